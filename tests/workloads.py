"""Query and workload descriptions shared by the tests (pure Python, no GPU)."""
from __future__ import annotations

import itertools
import random
from typing import Any, Dict, List

import starjoin as sj

ORDERS3 = list(itertools.permutations(range(3)))  # the reference's six join orders

# Join orders of the reference's six drivers over (S=0, C=1, D=2):
# src/ssb-jo/q33/{0..5}-{lip,naive}.cu header comments.
REF_DRIVER_ORDERS = {
    0: (0, 1, 2),  # S -> C -> D
    1: (0, 2, 1),  # S -> D -> C
    2: (2, 0, 1),  # D -> S -> C
    3: (2, 1, 0),  # D -> C -> S
    4: (1, 2, 0),  # C -> D -> S
    5: (1, 0, 2),  # C -> S -> D
}

SMALL = sj.StarSchema(seed=0x5EED0001, fact_rows=6_000_000, cust_rows=30_000, supp_rows=2_000)
FULL = sj.StarSchema(seed=0x5EED0002, fact_rows=120_000_000, cust_rows=600_000, supp_rows=40_000)
# SSB scale-factor-1 dimension sizes for the Q2.x / Q3.1 / Q3.2 / Q3.4 / Q4.x shapes
SHAPES_SMALL = sj.StarSchema(seed=0x5EED0009, fact_rows=6_000_000, cust_rows=30_000, supp_rows=2_000,
                             part_rows=200_000)
SHAPE_QUERIES = {21: sj.q21_query, 22: sj.q22_query, 23: sj.q23_query, 31: sj.q31_query, 32: sj.q32_query,
                 34: sj.q34_query, 41: sj.q41_query, 42: sj.q42_query, 43: sj.q43_query}
# integers per group line the reference drivers print
SHAPE_WIDTH = {21: 3, 22: 3, 23: 3, 31: 4, 32: 4, 34: 4, 41: 3, 42: 4, 43: 4}


shape_as_printed = sj.ssb_printed  # result tuples in the order the reference drivers print them


FOURDIM = sj.StarSchema(seed=0x5EED0003, fact_rows=120_000_000, cust_rows=600_000, supp_rows=40_000,
                        part_rows=1_000_000)


def random_query(rng: random.Random, schema: sj.StarSchema, n_dims: int | None = None) -> Dict[str, Any]:
    """A random star query over the schema: 1-4 dims, IN / range / all predicates
    on the city / year / category / sel attributes, random grouping, order, range."""
    pool = [
        {"fk": "fk_supp", "key": "s_key", "ht_len": schema.supp_rows, "key_min": 0,
         "attrs": [("s_city", 0, 249), ("s_sel", 0, 999)]},
        {"fk": "fk_cust", "key": "c_key", "ht_len": schema.cust_rows, "key_min": 0,
         "attrs": [("c_city", 0, 249), ("c_sel", 0, 999)]},
        {"fk": "fk_date", "key": "d_key", "ht_len": sj.DATE_MAX - sj.DATE_MIN + 1, "key_min": sj.DATE_MIN,
         "attrs": [("d_year", 1992, 1998), ("d_sel", 0, 999)]},
    ]
    if schema.part_rows:
        pool.append({"fk": "fk_part", "key": "p_key", "ht_len": schema.part_rows, "key_min": 0,
                     "attrs": [("p_category", 0, 24), ("p_sel", 0, 999)]})
    k = n_dims or rng.randint(1, len(pool))
    chosen = rng.sample(pool, k)
    dims = []
    for d in chosen:
        attr, lo, hi = rng.choice(d["attrs"])
        kind = rng.random()
        if kind < 0.5:
            n = rng.choice([1, 2, 3, 10, 50, (hi - lo + 1) // 2])
            pred = ("in", sorted(rng.sample(range(lo, hi + 1), max(1, min(n, hi - lo + 1)))))
        elif kind < 0.85:
            a = rng.randint(lo, hi)
            b = rng.randint(a, hi)
            pred = ("range", a, b)
        else:
            pred = ("all",)
        pattr, plo, phi = rng.choice(d["attrs"])
        group = rng.random() < 0.6
        dims.append({"fk": d["fk"], "key": d["key"], "attr": attr, "payload": pattr if group else None,
                     "key_min": d["key_min"], "ht_len": d["ht_len"], "pred": pred, "group": group,
                     "payload_range": (plo, phi)})
    # keep the dense group space within the engine's 2^26 limit
    span = 1
    for d in dims:
        if d["group"]:
            w = d["payload_range"][1] - d["payload_range"][0] + 1
            if span * w > (1 << 22):
                d["group"], d["payload"] = False, None
            else:
                span *= w
    order = list(range(k))
    rng.shuffle(order)
    n = schema.fact_rows
    if rng.random() < 0.5:
        b = rng.randint(0, n)
        e = rng.randint(b, n)
    else:
        b, e = 0, n
    return {"dims": dims, "measure": "revenue",
            "measure_sub": "supplycost" if (schema.part_rows and rng.random() < 0.3) else None,
            "row_range": (b, e), "order": order, "lip": rng.random() < 0.7,
            "adaptive": rng.random() < 0.5, "bf_bits_per_key": rng.choice([0, 4, 8, 16]),
            "bf_hashes": rng.randint(1, 4)}


def sel_query(schema: sj.StarSchema, sels: List[int], seed: int, order=None, lip=True, bpk=8, k=2,
              adaptive=False) -> Dict[str, Any]:
    """The 4-dimension variable-selectivity star join: dim i keeps the rows whose
    `sel` attribute (uniform over 1000 codes) lies in a seeded random subset of
    sels[i] codes (per mille); group by (s_city, c_city, d_year), part filter-only."""
    rng = random.Random(seed)
    spec = [("fk_supp", "s_key", "s_sel", "s_city", (0, 249), schema.supp_rows, 0, True),
            ("fk_cust", "c_key", "c_sel", "c_city", (0, 249), schema.cust_rows, 0, True),
            ("fk_date", "d_key", "d_sel", "d_year", (1992, 1998), sj.DATE_MAX - sj.DATE_MIN + 1, sj.DATE_MIN,
             True),
            ("fk_part", "p_key", "p_sel", None, (0, 0), schema.part_rows, 0, False)]
    dims = []
    for (fk, key, attr, payload, prange, ln, kmin, group), s in zip(spec, sels):
        codes = sorted(rng.sample(range(1000), s))
        dims.append({"fk": fk, "key": key, "attr": attr, "payload": payload, "key_min": kmin, "ht_len": ln,
                     "pred": ("in", codes), "group": group, "payload_range": prange})
    return {"dims": dims, "measure": "revenue", "measure_sub": None, "row_range": (0, schema.fact_rows),
            "order": list(order) if order is not None else list(range(len(dims))), "lip": lip,
            "adaptive": adaptive, "bf_bits_per_key": bpk, "bf_hashes": k}


def columns_of(query: Dict[str, Any]) -> List[str]:
    names = {query["measure"]}
    if query.get("measure_sub"):
        names.add(query["measure_sub"])
    for d in query["dims"]:
        for f in ("fk", "key", "attr", "payload"):
            if d.get(f):
                names.add(d[f])
    return sorted(names)
