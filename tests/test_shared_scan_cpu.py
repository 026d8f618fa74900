"""CPU checks of the shared-scan workload helpers: the seeded query generator
(selectivity, grouping and row-range bounds) and its restatement as a plain
query, run through the oracle."""
import math
import random

import numpy as np

import shared_scan as ss
import starjoin as sj

SC = sj.StarSchema(seed=0x5EED0004, fact_rows=400_000, cust_rows=30_000, supp_rows=2000, part_rows=20_000)


def test_generator_is_seeded_and_bounded():
    a = [ss.random_query(random.Random(7), SC) for _ in range(3)]
    b = [ss.random_query(random.Random(7), SC) for _ in range(3)]
    assert a == b
    rng = random.Random(1)
    dims = ss.schema_dims(SC)
    for _ in range(500):
        q = ss.random_query(rng, SC)
        assert 2 <= len(q["preds"]) <= 4
        assert len({p["dim"] for p in q["preds"]}) == len(q["preds"])
        b, e = q["row_range"]
        assert 0 <= b <= e <= SC.fact_rows
        span = 1
        for p in q["preds"]:
            attrs = dims[p["dim"]][5]
            lo, hi = attrs[p["attr"]][1]
            assert lo <= p["lo"] <= p["hi"] <= hi
            if p["group_attr"] >= 0:
                glo, ghi = attrs[p["group_attr"]][1]
                span *= ghi - glo + 1
        assert any(p["group_attr"] >= 0 for p in q["preds"])
        assert span <= 65536


def test_selectivities_are_log_uniform_over_the_range():
    rng = random.Random(3)
    dims = ss.schema_dims(SC)
    sels = []
    for _ in range(3000):
        for p in ss.random_query(rng, SC)["preds"]:
            lo, hi = dims[p["dim"]][5][p["attr"]][1]
            if p["attr"] == 2 and p["dim"] == len(dims) - 1:
                sels.append(1 / sj.DATE_DAYS)
            else:
                sels.append((p["hi"] - p["lo"] + 1) / (hi - lo + 1))
    logs = np.log(np.array(sels))
    assert min(sels) < 0.001 and max(sels) > 0.5
    # roughly uniform in log space between 0.05% and 60%
    lo, hi = math.log(0.0005), math.log(0.6)
    hist, _ = np.histogram(np.clip(logs, lo, hi), bins=4, range=(lo, hi))
    assert hist.min() > 0.15 * len(sels)


def test_plain_restatement_runs_through_the_oracle(oracle):
    cols = sj.gen_host(SC)
    rng = random.Random(11)
    for _ in range(6):
        q = ss.random_query(rng, SC, len_range=(10_000, None))
        plain = ss.to_plain(SC, q)
        got = oracle.run(plain, cols)
        # a direct numpy restatement of the same predicates and grouping
        dims = ss.schema_dims(SC)
        b, e = q["row_range"]
        keep = np.ones(e - b, dtype=bool)
        keys = []
        for p in q["preds"]:
            _, fk, key, kmin, ln, attrs = dims[p["dim"]]
            fkv = cols[fk][b:e].astype(np.int64)
            slot = (fkv - kmin) % ln
            table = np.full(ln, -1, dtype=np.int64)
            kv = cols[key].astype(np.int64)
            av = cols[attrs[p["attr"]][0]]
            ok = (av >= p["lo"]) & (av <= p["hi"]) & (kv != 0)
            table[((kv - kmin) % ln)[ok]] = np.nonzero(ok)[0]
            row = table[slot]
            keep &= row >= 0
            if p["group_attr"] >= 0:
                keys.append(np.where(row >= 0, cols[attrs[p["group_attr"]][0]][np.maximum(row, 0)], 0))
        rev = cols["revenue"][b:e].astype(np.uint64)
        groups = {}
        for i in np.nonzero(keep)[0]:
            k = tuple(int(x[i]) for x in keys)
            c, s = groups.get(k, (0, 0))
            groups[k] = (c + 1, (s + int(rev[i])) % (1 << 64))
        want = sorted(k + v for k, v in groups.items())
        assert got == want


def test_ssb_shapes_round_trip_through_shared_form(sj, oracle):
    """Every SSB query shape (Q2.1-Q4.3 as the reference's drivers run them)
    restated in shared-scan form over the SSB-attribute dimensions and back
    answers like the original on the oracle."""
    from workloads import SHAPE_QUERIES
    sc = sj.StarSchema(seed=0x5EED0011, fact_rows=200_000, cust_rows=3_000, supp_rows=200, part_rows=20_000)
    cols = sj.gen_host(sc)
    dims = ss.ssb_dims(sc)
    for q, make in SHAPE_QUERIES.items():
        plain = make(sc)
        shared = ss.from_plain(plain, dims)
        assert [p["dim"] for p in shared["preds"]] == [
            [d[1] for d in dims].index(x["fk"]) for x in plain["dims"]], q
        back = ss.to_plain(sc, shared, dims, plain["measure_sub"])
        assert oracle.run(back, cols) == oracle.run(plain, cols), q
