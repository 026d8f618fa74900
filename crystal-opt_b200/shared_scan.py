"""ctypes binding of the shared-scan forms (include/starjoin_batch.h): the batch
(many queries, one fact scan, one CUDA graph) and the serving loop (continuous
batching over a circular shared scan).

Also the workload helpers both forms are measured on: a 4-dimension star schema
(supplier, customer, part, date) whose dimensions expose a grouping attribute,
a selectivity attribute and the key, and seeded random queries with
log-uniform selectivities and fact row ranges.  `to_plain()` restates a
shared-scan query as a plain single-query description, so the same query runs
through the oracle and through the plain engine for parity checks.
"""
from __future__ import annotations

import ctypes as C
import math
import random
from typing import Any, Dict, List, Optional, Sequence, Tuple

import starjoin as sj

MAX_QUERIES = 64
MAX_ATTRS = 4


class SjbDim(C.Structure):
    _fields_ = [("fact_fk", C.c_void_p), ("key", C.c_void_p), ("rows", C.c_int64), ("key_min", C.c_int32),
                ("ht_len", C.c_int32), ("n_attrs", C.c_int32), ("attr", C.c_void_p * MAX_ATTRS)]


class SjbSchema(C.Structure):
    _fields_ = [("n_dims", C.c_int32), ("dims", SjbDim * sj.MAX_DIMS), ("measure", C.c_void_p),
                ("measure_sub", C.c_void_p), ("fact_rows", C.c_int64)]


class SjbPred(C.Structure):
    _fields_ = [("dim", C.c_int32), ("kind", C.c_int32), ("attr", C.c_int32), ("lo", C.c_int32),
                ("hi", C.c_int32), ("in_count", C.c_int32), ("in_codes", C.c_void_p), ("group_attr", C.c_int32)]


class SjbQuery(C.Structure):
    _fields_ = [("n_preds", C.c_int32), ("preds", SjbPred * sj.MAX_DIMS), ("row_begin", C.c_int64),
                ("row_end", C.c_int64)]


class SjbRow(C.Structure):
    _fields_ = [("query", C.c_int32), ("attr", C.c_int32 * sj.MAX_DIMS), ("pad_", C.c_int32),
                ("count", C.c_uint64), ("sum", C.c_uint64)]


class SjbLimits(C.Structure):
    _fields_ = [("group_entries", C.c_int64), ("result_rows", C.c_int64), ("filter_cache_bytes", C.c_int64),
                ("use_graph", C.c_int32), ("cache_filters", C.c_int32), ("threads", C.c_int32),
                ("smem_group_entries", C.c_int32)]


class SjbStats(C.Structure):
    _fields_ = [("ms_total", C.c_float), ("ms_probe", C.c_float), ("rows_scanned", C.c_uint64),
                ("filters_built", C.c_uint64), ("filters_cached", C.c_uint64), ("group_entries", C.c_uint64),
                ("error_flags", C.c_uint64)]


class SjsConfig(C.Structure):
    _fields_ = [("limits", SjbLimits), ("step_rows", C.c_int64), ("max_active", C.c_int32),
                ("plain", C.c_int32), ("hbm_reserve_bytes", C.c_int64), ("fault_admit_every", C.c_int32),
                ("solo_plain", C.c_int32)]


class SjsTicketInfo(C.Structure):
    _fields_ = [("done", C.c_int32), ("status", C.c_int32), ("n_rows", C.c_int64), ("submit_s", C.c_double),
                ("admit_s", C.c_double), ("finish_s", C.c_double)]


class SjsStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("admitted", C.c_uint64), ("finished", C.c_uint64),
                ("rejected", C.c_uint64), ("steps", C.c_uint64), ("rows_scanned", C.c_uint64),
                ("filters_built", C.c_uint64), ("filters_cached", C.c_uint64), ("peak_active", C.c_uint64),
                ("busy_s", C.c_double), ("admit_s", C.c_double), ("scan_s", C.c_double),
                ("probe_device_s", C.c_double), ("solo", C.c_uint64)]


class SjbTuneReport(C.Structure):
    _fields_ = [("candidates", C.c_int32), ("mismatches", C.c_int32), ("threads", C.c_int32),
                ("smem_group_entries", C.c_int32), ("best_probe_ms", C.c_float), ("default_probe_ms", C.c_float)]


SYMBOLS = ["sjb_batch_create", "sjb_batch_destroy", "sjb_batch_run", "sjb_batch_get_stats", "sjb_batch_tune",
           "sjs_server_create", "sjs_submit", "sjs_poll", "sjs_wait", "sjs_cancel", "sjs_get_stats", "sjs_now",
           "sjs_server_destroy"]


def load() -> C.CDLL:
    lib = sj.load()
    if getattr(lib, "_sjb_bound", False):
        return lib
    P = C.c_void_p
    sig = {
        "sjb_batch_create": (C.c_int, [P, C.POINTER(SjbSchema), C.POINTER(SjbLimits), C.POINTER(P)]),
        "sjb_batch_destroy": (None, [P]),
        "sjb_batch_run": (C.c_int, [P, C.POINTER(SjbQuery), C.c_int32, C.POINTER(SjbRow), C.c_int64,
                                    C.POINTER(C.c_int64), P]),
        "sjb_batch_get_stats": (C.c_int, [P, C.POINTER(SjbStats)]),
        "sjb_batch_tune": (C.c_int, [P, C.POINTER(SjbSchema), C.POINTER(SjbLimits), C.POINTER(SjbQuery), C.c_int32,
                                     C.c_int32, C.POINTER(SjbLimits), C.POINTER(SjbTuneReport)]),
        "sjs_server_create": (C.c_int, [P, C.POINTER(SjbSchema), C.POINTER(SjsConfig), C.POINTER(P)]),
        "sjs_submit": (C.c_int, [P, C.POINTER(SjbQuery), C.POINTER(C.c_uint64)]),
        "sjs_poll": (C.c_int, [P, C.c_uint64, C.POINTER(SjsTicketInfo), C.POINTER(SjbRow), C.c_int64]),
        "sjs_wait": (C.c_int, [P, C.c_uint64, C.c_double, C.POINTER(SjsTicketInfo), C.POINTER(SjbRow),
                               C.c_int64]),
        "sjs_cancel": (C.c_int, [P, C.c_uint64]),
        "sjs_get_stats": (C.c_int, [P, C.POINTER(SjsStats)]),
        "sjs_now": (C.c_double, []),
        "sjs_server_destroy": (None, [P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    lib._sjb_bound = True
    return lib


# ------------------------------------------------------------------ schema ----
# Dimension d of the shared-scan schema: (name, fact FK column, key column,
# key_min, ht_len, [(attribute column, (min, max)), ...]).  Attribute 0 is the
# grouping attribute, 1 the selectivity attribute, 2 the key itself.
def schema_dims(schema: sj.StarSchema) -> List[Tuple[str, str, str, int, int, List[Tuple[str, Tuple[int, int]]]]]:
    dims = [
        ("supp", "fk_supp", "s_key", 0, schema.supp_rows,
         [("s_city", (0, 249)), ("s_sel", (0, 999)), ("s_key", (1, schema.supp_rows))]),
        ("cust", "fk_cust", "c_key", 0, schema.cust_rows,
         [("c_city", (0, 249)), ("c_sel", (0, 999)), ("c_key", (1, schema.cust_rows))]),
    ]
    if schema.part_rows:
        dims.append(("part", "fk_part", "p_key", 0, schema.part_rows,
                     [("p_category", (0, 24)), ("p_sel", (0, 999)), ("p_key", (1, schema.part_rows))]))
    dims.append(("date", "fk_date", "d_key", sj.DATE_MIN, sj.DATE_MAX - sj.DATE_MIN + 1,
                 [("d_year", (1992, 1998)), ("d_sel", (0, 999)), ("d_key", (sj.DATE_MIN, sj.DATE_MAX))]))
    return dims


def ssb_dims(schema: sj.StarSchema) -> List[Tuple[str, str, str, int, int, List[Tuple[str, Tuple[int, int]]]]]:
    """The dimensions with SSB's attributes (the nested codes of the reference's
    queries: src/ssb-jo/q2x..q4x build kernels), in the layout of schema_dims."""
    dims = [
        ("supp", "fk_supp", "s_key", 0, schema.supp_rows,
         [("s_city", (0, 249)), ("s_nation", (0, 24)), ("s_region", (0, 4)), ("s_key", (1, schema.supp_rows))]),
        ("cust", "fk_cust", "c_key", 0, schema.cust_rows,
         [("c_city", (0, 249)), ("c_nation", (0, 24)), ("c_region", (0, 4)), ("c_key", (1, schema.cust_rows))]),
    ]
    if schema.part_rows:
        dims.append(("part", "fk_part", "p_key", 0, schema.part_rows,
                     [("p_brand1", (0, 999)), ("p_category", (0, 24)), ("p_mfgr", (0, 4)),
                      ("p_key", (1, schema.part_rows))]))
    dims.append(("date", "fk_date", "d_key", sj.DATE_MIN, sj.DATE_MAX - sj.DATE_MIN + 1,
                 [("d_year", (1992, 1998)), ("d_yearmonthnum", (199201, 199812)),
                  ("d_key", (sj.DATE_MIN, sj.DATE_MAX))]))
    return dims


def from_plain(q: Dict[str, Any], dims) -> Dict[str, Any]:
    """A plain single-query description (starjoin.q21_query ... q43_query) in
    shared-scan form over `dims`; predicates keep the plain query's dimension
    order, so result tuples compare with oracle.run / Engine.run directly."""
    where = {fk: i for i, (_, fk, *_rest) in enumerate(dims)}
    preds = []
    for d in q["dims"]:
        i = where[d["fk"]]
        names = [a for a, _ in dims[i][5]]
        pred = d["pred"]
        p: Dict[str, Any] = {"dim": i, "kind": pred[0]}
        if pred[0] == "in":
            p.update(attr=names.index(d["attr"]), codes=list(pred[1]))
        elif pred[0] == "range":
            p.update(attr=names.index(d["attr"]), lo=int(pred[1]), hi=int(pred[2]))
        p["group_attr"] = names.index(d["payload"]) if d.get("group") else -1
        preds.append(p)
    return {"preds": preds, "row_range": tuple(q["row_range"])}


def make_schema(schema: sj.StarSchema, cols: Dict[str, Any], dims=None,
                measure_sub: Optional[str] = None) -> Tuple[SjbSchema, list]:
    s = SjbSchema()
    keep = []

    def ptr(name):
        t = cols[name]
        keep.append(t)
        return t.data_ptr() if hasattr(t, "data_ptr") else t.ctypes.data

    dims = dims or schema_dims(schema)
    s.n_dims = len(dims)
    for i, (_, fk, key, kmin, ln, attrs) in enumerate(dims):
        d = s.dims[i]
        d.fact_fk = ptr(fk)
        d.key = ptr(key)
        d.rows = int(cols[key].shape[0])
        d.key_min = kmin
        d.ht_len = ln
        d.n_attrs = len(attrs)
        for a, (name, _) in enumerate(attrs):
            d.attr[a] = ptr(name)
    s.measure = ptr("revenue")
    s.measure_sub = ptr(measure_sub) if measure_sub else None
    s.fact_rows = schema.fact_rows
    return s, keep


# ----------------------------------------------------------------- queries ----
def random_query(rng: random.Random, schema: sj.StarSchema, n_dims: Optional[int] = None,
                 sel_range=(0.0005, 0.60), len_range=(1_000_000, None), max_span: int = 65536) -> Dict[str, Any]:
    """A seeded random shared-scan query: 2-4 dimensions, each predicate's
    selectivity log-uniform in sel_range (a range of the selectivity attribute
    when >= 0.1%, else a range of keys), a fact row range whose length is
    log-uniform in len_range, grouping by 1-3 dimensions' grouping attributes
    (worst-case key space <= max_span)."""
    dims = schema_dims(schema)
    nd = n_dims or rng.randint(2, min(4, len(dims)))
    chosen = sorted(rng.sample(range(len(dims)), nd))
    preds = []
    for d in chosen:
        _, _, _, _, _, attrs = dims[d]
        s = math.exp(rng.uniform(math.log(sel_range[0]), math.log(sel_range[1])))
        sel_lo, sel_hi = attrs[1][1]
        width = round(s * (sel_hi - sel_lo + 1))
        if s * (sel_hi - sel_lo + 1) >= 1:
            a = rng.randint(sel_lo, sel_hi - width + 1)
            pred = {"dim": d, "kind": "range", "attr": 1, "lo": a, "hi": a + width - 1}
        else:  # below the selectivity attribute's resolution: a range of keys
            klo, khi = attrs[2][1]
            if d == len(dims) - 1:  # date keys are yyyymmdd: one day
                day = rng.randint(0, sj.DATE_DAYS - 1)
                import datetime
                k = int((datetime.date(1992, 1, 1) + datetime.timedelta(days=day)).strftime("%Y%m%d"))
                pred = {"dim": d, "kind": "range", "attr": 2, "lo": k, "hi": k}
            else:
                w = max(1, round(s * (khi - klo + 1)))
                a = rng.randint(klo, khi - w + 1)
                pred = {"dim": d, "kind": "range", "attr": 2, "lo": a, "hi": a + w - 1}
        pred["group_attr"] = -1
        preds.append(pred)
    # grouping: 1-3 of the chosen dims, within max_span
    order = list(range(nd))
    rng.shuffle(order)
    span = 1
    for i in order[: rng.randint(1, min(3, nd))]:
        lo, hi = dims[preds[i]["dim"]][5][0][1]
        if span * (hi - lo + 1) <= max_span:
            preds[i]["group_attr"] = 0
            span *= hi - lo + 1
    n = schema.fact_rows
    lmin = min(len_range[0], n)
    lmax = min(len_range[1] or n, n)
    length = int(round(math.exp(rng.uniform(math.log(max(lmin, 1)), math.log(max(lmax, 1)))))) if n else 0
    length = max(0, min(length, n))
    b = rng.randint(0, n - length)
    return {"preds": preds, "row_range": (b, b + length)}


def q33_as_shared(schema: sj.StarSchema, cities=(231, 235)) -> Dict[str, Any]:
    """SSB Q3.3 (src/ssb-jo/q33/0-lip.cu:114-203) in shared-scan form."""
    dims = schema_dims(schema)
    di = {name: i for i, (name, *_rest) in enumerate(dims)}
    return {"preds": [
        {"dim": di["supp"], "kind": "in", "attr": 0, "codes": list(cities), "group_attr": 0},
        {"dim": di["cust"], "kind": "in", "attr": 0, "codes": list(cities), "group_attr": 0},
        {"dim": di["date"], "kind": "range", "attr": 0, "lo": -(2 ** 31), "hi": 1997, "group_attr": 0},
    ], "row_range": (0, schema.fact_rows)}


def fill_query(q: Dict[str, Any], out: SjbQuery, keep: list) -> None:
    out.n_preds = len(q["preds"])
    for k, p in enumerate(q["preds"]):
        sp = out.preds[k]
        sp.dim = p["dim"]
        kind = p["kind"]
        sp.kind = {"all": sj.PRED_ALL, "in": sj.PRED_IN, "range": sj.PRED_RANGE}[kind]
        sp.attr = p.get("attr", 0)
        sp.lo = p.get("lo", 0)
        sp.hi = p.get("hi", 0)
        if kind == "in":
            codes = (C.c_int32 * max(1, len(p["codes"])))(*p["codes"])
            keep.append(codes)
            sp.in_count = len(p["codes"])
            sp.in_codes = C.addressof(codes)
        else:
            sp.in_count = 0
            sp.in_codes = None
        sp.group_attr = p.get("group_attr", -1)
    out.row_begin, out.row_end = q["row_range"]


def to_plain(schema: sj.StarSchema, q: Dict[str, Any], dims=None, measure_sub: Optional[str] = None) -> Dict[str, Any]:
    """The same query as a plain single-query description (oracle / plain engine),
    with the dimensions in predicate order and a direct (exact) filter."""
    dims = dims or schema_dims(schema)
    out = []
    for p in q["preds"]:
        _, fk, key, kmin, ln, attrs = dims[p["dim"]]
        kind = p["kind"]
        if kind == "in":
            pred = ("in", list(p["codes"]))
        elif kind == "range":
            pred = ("range", p["lo"], p["hi"])
        else:
            pred = ("all",)
        g = p.get("group_attr", -1)
        out.append({"fk": fk, "key": key, "attr": attrs[p.get("attr", 0)][0] if kind != "all" else None,
                    "payload": attrs[g][0] if g >= 0 else None, "key_min": kmin, "ht_len": ln, "pred": pred,
                    "group": g >= 0, "payload_range": attrs[g][1] if g >= 0 else (0, 0)})
    return {"dims": out, "measure": "revenue", "measure_sub": measure_sub, "row_range": tuple(q["row_range"]),
            "order": list(range(len(out))), "lip": True, "adaptive": False, "bf_bits_per_key": 0,
            "bf_hashes": 2}


def rows_by_query(rows, n: int, queries: Sequence[Dict[str, Any]]) -> List[List[tuple]]:
    """Batch result rows -> per query sorted tuples (grouped attrs..., count, sum),
    the format of oracle.run / Engine.run."""
    out: List[List[tuple]] = [[] for _ in queries]
    for r in rows[:n]:
        q = queries[r.query]
        g = [k for k, p in enumerate(q["preds"]) if p.get("group_attr", -1) >= 0]
        out[r.query].append(tuple(int(r.attr[k]) for k in g) + (int(r.count), int(r.sum)))
    return [sorted(x) for x in out]


# ------------------------------------------------------------------- batch ----
class Batch:
    """A batch runner over one registered schema (device columns)."""

    def __init__(self, eng: sj.Engine, schema: sj.StarSchema, cols: Dict[str, Any], use_graph=True,
                 cache_filters=False, threads=0, group_entries=0, result_rows=0, smem_group_entries=0,
                 filter_cache_bytes=0, dims=None, measure_sub: Optional[str] = None):
        self.lib = load()
        self.eng, self.schema = eng, schema
        self._schema, self._keep = make_schema(schema, cols, dims, measure_sub)
        lim = SjbLimits(group_entries, result_rows, filter_cache_bytes, 1 if use_graph else 0,
                        1 if cache_filters else 0, threads, smem_group_entries)
        h = C.c_void_p()
        sj.check(self.lib.sjb_batch_create(eng.h, C.byref(self._schema), C.byref(lim), C.byref(h)))
        self.h = h
        self.result_rows = result_rows or (1 << 20)
        self._rows = (SjbRow * self.result_rows)()

    def describe(self, queries: Sequence[Dict[str, Any]]):
        """The C descriptions of a batch (kept alive by the returned tuple)."""
        arr = (SjbQuery * len(queries))()
        keep: list = []
        for i, q in enumerate(queries):
            fill_query(q, arr[i], keep)
        return arr, keep

    def run_raw(self, described, stream=None) -> int:
        """One sjb_batch_run call on a described batch; returns the row count
        (rows stay in the internal buffer until the next call)."""
        arr, _ = described
        n = C.c_int64()
        sj.check(self.lib.sjb_batch_run(self.h, arr, len(arr), self._rows, self.result_rows, C.byref(n), stream))
        return n.value

    def rows(self, n: int, queries: Sequence[Dict[str, Any]]) -> List[List[tuple]]:
        return rows_by_query(self._rows, n, queries)

    def run(self, queries: Sequence[Dict[str, Any]], stream=None) -> List[List[tuple]]:
        return self.rows(self.run_raw(self.describe(queries), stream), queries)

    def stats(self) -> SjbStats:
        s = SjbStats()
        sj.check(self.lib.sjb_batch_get_stats(self.h, C.byref(s)))
        return s

    def close(self):
        if self.h:
            self.lib.sjb_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tune_batch(eng: sj.Engine, schema: sj.StarSchema, cols: Dict[str, Any], queries: Sequence[Dict[str, Any]],
               reps: int = 3, use_graph=True, cache_filters=False, dims=None, measure_sub: Optional[str] = None):
    """sjb_batch_tune on a sample batch: returns ({"threads", "smem_group_entries"},
    SjbTuneReport) -- the probe shape to pass to Batch / Server."""
    lib = load()
    sch, keep = make_schema(schema, cols, dims, measure_sub)
    base = SjbLimits(0, 0, 0, 1 if use_graph else 0, 1 if cache_filters else 0, 0, 0)
    arr = (SjbQuery * len(queries))()
    qkeep: list = []
    for i, q in enumerate(queries):
        fill_query(q, arr[i], qkeep)
    chosen, rep = SjbLimits(), SjbTuneReport()
    sj.check(lib.sjb_batch_tune(eng.h, C.byref(sch), C.byref(base), arr, len(queries), reps, C.byref(chosen),
                                C.byref(rep)))
    return {"threads": chosen.threads, "smem_group_entries": chosen.smem_group_entries}, rep


# ----------------------------------------------------------------- serving ----
class Server:
    """The serving loop: submit() from any thread, wait()/poll() for results."""

    def __init__(self, eng: sj.Engine, schema: sj.StarSchema, cols: Dict[str, Any], plain=False, step_rows=0,
                 max_active=0, cache_filters=True, group_entries=0, filter_cache_bytes=0, threads=0,
                 hbm_reserve_bytes=0, fault_admit_every=0, solo_plain=False, smem_group_entries=0):
        self.lib = load()
        self.eng, self.schema = eng, schema
        self._schema, self._keep = make_schema(schema, cols)
        cfg = SjsConfig()
        cfg.limits = SjbLimits(group_entries, 0, filter_cache_bytes, 0, 1 if cache_filters else 0, threads,
                               smem_group_entries)
        cfg.step_rows = step_rows
        cfg.max_active = max_active
        cfg.plain = 1 if plain else 0
        cfg.hbm_reserve_bytes = hbm_reserve_bytes
        cfg.fault_admit_every = fault_admit_every
        cfg.solo_plain = 1 if solo_plain else 0
        h = C.c_void_p()
        sj.check(self.lib.sjs_server_create(eng.h, C.byref(self._schema), C.byref(cfg), C.byref(h)))
        self.h = h
        self.queries: Dict[int, Dict[str, Any]] = {}

    def submit(self, q: Dict[str, Any]) -> int:
        sq = SjbQuery()
        keep: list = []
        fill_query(q, sq, keep)
        t = C.c_uint64()
        sj.check(self.lib.sjs_submit(self.h, C.byref(sq), C.byref(t)))
        self.queries[t.value] = q
        return t.value

    def wait(self, ticket: int, timeout_s: float = 0.0, cap: int = 1 << 18):
        """(rows as sorted tuples, SjsTicketInfo)."""
        info = SjsTicketInfo()
        rows = (SjbRow * cap)()
        sj.check(self.lib.sjs_wait(self.h, ticket, timeout_s, C.byref(info), rows, cap))
        q = self.queries.pop(ticket)
        return rows_by_query_one(rows, info.n_rows, q), info

    def cancel(self, ticket: int) -> None:
        sj.check(self.lib.sjs_cancel(self.h, ticket))

    def stats(self) -> SjsStats:
        s = SjsStats()
        sj.check(self.lib.sjs_get_stats(self.h, C.byref(s)))
        return s

    def now(self) -> float:
        return float(self.lib.sjs_now())

    def close(self):
        if self.h:
            self.lib.sjs_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def rows_by_query_one(rows, n: int, q: Dict[str, Any]) -> List[tuple]:
    g = [k for k, p in enumerate(q["preds"]) if p.get("group_attr", -1) >= 0]
    return sorted(tuple(int(r.attr[k]) for k in g) + (int(r.count), int(r.sum)) for r in rows[:n])
