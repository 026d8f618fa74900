"""ctypes binding of the star-join engine's C ABI (include/starjoin.h).

Host-side harness for tests and benchmarks: loads the in-tree
_build/libstarjoin.so, mirrors the ABI structs, and offers helpers to describe
the star-schema workloads (synthetic columns with the reference's SSB shapes) and
queries (Q3.3 of src/ssb-jo/q33/*.cu, and its 4-dimension / variable-selectivity
forms).  Device buffers are torch CUDA tensors (plumbing only); every kernel that
computes the join is the engine's own CUDA code.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os
from typing import Any, Dict, List, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libstarjoin.so")

MAX_DIMS = 4
BF_AUTO = -1  # plan.bf_bits_per_key: filter layout chosen per dimension (SJ_BF_AUTO)
MAX_IN_CODES = 4096

SJ_OK = 0
SJ_ERR_INVALID_ARGUMENT = 1
SJ_ERR_UNSUPPORTED = 2
SJ_ERR_OUT_OF_MEMORY = 3
SJ_ERR_CUDA = 4
SJ_ERR_CAPACITY = 5
SJ_ERR_TIMEOUT = 6
SJ_ERR_NO_DEVICE = 7
SJ_ERR_REJECTED = 8
SJ_ERR_CANCELLED = 9

PRED_ALL, PRED_IN, PRED_RANGE = 0, 1, 2

# generator column ids / kinds (csrc/sj_datagen.h)
COL_FK_CUST, COL_FK_SUPP, COL_FK_PART, COL_FK_DATE, COL_REVENUE, COL_SUPPLYCOST = 1, 2, 3, 4, 5, 6
COL_CUST_CITY, COL_CUST_SEL = 11, 12
COL_SUPP_CITY, COL_SUPP_SEL = 21, 22
COL_PART_CATEGORY, COL_PART_SEL, COL_PART_BRAND = 31, 32, 33
COL_DATE_SEL = 42
GEN_UNIFORM, GEN_DATEKEY, GEN_SEQ, GEN_DATE_SEQ, GEN_DATE_YEAR = 0, 1, 2, 3, 4
DATE_DAYS, DATE_MIN, DATE_MAX = 2556, 19920101, 19981230


class StarJoinError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


class SjDim(C.Structure):
    _fields_ = [
        ("fact_fk", C.c_void_p), ("key", C.c_void_p), ("filter_attr", C.c_void_p),
        ("payload", C.c_void_p), ("rows", C.c_int64), ("key_min", C.c_int32),
        ("ht_len", C.c_int32), ("pred_kind", C.c_int32), ("pred_lo", C.c_int32),
        ("pred_hi", C.c_int32), ("in_count", C.c_int32), ("in_codes", C.c_void_p),
        ("group", C.c_int32), ("payload_min", C.c_int32), ("payload_max", C.c_int32),
    ]


class SjTuning(C.Structure):
    _fields_ = [("threads", C.c_int32), ("chunk_rows", C.c_int32), ("stages", C.c_int32),
                ("ctas_per_sm", C.c_int32), ("compact_threshold", C.c_int32),
                ("bf_smem_bytes", C.c_int32), ("record_events", C.c_int32)]


class SjPlan(C.Structure):
    _fields_ = [
        ("n_dims", C.c_int32), ("dims", SjDim * MAX_DIMS), ("measure", C.c_void_p),
        ("measure_sub", C.c_void_p), ("fact_rows", C.c_int64), ("row_begin", C.c_int64),
        ("row_end", C.c_int64), ("order", C.c_int32 * MAX_DIMS), ("lip", C.c_int32),
        ("adaptive", C.c_int32), ("bf_bits_per_key", C.c_int32), ("bf_hashes", C.c_int32),
        ("tune", SjTuning),
    ]


class SjAutotuneOpts(C.Structure):
    _fields_ = [("reps", C.c_int32), ("tune_filter", C.c_int32), ("tune_order", C.c_int32), ("verify", C.c_int32),
                ("cache_path", C.c_char_p)]


class SjAutotuneReport(C.Structure):
    _fields_ = [("candidates", C.c_int32), ("cache_hit", C.c_int32), ("mismatches", C.c_int32),
                ("default_ms", C.c_float), ("best_ms", C.c_float), ("selectivity", C.c_double * MAX_DIMS)]


class SjGroupRow(C.Structure):
    _fields_ = [("attr", C.c_int32 * MAX_DIMS), ("count", C.c_uint64), ("sum", C.c_uint64)]


class SjQueryStats(C.Structure):
    _fields_ = [
        ("rows_scanned", C.c_uint64), ("step_in", C.c_uint64 * 8), ("step_out", C.c_uint64 * 8),
        ("bf_inserted", C.c_uint64 * MAX_DIMS), ("bf_words", C.c_uint64 * MAX_DIMS),
        ("groups", C.c_uint64), ("reorders", C.c_uint64), ("error_flags", C.c_uint32),
        ("build_ms", C.c_float), ("probe_ms", C.c_float), ("bf_blocked", C.c_int32 * MAX_DIMS),
    ]


_lib: Optional[C.CDLL] = None


def load(build_if_missing: bool = True) -> C.CDLL:
    """Load the engine library (building it with nvcc when absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        if not build_if_missing:
            raise FileNotFoundError(LIB_PATH)
        import importlib.util
        spec = importlib.util.spec_from_file_location("sj_build_recipe", os.path.join(HERE, "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)  # type: ignore[union-attr]
        mod.build_engine()
    lib = C.CDLL(LIB_PATH)
    P = C.c_void_p
    sig = {
        "sj_engine_create": (C.c_int, [C.c_int, C.POINTER(P)]),
        "sj_engine_destroy": (None, [P]),
        "sj_status_string": (C.c_char_p, [C.c_int]),
        "sj_last_error": (C.c_char_p, []),
        "sj_device_sm_count": (C.c_int, [P]),
        "sj_query_prepare": (C.c_int, [P, C.POINTER(SjPlan), C.POINTER(P)]),
        "sj_query_build": (C.c_int, [P, P]),
        "sj_query_probe": (C.c_int, [P, P]),
        "sj_query_fetch": (C.c_int, [P, C.POINTER(SjGroupRow), C.c_int64, C.POINTER(C.c_int64), P]),
        "sj_query_get_stats": (C.c_int, [P, C.POINTER(SjQueryStats)]),
        "sj_query_release": (None, [P]),
        "sj_run_plain": (C.c_int, [P, C.POINTER(SjPlan), C.c_int, C.POINTER(SjGroupRow), C.c_int64,
                                   C.POINTER(C.c_int64), C.POINTER(C.c_float), P]),
        "sj_ssb_q33_run": (C.c_int, [P] + [P] * 4 + [C.c_int64] + [P] * 2 + [C.c_int64] + [P] * 2 +
                           [C.c_int64] + [P] * 2 + [C.c_int64] + [P, C.c_int32, C.c_int32,
                                                                 C.POINTER(SjGroupRow), C.c_int64,
                                                                 C.POINTER(C.c_int64),
                                                                 C.POINTER(C.c_float)]),
        "sj_bloom_test": (C.c_int, [P, P, C.c_int64, P, P, C.c_int64, C.c_int32, C.c_int32, C.c_int32,
                                    C.c_int32, P]),
        "sj_gen_column_device": (C.c_int, [P, C.c_int64, C.c_uint64, C.c_int32, C.c_int32, C.c_int32,
                                           C.c_int32, P]),
        "sj_gen_rows_device": (C.c_int, [P, C.c_int64, C.c_int64, C.c_uint64, C.c_int32, C.c_int32, C.c_int32,
                                         C.c_int32, P]),
        "sj_gen_column_host": (None, [P, C.c_int64, C.c_uint64, C.c_int32, C.c_int32, C.c_int32,
                                      C.c_int32, C.c_int]),
        "sj_ssb_q33_run_noalloc": (C.c_int, [C.c_int] + [P] * 4 + [C.c_int64] + [P] * 2 + [C.c_int64] +
                                   [P] * 2 + [C.c_int64] + [P] * 2 + [C.c_int64] +
                                   [P, C.c_int32, C.c_int32, C.POINTER(SjGroupRow), C.c_int64,
                                    C.POINTER(C.c_int64), P]),
        "sj_noalloc_last_error": (C.c_char_p, []),
        "sj_autotune": (C.c_int, [P, C.POINTER(SjPlan), C.POINTER(SjAutotuneOpts), C.POINTER(SjAutotuneReport), P]),
        "sj_ssb_column_file": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int64]),
        "sj_ssb_load_column": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int64, P]),
        "sj_ssb_store_column": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int64, P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def exported_symbols() -> List[str]:
    """Entry points declared in include/starjoin.h that the library must export."""
    return [
        "sj_engine_create", "sj_engine_destroy", "sj_status_string", "sj_last_error",
        "sj_device_sm_count", "sj_query_prepare", "sj_query_build", "sj_query_probe",
        "sj_query_fetch", "sj_query_get_stats", "sj_query_release", "sj_run_plain",
        "sj_ssb_q33_run", "sj_bloom_test", "sj_gen_column_device", "sj_gen_rows_device", "sj_gen_column_host",
        "sj_ssb_q33_run_noalloc", "sj_noalloc_last_error", "sj_autotune",
        "sj_ssb_column_file", "sj_ssb_load_column", "sj_ssb_store_column",
    ]


def check(status: int) -> None:
    if status != SJ_OK:
        lib = load()
        raise StarJoinError(status, lib.sj_last_error().decode(errors="replace"))


# ---------------------------------------------------------------- workload ----
@dataclasses.dataclass(frozen=True)
class StarSchema:
    """Sizes and seed of a synthetic star schema (BASE distributions of SSB Q3.x)."""
    seed: int
    fact_rows: int
    cust_rows: int
    supp_rows: int
    part_rows: int = 0
    date_rows: int = DATE_DAYS

    def column_specs(self) -> Dict[str, tuple]:
        """name -> (length, column id, kind, lo, hi)."""
        n = self.fact_rows
        specs = {
            "fk_cust": (n, COL_FK_CUST, GEN_UNIFORM, 1, self.cust_rows),
            "fk_supp": (n, COL_FK_SUPP, GEN_UNIFORM, 1, self.supp_rows),
            "fk_date": (n, COL_FK_DATE, GEN_DATEKEY, 0, 0),
            "revenue": (n, COL_REVENUE, GEN_UNIFORM, 1, 10_000_000),
            "c_key": (self.cust_rows, 0, GEN_SEQ, 1, 0),
            "c_city": (self.cust_rows, COL_CUST_CITY, GEN_UNIFORM, 0, 249),
            "c_sel": (self.cust_rows, COL_CUST_SEL, GEN_UNIFORM, 0, 999),
            "s_key": (self.supp_rows, 0, GEN_SEQ, 1, 0),
            "s_city": (self.supp_rows, COL_SUPP_CITY, GEN_UNIFORM, 0, 249),
            "s_sel": (self.supp_rows, COL_SUPP_SEL, GEN_UNIFORM, 0, 999),
            "d_key": (self.date_rows, 0, GEN_DATE_SEQ, 0, 0),
            "d_year": (self.date_rows, 0, GEN_DATE_YEAR, 0, 0),
            "d_sel": (self.date_rows, COL_DATE_SEL, GEN_UNIFORM, 0, 999),
        }
        if self.part_rows:
            specs.update({
                "fk_part": (n, COL_FK_PART, GEN_UNIFORM, 1, self.part_rows),
                "supplycost": (n, COL_SUPPLYCOST, GEN_UNIFORM, 1, 100_000),
                "p_key": (self.part_rows, 0, GEN_SEQ, 1, 0),
                "p_brand1": (self.part_rows, COL_PART_BRAND, GEN_UNIFORM, 0, 999),
                "p_sel": (self.part_rows, COL_PART_SEL, GEN_UNIFORM, 0, 999),
            })
        return specs

    def derived_specs(self) -> Dict[str, tuple]:
        """name -> (base column, divisor): SSB's nested codes.  A city's nation is
        city // 10 and its region nation // 5 (25 nations, 5 regions over 250
        cities); a brand's category is brand // 40 and its manufacturer
        category // 5 (1000 brands, 25 categories, 5 manufacturers); a date's
        d_yearmonthnum is datekey // 100 (19971231 -> 199712)."""
        d = {"c_nation": ("c_city", 10), "c_region": ("c_city", 50),
             "s_nation": ("s_city", 10), "s_region": ("s_city", 50), "d_yearmonthnum": ("d_key", 100)}
        if self.part_rows:
            d.update({"p_category": ("p_brand1", 40), "p_mfgr": ("p_brand1", 200)})
        return d

    def column_names(self) -> List[str]:
        return list(self.column_specs()) + list(self.derived_specs())


def _wanted(schema: StarSchema, names: Optional[Sequence[str]]):
    """Base columns to generate and derived columns to compute for `names`."""
    derived = schema.derived_specs()
    want = set(schema.column_names()) if names is None else set(names)
    bases = {n for n in want if n in schema.column_specs()}
    bases |= {derived[n][0] for n in want if n in derived}
    return bases, [n for n in derived if n in want], want


def gen_host(schema: StarSchema, names: Optional[Sequence[str]] = None, threads: int = 0) -> Dict[str, np.ndarray]:
    """Generate columns on the host (no GPU needed)."""
    lib = load()
    bases, derived, want = _wanted(schema, names)
    out = {}
    for name, (n, col, kind, lo, hi) in schema.column_specs().items():
        if name not in bases:
            continue
        a = np.empty(max(n, 0), dtype=np.int32)
        lib.sj_gen_column_host(a.ctypes.data, n, schema.seed, col, kind, lo, hi, threads)
        out[name] = a
    for name in derived:
        base, div = schema.derived_specs()[name]
        out[name] = (out[base] // div).astype(np.int32)
    return {k: v for k, v in out.items() if k in want}


def gen_device(schema: StarSchema, names: Optional[Sequence[str]] = None, device: int = 0,
               fact_range: Optional[Sequence[int]] = None):
    """Generate columns directly into torch CUDA tensors (same values as gen_host).
    fact_range=(b, e): only rows [b, e) of the fact columns (one shard of the
    schema's fact table); dimension columns are always whole."""
    import torch
    lib = load()
    bases, derived, want = _wanted(schema, names)
    out = {}
    for name, (n, col, kind, lo, hi) in schema.column_specs().items():
        if name not in bases:
            continue
        row0 = 0
        if fact_range is not None and n == schema.fact_rows:
            row0, n = int(fact_range[0]), int(fact_range[1]) - int(fact_range[0])
        t = torch.empty(max(n, 1), dtype=torch.int32, device=f"cuda:{device}")[:n]
        check(lib.sj_gen_rows_device(t.data_ptr(), row0, n, schema.seed, col, kind, lo, hi, None))
        out[name] = t
    for name in derived:
        base, div = schema.derived_specs()[name]
        out[name] = torch.div(out[base], div, rounding_mode="floor").to(torch.int32).contiguous()
    return {k: v for k, v in out.items() if k in want}


# ------------------------------------------------------------- SSB files ----
# Engine column names -> SSB column names (the reference's file layout).
SSB_NAMES = {"fk_cust": "lo_custkey", "fk_supp": "lo_suppkey", "fk_part": "lo_partkey", "fk_date": "lo_orderdate",
             "revenue": "lo_revenue", "supplycost": "lo_supplycost", "c_key": "c_custkey", "c_city": "c_city",
             "c_nation": "c_nation", "c_region": "c_region", "s_key": "s_suppkey", "s_city": "s_city",
             "s_nation": "s_nation", "s_region": "s_region", "p_key": "p_partkey", "p_brand1": "p_brand1",
             "p_category": "p_category", "p_mfgr": "p_mfgr", "d_key": "d_datekey", "d_year": "d_year",
             "d_yearmonthnum": "d_yearmonthnum"}


def ssb_file_name(column: str) -> str:
    buf = C.create_string_buffer(64)
    check(load().sj_ssb_column_file(column.encode(), buf, 64))
    return buf.value.decode()


def store_ssb_columns(directory: str, cols: Dict[str, np.ndarray]) -> None:
    """Write host columns (engine names) as the reference's column files."""
    for name, a in cols.items():
        if name not in SSB_NAMES:
            continue
        a = np.ascontiguousarray(a, dtype=np.int32)
        check(load().sj_ssb_store_column(directory.encode(), SSB_NAMES[name].encode(), a.size, a.ctypes.data))


def load_ssb_columns(directory: str, lengths: Dict[str, int]) -> Dict[str, np.ndarray]:
    """Read the reference's column files: engine name -> number of values."""
    out = {}
    for name, n in lengths.items():
        a = np.empty(max(n, 1), dtype=np.int32)[:n]
        check(load().sj_ssb_load_column(directory.encode(), SSB_NAMES[name].encode(), n, a.ctypes.data))
        out[name] = a
    return out


# ------------------------------------------------------------------ queries ----
def q33_query(schema: StarSchema, order=(0, 1, 2), lip=True, bf_bits_per_key=0, bf_hashes=2,
              adaptive=False, cities=(231, 235), row_range=None) -> Dict[str, Any]:
    """SSB Q3.3 as the reference drivers run it (src/ssb-jo/q33/0-lip.cu:114-203):
    dims 0 = supplier (s_city IN cities), 1 = customer (c_city IN cities),
    2 = date (d_year <= 1997, key-range table of 61130 slots from 19920101);
    group by (s_city, c_city, d_year); SUM(revenue)."""
    return {
        "dims": [
            {"fk": "fk_supp", "key": "s_key", "attr": "s_city", "payload": "s_city", "key_min": 0,
             "ht_len": schema.supp_rows, "pred": ("in", list(cities)), "group": True,
             "payload_range": (0, 249)},
            {"fk": "fk_cust", "key": "c_key", "attr": "c_city", "payload": "c_city", "key_min": 0,
             "ht_len": schema.cust_rows, "pred": ("in", list(cities)), "group": True,
             "payload_range": (0, 249)},
            {"fk": "fk_date", "key": "d_key", "attr": "d_year", "payload": "d_year",
             "key_min": DATE_MIN, "ht_len": DATE_MAX - DATE_MIN + 1,
             "pred": ("range", -(2 ** 31), 1997), "group": True, "payload_range": (1992, 1998)},
        ],
        "measure": "revenue", "measure_sub": None,
        "row_range": row_range if row_range is not None else (0, schema.fact_rows),
        "order": list(order), "lip": bool(lip), "adaptive": bool(adaptive),
        "bf_bits_per_key": int(bf_bits_per_key), "bf_hashes": int(bf_hashes),
    }


def _dim(fk, key, attr, pred, payload=None, prange=(0, 0), ht_len=0, key_min=0):
    return {"fk": fk, "key": key, "attr": attr, "payload": payload, "key_min": key_min, "ht_len": ht_len,
            "pred": pred, "group": payload is not None, "payload_range": prange}


def _date_dim(pred=("all",), attr="d_year"):
    return _dim("fk_date", "d_key", attr if pred[0] != "all" else None, pred, "d_year", (1992, 1998),
                DATE_MAX - DATE_MIN + 1, DATE_MIN)


def _shape(dims, schema, order, lip, bpk, k, adaptive, sub=None):
    return {"dims": dims, "measure": "revenue", "measure_sub": sub, "row_range": (0, schema.fact_rows),
            "order": list(order), "lip": bool(lip), "adaptive": bool(adaptive), "bf_bits_per_key": int(bpk),
            "bf_hashes": int(k)}


def q21_query(schema: StarSchema, order=(0, 1, 2), lip=True, bf_bits_per_key=0, bf_hashes=2,
              adaptive=False) -> Dict[str, Any]:
    """SSB Q2.1 as src/ssb-jo/q21/0-lip.cu runs it: dims 0 = supplier (s_region == 1,
    key-only table: BlockBuildSelectivePHT_1), 1 = part (p_category == 1, payload
    p_brand1), 2 = date (every day, payload d_year); group by (p_brand1, d_year);
    SUM(revenue).  Result tuples: (p_brand1, d_year, count, sum)."""
    dims = [_dim("fk_supp", "s_key", "s_region", ("in", [1]), ht_len=schema.supp_rows),
            _dim("fk_part", "p_key", "p_category", ("in", [1]), "p_brand1", (0, 999), schema.part_rows),
            _date_dim()]
    return _shape(dims, schema, order, lip, bf_bits_per_key, bf_hashes, adaptive)


def _q2x_query(schema, region, brand_pred, order, lip, bpk, k, adaptive):
    dims = [_dim("fk_supp", "s_key", "s_region", ("in", [region]), ht_len=schema.supp_rows),
            _dim("fk_part", "p_key", "p_brand1", brand_pred, "p_brand1", (0, 999), schema.part_rows),
            _date_dim()]
    return _shape(dims, schema, order, lip, bpk, k, adaptive)


def q22_query(schema: StarSchema, order=(0, 1, 2), lip=True, bf_bits_per_key=0, bf_hashes=2,
              adaptive=False) -> Dict[str, Any]:
    """SSB Q2.2 as src/ssb-jo/q22/0-lip.cu runs it: dims 0 = supplier (s_region == 2,
    key-only), 1 = part (260 <= p_brand1 <= 267, payload p_brand1), 2 = date (every
    day, payload d_year); group by (p_brand1, d_year); SUM(revenue).
    Result tuples: (p_brand1, d_year, count, sum)."""
    return _q2x_query(schema, 2, ("range", 260, 267), order, lip, bf_bits_per_key, bf_hashes, adaptive)


def q23_query(schema: StarSchema, order=(0, 1, 2), lip=True, bf_bits_per_key=0, bf_hashes=2,
              adaptive=False) -> Dict[str, Any]:
    """SSB Q2.3 as src/ssb-jo/q23/0-lip.cu runs it: as Q2.2 with s_region == 3 and
    p_brand1 == 260.  Result tuples: (p_brand1, d_year, count, sum)."""
    return _q2x_query(schema, 3, ("in", [260]), order, lip, bf_bits_per_key, bf_hashes, adaptive)


def q31_query(schema: StarSchema, order=(0, 1, 2), lip=True, bf_bits_per_key=0, bf_hashes=2,
              adaptive=False) -> Dict[str, Any]:
    """SSB Q3.1 as src/ssb-jo/q31/0-lip.cu runs it: dims 0 = customer (c_region == 2,
    payload c_nation), 1 = supplier (s_region == 2, payload s_nation), 2 = date
    (1992 <= d_year <= 1997); group by (c_nation, s_nation, d_year); SUM(revenue).
    Result tuples: (c_nation, s_nation, d_year, count, sum)."""
    dims = [_dim("fk_cust", "c_key", "c_region", ("in", [2]), "c_nation", (0, 24), schema.cust_rows),
            _dim("fk_supp", "s_key", "s_region", ("in", [2]), "s_nation", (0, 24), schema.supp_rows),
            _date_dim(("range", 1992, 1997))]
    return _shape(dims, schema, order, lip, bf_bits_per_key, bf_hashes, adaptive)


def q32_query(schema: StarSchema, order=(0, 1, 2), lip=True, bf_bits_per_key=0, bf_hashes=2,
              adaptive=False) -> Dict[str, Any]:
    """SSB Q3.2 as src/ssb-jo/q32/0-lip.cu runs it: dims 0 = supplier (s_nation == 24,
    payload s_city), 1 = customer (c_nation == 24, payload c_city), 2 = date
    (1992 <= d_year <= 1997); group by (s_city, c_city, d_year); SUM(revenue) (the
    driver sums in int32).  Result tuples: (s_city, c_city, d_year, count, sum)."""
    dims = [_dim("fk_supp", "s_key", "s_nation", ("in", [24]), "s_city", (0, 249), schema.supp_rows),
            _dim("fk_cust", "c_key", "c_nation", ("in", [24]), "c_city", (0, 249), schema.cust_rows),
            _date_dim(("range", 1992, 1997))]
    return _shape(dims, schema, order, lip, bf_bits_per_key, bf_hashes, adaptive)


def q34_query(schema: StarSchema, order=(0, 1, 2), lip=True, bf_bits_per_key=0, bf_hashes=2,
              adaptive=False) -> Dict[str, Any]:
    """SSB Q3.4 as src/ssb-jo/q34/0-lip.cu runs it: dims 0 = supplier (s_city IN
    {231, 235}), 1 = customer (c_city IN {231, 235}), 2 = date (d_yearmonthnum ==
    199712, payload d_year); group by (s_city, c_city, d_year); SUM(revenue) (int32
    in the driver).  Result tuples: (s_city, c_city, d_year, count, sum)."""
    dims = [_dim("fk_supp", "s_key", "s_city", ("in", [231, 235]), "s_city", (0, 249), schema.supp_rows),
            _dim("fk_cust", "c_key", "c_city", ("in", [231, 235]), "c_city", (0, 249), schema.cust_rows),
            _date_dim(("range", 199712, 199712), attr="d_yearmonthnum")]
    return _shape(dims, schema, order, lip, bf_bits_per_key, bf_hashes, adaptive)


def q41_query(schema: StarSchema, order=(0, 1, 2, 3), lip=True, bf_bits_per_key=0, bf_hashes=2,
              adaptive=False) -> Dict[str, Any]:
    """SSB Q4.1 as src/ssb-jo/q41/0-lip.cu runs it: dims 0 = supplier (s_region == 1,
    key-only), 1 = customer (c_region == 1, payload c_nation), 2 = part (p_mfgr IN
    {0, 1}, key-only), 3 = date (every day, payload d_year); group by (c_nation,
    d_year); SUM(revenue - supplycost).  Result tuples: (c_nation, d_year, count, sum)."""
    dims = [_dim("fk_supp", "s_key", "s_region", ("in", [1]), ht_len=schema.supp_rows),
            _dim("fk_cust", "c_key", "c_region", ("in", [1]), "c_nation", (0, 24), schema.cust_rows),
            _dim("fk_part", "p_key", "p_mfgr", ("in", [0, 1]), ht_len=schema.part_rows),
            _date_dim()]
    return _shape(dims, schema, order, lip, bf_bits_per_key, bf_hashes, adaptive, sub="supplycost")


def q42_query(schema: StarSchema, order=(0, 1, 2, 3), lip=False, bf_bits_per_key=0, bf_hashes=2,
              adaptive=False) -> Dict[str, Any]:
    """SSB Q4.2 as src/ssb-jo/q42/0-naive.cu runs it (the reference has no LIP
    driver for it): dims 0 = supplier (s_region == 1, payload s_nation), 1 =
    customer (c_region == 1, key-only), 2 = part (p_mfgr IN {0, 1}, payload
    p_category), 3 = date (d_year IN {1997, 1998}, payload d_year); group by
    (s_nation, p_category, d_year); SUM(revenue - supplycost) in uint64.
    Result tuples: (s_nation, p_category, d_year, count, sum)."""
    dims = [_dim("fk_supp", "s_key", "s_region", ("in", [1]), "s_nation", (0, 24), schema.supp_rows),
            _dim("fk_cust", "c_key", "c_region", ("in", [1]), ht_len=schema.cust_rows),
            _dim("fk_part", "p_key", "p_mfgr", ("in", [0, 1]), "p_category", (0, 24), schema.part_rows),
            _date_dim(("range", 1997, 1998))]
    return _shape(dims, schema, order, lip, bf_bits_per_key, bf_hashes, adaptive, sub="supplycost")


def q43_query(schema: StarSchema, order=(0, 1, 2, 3), lip=False, bf_bits_per_key=0, bf_hashes=2,
              adaptive=False) -> Dict[str, Any]:
    """SSB Q4.3 as src/ssb-jo/q43/q43.cu runs it (no Bloom filters): dims 0 =
    supplier (s_nation == 24, payload s_city), 1 = customer (c_region == 1,
    key-only), 2 = part (p_category == 3, payload p_brand1), 3 = date (d_year IN
    {1997, 1998}, payload d_year); group by (s_city, p_brand1, d_year);
    SUM(revenue - supplycost) (int32 in the driver).
    Result tuples: (s_city, p_brand1, d_year, count, sum)."""
    dims = [_dim("fk_supp", "s_key", "s_nation", ("in", [24]), "s_city", (0, 249), schema.supp_rows),
            _dim("fk_cust", "c_key", "c_region", ("in", [1]), ht_len=schema.cust_rows),
            _dim("fk_part", "p_key", "p_category", ("in", [3]), "p_brand1", (0, 999), schema.part_rows),
            _date_dim(("range", 1997, 1998))]
    return _shape(dims, schema, order, lip, bf_bits_per_key, bf_hashes, adaptive, sub="supplycost")


SSB_SHAPES = {21: q21_query, 22: q22_query, 23: q23_query, 31: q31_query, 32: q32_query, 33: q33_query,
              34: q34_query, 41: q41_query, 42: q42_query, 43: q43_query}


def _int32(v: int) -> int:
    return ((v + 2 ** 31) % 2 ** 32) - 2 ** 31


def ssb_printed(query: int, rows: List[tuple]) -> List[tuple]:
    """Result tuples (Engine.run / oracle order) in the order the reference's
    drivers print their groups (the result loops of src/ssb-jo/q*/ drivers):
    Q2.x (d_year, p_brand1, uint64 sum); Q3.1 (d_year, c_nation, s_nation, uint64
    sum); Q3.2 / Q3.3 / Q3.4 (d_year, c_city, s_city, int32 sum); Q4.1 (d_year,
    c_nation, uint64 sum); Q4.2 (d_year, s_nation, p_category, uint64 sum); Q4.3
    (d_year, s_city, p_brand1, int32 sum).  Drivers that accumulate in int32
    print the low 32 bits of the sum as a signed value."""
    if query in (21, 22, 23):
        return sorted((y, b, v) for (b, y, c, v) in rows)
    if query == 31:
        return sorted((y, cn, sn, v) for (cn, sn, y, c, v) in rows)
    if query in (32, 33, 34):
        return sorted((y, cc, sc, _int32(v)) for (sc, cc, y, c, v) in rows)
    if query == 41:
        return sorted((y, cn, v) for (cn, y, c, v) in rows)
    if query == 42:
        return sorted((y, sn, cat, v) for (sn, cat, y, c, v) in rows)
    if query == 43:
        return sorted((y, sc, b, _int32(v)) for (sc, b, y, c, v) in rows)
    raise ValueError(f"no SSB shape {query}")


def fill_plan(query: Dict[str, Any], cols: Dict[str, Any], fact_rows: int, tune: Optional[dict] = None):
    """Translate a query description into an SjPlan over device columns.
    Returns (plan, keepalive) -- keepalive holds ctypes arrays the plan points to."""
    def ptr(name):
        if name is None:
            return None
        t = cols[name]
        return t.data_ptr() if hasattr(t, "data_ptr") else t.ctypes.data

    def nrows(name):
        return int(cols[name].shape[0])

    plan = SjPlan()
    keep = []
    dims = query["dims"]
    plan.n_dims = len(dims)
    for i, d in enumerate(dims):
        sd = plan.dims[i]
        sd.fact_fk = ptr(d["fk"])
        sd.key = ptr(d["key"])
        sd.filter_attr = ptr(d.get("attr"))
        sd.payload = ptr(d.get("payload"))
        sd.rows = nrows(d["key"])
        sd.key_min = int(d.get("key_min", 0))
        sd.ht_len = int(d["ht_len"])
        pred = d.get("pred", ("all",))
        if pred[0] == "in":
            codes = (C.c_int32 * max(1, len(pred[1])))(*pred[1])
            keep.append(codes)
            sd.pred_kind, sd.in_count, sd.in_codes = PRED_IN, len(pred[1]), C.addressof(codes)
        elif pred[0] == "range":
            sd.pred_kind, sd.pred_lo, sd.pred_hi = PRED_RANGE, int(pred[1]), int(pred[2])
        else:
            sd.pred_kind = PRED_ALL
        sd.group = 1 if d.get("group") else 0
        if d.get("group"):
            sd.payload_min, sd.payload_max = d["payload_range"]
    plan.measure = ptr(query["measure"])
    plan.measure_sub = ptr(query.get("measure_sub"))
    plan.fact_rows = fact_rows
    plan.row_begin, plan.row_end = query["row_range"]
    for i, o in enumerate(query["order"]):
        plan.order[i] = o
    plan.lip = 1 if query["lip"] else 0
    plan.adaptive = 1 if query.get("adaptive") else 0
    plan.bf_bits_per_key = query.get("bf_bits_per_key", 0)
    plan.bf_hashes = query.get("bf_hashes", 2)
    if tune:
        for k, v in tune.items():
            setattr(plan.tune, k, int(v))
    return plan, keep


def rows_to_list(rows, n: int, query: Dict[str, Any]) -> List[tuple]:
    """Result rows as sorted tuples (grouped attrs in dim order..., count, sum)."""
    gdims = [i for i, d in enumerate(query["dims"]) if d.get("group")]
    out = []
    for r in rows[:n]:
        out.append(tuple(int(r.attr[i]) for i in gdims) + (int(r.count), int(r.sum)))
    return sorted(out)


class Engine:
    """One engine handle on one device."""

    def __init__(self, device: int = 0):
        self.lib = load()
        h = C.c_void_p()
        check(self.lib.sj_engine_create(device, C.byref(h)))
        self.h = h
        self.device = device

    def close(self):
        if self.h:
            self.lib.sj_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def sm_count(self) -> int:
        return int(self.lib.sj_device_sm_count(self.h))

    def run(self, query, cols, fact_rows, host_columns=False, tune=None, cap=1 << 20, stream=None):
        """Run one query end to end (sj_run_plain); returns (rows, ms)."""
        plan, keep = fill_plan(query, cols, fact_rows, tune)
        rows = (SjGroupRow * cap)()
        n = C.c_int64()
        ms = C.c_float()
        check(self.lib.sj_run_plain(self.h, C.byref(plan), 1 if host_columns else 0, rows, cap, C.byref(n),
                                    C.byref(ms), stream))
        return rows_to_list(rows, n.value, query), ms.value

    def autotune(self, query, cols, fact_rows, reps=5, tune_filter=False, tune_order=0, verify=True,
                 cache_path=None, stream=None):
        """sj_autotune: returns (query with the chosen filter / order, chosen tuning
        dict, SjAutotuneReport)."""
        plan, keep = fill_plan(query, cols, fact_rows)
        opts = SjAutotuneOpts(reps, 1 if tune_filter else 0, tune_order, 1 if verify else 0,
                              cache_path.encode() if cache_path else None)
        rep = SjAutotuneReport()
        check(self.lib.sj_autotune(self.h, C.byref(plan), C.byref(opts), C.byref(rep), stream))
        q = dict(query)
        q["bf_bits_per_key"] = plan.bf_bits_per_key
        q["bf_hashes"] = plan.bf_hashes
        q["order"] = [plan.order[i] for i in range(len(query["dims"]))]
        tune = {f: getattr(plan.tune, f) for f, _ in SjTuning._fields_}
        return q, tune, rep

    def prepare(self, query, cols, fact_rows, tune=None) -> "Query":
        plan, keep = fill_plan(query, cols, fact_rows, tune)
        h = C.c_void_p()
        check(self.lib.sj_query_prepare(self.h, C.byref(plan), C.byref(h)))
        return Query(self, h, query, keep, cols)


class Query:
    """A prepared query: build/probe can be re-run (device state is reused)."""

    def __init__(self, eng: Engine, h, query, keep, cols):
        self.eng, self.h, self.query, self._keep, self._cols = eng, h, query, keep, cols

    def build(self, stream=None):
        check(self.eng.lib.sj_query_build(self.h, stream))

    def probe(self, stream=None):
        check(self.eng.lib.sj_query_probe(self.h, stream))

    def fetch(self, cap=1 << 20, stream=None):
        rows = (SjGroupRow * cap)()
        n = C.c_int64()
        check(self.eng.lib.sj_query_fetch(self.h, rows, cap, C.byref(n), stream))
        return rows_to_list(rows, n.value, self.query)

    def stats(self) -> SjQueryStats:
        s = SjQueryStats()
        check(self.eng.lib.sj_query_get_stats(self.h, C.byref(s)))
        return s

    def release(self):
        if self.h:
            self.eng.lib.sj_query_release(self.h)
            self.h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass
