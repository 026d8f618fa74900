"""Python binding of the CPU oracle (oracle.c) -- TEST INFRASTRUCTURE.

Only the tests, the smoke check and the benchmark's CPU-baseline / reference
legs use this module, as the checker; the engine never imports it.  The query
description is the same plain dict the engine's harness uses (dims with column
names, predicate, group flag and payload range; measure; row range; order), so
one description drives both sides of a parity test.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Any, Dict, List, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "liboracle.so")
MAX_DIMS = 4


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "oracle.c")
    deps = [src, os.path.join(HERE, "oracle.h"),
            os.path.join(os.path.dirname(HERE), "crystal-opt_b200", "csrc", "sj_datagen.h")]
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(d) for d in deps):
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    tmp = LIB + ".tmp"
    subprocess.run(["gcc", "-O3", "-march=native", "-std=c11", "-fPIC", "-shared", "-pthread",
                    "-o", tmp, src], check=True)
    os.replace(tmp, LIB)
    return LIB


class OrDim(C.Structure):
    _fields_ = [
        ("fact_fk", C.c_void_p), ("key", C.c_void_p), ("filter_attr", C.c_void_p),
        ("payload", C.c_void_p), ("rows", C.c_int64), ("key_min", C.c_int32),
        ("ht_len", C.c_int32), ("pred_kind", C.c_int32), ("pred_lo", C.c_int32),
        ("pred_hi", C.c_int32), ("in_count", C.c_int32), ("in_codes", C.c_void_p),
        ("group", C.c_int32), ("payload_min", C.c_int32), ("payload_max", C.c_int32),
    ]


class OrPlan(C.Structure):
    _fields_ = [("n_dims", C.c_int32), ("dims", OrDim * MAX_DIMS), ("measure", C.c_void_p),
                ("measure_sub", C.c_void_p), ("row_begin", C.c_int64), ("row_end", C.c_int64),
                ("order", C.c_int32 * MAX_DIMS)]


class OrGroupRow(C.Structure):
    _fields_ = [("attr", C.c_int32 * MAX_DIMS), ("count", C.c_uint64), ("sum", C.c_uint64)]


_lib: Optional[C.CDLL] = None


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        lib = C.CDLL(build())
        lib.or_starjoin.restype = C.c_int
        lib.or_starjoin.argtypes = [C.POINTER(OrPlan), C.c_int, C.POINTER(OrGroupRow), C.c_int64,
                                    C.POINTER(C.c_int64)]
        lib.or_build_pht.restype = C.c_int
        lib.or_build_pht.argtypes = [C.POINTER(OrDim), C.c_void_p]
        lib.or_available_cores.restype = C.c_int
        lib.or_gen_column.restype = None
        lib.or_gen_column.argtypes = [C.c_void_p, C.c_int64, C.c_uint64, C.c_int32, C.c_int32, C.c_int32,
                                      C.c_int32, C.c_int]
        lib.or_gen_rows.restype = None
        lib.or_gen_rows.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_uint64, C.c_int32, C.c_int32, C.c_int32,
                                    C.c_int32, C.c_int]
        _lib = lib
    return _lib


def cores() -> int:
    return int(load().or_available_cores())


def gen_host(schema, names=None, threads: int = 0, fact_range=None) -> Dict[str, np.ndarray]:
    """The schema's seeded columns generated by this library (same values as the
    engine's generator), for CPU legs that must not load the engine.  `schema`
    is a starjoin.StarSchema (its column specs are plain Python).
    fact_range=(b, e): only rows [b, e) of the fact columns."""
    lib = load()
    derived_specs = schema.derived_specs()
    want = set(schema.column_names()) if names is None else set(names)
    bases = {n for n in want if n in schema.column_specs()} | {derived_specs[n][0] for n in want if n in derived_specs}
    out: Dict[str, np.ndarray] = {}
    for name, (n, col, kind, lo, hi) in schema.column_specs().items():
        if name in bases:
            row0 = 0
            if fact_range is not None and n == schema.fact_rows:
                row0, n = int(fact_range[0]), int(fact_range[1]) - int(fact_range[0])
            a = np.empty(max(n, 0), dtype=np.int32)
            lib.or_gen_rows(a.ctypes.data, row0, n, schema.seed, col, kind, lo, hi, threads)
            out[name] = a
    for name, (base, div) in derived_specs.items():
        if name in want:
            out[name] = (out[base] // div).astype(np.int32)
    return {k: v for k, v in out.items() if k in want}


def _plan(query: Dict[str, Any], cols: Dict[str, np.ndarray]):
    keep: List[Any] = []

    def ptr(name):
        if name is None:
            return None
        a = np.ascontiguousarray(cols[name], dtype=np.int32)
        keep.append(a)
        return a.ctypes.data

    p = OrPlan()
    p.n_dims = len(query["dims"])
    for i, d in enumerate(query["dims"]):
        od = p.dims[i]
        od.fact_fk = ptr(d["fk"])
        od.key = ptr(d["key"])
        od.filter_attr = ptr(d.get("attr"))
        od.payload = ptr(d.get("payload"))
        od.rows = int(len(cols[d["key"]]))
        od.key_min = int(d.get("key_min", 0))
        od.ht_len = int(d["ht_len"])
        pred = d.get("pred", ("all",))
        if pred[0] == "in":
            codes = np.asarray(pred[1], dtype=np.int32)
            keep.append(codes)
            od.pred_kind, od.in_count, od.in_codes = 1, len(codes), codes.ctypes.data
        elif pred[0] == "range":
            od.pred_kind, od.pred_lo, od.pred_hi = 2, int(pred[1]), int(pred[2])
        else:
            od.pred_kind = 0
        od.group = 1 if d.get("group") else 0
        if d.get("group"):
            od.payload_min, od.payload_max = d["payload_range"]
    p.measure = ptr(query["measure"])
    p.measure_sub = ptr(query.get("measure_sub"))
    p.row_begin, p.row_end = query["row_range"]
    for i, o in enumerate(query["order"]):
        p.order[i] = o
    return p, keep


def run(query: Dict[str, Any], cols: Dict[str, np.ndarray], threads: int = 0) -> List[tuple]:
    """Sorted result tuples (grouped attrs in dim order..., count, sum)."""
    lib = load()
    p, keep = _plan(query, cols)
    n = C.c_int64()
    cap = 1 << 16
    while True:
        rows = (OrGroupRow * cap)()
        rc = lib.or_starjoin(C.byref(p), threads, rows, cap, C.byref(n))
        if rc == 5 and n.value > cap:
            cap = n.value
            continue
        if rc != 0:
            raise RuntimeError(f"oracle error {rc}")
        break
    gdims = [i for i, d in enumerate(query["dims"]) if d.get("group")]
    return sorted(tuple(int(r.attr[i]) for i in gdims) + (int(r.count), int(r.sum))
                  for r in rows[:n.value])


def build_pht(query: Dict[str, Any], cols: Dict[str, np.ndarray], dim: int) -> np.ndarray:
    """The reference-layout PHT (2 x int32 per slot) of one dimension."""
    lib = load()
    p, keep = _plan(query, cols)
    ht = np.zeros(2 * int(query["dims"][dim]["ht_len"]), dtype=np.int32)
    if lib.or_build_pht(C.byref(p.dims[dim]), ht.ctypes.data) != 0:
        raise RuntimeError("oracle build failed")
    return ht
