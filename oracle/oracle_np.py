"""Vectorised numpy restatement of the reference star join -- TEST INFRASTRUCTURE.

An independent second oracle for small inputs, used to cross-check oracle.c.
It follows the same reference semantics: the PHT build of
BlockBuildSelectivePHT_2 (crystal/join.cuh:260-335: slot (key - key_min) % len,
first key claims the slot, last qualifying value stays), the PHT_2 probe
(crystal/join.cuh:108-131: a row joins iff its slot holds a nonzero key), and
the uint64 group-by SUM of src/ssb-jo/q31/0-lip.cu:98-113.
"""
from __future__ import annotations

from typing import Any, Dict, List

import numpy as np


def _slot(keys: np.ndarray, kmin: int, ln: int) -> np.ndarray:
    d = (keys.astype(np.int64) - kmin) & 0xFFFFFFFF  # unsigned 32-bit offset
    return (d % ln).astype(np.int64)


def _pred(d: Dict[str, Any], cols: Dict[str, np.ndarray]) -> np.ndarray:
    pred = d.get("pred", ("all",))
    n = len(cols[d["key"]])
    if pred[0] == "all":
        return np.ones(n, dtype=bool)
    a = cols[d["attr"]]
    if pred[0] == "range":
        return (a >= pred[1]) & (a <= pred[2])
    return np.isin(a, np.asarray(pred[1], dtype=np.int64))


def build_pht(d: Dict[str, Any], cols: Dict[str, np.ndarray]) -> np.ndarray:
    ln = int(d["ht_len"])
    ht = np.zeros(2 * ln, dtype=np.int32)
    q = np.nonzero(_pred(d, cols))[0]
    keys = cols[d["key"]][q]
    vals = cols[d["payload"]][q] if d.get("payload") else np.zeros(len(q), dtype=np.int32)
    s = _slot(keys, int(d.get("key_min", 0)), ln)
    # first key per slot (stable), last value per slot
    for i in range(len(q)):
        if ht[2 * s[i]] == 0:
            ht[2 * s[i]] = keys[i]
        ht[2 * s[i] + 1] = vals[i]
    return ht


def run(query: Dict[str, Any], cols: Dict[str, np.ndarray]) -> List[tuple]:
    b, e = query["row_range"]
    dims = query["dims"]
    live = np.ones(e - b, dtype=bool)
    payload = []
    for d in dims:
        ht = build_pht(d, cols)
        s = _slot(cols[d["fk"]][b:e], int(d.get("key_min", 0)), int(d["ht_len"]))
        live &= ht[2 * s] != 0
        payload.append(ht[2 * s + 1])
    m = cols[query["measure"]][b:e].astype(np.int64)
    if query.get("measure_sub"):
        m = m - cols[query["measure_sub"]][b:e].astype(np.int64)
    gd = [i for i, d in enumerate(dims) if d.get("group")]
    idx = np.nonzero(live)[0]
    if len(idx) == 0:
        return []
    keys = np.stack([payload[i][idx] for i in gd], axis=1) if gd else np.zeros((len(idx), 0), np.int64)
    mv = m[idx].astype(np.uint64)  # two's complement wrap, like the uint64 atomicAdd
    res: Dict[tuple, list] = {}
    for row, v in zip(map(tuple, keys.tolist()), mv.tolist()):
        acc = res.setdefault(row, [0, 0])
        acc[0] += 1
        acc[1] = (acc[1] + v) & 0xFFFFFFFFFFFFFFFF
    return sorted(k + (c, s) for k, (c, s) in res.items())
