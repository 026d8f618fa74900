"""Host logic of the multi-GPU star join: row sharding and the group merge.

The fact table partitions naturally: each rank scans a contiguous row range
against replicated dimension tables and produces exact group partials (counts
and two's-complement uint64 sums).  The one exchange step is the merge of those
partials.  Every rank lays its partials out densely over the query's group space
(the product of the grouped payload ranges, identical on every rank because the
dimensions are replicated) and one all-reduce adds them: on NCCL that is a
single ncclAllReduce over NVLink, on gloo the same call on the CPU.  The 64-bit
sums travel as two 32-bit halves in int64 lanes, so the reduction is exact for
any number of ranks and never relies on signed overflow.  Group spaces too large
to lay out densely fall back to an all-gather of the compact rows, merged with
numpy.  Integer addition is order-independent, so the merged result equals a
single-GPU run bit for bit.
"""
from __future__ import annotations

from typing import Any, Dict, List, Sequence, Tuple

import numpy as np
import torch

M64 = (1 << 64) - 1
DENSE_MAX = 1 << 24  # largest group space merged densely (3 x 8 B x 16M = 384 MB per rank)


def row_range(n_rows: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous shard of [0, n_rows) for `rank`; shard starts are multiples of 4
    rows so every shard's first column keeps 16-byte alignment."""
    def cut(r: int) -> int:
        return n_rows if r >= world else (n_rows * r // world) & ~3
    return cut(rank), cut(rank + 1)


def group_spans(query: Dict[str, Any]) -> List[Tuple[int, int]]:
    """(payload_min, span) of each grouped dimension, in dimension order: the
    axes of the query's dense group space."""
    out = []
    for d in query["dims"]:
        if d.get("group"):
            lo, hi = d["payload_range"]
            out.append((int(lo), int(hi) - int(lo) + 1))
    return out


def _rows_array(rows: Sequence[tuple], n_keys: int) -> np.ndarray:
    """Compact rows (keys..., count, uint64 sum) as int64 [n, n_keys + 3]:
    keys, count, low and high 32-bit halves of the sum."""
    a = np.zeros((len(rows), n_keys + 3), dtype=np.int64)
    if rows:
        r = np.array([list(x[:n_keys + 1]) for x in rows], dtype=np.int64).reshape(len(rows), n_keys + 1)
        s = np.array([x[n_keys + 1] & M64 for x in rows], dtype=np.uint64)
        a[:, : n_keys + 1] = r
        a[:, n_keys + 1] = (s & np.uint64(0xFFFFFFFF)).astype(np.int64)
        a[:, n_keys + 2] = (s >> np.uint64(32)).astype(np.int64)
    return a


def _rows_list(keys: np.ndarray, cnt: np.ndarray, lo: np.ndarray, hi: np.ndarray) -> List[tuple]:
    total = ((hi.astype(np.uint64) << np.uint64(32)) + lo.astype(np.uint64))  # wraps modulo 2^64
    out = [tuple(int(k) for k in keys[i]) + (int(cnt[i]), int(total[i])) for i in range(len(cnt))]
    return sorted(out)


def merge_dense(rows: Sequence[tuple], spans: Sequence[Tuple[int, int]], dist, device: str = "cpu") -> List[tuple]:
    """All-reduce every rank's group partials over the dense group space."""
    n_keys = len(spans)
    space = 1
    for _, s in spans:
        space *= s
    a = _rows_array(rows, n_keys)
    strides, st = [], 1
    for _, s in reversed(spans):
        strides.append(st)
        st *= s
    strides = strides[::-1]
    idx = np.zeros(len(a), dtype=np.int64)
    for j, ((lo, s), stride) in enumerate(zip(spans, strides)):
        k = a[:, j] - lo
        if np.any((k < 0) | (k >= s)):
            raise ValueError("group key outside its payload range")
        idx += k * stride
    dense = torch.zeros((3, max(space, 1)), dtype=torch.int64)
    if len(a):
        t = torch.from_numpy(idx)
        dense[0, t] = torch.from_numpy(a[:, n_keys].copy())
        dense[1, t] = torch.from_numpy(a[:, n_keys + 1].copy())
        dense[2, t] = torch.from_numpy(a[:, n_keys + 2].copy())
    dense = dense.to(device)
    dist.all_reduce(dense)  # SUM: one collective, the exchange step
    dense = dense.cpu().numpy()
    nz = np.nonzero(dense[0])[0]
    keys = np.zeros((len(nz), n_keys), dtype=np.int64)
    rem = nz.copy()
    for j, ((lo, s), stride) in enumerate(zip(spans, strides)):
        keys[:, j] = rem // stride + lo
        rem = rem % stride
    # carry the low halves' overflow into the high halves before recombining
    lo_sum = dense[1, nz]
    hi_sum = dense[2, nz] + (lo_sum >> 32)
    return _rows_list(keys, dense[0, nz], lo_sum & 0xFFFFFFFF, hi_sum & 0xFFFFFFFF)


def merge_gather(rows: Sequence[tuple], n_keys: int, dist, device: str = "cpu") -> List[tuple]:
    """All-gather every rank's compact rows and add them up (numpy)."""
    a = torch.from_numpy(_rows_array(rows, n_keys)).to(device)
    n = torch.tensor([a.shape[0]], dtype=torch.int64, device=device)
    world = dist.get_world_size()
    counts = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(counts, n)
    cap = max(int(c.item()) for c in counts)
    padded = torch.zeros((max(cap, 1), n_keys + 3), dtype=torch.int64, device=device)
    if a.shape[0]:
        padded[: a.shape[0]] = a
    parts = [torch.zeros_like(padded) for _ in range(world)]
    dist.all_gather(parts, padded)
    allrows = np.concatenate([p[: int(c.item())].cpu().numpy() for c, p in zip(counts, parts)], axis=0)
    if not len(allrows):
        return []
    keys, inv = np.unique(allrows[:, :n_keys], axis=0, return_inverse=True)
    inv = inv.reshape(-1)
    acc = np.zeros((len(keys), 3), dtype=np.int64)
    np.add.at(acc, inv, allrows[:, n_keys:])
    hi = acc[:, 2] + (acc[:, 1] >> 32)
    return _rows_list(keys, acc[:, 0], acc[:, 1] & 0xFFFFFFFF, hi & 0xFFFFFFFF)


def merge_groups(rows: Sequence[tuple], query: Dict[str, Any], dist, device: str = "cpu") -> List[tuple]:
    """Merge every rank's group rows of `query` (grouped attrs..., count, uint64
    sum); every rank returns the same sorted merged rows.  Dense all-reduce when
    the group space has at most DENSE_MAX slots, else an all-gather."""
    spans = group_spans(query)
    space = 1
    for _, s in spans:
        space *= s
    if space <= DENSE_MAX:
        return merge_dense(rows, spans, dist, device)
    return merge_gather(rows, len(spans), dist, device)
