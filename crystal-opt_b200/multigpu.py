"""Host logic of the multi-GPU star join: row sharding and the group merge.

The fact table partitions naturally: each rank scans a contiguous row range
against replicated dimension tables and produces exact group partials (counts
and two's-complement uint64 sums).  The one exchange step is the merge of those
partials: every rank all-gathers the compact rows of every other rank (a tensor
collective, so it runs on NCCL over NVLink as well as on gloo) and adds them.
Integer addition is order-independent, so the merged result equals a
single-GPU run bit for bit.
"""
from __future__ import annotations

from typing import Dict, List, Sequence, Tuple

import torch

M64 = (1 << 64) - 1


def row_range(n_rows: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous shard of [0, n_rows) for `rank`; shard starts are multiples of 4
    rows so every shard's first column keeps 16-byte alignment."""
    def cut(r: int) -> int:
        return n_rows if r >= world else (n_rows * r // world) & ~3
    return cut(rank), cut(rank + 1)


def _to_tensor(rows: Sequence[tuple], width: int) -> torch.Tensor:
    t = torch.zeros((len(rows), width), dtype=torch.int64)
    for i, r in enumerate(rows):
        vals = list(r[:-1]) + [r[-1] - (1 << 64) if r[-1] >= (1 << 63) else r[-1]]
        t[i] = torch.tensor(vals, dtype=torch.int64)
    return t


def merge_groups(rows: Sequence[tuple], n_keys: int, dist, device: str = "cpu") -> List[tuple]:
    """All-gather every rank's group rows (key attrs..., count, uint64 sum) and add
    them up; every rank returns the same sorted merged rows."""
    width = n_keys + 2
    local = _to_tensor(rows, width).to(device)
    n = torch.tensor([local.shape[0]], dtype=torch.int64, device=device)
    world = dist.get_world_size()
    counts = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(counts, n)
    cap = max(int(c.item()) for c in counts)
    padded = torch.zeros((max(cap, 1), width), dtype=torch.int64, device=device)
    if local.shape[0]:
        padded[: local.shape[0]] = local
    parts = [torch.zeros_like(padded) for _ in range(world)]
    dist.all_gather(parts, padded)
    merged: Dict[tuple, List[int]] = {}
    for c, p in zip(counts, parts):
        for row in p[: int(c.item())].cpu().tolist():
            key = tuple(row[:n_keys])
            acc = merged.setdefault(key, [0, 0])
            acc[0] += row[n_keys]
            acc[1] = (acc[1] + row[n_keys + 1]) & M64
    return sorted(k + (c, s) for k, (c, s) in merged.items())
