"""Measurements of the shared-scan forms, reported by bench.py.

batched(): 64 star-join queries (2-4 dimensions, selectivity log-uniform in
[0.05%, 60%], fact row range log-uniform in [1M, 120M]) over a shared 120M-row
fact table with supplier / customer / part / date dimensions, one batch = one
CUDA-graph replay; against the same queries run back to back through the plain
engine (sj_run_plain, device columns).  Results are compared query by query.

serving(): a resident 300M-row fact table; Poisson arrivals of such queries at
fixed rates; per-query latency (submit -> result available) from the server's
own clock, p50/p99, and throughput; the same schedule through the plain
one-at-a-time loop.
"""
from __future__ import annotations

import ctypes as C
import random
import statistics
import threading
import time
from typing import Any, Dict, List

import shared_scan as ss
import starjoin as sj

BATCH_SCHEMA = dict(seed=0x5EED0007, fact_rows=120_000_000, cust_rows=600_000, supp_rows=40_000,
                    part_rows=1_000_000)
SERVE_SCHEMA = dict(seed=0x5EED0008, fact_rows=300_000_000, cust_rows=1_500_000, supp_rows=100_000,
                    part_rows=1_400_000)
BYTES_PER_ROW_4DIM = 20  # 4 FK columns + revenue


class PlainRunner:
    """Back-to-back plain queries through sj_run_plain with prebuilt plans and
    one reusable result buffer (no per-query Python allocation in the loop)."""

    def __init__(self, eng: sj.Engine, sc: sj.StarSchema, dev: Dict[str, Any], queries: List[Dict[str, Any]]):
        self.eng, self.sc = eng, sc
        self.cap = 1 << 18
        self.rows = (sj.SjGroupRow * self.cap)()
        self.plans = []
        self.keep = []
        self.plain = [ss.to_plain(sc, q) for q in queries]
        for pq in self.plain:
            plan, keep = sj.fill_plan(pq, dev, sc.fact_rows)
            self.plans.append(plan)
            self.keep.append(keep)

    def run_all(self, stream=None):
        """(results, device ms per query, wall seconds of the loop of C calls)."""
        lib = self.eng.lib
        n = C.c_int64()
        ms = C.c_float()
        raw, dev_ms = [], []
        size = C.sizeof(sj.SjGroupRow)
        t0 = time.perf_counter()
        for plan in self.plans:
            sj.check(lib.sj_run_plain(self.eng.h, C.byref(plan), 0, self.rows, self.cap, C.byref(n), C.byref(ms),
                                      stream))
            dev_ms.append(ms.value)
            raw.append(C.string_at(self.rows, n.value * size))
        wall = time.perf_counter() - t0
        out = []
        for b, pq in zip(raw, self.plain):
            rows = (sj.SjGroupRow * max(1, len(b) // size)).from_buffer_copy(b.ljust(size, b"\0"))
            out.append(sj.rows_to_list(rows, len(b) // size, pq))
        return out, dev_ms, wall


def _tuned(eng: sj.Engine, sc: sj.StarSchema, dev, sample, threads: int, tune: bool):
    """The probe shape for the batched and served forms: sjb_batch_tune on a
    sample batch (outside every timed region) unless `threads` fixes it."""
    if threads or not tune:
        return {"threads": threads, "smem_group_entries": 0}, None
    shape, rep = ss.tune_batch(eng, sc, dev, sample, reps=3)
    return shape, {"candidates": rep.candidates, "mismatches": rep.mismatches, "threads": rep.threads,
                   "smem_group_entries": rep.smem_group_entries, "best_probe_ms": rep.best_probe_ms,
                   "default_probe_ms": rep.default_probe_ms}


def batched(eng: sj.Engine, n_batches: int = 6, per_batch: int = 64, seed: int = 2024,
            schema: Dict[str, int] = None, threads: int = 0, tune: bool = True) -> Dict[str, Any]:
    sc = sj.StarSchema(**(schema or BATCH_SCHEMA))
    dev = sj.gen_device(sc)
    rng = random.Random(seed)
    batches = [[ss.random_query(rng, sc) for _ in range(per_batch)] for _ in range(n_batches + 2)]
    shape, tuning = _tuned(eng, sc, dev, batches[0], threads, tune)
    b = ss.Batch(eng, sc, dev, use_graph=True, cache_filters=False, **shape)
    try:
        for qs in batches[:2]:  # warm-up: graph instantiation, first touches
            b.run_raw(b.describe(qs))
        dev_ms, wall, probe_ms, rows_read, results = [], [], [], [], []
        for qs in batches[2:]:
            desc = b.describe(qs)
            t0 = time.perf_counter()
            n = b.run_raw(desc)
            wall.append(time.perf_counter() - t0)
            res = b.rows(n, qs)
            st = b.stats()
            dev_ms.append(st.ms_total)
            probe_ms.append(st.ms_probe)
            rows_read.append(st.rows_scanned)
            results.append(res)
    finally:
        b.close()
    # the same queries back to back through the plain engine (two batches' worth)
    plain_dev, plain_wall, exact = [], [], True
    for qs, res in list(zip(batches[2:], results))[:2]:
        pr = PlainRunner(eng, sc, dev, qs)
        pr.run_all()  # warm-up
        out, ms, w = pr.run_all()
        plain_dev.append(sum(ms))
        plain_wall.append(w)
        exact = exact and out == res
    qps_dev = per_batch / (statistics.mean(dev_ms) / 1e3)
    qps_wall = per_batch / statistics.mean(wall)
    plain_qps_dev = per_batch / (statistics.mean(plain_dev) / 1e3)
    plain_qps_wall = per_batch / statistics.mean(plain_wall)
    sum_ranges = statistics.mean(sum(q["row_range"][1] - q["row_range"][0] for q in qs) for qs in batches[2:])
    probe = statistics.mean(probe_ms)
    del dev
    return {
        "workload": f"{per_batch} queries/batch, 2-4 dims, selectivity log-uniform [0.05%, 60%], "
                    f"row range log-uniform [1M, {sc.fact_rows // 1_000_000}M], fact {sc.fact_rows} rows",
        "queries_per_s": qps_dev, "queries_per_s_wall": qps_wall,
        "ms_per_batch": statistics.mean(dev_ms), "ms_per_batch_each": dev_ms, "probe_ms_per_batch": probe,
        "plain_queries_per_s": plain_qps_dev, "plain_queries_per_s_wall": plain_qps_wall,
        "plain_ms_per_batch": statistics.mean(plain_dev),
        "speedup_vs_plain": qps_dev / plain_qps_dev, "speedup_vs_plain_wall": qps_wall / plain_qps_wall,
        "bit_exact_vs_plain": exact, "batches_timed": n_batches,
        "shared_scan_rows": statistics.mean(rows_read), "sum_of_query_ranges": sum_ranges,
        "probe_hbm_gbs_algorithmic": BYTES_PER_ROW_4DIM * statistics.mean(rows_read) / (probe / 1e3) / 1e9,
        "cuda_graph": True, "filters_cached": False, "probe_shape": shape, "tuning": tuning,
    }


def _poisson_run(srv: ss.Server, queries: List[Dict[str, Any]], rate: float, seed: int):
    rng = random.Random(seed)
    tickets = []
    t_next = time.perf_counter()
    for q in queries:
        if rate == float("inf"):
            tickets.append(srv.submit(q))
            continue
        t_next += rng.expovariate(rate)
        while True:
            d = t_next - time.perf_counter()
            if d <= 0:
                break
            if d > 2e-4:
                time.sleep(d - 1e-4)
        tickets.append(srv.submit(q))
    lat, first, last, rows = [], None, None, []
    for t in tickets:
        r, info = srv.wait(t, timeout_s=600.0)
        rows.append(r)
        lat.append(info.finish_s - info.submit_s)
        first = info.submit_s if first is None else min(first, info.submit_s)
        last = info.finish_s if last is None else max(last, info.finish_s)
    lat.sort()
    return {
        "queries": len(queries), "offered_qps": rate,
        "throughput_qps": len(queries) / (last - first) if last > first else 0.0,
        "p50_ms": 1e3 * lat[len(lat) // 2], "p99_ms": 1e3 * lat[min(len(lat) - 1, int(0.99 * len(lat)))],
        "max_ms": 1e3 * lat[-1],
    }, rows


def serving(eng: sj.Engine, rates=(50.0, 200.0, 2000.0), seconds: float = 1.0, seed: int = 77,
            schema: Dict[str, int] = None, plain_cap: int = 300, flood: int = 2048, mixes: int = 3,
            threads: int = 0, tune: bool = True) -> Dict[str, Any]:
    sc = sj.StarSchema(**(schema or SERVE_SCHEMA))
    dev = sj.gen_device(sc)
    trng = random.Random(seed + 5)
    shape, tuning = _tuned(eng, sc, dev, [ss.random_query(trng, sc) for _ in range(64)], threads, tune)
    rng = random.Random(seed)
    out: Dict[str, Any] = {"workload": f"Poisson arrivals, 2-4 dims, selectivity log-uniform [0.05%, 60%], row "
                                       f"range log-uniform [1M, {sc.fact_rows // 1_000_000}M], resident fact "
                                       f"{sc.fact_rows} rows", "rates": []}
    exact = True
    for i, rate in enumerate(rates):
        n = max(20, int(rate * seconds))
        qs = [ss.random_query(rng, sc) for _ in range(n)]
        srv = ss.Server(eng, sc, dev, cache_filters=True, **shape)
        try:
            warm = [ss.random_query(random.Random(seed + 1000 + i), sc) for _ in range(8)]
            for t in [srv.submit(q) for q in warm]:
                srv.wait(t, timeout_s=600.0)
            shared, shared_rows = _poisson_run(srv, qs, rate, seed + i)
            st = srv.stats()
            shared.update({"steps": st.steps, "peak_active": st.peak_active, "rows_scanned": st.rows_scanned,
                           "filters_built": st.filters_built, "filters_cached": st.filters_cached})
        finally:
            srv.close()
        # the same arrivals with lone queries sent through the plain engine
        srv = ss.Server(eng, sc, dev, cache_filters=True, solo_plain=True, **shape)
        try:
            for t in [srv.submit(q) for q in warm]:
                srv.wait(t, timeout_s=600.0)
            solo, solo_rows = _poisson_run(srv, qs, rate, seed + i)
            st = srv.stats()
            solo.update({"steps": st.steps, "solo": st.solo, "peak_active": st.peak_active})
        finally:
            srv.close()
        exact = exact and solo_rows == shared_rows
        m = min(n, plain_cap)
        srv = ss.Server(eng, sc, dev, plain=True)
        try:
            plain, plain_rows = _poisson_run(srv, qs[:m], rate, seed + i)
        finally:
            srv.close()
        exact = exact and plain_rows == shared_rows[:m]
        out["rates"].append({"shared": shared, "shared_solo_plain": solo, "plain": plain})
    # saturation: every query of a mix submitted at once -- the loops' capacity,
    # over several seeded mixes of `flood` queries each
    if flood:
        runs = []
        for mix in range(mixes):
            mrng = random.Random(seed * 1009 + mix)
            qs = [ss.random_query(mrng, sc) for _ in range(flood)]
            res = {"seed": seed * 1009 + mix}
            for plain in (False, True):
                srv = ss.Server(eng, sc, dev, plain=plain, cache_filters=True, **shape)
                try:
                    r, rows = _poisson_run(srv, qs, float("inf"), seed)
                    st = srv.stats()
                    r.update({"steps": st.steps, "busy_s": st.busy_s, "admit_s": st.admit_s, "scan_s": st.scan_s,
                              "probe_device_s": st.probe_device_s, "peak_active": st.peak_active,
                              "rows_scanned": st.rows_scanned})
                finally:
                    srv.close()
                res["plain" if plain else "shared"] = r
                res["rows_plain" if plain else "rows_shared"] = rows
            exact = exact and res.pop("rows_plain") == res.pop("rows_shared")
            res["speedup_vs_plain"] = res["shared"]["throughput_qps"] / max(res["plain"]["throughput_qps"], 1e-9)
            runs.append(res)
        ratios = [r["speedup_vs_plain"] for r in runs]
        out["saturation"] = {"mixes": runs, "queries_per_mix": flood, "speedup_min": min(ratios),
                             "speedup_mean": statistics.mean(ratios),
                             "shared_qps_mean": statistics.mean(r["shared"]["throughput_qps"] for r in runs),
                             "plain_qps_mean": statistics.mean(r["plain"]["throughput_qps"] for r in runs)}
    out["bit_exact_vs_plain"] = exact
    out["probe_shape"], out["tuning"] = shape, tuning
    del dev
    return out
