#!/usr/bin/env python
"""Benchmark: the 3-dimension LIP star join (SSB Q3.3 shape) on 120M fact rows.

One step = one query through the engine: dimension builds (predicate ->
filter + PHT insert) and the fused scan/filter/probe/aggregate kernel, exactly
the span the reference's time_query covers (src/ssb-jo/q33/0-lip.cu:216-278).
Inputs (1.92 GB of fact columns) are resident in HBM and larger than the 126 MB
L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

Prints one JSON line (rank 0).  With N > 1 (torchrun), one seeded fact table of
N x 120M rows is sharded by contiguous row ranges, each rank scanning its own
120M-row shard (weak scaling) against replicated dimensions; the group partials
merge in one all-reduce and rank 0 checks the merge against the oracle.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "crystal-opt_b200"))

FACT_ROWS = 120_000_000
CUST_ROWS, SUPP_ROWS = 600_000, 40_000
SEED = 0x5EED0002
BYTES_PER_ROW = 16  # 3 FK columns + revenue, int32 (algorithmic bytes per fact row)
PROBE_EVERY = 20  # timed steps per probe-event sample
METRIC = "fact rows/s, 3-dim LIP star join (SSB Q3.3 shape)"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling in the background."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,utilization.gpu")

    def __init__(self, device: int):
        self.device = device
        self.samples = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 10:
                self.samples.append((time.time(), parts))

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self, t0: float, t1: float):
        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        window = [p for t, p in self.samples if t0 <= t <= t1]
        loaded = [p for p in window if (num(p[9]) or 0) > 0] or window
        if not loaded:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        sm = [num(p[1]) for p in loaded if num(p[1]) is not None]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for p in loaded:
            for name, v in zip(names, p[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": num(loaded[0][2]),
                "reasons": sorted(reasons), "samples": len(loaded),
                "power_w_max": max((num(p[3]) or 0) for p in loaded)}


def _traffic_from_profiles(bpk: int):
    """Per-launch DRAM bytes (read + write) of the probe kernel, from the committed
    ncu capture of one launch of this workload; (bytes, how) or (None, why)."""
    path = os.path.join(ROOT, "profiles", "probe_traffic.json")
    try:
        with open(path) as f:
            rec = json.load(f)
    except Exception:
        return None, "no profiles/probe_traffic.json"
    ent = rec.get(f"bpk{bpk}")
    if not ent or not ent.get("fact_rows"):
        return None, f"no capture for bf_bits_per_key={bpk}"
    if ent["fact_rows"] == FACT_ROWS:
        return ent["dram_bytes_per_launch"], f"ncu, one launch at {FACT_ROWS} rows ({ent.get('capture', '')})"
    return (ent["dram_bytes_per_launch"] * FACT_ROWS / ent["fact_rows"],
            f"ncu at {ent['fact_rows']} rows scaled by rows ({ent.get('capture', '')})")


def cpu_baseline(host_cols, query, budget_s: float = 12.0):
    """The oracle's multithreaded host plan on this box's cores, same workload;
    returns the baseline record and the oracle's groups."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    cores = oracle.cores()
    times = []
    t_end = time.perf_counter() + budget_s
    res = None
    while len(times) < 5 and (not times or time.perf_counter() < t_end):
        t0 = time.perf_counter()
        res = oracle.run(query, host_cols, threads=cores)
        times.append(time.perf_counter() - t0)
    t = statistics.median(times)
    return {"value": FACT_ROWS / t, "unit": "rows/s", "cores": cores, "kind": "port",
            "sample": f"full {FACT_ROWS // 1_000_000}M-row workload, median of {len(times)} runs, "
                      f"{t * 1e3:.1f} ms each"}, res


def _oracle_sharded(global_schema, world, bpk):
    """The single-process answer over the whole (world x FACT_ROWS)-row table: the
    oracle shard by shard on this host (one shard's columns in memory at a time),
    partial groups added modulo 2^64."""
    import starjoin as sj
    import multigpu
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    acc = {}
    dims = oracle.gen_host(global_schema, ["c_key", "c_city", "s_key", "s_city", "d_key", "d_year"])
    for r in range(world):
        b, e = multigpu.row_range(global_schema.fact_rows, r, world)
        cols = dict(dims)
        cols.update(oracle.gen_host(global_schema, ["fk_cust", "fk_supp", "fk_date", "revenue"], fact_range=(b, e)))
        local = sj.StarSchema(seed=SEED, fact_rows=e - b, cust_rows=CUST_ROWS, supp_rows=SUPP_ROWS)
        for row in oracle.run(sj.q33_query(local, order=(0, 1, 2), lip=True, bf_bits_per_key=bpk), cols):
            a = acc.setdefault(row[:3], [0, 0])
            a[0] += row[3]
            a[1] = (a[1] + row[4]) % (1 << 64)
        del cols
    return sorted(k + (c, v) for k, (c, v) in acc.items())


def run_reference(args):
    """Reference arm: the reference has no CPU implementation of the path, so the
    line's value is the oracle's port of its plan on the host cores; the
    reference's own CUDA drivers (oracle/_ref) are timed on the GPU beside it."""
    import numpy as np
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import starjoin as sj  # plan description only (plain Python); the engine library is never loaded here
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    schema = sj.StarSchema(seed=SEED, fact_rows=FACT_ROWS, cust_rows=CUST_ROWS, supp_rows=SUPP_ROWS)
    cols = oracle.gen_host(schema)
    query = sj.q33_query(schema, order=(0, 1, 2), lip=True)
    cores = oracle.cores()
    for _ in range(args.warmup):
        oracle.run(query, cols, threads=cores)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle.run(query, cols, threads=cores)
        times.append(time.perf_counter() - t0)
    ms = statistics.mean(times) * 1e3
    value = FACT_ROWS / (ms / 1e3)
    line = {"metric": METRIC, "value": value, "unit": "rows/s", "impl": "reference", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded SplitMix64)",
            "config": _config(args.bpk),
            "cpu_baseline": {"value": value, "unit": "rows/s", "cores": cores, "kind": "port",
                             "sample": f"full {FACT_ROWS // 1_000_000}M-row workload per step, {args.steps} steps"},
            "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    ref = _reference_cuda(args)
    if ref:
        line["reference_cuda"] = ref
    print(json.dumps(line), flush=True)


def _reference_cuda(args):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    try:
        import build_ref
    except Exception:
        return None
    exe = build_ref.binary(0, "lip")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref not built"}
    try:
        out = subprocess.run([exe, f"--seed={SEED}", f"--n={FACT_ROWS}", f"--c={CUST_ROWS}", f"--s={SUPP_ROWS}",
                              f"--t={max(3, min(args.steps, 10))}", f"--probe_t={max(3, min(args.steps, 20))}"],
                             capture_output=True, text=True, timeout=600, check=True).stdout
    except Exception as e:  # noqa: BLE001
        return {"unavailable": f"reference driver failed: {type(e).__name__}"}
    rec = build_ref.parse_output(out)
    tq = rec["time_query_ms"][1:] or rec["time_query_ms"]
    pr = rec["probe_ms"][1:] or rec["probe_ms"]
    return {"driver": "src/ssb-jo/q33/0-lip.cu (unmodified, sm_100a)",
            "time_query_ms": statistics.mean(tq), "rows_per_s": FACT_ROWS / (statistics.mean(tq) / 1e3),
            "probe_ms": statistics.mean(pr), "probe_rows_per_s": FACT_ROWS / (statistics.mean(pr) / 1e3),
            "probe_algorithmic_gbs": BYTES_PER_ROW * FACT_ROWS / (statistics.mean(pr) / 1e3) / 1e9,
            "groups": len(rec["groups"])}


def _bf_sweep(eng, schema, cols, args, sptr, stream, torch):
    """Probe time of the same query with each filter kind (config: direct bitmap,
    8 and 16 bits per inserted key), every join order of the reference's drivers
    for the chosen filter."""
    import starjoin as sj
    out = {}
    for bpk in (0, 8, 16):
        for order in ((0, 1, 2), (2, 1, 0), (1, 2, 0)):
            q = sj.q33_query(schema, order=order, lip=True, bf_bits_per_key=bpk, bf_hashes=2, adaptive=True)
            pq = eng.prepare(q, cols, FACT_ROWS)
            evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(30)]
            for _ in range(5):
                pq.build(sptr)
                pq.probe(sptr)
            for a, b in evs:
                pq.build(sptr)
                a.record(stream)
                pq.probe(sptr)
                b.record(stream)
            torch.cuda.synchronize()
            ms = statistics.median(a.elapsed_time(b) for a, b in evs)
            out[f"bpk{bpk}_order{''.join(map(str, order))}_probe_ms"] = ms
            pq.release()
    return out


def _config(bpk):
    return {"workload": f"3-dim LIP star join, SSB Q3.3 shape: {FACT_ROWS / 1e6:g}M fact rows (fk_cust U[1,600000], "
                        "fk_supp U[1,40000], fk_date over 2556 days, revenue U[1,1e7]); s_city/c_city IN "
                        "{231,235}, d_year<=1997; group by (s_city,c_city,d_year), SUM(revenue) uint64",
            "fact_rows": FACT_ROWS, "cust_rows": CUST_ROWS, "supp_rows": SUPP_ROWS, "date_rows": 2556,
            "join_order": "S>C>D", "bf_bits_per_key": bpk, "bf_hashes": 2,
            "l2": "no flush: fact columns (1.92 GB) exceed the 126 MB L2",
            "parallelism": "fact rows sharded per GPU (weak), dimensions replicated"}


def run_engine(args):
    import torch
    import torch.distributed as dist
    import starjoin as sj

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device(f"cuda:{local}"))
    eng = sj.Engine(local)
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream

    # one seeded fact table of world x FACT_ROWS rows, sharded by contiguous row
    # ranges (weak scaling); each rank generates only its shard, dimensions whole
    import multigpu
    global_schema = sj.StarSchema(seed=SEED, fact_rows=world * FACT_ROWS, cust_rows=CUST_ROWS, supp_rows=SUPP_ROWS)
    b, e = multigpu.row_range(global_schema.fact_rows, rank, world)
    schema = sj.StarSchema(seed=SEED, fact_rows=e - b, cust_rows=CUST_ROWS, supp_rows=SUPP_ROWS)
    cols = sj.gen_device(global_schema, [n for n in global_schema.column_specs()
                                         if not n.startswith("fk_") and n != "revenue"], device=local)
    cols.update(sj.gen_device(global_schema, ["fk_cust", "fk_supp", "fk_date", "revenue"], device=local,
                              fact_range=(b, e)))
    torch.cuda.synchronize()

    query = sj.q33_query(schema, order=(0, 1, 2), lip=True, bf_bits_per_key=args.bpk, bf_hashes=2,
                         adaptive=True)
    pq = eng.prepare(query, cols, FACT_ROWS)

    def step(ev=None):
        pq.build(sptr)
        if ev:
            ev[0].record(stream)
        pq.probe(sptr)
        if ev:
            ev[1].record(stream)

    # clock soak + warmup
    sampler = ClockSampler(local)
    sampler.start()
    t_soak = time.time()
    while time.time() - t_soak < 1.5:
        for _ in range(50):
            step()
        torch.cuda.synchronize()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    result = pq.fetch(stream=sptr)

    # the probe's own duration: CUDA events around it on every PROBE_EVERY-th timed
    # step (an event between the build and the probe holds the probe's launch until
    # the build drains, so sampling keeps that instrumentation out of ms_per_step)
    probe_every = PROBE_EVERY if args.steps >= 4 * PROBE_EVERY else 1
    probe_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                for _ in range(0, args.steps, probe_every)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t_wall0 = time.time()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for i in range(args.steps):
        step(probe_ev[i // probe_every] if i % probe_every == 0 else None)
    stop.record(stream)
    torch.cuda.synchronize()
    t_wall1 = time.time()
    if world > 1:
        dist.barrier()
    sampler.stop()
    total_ms = start.elapsed_time(stop)
    probe_ms = statistics.mean(a.elapsed_time(b) for a, b in probe_ev)
    stats = pq.stats()
    assert pq.fetch(stream=sptr) == result

    t = torch.tensor([total_ms, probe_ms], device=f"cuda:{local}", dtype=torch.float64)
    groups_ok = None
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        # the exchange step, outside the timed loop: one all-reduce of every rank's
        # group partials over the dense group space (NCCL over NVLink)
        merged = multigpu.merge_groups(result, query, dist, device=f"cuda:{local}")
        if rank == 0:
            groups_ok = merged == _oracle_sharded(global_schema, world, args.bpk)
        dist.barrier()
    total_ms, probe_ms = t.tolist()
    ms_per_step = total_ms / args.steps

    if rank == 0:
        peak, peak_kind = _peaks()
        rows = FACT_ROWS
        algorithmic = BYTES_PER_ROW * rows / (probe_ms / 1e3) / 1e9
        traffic, traffic_how = _traffic_from_profiles(args.bpk)
        achieved = traffic / (probe_ms / 1e3) / 1e9 if traffic else algorithmic
        line = {
            "metric": METRIC, "value": world * rows / (ms_per_step / 1e3), "unit": "rows/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded SplitMix64)",
            "config": _config(args.bpk),
            "probe_ms": probe_ms, "probe_ms_sampled_steps": len(probe_ev),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "algorithmic_gbs": algorithmic, "algorithmic_frac": algorithmic / peak,
                         "note": "probe kernel (sj_probe_kernel): achieved = DRAM bytes (read + write) of one launch, "
                                 f"{traffic_how}, / its mean duration (CUDA events on the launch stream); "
                                 "algorithmic_* use the full-load model of 16 B per fact row (3 FK columns + "
                                 "revenue), which this sector-skipping probe does not read (the first column "
                                 f"densely, later columns only at survivor rows); peak: {peak_kind} copy "
                                 "bandwidth" if traffic else
                                 "probe kernel: no DRAM capture for this setting, so achieved uses the 16 B/row "
                                 "algorithmic model"},
            "gpu_launches": 5 * args.steps,  # head clear, scan, insert, probe, compaction
            "groups": len(result), "groups_merged_ok": groups_ok,
            "stats": {"step_in": list(stats.step_in)[:6], "step_out": list(stats.step_out)[:6],
                      "bf_inserted": list(stats.bf_inserted)[:3], "bf_words": list(stats.bf_words)[:3],
                      "reorders": stats.reorders},
            "clocks": sampler.summary(t_soak, t_wall1),
        }
        if world == 1 and not args.no_e2e:
            line["e2e"] = _e2e(eng, schema, cols, query, args, torch)
        if world == 1 and not args.no_cpu_baseline:
            host = {k: v.cpu().numpy() for k, v in cols.items()}
            line["cpu_baseline"], want = cpu_baseline(host, query)
            line["groups_match_oracle"] = result == want
        if world == 1 and not args.no_shared:
            line["bf_sweep"] = _bf_sweep(eng, schema, cols, args, sptr, stream, torch)
    pq.release()
    if rank == 0 and world == 1 and not args.no_shared:
        import shared_bench as sb
        del cols
        torch.cuda.empty_cache()
        line["batched"] = sb.batched(eng, n_batches=args.batches)
        line["serving"] = sb.serving(eng)
    if rank == 0:
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        dist.destroy_process_group()


def _e2e(eng, schema, cols, query, args, torch):
    """Same query through the C ABI with HOST (pinned) columns: sj_run_plain stages
    every column host->device, builds, probes and reads the groups back."""
    names = sorted({query["measure"]} | {d[f] for d in query["dims"] for f in ("fk", "key", "attr", "payload")
                                         if d.get(f)})
    host = {}
    for n in names:
        h = torch.empty(cols[n].shape, dtype=torch.int32, pin_memory=True)
        h.copy_(cols[n])
        host[n] = h
    torch.cuda.synchronize()
    # explicit copies: the fact column tested first (streamed in pieces) and the
    # dimension columns; the other fact columns are read in place at survivor rows
    first = query["dims"][query["order"][0]]["fk"]
    dim_cols = sorted({d[f] for d in query["dims"] for f in ("key", "attr", "payload") if d.get(f)})
    h2d = 4 * host[first].numel() + sum(4 * host[n].numel() for n in dim_cols)
    reps = max(2, min(args.steps, 8))
    import ctypes as C
    import starjoin as sj
    plan, keep = sj.fill_plan(query, host, FACT_ROWS)
    cap = 4096
    rows = (sj.SjGroupRow * cap)()
    n = C.c_int64()
    ms = C.c_float()

    def call():  # the public C entry point, host buffers in and out
        sj.check(eng.lib.sj_run_plain(eng.h, C.byref(plan), 1, rows, cap, C.byref(n), C.byref(ms), None))

    call()  # warm
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        call()
        times.append(time.perf_counter() - t0)
    res = sj.rows_to_list(rows, n.value, query)
    t = statistics.mean(times)
    pq = eng.prepare(query, cols, FACT_ROWS)
    pq.build()
    pq.probe()
    pq.fetch()
    st = pq.stats()
    pq.release()
    # each row past the first test reads at most one 32-byte sector of each other fact column
    in_place = 32 * (len(query["dims"])) * int(st.step_out[0])
    return {"value": FACT_ROWS / t, "unit": "rows/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": 32 * len(res) + 256, "ms_per_step": t * 1e3,
            "in_place_read_bytes_upper_bound": in_place,
            "path": "sj_run_plain(host_columns=1) on pinned host columns: dimension tables copied, the first "
                    "join column streamed host->device in pieces overlapped with probe launches, the other fact "
                    "columns read in place (mapped pinned memory) at survivor rows, groups read back"}


def main():
    global FACT_ROWS
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--bpk", type=int, default=0,
                    help="filter: 0 = direct bitmap, one bit per key slot (the reference drivers' sizing, "
                         "src/ssb-jo/q33/0-lip.cu:221-223); >0 = blocked Bloom filter, bits per inserted key")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--rows", type=int, default=FACT_ROWS,
                    help="fact rows (default: the 120M-row workload; smaller values only for profiling captures)")
    ap.add_argument("--no-shared", action="store_true", help="skip the batched / serving measurements")
    ap.add_argument("--shared", choices=["batch", "serve"],
                    help="run only the batched or the serving measurement (--rows sets the fact table)")
    ap.add_argument("--batches", type=int, default=6, help="timed batches of the batched measurement")
    ap.add_argument("--rates", default="50,200,2000",
                    help="Poisson arrival rates (queries/s) of the serving measurement, comma-separated; "
                         "'none' measures saturation only")
    ap.add_argument("--sweep4", type=int, nargs="?", const=256, default=None,
                    help="run only the 4-dimension selectivity x filter sweep (optionally the first N of its "
                         "256 selectivity settings)")
    ap.add_argument("--shapes", action="store_true",
                    help="run only the SSB query shapes (Q2.1-Q4.3) at 120M rows: this engine, or with "
                         "--impl reference the reference's own CUDA drivers on the same schema")
    ap.add_argument("--queries", default="",
                    help="--shapes: comma-separated SSB query numbers (e.g. 41,43); default all ten")
    ap.add_argument("--no-autotune", action="store_true",
                    help="--shapes: skip the plan search (reference join order, LIP, automatic filter layout)")
    args = ap.parse_args()
    FACT_ROWS = args.rows
    args.warmup = max(3, args.warmup)
    if args.shapes:
        run_shapes(args)
    elif args.sweep4 is not None:
        import itertools
        import starjoin as sj
        import sweep_bench
        eng = sj.Engine(0)
        settings = list(itertools.product(sweep_bench.SELS, repeat=4))[: args.sweep4]
        print(json.dumps({"sweep4": sweep_bench.sweep4(eng, settings=settings)}), flush=True)
        eng.close()
    elif args.shared:
        run_shared(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_engine(args)


def run_shapes(args):
    """Every SSB query shape at 120M rows: this engine (shapes_bench), or the
    reference's own unmodified CUDA drivers (oracle/_ref) on the same seeded
    schema with their `time_query`; groups_sha1 digests compare the two."""
    import shapes_bench
    schema = dict(shapes_bench.SCHEMA)
    if args.rows != 120_000_000:
        schema["fact_rows"] = args.rows
    queries = tuple(int(x) for x in args.queries.split(",") if x) or shapes_bench.QUERIES
    if args.impl != "reference":
        import starjoin as sj
        eng = sj.Engine(0)
        print(json.dumps({"shapes": shapes_bench.shapes(eng, reps=max(3, min(args.steps, 20)), schema=schema,
                                                        queries=queries, autotune=not args.no_autotune)}), flush=True)
        eng.close()
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import build_ref
    sc = schema
    width = {21: 3, 22: 3, 23: 3, 31: 4, 32: 4, 33: 4, 34: 4, 41: 3, 42: 4, 43: 4}
    trials = max(3, min(args.steps, 10))
    out = {"impl": "reference", "workload": "SSB query shapes, reference CUDA drivers (unmodified, sm_100a)",
           "queries": {}}
    for q in queries:
        exe = build_ref.binary(0, "lip") if q == 33 else build_ref.shape_binary(q)
        if not os.path.exists(exe):
            out["queries"][str(q)] = {"unavailable": "oracle/_ref not built"}
            continue
        cmd = [exe, f"--seed={sc['seed']}", f"--n={sc['fact_rows']}", f"--c={sc['cust_rows']}",
               f"--s={sc['supp_rows']}", f"--t={trials}"]
        if q != 33:
            cmd.append(f"--p={sc['part_rows']}")
        try:
            text = subprocess.run(cmd, capture_output=True, text=True, timeout=600, check=True).stdout
        except Exception as e:  # noqa: BLE001
            out["queries"][str(q)] = {"unavailable": f"driver failed: {type(e).__name__}"}
            continue
        tq = build_ref.parse_output(text)["time_query_ms"]
        tq = tq[1:] or tq  # the first call also pays the caching allocator's first allocations
        groups = build_ref.parse_groups(text, width[q])
        out["queries"][str(q)] = {"driver": build_ref.SHAPE_SOURCES.get(q, "q33/0-lip.cu"),
                                  "time_query_ms": statistics.median(tq), "groups": len(groups),
                                  "groups_sha1": shapes_bench.groups_digest(groups)}
    print(json.dumps({"shapes": out}), flush=True)


def run_shared(args):
    """The shared-scan forms alone (for diagnostics and profiling captures)."""
    import starjoin as sj
    import shared_bench as sb
    eng = sj.Engine(0)
    if args.shared == "batch":
        schema = dict(sb.BATCH_SCHEMA)
        if args.rows != 120_000_000:
            schema["fact_rows"] = args.rows
        out = {"batched": sb.batched(eng, n_batches=args.batches, schema=schema)}
    else:
        schema = dict(sb.SERVE_SCHEMA)
        if args.rows != 120_000_000:
            schema["fact_rows"] = args.rows
        rates = () if args.rates == "none" else tuple(float(x) for x in args.rates.split(",") if x)
        out = {"serving": sb.serving(eng, schema=schema, rates=rates)}
    print(json.dumps(out), flush=True)
    eng.close()


if __name__ == "__main__":
    main()
