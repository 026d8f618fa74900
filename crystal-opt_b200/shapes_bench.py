"""Every SSB query shape through the plain engine, reported by `bench.py --shapes`.

Workload: the 120M-row four-dimension star schema (customer 600,000 rows,
supplier 40,000, part 1,000,000, the 2,556 SSB dates; seeded synthetic columns
with SSB's nested codes), and the ten queries as the reference's drivers run
them: Q2.1-Q2.3, Q3.1-Q3.4 and Q4.1-Q4.3 (src/ssb-jo/q*/ predicates, join
orders, groupings and sums).  Per query:

- plan: chosen by sj_autotune (filter kind including the per-dimension auto
  layout, probe geometry, every join order; each candidate verified bit for
  bit against the first) -- planning, outside the timed runs;
- query_ms: sj_run_plain's device time of that plan (filter and hash-table
  builds, probe, group compaction), the span the reference's own `time_query`
  measures;
- probe_ms: the probe kernel alone (prepared query, CUDA events);
  probe_ms_reference_plan: the same with the reference driver's join order,
  LIP setting and the direct (reference-sized) filter;
- groups / groups_sha1: the result in the order the reference's drivers print
  it, so a run of the reference's driver on the same schema compares by digest.
"""
from __future__ import annotations

import hashlib
import statistics
from typing import Any, Dict, Sequence

import starjoin as sj

SCHEMA = dict(seed=0x5EED0003, fact_rows=120_000_000, cust_rows=600_000, supp_rows=40_000, part_rows=1_000_000)
QUERIES = (21, 22, 23, 31, 32, 33, 34, 41, 42, 43)


def groups_digest(printed: Sequence[tuple]) -> str:
    """SHA-1 over the printed group lines ("a b c\\n" ...), sorted."""
    text = "".join(" ".join(str(x) for x in row) + "\n" for row in sorted(printed))
    return hashlib.sha1(text.encode()).hexdigest()


def _fact_bytes_per_row(q: Dict[str, Any]) -> int:
    return 4 * (len(q["dims"]) + 1 + (1 if q.get("measure_sub") else 0))


def shapes(eng: sj.Engine, reps: int = 10, schema: Dict[str, int] = None, queries=QUERIES,
           autotune: bool = True) -> Dict[str, Any]:
    """autotune=False runs the reference's join order with LIP, the per-dimension
    automatic filter layout and adaptive re-ranking, without the plan search
    (small profiling runs)."""
    import torch
    sc = sj.StarSchema(**(schema or SCHEMA))
    cols = sj.gen_device(sc)
    st = torch.cuda.current_stream()
    sp = st.cuda_stream
    out: Dict[str, Any] = {"workload": f"SSB query shapes, {sc.fact_rows // 1_000_000}M fact rows, customer "
                                       f"{sc.cust_rows}, supplier {sc.supp_rows}, part {sc.part_rows}, 2556 dates; "
                                       "seeded synthetic columns", "queries": {}}

    def probe_ms(q, tune):
        pq = eng.prepare(q, cols, sc.fact_rows, tune=tune)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
        for _ in range(3):
            pq.build(sp)
            pq.probe(sp)
        for a, b in evs:
            pq.build(sp)
            a.record(st)
            pq.probe(sp)
            b.record(st)
        torch.cuda.synchronize()
        pq.release()
        return statistics.median(a.elapsed_time(b) for a, b in evs)

    for qn in queries:
        ref_plan = sj.SSB_SHAPES[qn](sc)
        q0 = dict(ref_plan, lip=True)
        if autotune:
            q, tune, rep = eng.autotune(q0, cols, sc.fact_rows, reps=3, tune_filter=True, tune_order=2, verify=True,
                                        stream=sp)
            candidates = rep.candidates
        else:
            q, tune, candidates = dict(q0, bf_bits_per_key=sj.BF_AUTO, adaptive=True), {}, 0
        rows, _ = eng.run(q, cols, sc.fact_rows, tune=tune, stream=sp)
        ref_rows, _ = eng.run(ref_plan, cols, sc.fact_rows, stream=sp)
        times = []
        for _ in range(reps):
            _, ms = eng.run(q, cols, sc.fact_rows, tune=tune, stream=sp)
            times.append(ms)
        probe = probe_ms(q, tune)
        printed = sj.ssb_printed(qn, rows)
        qms = statistics.median(times)
        out["queries"][str(qn)] = {
            "query_ms": qms, "probe_ms": probe, "rows_per_s": sc.fact_rows / (qms / 1e3),
            "probe_algorithmic_gbs": _fact_bytes_per_row(q) * sc.fact_rows / (probe / 1e3) / 1e9,
            "probe_ms_reference_plan": probe_ms(ref_plan, None),
            "plan": {"order": q["order"], "lip": q["lip"], "bf_bits_per_key": q["bf_bits_per_key"],
                     "bf_hashes": q["bf_hashes"], "threads": tune.get("threads", 0),
                     "autotune_candidates": candidates},
            "same_as_reference_plan": rows == ref_rows,
            "groups": len(printed), "groups_sha1": groups_digest(printed),
        }
    del cols
    return out
