"""The N > 1 path on CPU: two gloo ranks shard the fact rows, compute their group
partials (the oracle stands in for each rank's GPU), and merge them with the
same all-gather the multi-GPU benchmark uses; the merge must equal a single run
over the whole table, bit for bit."""
import os
import socket
import time

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, queries, out):
    import sys
    for sub in ("crystal-opt_b200", "oracle", "tests"):
        sys.path.insert(0, os.path.join(ROOT, sub))
    import multigpu
    import oracle
    import starjoin as sj
    from workloads import SMALL
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sc = sj.StarSchema(seed=SMALL.seed, fact_rows=2_000_003, cust_rows=30_000, supp_rows=2_000)
        cols = sj.gen_host(sc)
        results = []
        for cities in queries:
            q = sj.q33_query(sc, cities=cities)
            b, e = multigpu.row_range(sc.fact_rows, rank, world)
            q["row_range"] = (b, e)
            part = oracle.run(q, cols, threads=2)
            results.append(multigpu.merge_groups(part, q, dist))
            results.append(multigpu.merge_gather(part, 3, dist))
        out[rank] = results
    finally:
        dist.destroy_process_group()


def test_row_ranges_tile_the_table():
    import multigpu
    for n in (0, 1, 5, 4097, 120_000_000):
        for world in (1, 2, 3, 8):
            ranges = [multigpu.row_range(n, r, world) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == n
            for (a, b), (c, d) in zip(ranges, ranges[1:]):
                assert b == c and a <= b
            assert all(a % 4 == 0 for a, _ in ranges)


@pytest.mark.parametrize("world", [2])
def test_two_gloo_ranks_merge_to_the_single_run(sj, oracle, world):
    queries = [(231, 235), tuple(range(0, 250, 3))]
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    port = _free_port()
    mp.start_processes(_rank_main, args=(world, port, queries, out), nprocs=world, join=True, start_method="spawn")
    sc = sj.StarSchema(seed=0x5EED0001, fact_rows=2_000_003, cust_rows=30_000, supp_rows=2_000)
    cols = sj.gen_host(sc)
    for i, cities in enumerate(queries):
        want = oracle.run(sj.q33_query(sc, cities=cities), cols)
        for r in range(world):
            assert out[r][2 * i] == want  # dense all-reduce
            assert out[r][2 * i + 1] == want  # all-gather fallback


def test_dense_merge_wraps_sums_modulo_2_64():
    """Sums near 2^64 from several ranks add modulo 2^64 (two's-complement
    uint64, as the engine's partials), through the 32-bit-halves layout."""
    import multigpu

    class FakeDist:  # all_reduce over three pretend ranks holding the same partials
        def all_reduce(self, t):
            t.mul_(3)

    spans = [(1992, 7)]
    rows = [(1995, 5, (1 << 64) - 7)]
    got = multigpu.merge_dense(rows, spans, FakeDist())
    assert got == [(1995, 15, (3 * ((1 << 64) - 7)) % (1 << 64))]


def _dying_rank(rank, world, port, out):
    import datetime
    import sys
    for sub in ("crystal-opt_b200",):
        sys.path.insert(0, os.path.join(ROOT, sub))
    import multigpu
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    if rank == 1:
        os._exit(3)  # the worker dies between steps, before the exchange
    t0 = time.time()
    try:
        multigpu.merge_dense([(1, 2, 1993, 4, 5)], [(0, 250), (0, 250), (1992, 7)], dist)
        out[rank] = ("merged", time.time() - t0)
    except Exception as e:  # noqa: BLE001
        out[rank] = ("error", time.time() - t0, type(e).__name__)


def test_surviving_rank_learns_of_a_dead_worker():
    """A rank that exits before the group merge: the surviving rank's collective
    ends with an error within the process-group timeout instead of hanging."""
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    port = _free_port()
    ctx = mp.start_processes(_dying_rank, args=(2, port, out), nprocs=2, join=False, start_method="spawn")
    deadline = time.time() + 60
    for p in ctx.processes:
        p.join(timeout=max(1.0, deadline - time.time()))
    alive = [p for p in ctx.processes if p.is_alive()]
    for p in alive:
        p.kill()
    assert not alive
    assert ctx.processes[1].exitcode == 3
    assert out[0][0] == "error" and out[0][1] < 30
