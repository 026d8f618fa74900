"""GPU parity: the engine (through its C ABI) against the CPU oracle, bit-exact
groups, counts and uint64 sums, for every join order, naive and LIP, each filter
layout, and the edge cases the reference's kernels meet (ragged tiles, key == len,
empty inputs)."""
import ctypes as C
import os
import random

import numpy as np
import pytest

from workloads import FULL, ORDERS3, REF_DRIVER_ORDERS, SMALL, columns_of, random_query, sel_query

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small(sj, torch_cuda):
    host = sj.gen_host(SMALL)
    dev = {k: torch_cuda.from_numpy(v).cuda() for k, v in host.items()}
    return host, dev


def test_device_generator_matches_host(sj, torch_cuda):
    sc = sj.StarSchema(seed=99, fact_rows=1_000_003, cust_rows=5000, supp_rows=300, part_rows=7000)
    host = sj.gen_host(sc)
    dev = sj.gen_device(sc)
    for k in host:
        np.testing.assert_array_equal(dev[k].cpu().numpy(), host[k], k)


@pytest.mark.parametrize("lip", [True, False])
@pytest.mark.parametrize("order", ORDERS3)
def test_q33_small_every_order(sj, oracle, engine, small, order, lip):
    host, dev = small
    q = sj.q33_query(SMALL, order=order, lip=lip)
    want = oracle.run(q, host)
    assert len(want) == 24
    for bpk, k in ([(0, 1), (8, 2), (16, 3)] if lip else [(0, 1)]):
        q["bf_bits_per_key"], q["bf_hashes"] = bpk, k
        got, _ = engine.run(q, dev, SMALL.fact_rows)
        assert got == want, (order, lip, bpk)


def test_q33_reference_call_form(sj, oracle, engine, small):
    """sj_ssb_q33_run: the reference runQuery argument list (0-lip.cu:205)."""
    host, dev = small
    want = oracle.run(sj.q33_query(SMALL), host)
    for drv, order in REF_DRIVER_ORDERS.items():
        for lip in (1, 0):
            rows = (sj.SjGroupRow * 64)()
            n = C.c_int64()
            ms = C.c_float()
            o = (C.c_int32 * 3)(*order)
            p = lambda name: dev[name].data_ptr()
            sj.check(engine.lib.sj_ssb_q33_run(
                engine.h, p("fk_date"), p("fk_cust"), p("fk_supp"), p("revenue"), SMALL.fact_rows,
                p("d_key"), p("d_year"), 2556, p("s_key"), p("s_city"), SMALL.supp_rows,
                p("c_key"), p("c_city"), SMALL.cust_rows, o, lip, 0, rows, 64, C.byref(n), C.byref(ms)))
            got = sorted((r.attr[0], r.attr[1], r.attr[2], r.count, r.sum) for r in rows[:n.value])
            assert got == want, (drv, lip)
            assert ms.value > 0


def test_host_columns_form(sj, oracle, engine, small):
    host, _ = small
    q = sj.q33_query(SMALL, order=(1, 0, 2), bf_bits_per_key=16, bf_hashes=2)
    got, ms = engine.run(q, host, SMALL.fact_rows, host_columns=True)
    assert got == oracle.run(q, host)


def test_host_columns_pinned_streamed(sj, oracle, engine, small, torch_cuda):
    """Pinned host columns: the first column streams to the device in pieces,
    the others are read in place at survivor rows."""
    host, _ = small
    pinned = {k: torch_cuda.from_numpy(v).pin_memory() for k, v in host.items()}
    for order, lip, bpk in (((0, 1, 2), True, 16), ((2, 1, 0), True, 0), ((1, 0, 2), False, 0)):
        q = sj.q33_query(SMALL, order=order, lip=lip, bf_bits_per_key=bpk)
        got, ms = engine.run(q, pinned, SMALL.fact_rows, host_columns=True)
        assert got == oracle.run(q, host), (order, lip, bpk)
        assert ms > 0
    q = sj.q33_query(SMALL, row_range=(3, 5_999_998), cities=tuple(range(0, 250, 7)), bf_bits_per_key=8)
    got, _ = engine.run(q, pinned, SMALL.fact_rows, host_columns=True)
    assert got == oracle.run(q, host)


@pytest.mark.parametrize("seed", range(40))
def test_random_queries(sj, oracle, engine, torch_cuda, seed):
    rng = random.Random(seed)
    sc = sj.StarSchema(seed=500 + seed % 4, fact_rows=rng.choice([1, 3, 4097, 300_001, 2_000_000]),
                       cust_rows=rng.choice([1, 33, 30_000]), supp_rows=rng.choice([1, 2000]),
                       part_rows=rng.choice([0, 10_000]))
    host = sj.gen_host(sc)
    dev = {k: torch_cuda.from_numpy(v).cuda() for k, v in host.items()}
    for _ in range(3):
        q = random_query(rng, sc)
        got, _ = engine.run(q, dev, sc.fact_rows)
        assert got == oracle.run(q, host), q


@pytest.mark.parametrize("begin,end", [(0, 0), (5, 5), (0, 1), (1, 2), (3, 4), (1, 4096), (2, 4099),
                                       (4095, 8193), (6_000_000 - 5, 6_000_000), (3, 6_000_000),
                                       (1_234_567, 4_567_891)])
def test_row_ranges_and_ragged_tails(sj, oracle, engine, small, begin, end):
    host, dev = small
    q = sj.q33_query(SMALL, cities=tuple(range(0, 250, 5)), row_range=(begin, end), bf_bits_per_key=8)
    got, _ = engine.run(q, dev, SMALL.fact_rows)
    assert got == oracle.run(q, host)


@pytest.mark.parametrize("tune", [dict(threads=256), dict(threads=768), dict(stages=2), dict(stages=12, chunk_rows=4096),
                                  dict(chunk_rows=4096), dict(chunk_rows=16384, stages=3),
                                  dict(bf_smem_bytes=0), dict(ctas_per_sm=2, stages=2, chunk_rows=4096),
                                  dict(record_events=1)])
def test_launch_geometry_does_not_change_results(sj, oracle, engine, small, tune):
    host, dev = small
    want = oracle.run(sj.q33_query(SMALL), host)
    for lip, bpk in ((True, 16), (True, 0), (False, 0)):
        q = sj.q33_query(SMALL, order=(2, 1, 0), lip=lip, bf_bits_per_key=bpk)
        got, _ = engine.run(q, dev, SMALL.fact_rows, tune=tune)
        assert got == want, (tune, lip, bpk)


def test_no_qualifying_rows_and_all_rows(sj, oracle, engine, small):
    host, dev = small
    q = sj.q33_query(SMALL, cities=(250, 251))  # no city matches
    assert engine.run(q, dev, SMALL.fact_rows)[0] == [] == oracle.run(q, host)
    q = sj.q33_query(SMALL, cities=tuple(range(250)))
    got, _ = engine.run(q, dev, SMALL.fact_rows)
    assert got == oracle.run(q, host) and len(got) > 370_000  # 375,000 possible groups


def test_key_equal_to_len_and_out_of_range_fks(sj, oracle, engine, torch_cuda):
    """FK values beyond the table alias slot (fk - min) % len, exactly as
    BlockProbeAndPHT_2 does (crystal/join.cuh:27,123); key == len is slot 0."""
    sc = sj.StarSchema(seed=11, fact_rows=100_000, cust_rows=97, supp_rows=13)
    host = sj.gen_host(sc)
    rng = np.random.default_rng(0)
    host["fk_cust"] = rng.integers(-300, 5000, size=sc.fact_rows).astype(np.int32)
    host["fk_supp"] = rng.integers(0, 60, size=sc.fact_rows).astype(np.int32)
    dev = {k: torch_cuda.from_numpy(v).cuda() for k, v in host.items()}
    for lip, bpk in ((True, 0), (True, 8), (False, 0)):
        q = sj.q33_query(sc, cities=tuple(range(0, 250, 2)), lip=lip, bf_bits_per_key=bpk)
        got, _ = engine.run(q, dev, sc.fact_rows)
        assert got == oracle.run(q, host), (lip, bpk)


def test_prepared_query_rebuild_and_reprobe(sj, oracle, engine, small):
    host, dev = small
    q = sj.q33_query(SMALL, order=(2, 0, 1), bf_bits_per_key=8)
    want = oracle.run(q, host)
    pq = engine.prepare(q, dev, SMALL.fact_rows)
    for _ in range(3):
        pq.build()
        pq.probe()
        assert pq.fetch() == want
    st = pq.stats()
    assert st.rows_scanned == SMALL.fact_rows
    assert st.groups == 24
    assert st.step_in[0] == SMALL.fact_rows
    assert st.error_flags == 0
    for _ in range(3):  # probes over one build: the same groups and per-probe counters each time
        pq.probe()
        assert pq.fetch() == want
        st = pq.stats()
        assert st.rows_scanned == SMALL.fact_rows and st.groups == 24 and st.step_in[0] == SMALL.fact_rows
    pq.release()


def test_rebuilds_follow_changed_dimension_rows(sj, oracle, engine, small, torch_cuda):
    """Prepared re-builds over dimension columns changed in place: every build
    clears the tables and filters the previous one set, so each round's groups
    match the oracle on that round's columns."""
    host, dev = small
    cols = {k: v.clone() for k, v in dev.items()}
    h = {k: v.copy() for k, v in host.items()}
    q = sj.q33_query(SMALL, order=(0, 1, 2), adaptive=False)
    pq = engine.prepare(q, cols, SMALL.fact_rows)
    rng = np.random.default_rng(11)
    try:
        for r in range(6):
            if r:  # new city attributes: a different set of customers and suppliers qualifies
                for col in ("c_city", "s_city"):
                    h[col] = rng.integers(0, 250, size=h[col].shape[0]).astype(np.int32)
                    cols[col].copy_(torch_cuda.from_numpy(h[col]))
            pq.build()
            pq.probe()
            assert pq.fetch() == oracle.run(q, h), r
    finally:
        pq.release()


def test_invalid_arguments_are_reported(sj, engine, small):
    host, dev = small
    q = sj.q33_query(SMALL)
    q["order"] = [0, 0, 1]
    with pytest.raises(sj.StarJoinError) as e:
        engine.run(q, dev, SMALL.fact_rows)
    assert e.value.status == sj.SJ_ERR_INVALID_ARGUMENT
    q = sj.q33_query(SMALL)
    q["dims"][0]["payload_range"] = (0, 100)  # s_city up to 249 falls outside
    with pytest.raises(sj.StarJoinError) as e:
        engine.run(q, dev, SMALL.fact_rows)
    assert e.value.status == sj.SJ_ERR_INVALID_ARGUMENT
    q = sj.q33_query(SMALL)
    dev2 = dict(dev)
    dev2["fk_supp"] = dev["fk_supp"][1:]  # 4-byte offset: not 16-byte aligned
    with pytest.raises(sj.StarJoinError) as e:
        engine.run(q, dev2, SMALL.fact_rows - 1)
    assert e.value.status == sj.SJ_ERR_INVALID_ARGUMENT


@pytest.mark.parametrize("bpk", [4, 8, 16])
@pytest.mark.parametrize("k", [1, 2, 3, 4])
def test_bloom_no_false_negatives(sj, engine, torch_cuda, bpk, k):
    """Every inserted key passes (the reference's bloom.cu expectation 'FN should be 0',
    src/ops/bloom.cu:241); the false-positive rate stays near the blocked-filter bound."""
    torch = torch_cuda
    n = 200_000
    keys = torch.arange(1, n + 1, dtype=torch.int32, device="cuda")
    flags = (torch.arange(n, device="cuda") % 3 == 0).to(torch.int32)
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    sj.check(engine.lib.sj_bloom_test(keys.data_ptr(), flags.data_ptr(), n, keys.data_ptr(), out.data_ptr(), n,
                                      bpk, k, 0, 0, None))
    f = flags.bool()
    assert bool(out[f].all()), "false negative"
    fpr = out[~f].float().mean().item()
    # k = 1 sets one bit in the low 32-bit half: a 32-bit block
    bound = ({4: 0.5, 8: 0.3, 16: 0.15} if k == 1 else {4: 0.2, 8: 0.06, 16: 0.02})[bpk]
    assert fpr < bound, fpr


def test_direct_bitmap_filter_is_exact(sj, engine, torch_cuda):
    torch = torch_cuda
    n = 1 << 16
    keys = torch.arange(n, dtype=torch.int32, device="cuda") + 19920101
    flags = (torch.arange(n, device="cuda") % 7 == 2).to(torch.int32)
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    sj.check(engine.lib.sj_bloom_test(keys.data_ptr(), flags.data_ptr(), n, keys.data_ptr(), out.data_ptr(), n,
                                      0, 1, 19920101, n // 32, None))
    assert torch.equal(out, flags)


def test_four_dim_selectivity_grid(sj, oracle, engine, torch_cuda):
    sc = sj.StarSchema(seed=77, fact_rows=3_000_000, cust_rows=60_000, supp_rows=4000, part_rows=100_000)
    host = sj.gen_host(sc)
    dev = {k: torch_cuda.from_numpy(v).cuda() for k, v in host.items()}
    rng = random.Random(5)
    for _ in range(12):
        sels = [rng.choice([1, 10, 100, 500]) for _ in range(4)]
        q = sel_query(sc, sels, seed=rng.randint(0, 1 << 30), order=rng.sample(range(4), 4),
                      bpk=rng.choice([4, 8, 16]), k=rng.randint(1, 4), adaptive=rng.random() < 0.5)
        got, _ = engine.run(q, dev, sc.fact_rows)
        assert got == oracle.run(q, host), sels


@pytest.fixture(scope="module")
def full(sj, torch_cuda):
    dev = sj.gen_device(FULL)
    host = {k: v.cpu().numpy() for k, v in dev.items()}
    return host, dev


@pytest.fixture(scope="module")
def full_want(sj, oracle, full):
    host, _ = full
    want = oracle.run(sj.q33_query(FULL), host)
    assert len(want) == 24
    return want


@pytest.mark.parametrize("order", ORDERS3)
def test_q33_full_size(sj, engine, full, full_want, order):
    """The bench workload (120M fact rows) at every join order: LIP with the
    direct bitmap and with 8 / 16 bits per key, with and without adaptive LIP,
    and naive -- bit-exact against the oracle."""
    _, dev = full
    for lip, bpk, adaptive in ((True, 0, False), (True, 0, True), (True, 8, False), (True, 16, True),
                               (False, 0, False)):
        q = sj.q33_query(FULL, order=order, lip=lip, bf_bits_per_key=bpk, adaptive=adaptive)
        got, _ = engine.run(q, dev, FULL.fact_rows)
        assert got == full_want, (order, lip, bpk, adaptive)


def _probe_ms(engine, q, cols, rows, reps=5):
    pq = engine.prepare(q, cols, rows, tune={"record_events": 1})  # build_ms / probe_ms in the stats
    times = []
    for _ in range(reps):
        pq.build()
        pq.probe()
        pq.fetch()
        times.append(pq.stats().probe_ms)
    assert min(times) > 0
    st = pq.stats()
    res = pq.fetch()
    pq.release()
    return sorted(times)[reps // 2], st, res


def test_adaptive_lip_starts_from_the_cheapest_order(sj, engine, full):
    """With adaptive LIP the starting order comes from each dimension's
    qualifying fraction: the reference's worst driver order (D first, 86% pass)
    runs about as fast as the best one."""
    host, dev = full
    for bpk in (0, 16):
        good, _, want = _probe_ms(engine, sj.q33_query(FULL, order=(0, 1, 2), bf_bits_per_key=bpk, adaptive=True),
                                  dev, FULL.fact_rows)
        bad, _, got = _probe_ms(engine, sj.q33_query(FULL, order=(2, 1, 0), bf_bits_per_key=bpk, adaptive=True),
                                dev, FULL.fact_rows)
        assert got == want
        assert bad < 1.3 * good + 0.02, (bpk, good, bad)


def test_adaptive_lip_reorders_when_the_estimate_misleads(sj, engine, full, torch_cuda):
    """Supplier FKs skewed onto qualifying suppliers: the supplier filter looks
    most selective (0.8% of suppliers qualify) but passes most fact rows, so the
    observed pass rates must re-rank the order during the scan."""
    torch = torch_cuda
    host, dev = full
    n = FULL.fact_rows
    keys = dev["s_key"][torch.isin(dev["s_city"], torch.tensor([231, 235], device="cuda", dtype=torch.int32))]
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    pick = keys[torch.randint(0, keys.numel(), (n,), device="cuda", generator=g)]
    skew = torch.where(torch.rand(n, device="cuda", generator=g) < 0.95, pick, dev["fk_supp"])
    cols = dict(dev)
    cols["fk_supp"] = skew
    q = sj.q33_query(FULL, order=(0, 1, 2), bf_bits_per_key=16, adaptive=True)
    _, st, got = _probe_ms(engine, q, cols, n, reps=2)
    assert st.reorders > 0
    fixed = sj.q33_query(FULL, order=(1, 0, 2), bf_bits_per_key=16, adaptive=False)
    _, _, want = _probe_ms(engine, fixed, cols, n, reps=1)
    assert got == want


def test_l2_set_aside_reserved_and_given_back(torch_cuda):
    """The engine reserves a persisting-L2 set-aside for the probes'
    access-policy windows while it lives and puts the previous limit back when
    the last engine of the process goes (checked in a fresh process, through
    the CUDA runtime's own cudaDeviceGetLimit)."""
    import subprocess
    import sys
    code = r'''
import ctypes, os, sys
sys.path.insert(0, os.path.join(sys.argv[1], "crystal-opt_b200"))
import nvidia.cuda_runtime
import starjoin as sj
rt = ctypes.CDLL(os.path.join(os.path.dirname(nvidia.cuda_runtime.__file__), "lib", "libcudart.so.12"))
lim = ctypes.c_size_t()
def get():
    assert rt.cudaDeviceGetLimit(ctypes.byref(lim), 6) == 0  # cudaLimitPersistingL2CacheSize
    return lim.value
rt.cudaFree(None)
before = get()
a = sj.Engine(0)
during = get()
b = sj.Engine(0)
a.close()
still = get()
b.close()
after = get()
print(before, during, still, after)
'''
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", code, root], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    before, during, still, after = map(int, out.stdout.split())
    assert during >= before and during > 0
    assert still == during  # a second engine keeps the set-aside
    assert after == before
