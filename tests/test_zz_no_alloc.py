"""The no-allocation Q3.3 entry point (sj_ssb_q33_run_noalloc).

It exists for callers that cannot allocate device memory while a query runs: a
fixed device-memory budget handed out up front, an allocator-free latency path,
or a runtime that owns every allocation.  All its scratch lives in one
fixed-size device array inside the library.  These tests call it through the C
ABI, twice in a row (the array keeps the previous call's contents, so the second
call checks that everything that must start at zero is cleared), and compare
each answer with the allocating entry point sj_ssb_q33_run: the results are
exact integers, so they must be identical.  The file is named to be collected
last, so that a stop-at-first-failure run has already run every other test.
"""
import ctypes as C

import pytest

from workloads import SMALL

pytestmark = pytest.mark.gpu


def _cols(sj, torch):
    host = sj.gen_host(SMALL)
    return {k: torch.from_numpy(v).cuda() for k, v in host.items()}


def _args(dev, order, lip, bpk):
    p = lambda name: dev[name].data_ptr()  # noqa: E731
    return (p("fk_date"), p("fk_cust"), p("fk_supp"), p("revenue"), SMALL.fact_rows,
            p("d_key"), p("d_year"), 2556, p("s_key"), p("s_city"), SMALL.supp_rows,
            p("c_key"), p("c_city"), SMALL.cust_rows, (C.c_int32 * 3)(*order), lip, bpk)


def _rows(rows, n):
    return [(r.attr[0], r.attr[1], r.attr[2], r.count, r.sum) for r in rows[:n]]


@pytest.mark.parametrize("order,lip,bpk", [((0, 1, 2), 1, 0), ((2, 1, 0), 1, 16), ((1, 0, 2), 0, 0)])
def test_noalloc_matches_allocating_entry_point_twice(sj, engine, torch_cuda, order, lip, bpk):
    dev = _cols(sj, torch_cuda)
    lib = engine.lib
    ref_rows = (sj.SjGroupRow * 64)()
    n_ref = C.c_int64()
    ms = C.c_float()
    sj.check(lib.sj_ssb_q33_run(engine.h, *_args(dev, order, lip, bpk), ref_rows, 64, C.byref(n_ref), C.byref(ms)))
    want = _rows(ref_rows, n_ref.value)
    assert len(want) == 24
    for _ in range(2):  # the second call reuses the scratch the first one left behind
        rows = (sj.SjGroupRow * 64)()
        n = C.c_int64()
        st = lib.sj_ssb_q33_run_noalloc(0, *_args(dev, order, lip, bpk), rows, 64, C.byref(n), None)
        assert st == sj.SJ_OK, lib.sj_noalloc_last_error()
        assert _rows(rows, n.value) == want


def test_noalloc_rejects_queries_beyond_its_scratch(sj, torch_cuda):
    """A customer table far larger than the fixed scratch allows is refused
    before any device work, with a message that names the limit."""
    lib = sj.load()
    dev = _cols(sj, torch_cuda)
    p = lambda name: dev[name].data_ptr()  # noqa: E731
    rows = (sj.SjGroupRow * 64)()
    n = C.c_int64()
    st = lib.sj_ssb_q33_run_noalloc(0, p("fk_date"), p("fk_cust"), p("fk_supp"), p("revenue"), SMALL.fact_rows,
                                    p("d_key"), p("d_year"), 2556, p("s_key"), p("s_city"), SMALL.supp_rows,
                                    p("c_key"), p("c_city"), 50_000_000, (C.c_int32 * 3)(0, 1, 2), 1, 0,
                                    rows, 64, C.byref(n), None)
    assert st == sj.SJ_ERR_CAPACITY
    assert b"scratch" in lib.sj_noalloc_last_error()
