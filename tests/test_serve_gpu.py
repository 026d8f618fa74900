"""GPU parity of the serving loop (sjs_*): queries admitted while others run
share the circular scan; each result equals the oracle, equals the same query
served alone, and equals the plain one-at-a-time loop."""
import random
import threading
import time

import pytest

import shared_scan as ss

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def star(sj, torch_cuda):
    sc = sj.StarSchema(seed=0x5EED0006, fact_rows=3_000_017, cust_rows=30_000, supp_rows=2000, part_rows=100_000)
    dev = sj.gen_device(sc)
    host = {k: v.cpu().numpy() for k, v in dev.items()}
    return sc, host, dev


def _serve(engine, sc, dev, queries, gaps=None, **kw):
    srv = ss.Server(engine, sc, dev, **kw)
    try:
        tickets = []
        for i, q in enumerate(queries):
            if gaps:
                time.sleep(gaps[i])
            tickets.append(srv.submit(q))
        out = [srv.wait(t, timeout_s=120.0) for t in tickets]
        return [r for r, _ in out], [i for _, i in out], srv.stats()
    finally:
        srv.close()


def test_burst_matches_oracle_and_shares_the_scan(oracle, engine, star):
    sc, host, dev = star
    rng = random.Random(10)
    qs = [ss.random_query(rng, sc, len_range=(100_000, None)) for _ in range(80)]
    got, info, st = _serve(engine, sc, dev, qs, step_rows=1 << 19)
    for i, q in enumerate(qs):
        assert got[i] == oracle.run(ss.to_plain(sc, q), host), i
        assert info[i].status == 0 and info[i].finish_s >= info[i].admit_s >= info[i].submit_s
    assert st.finished == 80 and st.peak_active > 1
    # shared: far fewer rows read than the queries' ranges add up to
    assert st.rows_scanned < sum(q["row_range"][1] - q["row_range"][0] for q in qs)


def test_alone_and_in_the_mix_are_equal(engine, star):
    sc, _, dev = star
    rng = random.Random(11)
    qs = [ss.random_query(rng, sc, len_range=(200_000, None)) for _ in range(30)]
    probe = qs[7]
    alone, _, _ = _serve(engine, sc, dev, [probe], step_rows=1 << 18)
    # arrivals spread over the scan so queries attach at different positions
    mix, info, st = _serve(engine, sc, dev, qs, gaps=[rng.uniform(0, 0.004) for _ in qs], step_rows=1 << 18)
    assert mix[7] == alone[0]
    assert st.steps > 1


def test_plain_loop_gives_the_same_results(engine, star):
    sc, _, dev = star
    rng = random.Random(12)
    qs = [ss.random_query(rng, sc, len_range=(100_000, None)) for _ in range(16)]
    shared, _, _ = _serve(engine, sc, dev, qs)
    plain, _, st = _serve(engine, sc, dev, qs, plain=True)
    assert shared == plain
    assert st.finished == 16


def test_small_memory_admits_in_turn(oracle, engine, star):
    """A filter cache that holds only a few queries' filters: the rest wait and
    are admitted as earlier queries leave (admission by device memory)."""
    sc, host, dev = star
    rng = random.Random(13)
    qs = [ss.random_query(rng, sc, len_range=(100_000, None)) for _ in range(20)]
    got, _, st = _serve(engine, sc, dev, qs, filter_cache_bytes=64 << 10, cache_filters=False,
                        step_rows=1 << 20)
    for i, q in enumerate(qs):
        assert got[i] == oracle.run(ss.to_plain(sc, q), host), i
    assert st.peak_active < 20


def test_refusals(sj, engine, star):
    sc, _, dev = star
    srv = ss.Server(engine, sc, dev, group_entries=1000)
    try:
        big = {"preds": [{"dim": 0, "kind": "all", "group_attr": 0}, {"dim": 1, "kind": "all", "group_attr": 0}],
               "row_range": (0, 10)}
        with pytest.raises(sj.StarJoinError) as e:
            srv.submit(big)
        assert e.value.status == sj.SJ_ERR_REJECTED
        assert srv.stats().rejected == 1
        ok = {"preds": [{"dim": 3, "kind": "all", "group_attr": 0}], "row_range": (0, 5000)}
        rows, info = srv.wait(srv.submit(ok), timeout_s=60.0)
        assert sum(r[-2] for r in rows) == 5000
    finally:
        srv.close()


def test_concurrent_submitters(oracle, engine, star):
    sc, host, dev = star
    srv = ss.Server(engine, sc, dev, step_rows=1 << 19)
    results = {}
    try:
        def client(seed):
            rng = random.Random(seed)
            for i in range(6):
                q = ss.random_query(rng, sc, len_range=(100_000, None))
                rows, _ = srv.wait(srv.submit(q), timeout_s=120.0)
                results[(seed, i)] = (q, rows)
        th = [threading.Thread(target=client, args=(s,)) for s in range(4)]
        for t in th:
            t.start()
        for t in th:
            t.join()
    finally:
        srv.close()
    assert len(results) == 24
    for q, rows in results.values():
        assert rows == oracle.run(ss.to_plain(sc, q), host)


def test_cancel_queued_and_running(sj, oracle, engine, star):
    """Cancelled tickets complete with SJ_ERR_CANCELLED (or with their full,
    correct result if they finished first); every other query is unaffected."""
    sc, host, dev = star
    rng = random.Random(14)
    qs = [ss.random_query(rng, sc, len_range=(1_000_000, None)) for _ in range(40)]
    srv = ss.Server(engine, sc, dev, step_rows=1 << 18, max_active=8)
    try:
        tickets = [srv.submit(q) for q in qs]
        for t in tickets[::3]:
            srv.cancel(t)
        cancelled = 0
        for i, (q, t) in enumerate(zip(qs, tickets)):
            try:
                rows, _ = srv.wait(t, timeout_s=120.0)
            except sj.StarJoinError as e:
                assert i % 3 == 0 and e.status == sj.SJ_ERR_CANCELLED, (i, e)
                cancelled += 1
                continue
            assert rows == oracle.run(ss.to_plain(sc, q), host), i
        assert cancelled >= 7  # with 8 slots most of the 14 cancelled tickets were still queued
    finally:
        srv.close()


def test_injected_allocation_failures(sj, oracle, engine, star):
    """Fault injection on the host: every 3rd admission fails as its device
    allocation would; those tickets report SJ_ERR_OUT_OF_MEMORY, the server keeps
    serving, and every other result stays exact."""
    sc, host, dev = star
    rng = random.Random(15)
    qs = [ss.random_query(rng, sc, len_range=(100_000, None)) for _ in range(24)]
    srv = ss.Server(engine, sc, dev, fault_admit_every=3, step_rows=1 << 19)
    try:
        tickets = [srv.submit(q) for q in qs]
        failed = 0
        for q, t in zip(qs, tickets):
            try:
                rows, _ = srv.wait(t, timeout_s=120.0)
            except sj.StarJoinError as e:
                assert e.status == sj.SJ_ERR_OUT_OF_MEMORY
                failed += 1
                continue
            assert rows == oracle.run(ss.to_plain(sc, q), host)
        assert failed == 8
    finally:
        srv.close()


def test_destroy_releases_blocked_waiters(sj, engine, star):
    sc, _, dev = star
    rng = random.Random(16)
    qs = [ss.random_query(rng, sc, len_range=(2_000_000, None)) for _ in range(64)]
    srv = ss.Server(engine, sc, dev, step_rows=1 << 17, max_active=2)
    tickets = [srv.submit(q) for q in qs]
    outcome = {}

    def waiter():
        try:
            srv.wait(tickets[-1])  # no timeout: only the shutdown can end this wait early
            outcome["status"] = 0
        except sj.StarJoinError as e:
            outcome["status"] = e.status

    th = threading.Thread(target=waiter)
    th.start()
    time.sleep(0.05)
    srv.close()
    th.join(timeout=30)
    assert not th.is_alive()
    assert outcome["status"] in (0, sj.SJ_ERR_CANCELLED)


def test_solo_plain_answers_lone_queries_exactly(oracle, engine, star):
    """solo_plain: a query that finds the scan idle and nothing else waiting,
    with a row range of at most one scan step, runs through the plain engine;
    a longer lone query and a burst share the scan.  Every answer equals the
    oracle's."""
    sc, host, dev = star
    rng = random.Random(16)
    step = 1 << 19
    lone = [ss.random_query(rng, sc, len_range=(100_000, step)) for _ in range(6)]
    srv = ss.Server(engine, sc, dev, solo_plain=True, step_rows=step)
    try:
        for q in lone:  # one at a time: each finds the server idle
            rows, info = srv.wait(srv.submit(q), timeout_s=120.0)
            assert info.status == 0
            assert rows == oracle.run(ss.to_plain(sc, q), host)
        st = srv.stats()
        assert st.solo == 6 and st.steps == 6 and st.finished == 6
        long_q = ss.random_query(rng, sc, len_range=(4 * step, None))
        rows, _ = srv.wait(srv.submit(long_q), timeout_s=120.0)
        assert rows == oracle.run(ss.to_plain(sc, long_q), host)
        st = srv.stats()
        assert st.solo == 6 and st.steps > 7  # the shared scan, in steps
        burst = [ss.random_query(rng, sc, len_range=(100_000, None)) for _ in range(40)]
        tickets = [srv.submit(q) for q in burst]
        for q, t in zip(burst, tickets):
            rows, info = srv.wait(t, timeout_s=120.0)
            assert rows == oracle.run(ss.to_plain(sc, q), host)
        st = srv.stats()
        assert st.finished == 47 and st.solo < 47 and st.peak_active > 1
    finally:
        srv.close()


def test_solo_plain_cancelled_ticket(sj, engine, star):
    """A lone query cancelled while the plain engine runs it completes as
    cancelled, with no rows."""
    sc, _, dev = star
    srv = ss.Server(engine, sc, dev, solo_plain=True)
    try:
        q = {"preds": [{"dim": 0, "kind": "all", "group_attr": 0}, {"dim": 3, "kind": "all", "group_attr": 0}],
             "row_range": (0, 1_000_000)}  # within one default step (fact_rows / 8, at least 2^20)
        t = srv.submit(q)
        srv.cancel(t)
        try:
            rows, info = srv.wait(t, timeout_s=60.0)
            assert info.status == 0  # finished before the cancel reached it
        except sj.StarJoinError as e:
            assert e.status == sj.SJ_ERR_CANCELLED
        ok = {"preds": [{"dim": 3, "kind": "all", "group_attr": 0}], "row_range": (0, 5000)}
        rows, _ = srv.wait(srv.submit(ok), timeout_s=60.0)
        assert sum(r[-2] for r in rows) == 5000
    finally:
        srv.close()


def test_cached_filter_regrouped_while_serving(oracle, engine, star):
    """Serving: a query that reuses a cached filter grouped by an attribute the
    filter has no statistics for gets them completed at admission; every answer
    equals the oracle's."""
    sc, host, dev = star
    srv = ss.Server(engine, sc, dev, cache_filters=True, step_rows=1 << 20)
    try:
        def q(g0, g1):
            return {"preds": [{"dim": 0, "kind": "range", "attr": 1, "lo": 50, "hi": 650, "group_attr": g0},
                              {"dim": 1, "kind": "range", "attr": 1, "lo": 100, "hi": 900, "group_attr": g1}],
                    "row_range": (0, sc.fact_rows)}
        # each query's worst group span (full attribute ranges) within the server's 1M result rows
        for g0, g1 in ((0, -1), (1, 0), (2, 0), (-1, 2)):
            qq = q(g0, g1)
            rows, info = srv.wait(srv.submit(qq), timeout_s=120.0, cap=1 << 20)
            assert info.status == 0
            assert rows == oracle.run(ss.to_plain(sc, qq), host)
        st = srv.stats()
        assert st.filters_built == 2 and st.filters_cached >= 6
    finally:
        srv.close()
