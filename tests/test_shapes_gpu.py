"""The reference's other query shapes through the engine: SSB Q2.1 (a key-only
supplier table, part grouped by brand), Q3.1 (nations and years) and Q4.1 (four
dimensions, SUM(revenue - supplycost)), bit-exact against the oracle for every
filter kind, LIP and naive probing and several join orders."""
import itertools

import pytest

from workloads import SHAPE_QUERIES, SHAPES_SMALL

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def shapes(sj, torch_cuda):
    dev = sj.gen_device(SHAPES_SMALL)
    host = {k: v.cpu().numpy() for k, v in dev.items()}
    return host, dev


@pytest.mark.parametrize("query", sorted(SHAPE_QUERIES))
def test_shape_matches_oracle(sj, oracle, engine, shapes, query):
    host, dev = shapes
    make = SHAPE_QUERIES[query]
    want = oracle.run(make(SHAPES_SMALL), host)
    assert want  # Q2.3 and Q3.4 select few groups at this size (7 and 2)
    n = len(make(SHAPES_SMALL)["dims"])
    orders = list(itertools.permutations(range(n)))[:: max(1, len(list(itertools.permutations(range(n)))) // 4)]
    for order in orders:
        for lip, bpk, k, adaptive in ((True, 0, 2, False), (True, 8, 3, True), (True, 16, 2, False),
                                      (False, 0, 2, False), (True, sj.BF_AUTO, 2, False),
                                      (True, sj.BF_AUTO, 3, True)):
            q = make(SHAPES_SMALL, order=order, lip=lip, bf_bits_per_key=bpk, bf_hashes=k, adaptive=adaptive)
            got, _ = engine.run(q, dev, SHAPES_SMALL.fact_rows)
            assert got == want, (query, order, lip, bpk, k, adaptive)


@pytest.mark.parametrize("query", sorted(SHAPE_QUERIES))
def test_shape_through_host_columns(sj, oracle, engine, shapes, query, torch_cuda):
    host, dev = shapes
    make = SHAPE_QUERIES[query]
    pinned = {k: torch_cuda.from_numpy(v).pin_memory() for k, v in host.items()}
    got, _ = engine.run(make(SHAPES_SMALL), pinned, SHAPES_SMALL.fact_rows, host_columns=True)
    assert got == oracle.run(make(SHAPES_SMALL), host)


def test_yearmonth_predicate_over_a_year(sj, oracle, engine, shapes):
    """Q3.4's d_yearmonthnum predicate widened from one month to all of 1997
    (the driver's month alone selects two rows at this size)."""
    host, dev = shapes
    q = sj.q34_query(SHAPES_SMALL)
    q["dims"][2]["pred"] = ("range", 199701, 199712)
    want = oracle.run(q, host)
    assert sum(r[-2] for r in want) > 10
    for order in ((0, 1, 2), (2, 1, 0)):
        for lip, bpk in ((True, 0), (True, 16), (False, 0)):
            q2 = dict(q, order=list(order), lip=lip, bf_bits_per_key=bpk)
            got, _ = engine.run(q2, dev, SHAPES_SMALL.fact_rows)
            assert got == want, (order, lip, bpk)


def test_ssb_shapes_in_one_shared_scan(sj, oracle, engine, shapes):
    """Every SSB shape through the shared scan: the revenue queries (Q2.x,
    Q3.x, with Q3.3) as one batch, the revenue - supplycost queries (Q4.x) as
    another, over the SSB-attribute dimensions.  Each query's groups equal the
    oracle's."""
    import shared_scan as ss
    host, dev = shapes
    dims = ss.ssb_dims(SHAPES_SMALL)
    groups = {None: [21, 22, 23, 31, 32, 34], "supplycost": [41, 42, 43]}
    for sub, qs in groups.items():
        plain = [SHAPE_QUERIES[q](SHAPES_SMALL) for q in qs]
        if sub is None:
            plain.append(sj.q33_query(SHAPES_SMALL))
        for p in plain:
            assert p["measure_sub"] == sub
        b = ss.Batch(engine, SHAPES_SMALL, dev, dims=dims, measure_sub=sub)
        try:
            got = b.run([ss.from_plain(p, dims) for p in plain])
        finally:
            b.close()
        for p, g in zip(plain, got):
            assert g == oracle.run(p, host)


def test_auto_filter_layout_per_dimension(sj, oracle, engine, shapes):
    """bf_bits_per_key = BF_AUTO with a 16 KB filter budget: Q2.3's part
    dimension (p_brand1 == 260, about 200 of 200,000 keys; a 32 KB direct
    bitmap over 2^18 slots) gets the blocked layout, the supplier (256 B) and
    date (8 KB) bitmaps stay direct, and the groups equal the oracle's."""
    host, dev = shapes
    q = sj.q23_query(SHAPES_SMALL, bf_bits_per_key=sj.BF_AUTO)
    pq = engine.prepare(q, dev, SHAPES_SMALL.fact_rows, tune={"bf_smem_bytes": 16384})
    try:
        pq.build()
        pq.probe()
        got = pq.fetch()
        st = pq.stats()
    finally:
        pq.release()
    assert got == oracle.run(q, host)
    assert list(st.bf_blocked)[:3] == [0, 1, 0]
    assert st.bf_words[1] * 4 < 32768 // 4  # blocked: 1,000 keys x 16 bits, far below the direct bitmap


@pytest.mark.parametrize("codes,expect_blocked", [([], 1), (list(range(25)), 0)])
def test_auto_filter_edges(sj, oracle, engine, shapes, codes, expect_blocked):
    """BF_AUTO at its edges, on a part dimension whose direct bitmap (2^18 slots,
    32 KB) is over a 16 KB budget: a predicate that accepts nothing gets a
    one-word blocked filter that rejects every row; one that accepts every row
    keeps the direct bitmap (the blocked one would not be smaller).  Groups equal
    the oracle's, under adaptive re-ranking too."""
    host, dev = shapes
    q = sj.q21_query(SHAPES_SMALL, bf_bits_per_key=sj.BF_AUTO, adaptive=True)
    q["dims"][1]["pred"] = ("in", codes) if codes else ("range", 1000, 2000)
    q["dims"][1]["attr"] = "p_category"
    pq = engine.prepare(q, dev, SHAPES_SMALL.fact_rows, tune={"bf_smem_bytes": 16384})
    try:
        pq.build()
        pq.probe()
        got = pq.fetch()
        st = pq.stats()
    finally:
        pq.release()
    want = oracle.run(q, host)
    assert got == want
    assert st.bf_blocked[1] == expect_blocked
    assert (len(want) == 0) == (not codes)
