"""GPU parity of the batch form (sjb_batch_run): many queries in one shared
scan, every query's groups bit-exact against the oracle and against the plain
engine, alone and in the mix, with and without the CUDA graph and the filter
cache."""
import random

import pytest

import shared_scan as ss

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def star(sj, torch_cuda):
    sc = sj.StarSchema(seed=0x5EED0005, fact_rows=4_000_003, cust_rows=30_000, supp_rows=2000, part_rows=100_000)
    dev = sj.gen_device(sc)
    host = {k: v.cpu().numpy() for k, v in dev.items()}
    return sc, host, dev


@pytest.fixture(scope="module")
def batch(sj, engine, star):
    sc, host, dev = star
    b = ss.Batch(engine, sc, dev, use_graph=True)
    yield b
    b.close()


def _oracle(oracle, sc, host, queries):
    return [oracle.run(ss.to_plain(sc, q), host) for q in queries]


def test_q33_in_shared_form(sj, oracle, batch, star):
    sc, host, dev = star
    q = ss.q33_as_shared(sc)
    got = batch.run([q])[0]
    want = oracle.run(ss.to_plain(sc, q), host)
    assert got == want and len(want) == 24


def test_64_random_queries_match_oracle(oracle, batch, star):
    sc, host, _ = star
    rng = random.Random(1)
    qs = [ss.random_query(rng, sc, len_range=(100_000, None)) for _ in range(64)]
    got = batch.run(qs)
    want = _oracle(oracle, sc, host, qs)
    for i, (g, w) in enumerate(zip(got, want)):
        assert g == w, i
    st = batch.stats()
    assert st.error_flags == 0 and st.filters_built > 0
    assert 0 < st.rows_scanned <= sc.fact_rows


def test_each_query_alone_equals_its_result_in_the_mix(batch, star):
    sc, _, _ = star
    rng = random.Random(2)
    qs = [ss.random_query(rng, sc, len_range=(50_000, None)) for _ in range(40)]
    mix = batch.run(qs)
    for i in range(0, 40, 5):
        assert batch.run([qs[i]])[0] == mix[i], i


def test_plain_engine_agrees(engine, batch, star):
    sc, _, dev = star
    rng = random.Random(3)
    qs = [ss.random_query(rng, sc, len_range=(100_000, None)) for _ in range(12)]
    got = batch.run(qs)
    for q, g in zip(qs, got):
        want, _ = engine.run(ss.to_plain(sc, q), dev, sc.fact_rows)
        assert g == want


@pytest.mark.parametrize("opts", [dict(use_graph=False), dict(cache_filters=True), dict(threads=256),
                                  dict(smem_group_entries=64), dict(threads=1024)])
def test_options_do_not_change_results(engine, batch, star, opts):
    sc, _, dev = star
    rng = random.Random(4)
    qs = [ss.random_query(rng, sc, len_range=(10_000, None)) for _ in range(33)]
    want = batch.run(qs)
    b = ss.Batch(engine, sc, dev, **opts)
    try:
        for _ in range(2):  # the second run serves cached filters when the cache is on
            assert b.run(qs) == want
        if opts.get("cache_filters"):
            assert b.stats().filters_built == 0 and b.stats().filters_cached > 0
    finally:
        b.close()


def test_edge_queries(sj, oracle, batch, star):
    sc, host, _ = star
    n = sc.fact_rows
    qs = [
        # empty row range
        {"preds": [{"dim": 0, "kind": "range", "attr": 1, "lo": 0, "hi": 999, "group_attr": 0}],
         "row_range": (100, 100)},
        # a predicate no row passes
        {"preds": [{"dim": 1, "kind": "range", "attr": 1, "lo": 5000, "hi": 6000, "group_attr": 0},
                   {"dim": 0, "kind": "all", "group_attr": -1}], "row_range": (0, n)},
        # no grouping: one group
        {"preds": [{"dim": 3, "kind": "in", "attr": 0, "codes": [1993, 1995], "group_attr": -1}],
         "row_range": (7, n - 5)},
        # ragged ends, one row, the last row
        {"preds": [{"dim": 2, "kind": "all", "group_attr": 0}], "row_range": (n - 1, n)},
        {"preds": [{"dim": 2, "kind": "all", "group_attr": 0}], "row_range": (3, 4)},
        # IN over the key attribute, grouped by every dimension
        {"preds": [{"dim": 0, "kind": "in", "attr": 2, "codes": list(range(1, 2000, 3)), "group_attr": 0},
                   {"dim": 3, "kind": "range", "attr": 0, "lo": 1992, "hi": 1997, "group_attr": 0},
                   {"dim": 2, "kind": "range", "attr": 1, "lo": 0, "hi": 99, "group_attr": 0}],
         "row_range": (129, n - 129)},
        # date keys at both ends of the calendar
        {"preds": [{"dim": 3, "kind": "range", "attr": 2, "lo": sj.DATE_MIN, "hi": sj.DATE_MIN, "group_attr": -1},
                   {"dim": 1, "kind": "all", "group_attr": -1}], "row_range": (0, n)},
        {"preds": [{"dim": 3, "kind": "range", "attr": 2, "lo": sj.DATE_MAX, "hi": sj.DATE_MAX, "group_attr": 0}],
         "row_range": (0, n)},
    ]
    got = batch.run(qs)
    want = _oracle(oracle, sc, host, qs)
    assert got == want
    assert got[0] == [] and got[1] == []
    assert len(got[2]) == 1


def test_capacity_and_argument_errors(sj, engine, star):
    sc, _, dev = star
    b = ss.Batch(engine, sc, dev, group_entries=1000)
    try:
        big = {"preds": [{"dim": 0, "kind": "all", "group_attr": 0}, {"dim": 1, "kind": "all", "group_attr": 0}],
               "row_range": (0, 10)}
        with pytest.raises(sj.StarJoinError) as e:
            b.run([big])
        assert e.value.status == sj.SJ_ERR_CAPACITY
        bad = {"preds": [{"dim": 0, "kind": "all", "group_attr": 0}, {"dim": 0, "kind": "all", "group_attr": -1}],
               "row_range": (0, 10)}
        with pytest.raises(sj.StarJoinError) as e:
            b.run([bad])
        assert e.value.status == sj.SJ_ERR_INVALID_ARGUMENT
        oob = {"preds": [{"dim": 1, "kind": "all", "group_attr": -1}], "row_range": (0, sc.fact_rows + 1)}
        with pytest.raises(sj.StarJoinError):
            b.run([oob])
        # the handle still works after refusals
        ok = {"preds": [{"dim": 3, "kind": "all", "group_attr": 0}], "row_range": (0, 1000)}
        assert sum(r[-2] for r in b.run([ok])[0]) == 1000
    finally:
        b.close()


def test_colliding_dimension_keys_are_refused(sj, engine, star, torch_cuda):
    sc, _, dev = star
    cols = dict(dev)
    k = cols["s_key"].clone()
    k[1] = k[0]  # two supplier rows in one slot
    cols["s_key"] = k
    with pytest.raises(sj.StarJoinError) as e:
        ss.Batch(engine, sc, cols)
    assert e.value.status == sj.SJ_ERR_UNSUPPORTED


def test_cached_filter_regrouped(oracle, engine, star):
    """A cached filter carries the min/max of the attributes its queries grouped
    by; a later batch that reuses it grouped by another attribute completes its
    statistics (a statistics-only build job, the bitmap untouched) and still
    answers like the oracle -- in the same batch and across batches."""
    sc, host, dev = star
    b = ss.Batch(engine, sc, dev, use_graph=True, cache_filters=True)
    try:
        def q(group_attr, other_group):
            return {"preds": [{"dim": 0, "kind": "range", "attr": 1, "lo": 100, "hi": 700, "group_attr": group_attr},
                              {"dim": 1, "kind": "range", "attr": 1, "lo": 0, "hi": 300, "group_attr": other_group}],
                    "row_range": (0, sc.fact_rows)}
        first = [q(0, -1)]                 # supplier filter, statistics of attribute 0
        later = [q(1, -1), q(2, 0)]        # the same filters grouped by attributes 1 and 2
        mixed = [q(0, 1), q(2, 1), q(-1, 2)]  # group spans within the batch's 16M accumulators
        for batch_qs in (first, later, mixed):
            got = b.run(batch_qs)
            for g, bq in zip(got, batch_qs):
                assert g == oracle.run(ss.to_plain(sc, bq), host)
        assert b.stats().filters_cached > 0
    finally:
        b.close()


def test_probe_shape_tuner(oracle, engine, star):
    """sjb_batch_tune: every candidate probe shape (CTA size x shared-memory group
    partials) gives the same groups, and a batch with the chosen shape matches
    the oracle."""
    sc, host, dev = star
    rng = random.Random(6)
    qs = [ss.random_query(rng, sc, len_range=(100_000, None)) for _ in range(24)]
    shape, rep = ss.tune_batch(engine, sc, dev, qs, reps=2)
    assert rep.mismatches == 0 and rep.candidates >= 6
    assert shape["threads"] in (256, 512, 1024) and shape["smem_group_entries"] in (2048, 6144, 12288)
    assert 0 < rep.best_probe_ms <= rep.default_probe_ms
    b = ss.Batch(engine, sc, dev, **shape)
    try:
        got = b.run(qs)
    finally:
        b.close()
    want = _oracle(oracle, sc, host, qs)
    for i, (g, w) in enumerate(zip(got, want)):
        assert g == w, i
