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
    assert len(want) > 20
    n = len(make(SHAPES_SMALL)["dims"])
    orders = list(itertools.permutations(range(n)))[:: max(1, len(list(itertools.permutations(range(n)))) // 4)]
    for order in orders:
        for lip, bpk, k, adaptive in ((True, 0, 2, False), (True, 8, 3, True), (True, 16, 2, False),
                                      (False, 0, 2, False)):
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
