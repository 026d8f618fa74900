"""CPU tests: the generator, the two oracle restatements, and the golden
vectors produced by running the reference's own CUDA drivers."""
import datetime
import json
import os
import random

import numpy as np
import pytest

import oracle_np
import starjoin as sj
from workloads import REF_DRIVER_ORDERS, SMALL, random_query

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
M64 = (1 << 64) - 1


def _splitmix_np(seed: int, col: int, n: int) -> np.ndarray:
    """SplitMix64 (Steele, Lea, Flood 2014) restated with numpy uint64 wraparound."""
    def mix(z):
        z = z + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))
    with np.errstate(over="ignore"):
        key = mix(np.uint64(seed) ^ (np.uint64(col) << np.uint64(40)))
        i = np.arange(n, dtype=np.uint64)
        return mix(key + i * np.uint64(0x9E3779B97F4A7C15))


def _uniform_np(draw: np.ndarray, lo: int, hi: int) -> np.ndarray:
    rng = np.uint64(hi - lo + 1)
    return (lo + ((draw >> np.uint64(32)) * rng >> np.uint64(32)).astype(np.int64)).astype(np.int32)


def test_generator_matches_numpy_restatement(sj):
    sc = sj.StarSchema(seed=12345, fact_rows=100_000, cust_rows=5000, supp_rows=700)
    cols = sj.gen_host(sc)
    for name, (n, col, kind, lo, hi) in sc.column_specs().items():
        if kind == sj.GEN_UNIFORM:
            np.testing.assert_array_equal(cols[name], _uniform_np(_splitmix_np(sc.seed, col, n), lo, hi), name)
        elif kind == sj.GEN_SEQ:
            np.testing.assert_array_equal(cols[name], np.arange(lo, lo + n, dtype=np.int32))
    # fact date keys: uniform day index -> calendar date
    days = _uniform_np(_splitmix_np(sc.seed, sj.COL_FK_DATE, sc.fact_rows), 0, sj.DATE_DAYS - 1)
    base = datetime.date(1992, 1, 1)
    want = np.array([int((base + datetime.timedelta(days=int(d))).strftime("%Y%m%d")) for d in days[:5000]])
    np.testing.assert_array_equal(cols["fk_date"][:5000], want)


def test_date_dimension_is_ssb_calendar(sj):
    cols = sj.gen_host(sj.StarSchema(seed=1, fact_rows=0, cust_rows=1, supp_rows=1), ["d_key", "d_year"])
    base = datetime.date(1992, 1, 1)
    want = [int((base + datetime.timedelta(days=i)).strftime("%Y%m%d")) for i in range(sj.DATE_DAYS)]
    assert cols["d_key"].tolist() == want
    assert cols["d_key"][-1] == 19981230  # the reference's date table ends here (0-lip.cu:219)
    assert (cols["d_year"] == cols["d_key"] // 10000).all()


@pytest.mark.parametrize("seed", range(12))
def test_c_oracle_matches_numpy_oracle(sj, oracle, seed):
    rng = random.Random(seed)
    sc = sj.StarSchema(seed=1000 + seed, fact_rows=rng.choice([0, 1, 7, 5000, 60_000]),
                       cust_rows=rng.choice([1, 31, 3000]), supp_rows=rng.choice([1, 64, 200]),
                       part_rows=rng.choice([0, 500]))
    cols = sj.gen_host(sc)
    for _ in range(4):
        q = random_query(rng, sc)
        assert oracle.run(q, cols) == oracle_np.run(q, cols)


def test_oracle_result_independent_of_order(sj, oracle):
    cols = sj.gen_host(SMALL)
    base = oracle.run(sj.q33_query(SMALL, order=(0, 1, 2)), cols)
    assert len(base) == 24  # 2 s_city x 2 c_city x 6 years
    for o in REF_DRIVER_ORDERS.values():
        assert oracle.run(sj.q33_query(SMALL, order=o), cols) == base


def test_oracle_pht_matches_reference_layout(sj, oracle):
    """BlockBuildSelectivePHT_2 layout: [key, payload] per slot (crystal/join.cuh:260-279)."""
    sc = sj.StarSchema(seed=3, fact_rows=10, cust_rows=1000, supp_rows=64)
    cols = sj.gen_host(sc)
    q = sj.q33_query(sc, cities=tuple(range(0, 250, 2)))
    ht = oracle.build_pht(q, cols, 1)
    np.testing.assert_array_equal(ht, oracle_np.build_pht(q["dims"][1], cols))
    keys = cols["c_key"]
    sel = np.isin(cols["c_city"], np.arange(0, 250, 2))
    slot = keys % sc.cust_rows
    assert (ht[2 * slot[sel]] == keys[sel]).all()
    assert (ht[2 * slot[sel] + 1] == cols["c_city"][sel]).all()
    assert (ht[2 * slot[~sel]] == 0).all()


def test_key_equal_to_len_wraps_to_slot_zero(sj, oracle):
    """HASH(len, len, 0) = 0 (crystal/join.cuh:27): key N lives in slot 0."""
    sc = sj.StarSchema(seed=4, fact_rows=50_000, cust_rows=10, supp_rows=10)
    cols = sj.gen_host(sc)
    q = sj.q33_query(sc, cities=tuple(range(250)))
    ht = oracle.build_pht(q, cols, 0)
    assert ht[0] == 10 and ht[2 * 1] == 1


def _golden(name):
    path = os.path.join(GOLDEN, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not generated yet")
    with open(path) as f:
        return json.load(f)


def test_oracle_matches_reference_cuda_golden(sj, oracle):
    """Pins the oracle: groups printed by the reference's own CUDA drivers
    (oracle/_ref, run on a B200) on the seeded small workload; the reference
    sums in int32 (src/ssb-jo/q33/0-lip.cu:108), so compare the low 32 bits."""
    g = _golden("q33_small_reference.json")
    sc = sj.StarSchema(**g["schema"])
    cols = sj.gen_host(sc)
    ours = oracle.run(sj.q33_query(sc), cols)
    want = sorted(tuple(r) for r in g["groups"])  # (year, c_city, s_city, int32 sum)
    got = sorted((y, c, s, ((v + 2 ** 31) % 2 ** 32) - 2 ** 31) for (s, c, y, cnt, v) in ours)
    assert got == want
    for drv in g["drivers"].values():
        assert sorted(tuple(r) for r in drv) == want  # every order, LIP and naive agree


def test_oracle_matches_reference_shape_golden(sj, oracle):
    """Pins the oracle on the other query shapes: groups printed by the
    reference's own drivers of Q2.1-Q2.3, Q3.1, Q3.2, Q3.4 and Q4.1-Q4.3
    (oracle/_ref, run on a B200) on the seeded SF1-sized schema.  Q2.x, Q3.1,
    Q4.1 and Q4.2 sum in uint64 (Q4.x: revenue - supplycost, two's complement);
    Q3.2, Q3.4 and Q4.3 print an int32 sum."""
    from workloads import SHAPE_QUERIES, shape_as_printed
    g = _golden("shapes_small_reference.json")
    sc = sj.StarSchema(**g["schema"])
    cols = sj.gen_host(sc)
    for q, make in SHAPE_QUERIES.items():
        want = sorted(tuple(r) for r in g["groups"][str(q)])
        assert want, q
        got = shape_as_printed(q, oracle.run(make(sc), cols))
        assert got == [tuple(w) for w in want], q


def test_oracle_generator_matches_engine_generator(sj):
    """The oracle library's copy of the seeded generator (used by the benchmark's
    reference arm, which must not load the engine) gives the engine's columns."""
    import oracle
    sc = sj.StarSchema(seed=424242, fact_rows=200_003, cust_rows=3001, supp_rows=401, part_rows=1501)
    a, b = oracle.gen_host(sc), sj.gen_host(sc)
    assert a.keys() == b.keys()
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    lo, hi = 70_001, 150_013  # one shard of the fact rows
    shard = oracle.gen_host(sc, ["fk_cust", "revenue", "c_city"], fact_range=(lo, hi))
    assert np.array_equal(shard["fk_cust"], a["fk_cust"][lo:hi])
    assert np.array_equal(shard["revenue"], a["revenue"][lo:hi])
    assert np.array_equal(shard["c_city"], a["c_city"])
