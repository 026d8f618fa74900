"""GPU checks of the autotuner (sj_autotune): every candidate plan gives the
same groups, the chosen plan matches the oracle, and the tuning cache returns
the stored choice for a plan with the same signature."""
import random

import pytest

from workloads import SMALL, sel_query

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small(sj, torch_cuda):
    dev = sj.gen_device(SMALL)
    host = {k: v.cpu().numpy() for k, v in dev.items()}
    return host, dev


def test_q33_search_is_exact_and_not_slower(sj, oracle, engine, small):
    host, dev = small
    q = sj.q33_query(SMALL, order=(2, 1, 0), bf_bits_per_key=16)
    tuned, tune, rep = engine.autotune(q, dev, SMALL.fact_rows, reps=3, tune_filter=True, tune_order=2)
    assert rep.mismatches == 0 and rep.candidates > 20 and rep.cache_hit == 0
    assert rep.best_ms <= rep.default_ms * 1.05 + 0.01
    got, _ = engine.run(tuned, dev, SMALL.fact_rows, tune=tune)
    assert got == oracle.run(q, host)
    assert 0.005 < rep.selectivity[0] < 0.012 and rep.selectivity[2] > 0.8  # 2/250 cities; 6 of 7 years


def test_cache_round_trip(sj, engine, small, tmp_path):
    host, dev = small
    path = str(tmp_path / "tuning.txt")
    q = sj.q33_query(SMALL, order=(0, 1, 2))
    t1, tune1, r1 = engine.autotune(q, dev, SMALL.fact_rows, reps=2, tune_filter=True, cache_path=path)
    assert r1.cache_hit == 0
    t2, tune2, r2 = engine.autotune(q, dev, SMALL.fact_rows, reps=2, tune_filter=True, cache_path=path)
    assert r2.cache_hit == 1 and r2.mismatches == 0
    assert tune1 == tune2 and t1["bf_bits_per_key"] == t2["bf_bits_per_key"] and t1["order"] == t2["order"]
    # different cities, same selectivity class: same signature, served from the cache
    q3 = sj.q33_query(SMALL, order=(0, 1, 2), cities=(17, 99))
    _, tune3, r3 = engine.autotune(q3, dev, SMALL.fact_rows, reps=2, tune_filter=True, cache_path=path)
    assert r3.cache_hit == 1 and tune3 == tune1


def test_four_dim_plans(sj, oracle, engine, torch_cuda):
    sc = sj.StarSchema(seed=78, fact_rows=2_000_000, cust_rows=60_000, supp_rows=4000, part_rows=100_000)
    host = sj.gen_host(sc)
    dev = {k: torch_cuda.from_numpy(v).cuda() for k, v in host.items()}
    rng = random.Random(9)
    for _ in range(3):
        q = sel_query(sc, [rng.choice([1, 10, 100, 500]) for _ in range(4)], seed=rng.randint(0, 1 << 30))
        tuned, tune, rep = engine.autotune(q, dev, sc.fact_rows, reps=2, tune_filter=True, tune_order=1)
        assert rep.mismatches == 0
        got, _ = engine.run(tuned, dev, sc.fact_rows, tune=tune)
        assert got == oracle.run(q, host)
