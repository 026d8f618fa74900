"""The reference's own CUDA drivers (oracle/_ref, compiled from its unmodified
src/ssb-jo/q33 sources) against the oracle on the same seeded inputs."""
import os
import sys

import pytest

import build_ref
from workloads import FULL, SMALL

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from make_golden import run_driver  # noqa: E402

pytestmark = pytest.mark.gpu


def _int32(v):
    return ((v + 2 ** 31) % 2 ** 32) - 2 ** 31


@pytest.mark.parametrize("method", ["lip", "naive"])
@pytest.mark.parametrize("order", range(6))
def test_reference_driver_agrees_with_oracle(sj, oracle, torch_cuda, order, method):
    if not os.path.exists(build_ref.binary(order, method)):
        pytest.skip("reference drivers not built")
    want = sorted((y, c, s, _int32(v)) for (s, c, y, cnt, v) in oracle.run(sj.q33_query(SMALL),
                                                                              sj.gen_host(SMALL)))
    got = run_driver(order, method, SMALL)["groups"]
    assert got == want


@pytest.fixture(scope="module")
def full_engine_groups(sj, engine, torch_cuda):
    """The engine's Q3.3 groups at the bench size (120M fact rows), as the
    reference drivers print them: (d_year, c_city, s_city, int32 SUM)."""
    dev = sj.gen_device(FULL)
    got, _ = engine.run(sj.q33_query(FULL), dev, FULL.fact_rows)
    del dev
    torch_cuda.cuda.empty_cache()
    assert len(got) == 24
    return sorted((y, c, s, _int32(v)) for (s, c, y, cnt, v) in got)


@pytest.mark.parametrize("method", ["lip", "naive"])
@pytest.mark.parametrize("order", range(6))
def test_reference_driver_at_full_size_agrees_with_engine(full_engine_groups, order, method):
    """Each of the reference's 12 Q3.3 drivers (unmodified, oracle/_ref) at 120M
    fact rows prints the engine's groups (its int32 sums, src/ssb-jo/q33/0-lip.cu:108,
    compared as the low 32 bits of the engine's uint64 sums)."""
    if not os.path.exists(build_ref.binary(order, method)):
        pytest.skip("reference drivers not built")
    got = run_driver(order, method, FULL, timeout=900)["groups"]
    assert got == full_engine_groups
