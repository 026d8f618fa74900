"""The reference's own CUDA drivers (oracle/_ref, compiled from its unmodified
src/ssb-jo/q33 sources) against the oracle on the same seeded inputs."""
import os
import sys

import pytest

import build_ref
from workloads import SMALL

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
