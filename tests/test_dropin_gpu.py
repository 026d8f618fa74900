"""The reference's own Q3.3 drivers, compiled unmodified against this
repository's crystal/*.cuh (tests/dropin_build.py), produce the reference's
answer: the same groups as the oracle and as the golden vectors printed by the
drivers built against the reference's own headers."""
import json
import os
import subprocess

import pytest

import dropin_build
from workloads import SMALL

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "q33_small_reference.json")


def _int32(v):
    return ((v + 2 ** 31) % 2 ** 32) - 2 ** 31


@pytest.mark.parametrize("method", ["lip", "naive"])
@pytest.mark.parametrize("order", range(6))
def test_reference_driver_on_b200_device_api(sj, oracle, torch_cuda, order, method):
    exe = dropin_build.binary(order, method)
    if not os.path.exists(exe):
        pytest.skip("drop-in drivers not built")
    import build_ref
    out = subprocess.run([exe, f"--seed={SMALL.seed}", f"--n={SMALL.fact_rows}", f"--c={SMALL.cust_rows}",
                          f"--s={SMALL.supp_rows}", "--t=1", "--probe_t=2"],
                         check=True, capture_output=True, text=True, timeout=300).stdout
    got = build_ref.parse_output(out)["groups"]
    want = sorted((y, c, s, _int32(v)) for (s, c, y, cnt, v) in oracle.run(sj.q33_query(SMALL), sj.gen_host(SMALL)))
    assert got == want
    with open(GOLDEN) as f:
        assert got == sorted(tuple(r) for r in json.load(f)["groups"])
