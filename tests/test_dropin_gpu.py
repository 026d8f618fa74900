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


@pytest.mark.parametrize("query", sorted(dropin_build.SHAPES))
def test_reference_shape_driver_on_b200_device_api(sj, oracle, torch_cuda, query):
    """The reference's own drivers of the other queries, compiled unmodified
    against crystal/*.cuh, print the oracle's groups and the golden vectors of
    the same drivers built against the reference's headers."""
    from workloads import SHAPE_QUERIES, SHAPE_WIDTH, SHAPES_SMALL, shape_as_printed
    exe = dropin_build.shape_binary(query)
    if not os.path.exists(exe):
        pytest.skip("drop-in drivers not built")
    import build_ref
    sc = SHAPES_SMALL
    out = subprocess.run([exe, f"--seed={sc.seed}", f"--n={sc.fact_rows}", f"--c={sc.cust_rows}",
                          f"--s={sc.supp_rows}", f"--p={sc.part_rows}"],
                         check=True, capture_output=True, text=True, timeout=300).stdout
    got = build_ref.parse_groups(out, SHAPE_WIDTH[query])
    want = shape_as_printed(query, oracle.run(SHAPE_QUERIES[query](sc), sj.gen_host(sc)))
    assert got == want
    golden = os.path.join(os.path.dirname(__file__), "golden", "shapes_small_reference.json")
    if os.path.exists(golden):
        with open(golden) as f:
            assert got == [tuple(r) for r in json.load(f)["groups"][str(query)]]
