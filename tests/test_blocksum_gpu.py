"""The drop-in BlockSum (crystal/reduce.cuh; the reference's crystal/reduce.cuh:25-75)
on the B200: both overloads, for int, unsigned and long long, on full and ragged
tiles at 32-1024 threads per block, against host sums (tests/cpp/blocksum_test.cu,
built by tests/dropin_build.py)."""
import os
import subprocess

import pytest

import dropin_build

pytestmark = pytest.mark.gpu

CASES = 9  # run_case calls in blocksum_test.cu's main()


def test_block_sum_matches_host_sums(torch_cuda):
    exe = dropin_build.BLOCKSUM
    if not os.path.exists(exe):
        pytest.skip("blocksum_test not built")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    lines = r.stdout.split("\n")
    assert r.returncode == 0, r.stdout + r.stderr
    oks = [ln for ln in lines if ln.startswith("ok ")]
    assert len(oks) == CASES, r.stdout
    assert {ln.split()[1] for ln in oks} == {"int", "unsigned", "long_long"}
