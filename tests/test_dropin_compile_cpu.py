"""Compile-only check: drivers of other query families and the reference's
micro-benchmarks build unmodified against crystal-opt_b200/crystal (sm_100a)."""
import os
import subprocess
import concurrent.futures as cf

import pytest

from build_ref import REF  # the reference tree the build recipe reads
from conftest import ROOT

DRIVERS = ["src/ssb-jo/q21/0-lip.cu", "src/ssb-jo/q31/0-lip.cu", "src/ssb-jo/q32/3-naive.cu",
           "src/ssb-jo/q34/5-lip.cu", "src/ssb-jo/q41/0-lip.cu", "src/ops/bloom_join.cu", "src/ops/join.cu"]


@pytest.mark.skipif(not REF or not os.path.isdir(REF), reason="reference tree not present (CRYSTAL_OPT_REF)")
def test_reference_drivers_compile_against_b200_device_api(tmp_path):
    def compile_one(rel):
        cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O1", "-c",
               "-I", os.path.join(ROOT, "crystal-opt_b200"), "-I", os.path.join(ROOT, "oracle", "ref_shim"),
               "-I", os.path.join(REF, "src", "ops"),
               "-o", str(tmp_path / (rel.replace("/", "_") + ".o")), os.path.join(REF, rel)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        return rel, r.returncode, r.stderr[-1500:]
    with cf.ThreadPoolExecutor(min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(compile_one, DRIVERS))
    failed = [(rel, err) for rel, rc, err in results if rc != 0]
    assert not failed, failed
