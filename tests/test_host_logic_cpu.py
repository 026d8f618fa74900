"""The shared-scan forms' host logic (range allocator, filter cache, circular-scan
coverage, group and step layouts) compiled with g++ and run on the CPU."""
import os
import subprocess

from conftest import ROOT


def test_host_logic(tmp_path):
    exe = str(tmp_path / "host_logic_test")
    cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-I", os.path.join(ROOT, "crystal-opt_b200", "csrc"),
                    "-I", os.path.join(ROOT, "include"), "-I", cuda_inc,
                    os.path.join(ROOT, "tests", "cpp", "host_logic_test.cpp"), "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == "OK"
