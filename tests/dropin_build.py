"""Build the reference's own SSB drivers (the 12 Q3.3 drivers and the drivers of
Q2.1-Q2.3, Q3.1, Q3.2, Q3.4 and Q4.1-Q4.3) against this repository's
crystal/*.cuh device functions (the drop-in check).

Each driver (src/ssb-jo/q33/<order>-<lip|naive>.cu, compiled where it lies in
the reference tree that oracle/build_ref.py locates) includes
"crystal/crystal.cuh"; with crystal-opt_b200/ first on the include path that
resolves to the sm_100a reimplementation here, while the driver source itself
stays unmodified.  The main() comes from oracle/ref_runner.cu (seeded synthetic
columns).  Binaries go to tests/_dropin/ (git-ignored; they travel with the
snapshot so the GPU tests can run them without the reference tree).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_dropin")


def binary(order: int, method: str) -> str:
    return os.path.join(OUT, f"q33_{order}_{method}")


def available() -> bool:
    return os.path.isdir(os.path.join(REF, "src", "ssb-jo", "q33"))


def _compile(order: int, method: str) -> str:
    src = os.path.join(REF, "src", "ssb-jo", "q33", f"{order}-{method}.cu")
    out = binary(order, method)
    hdrs = [os.path.join(ROOT, "crystal-opt_b200", "crystal", f) for f in os.listdir(
        os.path.join(ROOT, "crystal-opt_b200", "crystal"))]
    deps = [src, os.path.join(ROOT, "oracle", "ref_runner.cu")] + hdrs
    if os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(d) for d in deps):
        return out
    cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
           "-I", os.path.join(ROOT, "crystal-opt_b200"), "-I", os.path.join(ROOT, "oracle", "ref_shim"),
           f'-DREF_DRIVER="{src}"', f"-DREF_LIP={1 if method == 'lip' else 0}",
           "-o", out + ".tmp", os.path.join(ROOT, "oracle", "ref_runner.cu")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"{src}: {r.stderr[-2000:]}")
    os.replace(out + ".tmp", out)
    return out


sys.path.insert(0, os.path.join(ROOT, "oracle"))
from build_ref import REF, SHAPE_SOURCES  # noqa: E402  (reference tree; driver file of each other query)

SHAPES = tuple(SHAPE_SOURCES)


def shape_binary(query: int) -> str:
    return os.path.join(OUT, f"q{query}_ref")


def _compile_shape(query: int) -> str:
    """The query's reference driver against crystal/*.cuh, main() from oracle/ref_runner_shapes.cu."""
    src = os.path.join(REF, "src", "ssb-jo", SHAPE_SOURCES[query])
    out = shape_binary(query)
    runner = os.path.join(ROOT, "oracle", "ref_runner_shapes.cu")
    hdrs = [os.path.join(ROOT, "crystal-opt_b200", "crystal", f) for f in os.listdir(
        os.path.join(ROOT, "crystal-opt_b200", "crystal"))]
    deps = [src, runner] + hdrs
    if os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(d) for d in deps):
        return out
    cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
           "-I", os.path.join(ROOT, "crystal-opt_b200"), "-I", os.path.join(ROOT, "oracle", "ref_shim"),
           "-I", os.path.join(REF, "src", "ssb"),  # gpu_utils.h / ssb_utils.h named without src/ssb/
           f'-DREF_DRIVER="{src}"', f"-DREF_QUERY={query}", "-o", out + ".tmp", runner]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"{src}: {r.stderr[-2000:]}")
    os.replace(out + ".tmp", out)
    return out


BLOCKSUM = os.path.join(OUT, "blocksum_test")


def build_blocksum() -> str:
    """tests/cpp/blocksum_test.cu (the drop-in BlockSum on the GPU against host
    sums); needs no reference tree."""
    src = os.path.join(HERE, "cpp", "blocksum_test.cu")
    hdrs = [os.path.join(ROOT, "crystal-opt_b200", "crystal", f) for f in os.listdir(
        os.path.join(ROOT, "crystal-opt_b200", "crystal"))]
    if os.path.exists(BLOCKSUM) and os.path.getmtime(BLOCKSUM) >= max(os.path.getmtime(d) for d in [src] + hdrs):
        return BLOCKSUM
    os.makedirs(OUT, exist_ok=True)
    cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
           "-I", os.path.join(ROOT, "crystal-opt_b200"), "-o", BLOCKSUM + ".tmp", src]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"{src}: {r.stderr[-2000:]}")
    os.replace(BLOCKSUM + ".tmp", BLOCKSUM)
    return BLOCKSUM


def build(jobs: int = 0) -> list[str]:
    built = [build_blocksum()]
    if not available():
        return built
    os.makedirs(OUT, exist_ok=True)
    jobs = jobs or min(8, os.cpu_count() or 1)
    with cf.ThreadPoolExecutor(jobs) as ex:
        futs = [ex.submit(_compile, o, m) for o in range(6) for m in ("lip", "naive")]
        futs += [ex.submit(_compile_shape, q) for q in SHAPES]
        return built + [f.result() for f in futs]


if __name__ == "__main__":
    for p in build():
        print(p)
    if not available():
        print(f"reference tree not found at {REF}", file=sys.stderr)
