"""Build recipe for the star-join engine: nvcc -> in-tree shared library.

The CUDA sources under csrc/ compile for sm_100a only into
_build/libstarjoin.so (in-tree, so it travels with the repository snapshot).
A rebuild happens when any source or header is newer than the library.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "libstarjoin.so")

SOURCES = ["sj_engine.cu", "sj_build.cu", "sj_probe.cu", "sj_batch.cu", "sj_batch_host.cu", "sj_serve.cu",
           "sj_autotune.cu", "sj_ssbio.cu", "sj_noalloc.cu"]
HEADERS = ["sj_internal.h", "sj_ptx.cuh", "sj_datagen.h", "sj_shared.h", "sj_cache.h", "sj_l2.h"]
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-pthread"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _sources() -> list[str]:
    return [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build_engine(force: bool = False, verbose: bool = False) -> str:
    """Compile csrc/*.cu (one object each, in parallel) and link
    _build/libstarjoin.so; return its path."""
    from concurrent.futures import ThreadPoolExecutor

    srcs = _sources()
    common = [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(ROOT, "include", "starjoin.h"), os.path.join(ROOT, "include", "starjoin_batch.h")]
    objdir = os.path.join(BUILD, "obj")
    os.makedirs(objdir, exist_ok=True)
    objs = [os.path.join(objdir, os.path.basename(s)[:-3] + ".o") for s in srcs]
    todo = [(s, o) for s, o in zip(srcs, objs) if force or _stale(o, [s] + common)]

    def compile_one(so):
        src, obj = so
        cmd = [_nvcc(), *GENCODE, *NVCC_FLAGS, "-I", os.path.join(ROOT, "include"), "-c", "-o", obj + ".tmp", src]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        os.replace(obj + ".tmp", obj)

    with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 1))) as ex:
        list(ex.map(compile_one, todo))
    if force or todo or _stale(LIB, objs):
        tmp = LIB + ".tmp"
        cmd = [_nvcc(), *GENCODE, "-shared", "-Xcompiler", "-pthread", "-o", tmp, *objs]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build_engine(force="--force" in sys.argv, verbose=True))
