"""Compile the reference's own SSB drivers into oracle/_ref/ -- TEST INFRASTRUCTURE.

The driver sources are compiled where they lie under the reference tree named
by CRYSTAL_OPT_REF (nothing is built when it is unset); nothing is copied.
Each binary is one driver -- src/ssb-jo/q33/<order>-<lip|naive>.cu wrapped by
ref_runner.cu, or one of SHAPE_SOURCES (the other queries' drivers) wrapped by
ref_runner_shapes.cu -- the wrapper supplying main() and the synthetic columns.  The reference's
CUB 1.6.4 test header is replaced by ref_shim/cub/test/test_util.h.  Flags follow
the reference Makefile (-O3 -lineinfo -Xptxas -dlcm=ca, Makefile:23,35) with the
architecture switched to sm_100a.

The binaries need a GPU to run; they travel with the repository snapshot.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
REF = os.environ.get("CRYSTAL_OPT_REF", "")
ORDERS = range(6)
METHODS = ("lip", "naive")


def binary(order: int, method: str) -> str:
    return os.path.join(OUT, f"q33_{order}_{method}")


def available() -> bool:
    return bool(REF) and os.path.isdir(os.path.join(REF, "src", "ssb-jo", "q33"))


def _compile(order: int, method: str) -> str:
    src = os.path.join(REF, "src", "ssb-jo", "q33", f"{order}-{method}.cu")
    out = binary(order, method)
    deps = [src, os.path.join(HERE, "ref_runner.cu"), os.path.join(HERE, "ref_shim", "cub", "test", "test_util.h")]
    if os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(d) for d in deps):
        return out
    cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
           "-Xptxas", "-dlcm=ca", "-I", REF, "-I", os.path.join(HERE, "ref_shim"),
           f'-DREF_DRIVER="{src}"', f"-DREF_LIP={1 if method == 'lip' else 0}",
           "-o", out + ".tmp", os.path.join(HERE, "ref_runner.cu")]
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE)
    os.replace(out + ".tmp", out)
    return out


# The other queries' drivers under src/ssb-jo/: the order-0 LIP driver where the
# reference has one; Q4.2 has only a naive driver and Q4.3 a single q43.cu.
SHAPE_SOURCES = {21: "q21/0-lip.cu", 22: "q22/0-lip.cu", 23: "q23/0-lip.cu", 31: "q31/0-lip.cu",
                 32: "q32/0-lip.cu", 34: "q34/0-lip.cu", 41: "q41/0-lip.cu", 42: "q42/0-naive.cu",
                 43: "q43/q43.cu"}
SHAPES = tuple(SHAPE_SOURCES)


def shape_binary(query: int) -> str:
    return os.path.join(OUT, f"q{query}_ref")


def _compile_shape(query: int) -> str:
    src = os.path.join(REF, "src", "ssb-jo", SHAPE_SOURCES[query])
    out = shape_binary(query)
    runner = os.path.join(HERE, "ref_runner_shapes.cu")
    deps = [src, runner, os.path.join(HERE, "ref_shim", "cub", "test", "test_util.h")]
    if os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(d) for d in deps):
        return out
    cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
           "-Xptxas", "-dlcm=ca", "-I", REF, "-I", os.path.join(HERE, "ref_shim"),
           # q42/0-naive.cu and q43/q43.cu name gpu_utils.h / ssb_utils.h without their src/ssb/ directory
           "-I", os.path.join(REF, "src", "ssb"),
           f'-DREF_DRIVER="{src}"', f"-DREF_QUERY={query}", "-o", out + ".tmp", runner]
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE)
    os.replace(out + ".tmp", out)
    return out


def build(jobs: int = 0) -> list[str]:
    """Build the 12 Q3.3 drivers and the other queries' drivers (SHAPE_SOURCES);
    skipped when the reference tree is absent."""
    if not available():
        return []
    os.makedirs(OUT, exist_ok=True)
    jobs = jobs or min(8, os.cpu_count() or 1)
    with cf.ThreadPoolExecutor(jobs) as ex:
        futs = [ex.submit(_compile, o, m) for o in ORDERS for m in METHODS]
        futs += [ex.submit(_compile_shape, q) for q in SHAPES]
        return [f.result() for f in futs]


def parse_groups(text: str, width: int) -> list:
    """Group lines of a shape driver's output: `width` integers per line after
    the first "Result:" (other lines, e.g. "Num Matched ...", are skipped)."""
    groups, on = [], False
    for line in text.splitlines():
        line = line.strip()
        if line == "Result:":
            on = True
            continue
        if line.startswith("Res Count:"):
            break
        parts = line.split()
        if on and len(parts) == width and all(p.lstrip("-").isdigit() for p in parts):
            groups.append(tuple(int(p) for p in parts))
    return sorted(groups)


def parse_output(text: str) -> dict:
    """Parse a runner's stdout: result groups (year, c_city, s_city, int32 sum),
    time_query values and probe-only times."""
    import json
    groups = []
    times, probe = [], []
    in_res = False
    for line in text.splitlines():
        line = line.strip()
        if line == "Result:":
            in_res, groups = True, []
            continue
        if line.startswith("Res Count:"):
            in_res = False
            continue
        if in_res:
            parts = line.split()
            if len(parts) == 4:
                groups.append(tuple(int(x) for x in parts))
            continue
        if line.startswith("{"):
            rec = json.loads(line)
            if "time_query" in rec:
                times.append(rec["time_query"])
            if "probe_ms" in rec:
                probe.append(rec["probe_ms"])
    return {"groups": sorted(groups), "time_query_ms": times, "probe_ms": probe}


if __name__ == "__main__":
    for p in build():
        print(p)
    if not available():
        print(f"reference tree not found at {REF}", file=sys.stderr)
