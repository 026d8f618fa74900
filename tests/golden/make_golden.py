"""Regenerate the golden vectors from the reference's own CUDA drivers.

Runs every oracle/_ref/q33_<order>_<lip|naive> binary (the unmodified
src/ssb-jo/q33/*.cu drivers, built by oracle/build_ref.py) on the seeded small
star schema and records the groups each prints: (d_year, c_city, s_city, int32
SUM(lo_revenue)).  Needs a GPU; run from the repository root:

    python tests/golden/make_golden.py            # Q3.3, all 12 drivers
    python tests/golden/make_golden.py --shapes   # Q2.1-Q2.3, Q3.1, Q3.2, Q3.4, Q4.1-Q4.3
"""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "crystal-opt_b200"))

import build_ref  # noqa: E402
from workloads import SMALL  # noqa: E402


def run_driver(order: int, method: str, schema, trials: int = 1, probe_trials: int = 0, timeout=600) -> dict:
    exe = build_ref.binary(order, method)
    cmd = [exe, f"--seed={schema.seed}", f"--n={schema.fact_rows}", f"--c={schema.cust_rows}",
           f"--s={schema.supp_rows}", f"--t={trials}", f"--probe_t={probe_trials}"]
    out = subprocess.run(cmd, check=True, capture_output=True, text=True, timeout=timeout).stdout
    return build_ref.parse_output(out)


def shapes():
    """Groups printed by the reference's drivers for the other queries
    (oracle/_ref/q<query>_ref, built from build_ref.SHAPE_SOURCES) on the seeded
    SF1-sized schema."""
    from workloads import SHAPES_SMALL, SHAPE_WIDTH
    sc = SHAPES_SMALL
    rec = {"what": "groups printed by the reference's src/ssb-jo drivers " +
                   ", ".join(build_ref.SHAPE_SOURCES.values()) + " on the seeded schema; columns as each "
                   "driver prints them",
           "schema": {"seed": sc.seed, "fact_rows": sc.fact_rows, "cust_rows": sc.cust_rows,
                      "supp_rows": sc.supp_rows, "part_rows": sc.part_rows},
           "columns": {"21": ["d_year", "p_brand1", "sum_u64"], "22": ["d_year", "p_brand1", "sum_u64"],
                       "23": ["d_year", "p_brand1", "sum_u64"],
                       "31": ["d_year", "c_nation", "s_nation", "sum_u64"],
                       "32": ["d_year", "c_city", "s_city", "sum_int32"],
                       "34": ["d_year", "c_city", "s_city", "sum_int32"],
                       "41": ["d_year", "c_nation", "sum_u64(revenue-supplycost)"],
                       "42": ["d_year", "s_nation", "p_category", "sum_u64(revenue-supplycost)"],
                       "43": ["d_year", "s_city", "p_brand1", "sum_int32(revenue-supplycost)"]},
           "groups": {}}
    for q in build_ref.SHAPES:
        cmd = [build_ref.shape_binary(q), f"--seed={sc.seed}", f"--n={sc.fact_rows}", f"--c={sc.cust_rows}",
               f"--s={sc.supp_rows}", f"--p={sc.part_rows}"]
        out = subprocess.run(cmd, check=True, capture_output=True, text=True, timeout=600).stdout
        rec["groups"][str(q)] = build_ref.parse_groups(out, SHAPE_WIDTH[q])
    path = os.path.join(ROOT, "tests", "golden", "shapes_small_reference.json")
    with open(path, "w") as f:
        json.dump(rec, f, indent=1)
    print(path, {q: len(v) for q, v in rec["groups"].items()})


def main():
    drivers = {}
    for o in range(6):
        for m in ("lip", "naive"):
            drivers[f"{o}_{m}"] = run_driver(o, m, SMALL)["groups"]
    first = drivers["0_lip"]
    rec = {
        "what": "groups printed by the reference's src/ssb-jo/q33 drivers on the seeded small schema",
        "columns": ["d_year", "c_city", "s_city", "sum_int32"],
        "schema": {"seed": SMALL.seed, "fact_rows": SMALL.fact_rows, "cust_rows": SMALL.cust_rows,
                   "supp_rows": SMALL.supp_rows},
        "groups": first,
        "drivers": drivers,
    }
    path = os.path.join(ROOT, "tests", "golden", "q33_small_reference.json")
    with open(path, "w") as f:
        json.dump(rec, f, indent=1)
    print(path, len(first), "groups")


if __name__ == "__main__":
    if "--shapes" in sys.argv:
        shapes()
    else:
        main()
