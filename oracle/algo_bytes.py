"""Writes profiles/algo_bytes.json: the algorithmic bytes of the benchmark
workloads -- MEASUREMENT INFRASTRUCTURE, never imported by the product.

    python oracle/algo_bytes.py

For each (workload, k, result limit) it runs oracle/work_count (the per-thread
search restated on the host, one task per root in id order) and records the
adjacency words it reads.  The count is fixed per (graph, k, limit) and does
not depend on the GPU's schedule, so bench.py divides 4 x words by the
kernel's time for the roofline's achieved bandwidth.  For a result-limited
run it is the count up to that many results in root order.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)

from gmkbe_b200 import graphgen as gg  # noqa: E402

CASES = [
    ("cl20k_sub", os.path.join(ROOT, "tests", "golden", "cl20k_sub.graph.bin"), 1, 0),
    ("er200", os.path.join(ROOT, "tests", "golden", "er200.graph.bin"), 1, 0),
    ("cl20k", None, 1, 1_000_000),
]


def main() -> int:
    exe = os.path.join(HERE, "work_count")
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    out = {"what": "adjacency words read by the per-thread search restated on the host "
                   "(oracle/work_count.cpp over gmkbe_b200/csrc/enum_core.cuh), one task per "
                   "root in id order; algo_bytes = 4 x words",
           "command": "python oracle/algo_bytes.py", "cases": []}
    for name, path, k, limit in CASES:
        path = path or gg.cached_workload(name)
        r = json.loads(subprocess.run([exe, path, str(k), str(limit)], check=True,
                                      capture_output=True, text=True).stdout)
        r.update(workload=name)
        r["bytes_per_result"] = r["algo_bytes"] / max(1, r["results"])
        out["cases"].append(r)
        print(json.dumps(r), flush=True)
    with open(os.path.join(ROOT, "profiles", "algo_bytes.json"), "w") as f:
        json.dump(out, f, indent=1)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
