"""Regenerate the golden fixtures under tests/golden/.

Run in a checkout that has the reference tree at $GMK_REFERENCE (oracle/refpath.py)
and the BPPivot binary built by `make -C oracle ref`:

    python tests/golden/make_golden.py

It writes
  * <name>.graph.bin  -- the reference's KONECT fixtures
    (baselines/MaximalBiPlex/datas/*.txt, first line = size header, stripped)
    passed through the converter ordering (gmkbe_b200.graphgen.relabel), plus
    the seeded synthetic graphs small enough to enumerate completely;
  * golden.json       -- for every (graph, k): the number of maximal k-biplexes
    and the order-independent set summary (sum of h1, xor of h2) computed from
    the sets printed by the reference's BPPivot (`-q 1 -o 1`), and the same
    summary from the C oracle, which must agree.
  * southernwomen_k1_sets.txt -- BPPivot's 1256 k=1 sets, one "X | Y" per line.
"""
from __future__ import annotations

import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

import oracle as O  # noqa: E402
from gmkbe_b200 import graphgen as gg  # noqa: E402

from oracle.refpath import REFERENCE as REF  # noqa: E402
FIXTURES = {
    "southernwomen": "baselines/MaximalBiPlex/datas/opsahl_southernwomen.txt",
    "crime": "baselines/MaximalBiPlex/datas/moreno_crime.txt",
    "ucforum": "baselines/MaximalBiPlex/datas/opsahl_ucforum.txt",
}
# (graph, k) pairs whose complete result set is summarised; larger k on the
# bigger fixtures does not finish on one CPU core in reasonable time.
CASES = [("southernwomen", 1), ("southernwomen", 2), ("southernwomen", 3),
         ("crime", 1), ("er200", 1), ("cl20k_sub", 1), ("er60", 1), ("er60", 2)]


def load_konect(path: str) -> gg.Graph:
    rows = []
    with open(path) as f:
        f.readline()                                   # size header
        for line in f:
            t = line.split()
            if len(t) >= 2 and t[0][0] not in "%#":
                rows.append((int(t[0]), int(t[1])))
    e = np.array(rows, dtype=np.int64)
    return gg.relabel(e[:, 0], e[:, 1])


def graphs() -> dict[str, gg.Graph]:
    out = {name: load_konect(os.path.join(REF, rel)) for name, rel in FIXTURES.items()}
    out["er200"] = gg.make_workload("er200")
    out["cl20k_sub"] = gg.make_workload("cl20k_sub")
    out["er60"] = gg.erdos_renyi(30, 30, 0.15, 60)
    return out


def main() -> None:
    gs = graphs()
    meta = {}
    for name, g in gs.items():
        path = os.path.join(HERE, f"{name}.graph.bin")
        gg.write_graph_bin(g, path)
        meta[name] = {"n": g.n, "n_left": g.n_left, "edges": g.n_edges}
    golden = {"graphs": meta, "cases": []}
    for name, k in CASES:
        g = gs[name]
        path = os.path.join(HERE, f"{name}.graph.bin")
        t0 = time.time()
        r = O.run_bppivot(path, k, output=True)
        sets = list(O.parse_bppivot_sets(r["text"], g.n_left))
        ref = O.set_summary(sets)
        assert ref[0] == r["count"], (name, k, ref[0], r["count"])
        orc = O.enumerate_oracle(g, k)
        assert orc.summary() == ref, (name, k, orc.summary(), ref)
        if name == "southernwomen" and k == 1:
            with open(os.path.join(HERE, "southernwomen_k1_sets.txt"), "w") as f:
                for x, y in sorted(sets):
                    f.write(" ".join(map(str, x)) + " | " + " ".join(map(str, y)) + "\n")
        golden["cases"].append({"graph": name, "k": k, "count": ref[0],
                                "hash_sum": f"{ref[1]:016x}", "hash_xor": f"{ref[2]:016x}",
                                "bppivot_branch_ms": r["branch_ms"]})
        print(f"{name} k={k}: {ref[0]} sets, bppivot {r['branch_ms']} ms, "
              f"oracle agrees ({time.time() - t0:.1f}s)", flush=True)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(golden, f, indent=1)


if __name__ == "__main__":
    main()
