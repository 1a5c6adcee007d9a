"""Plain vs batched vs learned schedules on full enumerations, and a mixed
batch of graphs in one launch vs one launch per graph.

    python -m gmkbe_b200.compare_schedules [--json out.json]

Full enumeration is where scheduling matters: with a result limit every warp
stays busy until the limit, but a complete run ends with the last, largest
search tree.  Each case reports device time (CUDA events) per schedule and
checks that every schedule gives the same set summary.
  * plain   -- one task per root in id order, no splitting;
  * batched -- roots cut into chunks, chunk-major queue, unfinished trees
               split into the next round;
  * learned -- batched, roots ordered by the subtree-size model's predicted
               node count (largest first), the model trained on the
               plain-schedule subtree sizes of seeded graphs of the same
               families (seeds 10-19).
The mixed batch is 64 uneven graphs (seeds 100-163, sides log-uniform in
[6, 40], average degree uniform in [1.5, 3], half Erdos-Renyi and half
Chung-Lu, k in {1, 2, 3}), enumerated completely.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import graphgen as gg
from . import learned as L
from .api import Graph, enumerate_batch

GOLDEN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests",
                      "golden")
CASES = [("crime", 1), ("er200", 1), ("cl20k_sub", 1), ("southernwomen", 3), ("er60", 2)]


def _timed(g: Graph, reps: int = 3, **kw):
    best, st = None, None
    for _ in range(reps):
        st = g.enumerate(**kw)
        best = st.kernel_ms if best is None else min(best, st.kernel_ms)
    return best, st


def _train_model(k: int) -> L.SubtreeModel:
    xs, ys = [], []
    for seed in range(10, 20):
        for h in (gg.erdos_renyi(40, 40, 0.12, seed), gg.chung_lu(60, 120, 420, 2.1, seed, max_deg=25)):
            with Graph.from_graph(h) as dg:
                xs.append(L.root_features(dg, k))
                ys.append(L.target(L.subtree_nodes(dg, k)))
    m = L.SubtreeModel(seed=1)
    m.train(np.concatenate(xs), np.concatenate(ys), epochs=600, lr=3e-3)
    return m


def full_enumerations() -> list[dict]:
    out = []
    models: dict[int, L.SubtreeModel] = {}
    for name, k in CASES:
        with Graph.load(os.path.join(GOLDEN, f"{name}.graph.bin")) as g:
            if k not in models:
                models[k] = _train_model(k)
            t_plain, s_plain = _timed(g, k=k, schedule="plain")
            t_batch, s_batch = _timed(g, k=k, schedule="batched")
            nodes = L.subtree_nodes(g, k)
            cost = L.predicted_costs(models[k], g, k)
            t_learn, s_learn = _timed(g, k=k, schedule="ordered", task_cost=cost)
            same = s_plain.summary() == s_batch.summary() == s_learn.summary()
            out.append({"graph": name, "k": k, "results": s_plain.count,
                        "plain_ms": t_plain, "batched_ms": t_batch, "learned_ms": t_learn,
                        "batched_speedup": t_plain / t_batch, "learned_speedup": t_plain / t_learn,
                        "rounds_batched": s_batch.rounds, "same_set": same,
                        "spearman": L.spearman(cost, nodes),
                        "mean_relative_error": L.mean_relative_error(cost, nodes)})
    return out


def mixed_batch() -> dict:
    gs, ks = gg.mixed_batch(64, 100, size_lo=6, size_hi=40, deg_lo=1.5, deg_hi=3.0)
    pairs = [(g, k) for g, k in zip(gs, ks) if g.n_left not in (0, g.n)]
    dgs = [Graph.from_graph(g) for g, _ in pairs]
    ks = [k for _, k in pairs]
    try:
        enumerate_batch(dgs, ks)                        # warm-up
        t0 = time.perf_counter()
        batch = enumerate_batch(dgs, ks)
        wall_batch = time.perf_counter() - t0
        seq_ms, seq_wall, same = 0.0, 0.0, True
        for dg, k, st in zip(dgs, ks, batch):
            t0 = time.perf_counter()
            s = dg.enumerate(k=k, schedule="plain")
            seq_wall += time.perf_counter() - t0
            seq_ms += s.kernel_ms
            same &= s.summary() == st.summary()
        total = sum(st.count for st in batch)
        return {"graphs": len(dgs), "results": total, "batch_ms": batch[0].kernel_ms,
                "batch_wall_s": wall_batch, "one_launch_per_graph_ms": seq_ms,
                "one_launch_per_graph_wall_s": seq_wall,
                "speedup_device": seq_ms / batch[0].kernel_ms,
                "speedup_wall": seq_wall / wall_batch, "same_sets": same,
                "batch_results_per_s": total / (batch[0].kernel_ms / 1e3)}
    finally:
        for dg in dgs:
            dg.close()


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--json", help="also write the results here")
    a = ap.parse_args(argv)
    res = {"full_enumeration": full_enumerations(), "mixed_batch": mixed_batch()}
    print(json.dumps(res, indent=1))
    if a.json:
        with open(a.json, "w") as f:
            json.dump(res, f, indent=1)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
