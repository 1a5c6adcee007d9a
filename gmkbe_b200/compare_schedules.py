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
CASES = [("er200", 1), ("cl20k_sub", 1), ("southernwomen", 3), ("er60", 2), ("crime", 1)]
WATCHDOG_MS = 30_000   # a schedule that has not finished by then is reported as such


def _timed(g: Graph, **kw):
    """(device ms, stats) of one run, or (None, None) when the watchdog ended it."""
    from .api import GmkError
    try:
        st = g.enumerate(watchdog_ms=WATCHDOG_MS, **kw)
    except GmkError as e:
        if e.code == -8:
            return None, None
        raise
    return st.kernel_ms, st


def _ratio(a, b):
    return None if a is None or b is None else a / b


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
            t_batch, s_batch = _timed(g, k=k, schedule="batched")
            cost = L.predicted_costs(models[k], g, k)
            t_learn, s_learn = _timed(g, k=k, schedule="ordered", task_cost=cost)
            t_plain, s_plain = _timed(g, k=k, schedule="plain")
            sums = {s.summary() for s in (s_plain, s_batch, s_learn) if s is not None}
            row = {"graph": name, "k": k, "results": (s_batch or s_plain).count if (s_batch or s_plain) else None,
                   "plain_ms": t_plain, "batched_ms": t_batch, "learned_ms": t_learn,
                   "batched_speedup": _ratio(t_plain, t_batch),
                   "learned_speedup": _ratio(t_plain, t_learn),
                   "rounds_batched": s_batch.rounds if s_batch else None,
                   "same_set": len(sums) == 1, "watchdog_ms": WATCHDOG_MS}
            if s_plain is not None:
                nodes = L.subtree_nodes(g, k, watchdog_ms=WATCHDOG_MS)
                row["spearman"] = L.spearman(cost, nodes)
                row["mean_relative_error"] = L.mean_relative_error(cost, nodes)
            print(json.dumps(row), flush=True)
            out.append(row)
    return out


def mixed_batch() -> dict:
    gs, ks = gg.mixed_batch(64, 100, size_lo=6, size_hi=40, deg_lo=1.5, deg_hi=3.0)
    from .api import GmkError
    pairs = [(g, k) for g, k in zip(gs, ks) if g.n_left not in (0, g.n)]
    dgs = [Graph.from_graph(g) for g, _ in pairs]
    ks = [k for _, k in pairs]
    try:
        enumerate_batch(dgs, ks)                        # warm-up
        t0 = time.perf_counter()
        batch = enumerate_batch(dgs, ks)
        wall_batch = time.perf_counter() - t0
        seq_ms, seq_wall, same, unfinished = 0.0, 0.0, True, 0
        for dg, k, st in zip(dgs, ks, batch):
            t0 = time.perf_counter()
            try:
                s = dg.enumerate(k=k, schedule="plain", watchdog_ms=10_000)
            except GmkError as e:
                if e.code != -8:
                    raise
                unfinished += 1
                seq_ms += 10_000
                seq_wall += time.perf_counter() - t0
                continue
            seq_wall += time.perf_counter() - t0
            seq_ms += s.kernel_ms
            same &= s.summary() == st.summary()
        total = sum(st.count for st in batch)
        return {"graphs": len(dgs), "results": total, "batch_ms": batch[0].kernel_ms,
                "batch_wall_s": wall_batch, "one_launch_per_graph_ms": seq_ms,
                "one_launch_per_graph_wall_s": seq_wall,
                "speedup_device": seq_ms / batch[0].kernel_ms,
                "speedup_wall": seq_wall / wall_batch, "same_sets": same,
                "plain_runs_unfinished_at_watchdog": unfinished,
                "batch_results_per_s": total / (batch[0].kernel_ms / 1e3)}
    finally:
        for dg in dgs:
            dg.close()


def mixed_batch_stated(cap: int = 1_000_000, n_graphs: int = 64) -> dict:
    """The mixed batch at its stated sizes (|U|, |V| log-uniform in [1k, 50k],
    average degree 5-30, half ER and half Chung-Lu, k in {1,2,3}, seeds
    100-163) in one launch with learned ordering and a per-graph result cap
    (complete enumeration of these graphs does not end: each has far more
    maximal k-biplexes than any cap), against one capped launch per graph."""
    gs, ks = gg.mixed_batch(n_graphs, 100)
    pairs = [(g, k) for g, k in zip(gs, ks) if g.n_left not in (0, g.n)]
    dgs = [Graph.from_graph(g) for g, _ in pairs]
    ks = [k for _, k in pairs]
    model = L.load_default()
    try:
        costs = [L.predicted_costs(model, dg, k) for dg, k in zip(dgs, ks)]
        caps = [cap] * len(dgs)
        enumerate_batch(dgs, ks, schedule="ordered", task_costs=costs, limits=caps)   # warm-up
        t0 = time.perf_counter()
        batch = enumerate_batch(dgs, ks, schedule="ordered", task_costs=costs, limits=caps)
        wall_batch = time.perf_counter() - t0
        enumerate_batch(dgs, ks, schedule="batched", limits=caps)
        chunk_major = enumerate_batch(dgs, ks, schedule="batched", limits=caps)
        seq_ms, seq_wall, same_counts = 0.0, 0.0, True
        for dg, k, st in zip(dgs, ks, batch):
            t0 = time.perf_counter()
            s = dg.enumerate(k=k, result_limit=cap, schedule="plain")
            seq_wall += time.perf_counter() - t0
            seq_ms += s.kernel_ms
            same_counts &= s.count == st.count
        total = sum(st.count for st in batch)
        return {"graphs": len(dgs), "cap": cap, "results": total,
                "edges": [g.n_edges for g, _ in pairs], "counts": [st.count for st in batch],
                "truncated": sum(st.truncated for st in batch),
                "batch_ms": batch[0].kernel_ms, "batch_wall_s": wall_batch,
                "batch_chunk_major_ms": chunk_major[0].kernel_ms,
                "one_plain_launch_per_graph_ms": seq_ms, "one_launch_per_graph_wall_s": seq_wall,
                "speedup_device": seq_ms / batch[0].kernel_ms, "same_counts": same_counts,
                "batch_results_per_s": total / (batch[0].kernel_ms / 1e3)}
    finally:
        for dg in dgs:
            dg.close()


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--json", help="also write the results here")
    ap.add_argument("--stated", action="store_true",
                    help="only the mixed batch at its stated sizes, with per-graph caps")
    ap.add_argument("--cap", type=int, default=1_000_000)
    a = ap.parse_args(argv)
    if a.stated:
        res = {"mixed_batch_stated": mixed_batch_stated(a.cap)}
        print(json.dumps(res["mixed_batch_stated"]), flush=True)
    else:
        res = {"full_enumeration": full_enumerations()}
        res["mixed_batch"] = mixed_batch()
        print(json.dumps(res["mixed_batch"]), flush=True)
    if a.json:
        with open(a.json, "w") as f:
            json.dump(res, f, indent=1)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
