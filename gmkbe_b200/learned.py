"""Learned schedule: a subtree-size model that orders the root tasks.

Each root task x (all maximal k-biplexes whose smallest U vertex is x) gets 16
integer-derived features (gmk_root_features, computed on the GPU: k, depth,
degree of x, candidate and exclusion set sizes, 2-hop sizes, neighbour degree
statistics).  A 16-64-64-1 perceptron with FP16 weights and FP32 accumulation
(gmk_mlp_*, trained on the GPU by the library's own forward, backward and
Adam kernels) predicts log1p of the task's search-tree nodes.  The targets are
the node counts the plain schedule logs per root (gmk_opts.root_nodes).

The predictions only order the work: GMK_SCHEDULE_ORDERED starts the largest
predicted roots first (longest-processing-time order), which shortens the
tail of a full enumeration.  Nothing is pruned, so the result set is the
same with or without the model.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .api import GmkError, Graph, _check, load_library

N_FEATURES = 16
N_PARAMS = 5313
_PF = ctypes.POINTER(ctypes.c_float)


def _fp(a: np.ndarray):
    return a.ctypes.data_as(_PF)


def root_features(g: Graph, k: int) -> np.ndarray:
    """(n_left, 16) float32 features of every root of g (FP16-rounded)."""
    lib = load_library()
    out = np.zeros((g.n_left, N_FEATURES), np.float32)
    _check(lib.gmk_root_features(g._h, k, _fp(out)))
    return out


def subtree_nodes(g: Graph, k: int, **kw) -> np.ndarray:
    """Search nodes of every root task, logged by a batched run (split records
    carry their root, so the log is per root whatever the schedule)."""
    nodes = np.zeros(g.n_left, np.uint64)
    g.enumerate(k=k, schedule="batched", root_nodes=nodes, **kw)
    return nodes


class SubtreeModel:
    """The 16-64-64-1 model on one GPU (gmk_mlp)."""

    def __init__(self, device: int = 0, seed: int = 0):
        self._lib = load_library()
        h = ctypes.c_void_p()
        _check(self._lib.gmk_mlp_create(device, seed, ctypes.byref(h)))
        self._h = h

    def close(self) -> None:
        if self._h:
            self._lib.gmk_mlp_free(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        p = np.zeros(N_PARAMS, np.float32)
        _check(self._lib.gmk_mlp_params(self._h, _fp(p), None))
        return p

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        if p.size != N_PARAMS:
            raise ValueError(f"expected {N_PARAMS} parameters")
        _check(self._lib.gmk_mlp_params(self._h, None, _fp(p)))

    def gradient(self, x: np.ndarray, y: np.ndarray) -> tuple[np.ndarray, float]:
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        g = np.zeros(N_PARAMS, np.float32)
        loss = ctypes.c_float()
        _check(self._lib.gmk_mlp_gradient(self._h, _fp(x), _fp(y), len(y), _fp(g),
                                          ctypes.byref(loss)))
        return g, loss.value

    def train(self, x: np.ndarray, y: np.ndarray, epochs: int = 400, lr: float = 3e-3) -> float:
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        loss = ctypes.c_float()
        _check(self._lib.gmk_mlp_train(self._h, _fp(x), _fp(y), len(y), epochs, lr,
                                       ctypes.byref(loss)))
        return loss.value

    def predict(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32)
        out = np.zeros(x.shape[0], np.float32)
        _check(self._lib.gmk_mlp_predict(self._h, _fp(x), x.shape[0], _fp(out)))
        return out

    def predict_roots(self, g: Graph, k: int) -> np.ndarray:
        """The prediction for every root of g, features and forward pass on the
        device (gmk_mlp_predict_roots): predict(root_features(g, k)) without
        the host round trip."""
        out = np.zeros(g.n_left, np.float32)
        _check(self._lib.gmk_mlp_predict_roots(self._h, g._h, k, _fp(out)))
        return out


def target(nodes: np.ndarray) -> np.ndarray:
    """Training target: log1p of the node count."""
    return np.log1p(nodes.astype(np.float64)).astype(np.float32)


def spearman(a, b) -> float:
    """Spearman rank correlation (average ranks for ties)."""
    def ranks(v):
        v = np.asarray(v, np.float64)
        order = np.argsort(v, kind="mergesort")
        r = np.empty(v.size, np.float64)
        r[order] = np.arange(v.size, dtype=np.float64)
        _, inv, cnt = np.unique(v, return_inverse=True, return_counts=True)
        sums = np.zeros(cnt.size)
        np.add.at(sums, inv, r)
        return (sums / cnt)[inv]
    ra, rb = ranks(a), ranks(b)
    ra -= ra.mean()
    rb -= rb.mean()
    den = np.sqrt((ra * ra).sum() * (rb * rb).sum())
    return float((ra * rb).sum() / den) if den > 0 else 0.0


def mean_relative_error(pred_nodes, true_nodes) -> float:
    """Mean of |pred - true| / true over roots with true > 0."""
    p = np.asarray(pred_nodes, np.float64)
    t = np.asarray(true_nodes, np.float64)
    m = t > 0
    return float(np.mean(np.abs(p[m] - t[m]) / t[m])) if m.any() else 0.0


def makespan(costs, order, workers: int) -> float:
    """Finish time of list scheduling: tasks taken in `order` by the first
    free of `workers` identical workers (what the device work queue does)."""
    import heapq
    loads = [0.0] * workers
    heapq.heapify(loads)
    for i in order:
        t = heapq.heappop(loads)
        heapq.heappush(loads, t + float(costs[i]))
    return max(loads)


def predicted_costs(model: SubtreeModel, g: Graph, k: int) -> np.ndarray:
    """Predicted node counts of every root (task_cost for the ordered schedule)."""
    return np.expm1(np.maximum(model.predict_roots(g, k), 0.0)).astype(np.float32)


__all__ = ["SubtreeModel", "root_features", "subtree_nodes", "target", "spearman",
           "mean_relative_error", "makespan", "predicted_costs", "GmkError", "MODEL_PATH",
           "training_set", "train_default", "load_default"]


# ----------------------------------------------------------------------------- training
MODEL_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "models", "subtree.npy")


def _families():
    """Training families: seeded graphs of the benchmark configurations'
    generators, cut to induced prefixes whose complete enumeration finishes in
    seconds (the full graphs have ~|E|.|V| maximal k-biplexes).  Each entry:
    (name, builder(seed) -> graphgen.Graphs, the ks of each graph, seeds)."""
    from . import graphgen as gg

    def er200(seed):
        return [gg.erdos_renyi(200, 200, 0.05, seed)]

    def cl20k(seed):
        return [gg.induced_prefix(gg.chung_lu(20_000, 50_000, 500_000, 2.1, seed, 2000),
                                  5_000, 12_000)]

    def cl100k(seed):
        full = gg.chung_lu(100_000, 300_000, 3_000_000, 2.2, seed)
        return [gg.induced_prefix(full, 20_000, 60_000), gg.induced_prefix(full, 4_000, 12_000)]

    def cl500k(seed):
        full = gg.chung_lu(500_000, 1_000_000, 20_000_000, 2.0, seed)
        return [gg.induced_prefix(full, 20_000, 40_000), gg.induced_prefix(full, 10_000, 20_000)]

    # (name, builder, k of each graph the builder returns, seeds)
    return [("er200", er200, ((1,),), range(10, 20)),
            ("cl20k", cl20k, ((1,),), range(10, 20)),
            ("cl100k", cl100k, ((1,), (2,)), range(10, 20)),
            ("cl500k", cl500k, ((2,), (3,)), range(10, 13))]


def training_set(watchdog_ms: int = 20_000, device: int = 0, log=None):
    """(features, targets, info) over the training families: per root task, its
    16 features and log1p of its search nodes, logged by complete runs."""
    xs, ys, info = [], [], []
    for name, build, kss, seeds in _families():
        for seed in seeds:
            for h, ks in zip(build(seed), kss):
                if h.n_left in (0, h.n):
                    continue
                _log_graph(h, ks, name, seed, watchdog_ms, device, xs, ys, info, log)
    return np.concatenate(xs), np.concatenate(ys), info


def _log_graph(h, ks, name, seed, watchdog_ms, device, xs, ys, info, log):
    """Appends graph h's features and logged subtree sizes for each k."""
    with Graph.from_graph(h, device=device) as g:
        for k in ks:
            try:
                nodes = subtree_nodes(g, k, watchdog_ms=watchdog_ms)
            except GmkError as e:
                if e.code != -8:      # watchdog: this case is skipped
                    raise
                info.append({"family": name, "seed": seed, "k": k, "skipped": "watchdog"})
                continue
            xs.append(root_features(g, k))
            ys.append(target(nodes))
            info.append({"family": name, "seed": seed, "k": k, "roots": int(h.n_left),
                         "nodes": int(nodes.sum())})
            if log:
                log(info[-1])


def train_default(out_path: str = MODEL_PATH, epochs: int = 1500, lr: float = 3e-3, seed: int = 1,
                  device: int = 0, log=None) -> dict:
    """Trains the shipped model on the training families (seeds 10-19) with the
    library's GPU kernels and saves its FP32 master weights."""
    x, y, info = training_set(device=device, log=log)
    m = SubtreeModel(device=device, seed=seed)
    loss = m.train(x, y, epochs=epochs, lr=lr)
    os.makedirs(os.path.dirname(out_path), exist_ok=True)
    np.save(out_path, m.params())
    return {"samples": int(len(y)), "loss": float(loss), "epochs": epochs, "lr": lr, "cases": info}


def load_default(device: int = 0, path: str = MODEL_PATH) -> SubtreeModel:
    """The shipped model (weights trained by train_default)."""
    m = SubtreeModel(device=device, seed=0)
    m.set_params(np.load(path))
    return m


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser(description="train the subtree-size model on the GPU")
    ap.add_argument("--out", default=MODEL_PATH)
    ap.add_argument("--epochs", type=int, default=1500)
    a = ap.parse_args()
    res = train_default(a.out, epochs=a.epochs, log=lambda r: print(json.dumps(r), flush=True))
    print(json.dumps({k: v for k, v in res.items() if k != "cases"}), flush=True)
