"""Autotuner for the warp engine's schedule knobs.

For one (graph, k) it times short result-limited enumerations over a small
grid of settings and keeps the fastest:
  * chunk           first-level children per root task (0 = about 8 tasks per warp);
  * split_min_nodes nodes a task must have run before a hungry round splits it;
  * pair_limit      largest |S u C_U| x |S u C_V| at which the node rules
                    (shortcut, forcing, exclusion prune) run.
None of them changes the result set, only the schedule and the pruning
effort.  Winners are cached in a JSON file keyed by the graph's fingerprint,
k and the result limit, so a graph is tuned once.
"""
from __future__ import annotations

import json
import os
import time

from .api import Graph

DEFAULT_GRID = [
    dict(chunk=0, split_min_nodes=64, pair_limit=4096),
    dict(chunk=0, split_min_nodes=16, pair_limit=4096),
    dict(chunk=0, split_min_nodes=512, pair_limit=4096),
    dict(chunk=64, split_min_nodes=64, pair_limit=4096),
    dict(chunk=4096, split_min_nodes=64, pair_limit=4096),
    dict(chunk=0, split_min_nodes=64, pair_limit=1024),
    dict(chunk=0, split_min_nodes=64, pair_limit=16384),
]


def _key(g: Graph, k: int, limit: int) -> str:
    return f"{g.fingerprint():016x}:k{k}:r{limit}"


def tune(g: Graph, k: int, result_limit: int = 200_000, grid=None, repeats: int = 2,
         cache_path: str | None = None) -> dict:
    """Best settings for enumerating g at k (device time per result, lower is
    better).  Returns {"settings": {...}, "ms": best_ms, "results": count,
    "cached": bool, "trials": [...]}."""
    cache_path = cache_path or os.environ.get("GMK_AUTOTUNE_CACHE")
    key = _key(g, k, result_limit)
    cache = {}
    if cache_path and os.path.exists(cache_path):
        with open(cache_path) as f:
            cache = json.load(f)
        if key in cache:
            return dict(cache[key], cached=True)
    trials = []
    for s in grid or DEFAULT_GRID:
        ms = []
        count = 0
        for _ in range(repeats):
            st = g.enumerate(k=k, result_limit=result_limit, schedule="batched", **s)
            ms.append(st.kernel_ms)
            count = st.count
        # per result: a setting that stops early on fewer results is not better
        trials.append({"settings": s, "ms": min(ms), "results": count,
                       "ms_per_result": min(ms) / max(1, count)})
    best = min(trials, key=lambda t: t["ms_per_result"])
    out = {"settings": best["settings"], "ms": best["ms"], "results": best["results"],
           "trials": trials, "tuned_at": time.time()}
    if cache_path:
        cache[key] = out
        tmp = cache_path + f".tmp{os.getpid()}"
        with open(tmp, "w") as f:
            json.dump(cache, f, indent=1)
        os.replace(tmp, cache_path)
    return dict(out, cached=False)
