"""The task planner (gmk_plan_tasks, host-only: no GPU needed) that the
ordered schedule, sharding and shard recovery use: chunks cover every root's
first-level V children exactly once, shards partition the plan, the
longest-processing-time assignment is balanced, and the ctypes mirror's
structs match include/gmk.h."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import gmkbe_b200 as G
from gmkbe_b200 import graphgen as gg
from gmkbe_b200.api import _Opts, _Stats, _Task
from gmkbe_b200.shard import lpt_split
from conftest import ROOT, golden_graph_path


def proxy_cost(g) -> np.ndarray:
    """1 + sum over x's neighbours y of |N(y) above x| (gmk_root_costs)."""
    out = np.ones(g.n_left, np.float64)
    for x in range(g.n_left):
        for y in g.nbrs(x):
            out[x] += int((g.nbrs(int(y)) > x).sum())
    return out.astype(np.float32)


def _key(t):
    return int(t["root"]), int(t["first"]), int(t["last"])


@pytest.mark.parametrize("name", ["er200", "crime", "southernwomen"])
@pytest.mark.parametrize("target", [1, 100, 5000])
def test_chunks_cover_each_root_once(name, target):
    g = gg.read_graph_bin(golden_graph_path(name))
    cost = proxy_cost(g)
    plan = G.plan_tasks(g.n, g.n_left, cost, target_tasks=target)
    assert set(plan["root"].tolist()) == set(range(g.n_left))
    for r in range(g.n_left):
        t = sorted(_key(x) for x in plan[plan["root"] == r])
        assert t[0][1] == g.n_left and t[-1][2] == g.n
        assert all(a[2] == b[1] for a, b in zip(t, t[1:]))          # contiguous, disjoint
        assert all(x[2] - x[1] >= min(16, g.n - g.n_left) for x in t[:-1])
    assert np.all(np.diff(plan["cost"]) <= 0)                       # largest first
    if target == 1:
        assert len(plan) == g.n_left


@pytest.mark.parametrize("nshards", [2, 3, 8])
def test_shards_partition_the_plan_and_balance(nshards):
    g = gg.read_graph_bin(golden_graph_path("crime"))
    cost = proxy_cost(g)
    full = G.plan_tasks(g.n, g.n_left, cost, target_tasks=400)
    parts = [G.plan_tasks(g.n, g.n_left, cost, target_tasks=400, nshards=nshards, shard=s)
             for s in range(nshards)]
    keys = [set(map(_key, p)) for p in parts]
    assert sum(len(k) for k in keys) == len(full)
    assert set().union(*keys) == set(map(_key, full))
    loads = [float(p["cost"].astype(np.float64).sum()) for p in parts]
    total = float(full["cost"].astype(np.float64).sum())
    assert max(loads) <= total / nshards + float(full["cost"].max()) + 1e-3


def test_root_range_selects_positions_of_the_cost_order():
    g = gg.read_graph_bin(golden_graph_path("er60"))
    cost = proxy_cost(g)
    order = np.argsort(-cost.astype(np.float64), kind="stable")
    a = G.plan_tasks(g.n, g.n_left, cost, root_begin=0, root_end=7, target_tasks=1)
    b = G.plan_tasks(g.n, g.n_left, cost, root_begin=7, target_tasks=1)
    assert sorted(a["root"].tolist()) == sorted(order[:7].tolist())
    assert sorted(b["root"].tolist()) == sorted(order[7:].tolist())


def test_plain_planning_keeps_one_task_per_root():
    g = gg.read_graph_bin(golden_graph_path("er200"))
    plan = G.plan_tasks(g.n, g.n_left, proxy_cost(g), target_tasks=10 ** 6, max_chunks=1)
    assert len(plan) == g.n_left and np.all(plan["first"] == g.n_left) and np.all(plan["last"] == g.n)


def test_lpt_split_partitions_a_shard():
    g = gg.read_graph_bin(golden_graph_path("crime"))
    shard = G.plan_tasks(g.n, g.n_left, proxy_cost(g), target_tasks=300, nshards=3, shard=1)
    parts = [lpt_split(shard, 2, i) for i in range(2)]
    assert sorted(map(_key, np.concatenate(parts))) == sorted(map(_key, shard))


def test_invalid_plan_arguments_raise():
    with pytest.raises(G.GmkError):
        G.plan_tasks(10, 4, np.ones(4, np.float32), nshards=2, shard=2)
    with pytest.raises(G.GmkError):
        G.plan_tasks(10, 4, np.ones(4, np.float32), root_begin=3, root_end=2)


def test_ctypes_structs_match_the_header(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text('#include <stdio.h>\n#include "gmk.h"\n'
                   'int main(void){printf("%zu %zu %zu\\n", sizeof(gmk_opts), sizeof(gmk_stats),'
                   ' sizeof(gmk_task)); return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True)
    sizes = tuple(int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True,
                                                 check=True).stdout.split())
    assert sizes == (ctypes.sizeof(_Opts), ctypes.sizeof(_Stats), ctypes.sizeof(_Task))


def _plan_restated(n, nl, cost, target):
    """The planner restated: roots by cost, largest first (stable); root r cut
    into m = clamp(ceil(cost / unit), 1, (n - nl) // 16) equal chunks, unit =
    total cost / target; all tasks stably sorted by their per-task cost
    float32(cost / m), largest first."""
    nv = n - nl
    c64 = np.maximum(cost.astype(np.float64), 0.0)
    roots = np.argsort(-cost, kind="stable")
    unit = c64[roots].sum() / max(1, target)
    wide = max(1, nv // 16)
    tasks = []
    for r in roots:
        m = int(max(1.0, min(np.ceil(c64[r] / unit) if unit > 0 else 1.0, float(wide))))
        width = (nv + m - 1) // m
        for i in range(m):
            first = nl + i * width
            if first >= n:
                break
            tasks.append((int(r), first, min(n, first + width), float(np.float32(c64[r] / m))))
    tasks.sort(key=lambda t: -t[3])     # stable
    return tasks


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_plan_order_is_a_stable_sort_of_the_tasks_by_cost(seed):
    # The planner sorts roots by per-task cost instead of sorting every task;
    # a root's chunks share one cost, so the order must be exactly that of a
    # stable sort of all tasks (ties included: costs are rounded here).
    rng = np.random.default_rng(seed)
    nl, nv = int(rng.integers(50, 400)), int(rng.integers(40, 900))
    cost = np.round(np.exp(rng.uniform(0, 6, nl)) / 20).astype(np.float32)
    for target in (1, 37, 2000):
        plan = G.plan_tasks(nl + nv, nl, cost, target_tasks=target)
        want = _plan_restated(nl + nv, nl, cost, target)
        got = [(int(t["root"]), int(t["first"]), int(t["last"]), float(t["cost"])) for t in plan]
        assert got == want, (seed, target)
