"""The library's own sharding on one GPU: for N shards, gmk_enumerate with
shard = s, nshards = N (the longest-processing-time partition of the planned
tasks) run for every s combines (counts and h1 sums add, h2 xors) to the
golden summary, and the shards' result sets are disjoint.  Also: the device
cost proxy equals its restatement, explicit task lists (the recovery path)
cover the set, and the ordered schedule over the proxy costs is bit-exact."""
import numpy as np
import pytest

import gmkbe_b200 as G
from gmkbe_b200 import graphgen as gg
from gmkbe_b200.shard import MASK64, lpt_split
from conftest import golden_graph_path
from test_plan import proxy_cost

pytestmark = pytest.mark.gpu


def _want(golden, name, k):
    case = next(c for c in golden["cases"] if c["graph"] == name and c["k"] == k)
    return case["count"], int(case["hash_sum"], 16), int(case["hash_xor"], 16)


def _combine(stats):
    c = s = x = 0
    for st in stats:
        c += st.count
        s = (s + st.hash_sum) & MASK64
        x ^= st.hash_xor
    return c, s, x


@pytest.mark.parametrize("name,k", [("southernwomen", 2), ("er60", 2), ("er200", 1),
                                    ("cl20k_sub", 1)])
@pytest.mark.parametrize("nshards", [2, 3, 8])
def test_shards_combine_to_the_golden_summary(golden, name, k, nshards):
    with G.Graph.load(golden_graph_path(name)) as g:
        parts = [g.enumerate(k=k, shard=s, nshards=nshards) for s in range(nshards)]
    assert _combine(parts) == _want(golden, name, k)
    assert sum(1 for p in parts if p.count) >= min(2, nshards)   # the work is spread


@pytest.mark.parametrize("schedule", ["plain", "batched"])
def test_shard_result_sets_are_disjoint(golden, schedule):
    with G.Graph.load(golden_graph_path("southernwomen")) as g:
        sets = [set(g.enumerate(k=2, shard=s, nshards=3, schedule=schedule, collect=True).results)
                for s in range(3)]
    assert sum(len(p) for p in sets) == len(set().union(*sets)) == _want(golden, "southernwomen", 2)[0]


def test_device_cost_proxy_matches_its_restatement():
    for name in ("er200", "crime", "southernwomen"):
        h = gg.read_graph_bin(golden_graph_path(name))
        with G.Graph.from_graph(h) as g:
            assert np.array_equal(g.root_costs(), proxy_cost(h)), name


def test_explicit_task_lists_cover_the_set(golden):
    # the recovery path: a missing shard's tasks split among survivors and run
    # as explicit task lists
    h = gg.read_graph_bin(golden_graph_path("er200"))
    with G.Graph.from_graph(h) as g:
        cost = g.root_costs()
        parts = []
        for s in range(3):
            tasks = G.plan_tasks(h.n, h.n_left, cost, target_tasks=2000, nshards=3, shard=s)
            if s == 2:
                parts += [g.enumerate(k=1, tasks=lpt_split(tasks, 2, i)) for i in range(2)]
            else:
                parts.append(g.enumerate(k=1, tasks=tasks))
    assert _combine(parts) == _want(golden, "er200", 1)


@pytest.mark.parametrize("name,k", [("er200", 1), ("southernwomen", 3), ("crime", 1)])
def test_ordered_schedule_over_proxy_costs_is_exact(golden, name, k):
    with G.Graph.load(golden_graph_path(name)) as g:
        st = g.enumerate(k=k, schedule="ordered", task_cost=g.root_costs())
    assert st.summary() == _want(golden, name, k)
