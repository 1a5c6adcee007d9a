"""The Chung-Lu 100k x 300k (exponent 2.2, seed 3) and 500k x 1M (exponent
2.0, seed 4) workloads on the GPU.  Their complete result
sets are far too large to enumerate, so:
  * on the full graphs, the first 50 000 results of a record-mode run (and of a
    run that splits after every two nodes) are distinct, and every sampled one
    is a maximal k-biplex by the oracle's direct classifier;
  * on subgraphs induced by their first ids (as cl20k's exactness case is), complete count-mode enumerations -- the k >= 2 filter-bitmap
    kernel with in-launch sharing -- equal the C oracle's set summary."""
import numpy as np
import pytest

import gmkbe_b200 as G
import oracle as O
from gmkbe_b200 import graphgen as gg

pytestmark = pytest.mark.gpu

_cache = {}


def _graph(name):
    if name not in _cache:
        _cache[name] = gg.read_graph_bin(gg.cached_workload(name))
    return _cache[name]


@pytest.mark.parametrize("name,k", [("cl100k", 2), ("cl500k", 1), ("cl500k", 2), ("cl500k", 3)])
@pytest.mark.parametrize("split", [False, True])
def test_full_graph_results_are_distinct_and_maximal(name, k, split):
    h = _graph(name)
    kw = dict(split_min_nodes=2, chunk=1) if split else {}
    with G.Graph.load(gg.cached_workload(name)) as g:
        st = g.enumerate(k=k, result_limit=50_000, collect=True, **kw)
    res = st.results
    assert st.count == len(res) == 50_000 and st.truncated
    assert len(set(res)) == len(res)
    rng = np.random.default_rng(k + 10 * split)
    for i in rng.choice(len(res), size=40, replace=False):
        x, y = res[i]
        assert x and y and max(x) < h.n_left <= min(y)
        assert O.classify(h, k, x, y) == 2, (name, k, x, y)


@pytest.mark.parametrize("name,k,sub", [("cl100k", 1, (8_000, 24_000)), ("cl100k", 2, (4_000, 12_000)),
                                        ("cl500k", 2, (20_000, 40_000)), ("cl500k", 3, (10_000, 20_000))])
def test_family_subgraph_complete_runs_match_the_oracle(name, k, sub):
    h = gg.induced_prefix(_graph(name), *sub)
    want = O.enumerate_oracle(h, k).summary()
    with G.Graph.from_graph(h) as g:
        assert g.enumerate(k=k).summary() == want
        assert g.enumerate(k=k, schedule="ordered", task_cost=g.root_costs()).summary() == want
        assert g.enumerate(k=k, donate_min_nodes=1, bits_min_list=2).summary() == want
