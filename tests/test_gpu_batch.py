"""Mixed batch in one launch (gmk_enumerate_batch): uneven graphs with their own
k share one device work queue; every graph's result set must be bit-exact
with its own single-graph run and, where small enough, with the oracle."""
import numpy as np
import pytest

import gmkbe_b200 as G
import oracle as O
from gmkbe_b200 import graphgen as gg
from gmkbe_b200 import learned as L

pytestmark = pytest.mark.gpu


def _batch(n=16, seed0=100):
    gs, ks = gg.mixed_batch(n, seed0, size_lo=6, size_hi=30, deg_lo=1.5, deg_hi=3.0)
    keep = [(g, k) for g, k in zip(gs, ks) if g.n_left not in (0, g.n)]
    return [g for g, _ in keep], [k for _, k in keep]


@pytest.mark.parametrize("schedule", ["batched", "plain"])
def test_batch_matches_single_runs_and_oracle(schedule):
    gs, ks = _batch()
    dgs = [G.Graph.from_graph(g) for g in gs]
    try:
        got = G.enumerate_batch(dgs, ks, schedule=schedule)
        for g, dg, k, st in zip(gs, dgs, ks, got):
            single = dg.enumerate(k=k, schedule="plain").summary()
            assert st.summary() == single
            if single[0] < 200_000:
                assert st.summary() == O.enumerate_oracle(g, k).summary()
        assert len({st.rounds for st in got}) == 1       # one run of launches
    finally:
        for dg in dgs:
            dg.close()


def test_batch_with_learned_order_and_forced_splits():
    gs, ks = _batch(12, 300)
    dgs = [G.Graph.from_graph(g) for g in gs]
    try:
        model = L.SubtreeModel(seed=3)
        xs = np.concatenate([L.root_features(dg, k) for dg, k in zip(dgs, ks)])
        ys = np.concatenate([L.target(L.subtree_nodes(dg, k)) for dg, k in zip(dgs, ks)])
        model.train(xs, ys, epochs=200)
        costs = [L.predicted_costs(model, dg, k) for dg, k in zip(dgs, ks)]
        got = G.enumerate_batch(dgs, ks, schedule="ordered", task_costs=costs, split_min_nodes=2,
                                chunk=1)
        for dg, k, st in zip(dgs, ks, got):
            assert st.summary() == dg.enumerate(k=k, schedule="plain").summary()
    finally:
        for dg in dgs:
            dg.close()


def test_batch_rejects_unsupported_options():
    g = gg.read_graph_bin(__import__("conftest").golden_graph_path("er60"))
    with G.Graph.from_graph(g) as dg:
        with pytest.raises(G.GmkError):
            G.enumerate_batch([dg, dg], [1, 1])        # the same graph twice
        lib = G.load_library()
        assert lib.gmk_enumerate_batch(None, 0, None, None, None, None, None) == -1


def test_per_graph_caps_stop_each_graph_alone():
    # graph i stops at its own cap; graphs whose full set is below their cap
    # are enumerated completely and stay bit-exact
    gs, ks = _batch(16, 500)
    dgs = [G.Graph.from_graph(g) for g in gs]
    try:
        full = [dg.enumerate(k=k, schedule="plain") for dg, k in zip(dgs, ks)]
        caps = [max(1, f.count // 3) if i % 2 else f.count + 10 for i, f in enumerate(full)]
        got = G.enumerate_batch(dgs, ks, limits=caps)
        for f, cap, st in zip(full, caps, got):
            if cap > f.count:
                assert st.summary() == f.summary() and not st.truncated
            else:
                assert st.count == cap and st.truncated
    finally:
        for dg in dgs:
            dg.close()


def test_stated_size_mixed_batch_with_caps():
    # the mixed batch at its stated sizes (|U|, |V| log-uniform in [1k, 50k],
    # average degree 5-30, half Erdos-Renyi and half Chung-Lu, k in {1,2,3};
    # 16 of the 64 seeds): every graph has far more maximal k-biplexes than
    # the cap, so each must stop at exactly its cap, as its own capped run does
    gs, ks = gg.mixed_batch(16, 100)
    cap = 50_000
    dgs = [G.Graph.from_graph(g) for g in gs]
    try:
        got = G.enumerate_batch(dgs, ks, limits=[cap] * len(dgs))
        for dg, k, st in zip(dgs, ks, got):
            single = dg.enumerate(k=k, result_limit=cap)
            assert st.count == single.count
            assert st.truncated == single.truncated
        assert sum(st.count for st in got) > 0
    finally:
        for dg in dgs:
            dg.close()
