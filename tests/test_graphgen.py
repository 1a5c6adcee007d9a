"""The seeded graph generators behind the fixtures, the benchmark workloads and
the training families (CPU only)."""
import numpy as np

from gmkbe_b200 import graphgen as gg
from conftest import golden_graph_path


def test_small_erdos_renyi_is_the_committed_fixture():
    # graphs up to DENSE_ER_PAIRS pairs draw every pair, as when er200 was made
    g = gg.erdos_renyi(200, 200, 0.05, 1)
    h = gg.read_graph_bin(golden_graph_path("er200"))
    assert np.array_equal(g.offsets, h.offsets) and np.array_equal(g.adj, h.adj)


def test_large_erdos_renyi_is_sampled_edge_by_edge():
    nu, nv, p = 6000, 4000, 0.002
    assert nu * nv > gg.DENSE_ER_PAIRS
    a = gg.erdos_renyi(nu, nv, p, 9)
    b = gg.erdos_renyi(nu, nv, p, 9)
    assert np.array_equal(a.adj, b.adj)                       # seeded
    mean, sd = nu * nv * p, np.sqrt(nu * nv * p * (1 - p))
    assert abs(a.n_edges - mean) < 5 * sd
    e = a.edges()
    assert len({(int(x), int(y)) for x, y in e}) == a.n_edges  # no parallel edges
    # degrees look binomial: U-side mean close to nv * p
    deg = a.degree()[: a.n_left].astype(np.float64)
    assert abs(deg.mean() - a.n_edges / a.n_left) < 1e-9
    assert abs(a.n_edges / nu - nv * p) < 0.5


def test_mixed_batch_at_its_stated_sizes_is_generated_quickly():
    gs, ks = gg.mixed_batch(4, 100)
    assert len(gs) == 4 and set(ks) <= {1, 2, 3}
    for g in gs:
        assert 0 < g.n_left < g.n and g.n_edges > 0
