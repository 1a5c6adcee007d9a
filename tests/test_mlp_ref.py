"""The CPU restatement of the subtree-size model (the oracle of the GPU MLP
kernels) against central finite differences, and the ranking / scheduling
helpers of gmkbe_b200.learned."""
import numpy as np

from oracle import mlp_ref
from gmkbe_b200 import learned as L


def test_reference_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.3, mlp_ref.NP)
    x = rng.uniform(0, 2, (9, 16))
    y = rng.normal(0, 1, 9)
    _, g = mlp_ref.loss_and_gradient(p, x, y, fp16=False)
    for i in rng.choice(mlp_ref.NP, 60, replace=False):
        e = np.zeros(mlp_ref.NP)
        e[i] = 1e-6
        lp, _ = mlp_ref.loss_and_gradient(p + e, x, y, fp16=False)
        lm, _ = mlp_ref.loss_and_gradient(p - e, x, y, fp16=False)
        assert abs((lp - lm) / 2e-6 - g[i]) <= 1e-6 + 1e-5 * abs(g[i])


def test_spearman_and_relative_error():
    assert L.spearman([1, 2, 3, 4], [10, 20, 30, 40]) == 1.0
    assert L.spearman([1, 2, 3, 4], [4, 3, 2, 1]) == -1.0
    assert abs(L.spearman([1, 1, 2], [5, 5, 9]) - 1.0) < 1e-12
    assert L.mean_relative_error([2, 4], [1, 4]) == 0.5


def test_longest_first_order_shortens_the_makespan():
    costs = np.array([1, 1, 1, 1, 1, 1, 1, 1, 8], float)
    ident = L.makespan(costs, np.arange(9), 4)       # the big task starts last
    lpt = L.makespan(costs, np.argsort(-costs), 4)   # the big task starts first
    assert ident == 10 and lpt == 8
