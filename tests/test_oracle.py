"""CPU checks of the oracles themselves: the C oracle against the definition
(brute force) and against the golden summaries taken from the reference's
BPPivot, plus the graph format and converter-ordering helpers."""
import os

import numpy as np
import pytest

import oracle as O
from gmkbe_b200 import graphgen as gg
from conftest import golden_graph_path


def _tiny(seed):
    rng = np.random.default_rng(seed)
    nu, nv = int(rng.integers(1, 8)), int(rng.integers(1, 8))
    return gg.erdos_renyi(nu, nv, float(rng.uniform(0.15, 0.8)), seed)


@pytest.mark.parametrize("k", [1, 2, 3])
def test_oracle_equals_definition_on_tiny_graphs(k):
    checked = 0
    for seed in range(60):
        g = _tiny(seed)
        if g.n == 0 or g.n > 14 or g.n_left in (0, g.n):
            continue
        bf = sorted(O.brute_force(g, k))
        got = sorted(O.enumerate_oracle(g, k, collect=True).results)
        assert got == bf, (seed, k)
        checked += 1
    assert checked >= 30


@pytest.mark.parametrize("args,k", [((2, 3, 8, 2, 1), 2), ((3, 3, 9, 2, 2), 2),
                                    ((3, 2, 8, 3, 3), 3)])
def test_oracle_equals_definition_on_hub_graphs(args, k):
    # small members of the family the GPU filter-bitmap tests compare against
    g = gg.hubs_and_sparse(*args)
    assert g.n <= 15
    assert sorted(O.enumerate_oracle(g, k, collect=True).results) == sorted(O.brute_force(g, k))


def test_every_oracle_result_is_maximal():
    g = gg.read_graph_bin(golden_graph_path("southernwomen"))
    for k in (1, 2):
        res = O.enumerate_oracle(g, k, collect=True).results
        assert len(res) == len(set(res))
        for x, y in res[:: max(1, len(res) // 300)]:
            assert O.classify(g, k, x, y) == 2


@pytest.mark.parametrize("name,k", [("southernwomen", 1), ("southernwomen", 2), ("er60", 1),
                                    ("er60", 2), ("cl20k_sub", 1)])
def test_oracle_matches_golden(golden, name, k):
    case = next(c for c in golden["cases"] if c["graph"] == name and c["k"] == k)
    g = gg.read_graph_bin(golden_graph_path(name))
    st = O.enumerate_oracle(g, k)
    assert st.summary() == (case["count"], int(case["hash_sum"], 16), int(case["hash_xor"], 16))


def test_southernwomen_sets_file_matches_oracle():
    g = gg.read_graph_bin(golden_graph_path("southernwomen"))
    want = []
    with open(os.path.join(os.path.dirname(golden_graph_path("x")), "southernwomen_k1_sets.txt")) as f:
        for line in f:
            xs, ys = line.split("|")
            want.append((tuple(map(int, xs.split())), tuple(map(int, ys.split()))))
    got = sorted(O.enumerate_oracle(g, 1, collect=True).results)
    assert got == sorted(want) and len(got) == 1256


def test_bppivot_agrees_when_built():
    if not os.path.exists(O.bppivot_path()):
        pytest.skip("oracle/_ref/bppivot not built (needs the reference sources)")
    path = golden_graph_path("er60")
    g = gg.read_graph_bin(path)
    r = O.run_bppivot(path, 1, output=True)
    sets = list(O.parse_bppivot_sets(r["text"], g.n_left))
    assert O.set_summary(sets) == O.enumerate_oracle(g, 1).summary()


def test_limit_counts_exactly():
    g = gg.read_graph_bin(golden_graph_path("er60"))
    st = O.enumerate_oracle(g, 2, result_limit=1000)
    assert st.count == 1000 and st.truncated


def test_graph_bin_roundtrip(tmp_path):
    g = gg.chung_lu(300, 500, 2000, 2.1, 7, max_deg=50)
    p = str(tmp_path / "g.graph.bin")
    gg.write_graph_bin(g, p)
    h = gg.read_graph_bin(p)
    assert (h.offsets == g.offsets).all() and (h.adj == g.adj).all() and h.n_left == g.n_left


def test_truncated_graph_bin_rejected(tmp_path):
    g = gg.erdos_renyi(20, 20, 0.2, 3)
    p = str(tmp_path / "g.graph.bin")
    gg.write_graph_bin(g, p)
    raw = open(p, "rb").read()
    open(p, "wb").write(raw[:-8])
    with pytest.raises(ValueError):
        gg.read_graph_bin(p)


def test_converter_ordering_rules():
    # left vertices sort by (bucket(deg-2), deg-2, id) with unsigned wrap, so
    # degree-1 left vertices come last; right vertices by (bucket(deg-1), deg-1, id)
    left = np.array([0, 0, 0, 1, 2, 2, 3])
    right = np.array([0, 1, 2, 0, 0, 1, 2])
    g = gg.relabel(left, right)
    d = g.degree()
    dl = list(d[: g.n_left])
    assert dl == [2, 3, 1, 1]
    dr = list(d[g.n_left:])
    assert dr == sorted(dr)
    for v in range(g.n):
        row = g.nbrs(v)
        assert (np.diff(row.astype(np.int64)) > 0).all()


def test_parallel_edges_and_isolated_vertices_dropped():
    g = gg.relabel(np.array([5, 5, 9]), np.array([1, 1, 1]))
    assert g.n_left == 2 and g.n_right == 1 and g.n_edges == 2


def test_workload_definitions_are_seeded():
    a = gg.make_workload("er200")
    b = gg.make_workload("er200")
    assert (a.adj == b.adj).all()
    assert a.n_left == 200 and a.n_right == 200
