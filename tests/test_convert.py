"""The edge-list converter port against the reference's own `graph_convert`
(compiled from preprocess/graph_conver.cpp by oracle/Makefile into
oracle/_ref): byte-identical .graph.bin on the reference's KONECT fixtures and
on random edge lists with duplicates, degree-1 vertices (whose deg-2 key wraps)
and comment lines."""
import os
import subprocess

import numpy as np
import pytest

from gmkbe_b200 import convert as C
from gmkbe_b200 import graphgen as gg
from conftest import ROOT, golden_graph_path
from oracle.refpath import ref_path

REF_CONVERT = os.path.join(ROOT, "oracle", "_ref", "graph_convert")
needs_ref = pytest.mark.skipif(not os.path.exists(REF_CONVERT),
                               reason="reference converter not built (no reference sources)")


def _ref_convert(txt: str, prefix: str) -> bytes:
    subprocess.run([REF_CONVERT, "-i", txt, "-o", prefix], check=True, capture_output=True)
    with open(prefix + ".graph.bin", "rb") as f:
        return f.read()


def _ours(txt: str, prefix: str) -> bytes:
    with open(C.convert(txt, prefix), "rb") as f:
        return f.read()


def test_parser_follows_reference_scanner():
    u, v = C.parse_edge_list(b"% c\n# d\n 3 4 9\n\t5\t6\r\n7 8")
    assert u.tolist() == [3, 5, 7] and v.tolist() == [4, 6, 8]


def test_golden_graphs_are_converter_ordered():
    # the committed fixtures were written through the same ordering
    g = gg.read_graph_bin(golden_graph_path("southernwomen"))
    e = g.edges()
    again = gg.relabel(e[:, 0], e[:, 1] - g.n_left)
    assert np.array_equal(again.offsets, g.offsets) and np.array_equal(again.adj, g.adj)


@needs_ref
@pytest.mark.parametrize("fixture", ["opsahl_southernwomen", "moreno_crime", "opsahl_ucforum"])
def test_konect_fixtures_byte_identical(tmp_path, fixture):
    src = ref_path("baselines", "MaximalBiPlex", "datas", fixture + ".txt")
    if not os.path.exists(src):
        pytest.skip("reference fixtures absent")
    lines = open(src).read().splitlines()[1:]             # size header removed
    txt = tmp_path / "e.txt"
    txt.write_text("\n".join(lines) + "\n")
    assert _ours(str(txt), str(tmp_path / "ours")) == _ref_convert(str(txt), str(tmp_path / "ref"))


@needs_ref
@pytest.mark.parametrize("seed", range(6))
def test_random_edge_lists_byte_identical(tmp_path, seed):
    rng = np.random.default_rng(seed)
    m = int(rng.integers(1, 3000))
    u = rng.integers(0, int(rng.integers(1, 400)), m)
    v = rng.integers(0, int(rng.integers(1, 900)), m)
    u = np.concatenate([u, u[: m // 5]])                  # parallel edges
    v = np.concatenate([v, v[: m // 5]])
    rows = [f"{a} {b}" for a, b in zip(u, v)]
    rows.insert(len(rows) // 2, "% a comment")
    txt = tmp_path / "e.txt"
    txt.write_text("\n".join(rows) + "\n")
    assert _ours(str(txt), str(tmp_path / "ours")) == _ref_convert(str(txt), str(tmp_path / "ref"))
