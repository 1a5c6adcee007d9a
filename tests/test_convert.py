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


# ---- the multi-threaded C++ converter (gmk-convert)

needs_native = pytest.mark.skipif(not os.path.exists(C.NATIVE), reason="gmk-convert not built")


def _ref_convert_threads(txt: str, prefix: str, threads: int) -> bytes:
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    subprocess.run([REF_CONVERT, "-i", txt, "-o", prefix], check=True, capture_output=True, env=env)
    with open(prefix + ".graph.bin", "rb") as f:
        return f.read()


def _native(txt: str, prefix: str, threads: int, min_chunk: int = 0) -> bytes:
    with open(C.convert_native(txt, prefix, threads=threads, min_chunk=min_chunk), "rb") as f:
        return f.read()


@needs_ref
@needs_native
@pytest.mark.parametrize("fixture", ["opsahl_southernwomen", "moreno_crime", "opsahl_ucforum"])
def test_native_konect_fixtures_byte_identical(tmp_path, fixture):
    src = ref_path("baselines", "MaximalBiPlex", "datas", fixture + ".txt")
    if not os.path.exists(src):
        pytest.skip("reference fixtures absent")
    txt = tmp_path / "e.txt"
    txt.write_text("\n".join(open(src).read().splitlines()[1:]) + "\n")
    want = _ref_convert(str(txt), str(tmp_path / "ref"))
    for threads in (1, 3, 8):
        assert _native(str(txt), str(tmp_path / "n"), threads, min_chunk=64) == want


@needs_ref
@needs_native
@pytest.mark.parametrize("seed", range(8))
def test_native_random_edge_lists_byte_identical(tmp_path, seed):
    # comment lines, parallel edges, sparse id ranges, trailing fields and CRs;
    # small chunks so that several threads and the boundary repair run
    rng = np.random.default_rng(100 + seed)
    m = int(rng.integers(1, 6000))
    u = rng.integers(0, int(rng.integers(1, 500)), m)
    v = rng.integers(0, int(rng.integers(1, 900)), m)
    if seed % 3 == 2:
        u = u * 1000003 + 7
    u = np.concatenate([u, u[: m // 5]])
    v = np.concatenate([v, v[: m // 5]])
    rows = [f"{a} {b}" for a, b in zip(u, v)]
    for i in range(0, len(rows), 97):
        rows.insert(i, "% comment" if i % 2 else "#another")
    if seed % 2:
        rows = [r + " 9 extra\r" if i % 5 == 0 else r for i, r in enumerate(rows)]
    txt = tmp_path / "e.txt"
    txt.write_text("\n".join(rows) + "\n")
    want = _ref_convert(str(txt), str(tmp_path / "ref"))
    for threads, chunk in ((1, 0), (4, 97), (16, 31)):
        assert _native(str(txt), str(tmp_path / "n"), threads, chunk) == want, (threads, chunk)


@needs_ref
@needs_native
def test_native_reads_split_records_like_the_single_threaded_reference(tmp_path):
    # a line with one number takes the second from the next line; the
    # reference cuts such records at its thread chunks' ends, so its own output
    # depends on its thread count -- ours equals its one-thread output, at any
    # thread count and chunk size (the boundary repair re-reads them whole)
    rng = np.random.default_rng(7)
    u = rng.integers(0, 300, 4000)
    v = rng.integers(0, 800, 4000)
    rows = [f"{a}\n{b}" if i % 3 == 0 else f"{a} {b}" for i, (a, b) in enumerate(zip(u, v))]
    txt = tmp_path / "e.txt"
    txt.write_text("\n".join(rows) + "\n")
    want = _ref_convert_threads(str(txt), str(tmp_path / "ref"), 1)
    assert open(C.convert(str(txt), str(tmp_path / "py")), "rb").read() == want
    for threads, chunk in ((1, 0), (2, 50), (8, 13), (32, 7)):
        assert _native(str(txt), str(tmp_path / "n"), threads, chunk) == want, (threads, chunk)


@needs_native
def test_native_empty_and_comment_only_inputs(tmp_path):
    for text in ("", "% only\n# comments\n", "\n\n  \t\n"):
        txt = tmp_path / "e.txt"
        txt.write_text(text)
        assert _native(str(txt), str(tmp_path / "n"), 4, 1) == \
            open(C.convert(str(txt), str(tmp_path / "p")), "rb").read()
