"""CPU checks of the C ABI library: it loads, exports every entry point that
include/gmk.h declares, hashes like the oracle, and fails loudly (never falls
back) when no GPU is present."""
import os
import re
import subprocess

import pytest

import gmkbe_b200 as G
import oracle as O
from conftest import ROOT, golden_graph_path

HEADER = os.path.join(ROOT, "include", "gmk.h")


def _declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(gmk_[a-z_]+)\s*\(", text)) - {"gmk_sink"})


def test_library_is_built_in_tree():
    assert os.path.exists(G.LIB_PATH), "run python -m gmkbe_b200.build"


def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", G.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s(gmk_\w+)", out))
    declared = _declared()
    assert declared, "no declarations parsed"
    missing = [s for s in declared if s not in exported]
    assert not missing, missing
    assert set(G.EXPORTS) == set(declared)


def test_abi_version_and_strerror():
    lib = G.load_library()
    assert lib.gmk_abi_version() == 3
    for code in list(range(0, -13, -1)) + [1]:
        assert lib.gmk_strerror(code).decode() != "unknown error"


def test_result_hash_matches_oracle():
    for x, y in [((0,), (5,)), ((1, 2, 3), (10, 11)), ((7,), (8, 9, 12, 15))]:
        assert G.result_hash(x, y) == O.result_hash(x, y)


def test_no_silent_cpu_path_without_gpu():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(G.GmkError) as e:
        G.Graph.load(golden_graph_path("er60"))
    assert e.value.code in (-11, -4)


def test_malformed_file_rejected_before_device_use(tmp_path):
    p = tmp_path / "bad.graph.bin"
    p.write_bytes(b"\x01\x00")
    with pytest.raises(G.GmkError) as e:
        G.Graph.load(str(p))
    assert e.value.code in (-3, -2)


def test_missing_file_is_io_error():
    with pytest.raises(G.GmkError) as e:
        G.Graph.load("/nonexistent/x.graph.bin")
    assert e.value.code == -2


def test_cli_usage():
    cli = os.path.join(ROOT, "gmkbe_b200", "gmk")
    assert os.path.exists(cli)
    p = subprocess.run([cli], capture_output=True, text=True)
    assert p.returncode == 2 and "usage" in p.stderr
