"""The CLI's time file (<dir>/<stem>.gpu<k>.json, the reference's
include/timer.cuh:85-185), on the CPU: gmkbe_b200/csrc/time_file.h compiled
alone with g++ into a small driver that reads a file, sets one entry and
writes it back -- the CLI's two steps.  Other entries survive, unreadable
files start empty, the output is JSON, and the path is named for the graph."""
import json
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

DRIVER = r"""
#include "time_file.h"
#include <cstdio>
int main(int argc, char** argv) {
    if (argc == 3) {   // path of the time file for graph argv[1], k argv[2]
        std::printf("%s\n", gmk_cli::time_file_path(argv[1], (uint32_t)std::atoi(argv[2])).c_str());
        return 0;
    }
    // argv: file k limit value
    gmk_cli::TimeTable t = gmk_cli::read_time_table(argv[1]);
    t[argv[2]][argv[3]] = argv[4];
    gmk_cli::write_time_table(argv[1], t);
    return 0;
}
"""


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("tf")
    src = d / "drv.cpp"
    src.write_text(DRIVER)
    exe = d / "drv"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "gmkbe_b200", "csrc"),
                    str(src), "-o", str(exe)], check=True)
    return str(exe)


def _set(driver, path, k, limit, value):
    subprocess.run([driver, str(path), str(k), str(limit), value], check=True)
    return json.loads(path.read_text())


def test_entries_are_set_and_merged(driver, tmp_path):
    f = tmp_path / "g.gpu1.json"
    assert _set(driver, f, 1, 100, "18000000") == {"1": {"100": 18000000}}
    assert _set(driver, f, 1, 100, "12.5") == {"1": {"100": 12.5}}
    assert _set(driver, f, 2, 7, "3") == {"1": {"100": 12.5}, "2": {"7": 3}}
    assert _set(driver, f, 1, 1000, "1e-3") == {"1": {"100": 12.5, "1000": 0.001}, "2": {"7": 3}}


def test_reads_the_reference_layout(driver, tmp_path):
    # the reference writes nlohmann's dump(4): four-space indents, one key a line
    f = tmp_path / "g.gpu2.json"
    f.write_text(json.dumps({"2": {"1000000": 38666.0, "5": 18000000}}, indent=4))
    assert _set(driver, f, 2, 10, "1.25") == {"2": {"1000000": 38666.0, "5": 18000000, "10": 1.25}}
    text = f.read_text()
    assert text.startswith("{\n    \"2\": {\n        \"10\": 1.25,")


@pytest.mark.parametrize("junk", ["", "not json", "{\"1\": [1, 2]}", "{\"1\": {\"2\": }"])
def test_unreadable_files_start_empty(driver, tmp_path, junk):
    f = tmp_path / "g.gpu1.json"
    f.write_text(junk)
    assert _set(driver, f, 1, 5, "2") == {"1": {"5": 2}}


def test_path_is_named_for_the_graph(driver):
    def path(graph, k):
        return subprocess.run([driver, graph, str(k)], capture_output=True, text=True,
                              check=True).stdout.strip()
    assert path("/data/x/cl20k.graph.bin", 1) == "/data/x/cl20k.graph.gpu1.json"
    assert path("sw.bin", 3) == "sw.gpu3.json"
    assert path("dir/noext", 2) == "dir/noext.gpu2.json"
