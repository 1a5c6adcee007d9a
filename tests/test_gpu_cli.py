"""The drop-in executable `gmk` (same -f/-k/-r/-q/-d flags as the reference's
gmkbpe, src/main.cu:1719-1775) on the GPU: its `-q 1` result lines have the
reference's format (include/output.cuh:102-145: "Result <n>: X: x1 x2 | Y:
y1 y2 "), are numbered 1..N, and hold exactly BPPivot's result set; the header
and `Running Time:` lines follow src/main.cu:1593 and :1709; -r stops at the
limit; and the buffered writer's rate is reported."""
import os
import re
import subprocess

import pytest

from conftest import GOLDEN, ROOT, golden_graph_path

pytestmark = pytest.mark.gpu

CLI = os.path.join(ROOT, "gmkbe_b200", "gmk")
RESULT = re.compile(r"^Result (\d+): X:((?: \d+)+) \| Y: ((?:\d+ )+)$")
HEADER = re.compile(r"^Graph size: (\d+), edge num: (\d+), bipartite index: (\d+), k = (\d+), "
                    r"theta = 1$")
RUNNING = re.compile(r"^Running Time: (\d+(?:\.\d+)?(?:e[-+]?\d+)?) ms$")


def _run(*args):
    # --no-time-file: no side file next to the committed fixtures
    p = subprocess.run([CLI, *args, "--no-time-file"], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    return p.stdout.splitlines()


def _parse(lines):
    results, other = [], []
    for line in lines:
        m = RESULT.match(line)
        if m:
            results.append((int(m.group(1)), tuple(int(v) for v in m.group(2).split()),
                            tuple(int(v) for v in m.group(3).split())))
        else:
            other.append(line)
    return results, other


def test_result_lines_match_the_reference_format_and_set():
    lines = _run("-f", golden_graph_path("southernwomen"), "-k", "1", "-q", "1", "--all")
    results, other = _parse(lines)
    assert re.match(r"^Using GPU: .+, GPU id: 0$", other[0]), other[0]
    assert HEADER.match(other[1]), other[1]
    assert RUNNING.match(other[-1]), other[-1]
    assert len(other) == 3, other
    assert [n for n, _, _ in results] == list(range(1, len(results) + 1))
    got = {(x, y) for _, x, y in results}
    want = set()
    with open(os.path.join(GOLDEN, "southernwomen_k1_sets.txt")) as f:
        for line in f:
            xs, ys = line.split("|")
            want.add((tuple(int(v) for v in xs.split()), tuple(int(v) for v in ys.split())))
    assert len(results) == len(got) == 1256
    assert got == want
    # ids ascending within each side, X in U and Y in V
    n, _, nl, _ = (int(v) for v in HEADER.match(other[1]).groups())
    for _, x, y in results:
        assert list(x) == sorted(x) and list(y) == sorted(y)
        assert x[-1] < nl <= y[0] and y[-1] < n


def test_result_limit_and_quiet_mode():
    results, other = _parse(_run("-f", golden_graph_path("southernwomen"), "-k", "2", "-q", "1",
                                 "-r", "100"))
    assert len(results) == 100 and len({(x, y) for _, x, y in results}) == 100
    results, other = _parse(_run("-f", golden_graph_path("southernwomen"), "-k", "2", "-r", "100"))
    assert results == [] and RUNNING.match(other[-1])


def test_million_line_output_rate(golden, tmp_path):
    # er200, k = 1: 1 891 002 lines; the set summary of the printed run equals
    # the golden one and the writer's lines per second are reported
    case = next(c for c in golden["cases"] if c["graph"] == "er200" and c["k"] == 1)
    out = tmp_path / "out.txt"
    with open(out, "w") as f:
        p = subprocess.run([CLI, "-f", golden_graph_path("er200"), "-k", "1", "-q", "1", "--all",
                            "--stats", "--no-time-file"], stdout=f, stderr=subprocess.PIPE,
                           text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    tail = subprocess.run(["tail", "-n", "2", str(out)], capture_output=True, text=True).stdout
    stats = dict(zip(*[iter(tail.splitlines()[-1].split())] * 2))
    assert int(stats["results"]) == int(stats["lines"]) == case["count"]
    assert int(stats["hash_sum"], 16) == int(case["hash_sum"], 16)
    assert int(stats["hash_xor"], 16) == int(case["hash_xor"], 16)
    wc = subprocess.run(["wc", "-l", str(out)], capture_output=True, text=True).stdout.split()[0]
    assert int(wc) == case["count"] + 4   # + the GPU line, header, running time, stats
    print(f"gmk -q 1: {stats['lines']} lines, {float(stats['lines_per_s']) / 1e6:.2f} M lines/s "
          f"(wall {stats['wall_ms']} ms)")


def test_progress_marks_and_time_file(tmp_path):
    # The reference reports "Output <n>, cost Time: <ms> ms" on stderr at 10^i
    # results and at the limit (src/main.cu:1752-1760, include/output.cuh:350-372)
    # and keeps the time to the limit in <stem>.gpu<k>.json next to the graph
    # (include/timer.cuh:85-185): 5 h until the limit is reached, other
    # entries of the file kept.
    import json
    import shutil
    graph = tmp_path / "sw.graph.bin"
    shutil.copy(golden_graph_path("southernwomen"), graph)
    side = tmp_path / "sw.graph.gpu1.json"   # the stem drops the last extension only
    side.write_text(json.dumps({"2": {"5": 1.5}}))
    p = subprocess.run([CLI, "-f", str(graph), "-k", "1", "-r", "100", "-q", "1"],
                       capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    marks = re.findall(r"^Output (\d+), cost Time: ([0-9.e+-]+) ms$", p.stderr, re.M)
    assert [int(n) for n, _ in marks] == [1, 10, 100]
    table = json.loads(side.read_text())
    assert table["2"] == {"5": 1.5}
    assert 0 < table["1"]["100"] < 18_000_000
    # count mode, limit above the total (1 256 results): the final mark only,
    # and the 5 h placeholder stays for that limit
    p = subprocess.run([CLI, "-f", str(graph), "-k", "1", "-r", "1000000"],
                       capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    assert re.findall(r"^Output (\d+),", p.stderr, re.M) == ["1256"]
    table = json.loads(side.read_text())
    assert table["1"]["1000000"] == 18_000_000 and table["1"]["100"] < 18_000_000
