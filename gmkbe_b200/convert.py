"""Edge list -> `.graph.bin`, with the ordering of the reference's converter.

    python -m gmkbe_b200.convert -i edges.txt -o out[.graph.bin]   # gmk-convert, threaded
    gmkbe_b200/gmk-convert -i edges.txt -o out [--threads N]        # the same, directly

Reads text lines "u v ..." (lines starting with % or # are comments; a size
header line such as KONECT's must be removed first, as for the reference's
`graph_convert`, preprocess/graph_conver.cpp:819-850).  Parsing follows that
converter's scanner (graph_conver.cpp:433-441, :529-549): after skipping
blanks, a line's first two decimal digit runs are the edge (u, v) and the
rest of the line is ignored.  The output is byte-identical to the
converter's: per-side compaction, parallel edges removed, and each side
ordered by (log32 bucket of d', d', compact id) with d' = deg-2 (left) or
deg-1 (right) in wrapping 32-bit arithmetic (gmkbe_b200.graphgen.relabel).
"""
from __future__ import annotations

import argparse
import os
import re
import subprocess
import sys

import numpy as np

from . import graphgen as gg

_DIGITS = re.compile(rb"[0-9]+")


def parse_edge_list(data: bytes) -> tuple[np.ndarray, np.ndarray]:
    """(u, v) arrays of a text edge list, read as the reference's scanner does."""
    us: list[int] = []
    vs: list[int] = []
    p, n = 0, len(data)
    while p < n:
        c = data[p]
        if c in b"\n\r \t":
            p += 1
            continue
        if c in b"%#":
            e = data.find(b"\n", p)
            p = n if e < 0 else e
            continue
        vals = []
        for _ in range(2):
            m = _DIGITS.search(data, p)
            if m is None:
                vals.append(0)
                p = n
            else:
                vals.append(int(m.group()) & 0xFFFFFFFF)
                p = m.end()
        us.append(vals[0])
        vs.append(vals[1])
        e = data.find(b"\n", p)
        p = n if e < 0 else e
    return np.asarray(us, dtype=np.int64), np.asarray(vs, dtype=np.int64)


NATIVE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "gmk-convert")


def convert_native(infile: str, outfile: str, threads: int = 0, min_chunk: int = 0) -> str:
    """The multi-threaded C++ converter (gmk-convert, built by gmkbe_b200.build);
    same output as convert().  Returns the output path."""
    if not os.path.exists(NATIVE):
        raise FileNotFoundError(f"{NATIVE} not built; run `python -m gmkbe_b200.build`")
    cmd = [NATIVE, "-i", infile, "-o", outfile]
    if threads:
        cmd += ["--threads", str(threads)]
    if min_chunk:
        cmd += ["--min-chunk", str(min_chunk)]
    return subprocess.run(cmd, check=True, capture_output=True, text=True).stdout.strip()


def convert(infile: str, outfile: str) -> str:
    """Writes the `.graph.bin` of an edge-list file; returns the output path."""
    if not outfile.endswith(".graph.bin"):
        outfile += ".graph.bin"
    with open(infile, "rb") as f:
        u, v = parse_edge_list(f.read())
    gg.write_graph_bin(gg.relabel(u, v), outfile)
    return outfile


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("-i", required=True, help="edge list")
    ap.add_argument("-o", required=True, help="output prefix or .graph.bin path")
    ap.add_argument("--python", action="store_true", help="the single-threaded numpy port")
    a = ap.parse_args(argv)
    print(convert(a.i, a.o) if a.python or not os.path.exists(NATIVE) else convert_native(a.i, a.o))
    return 0


if __name__ == "__main__":
    sys.exit(main())
