"""Edge list -> `.graph.bin`, with the ordering of the reference's converter.

    python -m gmkbe_b200.convert -i edges.txt -o out[.graph.bin]

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
import re
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
    a = ap.parse_args(argv)
    print(convert(a.i, a.o))
    return 0


if __name__ == "__main__":
    sys.exit(main())
