"""ctypes front end of the C oracle, the BPPivot runner and a brute-force check.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU legs, never by the gmkbe_b200 package.
"""
from __future__ import annotations

import ctypes
import itertools
import os
import re
import subprocess
import tempfile
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
MASK64 = (1 << 64) - 1


def liboracle_path() -> str:
    return os.path.join(HERE, "liboracle.so")


def bppivot_path() -> str:
    return os.path.join(HERE, "_ref", "bppivot")


def refgpu_path() -> str:
    """The reference's own GPU enumerator (make -C oracle refgpu)."""
    return os.path.join(HERE, "_ref", "gmkbpe")


# ----------------------------------------------------------------------------- hashing

def _mix64(z: int) -> int:
    z = (z + 0x9E3779B97F4A7C15) & MASK64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
    return z ^ (z >> 31)


def result_hash(x, y) -> tuple[int, int]:
    """(h1, h2) of one result; same definition as oracle_result_hash() in C and
    gmk_result_hash() in the CUDA library."""
    a = b = 0
    for v in list(x) + list(y):
        e = _mix64((int(v) * 2 + 1) & MASK64)
        a = (a + e) & MASK64
        b = (b + _mix64(e ^ 0x5851F42D4C957F2D)) & MASK64
    nx, ny = len(x), len(y)
    h1 = _mix64((a + nx * 0x100000001B3 + ny) & MASK64)
    h2 = _mix64(b ^ ((nx << 32) | ny))
    return h1, h2


def set_summary(results) -> tuple[int, int, int]:
    """(count, wrapping sum of h1, xor of h2) over an iterable of (X, Y)."""
    c = s = xr = 0
    for x, y in results:
        h1, h2 = result_hash(x, y)
        c += 1
        s = (s + h1) & MASK64
        xr ^= h2
    return c, s, xr


# ----------------------------------------------------------------------------- C oracle

class _Stats(ctypes.Structure):
    _fields_ = [("count", ctypes.c_uint64), ("hash_sum", ctypes.c_uint64),
                ("hash_xor", ctypes.c_uint64), ("nodes", ctypes.c_uint64),
                ("truncated", ctypes.c_int)]


@dataclass
class OracleStats:
    count: int
    hash_sum: int
    hash_xor: int
    nodes: int
    truncated: bool
    results: list | None = None

    def summary(self) -> tuple[int, int, int]:
        return self.count, self.hash_sum, self.hash_xor


_SINK = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32),
                         ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32), ctypes.c_uint32)
_lib = None


def _load():
    global _lib
    if _lib is None:
        path = liboracle_path()
        if not os.path.exists(path):
            subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
        lib = ctypes.CDLL(path)
        lib.oracle_enumerate.restype = ctypes.c_int
        lib.oracle_enumerate.argtypes = [
            ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32), ctypes.c_uint32,
            ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, _SINK, ctypes.c_void_p,
            ctypes.POINTER(_Stats)]
        lib.oracle_enumerate_shard.restype = ctypes.c_int
        lib.oracle_enumerate_shard.argtypes = [
            ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32), ctypes.c_uint32,
            ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32,
            _SINK, ctypes.c_void_p, ctypes.POINTER(_Stats)]
        lib.oracle_classify.restype = ctypes.c_int
        lib.oracle_classify.argtypes = [
            ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32), ctypes.c_uint32,
            ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32), ctypes.c_uint32,
            ctypes.POINTER(ctypes.c_uint32), ctypes.c_uint32]
        _lib = lib
    return _lib


def _csr32(g):
    off = np.ascontiguousarray(g.offsets, dtype=np.uint32)
    adj = np.ascontiguousarray(g.adj, dtype=np.uint32)
    if adj.size == 0:
        adj = np.zeros(1, np.uint32)
    P = ctypes.POINTER(ctypes.c_uint32)
    return off, adj, off.ctypes.data_as(P), adj.ctypes.data_as(P)


def enumerate_oracle(g, k: int, result_limit: int = 0, collect: bool = False,
                     shard: int = 0, nshards: int = 1) -> OracleStats:
    """All maximal k-biplexes of g (or, with nshards > 1, those whose smallest U
    vertex x has x % nshards == shard)."""
    lib = _load()
    off, adj, poff, padj = _csr32(g)
    out = []
    if collect:
        def sink(_u, xp, nx, yp, ny):
            out.append((tuple(xp[i] for i in range(nx)), tuple(yp[i] for i in range(ny))))
            return 0
        cb = _SINK(sink)
    else:
        cb = _SINK(0)
    st = _Stats()
    rc = lib.oracle_enumerate_shard(poff, padj, g.n, g.n_left, k, result_limit, shard, nshards,
                                    cb, None, ctypes.byref(st))
    if rc != 0:
        raise ValueError(f"oracle_enumerate failed ({rc}); n={g.n} (max 16384), k={k}")
    return OracleStats(st.count, st.hash_sum, st.hash_xor, st.nodes, bool(st.truncated),
                       out if collect else None)


def classify(g, k: int, x, y) -> int:
    """0 = not a k-biplex, 1 = k-biplex but not maximal, 2 = maximal."""
    lib = _load()
    off, adj, poff, padj = _csr32(g)
    xa = np.ascontiguousarray(list(x) or [0], dtype=np.uint32)
    ya = np.ascontiguousarray(list(y) or [0], dtype=np.uint32)
    P = ctypes.POINTER(ctypes.c_uint32)
    return lib.oracle_classify(poff, padj, g.n, g.n_left, k, xa.ctypes.data_as(P), len(x),
                               ya.ctypes.data_as(P), len(y))


# ----------------------------------------------------------------------------- BPPivot

_SL = re.compile(r"^\s*SL:\s*(.*)$")
_SR = re.compile(r"^\s*SR:\s*(.*)$")


def parse_bppivot_sets(text: str, n_left: int):
    """BPPivot -o 1 prints 'SL: a, b, ' (U ids) then 'SR: c, d, ' (V ids local to
    the right side); yield (X, Y) in global ids, sorted."""
    x = None
    for line in text.splitlines():
        m = _SL.match(line)
        if m:
            x = tuple(sorted(int(t) for t in m.group(1).replace(",", " ").split()))
            continue
        m = _SR.match(line)
        if m and x is not None:
            y = tuple(sorted(int(t) + n_left for t in m.group(1).replace(",", " ").split()))
            yield x, y
            x = None


def run_bppivot(graph_path: str, k: int, result_limit: int = 0, output: bool = False,
                timeout: float | None = None) -> dict:
    """Run the reference BPPivot binary with lower bound q=1 (every maximal
    k-biplex).  Returns count, branch_ms, wall-clock and (if output) the text."""
    exe = bppivot_path()
    if not os.path.exists(exe):
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)
    # BPPivot's search logger writes next to its input: give it a private directory
    tmpdir = tempfile.mkdtemp(prefix="bppivot_")
    link = os.path.join(tmpdir, os.path.basename(graph_path))
    os.symlink(os.path.abspath(graph_path), link)
    cmd = [exe, "-d", link, "-q", "1", "-k", str(k)]
    if result_limit:
        cmd += ["-n", str(result_limit)]
    if output:
        cmd += ["-o", "1"]
    import resource
    import time

    def _unlimited_stack():
        # the recursion depth reaches |V| on large graphs
        resource.setrlimit(resource.RLIMIT_STACK, (resource.RLIM_INFINITY, resource.RLIM_INFINITY))

    t0 = time.perf_counter()
    with tempfile.TemporaryFile() as f:
        p = subprocess.run(cmd, stdout=f, stderr=subprocess.STDOUT, timeout=timeout,
                           preexec_fn=_unlimited_stack)
        wall = time.perf_counter() - t0
        f.seek(0)
        text = f.read().decode(errors="replace")
    import shutil
    shutil.rmtree(tmpdir, ignore_errors=True)
    if p.returncode != 0:
        raise RuntimeError(f"bppivot exited {p.returncode}: {text[-400:]}")
    cnt = re.search(r"Number of biplexes:\s*(\d+)", text)
    br = re.search(r"Branch time:\s*(\d+)", text)
    return {"count": int(cnt.group(1)) if cnt else None,
            "branch_ms": int(br.group(1)) if br else None,
            "wall_s": wall, "text": text if output else None}


# ----------------------------------------------------------------------------- reference GPU binary

_RESULT = re.compile(r"^Result \d+: X: ([0-9 ]*)\| Y: ([0-9 ]*)$")
_RUNTIME = re.compile(r"Running Time:\s*([0-9.eE+-]+)\s*ms")


def parse_reference_results(text: str, n_left: int):
    """The reference's `Result N: X: x.. | Y: y..` lines (src/output.cuh) as
    sorted (X, Y) tuples of global ids (Y ids below n_left are shifted)."""
    for line in text.splitlines():
        m = _RESULT.match(line.rstrip("\n"))
        if not m:
            continue
        x = tuple(sorted(int(t) for t in m.group(1).split()))
        y = [int(t) for t in m.group(2).split()]
        y = tuple(sorted(v if v >= n_left else v + n_left for v in y))
        yield x, y


def run_reference_gpu(graph_path: str, k: int, result_limit: int = 10_000_000,
                      output: bool = False, device: int = 0, timeout: float | None = None) -> dict:
    """Runs `gmkbpe -f <graph> -k k -r limit -q 0|1 -d device` on a private
    copy of the graph's directory (its time recorder writes a JSON next to the
    input).  Returns running_ms, the printed result lines' text (output=True)
    and the exit status."""
    exe = refgpu_path()
    tmpdir = tempfile.mkdtemp(prefix="gmkbpe_")
    link = os.path.join(tmpdir, "g.graph.bin")
    os.symlink(os.path.abspath(graph_path), link)
    cmd = [exe, "-f", link, "-k", str(k), "-r", str(result_limit), "-q", "1" if output else "0",
           "-d", str(device)]
    import shutil
    import time
    t0 = time.perf_counter()
    with tempfile.TemporaryFile() as f:
        p = subprocess.run(cmd, stdout=f, stderr=subprocess.STDOUT, timeout=timeout)
        wall = time.perf_counter() - t0
        f.seek(0)
        text = f.read().decode(errors="replace")
    shutil.rmtree(tmpdir, ignore_errors=True)
    m = _RUNTIME.search(text)
    return {"returncode": p.returncode, "running_ms": float(m.group(1)) if m else None,
            "wall_s": wall, "text": text}


# ----------------------------------------------------------------------------- brute force

def brute_force(g, k: int):
    """Every maximal k-biplex with both sides non-empty, by exhaustive search over
    all vertex subsets (the definition itself).  Only for n <= 16."""
    n, nl = g.n, g.n_left
    if n > 16:
        raise ValueError("brute force is limited to 16 vertices")
    adj = [set(int(w) for w in g.nbrs(v)) for v in range(n)]
    U, V = list(range(nl)), list(range(nl, n))

    def is_biplex(X, Y):
        return all(len(set(Y) - adj[x]) <= k for x in X) and \
            all(len(set(X) - adj[y]) <= k for y in Y)

    plexes = []
    for mx in range(1, 1 << len(U)):
        X = [U[i] for i in range(len(U)) if mx >> i & 1]
        for my in range(1, 1 << len(V)):
            Y = [V[i] for i in range(len(V)) if my >> i & 1]
            if is_biplex(X, Y):
                plexes.append((X, Y))
    out = []
    for X, Y in plexes:
        maximal = True
        for w in itertools.chain(U, V):
            if w in X or w in Y:
                continue
            X2, Y2 = (X + [w], Y) if w < nl else (X, Y + [w])
            if is_biplex(X2, Y2):
                maximal = False
                break
        if maximal:
            out.append((tuple(X), tuple(Y)))
    return out
