"""Seeded synthetic bipartite graphs and the `.graph.bin` format.

`.graph.bin` layout (little-endian u32), as read by the reference loader
`data/src/tmp_load.h:213-295` and written by `preprocess/graph_conver.cpp:786-810`:

    header: 2|E|, N, |U|
    then for every vertex i in 0..N-1:  id (=i), deg, deg sorted neighbour ids

U vertices have ids [0, |U|), V vertices [|U|, N).  Neighbour lists hold global
ids.  The reference enumerator relies on the converter's per-side order
(`src/main.cu:1611` reads the max degree from the last id of each side), so
`relabel` below applies the same ordering rules as the converter
(`preprocess/graph_conver.cpp:566-733`): ids are compacted per side in numeric
order, parallel edges are dropped, isolated vertices disappear, and each side
is sorted by (log32 bucket of d', d', compact id) with d' = deg-2 on the left
and deg-1 on the right, computed in unsigned 32-bit arithmetic (so left
vertices of degree 1 wrap around and sort last).
"""
from __future__ import annotations

import os
import struct
from dataclasses import dataclass

import numpy as np


@dataclass
class Graph:
    """CSR over both sides; `offsets` has N+1 entries, `adj` 2|E| global ids."""
    n_left: int
    n: int
    offsets: np.ndarray  # uint64 [N+1]
    adj: np.ndarray      # uint32 [2|E|]

    @property
    def n_right(self) -> int:
        return self.n - self.n_left

    @property
    def n_edges(self) -> int:
        return int(self.adj.shape[0] // 2)

    def degree(self) -> np.ndarray:
        return np.diff(self.offsets).astype(np.uint32)

    def nbrs(self, v: int) -> np.ndarray:
        return self.adj[self.offsets[v]:self.offsets[v + 1]]

    def edges(self) -> np.ndarray:
        """(|E|, 2) array of (u, v) with u < n_left <= v."""
        deg = self.degree()[: self.n_left]
        src = np.repeat(np.arange(self.n_left, dtype=np.uint32), deg)
        dst = self.adj[: int(self.offsets[self.n_left])]
        return np.stack([src, dst], axis=1)


def _degree_bucket(d: np.ndarray) -> np.ndarray:
    """Bucket b = smallest b with d <= 32^(b+1), capped at 8 (graph_conver.cpp:443-451)."""
    d = d.astype(np.uint64)
    b = np.zeros(d.shape, dtype=np.uint64)
    limit = np.full(d.shape, 32, dtype=np.uint64)
    for _ in range(8):
        m = (d > limit) & (b < 8)
        if not m.any():
            break
        b[m] += 1
        limit[m] *= 32
    return b


def relabel(left_ids: np.ndarray, right_ids: np.ndarray) -> Graph:
    """Edge list (arbitrary non-negative ids per side) -> converter-ordered CSR."""
    left_ids = np.asarray(left_ids, dtype=np.int64)
    right_ids = np.asarray(right_ids, dtype=np.int64)
    if left_ids.size == 0:
        return Graph(0, 0, np.zeros(1, np.uint64), np.zeros(0, np.uint32))
    lu, li = np.unique(left_ids, return_inverse=True)
    ru, ri = np.unique(right_ids, return_inverse=True)
    nl, nr = lu.size, ru.size
    key = np.unique(li.astype(np.int64) * nr + ri)          # drops parallel edges
    li, ri = key // nr, key % nr
    degl = np.bincount(li, minlength=nl).astype(np.uint32)
    degr = np.bincount(ri, minlength=nr).astype(np.uint32)
    with np.errstate(over="ignore"):
        dl = (degl - np.uint32(2)).astype(np.uint32)
        dr = (degr - np.uint32(1)).astype(np.uint32)
    ordl = np.lexsort((np.arange(nl), dl, _degree_bucket(dl)))
    ordr = np.lexsort((np.arange(nr), dr, _degree_bucket(dr)))
    newl = np.empty(nl, np.int64); newl[ordl] = np.arange(nl)
    newr = np.empty(nr, np.int64); newr[ordr] = np.arange(nr) + nl
    return from_edges(newl[li], newr[ri], nl, nl + nr)


def from_edges(u: np.ndarray, v: np.ndarray, n_left: int, n: int) -> Graph:
    """CSR from global-id edges (u in [0,n_left), v in [n_left,n)); rows sorted."""
    u = np.asarray(u, dtype=np.int64)
    v = np.asarray(v, dtype=np.int64)
    src = np.concatenate([u, v])
    dst = np.concatenate([v, u])
    order = np.lexsort((dst, src))
    src, dst = src[order], dst[order]
    if src.size:
        keep = np.ones(src.size, bool)
        keep[1:] = (src[1:] != src[:-1]) | (dst[1:] != dst[:-1])
        src, dst = src[keep], dst[keep]
    counts = np.bincount(src, minlength=n)
    offsets = np.zeros(n + 1, np.uint64)
    np.cumsum(counts, out=offsets[1:])
    return Graph(int(n_left), int(n), offsets, dst.astype(np.uint32))


def write_graph_bin(g: Graph, path: str) -> None:
    deg = g.degree().astype(np.int64)
    out = np.empty(3 + 2 * g.n + g.adj.size, dtype="<u4")
    out[:3] = (g.adj.size, g.n, g.n_left)
    start = 3 + 2 * np.arange(g.n, dtype=np.int64) + g.offsets[:-1].astype(np.int64)
    out[start] = np.arange(g.n, dtype=np.uint32)
    out[start + 1] = deg
    # neighbour j of vertex i lands at start[i] + 2 + (j - offsets[i])
    owner = np.repeat(np.arange(g.n, dtype=np.int64), deg)
    pos = np.arange(g.adj.size, dtype=np.int64) + 3 + 2 * owner + 2
    out[pos] = g.adj
    with open(path, "wb") as f:
        f.write(out.tobytes())


def read_graph_bin(path: str) -> Graph:
    raw = np.fromfile(path, dtype="<u4")
    if raw.size < 3:
        raise ValueError(f"{path}: truncated header")
    n2e, n, nl = (int(x) for x in raw[:3])
    if nl > n:
        raise ValueError(f"{path}: bipartite index {nl} > N {n}")
    offsets = np.zeros(n + 1, np.uint64)
    adj = np.empty(n2e, np.uint32)
    pos, w = 3, 0
    for i in range(n):
        if pos + 2 > raw.size:
            raise ValueError(f"{path}: truncated vertex record {i}")
        d = int(raw[pos + 1]); pos += 2
        if pos + d > raw.size or w + d > n2e:
            raise ValueError(f"{path}: truncated neighbours of {i}")
        adj[w:w + d] = raw[pos:pos + d]
        pos += d; w += d
        offsets[i + 1] = w
    return Graph(nl, n, offsets, adj[:w])


# ----------------------------------------------------------------------------- generators

DENSE_ER_PAIRS = 1 << 24   # larger ER graphs are sampled edge by edge


def erdos_renyi(nu: int, nv: int, p: float, seed: int) -> Graph:
    """Each of the nu*nv pairs independently with probability p (PCG64(seed)).
    Up to DENSE_ER_PAIRS pairs every pair is drawn (the committed fixtures were
    made that way); above it the edge count is drawn from Binomial(nu*nv, p)
    and that many distinct pairs are drawn uniformly -- the same distribution
    without a dense nu x nv draw."""
    rng = np.random.Generator(np.random.PCG64(seed))
    if nu * nv <= DENSE_ER_PAIRS:
        mask = rng.random((nu, nv)) < p
        li, ri = np.nonzero(mask)
        return relabel(li, ri)
    total = nu * nv
    m = int(rng.binomial(total, p))
    keys = np.unique(rng.integers(0, total, size=m + m // 8 + 16, dtype=np.int64))
    while keys.size < m:
        keys = np.unique(np.concatenate([keys, rng.integers(0, total, size=m - keys.size + 16,
                                                            dtype=np.int64)]))
    keys = rng.permutation(keys)[:m]
    return relabel(keys // nv, keys % nv)


def _chung_lu_weights(n: int, gamma: float, mean_deg: float, cap: float | None) -> np.ndarray:
    i = np.arange(1, n + 1, dtype=np.float64)
    w = i ** (-1.0 / (gamma - 1.0))
    w *= mean_deg * n / w.sum()
    if cap is not None:
        for _ in range(50):                     # clip and re-normalise to keep the mean
            over = w > cap
            if not over.any():
                break
            w[over] = cap
            free = ~over
            need = mean_deg * n - w[over].sum()
            w[free] *= need / w[free].sum()
        w = np.minimum(w, cap)
    return w


def chung_lu(nu: int, nv: int, m: int, gamma: float, seed: int,
             max_deg: int | None = None) -> Graph:
    """Bipartite Chung-Lu: m endpoint pairs drawn with P(u) ~ w_u, P(v) ~ w_v,
    w_i ~ i^(-1/(gamma-1)) on each side, expected degrees capped at max_deg;
    parallel edges collapse, so the edge count ends slightly below m."""
    rng = np.random.Generator(np.random.PCG64(seed))
    wu = _chung_lu_weights(nu, gamma, m / nu, max_deg)
    wv = _chung_lu_weights(nv, gamma, m / nv, max_deg)
    u = rng.choice(nu, size=m, p=wu / wu.sum())
    v = rng.choice(nv, size=m, p=wv / wv.sum())
    return relabel(u, v)


def hubs_and_sparse(n_hubs: int, n_sparse: int, n: int, d_sparse: int, seed: int) -> Graph:
    """n_hubs V vertices adjacent to all n U vertices, plus n_sparse V vertices
    of d_sparse random U neighbours each.  Once S holds k + 1 hubs, a node's
    U candidates are a local list of about n entries (the union of the hubs'
    rows), and a sparse member one miss short of k makes every child that
    misses it filter that list: the long-list filter with few results."""
    rng = np.random.Generator(np.random.PCG64(seed))
    left, right = [], []
    for h in range(n_hubs):
        left.append(np.arange(n, dtype=np.int64))
        right.append(np.full(n, h, dtype=np.int64))
    for y in range(n_hubs, n_hubs + n_sparse):
        left.append(rng.choice(n, size=d_sparse, replace=False).astype(np.int64))
        right.append(np.full(d_sparse, y, dtype=np.int64))
    return relabel(np.concatenate(left), np.concatenate(right))


def induced_prefix(g: Graph, nu: int, nv: int) -> Graph:
    """Subgraph induced by the first nu U ids and first nv V ids, re-run through
    the converter ordering (isolated vertices dropped)."""
    e = g.edges().astype(np.int64)
    keep = (e[:, 0] < nu) & (e[:, 1] < g.n_left + nv)
    e = e[keep]
    return relabel(e[:, 0], e[:, 1] - g.n_left)


# ----------------------------------------------------------------------------- named workloads
# Sizes, exponents and seeds of the five synthetic workloads the enumerator is
# measured on; "full" marks whole-set enumeration, otherwise result_limit caps it.

WORKLOADS = {
    "er200": dict(kind="er", nu=200, nv=200, p=0.05, seed=1, k=1, result_limit=0),
    "cl20k": dict(kind="cl", nu=20_000, nv=50_000, m=500_000, gamma=2.1, max_deg=2000,
                  seed=2, k=1, result_limit=1_000_000),
    "cl20k_sub": dict(kind="cl_sub", base="cl20k", sub_u=5_000, sub_v=12_000, k=1,
                      result_limit=0),
    "cl100k": dict(kind="cl", nu=100_000, nv=300_000, m=3_000_000, gamma=2.2, max_deg=None,
                   seed=3, k=2, result_limit=10_000_000),
    "cl500k": dict(kind="cl", nu=500_000, nv=1_000_000, m=20_000_000, gamma=2.0,
                   max_deg=None, seed=4, k=1, result_limit=100_000_000),
}


def mixed_batch(n_graphs: int = 64, seed0: int = 100, size_lo: int = 1_000,
                size_hi: int = 50_000, deg_lo: float = 5.0, deg_hi: float = 30.0,
                gamma: float = 2.1) -> tuple[list[Graph], list[int]]:
    """A batch of uneven graphs and their k: graph i (seed seed0 + i) has |U|
    and |V| log-uniform in [size_lo, size_hi], average U-side degree uniform in
    [deg_lo, deg_hi] (capped by |V|), Erdos-Renyi for even i and Chung-Lu with
    exponent gamma for odd i, and k drawn from {1, 2, 3}."""
    graphs, ks = [], []
    for i in range(n_graphs):
        seed = seed0 + i
        rng = np.random.Generator(np.random.PCG64(seed))
        nu = int(round(np.exp(rng.uniform(np.log(size_lo), np.log(size_hi)))))
        nv = int(round(np.exp(rng.uniform(np.log(size_lo), np.log(size_hi)))))
        deg = min(float(rng.uniform(deg_lo, deg_hi)), 0.9 * nv)
        k = int(rng.integers(1, 4))
        if i % 2 == 0:
            g = erdos_renyi(nu, nv, deg / nv, seed)
        else:
            g = chung_lu(nu, nv, max(1, int(deg * nu)), gamma, seed)
        graphs.append(g)
        ks.append(k)
    return graphs, ks


def make_workload(name: str) -> Graph:
    w = WORKLOADS[name]
    if w["kind"] == "er":
        return erdos_renyi(w["nu"], w["nv"], w["p"], w["seed"])
    if w["kind"] == "cl":
        return chung_lu(w["nu"], w["nv"], w["m"], w["gamma"], w["seed"], w["max_deg"])
    if w["kind"] == "cl_sub":
        return induced_prefix(make_workload(w["base"]), w["sub_u"], w["sub_v"])
    raise KeyError(name)


def cached_workload(name: str, cache_dir: str | None = None) -> str:
    """Path of the workload's .graph.bin, generating it on first use."""
    cache_dir = cache_dir or os.environ.get("GMK_GRAPH_CACHE") or os.path.join(
        os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "_graphs")
    os.makedirs(cache_dir, exist_ok=True)
    path = os.path.join(cache_dir, f"{name}.graph.bin")
    if not os.path.exists(path):
        tmp = path + f".tmp{os.getpid()}"
        write_graph_bin(make_workload(name), tmp)
        os.replace(tmp, path)
    return path
