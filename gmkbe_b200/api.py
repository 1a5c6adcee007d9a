"""Python host mirror of the enumerator's C ABI (include/gmk.h), via ctypes.

    g = gmkbe_b200.Graph.load("g.graph.bin", device=0)
    st = g.enumerate(k=1, result_limit=10**6)
    st.count, st.hash_sum, st.hash_xor

Argument meanings and errors follow the reference executable (-f/-k/-r/-d,
src/main.cu:1719-1775): k >= 1, a result limit of 0 means "all", a CUDA or
file error raises GmkError.  There is no CPU path: without libgmk.so or a
GPU, every call raises.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
# GMK_LIBRARY names another build of the library (for A/B measurements)
LIB_PATH = os.environ.get("GMK_LIBRARY") or os.path.join(_PKG, "libgmk.so")

# entry points declared in include/gmk.h
EXPORTS = ("gmk_graph_load", "gmk_graph_from_csr", "gmk_graph_info", "gmk_graph_fingerprint",
           "gmk_graph_free",
           "gmk_opts_default", "gmk_enumerate", "gmk_enumerate_batch", "gmk_enumerate_resumable",
           "gmk_enumerate_noalloc", "gmk_result_hash", "gmk_strerror", "gmk_last_cuda_error",
           "gmk_abi_version", "gmk_root_features", "gmk_mlp_create", "gmk_mlp_free",
           "gmk_mlp_params", "gmk_mlp_gradient", "gmk_mlp_train", "gmk_mlp_predict",
           "gmk_mlp_predict_roots",
           "gmk_root_costs", "gmk_plan_tasks", "gmk_graph_set_hash_load")

SCHEDULES = {"plain": 0, "batched": 1, "ordered": 2}
ENGINES = {"warp": 0, "thread": 1}

E_OUTBUF = -9
E_SINK = -10
E_CHECKPOINT = -12
PAUSED = 1


class GmkError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"gmk error {code}: {msg}")
        self.code = code


class _Opts(ctypes.Structure):
    _fields_ = [("k", ctypes.c_uint32), ("result_limit", ctypes.c_uint64),
                ("schedule", ctypes.c_int32), ("emit", ctypes.c_int32),
                ("chunk", ctypes.c_uint32), ("threads", ctypes.c_uint32),
                ("arena_words", ctypes.c_uint32), ("max_members", ctypes.c_uint32),
                ("watchdog_ms", ctypes.c_uint32), ("out_words", ctypes.c_uint64),
                ("task_cost", ctypes.POINTER(ctypes.c_float)), ("pair_limit", ctypes.c_uint32),
                ("shard", ctypes.c_uint32), ("nshards", ctypes.c_uint32),
                ("engine", ctypes.c_int32), ("split_min_nodes", ctypes.c_uint32),
                ("root_begin", ctypes.c_uint32), ("root_end", ctypes.c_uint32),
                ("root_nodes", ctypes.POINTER(ctypes.c_uint64)),
                ("donate_min_nodes", ctypes.c_uint32), ("no_sharing", ctypes.c_int32),
                ("tasks", ctypes.c_void_p), ("n_tasks", ctypes.c_uint64),
                ("tasks_per_worker", ctypes.c_uint32), ("bits_min_list", ctypes.c_uint32)]


class _Stats(ctypes.Structure):
    _fields_ = [("count", ctypes.c_uint64), ("hash_sum", ctypes.c_uint64),
                ("hash_xor", ctypes.c_uint64), ("nodes", ctypes.c_uint64),
                ("algo_bytes", ctypes.c_uint64), ("tasks", ctypes.c_uint64),
                ("tasks_done", ctypes.c_uint64), ("kernel_ms", ctypes.c_double),
                ("truncated", ctypes.c_int32), ("threads", ctypes.c_uint32),
                ("rounds", ctypes.c_uint32), ("donations", ctypes.c_uint64)]


class _Task(ctypes.Structure):
    _fields_ = [("root", ctypes.c_uint32), ("first", ctypes.c_uint32), ("last", ctypes.c_uint32),
                ("graph", ctypes.c_uint32), ("cost", ctypes.c_float)]


SINK = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32),
                        ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32), ctypes.c_uint32)

_lib = None


def load_library(path: str = LIB_PATH):
    """Load libgmk.so; raises if it is missing (no fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise GmkError(-11, f"{path} not built; run `python -m gmkbe_b200.build`")
    lib = ctypes.CDLL(path)
    P32 = ctypes.POINTER(ctypes.c_uint32)
    lib.gmk_graph_load.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    lib.gmk_graph_from_csr.argtypes = [P32, P32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_void_p)]
    lib.gmk_graph_info.argtypes = [ctypes.c_void_p, P32, P32, ctypes.POINTER(ctypes.c_uint64)]
    lib.gmk_graph_fingerprint.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)]
    lib.gmk_graph_free.argtypes = [ctypes.c_void_p]
    lib.gmk_graph_free.restype = None
    lib.gmk_opts_default.argtypes = [ctypes.POINTER(_Opts)]
    lib.gmk_opts_default.restype = None
    lib.gmk_enumerate.argtypes = [ctypes.c_void_p, ctypes.POINTER(_Opts), SINK, ctypes.c_void_p,
                                  ctypes.POINTER(_Stats)]
    lib.gmk_enumerate_batch.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_uint32, P32,
                                        ctypes.POINTER(ctypes.c_uint64),
                                        ctypes.POINTER(ctypes.POINTER(ctypes.c_float)),
                                        ctypes.POINTER(_Opts), ctypes.POINTER(_Stats)]
    lib.gmk_enumerate_resumable.argtypes = [ctypes.c_void_p, ctypes.POINTER(_Opts), ctypes.c_char_p,
                                            ctypes.c_uint32, ctypes.c_uint32, SINK,
                                            ctypes.c_void_p, ctypes.POINTER(_Stats)]
    lib.gmk_enumerate_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                          ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64,
                                          ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                          ctypes.c_void_p, ctypes.POINTER(_Stats)]
    PF = ctypes.POINTER(ctypes.c_float)
    lib.gmk_root_features.argtypes = [ctypes.c_void_p, ctypes.c_uint32, PF]
    lib.gmk_mlp_create.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p)]
    lib.gmk_mlp_free.argtypes = [ctypes.c_void_p]
    lib.gmk_mlp_free.restype = None
    lib.gmk_mlp_params.argtypes = [ctypes.c_void_p, PF, PF]
    lib.gmk_mlp_gradient.argtypes = [ctypes.c_void_p, PF, PF, ctypes.c_uint32, PF, PF]
    lib.gmk_mlp_train.argtypes = [ctypes.c_void_p, PF, PF, ctypes.c_uint32, ctypes.c_uint32,
                                  ctypes.c_float, PF]
    lib.gmk_mlp_predict.argtypes = [ctypes.c_void_p, PF, ctypes.c_uint32, PF]
    if hasattr(lib, "gmk_mlp_predict_roots"):
        lib.gmk_mlp_predict_roots.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, PF]
    lib.gmk_result_hash.argtypes = [P32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                    ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
    lib.gmk_result_hash.restype = None
    if hasattr(lib, "gmk_graph_set_hash_load"):
        lib.gmk_graph_set_hash_load.argtypes = [ctypes.c_void_p, ctypes.c_uint32]
    if hasattr(lib, "gmk_plan_tasks"):   # (a library build from before the planner lacks them)
        lib.gmk_root_costs.argtypes = [ctypes.c_void_p, PF]
        lib.gmk_plan_tasks.argtypes = [ctypes.c_uint32, ctypes.c_uint32, PF, ctypes.c_uint32,
                                       ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint32,
                                       ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(_Task),
                                       ctypes.POINTER(ctypes.c_uint64)]
    lib.gmk_strerror.restype = ctypes.c_char_p
    lib.gmk_last_cuda_error.restype = ctypes.c_char_p
    _lib = lib
    return lib


def _check(rc: int) -> None:
    if rc:
        lib = load_library()
        raise GmkError(rc, f"{lib.gmk_strerror(rc).decode()} ({lib.gmk_last_cuda_error().decode()})")


@dataclass
class Stats:
    count: int
    hash_sum: int
    hash_xor: int
    nodes: int
    algo_bytes: int
    tasks: int
    tasks_done: int
    kernel_ms: float
    truncated: bool
    threads: int
    rounds: int = 1
    results: list | None = None
    donations: int = 0

    def summary(self) -> tuple[int, int, int]:
        return self.count, self.hash_sum, self.hash_xor


def enumerate_batch(graphs, ks, schedule: str = "batched", task_costs=None, limits=None,
                    **tuning) -> list:
    """gmk_enumerate_batch: several graphs (all on one device) in one run of
    launches; ks[i] is graph i's k, limits[i] its result cap (None: complete
    enumeration of every graph).  Returns one Stats per graph."""
    lib = load_library()
    n = len(graphs)
    o, _ = graphs[0]._opts(int(ks[0]), 0, schedule, tuning.get("chunk", 0), tuning.get("threads", 0),
                           tuning.get("arena_words", 0), tuning.get("max_members", 0),
                           tuning.get("watchdog_ms", 0), tuning.get("pair_limit", 0), None, 0, 1,
                           "warp", tuning.get("split_min_nodes", 0), 0, 0)
    hs = (ctypes.c_void_p * n)(*[g._h.value for g in graphs])
    karr = np.ascontiguousarray(ks, dtype=np.uint32)
    PF = ctypes.POINTER(ctypes.c_float)
    costs_keep = []
    costs = None
    if task_costs is not None:
        costs = (PF * n)()
        for i, c in enumerate(task_costs):
            c = np.ascontiguousarray(c, dtype=np.float32)
            costs_keep.append(c)
            costs[i] = c.ctypes.data_as(PF)
    outs = (_Stats * n)()
    lim = None
    if limits is not None:
        larr = np.ascontiguousarray(limits, dtype=np.uint64)
        lim = larr.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
    _check(lib.gmk_enumerate_batch(hs, n, karr.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                                   lim, costs, ctypes.byref(o), outs))
    return [Graph._stats(outs[i], None) for i in range(n)]


def plan_tasks(n: int, n_left: int, root_cost, root_begin: int = 0, root_end: int | None = None,
               target_tasks: int = 1, max_chunks: int = 0, nshards: int = 1,
               shard: int = 0) -> np.ndarray:
    """gmk_plan_tasks (host only, no GPU needed): this shard's planned tasks as
    a structured array with fields root, first, last, graph, cost, largest
    cost first."""
    lib = load_library()
    cost = np.ascontiguousarray(root_cost, dtype=np.float32)
    if cost.size != n_left:
        raise ValueError("root_cost needs one value per U vertex")
    re_ = n_left if root_end is None else root_end
    PF = ctypes.POINTER(ctypes.c_float)
    cnt = ctypes.c_uint64()
    args = (n, n_left, cost.ctypes.data_as(PF), root_begin, re_, target_tasks, max_chunks,
            nshards, shard)
    _check(lib.gmk_plan_tasks(*args, None, ctypes.byref(cnt)))
    buf = (_Task * max(1, cnt.value))()
    _check(lib.gmk_plan_tasks(*args, buf, ctypes.byref(cnt)))
    dt = np.dtype([("root", np.uint32), ("first", np.uint32), ("last", np.uint32),
                   ("graph", np.uint32), ("cost", np.float32)])
    return np.frombuffer(bytes(buf), dtype=dt, count=cnt.value).copy()


def result_hash(x, y) -> tuple[int, int]:
    """The library's per-result hash pair (gmk_result_hash)."""
    lib = load_library()
    ids = np.ascontiguousarray(list(x) + list(y) or [0], dtype=np.uint32)
    h1, h2 = ctypes.c_uint64(), ctypes.c_uint64()
    lib.gmk_result_hash(ids.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), len(x) + len(y),
                        len(x), len(y), ctypes.byref(h1), ctypes.byref(h2))
    return h1.value, h2.value


class Graph:
    """A bipartite graph resident on one GPU (gmk_graph)."""

    def __init__(self, handle: int, device: int):
        self._h = ctypes.c_void_p(handle)
        self.device = device
        lib = load_library()
        n, nl, m = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint64()
        _check(lib.gmk_graph_info(self._h, ctypes.byref(n), ctypes.byref(nl), ctypes.byref(m)))
        self.n, self.n_left, self.adj_len = n.value, nl.value, m.value

    def set_hash_load(self, load_pct: int) -> None:
        """gmk_graph_set_hash_load: rebuild the edge hash at this maximum load (%)."""
        _check(load_library().gmk_graph_set_hash_load(self._h, load_pct))

    def root_costs(self) -> np.ndarray:
        """gmk_root_costs: the 2-hop cost proxy of every root (float32, n_left)."""
        out = np.zeros(self.n_left, np.float32)
        _check(load_library().gmk_root_costs(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def fingerprint(self) -> int:
        """64-bit hash of the CSR (the identity checkpoints and tuning caches record)."""
        v = ctypes.c_uint64()
        _check(load_library().gmk_graph_fingerprint(self._h, ctypes.byref(v)))
        return v.value

    @classmethod
    def load(cls, path: str, device: int = 0) -> "Graph":
        lib = load_library()
        h = ctypes.c_void_p()
        _check(lib.gmk_graph_load(os.fsencode(path), device, ctypes.byref(h)))
        return cls(h.value, device)

    @classmethod
    def from_csr(cls, offsets, adj, n: int, n_left: int, device: int = 0) -> "Graph":
        lib = load_library()
        off = np.ascontiguousarray(offsets, dtype=np.uint32)
        a = np.ascontiguousarray(adj, dtype=np.uint32)
        if a.size == 0:
            a = np.zeros(1, np.uint32)
        P = ctypes.POINTER(ctypes.c_uint32)
        h = ctypes.c_void_p()
        _check(lib.gmk_graph_from_csr(off.ctypes.data_as(P), a.ctypes.data_as(P), n, n_left,
                                      device, ctypes.byref(h)))
        return cls(h.value, device)

    @classmethod
    def from_graph(cls, g, device: int = 0) -> "Graph":
        """From a gmkbe_b200.graphgen.Graph."""
        return cls.from_csr(g.offsets, g.adj, g.n, g.n_left, device)

    def close(self) -> None:
        if self._h:
            load_library().gmk_graph_free(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _opts(self, k, result_limit, schedule, chunk, threads, arena_words, max_members,
              watchdog_ms, pair_limit, task_cost, shard, nshards, engine, split_min_nodes,
              root_begin, root_end):
        lib = load_library()
        o = _Opts()
        lib.gmk_opts_default(ctypes.byref(o))
        o.k, o.result_limit, o.schedule = k, result_limit, SCHEDULES[schedule]
        o.chunk, o.threads, o.arena_words = chunk, threads, arena_words
        o.max_members, o.watchdog_ms, o.pair_limit = max_members, watchdog_ms, pair_limit
        o.shard, o.nshards = shard, nshards
        o.engine, o.split_min_nodes = ENGINES[engine], split_min_nodes
        o.root_begin, o.root_end = root_begin, root_end
        cost = None
        if task_cost is not None:
            cost = np.ascontiguousarray(task_cost, dtype=np.float32)
            if cost.size != self.n_left:
                raise ValueError("task_cost needs one value per U vertex")
            o.task_cost = cost.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        return o, cost

    @staticmethod
    def _sink(collect, sink, out):
        if not (collect or sink is not None):
            return SINK(0)

        def _cb(_u, xp, nx, yp, ny):
            x = tuple(xp[i] for i in range(nx))
            y = tuple(yp[i] for i in range(ny))
            if collect:
                out.append((x, y))
                return 0
            return 1 if sink(x, y) else 0
        return SINK(_cb)

    @staticmethod
    def _stats(st, results):
        return Stats(st.count, st.hash_sum, st.hash_xor, st.nodes, st.algo_bytes, st.tasks,
                     st.tasks_done, st.kernel_ms, bool(st.truncated), st.threads, st.rounds,
                     results, st.donations)

    def enumerate(self, k: int = 1, result_limit: int = 0, schedule: str = "batched",
                  collect: bool = False, chunk: int = 0, threads: int = 0, arena_words: int = 0,
                  max_members: int = 0, watchdog_ms: int = 0, pair_limit: int = 0,
                  task_cost=None, sink=None, shard: int = 0, nshards: int = 1,
                  engine: str = "warp", split_min_nodes: int = 0, root_begin: int = 0,
                  root_end: int = 0, root_nodes=None, out_words: int = 0,
                  donate_min_nodes: int = 0, sharing: bool = True, tasks=None,
                  tasks_per_worker: int = 0, bits_min_list: int = 0) -> Stats:
        """Enumerate maximal k-biplexes.  collect=True returns the result list
        (sorted X, Y tuples) in Stats.results; `sink(x, y)` is called per
        result otherwise (return True to stop).  root_nodes: a uint64 numpy
        array of n_left entries to which each root's search nodes are added."""
        lib = load_library()
        o, _cost = self._opts(k, result_limit, schedule, chunk, threads, arena_words, max_members,
                              watchdog_ms, pair_limit, task_cost, shard, nshards, engine,
                              split_min_nodes, root_begin, root_end)
        if root_nodes is not None:
            if root_nodes.dtype != np.uint64 or root_nodes.size != self.n_left or \
                    not root_nodes.flags.c_contiguous:
                raise ValueError("root_nodes must be a contiguous uint64 array of n_left entries")
            o.root_nodes = root_nodes.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
        o.donate_min_nodes = donate_min_nodes
        o.no_sharing = 0 if sharing else 1
        o.tasks_per_worker, o.bits_min_list = tasks_per_worker, bits_min_list
        task_buf = None
        if tasks is not None:
            # an explicit task list (structured array from plan_tasks, or rows of
            # (root, first, last)): run exactly these tasks
            rows = [(int(t[0]), int(t[1]), int(t[2])) for t in tasks]
            task_buf = (_Task * max(1, len(rows)))()
            for i, (r, f, l) in enumerate(rows):
                task_buf[i] = _Task(r, f, l, 0, 0.0)
            o.tasks = ctypes.cast(task_buf, ctypes.c_void_p)
            o.n_tasks = len(rows)
        out: list = []
        cb = self._sink(collect, sink, out)
        o.emit = 1 if (collect or sink is not None) else 0
        o.out_words = out_words
        st = _Stats()
        while True:
            out.clear()
            rc = lib.gmk_enumerate(self._h, ctypes.byref(o), cb, None, ctypes.byref(st))
            # a record buffer overflow is retried with a larger buffer only when
            # no caller sink has seen results yet
            if rc != E_OUTBUF or sink is not None:
                break
            o.out_words = (o.out_words or (64 << 20)) * 4
        if rc != E_SINK:
            _check(rc)
        return self._stats(st, out if collect else None)

    def enumerate_resumable(self, checkpoint: str, batch_roots: int = 0, max_batches: int = 0,
                            k: int = 1, result_limit: int = 0, schedule: str = "batched",
                            collect: bool = False, sink=None, task_cost=None,
                            engine: str = "warp", **tuning) -> tuple[Stats, bool]:
        """gmk_enumerate_resumable: batches of roots with a checkpoint file after
        each.  Returns (totals of the whole run, paused); paused is True when
        max_batches stopped the call with work left (call again to resume)."""
        lib = load_library()
        o, _cost = self._opts(k, result_limit, schedule, tuning.get("chunk", 0),
                              tuning.get("threads", 0), tuning.get("arena_words", 0),
                              tuning.get("max_members", 0), tuning.get("watchdog_ms", 0),
                              tuning.get("pair_limit", 0), task_cost, tuning.get("shard", 0),
                              tuning.get("nshards", 1), engine, tuning.get("split_min_nodes", 0),
                              0, 0)
        out: list = []
        cb = self._sink(collect, sink, out)
        o.emit = 1 if (collect or sink is not None) else 0
        if o.emit:
            o.out_words = tuning.get("out_words", 0)
        st = _Stats()
        rc = lib.gmk_enumerate_resumable(self._h, ctypes.byref(o), os.fsencode(checkpoint),
                                         batch_roots, max_batches, cb, None, ctypes.byref(st))
        if rc not in (0, PAUSED, E_SINK):
            _check(rc)
        return self._stats(st, out if collect else None), rc == PAUSED
