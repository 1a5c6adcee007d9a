"""gmk_enumerate_noalloc: the entry point for callers that cannot allocate
device memory (code running under an external pool that owns the device
memory, or inside an allocator's own callbacks).  The test plays such a
caller: it holds the graph in device memory it allocated itself (torch), calls
the C ABI with those device pointers, and checks that two calls in a row give
the same set summary as the allocating entry point gmk_enumerate.  It also
checks that an oversized request is refused with GMK_E_SCRATCH.  This file is
collected last on purpose."""
import ctypes

import numpy as np
import pytest

import gmkbe_b200 as G
from gmkbe_b200.api import _Stats
from conftest import golden_graph_path
from gmkbe_b200 import graphgen as gg

pytestmark = pytest.mark.gpu

E_SCRATCH = -13
E_FORMAT = -3
E_ARENA = -6
SCRATCH_BYTES = 64 << 20


def _device_csr(g):
    import torch
    off = torch.from_numpy(np.ascontiguousarray(g.offsets, dtype=np.uint32).view(np.int32)).cuda()
    adj_np = np.ascontiguousarray(g.adj, dtype=np.uint32)
    if adj_np.size == 0:
        adj_np = np.zeros(1, np.uint32)
    adj = torch.from_numpy(adj_np.view(np.int32)).cuda()
    torch.cuda.synchronize()
    return off, adj


def _noalloc(lib, off, adj, g, k, limit=0, threads=0, arena=0, members=0):
    st = _Stats()
    rc = lib.gmk_enumerate_noalloc(ctypes.c_void_p(off.data_ptr()), ctypes.c_void_p(adj.data_ptr()),
                                   g.n, g.n_left, k, limit, threads, arena, members, None,
                                   ctypes.byref(st))
    return rc, st


@pytest.mark.parametrize("name,k", [("southernwomen", 2), ("er60", 1), ("er200", 1)])
def test_noalloc_matches_allocating_entry_point_twice(name, k):
    import torch
    torch.cuda.set_device(0)
    lib = G.load_library()
    g = gg.read_graph_bin(golden_graph_path(name))
    off, adj = _device_csr(g)
    with G.Graph.from_graph(g) as dg:
        want = dg.enumerate(k=k).summary()
    for _ in range(2):                      # the shared scratch keeps the last call's state
        rc, st = _noalloc(lib, off, adj, g, k)
        assert rc == 0, lib.gmk_strerror(rc)
        assert (st.count, st.hash_sum, st.hash_xor) == want
        assert not st.truncated


def test_noalloc_result_limit_and_oversized_request():
    import torch
    torch.cuda.set_device(0)
    lib = G.load_library()
    g = gg.read_graph_bin(golden_graph_path("er200"))
    off, adj = _device_csr(g)
    rc, st = _noalloc(lib, off, adj, g, 1, limit=1000)
    assert rc == 0 and st.count == 1000 and st.truncated
    rc, st = _noalloc(lib, off, adj, g, 1, threads=1 << 20, arena=1 << 16)
    assert rc == E_SCRATCH
    rc, st = _noalloc(lib, off, adj, g, 1)   # still usable after the refusal
    assert rc == 0 and st.count > 1000


def test_noalloc_empty_side_returns_nothing():
    import torch
    torch.cuda.set_device(0)
    lib = G.load_library()
    # three U vertices and no V side; then three V vertices and no U side
    for n, nl in ((3, 3), (3, 0)):
        off = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
        adj = torch.zeros(1, dtype=torch.int32, device="cuda")
        st = _Stats()
        rc = lib.gmk_enumerate_noalloc(ctypes.c_void_p(off.data_ptr()),
                                       ctypes.c_void_p(adj.data_ptr()), n, nl, 1, 0, 0, 0, 0,
                                       None, ctypes.byref(st))
        assert rc == 0 and st.count == 0


def test_noalloc_refuses_a_malformed_csr_before_the_search():
    # adj holds exactly d_offsets[n] words, so the device check reads only
    # valid memory; it must catch the bad rows before the search runs
    import torch
    torch.cuda.set_device(0)
    lib = G.load_library()
    g = gg.read_graph_bin(golden_graph_path("southernwomen"))
    off, adj = _device_csr(g)
    row0 = int(g.offsets[0]), int(g.offsets[1])
    bad_id = adj.clone()
    bad_id[row0[0]] = 0                       # a U id in a U row (wrong side)
    unsorted = adj.clone()
    unsorted[row0[0]], unsorted[row0[0] + 1] = adj[row0[0] + 1].item(), adj[row0[0]].item()
    for a in (bad_id, unsorted):
        rc, _ = _noalloc(lib, off, a, g, 1)
        assert rc == E_FORMAT
    bad_off = off.clone()
    bad_off[1] = bad_off[2] + 1               # offsets decrease
    rc, _ = _noalloc(lib, bad_off, adj, g, 1)
    assert rc == E_FORMAT
    rc, st = _noalloc(lib, off, adj, g, 1)    # the good CSR still runs
    assert rc == 0 and st.count == 1256


def test_noalloc_near_the_scratch_limit_and_arena_overflow():
    import torch
    torch.cuda.set_device(0)
    lib = G.load_library()
    g = gg.read_graph_bin(golden_graph_path("er60"))
    off, adj = _device_csr(g)
    with G.Graph.from_graph(g) as dg:
        want = dg.enumerate(k=2).summary()
    # 1024 threads x (4 x 15000 + 8 x 512) bytes + 256 = 65.6 MB of the 67.1 MB
    threads, arena, members = 1024, 15000, 512
    assert 256 + threads * (4 * arena + 8 * members) <= SCRATCH_BYTES
    rc, st = _noalloc(lib, off, adj, g, 2, threads=threads, arena=arena, members=members)
    assert rc == 0 and (st.count, st.hash_sum, st.hash_xor) == want
    rc, _ = _noalloc(lib, off, adj, g, 2, threads=threads, arena=arena + 1000, members=members)
    assert rc == E_SCRATCH
    # an arena of 40 words cannot hold a search frame and its lists
    rc, _ = _noalloc(lib, off, adj, g, 2, arena=40)
    assert rc == E_ARENA
    rc, st = _noalloc(lib, off, adj, g, 2)    # usable again after the failure
    assert rc == 0 and (st.count, st.hash_sum, st.hash_xor) == want
