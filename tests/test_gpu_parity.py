"""Parity of the CUDA enumerator (through the C ABI) with the oracle and with
the golden summaries of the reference's BPPivot output."""
import os

import numpy as np
import pytest

import gmkbe_b200 as G
import oracle as O
from gmkbe_b200 import graphgen as gg
from conftest import GOLDEN, golden_graph_path

pytestmark = pytest.mark.gpu


def _summary(case):
    return case["count"], int(case["hash_sum"], 16), int(case["hash_xor"], 16)


@pytest.fixture(scope="module")
def graphs():
    cache = {}

    def get(name):
        if name not in cache:
            cache[name] = G.Graph.load(golden_graph_path(name))
        return cache[name]
    yield get
    for g in cache.values():
        g.close()


GOLDEN_CASES = [("southernwomen", 1), ("southernwomen", 2), ("southernwomen", 3), ("crime", 1),
                ("er200", 1), ("cl20k_sub", 1), ("er60", 1), ("er60", 2)]


@pytest.mark.parametrize("name,k", GOLDEN_CASES)
def test_golden_full_enumeration(golden, graphs, name, k):
    case = next(c for c in golden["cases"] if c["graph"] == name and c["k"] == k)
    st = graphs(name).enumerate(k=k)
    assert not st.truncated
    assert st.summary() == _summary(case)


@pytest.mark.parametrize("schedule,chunk", [("plain", 0), ("batched", 1), ("batched", 3),
                                            ("batched", 64)])
def test_schedule_does_not_change_the_set(golden, graphs, schedule, chunk):
    case = next(c for c in golden["cases"] if c["graph"] == "southernwomen" and c["k"] == 2)
    st = graphs("southernwomen").enumerate(k=2, schedule=schedule, chunk=chunk)
    assert st.summary() == _summary(case)


@pytest.mark.parametrize("split_min_nodes", [1, 7])
def test_tree_splitting_does_not_change_the_set(golden, graphs, split_min_nodes):
    # a tiny split threshold splits almost every task into the next round
    for name, k in [("southernwomen", 2), ("er60", 2), ("er200", 1)]:
        case = next(c for c in golden["cases"] if c["graph"] == name and c["k"] == k)
        st = graphs(name).enumerate(k=k, chunk=2, split_min_nodes=split_min_nodes)
        assert st.summary() == _summary(case), (name, k, split_min_nodes)
        assert st.rounds >= 1


@pytest.mark.parametrize("k", [1, 2])
def test_thread_engine_matches_warp_engine(golden, graphs, k):
    # crime has over 10^8 maximal 2-biplexes: it is compared at k = 1 only
    for name in ("southernwomen", "er60") + (("crime",) if k == 1 else ()):
        hit = [c for c in golden["cases"] if c["graph"] == name and c["k"] == k]
        st_t = graphs(name).enumerate(k=k, engine="thread")
        st_w = graphs(name).enumerate(k=k, engine="warp")
        assert st_t.summary() == st_w.summary(), name
        if hit:
            assert st_w.summary() == _summary(hit[0]), name


def test_ordered_schedule_same_set(golden, graphs):
    case = next(c for c in golden["cases"] if c["graph"] == "er60" and c["k"] == 2)
    g = graphs("er60")
    cost = np.random.default_rng(0).random(g.n_left).astype(np.float32)
    st = g.enumerate(k=2, schedule="ordered", task_cost=cost)
    assert st.summary() == _summary(case)


def test_thread_and_arena_shapes_do_not_change_the_set(golden, graphs):
    case = next(c for c in golden["cases"] if c["graph"] == "er200" and c["k"] == 1)
    # 4096 threads = 128 warps: few enough that warps take many tasks each
    for threads, pair_limit in [(4096, 64), (8192, 256), (0, 1 << 20)]:
        st = graphs("er200").enumerate(k=1, threads=threads, pair_limit=pair_limit)
        assert st.summary() == _summary(case), (threads, pair_limit)
    # pair_limit 1 turns the node rules off almost everywhere: a far larger tree
    small = next(c for c in golden["cases"] if c["graph"] == "er60" and c["k"] == 1)
    assert graphs("er60").enumerate(k=1, pair_limit=1).summary() == _summary(small)


@pytest.mark.parametrize("out_words", [600, 4096])
def test_streamed_records_through_small_buffers(golden, graphs, out_words):
    # a record buffer far smaller than the output: rounds wind down whenever
    # it is half full, and the host drains it while the next round runs
    case = next(c for c in golden["cases"] if c["graph"] == "er60" and c["k"] == 2)
    got = []
    st = graphs("er60").enumerate(k=2, sink=lambda x, y: got.append((x, y)) and False,
                                  out_words=out_words)
    assert st.rounds > 5
    assert O.set_summary(got) == _summary(case) == st.summary()
    assert len(got) == len(set(got))


def test_streamed_records_with_limit(graphs):
    got = []
    st = graphs("er200").enumerate(k=1, result_limit=30_000, out_words=2048,
                                   sink=lambda x, y: got.append((x, y)) and False)
    assert st.count == 30_000 == len(got) == len(set(got))


def test_emitted_sets_equal_reference_sets(graphs):
    want = []
    with open(os.path.join(GOLDEN, "southernwomen_k1_sets.txt")) as f:
        for line in f:
            xs, ys = line.split("|")
            want.append((tuple(map(int, xs.split())), tuple(map(int, ys.split()))))
    st = graphs("southernwomen").enumerate(k=1, collect=True)
    assert sorted(st.results) == sorted(want)


@pytest.mark.parametrize("k", [1, 2, 3])
def test_random_graphs_against_oracle(k):
    # the search tree grows steeply with k; sides are kept small enough that
    # the oracle finishes each graph in well under a second
    hi = {1: 25, 2: 20, 3: 12}[k]
    for seed in range(12):
        rng = np.random.default_rng(100 + seed)
        nu, nv = int(rng.integers(3, hi)), int(rng.integers(3, hi))
        g = gg.erdos_renyi(nu, nv, float(rng.uniform(0.1, 0.5)), 100 + seed)
        if g.n_left in (0, g.n):
            continue
        want = O.enumerate_oracle(g, k).summary()
        with G.Graph.from_graph(g) as dg:
            got = dg.enumerate(k=k, chunk=int(rng.integers(1, 6))).summary()
        assert got == want, (seed, k)


def test_chung_lu_small_against_oracle():
    g = gg.chung_lu(400, 700, 1500, 2.1, 11, max_deg=80)
    want = O.enumerate_oracle(g, 1).summary()
    with G.Graph.from_graph(g) as dg:
        assert dg.enumerate(k=1).summary() == want


@pytest.mark.parametrize("seed", [21, 22, 23])
def test_small_subtree_solver_against_oracle_and_records(seed):
    # Sparse k = 1 graphs: most local nodes hold at most six candidates, so the
    # k = 1 kernels test their subsets at once (solve_small).  Count mode, record
    # mode (streamed through the smallest record buffer the warp engine takes,
    # so rounds wind down and nodes defer), a limited record run, and the
    # thread engine (no solver) must all give the oracle's set.
    g = gg.chung_lu(150, 260, 420, 2.1, seed, max_deg=30)   # 65-73 k results each
    want = O.enumerate_oracle(g, 1).summary()
    with G.Graph.from_graph(g) as dg:
        assert dg.enumerate(k=1).summary() == want
        assert dg.enumerate(k=1, engine="thread").summary() == want
        for out_words in (0, 160):
            sets = []
            st = dg.enumerate(k=1, sink=lambda x, y: sets.append((tuple(x), tuple(y))),
                              out_words=out_words)
            assert st.summary() == want
            assert len(sets) == want[0] and O.set_summary(sets) == want
        st = dg.enumerate(k=1, result_limit=max(1, want[0] // 3), collect=True)
        assert st.count == len(st.results) == max(1, want[0] // 3)
        assert len(set(st.results)) == st.count


HUB_CASES = [(3, 6, 72, 4, 2, 1), (4, 8, 80, 4, 2, 2), (4, 4, 66, 4, 3, 5), (4, 5, 70, 5, 3, 3)]


@pytest.mark.parametrize("n_hubs,n_sparse,n,d,k,seed", HUB_CASES)
def test_long_list_filter_bitmaps_against_oracle(n_hubs, n_sparse, n, d, k, seed):
    # k >= 2 nodes that branch on a list of 64 or more candidates filter their
    # children through per-frame bitmaps; with k + 1 hubs in S the U list holds
    # all n U vertices.  Count mode, split records (restored frames carry no
    # bitmaps) and streamed records must all give the oracle's set.
    g = gg.hubs_and_sparse(n_hubs, n_sparse, n, d, seed)
    want = O.enumerate_oracle(g, k).summary()
    with G.Graph.from_graph(g) as dg:
        assert dg.enumerate(k=k).summary() == want
        assert dg.enumerate(k=k, chunk=4, split_min_nodes=3).summary() == want
        if k == 2:   # the k = 3 cases hold 0.5-1 M sets: count mode only
            sets = []
            st = dg.enumerate(k=k, sink=lambda x, y: sets.append((tuple(x), tuple(y))))
            assert st.summary() == want
            assert len(sets) == want[0] and O.set_summary(sets) == want


# ---------------------------------------------------------------- edge cases

def test_single_edge():
    g = gg.relabel(np.array([0]), np.array([0]))
    with G.Graph.from_graph(g) as dg:
        st = dg.enumerate(k=1, collect=True)
    assert st.results == [((0,), (1,))]


def test_complete_bipartite_is_one_result():
    u, v = np.meshgrid(np.arange(6), np.arange(5), indexing="ij")
    g = gg.relabel(u.ravel(), v.ravel())
    for k in (1, 2, 3):
        with G.Graph.from_graph(g) as dg:
            st = dg.enumerate(k=k, collect=True)
        assert st.results == [(tuple(range(6)), tuple(range(6, 11)))]


def test_star_and_matching_against_definition():
    # a star plus a perfect matching: many disconnected maximal 1-biplexes
    u = np.array([0, 0, 0, 0, 1, 2, 3, 4])
    v = np.array([0, 1, 2, 3, 4, 5, 6, 7])
    g = gg.relabel(u, v)
    for k in (1, 2):
        want = sorted(O.brute_force(g, k)) if g.n <= 16 else None
        with G.Graph.from_graph(g) as dg:
            got = sorted(dg.enumerate(k=k, collect=True).results)
        assert got == want


def test_empty_side_has_no_results():
    off = np.zeros(4, np.uint32)          # three U vertices, no V, no edges
    with G.Graph.from_csr(off, np.zeros(0, np.uint32), 3, 3) as dg:
        assert dg.enumerate(k=1).count == 0


def test_bad_csr_rejected():
    off = np.array([0, 1, 2], np.uint32)
    adj = np.array([0, 0], np.uint32)     # U vertex 0 adjacent to itself: not bipartite
    with pytest.raises(G.GmkError) as e:
        G.Graph.from_csr(off, adj, 2, 1)
    assert e.value.code == -3


def test_result_limit_exact_in_record_mode(graphs):
    st = graphs("er200").enumerate(k=1, result_limit=5000, collect=True)
    assert st.count == 5000 and len(st.results) == 5000 and st.truncated
    g = gg.read_graph_bin(golden_graph_path("er200"))
    for x, y in st.results[::250]:
        assert O.classify(g, 1, x, y) == 2


def test_result_limit_count_mode(graphs):
    st = graphs("er200").enumerate(k=1, result_limit=100000)
    assert st.count == 100000 and st.truncated


def test_small_arena_reports_error_not_fault(graphs):
    # the per-thread engine cannot split: an arena too small for its search
    # is an error; for the warp engine, 20 words cannot hold a task's base
    # frame and its first child
    with pytest.raises(G.GmkError) as e:
        graphs("er200").enumerate(k=1, arena_words=40, engine="thread")
    assert e.value.code == -6
    with pytest.raises(G.GmkError) as e:
        graphs("er200").enumerate(k=1, arena_words=20)
    assert e.value.code == -6
    # the context stays usable
    assert graphs("er60").enumerate(k=1).count == 8041


@pytest.mark.parametrize("schedule", ["batched", "plain"])
def test_paths_that_outgrow_the_arena_move_to_the_next_round(golden, graphs, schedule):
    # a child (or a node's scratch) that does not fit sends the task's path to
    # the next round, each frame at the bottom of an empty arena: the set is
    # unchanged and only extra rounds show it.  Arenas from barely two frames
    # up: every run that succeeds is exact, the rest report GMK_E_ARENA (a
    # base frame that cannot hold one child), and some succeed after moving
    # paths (more than one round).
    moved = 0
    for name, k in [("er200", 1), ("crime", 1), ("southernwomen", 2), ("er60", 2)]:
        case = next(c for c in golden["cases"] if c["graph"] == name and c["k"] == k)
        for arena in (36, 48, 64, 96, 128, 192):
            try:
                st = graphs(name).enumerate(k=k, arena_words=arena, schedule=schedule)
            except G.GmkError as e:
                assert e.code == -6, (name, arena, e)
                continue
            assert st.summary() == _summary(case), (name, k, arena)
            moved += st.rounds > 1
    assert moved > 0


def test_watchdog_returns_status():
    g = gg.erdos_renyi(300, 300, 0.05, 5)
    with G.Graph.from_graph(g) as dg:
        with pytest.raises(G.GmkError) as e:
            dg.enumerate(k=3, watchdog_ms=20)
        assert e.value.code == -8
        assert dg.enumerate(k=1, result_limit=10).count == 10


def test_limited_run_at_full_size():
    path = gg.cached_workload("cl20k")
    with G.Graph.load(path) as dg:
        st = dg.enumerate(k=1, result_limit=1_000_000)
        assert st.count == 1_000_000 and st.truncated
        sample = dg.enumerate(k=1, result_limit=2000, collect=True)
    g = gg.read_graph_bin(path)
    assert len(set(sample.results)) == 2000
    for x, y in sample.results[::100]:
        assert O.classify(g, 1, x, y) == 2


def test_autotuner_picks_a_setting_and_caches_it(golden, tmp_path):
    # every knob is tried (k = 2 also tries the intersection strategy); the
    # winner is cached per fingerprint, and no setting changes the result set
    from gmkbe_b200 import autotune
    cache = str(tmp_path / "tune.json")
    want = _summary(next(c for c in golden["cases"] if c["graph"] == "er60" and c["k"] == 2))
    h = gg.read_graph_bin(golden_graph_path("er60"))
    with G.Graph.from_graph(h) as g:
        cost = g.root_costs()
        first = autotune.tune(g, h, 2, cost, repeats=1, cache_path=cache)
        assert not first["cached"] and first["results"] == want[0]
        assert first["settings"] in [t["settings"] for t in first["trials"]]
        tried = {kn for t in first["trials"] for kn, v in t["settings"].items()
                 if v != autotune.DEFAULTS[kn]}
        assert tried == set(autotune.CHOICES)
        again = autotune.tune(g, h, 2, cost, cache_path=cache)
        assert again["cached"] and again["settings"] == first["settings"]
        buckets = autotune.degree_buckets(h, g.n_left)
        for t in first["trials"]:
            kw = autotune.apply(g, t["settings"], cost, buckets, 4144 * 32)
            assert g.enumerate(k=2, **kw).summary() == want, t["settings"]


@pytest.mark.parametrize("load", [10, 25, 90, 100])
def test_edge_hash_load_keeps_the_set(golden, load):
    with G.Graph.load(golden_graph_path("crime")) as g:
        g.set_hash_load(load)
        st = g.enumerate(k=1)
    assert st.summary() == _summary(next(c for c in golden["cases"] if c["graph"] == "crime"
                                         and c["k"] == 1))


@pytest.mark.parametrize("bits_min", [1, 2, 32, 0xFFFFFFFF])
def test_intersection_strategy_keeps_the_set(bits_min):
    # bitmaps for every list (1), for lists of two or more, or never (probes)
    g = gg.hubs_and_sparse(4, 60, 150, 3, 7)
    with G.Graph.from_graph(g) as dg:
        want = O.enumerate_oracle(g, 2).summary()
        assert dg.enumerate(k=2, bits_min_list=bits_min).summary() == want
