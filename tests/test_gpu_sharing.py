"""In-launch work sharing: busy warps hand the shallowest unexplored part of
their search tree to idle warps inside the same launch.  The result set must
not depend on it -- with aggressive donation (after 1 node), the default, or
none -- and on complete enumerations donations must actually happen."""
import pytest

import gmkbe_b200 as G
from conftest import golden_graph_path

pytestmark = pytest.mark.gpu

CASES = [("southernwomen", 1), ("southernwomen", 2), ("southernwomen", 3), ("crime", 1),
         ("er200", 1), ("cl20k_sub", 1), ("er60", 1), ("er60", 2)]


def _want(golden, name, k):
    case = next(c for c in golden["cases"] if c["graph"] == name and c["k"] == k)
    return case["count"], int(case["hash_sum"], 16), int(case["hash_xor"], 16)


@pytest.mark.parametrize("name,k", CASES)
@pytest.mark.parametrize("donate_min_nodes", [1, 0, 512])
def test_sharing_leaves_the_set_unchanged(golden, name, k, donate_min_nodes):
    with G.Graph.load(golden_graph_path(name)) as g:
        st = g.enumerate(k=k, donate_min_nodes=donate_min_nodes)
    assert st.summary() == _want(golden, name, k)


@pytest.mark.parametrize("name,k", [("er200", 1), ("southernwomen", 3), ("er60", 2)])
def test_complete_runs_donate_and_need_fewer_launches(golden, name, k):
    with G.Graph.load(golden_graph_path(name)) as g:
        shared = g.enumerate(k=k)
        rounds_only = g.enumerate(k=k, sharing=False)
    assert shared.summary() == rounds_only.summary() == _want(golden, name, k)
    assert shared.donations > 0
    assert rounds_only.donations == 0
    assert shared.rounds < rounds_only.rounds


def test_sharing_with_small_chunks_and_thread_counts(golden):
    # few warps and many tiny tasks: donation and the root queue interleave
    with G.Graph.load(golden_graph_path("er200")) as g:
        for threads in (64, 1024, 8192):
            st = g.enumerate(k=1, chunk=2, threads=threads, donate_min_nodes=4)
            assert st.summary() == _want(golden, "er200", 1), threads


def test_sharing_under_a_result_limit_stops_exactly():
    with G.Graph.load(golden_graph_path("er200")) as g:
        st = g.enumerate(k=1, result_limit=100_000, donate_min_nodes=1)
    assert st.count == 100_000 and st.truncated
