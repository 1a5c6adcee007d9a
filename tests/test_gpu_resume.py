"""Checkpoint / resume (gmk_enumerate_resumable) on the GPU: a run paused
after a few batches of roots and resumed from its checkpoint file gives the
same set as one uninterrupted run; a checkpoint written for another k or graph
is refused."""
import os

import pytest

import gmkbe_b200 as G
from conftest import golden_graph_path

pytestmark = pytest.mark.gpu


def _summary(case):
    return case["count"], int(case["hash_sum"], 16), int(case["hash_xor"], 16)


def test_pause_and_resume_gives_the_full_set(golden, tmp_path):
    case = next(c for c in golden["cases"] if c["graph"] == "er200" and c["k"] == 1)
    ck = str(tmp_path / "run.ckpt")
    with G.Graph.load(golden_graph_path("er200")) as g:
        st, paused = g.enumerate_resumable(ck, batch_roots=16, max_batches=3, k=1)
        assert paused and 0 < st.count < case["count"]
        text = open(ck).read()
        assert "next_root 48" in text and "done 0" in text
        st, paused = g.enumerate_resumable(ck, batch_roots=16, max_batches=2, k=1)
        assert paused
        st, paused = g.enumerate_resumable(ck, batch_roots=16, k=1)
        assert not paused
        assert st.summary() == _summary(case)
        assert "done 1" in open(ck).read()
        # a finished checkpoint returns the totals without work
        st2, paused = g.enumerate_resumable(ck, batch_roots=16, k=1)
        assert not paused and st2.summary() == _summary(case) and st2.rounds == 0


def test_resume_delivers_each_result_once(tmp_path):
    ck = str(tmp_path / "sw.ckpt")
    with G.Graph.load(golden_graph_path("southernwomen")) as g:
        want = sorted(g.enumerate(k=2, collect=True).results)
        got = []
        paused = True
        while paused:
            st, paused = g.enumerate_resumable(ck, batch_roots=2, max_batches=1, k=2,
                                               sink=lambda x, y: got.append((x, y)) and False)
        assert sorted(got) == want and len(got) == len(set(got))


def test_checkpoint_for_other_k_or_graph_is_refused(tmp_path):
    ck = str(tmp_path / "x.ckpt")
    with G.Graph.load(golden_graph_path("er60")) as g:
        g.enumerate_resumable(ck, batch_roots=4, max_batches=1, k=1)
        with pytest.raises(G.GmkError) as e:
            g.enumerate_resumable(ck, batch_roots=4, k=2)
        assert e.value.code == -12
    with G.Graph.load(golden_graph_path("southernwomen")) as g2:
        with pytest.raises(G.GmkError) as e:
            g2.enumerate_resumable(ck, batch_roots=4, k=1)
        assert e.value.code == -12
    with open(ck, "w") as f:
        f.write("garbage\n")
    with G.Graph.load(golden_graph_path("er60")) as g:
        with pytest.raises(G.GmkError) as e:
            g.enumerate_resumable(ck, k=1)
        assert e.value.code == -12


def test_result_limit_across_resume(tmp_path):
    ck = str(tmp_path / "lim.ckpt")
    with G.Graph.load(golden_graph_path("er200")) as g:
        paused = True
        while paused:
            st, paused = g.enumerate_resumable(ck, batch_roots=8, max_batches=2, k=1,
                                               result_limit=50_000)
        assert st.count == 50_000 and st.truncated
    assert os.path.exists(ck)


def test_checkpoint_for_other_shard_or_limit_is_refused(tmp_path):
    # a checkpoint records the task set it covers: shard, shard count and
    # result limit must match, or counts from two task sets would mix
    ck = str(tmp_path / "sh.ckpt")
    with G.Graph.load(golden_graph_path("er60")) as g:
        g.enumerate_resumable(ck, batch_roots=4, max_batches=1, k=1, shard=0, nshards=2)
        text = open(ck).read()
        assert "shard 0\nnshards 2\nresult_limit 0\n" in text
        for kw in (dict(shard=1, nshards=2), dict(shard=0, nshards=3), dict(shard=0, nshards=1),
                   dict(shard=0, nshards=2, result_limit=10)):
            with pytest.raises(G.GmkError) as e:
                g.enumerate_resumable(ck, batch_roots=4, k=1, **kw)
            assert e.value.code == -12, kw
        # the matching run resumes
        st, paused = g.enumerate_resumable(ck, batch_roots=4, k=1, shard=0, nshards=2)
        assert not paused and st.count > 0
