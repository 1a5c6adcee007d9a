"""Multi-rank path on CPU: two gloo ranks each enumerate their shard of the
roots (the oracle stands in for a GPU's shard of the search tasks), then
combine their set summaries with gmkbe_b200.shard.  The combined summary must
equal the single-process summary, and the slowest rank's time must be the
maximum.  No GPU is touched."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import ROOT, golden_graph_path


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, name, k, q):
    import sys
    sys.path.insert(0, ROOT)
    import datetime
    import torch.distributed as dist
    import oracle as O
    from gmkbe_b200 import graphgen as gg
    from gmkbe_b200.shard import combine_max, combine_summary
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        g = gg.read_graph_bin(golden_graph_path(name))
        st = O.enumerate_oracle(g, k, shard=rank, nshards=world)
        summ = combine_summary(st.count, st.hash_sum, st.hash_xor)
        slowest = combine_max(float(rank + 1))
        if rank == 0:
            q.put((summ, slowest, st.count))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name,k", [("southernwomen", 2), ("er60", 1)])
def test_two_gloo_ranks_combine_to_the_full_set(golden, name, k):
    case = next(c for c in golden["cases"] if c["graph"] == name and c["k"] == k)
    want = (case["count"], int(case["hash_sum"], 16), int(case["hash_xor"], 16))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, name, k, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    summ, slowest, rank0_count = q.get(timeout=5)
    assert summ == want
    assert slowest == 2.0
    assert 0 < rank0_count < want[0]      # both shards did real work


def test_shards_partition_the_result_set(golden):
    import oracle as O
    from gmkbe_b200 import graphgen as gg
    g = gg.read_graph_bin(golden_graph_path("er60"))
    full = set(O.enumerate_oracle(g, 2, collect=True).results)
    parts = [set(O.enumerate_oracle(g, 2, collect=True, shard=s, nshards=3).results)
             for s in range(3)]
    assert sum(len(p) for p in parts) == len(full)
    assert set().union(*parts) == full
