"""Multi-rank path on CPU (no GPU touched).

Each gloo rank takes its shard of the library's own task partition
(gmk_plan_tasks: longest processing time over the root-cost proxy, the
partition gmk_enumerate uses for shard/nshards) and enumerates exactly those
tasks -- the oracle stands in for the GPU: a result belongs to the task whose
root is its smallest U vertex and whose child range holds its smallest V
vertex.  The combined summary must equal the golden one.  A second test makes
a rank leave between steps: the survivors see its summary missing from the
store, split its shard among themselves and still combine to the full set."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT, golden_graph_path


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _task_runner(name, k):
    """(plan(shard, nshards), run_tasks(tasks)) over the oracle's result set."""
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle as O
    import gmkbe_b200 as G
    from gmkbe_b200 import graphgen as gg
    from test_plan import proxy_cost
    g = gg.read_graph_bin(golden_graph_path(name))
    cost = proxy_cost(g)
    results = O.enumerate_oracle(g, k, collect=True).results

    def plan(shard, nshards):
        return G.plan_tasks(g.n, g.n_left, cost, target_tasks=64, nshards=nshards, shard=shard)

    def run_tasks(tasks):
        keys = {(int(t["root"]), int(t["first"]), int(t["last"])) for t in tasks}
        roots = {}
        for r, f, l in keys:
            roots.setdefault(r, []).append((f, l))
        mine = [(x, y) for x, y in results
                if any(f <= min(y) < l for f, l in roots.get(min(x), ()))]
        return O.set_summary(mine)
    return plan, run_tasks


def _rank_main(rank, world, port, name, k, q):
    import sys
    sys.path.insert(0, ROOT)
    import datetime
    import torch.distributed as dist
    from gmkbe_b200.shard import combine_max, combine_summary
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        plan, run_tasks = _task_runner(name, k)
        c, s, x = run_tasks(plan(rank, world))
        summ = combine_summary(c, s, x)
        slowest = combine_max(float(rank + 1))
        if rank == 0:
            q.put((summ, slowest, c))
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


def _recovery_main(rank, world, port, store_port, name, k, leaver, q):
    import sys
    sys.path.insert(0, ROOT)
    import datetime
    import torch.distributed as dist
    from gmkbe_b200.shard import run_with_recovery
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=30))
    store = dist.TCPStore("127.0.0.1", store_port, world, rank == 0,
                          timeout=datetime.timedelta(seconds=30))
    if rank == leaver:
        # leaves between steps: joined the job, runs nothing, publishes nothing
        os._exit(3)
    plan, run_tasks = _task_runner(name, k)
    summ, missing = run_with_recovery(store, rank, world, plan, run_tasks, wait_s=5.0)
    q.put((rank, summ, missing))
    q.close()
    q.join_thread()        # the queue's feeder thread must deliver before os._exit
    # the store's host stays up until every survivor has combined
    store.add("gmk/finished", 1)
    if rank == 0:
        import time
        t_end = time.monotonic() + 30
        while store.add("gmk/finished", 0) < world - 1 and time.monotonic() < t_end:
            time.sleep(0.05)
    os._exit(0)


def test_a_rank_that_leaves_is_covered_by_the_survivors(golden):
    case = next(c for c in golden["cases"] if c["graph"] == "er60" and c["k"] == 2)
    want = (case["count"], int(case["hash_sum"], 16), int(case["hash_xor"], 16))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port, store_port = _free_port(), _free_port()
    world, leaver = 3, 2
    procs = [ctx.Process(target=_recovery_main,
                         args=(r, world, port, store_port, "er60", 2, leaver, q))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    codes = [p.exitcode for p in procs]
    assert codes == [0, 0, 3], codes
    got = sorted(q.get(timeout=5) for _ in range(world - 1))
    for rank, summ, missing in got:
        assert missing == [leaver]
        assert summ == want, rank
