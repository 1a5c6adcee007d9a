"""Multi-GPU runs: one process per GPU, each enumerating its shard of the
search tasks (gmk_opts.shard / nshards: task t goes to rank t % world).

The shards share nothing while they run.  At the end the per-rank set
summaries are combined once: counts and h1 sums add (mod 2^64), h2 values
xor.  NCCL and gloo have no xor reduction, so the three words of every rank
are all-gathered and combined on the host.  The combined summary equals the
single-GPU summary of the whole result set.
"""
from __future__ import annotations

MASK64 = (1 << 64) - 1


def _to_i64(v: int) -> int:
    v &= MASK64
    return v - (1 << 64) if v >= 1 << 63 else v


def combine_summary(count: int, hash_sum: int, hash_xor: int, device=None,
                    group=None) -> tuple[int, int, int]:
    """(count, sum of h1 mod 2^64, xor of h2) over all ranks of the default
    process group.  `device` is where the all-gather buffer lives (a CUDA
    device for nccl, None = CPU for gloo)."""
    import torch
    import torch.distributed as dist
    mine = torch.tensor([_to_i64(count), _to_i64(hash_sum), _to_i64(hash_xor)],
                        dtype=torch.int64, device=device)
    world = dist.get_world_size(group)
    parts = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(parts, mine, group=group)
    c = s = x = 0
    for p in parts:
        a, b, h = (int(v) & MASK64 for v in p.cpu().tolist())
        c += a
        s = (s + b) & MASK64
        x ^= h
    return c, s, x


def combine_max(value: float, device=None, group=None) -> float:
    """Largest value over the ranks (the slowest rank's time)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


# ----------------------------------------------------------------------------- recovery

def lpt_split(tasks, parts: int, part: int):
    """Part `part` of `parts` of a task array (fields root, first, last, cost,
    as gmk_plan_tasks returns), by the planner's rule: largest cost first, each
    task to the least-loaded part, lowest index on ties."""
    import numpy as np
    order = np.argsort(-np.asarray(tasks["cost"], np.float64), kind="stable")
    load = [0.0] * parts
    mine = []
    for i in order:
        best = min(range(parts), key=lambda p: (load[p], p))
        load[best] += max(float(tasks["cost"][i]), 1e-9)
        if best == part:
            mine.append(i)
    return tasks[np.asarray(mine, dtype=np.int64)]


def _put(store, key: str, summary) -> None:
    store.set(key, ",".join(str(int(v)) for v in summary))


def _get(store, key: str):
    return tuple(int(v) for v in store.get(key).decode().split(","))


def _wait(store, keys, deadline: float, poll_s: float) -> list:
    """Keys present by the deadline (polls; never blocks past it)."""
    import time
    while True:
        have = [k for k in keys if store.check([k])]
        if len(have) == len(keys) or time.monotonic() >= deadline:
            return have
        time.sleep(poll_s)


def run_with_recovery(store, rank: int, world: int, plan, run_tasks, wait_s: float = 30.0,
                      poll_s: float = 0.05, tag: str = "gmk"):
    """One sharded enumeration that survives ranks leaving between steps.

    plan(shard, nshards) -> that shard's task array (gmk_plan_tasks);
    run_tasks(tasks) -> (count, hash_sum, hash_xor) of exactly those tasks
    (Graph.enumerate(tasks=...) on a GPU).  Everything goes through the
    key-value store (a torch.distributed.TCPStore), so no collective ever
    waits on a rank that is gone.
      1. each rank runs its own shard and publishes its summary;
      2. ranks whose summary has not appeared within wait_s are taken as
         gone; the survivors (in rank order) split each missing shard's tasks
         by longest processing time, run their parts and publish them;
      3. every survivor combines all parts (counts and h1 add mod 2^64, h2
         xor).
    Returns (summary, missing ranks).  The store's host must survive; a rank
    that leaves during step 2 makes the others raise TimeoutError."""
    import time
    _put(store, f"{tag}/sum/{rank}", run_tasks(plan(rank, world)))
    keys = [f"{tag}/sum/{r}" for r in range(world)]
    have = _wait(store, keys, time.monotonic() + wait_s, poll_s)
    alive = sorted(int(k.rsplit("/", 1)[1]) for k in have)
    missing = [r for r in range(world) if r not in alive]
    me = alive.index(rank)
    for d in missing:
        part = lpt_split(plan(d, world), len(alive), me)
        _put(store, f"{tag}/rerun/{d}/{me}", run_tasks(part))
    parts = [f"{tag}/sum/{r}" for r in alive]
    parts += [f"{tag}/rerun/{d}/{i}" for d in missing for i in range(len(alive))]
    got = _wait(store, parts, time.monotonic() + wait_s, poll_s)
    if len(got) != len(parts):
        raise TimeoutError(f"rank {rank}: parts missing after recovery: "
                           f"{sorted(set(parts) - set(got))}")
    c = s = x = 0
    for k in parts:
        a, b, h = _get(store, k)
        c += a
        s = (s + b) & MASK64
        x ^= h & MASK64
    return (c, s, x), missing
