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
