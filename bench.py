#!/usr/bin/env python
"""Benchmark: maximal k-biplexes/s of the B200 enumerator on the Chung-Lu
20k x 50k workload (gamma 2.1, max degree 2k, seed 2; k = 1, first 10^6
results), one JSON line on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gmk|reference]

A step is one enumeration of the workload up to the result limit.  `value` is
device-timed (CUDA events around the kernel, graph already resident);
`e2e` is the same metric through the public C ABI from pinned host CSR
arrays, host->device copy and the statistics read-back inside the timed
region.  L2 is flushed (256 MB write) between timed steps.  With N > 1 (one
process per GPU under torchrun) every rank enumerates its own shard of the
search tasks to the same result limit (weak scaling) and the slowest rank's
time is used.  `--impl reference` times the reference's own CPU enumerator
(BPPivot, built from its sources under oracle/_ref) on samples of the same
workload; under torchrun only rank 0 runs it.
"""
from __future__ import annotations

import argparse
import csv
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "maximal k-biplexes/sec, learned+batched vs plain GPU, bit-exact result set"
UNIT = "results/s"
WORKLOAD = "cl20k"
CONFIG_DESC = ("Chung-Lu bipartite |U|=20k |V|=50k ~500k edges (463,390 after dedup), "
               "exponent 2.1 both sides, max degree 2k, seed 2; k=1, first 10^6 results")
REF_STEP_SAMPLE = 100_000      # results per reference-arm step
CPU_BASELINE_SAMPLE = 200_000  # results in the GPU arm's cpu_baseline leg


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _traffic_per_launch(kernel: str):
    """DRAM bytes (read + write) per launch of `kernel` on this workload, from
    the committed ncu summary (profiles/<kernel>_cl20k.json), or None."""
    p = os.path.join(ROOT, "profiles", f"{kernel}_cl20k.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f).get("dram_bytes_per_launch")
    return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 50 ms, each sample
    time-stamped on arrival; stop() keeps the samples inside the timed window
    (the nearest one when the window is shorter than the sampling interval)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.p = None
        self.rows = []
        self.thread = None

    def _read(self):
        for line in self.p.stdout:
            r = next(csv.reader([line]), [])
            if len(r) >= 9:
                self.rows.append((time.perf_counter(), r))

    def start(self):
        """Starts sampling and waits (up to 5 s) for the first sample, so that
        the timed window that follows is covered."""
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "50"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        t_end = time.perf_counter() + 5.0
        while not self.rows and time.perf_counter() < t_end and self.p.poll() is None:
            time.sleep(0.01)

    def stop(self, t0: float, t1: float):
        if not self.p:
            return None
        time.sleep(0.06)                       # one more sample after the window
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.thread.join(timeout=5)
        if not self.rows:
            return None
        inside = [r for t, r in self.rows if t0 <= t <= t1]
        if not inside:
            mid = 0.5 * (t0 + t1)
            inside = [min(self.rows, key=lambda tr: abs(tr[0] - mid))[1]]
        sm = [float(r[1]) for r in inside if r[1].strip().replace(".", "").isdigit()]
        mx = max((float(r[2]) for r in inside if r[2].strip().replace(".", "").isdigit()), default=None)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in inside for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": reasons, "samples": len(inside)}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_reference(args, world, rank):
    """Reference arm: BPPivot (the reference's CPU enumerator) on the same workload."""
    if rank != 0:
        return
    import oracle as O
    from gmkbe_b200 import graphgen as gg
    path = gg.cached_workload(WORKLOAD)
    sample = min(args.limit, REF_STEP_SAMPLE)
    config = {"workload": CONFIG_DESC, "k": args.k, "result_limit": args.limit,
              "reference_sample_per_step": sample}
    if not os.path.exists(O.bppivot_path()):
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/bppivot not built (reference sources absent at build time)"}))
        return
    for _ in range(args.warmup):
        O.run_bppivot(path, args.k, result_limit=1000)
    tot_res = tot_ms = 0
    walls = []
    for _ in range(args.steps):
        r = O.run_bppivot(path, args.k, result_limit=sample)
        tot_res += r["count"]
        tot_ms += max(r["branch_ms"], 1)
        walls.append(r["wall_s"])
    value = tot_res / (tot_ms / 1e3)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded Chung-Lu, converter ordering)", "config": config,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                             "sample": f"first {sample} results of the workload per step, "
                                       "BPPivot -q 1 -k 1 -n <sample>, branch time "
                                       "(single-threaded; it has no parallel mode)"},
            "e2e": {"value": tot_res / sum(walls), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline(k):
    import oracle as O
    from gmkbe_b200 import graphgen as gg
    if not os.path.exists(O.bppivot_path()):
        return None
    r = O.run_bppivot(gg.cached_workload(WORKLOAD), k, result_limit=CPU_BASELINE_SAMPLE)
    return {"value": r["count"] / (max(r["branch_ms"], 1) / 1e3), "unit": UNIT, "cores": 1,
            "kind": "reference",
            "sample": f"first {CPU_BASELINE_SAMPLE} results of the workload (BPPivot -q 1 -k {k} "
                      f"-n {CPU_BASELINE_SAMPLE}), branch time {r['branch_ms']} ms, 1 thread"}


def run_gmk(args, world, rank, local):
    import numpy as np
    import torch
    import gmkbe_b200 as G
    from gmkbe_b200 import graphgen as gg

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    path = gg.cached_workload(WORKLOAD) if rank == 0 else None
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        path = gg.cached_workload(WORKLOAD)
    host = gg.read_graph_bin(path)
    off = torch.from_numpy(host.offsets.astype(np.uint32).view(np.int32)).pin_memory()
    adj = torch.from_numpy(host.adj.view(np.int32)).pin_memory()
    off_np = off.numpy().view(np.uint32)
    adj_np = adj.numpy().view(np.uint32)
    h2d = 4 * (off_np.size + adj_np.size)
    kw = dict(k=args.k, result_limit=args.limit, schedule=args.schedule, engine=args.engine)
    if world > 1:
        kw.update(shard=rank, nshards=world)

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    dg = G.Graph.from_csr(off_np, adj_np, host.n, host.n_left, device=local)
    flush_buf = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    for _ in range(args.warmup):
        dg.enumerate(**kw)
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    t_clk0 = time.perf_counter()
    ms, count, algo, launches = [], 0, 0, 0
    for _ in range(args.steps):
        flush_buf.zero_()          # L2 flush, outside the timed kernel
        torch.cuda.synchronize()
        st = dg.enumerate(**kw)
        ms.append(st.kernel_ms)
        count += st.count
        algo += st.algo_bytes
        launches += st.rounds
    barrier()
    clk = clocks.stop(t_clk0, time.perf_counter())
    # the plain static schedule on the same GPU (one task per root, no splitting)
    plain = None
    if args.schedule != "plain" and not args.no_plain:
        flush_buf.zero_()
        torch.cuda.synchronize()
        sp = dg.enumerate(**dict(kw, schedule="plain"))
        plain = {"value": sp.count / (sp.kernel_ms / 1e3), "ms": sp.kernel_ms,
                 "results": sp.count}
    # end to end through the C ABI: host CSR -> device, enumerate, read back.
    # W untimed steps first, like the device arm (the first upload of a second
    # graph fills the device buffer cache)
    for _ in range(args.warmup):
        with G.Graph.from_csr(off_np, adj_np, host.n, host.n_left, device=local) as g2:
            g2.enumerate(**kw)
    barrier()
    e2e_s, e2e_rounds = 0.0, 0
    for _ in range(args.steps):
        flush_buf.zero_()
        barrier()
        t0 = time.perf_counter()
        g2 = G.Graph.from_csr(off_np, adj_np, host.n, host.n_left, device=local)
        st2 = g2.enumerate(**kw)
        g2.close()
        e2e_s += time.perf_counter() - t0
        e2e_rounds += st2.rounds
    barrier()
    tot_ms = sum(ms)
    if world > 1:
        from gmkbe_b200.shard import combine_max, combine_summary
        dev = f"cuda:{local}"
        tot_ms_max = combine_max(tot_ms, device=dev)
        e2e_max = combine_max(e2e_s, device=dev)
        count_all = float(combine_summary(count, 0, 0, device=dev)[0])
    else:
        tot_ms_max, e2e_max, count_all = tot_ms, e2e_s, float(count)
    # counters read back after every round: 32 B round counters + 88 B totals
    d2h = 120 * e2e_rounds / max(1, args.steps)
    if rank == 0:
        peak, peak_kind = _peaks()
        achieved = (algo / args.steps) / (tot_ms / args.steps / 1e3) / 1e9
        line = {
            "metric": METRIC, "value": count_all / (tot_ms_max / 1e3), "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": tot_ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded Chung-Lu, converter ordering)",
            "config": {"workload": CONFIG_DESC, "k": args.k, "result_limit": args.limit,
                       "schedule": args.schedule, "l2": "flushed between steps (256 MB write)",
                       "parallelism": f"task shards x{world}" if world > 1 else "1 GPU"},
            "e2e": {"value": count_all / e2e_max, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": _traffic_per_launch("enumerate_warp_kernel" if args.engine == "warp"
                                                        else "enumerate_kernel"),
                         "peak_source": peak_kind,
                         "kernel": ("enumerate_warp_kernel" if args.engine == "warp"
                                    else "enumerate_kernel"),
                         "algorithmic_bytes_per_launch": algo / args.steps},
            "clocks": clk,
            "stats": {"nodes_per_step": st.nodes, "tasks": st.tasks, "tasks_done": st.tasks_done,
                      "threads": st.threads, "rounds_per_step": launches / args.steps,
                      "engine": args.engine},
            "plain_schedule": plain,
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(args.k)
        print(json.dumps(line), flush=True)
    dg.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gmk", choices=["gmk", "reference"])
    ap.add_argument("--k", type=int, default=1)
    ap.add_argument("--limit", type=int, default=1_000_000)
    ap.add_argument("--schedule", default="batched", choices=["plain", "batched"])
    ap.add_argument("--engine", default="warp", choices=["warp", "thread"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-schedule comparison")
    args = ap.parse_args()
    world, rank, local = _dist()
    if args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_gmk(args, world, rank, local)


if __name__ == "__main__":
    main()
