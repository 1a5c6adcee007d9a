#!/usr/bin/env python
"""Benchmark: maximal k-biplexes/s of the B200 enumerator, learned+batched
schedule against the plain GPU schedule, bit-exact result set; one JSON line
on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gmk|reference]

Workload (the headline `value`): the exactness case of cl20k -- the
Chung-Lu graph |U| = 20k, |V| = 50k (exponent 2.1, max degree 2k, seed 2),
complete enumeration of the subgraph induced by its first 5k U and 12k V ids
(tests/golden/cl20k_sub.graph.bin: 623 x 653 vertices, 660 edges, 245 860
maximal 1-biplexes), k = 1.  A step is one complete enumeration; every step's
set summary (count, sum and xor of per-result hashes) is checked against the
golden summary of the reference's BPPivot output, so each timed step is
bit-exact.  The schedule is learned+batched: the shipped subtree-size model
(gmkbe_b200/models/subtree.npy) predicts every root's cost, the planner splits
and orders the tasks by it, and the persistent kernel shares work inside the
launch.  `value` is device-timed (CUDA events around the enumeration's
launches, graph and predictions resident); `e2e` is the same metric through the
public API from pinned host CSR arrays: upload, device CSR check, edge-hash
build, root features, model prediction, planning, enumeration and read-back
all inside the timed region.  L2 is flushed (256 MB write) between steps.

Beside it: the plain schedule (one task per root, id order, no splitting) and
the batched schedule without the model on the same graph; cl20k's throughput
run (full graph, first 10^6 results) and the Chung-Lu 100k x 300k (cl100k) and
500k x 1M (cl500k) graphs (first 10^7 / 10^8 results) under the three
schedules; and complete enumerations of the Erdos-Renyi 200 x 200 graph (er200)
and of subgraphs of cl100k and cl500k.
`--impl reference` times the reference's own CPU enumerator (BPPivot, built
from its sources under oracle/_ref) on the same complete enumeration.  With
N > 1 (one process per GPU under torchrun) every rank runs its shard of the
planned tasks of the same complete enumeration (strong scaling: the total work
is fixed) and the slowest rank's time is used.
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
WORKLOAD = "cl20k_sub"
WORKLOAD_PATH = os.path.join(ROOT, "tests", "golden", "cl20k_sub.graph.bin")
CONFIG_DESC = ("cl20k: Chung-Lu bipartite |U|=20k |V|=50k ~500k edges, exponent 2.1, max "
               "degree 2k, seed 2; complete enumeration of the subgraph induced by the first 5k U "
               "and 12k V ids (623 x 653 vertices, 660 edges after dropping isolated vertices), "
               "k=1, 245860 maximal 1-biplexes, bit-exact against BPPivot")
K = 1


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured", float(d.get("sm_max_mhz", 1965.0))
    return 6650.0, "fallback", 1965.0


def _profile(name: str):
    """A committed ncu summary (profiles/<name>.json), or None."""
    p = os.path.join(ROOT, "profiles", name + ".json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return None


def _algo_bytes(workload: str, k: int, limit: int):
    """Algorithmic bytes of (workload, k, limit) counted by the host restatement
    (profiles/algo_bytes.json, written by oracle/algo_bytes.py), or None."""
    d = _profile("algo_bytes")
    for c in (d or {}).get("cases", []):
        if c["workload"] == workload and c["k"] == k and c["result_limit"] == limit:
            return c
    return None


def _golden(name: str, k: int):
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        for c in json.load(f)["cases"]:
            if c["graph"] == name and c["k"] == k:
                return c["count"], int(c["hash_sum"], 16), int(c["hash_xor"], 16)
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
    """Reference arm: BPPivot (the reference's CPU enumerator) on the same
    complete enumeration, one thread (it has no parallel mode)."""
    if rank != 0:
        return
    import oracle as O
    config = {"workload": CONFIG_DESC, "k": K, "result_limit": 0, "complete": True}
    if not os.path.exists(O.bppivot_path()):
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/bppivot not built (reference sources absent at build time)"}))
        return
    want = _golden(WORKLOAD, K)
    for _ in range(args.warmup):
        O.run_bppivot(WORKLOAD_PATH, K)
    tot_res = tot_ms = 0
    walls = []
    for _ in range(args.steps):
        r = O.run_bppivot(WORKLOAD_PATH, K)
        assert r["count"] == want[0], (r["count"], want)
        tot_res += r["count"]
        tot_ms += max(r["branch_ms"], 1)
        walls.append(r["wall_s"])
    value = tot_res / (tot_ms / 1e3)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot_ms / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded Chung-Lu, converter ordering)", "config": config,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                             "sample": "the complete enumeration per step (BPPivot -q 1 -k 1, "
                                       "branch time; single-threaded, it has no parallel mode)"},
            "e2e": {"value": tot_res / sum(walls), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline():
    """BPPivot's complete enumeration of the workload on this host, one thread."""
    import oracle as O
    if not os.path.exists(O.bppivot_path()):
        return None
    r = O.run_bppivot(WORKLOAD_PATH, K)
    return {"value": r["count"] / (max(r["branch_ms"], 1) / 1e3), "unit": UNIT, "cores": 1,
            "kind": "reference",
            "sample": f"the complete enumeration ({r['count']} results), BPPivot -q 1 -k {K}, "
                      f"branch time {r['branch_ms']} ms, wall {r['wall_s']:.2f} s, 1 thread",
            "cpu": _cpu_model()}


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip() + f" ({os.cpu_count()} threads)"
    except OSError:
        pass
    return None


def _model(device: int):
    """The shipped subtree-size model, or one trained now (and said so)."""
    from gmkbe_b200 import learned as L
    if os.path.exists(L.MODEL_PATH):
        return L.load_default(device), "shipped (gmkbe_b200/models/subtree.npy)"
    L.train_default(os.path.join(ROOT, "_graphs", "subtree.npy"), device=device)
    return L.load_default(device, os.path.join(ROOT, "_graphs", "subtree.npy")), "trained at start"


def _schedules(g, k, limit, cost, reps, flush, check=None, **kw):
    """plain / batched / learned device times of one (graph, k, limit): the
    median of `reps` runs after one untimed run each; sets compared."""
    import torch
    out, summ = {}, {}
    import gmkbe_b200 as G
    for name, extra in (("learned", dict(schedule="ordered", task_cost=cost)),
                        ("batched", dict(schedule="batched")), ("plain", dict(schedule="plain"))):
        try:
            g.enumerate(k=k, result_limit=limit, **extra, **kw)
            ms, st = [], None
            for _ in range(reps):
                flush.zero_()
                torch.cuda.synchronize()
                st = g.enumerate(k=k, result_limit=limit, **extra, **kw)
                ms.append(st.kernel_ms)
        except G.GmkError as e:          # reported in the line, not hidden
            out[name] = {"error": str(e)}
            continue
        m = statistics.median(ms)
        out[name] = {"ms": m, "results": st.count, "value": st.count / (m / 1e3),
                     "rounds": st.rounds, "donations": st.donations, "tasks": st.tasks}
        summ[name] = st.summary()
    if any("error" in out[n] for n in ("learned", "batched", "plain")):
        return out
    out["learned_vs_plain"] = out["plain"]["ms"] / out["learned"]["ms"]
    out["batched_vs_plain"] = out["plain"]["ms"] / out["batched"]["ms"]
    out["learned_vs_batched"] = out["batched"]["ms"] / out["learned"]["ms"]
    if not limit:
        out["same_set"] = len(set(summ.values())) == 1
        if check is not None:
            out["bit_exact_vs_golden"] = summ["learned"] == check
    return out


def _extras(model, flush, device):
    """cl20k's throughput run and cl100k / cl500k, result-limited, and complete
    enumerations of er200 and of cl100k / cl500k subgraphs, under the three
    schedules."""
    import gmkbe_b200 as G
    from gmkbe_b200 import graphgen as gg
    from gmkbe_b200 import learned as L
    limited, complete = [], []
    for name, k, limit in (("cl20k", 1, 1_000_000), ("cl100k", 2, 10_000_000),
                           ("cl500k", 1, 100_000_000), ("cl500k", 2, 100_000_000)):
        with G.Graph.load(gg.cached_workload(name), device=device) as g:
            r = _schedules(g, k, limit, L.predicted_costs(model, g, k), 3, flush)
            r.update(workload=name, k=k, result_limit=limit)
            limited.append(r)
    for name, k, sub in COMPLETE_CASES:
        h = gg.read_graph_bin(os.path.join(ROOT, "tests", "golden", name + ".graph.bin")) \
            if sub is None else gg.induced_prefix(gg.read_graph_bin(gg.cached_workload(name)), *sub)
        with G.Graph.from_graph(h, device=device) as g:
            r = _schedules(g, k, 0, L.predicted_costs(model, g, k), 3, flush,
                           check=_golden(name, k) if sub is None else None)
            r.update(workload=name if sub is None else f"{name} induced {sub[0]}x{sub[1]}", k=k,
                     vertices=[h.n_left, h.n - h.n_left], edges=h.n_edges)
            complete.append(r)
    return limited, complete


# complete enumerations beside the headline: (workload, k, induced prefix or None).  As for
# cl20k's exactness case, a prefix is the subgraph induced by the first U and V ids
# (the converter's order: lowest degrees first), sized so that the run ends in well under a second.
COMPLETE_CASES = [("er200", 1, None), ("cl100k", 1, (20000, 60000)), ("cl100k", 2, (4000, 12000)),
                  ("cl500k", 2, (20000, 40000)), ("cl500k", 3, (10000, 20000))]


def run_gmk(args, world, rank, local):
    import numpy as np
    import torch
    import gmkbe_b200 as G
    from gmkbe_b200 import graphgen as gg
    from gmkbe_b200 import learned as L

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    host = gg.read_graph_bin(WORKLOAD_PATH)
    off = torch.from_numpy(host.offsets.astype(np.uint32).view(np.int32)).pin_memory()
    adj = torch.from_numpy(host.adj.view(np.int32)).pin_memory()
    off_np = off.numpy().view(np.uint32)
    adj_np = adj.numpy().view(np.uint32)
    shard = dict(shard=rank, nshards=world) if world > 1 else {}

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    model, model_src = _model(local)
    flush_buf = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    want = _golden(WORKLOAD, K)
    dg = G.Graph.from_csr(off_np, adj_np, host.n, host.n_left, device=local)
    cost = L.predicted_costs(model, dg, K)        # the learned schedule's input, resident
    kw = dict(k=K, schedule="ordered", task_cost=cost, **shard)
    for _ in range(args.warmup):
        dg.enumerate(**kw)
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    t_clk0 = time.perf_counter()
    ms, count, launches, exact = [], 0, 0, True
    for _ in range(args.steps):
        flush_buf.zero_()          # L2 flush, outside the timed kernels
        torch.cuda.synchronize()
        st = dg.enumerate(**kw)
        ms.append(st.kernel_ms)
        count += st.count
        launches += st.rounds
        if world == 1:
            exact &= st.summary() == want
    barrier()
    clk = clocks.stop(t_clk0, time.perf_counter())
    if world > 1:
        from gmkbe_b200.shard import combine_summary
        exact = combine_summary(*st.summary(), device=f"cuda:{local}") == want
    # the same graph under the plain and the batched schedule (this rank's shard)
    sched = _schedules(dg, K, 0, cost, min(args.steps, 5), flush_buf, check=want, **shard)
    # end to end through the public API, from pinned host arrays: upload + CSR
    # check + edge hash, root features + model prediction, planning,
    # enumeration, statistics read-back
    for _ in range(args.warmup):
        with G.Graph.from_csr(off_np, adj_np, host.n, host.n_left, device=local) as g2:
            g2.enumerate(k=K, schedule="ordered", task_cost=L.predicted_costs(model, g2, K), **shard)
    barrier()
    e2e_s, e2e_rounds, e2e_tasks = 0.0, 0, 0
    for _ in range(args.steps):
        flush_buf.zero_()
        barrier()
        t0 = time.perf_counter()
        g2 = G.Graph.from_csr(off_np, adj_np, host.n, host.n_left, device=local)
        c2 = L.predicted_costs(model, g2, K)
        st2 = g2.enumerate(k=K, schedule="ordered", task_cost=c2, **shard)
        g2.close()
        e2e_s += time.perf_counter() - t0
        e2e_rounds += st2.rounds
        e2e_tasks += st2.tasks
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
    # bytes copied per end-to-end step: host -> device the CSR (n+1 offsets and
    # 2|E| ids) and the task table (16 B a task); device -> host the
    # predictions (n_left FP32; features and forward pass stay on the device),
    # the CSR check (16 B) and per launch the round counters (512 B) and
    # totals (88 B)
    nl = host.n_left
    h2d = 4 * (off_np.size + adj_np.size) + 16 * e2e_tasks / args.steps
    d2h = 4 * nl + 16 + 600 * e2e_rounds / args.steps
    if rank == 0:
        peak, peak_kind, sm_max = _peaks()
        ab = _algo_bytes(WORKLOAD, K, 0)
        prof = _profile("enumerate_warp_kernel_cl20k_sub") or {}
        mean_ms = tot_ms / args.steps
        achieved = (ab["algo_bytes"] / world / (mean_ms / 1e3) / 1e9) if ab else None
        line = {
            "metric": METRIC, "value": count_all / (tot_ms_max / 1e3), "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": tot_ms_max / args.steps, "higher_is_better": True,
            # N GPUs share the one complete enumeration (LPT shards of its tasks)
            "scaling": "strong",
            "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded Chung-Lu, converter ordering)",
            "config": {"workload": CONFIG_DESC, "k": K, "result_limit": 0, "complete": True,
                       "schedule": "learned+batched (ordered planner over the model's predicted "
                                   "subtree sizes, in-launch work sharing)",
                       "model": model_src, "l2": "flushed between steps (256 MB write)",
                       "parallelism": f"task shards x{world}" if world > 1 else "1 GPU"},
            "bit_exact": bool(exact),
            "e2e": {"value": count_all / e2e_max, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "learned_vs_plain": sched.get("learned_vs_plain"),
            "schedules": sched,
            "roofline": {
                "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak if achieved else None,
                "traffic": prof.get("dram_bytes_per_launch"), "peak_source": peak_kind,
                "kernel": "enumerate_warp_kernel",
                "algorithmic_bytes_per_step": ab["algo_bytes"] if ab else None,
                "algorithmic_bytes_source": "profiles/algo_bytes.json (oracle/algo_bytes.py)",
                "l2_hit_rate": prof.get("l2_hit_rate_pct"),
                "issue_active_frac": prof.get("issue_active_frac"),
                "warp_inst_per_launch": prof.get("warp_inst_per_launch"),
                "binding_ceiling": prof.get("binding_ceiling")},
            "clocks": clk,
            "stats": {"nodes_per_step": st.nodes, "tasks": st.tasks, "threads": st.threads,
                      "rounds_per_step": launches / args.steps, "donations": st.donations},
        }
        if world == 1 and not args.no_extras:
            line["limited"], line["complete_runs"] = _extras(model, flush_buf, local)
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline()
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
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the result-limited configurations and the complete-run table")
    args = ap.parse_args()
    world, rank, local = _dist()
    if args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_gmk(args, world, rank, local)


if __name__ == "__main__":
    main()
