"""Runs every kernel of the library once on one workload, for profiling.

    python -m gmkbe_b200.profile_kernels [--workload cl500k] [--k 1] [--limit 100000]
                                         [--samples 262144]

In launch order: csr_check_kernel and build_edge_hash (loading the graph),
root_cost_kernel (gmk_root_costs), root_features_kernel (gmk_root_features),
float_to_half_kernel + forward_kernel (a prediction over every root),
float_to_half_kernel, forward_kernel, backward_kernel, adam_kernel (one
training epoch over `samples` feature rows), forward_kernel + backward_kernel
again (the loss after the epoch), and the enumeration (enumerate_warp_kernel,
result limit `limit`).  Prints the times the API reports.  Under ncu, select
kernels with -k and count launches with -c.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import graphgen as gg
from . import learned as L
from .api import Graph


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--workload", default="cl500k", choices=sorted(gg.WORKLOADS))
    ap.add_argument("--k", type=int, default=1)
    ap.add_argument("--limit", type=int, default=100_000)
    ap.add_argument("--samples", type=int, default=1 << 18)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--no-enumerate", action="store_true",
                    help="skip the enumeration (and the search workspace it allocates)")
    a = ap.parse_args(argv)
    path = gg.cached_workload(a.workload)
    out = {"workload": a.workload}
    t0 = time.perf_counter()
    g = Graph.load(path, device=a.device)
    out["load_s"] = time.perf_counter() - t0
    out["n"], out["n_left"], out["adj_len"] = g.n, g.n_left, g.adj_len
    t0 = time.perf_counter()
    g.root_costs()
    out["root_costs_s"] = time.perf_counter() - t0
    feats = L.root_features(g, a.k)
    model = L.SubtreeModel(device=a.device, seed=1)
    model.predict(feats)
    rows = np.resize(feats, (a.samples, feats.shape[1])).astype(np.float32)
    y = np.log1p(np.arange(a.samples, dtype=np.float32) % 1000)
    out["train_loss"] = model.train(rows, y, epochs=1, lr=1e-3)
    if not a.no_enumerate:
        st = g.enumerate(k=a.k, result_limit=a.limit)
        out.update(results=st.count, enumerate_ms=st.kernel_ms, rounds=st.rounds)
    model.close()
    g.close()
    print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
