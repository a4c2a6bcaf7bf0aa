#!/usr/bin/env python
"""Benchmark of the likelihood path on one B200 (or N, pattern-sharded).

Workload: DNA GTR+G4 (Gamma shape 0.5) on a seeded 512-taxon tree with branch lengths
~Exp(0.05), 1,000,000 simulated sites with 5% gap cells, compressed to unique patterns
(the "FP64 vs mixed-precision DNA at scale" configuration).  A step is one full-tree
log-likelihood evaluated from scratch: every partial of the tree recomputed (510 node
updates over all patterns), then the branch log-likelihood and its pattern-weighted sum.

Metric: site-partial updates/s (patterns x node updates per second, whole job) and lnL
evaluations/s.  `value` is measured with the inputs resident in HBM; `e2e` runs the same
step through the public PhyloTree API from host buffers (tips, weights up; pattern lnL
down) every step.  Timing uses CUDA events on the session's stream; partial buffers
(~39 GB) exceed L2 many times over, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gems|reference]

Under torchrun each rank holds its own 1,000,000-site slab of the same tree and model
(weak scaling); the per-evaluation exchange is one NCCL all-reduce of the lnL.
`--impl reference` times the CPU restatement of the reference kernels (oracle/, FP64, all
host threads) on the same workload, bounded to a pattern sample per step.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from gems_b200 import synth  # noqa: E402

NSITES = 1_000_000
NTAXA = 512


def update_bytes(s, n=4, C=4, safe=False):
    """Algorithmic bytes of one site-partial update: internal-internal 3*C*n*s + 3*sigma,
    tip-internal 2*C*n*s + 1 + 2*sigma, tip-tip C*n*s + 2 + sigma, with s = 8 (FP64) or 4
    (FP32 partials) and sigma = 2 B (NORM counter) or 2*C B (SAFE counters)."""
    sig = 2 * C if safe else 2
    return 3 * C * n * s + 3 * sig, 2 * C * n * s + 1 + 2 * sig, C * n * s + 2 + sig


def update_flops(n=4, C=4):
    """Algorithmic flops of one site-partial update (eigen-space form): 6*C*n^2 + C*n."""
    return 6 * C * n * n + C * n


CONFIGS = {
    "dna512": "DNA GTR+G4 (alpha 0.5), 512 taxa, Exp(0.05) lengths, {sites} sites/rank with 5% "
              "gaps, from-scratch full-tree lnL",
    "protein128": "20-state protein +G4 (alpha 0.8), log-normal exchangeabilities, Dirichlet "
                  "frequencies, 128 taxa, Exp(0.15) lengths, {sites} sites/rank, from-scratch "
                  "full-tree lnL",
}


def env_rank():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def op_kinds(tree):
    """(internal-internal, tip-internal, tip-tip) node updates of a from-scratch
    computeLikelihood, rooted at the leaf that findFarthestLeaf returns."""
    n = tree.nnodes
    adj = [[] for _ in range(n)]
    for u, v in zip(tree.eu, tree.ev):
        adj[int(u)].append(int(v))
        adj[int(v)].append(int(u))
    h = [0] * n
    sys.setrecursionlimit(10000)

    def far(node, dad):
        if dad >= 0 and len(adj[node]) == 1:
            h[node] = 0
            return node
        res = -1
        h[node] = 0
        for c in adj[node]:
            if c == dad:
                continue
            lf = far(c, node)
            if h[node] < h[c] + 1:
                h[node] = h[c] + 1
                res = lf
        return res

    root = far(0, -1)
    counts = [0, 0, 0]
    stack = [(adj[root][0], root)]
    while stack:
        node, dad = stack.pop()
        kids = [c for c in adj[node] if c != dad]
        if not kids:
            continue
        nleaf = sum(1 for c in kids if len(adj[c]) == 1)
        counts[nleaf] += 1
        stack.extend((c, node) for c in kids)
    return counts


def read_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def read_traffic(name):
    """traffic (DRAM bytes per launch) from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", open(path).read())
        return float(m.group(1)) if m else None
    except OSError:
        return None


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_bench_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()
            self.f.close()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().split("\n") if r]
            sm = [float(r[0]) for r in rows]
            reasons = set()
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for r in rows:
                for k, nm in enumerate(names):
                    if "Active" in r[3 + k] and "Not" not in r[3 + k]:
                        reasons.add(nm)
            return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][1]),
                    "reasons": sorted(reasons), "samples": len(rows)}
        except Exception:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}


def make_workload(rank, nsites, config="dna512"):
    """Same tree and model on every rank; each rank simulates its own site slab."""
    if config == "protein128":
        rng = np.random.default_rng(3)
        model = synth.protein(rng, 4, 0.8)
        tree = synth.random_tree(128, 0.15, 14)
        aln = synth.simulate(tree, model, nsites, 26 + 1000 * rank)
        return tree, model, aln
    rng = np.random.default_rng(2)
    model = synth.dna_gtr(rng, 4, 0.5)
    tree = synth.random_tree(NTAXA, 0.05, 13)
    aln = synth.simulate(tree, model, nsites, 25 + 1000 * rank, gap_frac=0.05)
    return tree, model, aln


def cpu_baseline(tree, model, aln, target_s=12.0):
    """The oracle (CPU restatement of the reference kernels) on a bounded pattern sample."""
    from oracle import oracle as orc
    threads = os.cpu_count() or 1
    orc.set_threads(threads)
    nsamp = min(aln.npat, 40_000)
    sub = synth.Alignment(aln.ntaxa, model.nstates, int(aln.weights[:nsamp].sum()),
                          np.ascontiguousarray(aln.patterns[:, :nsamp]), aln.weights[:nsamp])
    ot = orc.OracleTree(tree, model, sub)
    nops = sum(op_kinds(tree))
    t0 = time.perf_counter()
    k = 0
    while True:
        ot.clearAllPartialLH()
        ot.computeLikelihood()
        k += 1
        el = time.perf_counter() - t0
        if el > target_s or k >= 50:
            break
    ups = k * nops * nsamp / el
    return {"value": ups, "unit": "site-partial updates/s", "cores": threads, "kind": "port",
            "sample": f"{nsamp} of {aln.npat} patterns, {k} from-scratch lnL evaluations "
                      f"({nops} node updates each), oracle FP64, {threads} threads",
            "lnl_evals_per_s": k / el}


def run_reference(args):
    rank, world, _ = env_rank()
    if rank != 0:
        return
    tree, model, aln = make_workload(0, args.sites, args.config)
    for _ in range(args.warmup):
        pass
    res = []
    for _ in range(args.steps):
        res.append(cpu_baseline(tree, model, aln, target_s=max(3.0, 30.0 / args.steps)))
    v = statistics.median(r["value"] for r in res)
    nops = sum(op_kinds(tree))
    line = {
        "impl": "reference", "metric": "site-partial updates/s", "value": v,
        "unit": "site-partial updates/s", "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "ms_per_step": 1e3 * nops * aln.npat / v, "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": {"workload": "DNA GTR+G4, 512 taxa, 1,000,000 sites (5% gaps), "
                               "from-scratch full-tree lnL", "npat": aln.npat},
        "cpu_baseline": {**res[0], "value": v},
        "e2e": {"value": v, "unit": "site-partial updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gems", choices=["gems", "reference"])
    ap.add_argument("--sites", type=int, default=None)
    ap.add_argument("--config", default="dna512", choices=sorted(CONFIGS))
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-tc", action="store_true",
                    help="20-state mixed traversal on CUDA cores instead of tcgen05")
    args = ap.parse_args()
    if args.sites is None:
        args.sites = NSITES if args.config == "dna512" else 100_000
    if args.impl == "reference":
        return run_reference(args)

    import torch
    from gems_b200 import PhyloTree
    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    tree, model, aln = make_workload(rank, args.sites, args.config)
    gt = PhyloTree.from_case(tree, model, aln, precision=args.precision, device=local)
    s = gt.session
    if args.no_tc:
        s.set_tensor_cores(False)
    stream = torch.cuda.ExternalStream(s.stream_handle(), device=local)
    kinds = op_kinds(tree)
    nops = sum(kinds)
    P = aln.npat
    lnl_buf = torch.zeros(1, dtype=torch.float64, device=f"cuda:{local}")

    def step():
        gt.clearAllPartialLH()
        v = gt.computeLikelihood()
        if dist is not None:
            lnl_buf.fill_(v)
            dist.all_reduce(lnl_buf)
            return float(lnl_buf.item())
        return v

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    s.profile(True)
    s.profile_read(0)
    l0 = s.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            lnl = step()
        e1.record(stream)
        torch.cuda.synchronize()
    s.profile(False)
    ms = e0.elapsed_time(e1) / args.steps
    trav_ms, trav_n = s.profile_read(0)
    launches = s.launch_count() - l0
    # max over ranks
    t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local}")
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())

    # end to end through the public API from host buffers
    pin_pat = torch.empty(aln.patterns.shape, dtype=torch.uint8, pin_memory=True)
    pin_w = torch.empty(aln.weights.shape, dtype=torch.float64, pin_memory=True)
    pat_host = pin_pat.numpy()
    w_host = pin_w.numpy()
    pat_host[:] = aln.patterns
    w_host[:] = aln.weights
    h2d = pat_host.nbytes + w_host.nbytes
    d2h = 8 * P + 8
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e2.record(stream)
    for _ in range(args.steps):
        s.upload_tips(pat_host)
        s.upload_patterns(w_host)
        gt.clearAllPartialLH()
        lnl_e2e, plh = gt.computeLikelihood(pattern_lh=True)
    e3.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e2.elapsed_time(e3) / args.steps
    t = torch.tensor([ms_e2e], dtype=torch.float64, device=f"cuda:{local}")
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_e2e = float(t.item())

    ups = world * nops * P / (ms * 1e-3)
    ups_e2e = world * nops * P / (ms_e2e * 1e-3)
    b_ii, b_ti, b_tt = update_bytes(8 if args.precision == "fp64" else 4, model.nstates,
                                    model.ncat)
    alg_bytes = P * (kinds[0] * b_ii + kinds[1] * b_ti + kinds[2] * b_tt)
    peak, peak_kind = read_peaks()
    achieved = alg_bytes / (trav_ms / max(trav_n, 1) * 1e-3) / 1e9 if trav_n else None
    line = {
        "metric": "site-partial updates/s", "value": ups, "unit": "site-partial updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32+f64",
        "data": "synthetic (seeded generator; no public dataset)",
        "config": {"workload": CONFIGS[args.config].format(sites=f"{args.sites:,}"),
                   "npat_per_rank": P, "node_updates_per_step": nops,
                   "precision": args.precision, "parallelism": f"pattern-shard x{world}",
                   "l2": "inputs larger than L2 (partials ~39 GB)"},
        "lnl_evals_per_s": 1.0 / (ms * 1e-3),
        "lnl": lnl,
        "gpu_launches": launches,
        "e2e": {"value": ups_e2e, "unit": "site-partial updates/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": ms_e2e},
        "roofline": {"bound": "hbm", "kernel": "k_traverse", "achieved": achieved,
                     "peak": peak, "peak_source": peak_kind, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None,
                     "algorithmic_bytes_per_launch": alg_bytes,
                     "avg_launch_ms": trav_ms / max(trav_n, 1),
                     "traffic": read_traffic(f"traverse_{args.precision}_{args.config}.md")},
        "clocks": clk.summary(),
    }
    if rank == 0 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(tree, model, aln)
    if rank == 0:
        print(json.dumps(line), flush=True)
    gt.close()
    s.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
