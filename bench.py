#!/usr/bin/env python
"""Benchmark: GTEPS of BFS / SSSP / CC / PageRank on one B200 (per GPU).

Workload (the reference's headline configuration at scale): RMAT scale 24,
edge factor 16, a=.57 b=.19 c=.19, self-loops and duplicates removed,
uint32 weights uniform in [1, 64], seeded; BFS and SSSP from seeded random
non-isolated roots on the directed graph, CC on the symmetrised graph,
PageRank (d = 0.85, 20 iterations, FP64) on the directed graph.

One step = BFS(root) + SSSP(root) + CC + PageRank(20) with the step's root
(roots cycle through 10 seeded roots).  GTEPS numerators: BFS/SSSP = sum of
out-degrees of reached vertices; CC = edges of the symmetrised graph;
PageRank = E x iterations.  `value` = all numerators of the K timed steps /
their device time (CUDA events on the engine's stream, max over ranks).
`e2e` = the same through the C ABI from pinned host buffers: every step
uploads both CSRs (cgb_graph_create), runs the four algorithms and reads
every result back into host memory.  Uploads run back to back on a second
host thread (the symmetrised graph, then the directed graph's weights,
which only SSSP reads) while the directed graph's algorithms run.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GTEPS (BFS/SSSP/WCC/PR) on 1 B200: learned vs heuristic schedule, % HBM peak"
BFS, SSSP, CC, PR = 0, 1, 2, 3
ALG_NAMES = ["bfs", "sssp", "cc", "pagerank"]
N_ROOTS = 10


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["cgb200", "reference"], default="cgb200")
    p.add_argument("--scale", type=int, default=24)
    p.add_argument("--edge-factor", type=int, default=16)
    p.add_argument("--seed", type=int, default=1)
    p.add_argument("--pr-iters", type=int, default=20)
    p.add_argument("--schedule", choices=["heuristic", "learned"], default="heuristic",
                   help="schedule of the timed steps (both are compared in 'schedules')")
    p.add_argument("--no-compare", action="store_true", help="skip the learned-vs-heuristic comparison")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--e2e-steps", type=int, default=0, help="0 = same as --steps")
    p.add_argument("--no-autotune", action="store_true",
                   help="keep the default launch parameters (else cgb_autotune per algorithm, untimed)")
    p.add_argument("--no-batching", action="store_true", help="skip the multi-root and graph-batch section")
    p.add_argument("--no-serving", action="store_true", help="skip the request-server section")
    p.add_argument("--no-shapes", action="store_true",
                   help="skip the skewed / high-diameter shapes (Chung-Lu 41.6 M vertices / 1.47 B edges, 4800 x 5000 grid)")
    p.add_argument("--shapes-scale", type=float, default=1.0,
                   help="fraction of the Chung-Lu vertices and edges (1.0 = 41.6 M / 1.47 B)")
    p.add_argument("--serve-scale", type=int, default=25, help="RMAT scale of the served graph")
    p.add_argument("--serve-requests", type=int, default=256, help="queries per arrival rate")
    p.add_argument("--algorithms", default="bfs,sssp,cc,pr",
                   help="comma list of bfs,sssp,cc,pr run in each step (default: all four)")
    return p.parse_args()


# ------------------------------------------------------------------ helpers
class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        mx = [num(r[2]) for r in rows if num(r[2]) is not None]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for i, n in enumerate(names):
                if r[5 + i].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def pick_roots(offsets: np.ndarray, seed: int, n: int) -> list:
    deg = np.diff(offsets.astype(np.int64))
    cand = np.nonzero(deg)[0]
    rng = np.random.default_rng(seed + 1000)
    return [int(x) for x in rng.choice(cand, size=min(n, cand.size), replace=False)]


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one k_pr_pull
# launch, from a one-pass ncu capture of this bench with --algorithms pr on the
# same graph, keyed by (scale, edge factor, seed).
PR_PULL_DRAM_BYTES = {(24, 16, 1): 1166656256 + 225822208, (22, 16, 1): 250001920 + 20899072}


def load_peaks() -> dict:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return {"hbm_gbs": d["hbm_gbs"], "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


# ------------------------------------------------------------------ dist
class Dist:
    """One process per GPU (torchrun); replicas only, so the collectives are
    the barrier and the max / sum reductions of cggraph_b200.replicas."""

    def __init__(self, want_gpus: int):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        if want_gpus != self.world:
            raise SystemExit(f"--gpus {want_gpus} but WORLD_SIZE={self.world}: launch one process per GPU with "
                             f"python -m torch.distributed.run --nproc-per-node {want_gpus} bench.py --gpus {want_gpus}")
        self.pg = False
        if self.world > 1:
            import torch
            import torch.distributed as dist
            torch.cuda.set_device(self.local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device("cuda", self.local))
            self.pg = True

    def shard(self, items):
        from cggraph_b200.replicas import shard
        return shard(items, self.rank, self.world)

    def barrier(self):
        if self.pg:
            import torch.distributed as dist
            dist.barrier(device_ids=[self.local])

    def reduce(self, x: float, op: str) -> float:
        from cggraph_b200.replicas import max_over_ranks, sum_over_ranks
        dev = f"cuda:{self.local}" if self.pg else None
        return max_over_ranks(x, dev) if op == "max" else sum_over_ranks(x, dev)

    def close(self):
        if self.pg:
            import torch.distributed as dist
            dist.destroy_process_group()


def workload_config(args, V, Ed, Es, roots, algs) -> dict:
    """The workload both arms run (the same dict in each arm's JSON line)."""
    return {"workload": f"rmat{args.scale}_ef{args.edge_factor}_"
                        + "_".join(ALG_NAMES[a] for a in algs).replace("pagerank", f"pr{args.pr_iters}"),
            "scale": args.scale, "edge_factor": args.edge_factor, "rmat_abc": [0.57, 0.19, 0.19],
            "seed": args.seed, "vertices": V, "edges_directed": Ed, "edges_symmetrised": Es,
            "weights": "uniform [1,64]", "roots": roots, "pr_iterations": args.pr_iters,
            "algorithms": [ALG_NAMES[a] for a in algs],
            "cc": "components of the symmetrised graph",
            "l2": "inputs larger than L2 (directed CSR %.2f GB)" % ((4 * (V + 1) + 8 * Ed) / 1e9),
            "parallelism": f"replicas x{args.gpus}"}


# ---------------------------------------------------------------- our arm
def parse_algs(spec: str) -> list:
    names = {"bfs": BFS, "sssp": SSSP, "cc": CC, "wcc": CC, "pr": PR, "pagerank": PR}
    return sorted({names[a.strip().lower()] for a in spec.split(",") if a.strip()})


def run_step(gd, root, opts, cc_opts, pr_iters, algs=(BFS, SSSP, CC, PR)):
    """One step on the resident graph; returns [(algorithm, run stats)].  CC
    runs as weak components of the directed graph (CGB_FLAG_CC_WEAK): the
    labels of CC on the symmetrised graph, with no symmetrised copy."""
    out = []
    for alg in algs:
        arg = {BFS: root, SSSP: root, CC: 0, PR: pr_iters}[alg]
        gd.run(alg, arg, cc_opts if alg == CC else opts, to_host=False)
        out.append((alg, gd.stats()))
    return out


def symmetrised_edges(cg, args, dev, keep_host=False):
    """Edge count of the symmetrised graph (the CC numerator), from the
    device generator; with keep_host, also its CSR in host memory."""
    gs = cg.Graph.rmat(args.scale, args.edge_factor, args.seed, symmetrise=True, wmax=0, device=dev)
    Es = gs.edgeNum
    host = gs.download(with_weight=False)[:2] if keep_host else None
    gs.close()
    return Es, host


def bench_cgb200(args, d: Dist):
    import torch
    import cggraph_b200 as cg
    from cggraph_b200 import _lib as L

    dev = d.local
    torch.cuda.set_device(dev)
    algs = parse_algs(args.algorithms)
    Es, sym_host = symmetrised_edges(cg, args, dev, keep_host=d.world == 1 and not args.no_cpu_baseline)
    gd = cg.Graph.rmat(args.scale, args.edge_factor, args.seed, wmax=64, device=dev)
    off_h, dst_h, w_h = gd.download()
    roots_all = pick_roots(off_h, args.seed, N_ROOTS * d.world)
    roots = d.shard(roots_all)
    V, Ed = gd.vertexNum, gd.edgeNum

    stream = torch.cuda.current_stream()
    gd.set_stream(stream)
    sched = L.SCHED_LEARNED if args.schedule == "learned" else L.SCHED_HEURISTIC
    if args.schedule == "learned":
        from cggraph_b200 import policy
        if not policy.load_default():
            raise SystemExit("--schedule learned: no trained policy (python -m cggraph_b200.train_policy)")
    warm_opts = cg.make_options(schedule=sched)
    timed_opts = cg.make_options(schedule=sched, flags=L.FLAG_KERNEL_TIMING)
    warm_cc = cg.make_options(schedule=sched, flags=L.FLAG_CC_WEAK)
    timed_cc = cg.make_options(schedule=sched, flags=L.FLAG_KERNEL_TIMING | L.FLAG_CC_WEAK)

    # launch parameters: the project's autotuner, per algorithm, before timing
    autotune = None
    if not args.no_autotune:
        autotune = {}
        tune_roots = pick_roots(off_h, args.seed + 13, 4)  # not the timed roots
        for alg, rts in ((BFS, tune_roots), (SSSP, tune_roots), (CC, [0]), (PR, [5, 5])):
            if alg in algs:
                best, bms, sms = gd.autotune(alg, rts, cc_weak=alg == CC)
                autotune[ALG_NAMES[alg]] = {"default_ms": sms, "tuned_ms": bms, "speedup": sms / bms,
                                            "tuning": best}

    for i in range(args.warmup):
        run_step(gd, roots[i % len(roots)], warm_opts, warm_cc, args.pr_iters, algs)

    clocks = Clocks(dev)
    clocks.start()
    per_alg_edges = [0] * 4
    per_alg_ms = [0.0] * 4
    kclass_ms = [0.0] * 8
    kclass_launches = [0] * 8
    launches = 0
    pr_launch_ms = 0.0
    pr_launches = 0
    d.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for k in range(args.steps):
        for alg, st in run_step(gd, roots[k % len(roots)], timed_opts, timed_cc, args.pr_iters, algs):
            # CC: the edges of the symmetrised graph, whose components it computes
            per_alg_edges[alg] += Es if alg == CC else st.traversed_edges
            per_alg_ms[alg] += st.ms
            launches += st.launches
            for c in range(8):
                kclass_ms[c] += st.kernel_ms[c]
                kclass_launches[c] += st.kernel_launches[c]
            if alg == PR:
                pr_launch_ms += st.kernel_ms[L.K_PR]
                pr_launches += st.kernel_launches[L.K_PR]
    ev1.record(stream)
    torch.cuda.synchronize()
    d.barrier()
    clk = clocks.stop()
    ms_local = ev0.elapsed_time(ev1)
    ms_max = d.reduce(ms_local, "max")
    edges_total = d.reduce(sum(per_alg_edges), "sum")
    value = edges_total / (ms_max / 1e3) / 1e9

    # roofline of the dominant kernel class
    peaks = load_peaks()
    dom = int(np.argmax(kclass_ms))
    roof = {"bound": "hbm", "unit": "GB/s", "peak": peaks["hbm_gbs"], "peak_source": peaks["source"]}
    if pr_launches:
        bytes_per_launch = 12 * Ed + 20 * V + 4
        avg_s = pr_launch_ms / pr_launches / 1e3
        achieved = bytes_per_launch / avg_s / 1e9
        roof.update({"kernel": "k_pr_pull (+ hub-row chunk kernels), one PageRank iteration",
                     "alg_bytes_per_launch": bytes_per_launch, "avg_launch_ms": pr_launch_ms / pr_launches,
                     "achieved": achieved, "frac": achieved / peaks["hbm_gbs"],
                     "traffic": PR_PULL_DRAM_BYTES.get((args.scale, args.edge_factor, args.seed)),
                     "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of one k_pr_pull launch, "
                                       "ncu capture of this workload (hub-row chunk kernels not included)",
                     "dominant_class": L.KERNEL_CLASS_NAMES[dom],
                     "class_share": {L.KERNEL_CLASS_NAMES[c]: round(kclass_ms[c] / max(1e-9, sum(kclass_ms)), 4)
                                     for c in range(8) if kclass_ms[c] > 0}})

    per_alg = {ALG_NAMES[a]: {"gteps": per_alg_edges[a] / (per_alg_ms[a] / 1e3) / 1e9 if per_alg_ms[a] else None,
                              "ms_per_run": per_alg_ms[a] / args.steps} for a in algs}
    full = algs == [BFS, SSSP, CC, PR]

    schedules = None
    if not args.no_compare and d.world == 1 and (BFS in algs or SSSP in algs):
        schedules = compare_schedules(args, cg, L, gd, roots[:4], dev)
        if args.schedule == "learned":
            from cggraph_b200 import policy
            policy.load_default()

    # end to end through the C ABI with pinned host buffers
    e2e = None
    if not args.no_e2e and full:
        e2e = bench_e2e(args, d, cg, gd, roots, off_h, dst_h, w_h, Es, sched)

    # CPU baseline: the reference's own engine on this host (rank 0, N = 1)
    cpu = None
    if d.world == 1 and not args.no_cpu_baseline and full:
        try:
            cpu = cpu_baseline(args, V, Ed, Es, off_h, dst_h, w_h, sym_host, roots)
        except Exception as e:  # reported, not fatal
            cpu = {"value": None, "error": str(e)[-300:]}
    sym_host = None

    batching = None
    if d.world == 1 and not args.no_batching and (BFS in algs or SSSP in algs):
        batching = bench_batching(args, cg, L, gd, roots, dev)

    gd.set_stream(None)
    gd.close()
    serving = None
    if d.world == 1 and not args.no_serving and (BFS in algs or SSSP in algs):
        serving = bench_serving(args, cg, L, dev)
    shapes = None
    if d.world == 1 and not args.no_shapes and algs == [BFS, SSSP, CC, PR]:
        shapes = bench_shapes(args, cg, L, dev)
    result = {
        "metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": d.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32 (BFS/SSSP/CC), f64 (PageRank)",
        "data": "synthetic (seeded RMAT)",
        "config": workload_config(args, V, Ed, Es, roots_all, algs),
        "engine": {"schedule": args.schedule, "roots_this_rank": roots,
                   "launch_parameters": "default" if args.no_autotune else "cgb_autotune per algorithm (untimed)",
                   "cc": "weak components of the directed graph (CGB_FLAG_CC_WEAK)"},
        "per_algorithm": per_alg,
        "schedules": schedules,
        "autotune": autotune,
        "batching": batching,
        "serving": serving,
        "shapes": shapes,
        "roofline": roof,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": int(d.reduce(launches, "sum")),
        "clocks": clk,
    }
    return result


def _best_of(g, alg, root, opts, reps=2):
    g.run(alg, root, opts, to_host=False)
    best, st = 1e30, None
    for _ in range(reps):
        g.run(alg, root, opts, to_host=False)
        s = g.stats()
        if s.ms < best:
            best, st = s.ms, s
    return best, st


def compare_schedules(args, cg, L, gd, roots, dev):
    """BFS and SSSP under the heuristic and the learned schedule: on the
    benchmark graph from its roots, and on the 4800 x 5000 grid (24 M
    vertices, weights U[1,1000]) from a corner.  Results are bit-identical;
    only time differs."""
    from cggraph_b200 import policy
    if not policy.load_default():
        return {"note": "no trained policy shipped: learned runs fall back to the heuristic"}
    out = {}
    try:
        cases = [(f"rmat{args.scale}", gd, roots, False)]
        grid = cg.Graph.grid(4800, 5000, seed=1, device=dev) if args.scale >= 20 else None
        if grid is not None:
            cases.append(("grid4800x5000", grid, [0], True))
        for name, g, rts, own in cases:
            res = {}
            for alg, an in ((BFS, "bfs"), (SSSP, "sssp")):
                t = {}
                edges = 0
                for sched, sn in ((L.SCHED_HEURISTIC, "heuristic"), (L.SCHED_LEARNED, "learned")):
                    tot = 0.0
                    e = 0
                    for r in rts:
                        ms, st = _best_of(g, alg, r, cg.make_options(schedule=sched))
                        tot += ms
                        e += st.traversed_edges
                    t[sn] = tot
                    edges = e
                res[an] = {"heuristic_ms": t["heuristic"], "learned_ms": t["learned"],
                           "heuristic_gteps": edges / t["heuristic"] / 1e6, "learned_gteps": edges / t["learned"] / 1e6,
                           "learned_speedup": t["heuristic"] / t["learned"]}
            # the best fixed delta: the heuristic schedule with the default delta
            # scaled by 1/4 ... 16 (the learned schedule's own choices per bucket)
            _, st0 = _best_of(g, SSSP, rts[0], cg.make_options(schedule=L.SCHED_HEURISTIC), reps=1)
            base = st0.sssp_delta
            sweep = {}
            for sc in (0.25, 0.5, 1, 2, 4, 8, 16):
                dk = max(1, int(base * sc))
                sweep[str(sc)] = sum(_best_of(g, SSSP, r, cg.make_options(schedule=L.SCHED_HEURISTIC,
                                                                            sssp_delta=dk))[0] for r in rts)
            best = min(sweep, key=sweep.get)
            res["sssp"].update({"default_delta": base, "fixed_delta_ms": sweep, "best_fixed_scale": float(best),
                                "best_fixed_ms": sweep[best],
                                "learned_vs_best_fixed": sweep[best] / t_sssp if (t_sssp := res["sssp"]["learned_ms"]) else None})
            out[name] = res
            if own:
                g.close()
    finally:
        policy.load(None)
    return out


def bench_batching(args, cg, L, gd, roots, dev):
    """Batching: 64 BFS and 64 SSSP roots on the benchmark graph in
    multi-root passes (bit-packed per-vertex root masks) against one run per
    root; and 256 uneven graphs (RMAT scales 10-16, grids 32x32 to 512x512)
    as one disjoint-union graph, BFS/SSSP from one root per graph in one
    captured launch, against one run per graph.  Results are identical
    (tests); only time differs."""
    import torch
    out = {}
    V = gd.vertexNum
    off_h, _, _ = gd.download(with_weight=False)
    rts = pick_roots(off_h, args.seed + 7, 64)
    tune_rts = pick_roots(off_h, args.seed + 17, 64)
    d_out = torch.empty((64, V), dtype=torch.int32, device=f"cuda:{dev}")
    seq = cg.make_options(flags=L.FLAG_BATCH_SEQUENTIAL)
    for alg, an in ((BFS, "bfs"), (SSSP, "sssp")):
        tuned = None
        if not args.no_autotune:
            best, bms, sms = gd.autotune(alg, tune_rts, batch=True)
            tuned = {"default_ms": sms, "tuned_ms": bms, "tuning": best}
        gd.run_batch(alg, rts, out=d_out)  # warm-up
        _, ms_multi = gd.run_batch(alg, rts, out=d_out)
        edges = gd.stats().traversed_edges
        _, ms_seq = gd.run_batch(alg, rts, seq, out=d_out)
        out[f"roots64_{an}"] = {"multi_ms": ms_multi, "one_by_one_ms": ms_seq, "multi_gteps": edges / ms_multi / 1e6,
                                "one_by_one_gteps": edges / ms_seq / 1e6, "speedup": ms_seq / ms_multi,
                                "autotune": tuned}
    # 256 uneven graphs
    rng = np.random.default_rng(args.seed + 11)
    graphs = []
    for i in range(256):
        if i % 2 == 0:
            h = cg.Graph.rmat(int(rng.integers(10, 17)), 16, seed=1000 + i, wmax=64, device=dev)
        else:
            side = int(rng.integers(32, 513))
            h = cg.Graph.grid(side, side, seed=1000 + i, device=dev)
        graphs.append(h)
    csrs = [h.download() for h in graphs]
    roots_b = [int(rng.integers(0, o.size - 1)) for o, _, _ in csrs]
    with cg.Batch(csrs, device=dev) as b:
        tv, te, _ = b.info()
        res = {"graphs": 256, "vertices": tv, "edges": te}
        for alg, an in ((BFS, "bfs"), (SSSP, "sssp")):
            b.run(alg, roots_b)  # first run captures the CUDA graph
            _, ms_b = b.run(alg, roots_b)
            edges = b.stats().traversed_edges
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ms_one = 0.0
            for h, r in zip(graphs, roots_b):
                h.run(alg, r, to_host=False)
                ms_one += h.stats().ms
            torch.cuda.synchronize()
            wall_one = (time.perf_counter() - t0) * 1e3
            res[an] = {"batch_ms": ms_b, "one_by_one_device_ms": ms_one, "one_by_one_wall_ms": wall_one,
                       "batch_gteps": edges / ms_b / 1e6, "one_by_one_gteps": edges / wall_one / 1e6,
                       "speedup_vs_wall": wall_one / ms_b}
        res["captured"] = b.info()[2]
        out["graphs256"] = res
    for h in graphs:
        h.close()
    return out


def bench_shapes(args, cg, L, dev):
    """Skewed and high-diameter shapes, all four algorithms under the plain
    heuristic schedule: a Chung-Lu power-law directed graph of 41.6 M
    vertices and about 1.47 B distinct edges (about 1.96 B draws before
    duplicates are removed; degree-distribution exponent 2, largest
    out-degree about 3 M, weights [1,64]; its symmetrised copy for CC),
    and the 4800 x 5000 grid (weights [1,1000]).  One untimed run, then the
    best of two; GTEPS numerators as in the main line."""
    out = {}

    def best2(g, alg, arg):
        g.run(alg, arg, to_host=False)
        ms = []
        for _ in range(2):
            g.run(alg, arg, to_host=False)
            ms.append(g.stats().ms)
        return min(ms), g.stats().traversed_edges

    Vc = int(41_600_000 * args.shapes_scale)
    draws, i0 = cg.chunglu_draws_for_edges(Vc, int(1_470_000_000 * args.shapes_scale),
                                           int(3_000_000 * args.shapes_scale) or 1)
    t0 = time.perf_counter()
    g = cg.Graph.chunglu(Vc, draws, i0, seed=args.seed, wmax=64, device=dev)
    gen_s = time.perf_counter() - t0
    off_h, _, _ = g.download(with_weight=False)
    deg = np.diff(off_h.astype(np.int64))
    roots = pick_roots(off_h, args.seed + 23, 2)
    res = {"vertices": g.vertexNum, "draws": draws, "edges": g.edgeNum, "weight_offset": i0,
           "max_out_degree": int(deg.max()), "generate_s": gen_s}
    for alg in (BFS, SSSP):
        tot_ms = tot_e = 0
        for r in roots:
            ms, e = best2(g, alg, r)
            tot_ms += ms
            tot_e += e
        res[ALG_NAMES[alg]] = {"ms_per_run": tot_ms / len(roots), "gteps": tot_e / tot_ms / 1e6}
    ms, e = best2(g, PR, args.pr_iters)
    res["pagerank"] = {"ms_per_run": ms, "gteps": e / ms / 1e6}
    g.close()
    s = cg.Graph.chunglu(Vc, draws, i0, seed=args.seed, symmetrise=True, wmax=0, device=dev)
    ms, e = best2(s, CC, 0)
    res["cc"] = {"ms_per_run": ms, "gteps": e / ms / 1e6, "edges_symmetrised": s.edgeNum}
    s.close()
    out["chunglu"] = res
    if args.shapes_scale >= 1.0:
        gr = cg.Graph.grid(4800, 5000, seed=1, device=dev)
        res = {"vertices": gr.vertexNum, "edges": gr.edgeNum}
        for alg, arg in ((BFS, 0), (SSSP, 0), (CC, 0), (PR, args.pr_iters)):
            ms, e = best2(gr, alg, arg)
            res[ALG_NAMES[alg]] = {"ms_per_run": ms, "gteps": e / ms / 1e6}
        gr.close()
        out["grid4800x5000"] = res
    return out


def bench_serving(args, cg, L, dev):
    """Serving: BFS/SSSP queries (half each, seeded uniform non-isolated
    roots) with Poisson arrivals against a resident RMAT graph (scale
    --serve-scale, weights [1,64]) at 25, 50 and 100 req/s (below the
    server's capacity, so latency is service time) and at 1k, 5k and 20k
    req/s (above it: throughput), and at 2 and 1k req/s against the
    4800 x 5000 grid (weights [1,1000]); latency = completion - arrival.
    Each rate also reports the lone-run latency of its queries' median
    (one cgb_run) for comparison."""
    out = {}
    n_sub = max(32, args.serve_requests // 4)
    cases = [(f"rmat{args.serve_scale}", lambda: cg.Graph.rmat(args.serve_scale, 16, args.seed + 3, wmax=64,
                                                                   device=dev),
              ((25, n_sub), (50, n_sub), (100, n_sub), (1000, args.serve_requests), (5000, args.serve_requests),
               (20000, args.serve_requests)))]
    if args.serve_scale >= 20:
        cases.append(("grid4800x5000", lambda: cg.Graph.grid(4800, 5000, seed=1, device=dev),
                      ((2, 16), (1000, max(64, args.serve_requests // 2)))))
    for name, make, rates in cases:
        g = make()
        off_h, _, _ = g.download(with_weight=False)
        deg = np.diff(off_h.astype(np.int64))
        nzv = np.nonzero(deg)[0]
        res = {"vertices": g.vertexNum, "edges": g.edgeNum}
        with cg.Server(g) as srv:
            st = srv.stats()
            res["slots"] = {"bfs": st["bfs_slots"], "sssp": st["sssp_slots"]}
        # lone runs: the service time a query has on an idle engine
        lone = {}
        rng0 = np.random.default_rng(args.seed + 99)
        for a, an in ((BFS, "bfs"), (SSSP, "sssp")):
            ms = []
            for r in nzv[rng0.integers(0, nzv.size, 6)]:
                g.run(a, int(r), to_host=False)
                ms.append(g.stats().ms)
            lone[an] = {"median_ms": float(np.median(ms)), "max_ms": float(np.max(ms))}
        res["lone_run"] = lone
        # the batch engines' rate for the same mix: 64 BFS and 64 SSSP roots as
        # two cgb_run_batch passes (results left on the device)
        import torch
        buf = torch.empty((64, g.vertexNum), dtype=torch.int32, device=f"cuda:{dev}")
        rngb = np.random.default_rng(args.seed + 98)
        bt = {}
        for a, an in ((BFS, "bfs"), (SSSP, "sssp")):
            rb = [int(x) for x in nzv[rngb.integers(0, nzv.size, 64)]]
            g.run_batch(a, rb, out=buf)
            bt[an] = min(g.run_batch(a, rb, out=buf)[1] for _ in range(2))
        del buf
        torch.cuda.empty_cache()
        batch_rate = 128.0 / (bt["bfs"] + bt["sssp"]) * 1e3
        res["batch64"] = {"bfs_ms": bt["bfs"], "sssp_ms": bt["sssp"], "mix_rate_req_s": batch_rate}
        for rate, nreq in rates:
            rng = np.random.default_rng(args.seed * 1000 + rate)
            arrivals = np.cumsum(rng.exponential(1e6 / rate, nreq))
            algs_q = rng.integers(0, 2, nreq)
            roots_q = nzv[rng.integers(0, nzv.size, nreq)]
            with cg.Server(g) as srv:
                for a, r, t in zip(algs_q, roots_q, arrivals):
                    srv.submit(int(a), int(r), float(t))
                srv.start()
                srv.wait(600000)
                recs = srv.poll()
                sst = srv.stats()
            lat = np.array([r["done_us"] - r["arrival_us"] for r in recs]) / 1e3
            makespan = (max(r["done_us"] for r in recs) - min(r["arrival_us"] for r in recs)) / 1e6
            edges = sum(r["traversed_edges"] for r in recs)
            per = {}
            for a, an in ((BFS, "bfs"), (SSSP, "sssp")):
                la = np.array([r["done_us"] - r["arrival_us"] for r in recs if r["algorithm"] == a]) / 1e3
                if la.size:
                    per[an] = {"p50_ms": float(np.percentile(la, 50)), "p99_ms": float(np.percentile(la, 99))}
            for an in per:
                per[an]["p50_vs_lone"] = per[an]["p50_ms"] / lone[an]["median_ms"]
            res[f"rate{rate}"] = {"requests": nreq, "completed": len(recs),
                                  "errors": sum(1 for r in recs if r["status"] != 0),
                                  "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                                  "throughput_req_s": len(recs) / makespan, "gteps": edges / makespan / 1e9,
                                  "served_vs_batch_rate": len(recs) / makespan / batch_rate,
                                  "ticks": sst["ticks"], "per_algorithm": per}
        g.close()
        out[name] = res
    return out


E2E_POOL_HEADROOM = 32 << 30  # bytes added to the pool before the e2e steps


def bench_e2e(args, d, cg, gd, roots, off_h, dst_h, w_h, Es, sched):
    import torch
    from cggraph_b200 import _lib as L
    V = gd.vertexNum
    pin = lambda a: torch.from_numpy(a.view(np.int32)).pin_memory()  # noqa: E731
    t_off, t_dst, t_w = pin(off_h), pin(dst_h), pin(w_h)
    out_b = torch.empty(V, dtype=torch.int32).pin_memory()
    out_s = torch.empty(V, dtype=torch.int32).pin_memory()
    out_c = torch.empty(V, dtype=torch.int32).pin_memory()
    out_p = torch.empty(V, dtype=torch.float64).pin_memory()
    # each result lands in device memory and goes to its pinned host buffer on a
    # copy stream while the next algorithm runs (cgb_run returns once its result
    # is complete; the step waits for the copies before it ends)
    dev = f"cuda:{d.local}"
    res_b, res_s, res_c = (torch.empty(V, dtype=torch.int32, device=dev) for _ in range(3))
    res_p = torch.empty(V, dtype=torch.float64, device=dev)
    copy_stream = torch.cuda.Stream(device=dev)

    def to_host(host, res):
        with torch.cuda.stream(copy_stream):
            host.copy_(res, non_blocking=True)

    opts = cg.make_options(schedule=sched)
    cc_opts = cg.make_options(schedule=sched, flags=L.FLAG_CC_WEAK)
    steps = args.e2e_steps or args.steps

    def step(root):
        # The host-to-device link is the step's serial resource.  The graph's
        # structure goes first; a second host thread then uploads the weights
        # (only SSSP reads them; cgb_graph_set_weights) while BFS, PageRank and
        # CC (weak components of the directed graph) run; SSSP follows.
        box = {}
        weights_in = threading.Event()
        g = cg.Graph.from_csr(t_off, t_dst, None, vertexNum=V, edgeNum=gd.edgeNum, device=d.local)

        def upload_weights():
            try:
                g.set_weights(t_w)
            except BaseException as e:  # re-raised on the main thread
                box["error"] = e
            finally:
                weights_in.set()

        edges = 0
        th = threading.Thread(target=upload_weights)
        th.start()
        try:
            g.run(BFS, root, opts, out=res_b)
            to_host(out_b, res_b)
            edges += g.stats().traversed_edges
            g.run(PR, args.pr_iters, opts, out=res_p)
            to_host(out_p, res_p)
            edges += g.stats().traversed_edges
            g.run(CC, 0, cc_opts, out=res_c)
            to_host(out_c, res_c)
            edges += Es
            weights_in.wait()
            if "error" not in box:
                g.run(SSSP, root, opts, out=res_s)
                to_host(out_s, res_s)
                edges += g.stats().traversed_edges
            copy_stream.synchronize()
            g.close()
        finally:
            th.join()
        if "error" in box:
            raise box["error"]
        return edges

    # The pool is grown once, up front, to hold a step's graph at its peak
    # (as a long-running process would): growing it costs driver time.
    r0, _ = cg.memory_info(d.local)
    cg.memory_reserve(r0 + E2E_POOL_HEADROOM, d.local)
    for k in range(max(1, args.warmup)):  # warm-up: pinned pages touched, layouts of the same size cached
        step(roots[k % len(roots)])
    torch.cuda.synchronize()
    d.barrier()
    t0 = time.perf_counter()
    edges = 0
    marks = [t0]
    pool_gb = []
    for k in range(steps):
        edges += step(roots[k % len(roots)])
        marks.append(time.perf_counter())
        pool_gb.append(round(cg.memory_info(d.local)[0] / 2**30, 1))
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    d.barrier()
    s_max = d.reduce(t1 - t0, "max")
    edges = d.reduce(edges, "sum")
    h2d = 4 * (V + 1) + 8 * gd.edgeNum
    d2h = 4 * V * 3 + 8 * V
    return {"value": edges / s_max / 1e9, "unit": "GTEPS", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "ms_per_step": s_max * 1e3 / steps, "steps": steps,
            "step_ms": [round((b - a) * 1e3, 1) for a, b in zip(marks, marks[1:])],
            "pool_reserved_gb_after_step": pool_gb,
            "what": "cgb_graph_create(directed CSR structure, host pinned) + BFS + PR(20) + CC (weak components) "
                    "while a second host thread uploads the weights (cgb_graph_set_weights); SSSP once they are "
                    "in; each result -> pinned host on a copy stream during the next run; destroy; wall clock"}


def write_csr_files(dirpath, prefix, off, dst, w):
    paths = [os.path.join(dirpath, f"{prefix}_{n}.bin") for n in ("off", "dst", "w")]
    off.tofile(paths[0])
    dst.tofile(paths[1])
    if w is not None:
        w.tofile(paths[2])
    else:
        paths[2] = None
    return paths


def cpu_baseline(args, V, Ed, Es, off_h, dst_h, w_h, sym_host, roots):
    from oracle import oracle as O
    if not O.ref_available():
        return {"value": None, "unit": "GTEPS", "error": "reference harness oracle/_ref/cgref_oracle not built"}
    threads = os.cpu_count() or 1
    soff, sdst = sym_host
    tmp = "/dev/shm" if os.path.isdir("/dev/shm") else None
    with tempfile.TemporaryDirectory(dir=tmp) as dd:
        pd = write_csr_files(dd, "d", off_h, dst_h, w_h)
        ps = write_csr_files(dd, "s", soff, sdst, None)
        r3 = roots[:3]
        ib = O.ref_run_files(pd, V, Ed, 0, r3, len(r3), threads)
        isp = O.ref_run_files(pd, V, Ed, 1, r3, len(r3), threads)
        ic = O.ref_run_files(ps, V, Es, 2, [0], 2, threads)
    in_off, in_src = O.csc(off_h, dst_h)
    t0 = time.perf_counter()
    O.pagerank_pull_omp(off_h, in_off, in_src, 2, threads)
    pr_s = time.perf_counter() - t0
    edges = sum(ib["edges"]) + sum(isp["edges"]) + Es * len(ic["ms"]) + Ed * 2
    secs = (sum(ib["ms"]) + sum(isp["ms"]) + sum(ic["ms"])) / 1e3 + pr_s
    return {"value": edges / secs / 1e9, "unit": "GTEPS", "cores": int(ib["threads"]), "kind": "reference",
            "sample": f"reference Graph_Numa (MULTI_CORE) on the same RMAT-{args.scale} CSR: BFS x3 roots, "
                      f"SSSP x3 roots, CC x2 (symmetrised); PageRank by the FP64 OpenMP port (2 iterations, "
                      f"the reference's own PageRank does not build); times from the reference's own timer",
            "per_algorithm_gteps": {
                "bfs": sum(ib["edges"]) / (sum(ib["ms"]) / 1e3) / 1e9,
                "sssp": sum(isp["edges"]) / (sum(isp["ms"]) / 1e3) / 1e9,
                "cc": Es * len(ic["ms"]) / (sum(ic["ms"]) / 1e3) / 1e9,
                "pagerank_port": Ed * 2 / pr_s / 1e9}}


# ------------------------------------------------------------ reference arm
def bench_reference(args):
    """The reference's own CPU implementation (Graph_Numa, built from the
    reference sources into oracle/_ref) on this host's cores, same workload
    and metric.  PageRank uses the FP64 OpenMP port because the reference's
    PageRank does not build.  The input (the seeded RMAT CSR and its
    symmetrised copy, which the reference's CC needs) is made before any
    timing by the oracle's CPU twin of the generator, so nothing of the
    engine is loaded in this arm."""
    from oracle import oracle as O
    if not O.ref_available():
        return {"impl": "reference", "unavailable": "reference harness oracle/_ref/cgref_oracle was not built"}
    threads = os.cpu_count() or 1
    algs = [BFS, SSSP, CC, PR]
    off_h, dst_h, w_h = O.rmat_graph(args.scale, args.edge_factor, args.seed, wmax=64)
    soff, sdst, _ = O.rmat_graph(args.scale, args.edge_factor, args.seed, symmetrise=True, wmax=0)
    V, Ed, Es = off_h.size - 1, dst_h.size, sdst.size
    roots_all = pick_roots(off_h, args.seed, N_ROOTS * args.gpus)
    n = args.warmup + args.steps
    seq = [roots_all[i % len(roots_all)] for i in range(n)]
    tmp = "/dev/shm" if os.path.isdir("/dev/shm") else None
    with tempfile.TemporaryDirectory(dir=tmp) as dd:
        pd = write_csr_files(dd, "d", off_h, dst_h, w_h)
        ps = write_csr_files(dd, "s", soff, sdst, None)
        del soff, sdst
        ib = O.ref_run_files(pd, V, Ed, 0, seq, n, threads)
        isp = O.ref_run_files(pd, V, Ed, 1, seq, n, threads)
        ic = O.ref_run_files(ps, V, Es, 2, [0], n, threads)
    in_off, in_src = O.csc(off_h, dst_h)
    pr_ms = []
    for _ in range(n):
        t0 = time.perf_counter()
        O.pagerank_pull_omp(off_h, in_off, in_src, args.pr_iters, threads)
        pr_ms.append((time.perf_counter() - t0) * 1e3)
    w = args.warmup
    edges = sum(ib["edges"][w:]) + sum(isp["edges"][w:]) + Es * args.steps + Ed * args.pr_iters * args.steps
    ms = sum(ib["ms"][w:]) + sum(isp["ms"][w:]) + sum(ic["ms"][w:]) + sum(pr_ms[w:])
    value = edges / (ms / 1e3) / 1e9
    return {
        "metric": METRIC, "value": value, "unit": "GTEPS", "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32 (BFS/SSSP/CC), f64 (PageRank)",
        "data": "synthetic (seeded RMAT)",
        "config": workload_config(args, V, Ed, Es, roots_all, algs),
        "per_algorithm": {
            "bfs": sum(ib["edges"][w:]) / (sum(ib["ms"][w:]) / 1e3) / 1e9,
            "sssp": sum(isp["edges"][w:]) / (sum(isp["ms"][w:]) / 1e3) / 1e9,
            "cc": Es * args.steps / (sum(ic["ms"][w:]) / 1e3) / 1e9,
            "pagerank_port": Ed * args.pr_iters * args.steps / (sum(pr_ms[w:]) / 1e3) / 1e9},
        "cpu_baseline": {"value": value, "unit": "GTEPS", "cores": int(ib["threads"]), "kind": "reference",
                         "sample": "each step: reference Graph_Numa BFS + SSSP from the step's root and CC on the "
                                   "symmetrised graph, plus the FP64 OpenMP PageRank port; reference's own timer"},
        "e2e": {"value": value, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    args = parse_args()
    if args.impl == "reference":
        # CPU only: under torchrun rank 0 alone runs it, the other ranks exit at once
        if int(os.environ.get("RANK", "0")) == 0:
            print(json.dumps(bench_reference(args)), flush=True)
        return
    d = Dist(args.gpus)
    try:
        res = bench_cgb200(args, d)
        if d.rank == 0 and res is not None:
            print(json.dumps(res), flush=True)
    finally:
        d.close()


if __name__ == "__main__":
    main()
