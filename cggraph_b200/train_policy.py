"""Trains the learned scheduler and writes cggraph_b200/policy_weights.npy.

Training graphs (seeded, none of them a benchmark input):
  RMAT scales 18, 20, 22 and 24 (a=.57, b=.19, c=.19, edge factor 16,
  weights U[1,64]; seeds 2..5, the benchmark uses seed 1) and scales 20 and
  22 with edge factors 4 and 8, Chung-Lu power-law graphs of 1, 2 and 4 M
  vertices (the benchmark's degree exponent, seeds 2..4) and 2-D grids
  256x256 to 4096x4096, 1024x4096 and 4800x5000 (weights U[1,1000]; the
  benchmark's grid is seed 1, this one seed 9).
For each graph and a few seeded roots (3 for BFS, 8 for SSSP) the engine
records counterfactual samples (cgb_policy_collect): every BFS level timed as
a binned push, a chunked push and a pull; at the first SSSP bucket boundary
the rest of the run timed with delta x {1/4, 1/2, 1, 2, 4, 8, 16}; every
large SSSP near round timed as each of its four variants.
The network is trained on the GPU by the engine's own kernels
(cgb_policy_train).

  python -m cggraph_b200.train_policy [--quick] [--out PATH] [--epochs N]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time
import zlib

import numpy as np

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import cggraph_b200 as cg  # noqa: E402
from cggraph_b200 import policy  # noqa: E402

BFS, SSSP = 0, 1


def training_graphs(quick: bool):
    if quick:
        yield "rmat16_s2", lambda: cg.Graph.rmat(16, 16, seed=2)
        yield "grid128_s2", lambda: cg.Graph.grid(128, 128, seed=2)
        return
    for scale, seed in ((18, 2), (20, 3), (22, 4), (24, 5)):
        yield f"rmat{scale}_s{seed}", (lambda s=scale, d=seed: cg.Graph.rmat(s, 16, seed=d))
    for scale, ef, seed in ((20, 4, 6), (20, 8, 7), (22, 4, 8), (22, 8, 9)):
        yield f"rmat{scale}_ef{ef}_s{seed}", (lambda s=scale, e=ef, d=seed: cg.Graph.rmat(s, e, seed=d))
    for vc, seed in ((1_000_000, 2), (2_000_000, 4), (4_000_000, 3)):
        draws = int(vc * 35.3)  # the benchmark's draws per vertex (1.47 B / 41.6 M)
        i0 = cg.chunglu_weight_offset(vc, draws, max(1, int(vc * 0.072)))
        yield f"chunglu{vc // 1_000_000}m_s{seed}", (lambda v=vc, n=draws, o=i0, d=seed: cg.Graph.chunglu(v, n, o, seed=d))
    for n, seed in ((256, 2), (512, 3), (1024, 4), (2048, 6), (4096, 7)):
        yield f"grid{n}_s{seed}", (lambda n=n, d=seed: cg.Graph.grid(n, n, seed=d))
    yield "grid1024x4096_s8", lambda: cg.Graph.grid(1024, 4096, seed=8)
    # the benchmark's grid shape with another seed (2 BFS and 4 SSSP roots)
    yield "grid4800x5000_s9", lambda: cg.Graph.grid(4800, 5000, seed=9)


def collect_all(quick: bool, roots_per_graph: int = 3, sssp_roots: int = 8, log=print):
    Xs, Ts, Ms, info = [], [], [], []
    for name, make in training_graphs(quick):
        g = make()
        off, _, _ = g.download(with_weight=False)
        deg = np.diff(off.astype(np.int64))
        rng = np.random.default_rng(zlib.crc32(name.encode()))
        cand = np.nonzero(deg)[0]
        nb, ns = (2, 4) if name.startswith("grid4800") else (roots_per_graph, sssp_roots)
        nr = max(nb, ns)
        roots = [int(deg.argmax())] + [int(x) for x in rng.choice(cand, nr - 1, replace=False)]
        for i, r in enumerate(roots):
            for alg in (BFS, SSSP):
                if i >= (nb if alg == BFS else ns):
                    continue
                t0 = time.time()
                X, T, M = policy.collect(g, alg, r)
                Xs.append(X)
                Ts.append(T)
                Ms.append(M)
                info.append({"graph": name, "root": r, "alg": ["bfs", "sssp"][alg], "samples": len(X)})
                log(f"  {name} root {r} {['bfs', 'sssp'][alg]}: {len(X)} samples ({time.time() - t0:.1f} s)")
        g.close()
    return np.concatenate(Xs), np.concatenate(Ts), np.concatenate(Ms), info


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--quick", action="store_true")
    ap.add_argument("--out", default=policy.DEFAULT_WEIGHTS)
    ap.add_argument("--epochs", type=int, default=400)
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args(argv)
    X, T, M, info = collect_all(args.quick)
    print(f"{len(X)} samples; training {args.epochs} epochs on the GPU")
    t0 = time.time()
    params, loss = policy.train(X, T, M, epochs=args.epochs, batch=256, lr=3e-3, seed=args.seed)
    print(f"final mean squared error of log-costs {loss:.4f} ({time.time() - t0:.1f} s)")
    np.save(args.out, params)
    np.savez_compressed(os.path.splitext(args.out)[0] + "_data.npz", X=X, T=T, M=M)
    summary = {"samples": int(len(X)), "epochs": args.epochs, "final_loss": loss, "runs": info}
    with open(os.path.splitext(args.out)[0] + ".json", "w") as f:
        json.dump(summary, f, indent=1)
    return params, loss


if __name__ == "__main__":
    main()
