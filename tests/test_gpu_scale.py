"""Parity at the benchmark's sizes.

RMAT scale 20 (1,048,576 vertices, ~16.8 M edges before dedup): every value
compared with the oracle.  RMAT scale 24 (16.8 M vertices, ~268 M edges):
size-independent properties checked on the GPU -- BFS levels and SSSP
distances satisfy their Bellman fixpoint equation exactly (which has a unique
solution for positive weights), CC labels are constant along every edge and
each label is its class's minimum vertex and its own label, and the
20-iteration PageRank equals one FP64 pull step applied to the engine's own
19-iteration result."""
import numpy as np
import pytest

import cggraph_b200 as cg

pytestmark = pytest.mark.gpu

BFS, SSSP, CC, PR = 0, 1, 2, 3
VMAX = 999999999


def test_rmat20_full_parity(oracle):
    off, dst, w = oracle.rmat_graph(20, 16, seed=1)
    with cg.Graph.rmat(20, 16, seed=1) as g:
        o2, d2, w2 = g.download()
        np.testing.assert_array_equal(o2, off)
        np.testing.assert_array_equal(d2, dst)
        np.testing.assert_array_equal(w2, w)
        root = int(np.diff(off.astype(np.int64)).argmax())
        np.testing.assert_array_equal(g.run(BFS, root)[0], oracle.bfs(off, dst, root))
        np.testing.assert_array_equal(g.run(SSSP, root)[0], oracle.sssp(off, dst, w, root))
        np.testing.assert_array_equal(g.run(CC)[0], oracle.cc(off, dst))
        exp = oracle.pagerank(off, dst, 20)
        got = g.run(PR, 20)[0]
        assert np.max(np.abs(got - exp) / exp) <= 1e-6
    so, sd, sw = oracle.rmat_graph(20, 16, seed=1, symmetrise=True)
    with cg.Graph.rmat(20, 16, seed=1, symmetrise=True) as g:
        np.testing.assert_array_equal(g.run(CC)[0], oracle.wcc_unionfind(so, sd))


def _edge_tensors(g):
    import torch
    o, d, w = g.download()
    off = torch.from_numpy(o.astype(np.int64)).cuda()
    dst = torch.from_numpy(d.astype(np.int64)).cuda()
    wt = torch.from_numpy(w.astype(np.int64)).cuda() if w is not None else None
    deg = off[1:] - off[:-1]
    src = torch.repeat_interleave(torch.arange(g.vertexNum, device="cuda"), deg)
    return src, dst, wt, deg


def _bellman_ok(val, src, dst, wt, root):
    import torch
    V = val.numel()
    v = val.to(torch.int64)
    reached = v[src] != VMAX
    cand = torch.where(reached, v[src] + wt, torch.full_like(src, VMAX))
    cand = torch.clamp(cand, max=VMAX)
    best = torch.full((V,), VMAX, dtype=torch.int64, device="cuda")
    best.scatter_reduce_(0, dst, cand, reduce="amin")
    best[root] = 0
    return bool(torch.equal(best, v))


def test_rmat24_properties():
    import torch
    with cg.Graph.rmat(24, 16, seed=1) as g:
        src, dst, wt, deg = _edge_tensors(g)
        rng = np.random.default_rng(0)
        nz = torch.nonzero(deg).flatten().cpu().numpy()
        for root in [int(torch.argmax(deg).item()), int(rng.choice(nz))]:
            bfs = torch.from_numpy(g.run(BFS, root)[0].astype(np.int64)).cuda()
            assert _bellman_ok(bfs, src, dst, torch.ones_like(dst), root)
            sssp = torch.from_numpy(g.run(SSSP, root)[0].astype(np.int64)).cuda()
            assert _bellman_ok(sssp, src, dst, wt, root)
            # a vertex is reached by SSSP iff it is reached by BFS
            assert torch.equal(bfs == VMAX, sssp == VMAX)
        # PageRank: pr20 == one pull step of pr19
        pr19 = torch.from_numpy(g.run(PR, 19)[0]).cuda()
        pr20 = torch.from_numpy(g.run(PR, 20)[0]).cuda()
        V = g.vertexNum
        contrib = torch.where(deg > 0, pr19 / deg.clamp(min=1).double(), torch.zeros_like(pr19))
        acc = torch.zeros(V, dtype=torch.float64, device="cuda").index_add_(0, dst, contrib[src])
        step = 0.15 / V + 0.85 * acc
        assert float(torch.max(torch.abs(step - pr20) / pr20)) < 1e-9
        del src, dst, wt
    with cg.Graph.rmat(24, 16, seed=1, symmetrise=True, wmax=0) as g:
        src, dst, _, _ = _edge_tensors(g)
        lab = torch.from_numpy(g.run(CC)[0].astype(np.int64)).cuda()
        V = g.vertexNum
        ids = torch.arange(V, device="cuda")
        assert torch.equal(lab[src], lab[dst])              # constant along edges
        assert bool(torch.all(lab <= ids))
        assert torch.equal(lab[lab], lab)                   # the label is its own label
        mn = torch.full((V,), V, dtype=torch.int64, device="cuda").scatter_reduce_(0, lab, ids, reduce="amin")
        assert torch.equal(mn[lab], lab)                    # and the class minimum
