"""Parity at the benchmark's sizes, bit for bit against the oracle.

* RMAT scale 20 (1,048,576 vertices): every value of all four algorithms,
  and the device generator equal to the oracle's CPU twin.
* RMAT scale 24 (16.8 M vertices, 263 M directed edges), the benchmark's own
  graph (seed 1) and roots: BFS and SSSP from two of the timed roots under
  the heuristic and the learned schedule, equal to the oracle's queue BFS and
  Dijkstra, and for one root to the reference's own engine (Graph_Numa) where
  its harness is built; CC as weak components of the directed graph
  (CGB_FLAG_CC_WEAK, the benchmark's CC) and on the symmetrised graph, each
  equal to union-find, and the reference's directed label propagation equal
  to the oracle's; PageRank(20) within 1e-6 relative of the oracle's FP64
  pull, and equal (1e-9) to one FP64 pull step of the engine's own PR(19).
* The 4800 x 5000 grid (24 M vertices, diameter ~9,800): BFS and SSSP from a
  corner and from the centre, CC, PageRank.
* Chung-Lu at a tenth of the benchmark's shape (4.16 M vertices, 147 M edge
  draws, the same degree exponent and weights): all four algorithms, CC both
  as reference label propagation and as weak components.

The engine's device generators build the graphs (their CPU twin equality is
checked at scale 20 here and at smaller sizes elsewhere); the CSR is then
downloaded and handed to the oracle.
"""
import os

import numpy as np
import pytest

import cggraph_b200 as cg
from cggraph_b200 import _lib as L

pytestmark = pytest.mark.gpu

BFS, SSSP, CC, PR = 0, 1, 2, 3
VMAX = 999999999


def bench_roots(off, seed, n):
    """The benchmark's roots: seeded uniform choice among non-isolated vertices."""
    deg = np.diff(off.astype(np.int64))
    cand = np.nonzero(deg)[0]
    rng = np.random.default_rng(seed + 1000)
    return [int(x) for x in rng.choice(cand, size=min(n, cand.size), replace=False)]


def _n_labels(lab):
    return int(np.unique(lab).size)


def _pr_close(got, exp, tol=1e-6):
    rel = float(np.max(np.abs(got - exp) / exp))
    assert rel <= tol, f"PageRank max relative error {rel}"
    return rel


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
        weak = cg.make_options(flags=L.FLAG_CC_WEAK)
        np.testing.assert_array_equal(g.run(CC, 0, weak)[0], oracle.wcc_unionfind(off, dst))
        _pr_close(g.run(PR, 20)[0], oracle.pagerank(off, dst, 20))
    so, sd, sw = oracle.rmat_graph(20, 16, seed=1, symmetrise=True)
    with cg.Graph.rmat(20, 16, seed=1, symmetrise=True) as g:
        np.testing.assert_array_equal(g.run(CC)[0], oracle.wcc_unionfind(so, sd))


@pytest.fixture(scope="module")
def rmat24():
    g = cg.Graph.rmat(24, 16, seed=1)
    off, dst, w = g.download()
    yield g, off, dst, w
    g.close()


def test_rmat24_bfs_sssp_bench_roots(oracle, rmat24):
    g, off, dst, w = rmat24
    from cggraph_b200 import policy
    roots = bench_roots(off, 1, 10)[:2]
    for r in roots:
        exp_b = oracle.bfs(off, dst, r)
        exp_s = oracle.sssp(off, dst, w, r)
        np.testing.assert_array_equal(g.run(BFS, r)[0], exp_b, err_msg=f"BFS root {r}")
        np.testing.assert_array_equal(g.run(SSSP, r)[0], exp_s, err_msg=f"SSSP root {r}")
        if policy.load_default():
            try:
                learned = cg.make_options(schedule=L.SCHED_LEARNED)
                np.testing.assert_array_equal(g.run(BFS, r, learned)[0], exp_b, err_msg=f"learned BFS root {r}")
                np.testing.assert_array_equal(g.run(SSSP, r, learned)[0], exp_s, err_msg=f"learned SSSP root {r}")
            finally:
                policy.load(None)
        # a vertex is reached by SSSP iff it is reached by BFS
        assert np.array_equal(exp_b == VMAX, exp_s == VMAX)


def test_rmat24_matches_reference_engine(oracle, rmat24):
    """The reference's own MULTI_CORE engine (Graph_Numa) on the benchmark's
    graph and first timed root: BFS levels and SSSP distances."""
    if not oracle.ref_available():
        pytest.skip("reference engine harness (oracle/_ref/cgref_oracle) not built")
    g, off, dst, w = rmat24
    r = bench_roots(off, 1, 10)[0]
    tmp = "/dev/shm" if os.path.isdir("/dev/shm") else None
    for alg in (BFS, SSSP):
        ref, _, _ = oracle.ref_run(off, dst, w, alg, r, runs=1, tmpdir=tmp)
        np.testing.assert_array_equal(g.run(alg, r)[0], ref, err_msg=f"alg {alg} root {r}")


def test_rmat24_cc(oracle, rmat24):
    g, off, dst, _ = rmat24
    exp_weak = oracle.wcc_unionfind(off, dst)
    got = g.run(CC, 0, cg.make_options(flags=L.FLAG_CC_WEAK))[0]
    np.testing.assert_array_equal(got, exp_weak)
    assert g.stats().cc_path == 2
    # the reference's semantics on the directed graph: label = min{u : u reaches v}
    np.testing.assert_array_equal(g.run(CC)[0], oracle.cc(off, dst))
    with cg.Graph.rmat(24, 16, seed=1, symmetrise=True, wmax=0) as s:
        so, sd, _ = s.download(with_weight=False)
        exp = oracle.wcc_unionfind(so, sd)
        lab = s.run(CC)[0]
        np.testing.assert_array_equal(lab, exp)
        assert _n_labels(lab) == _n_labels(exp)
        # weak components of the directed graph are the symmetrised graph's components
        np.testing.assert_array_equal(exp, exp_weak)


def test_rmat24_pagerank(oracle, rmat24):
    import torch
    g, off, dst, _ = rmat24
    in_off, in_src = oracle.csc(off, dst)
    exp = oracle.pagerank_pull_omp(off, in_off, in_src, 20)
    pr20 = g.run(PR, 20)[0]
    _pr_close(pr20, exp)
    # pr20 == one FP64 pull step of the engine's own pr19
    pr19 = torch.from_numpy(g.run(PR, 19)[0]).cuda()
    o = torch.from_numpy(off.astype(np.int64)).cuda()
    d = torch.from_numpy(dst.astype(np.int64)).cuda()
    deg = o[1:] - o[:-1]
    src = torch.repeat_interleave(torch.arange(g.vertexNum, device="cuda"), deg)
    V = g.vertexNum
    contrib = torch.where(deg > 0, pr19 / deg.clamp(min=1).double(), torch.zeros_like(pr19))
    acc = torch.zeros(V, dtype=torch.float64, device="cuda").index_add_(0, d, contrib[src])
    step = 0.15 / V + 0.85 * acc
    got = torch.from_numpy(pr20).cuda()
    assert float(torch.max(torch.abs(step - got) / got)) < 1e-9


def test_grid4800x5000(oracle):
    with cg.Graph.grid(4800, 5000, seed=1) as g:
        off, dst, w = g.download()
        go, gd, gw = oracle.grid_graph(4800, 5000, seed=1)
        np.testing.assert_array_equal(off, go)
        np.testing.assert_array_equal(dst, gd)
        np.testing.assert_array_equal(w, gw)
        V = g.vertexNum
        for r in (0, (4800 // 2) * 5000 + 2500):
            np.testing.assert_array_equal(g.run(BFS, r)[0], oracle.bfs(off, dst, r), err_msg=f"BFS root {r}")
            np.testing.assert_array_equal(g.run(SSSP, r)[0], oracle.sssp(off, dst, w, r), err_msg=f"SSSP root {r}")
        lab = g.run(CC)[0]
        np.testing.assert_array_equal(lab, oracle.wcc_unionfind(off, dst))
        assert np.all(lab == 0)
        np.testing.assert_array_equal(g.run(CC, 0, cg.make_options(flags=L.FLAG_CC_WEAK))[0], lab)
        in_off, in_src = oracle.csc(off, dst)
        _pr_close(g.run(PR, 20)[0], oracle.pagerank_pull_omp(off, in_off, in_src, 20))
        assert V == 24_000_000


def test_chunglu_tenth_of_bench_shape(oracle):
    Vc = 4_160_000
    draws, i0 = cg.chunglu_draws_for_edges(Vc, 147_000_000, 300_000)
    with cg.Graph.chunglu(Vc, draws, i0, seed=1) as g:
        off, dst, w = g.download()
        deg = np.diff(off.astype(np.int64))
        roots = [int(deg.argmax())] + bench_roots(off, 23, 2)
        for r in roots:
            np.testing.assert_array_equal(g.run(BFS, r)[0], oracle.bfs(off, dst, r), err_msg=f"BFS root {r}")
            np.testing.assert_array_equal(g.run(SSSP, r)[0], oracle.sssp(off, dst, w, r), err_msg=f"SSSP root {r}")
        np.testing.assert_array_equal(g.run(CC)[0], oracle.cc(off, dst))
        weak = g.run(CC, 0, cg.make_options(flags=L.FLAG_CC_WEAK))[0]
        np.testing.assert_array_equal(weak, oracle.wcc_unionfind(off, dst))
        in_off, in_src = oracle.csc(off, dst)
        _pr_close(g.run(PR, 20)[0], oracle.pagerank_pull_omp(off, in_off, in_src, 20))
    # the CPU twin builds the same graph
    co, cd, cw = oracle.chunglu_graph(Vc, draws, i0, seed=1)
    np.testing.assert_array_equal(co, off)
    np.testing.assert_array_equal(cd, dst)
    np.testing.assert_array_equal(cw, w)
