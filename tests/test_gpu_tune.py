"""Launch-parameter tuning: every tuning gives the same results, and the
autotuner returns a tuning no slower than where it started."""
import numpy as np
import pytest

import cggraph_b200 as cg

pytestmark = pytest.mark.gpu

BFS, SSSP, CC, PR = 0, 1, 2, 3

TUNINGS = [
    {},
    {"push_big_deg": 128, "push_chunk": 256, "push_ctas_per_sm": 1, "persist_enter": 0, "ms_edges": 64,
     "pr_unroll": 4, "pr_ctas_per_sm": 1},
    {"push_big_deg": 65536, "push_chunk": 65536, "push_ctas_per_sm": 32, "persist_enter": 1 << 30,
     "persist_deg": 65536, "ms_edges": 4096, "pr_unroll": 16, "pr_ctas_per_sm": 1024},
    {"push_big_deg": 300, "push_chunk": 512, "push_ctas_per_sm": 3, "persist_enter": 100, "persist_deg": 64,
     "persist_ctas": 5},
    {"persist_ctas": 1},
    {"sssp_pull_alpha": 1000, "persist_enter": 0},
    {"sssp_pull_alpha": 0},
    {"cluster_enter": 0},
    {"sssp_dense_alpha": 1000},
    {"sssp_dense_alpha": 0, "sssp_pull_alpha": 0},
    {"cluster_enter": 1 << 20},
    {"push_block": 128},
    {"push_block": 512, "push_ctas_per_sm": 2},
]


@pytest.mark.parametrize("sym", [False, True])
def test_results_identical_under_every_tuning(oracle, sym):
    off, dst, w = oracle.rmat_graph(15, 16, seed=17, symmetrise=sym)
    deg = np.diff(off.astype(np.int64))
    roots = [int(deg.argmax()), int(np.nonzero(deg)[0][3])]
    exp_b = [oracle.bfs(off, dst, r) for r in roots]
    exp_s = [oracle.sssp(off, dst, w, r) for r in roots]
    exp_c = oracle.cc(off, dst)
    pr_ref = None
    with cg.Graph.from_csr(off, dst, w) as g:
        for t in TUNINGS:
            g.set_tuning({**cg.DEFAULT_TUNING, **t})
            for r, eb, es in zip(roots, exp_b, exp_s):
                np.testing.assert_array_equal(g.run(BFS, r)[0], eb, err_msg=str(t))
                np.testing.assert_array_equal(g.run(SSSP, r)[0], es, err_msg=str(t))
            np.testing.assert_array_equal(g.run(CC)[0], exp_c, err_msg=str(t))
            pr, _ = g.run(PR, 20)
            if pr_ref is None:
                pr_ref = pr
            np.testing.assert_array_equal(pr, pr_ref, err_msg=str(t))  # fixed summation order: bit-identical
            out, _ = g.run_batch(SSSP, roots)
            np.testing.assert_array_equal(out, np.stack(exp_s), err_msg=str(t))
            out, _ = g.run_batch(BFS, roots)
            np.testing.assert_array_equal(out, np.stack(exp_b), err_msg=str(t))


def test_grid_under_tunings(oracle):
    off, dst, w = oracle.grid_graph(50, 70, seed=8)
    with cg.Graph.from_csr(off, dst, w) as g:
        for t in TUNINGS:
            g.set_tuning({**cg.DEFAULT_TUNING, **t})
            np.testing.assert_array_equal(g.run(BFS, 17)[0], oracle.bfs(off, dst, 17))
            np.testing.assert_array_equal(g.run(SSSP, 17)[0], oracle.sssp(off, dst, w, 17))


def test_autotune_and_range_checks(oracle):
    off, dst, w = oracle.rmat_graph(14, 16, seed=3)
    deg = np.diff(off.astype(np.int64))
    roots = [int(x) for x in np.nonzero(deg)[0][:2]]
    with cg.Graph.from_csr(off, dst, w) as g:
        assert g.get_tuning(BFS) == cg.DEFAULT_TUNING
        best, best_ms, start_ms = g.autotune(BFS, roots, keep=False)
        assert best_ms <= start_ms
        assert g.get_tuning(BFS) == cg.DEFAULT_TUNING
        best, best_ms, start_ms = g.autotune(SSSP, roots * 3, batch=True)
        assert best_ms <= start_ms
        assert g.get_tuning(SSSP) == best
        assert g.get_tuning(BFS) == cg.DEFAULT_TUNING  # tunings are per algorithm
        np.testing.assert_array_equal(g.run(SSSP, roots[0])[0], oracle.sssp(off, dst, w, roots[0]))
        best_pr, pms, psms = g.autotune(PR, [5, 5])
        assert pms <= psms and g.get_tuning(PR) == best_pr
        for bad in ({"push_big_deg": 64}, {"push_chunk": 1000}, {"push_ctas_per_sm": 0}, {"ms_edges": 8192},
                    {"persist_deg": 1}, {"pr_unroll": 6}, {"pr_ctas_per_sm": 1025}, {"push_block": 300},
                    {"push_block": 1024}):
            with pytest.raises(cg.CgbError):
                g.set_tuning(bad, SSSP)
        assert g.get_tuning(SSSP) == best
