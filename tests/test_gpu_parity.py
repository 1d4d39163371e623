"""Engine vs oracle parity on the GPU, through the C ABI.

BFS / SSSP / CC results must be bit-identical to the reference (golden
fixtures from its Graph_Numa engine, and the oracle's restatement, itself
pinned to those fixtures); PageRank must be within a max per-vertex relative
error of 1e-6 of the FP64 oracle."""
import numpy as np
import pytest

import cggraph_b200 as cg
from cggraph_b200 import _lib as L
from conftest import GOLDEN, load_golden

pytestmark = pytest.mark.gpu

BFS, SSSP, CC, PR = 0, 1, 2, 3
PR_RTOL = 1e-6  # max per-vertex relative error allowed for PageRank


def pr_close(a, b):
    rel = np.max(np.abs(a - b) / np.abs(b))
    assert rel <= PR_RTOL, rel
    return rel


SCHEDULES = {
    "heuristic": None,
    "push_only": lambda: cg.make_options(schedule=L.SCHED_FIXED, variant=L.VAR_PUSH),
    "pull_only": lambda: cg.make_options(schedule=L.SCHED_FIXED, variant=L.VAR_PULL),
    "learned": lambda: cg.make_options(schedule=L.SCHED_LEARNED),
}


@pytest.mark.parametrize("name", GOLDEN)
def test_golden_bfs_sssp_cc(name):
    gd = load_golden(name)
    with cg.Graph.from_csr(gd["offsets"], gd["dest"], gd["weight"]) as g:
        for r in gd["roots"].tolist():
            for sname, mk in SCHEDULES.items():
                got, _ = g.run(BFS, r, mk() if mk else None)
                np.testing.assert_array_equal(got, gd[f"bfs_{r}"], err_msg=f"BFS root {r} {sname}")
            got, _ = g.run(SSSP, r)
            np.testing.assert_array_equal(got, gd[f"sssp_{r}"], err_msg=f"SSSP root {r}")
        got, _ = g.run(CC)
        np.testing.assert_array_equal(got, gd["cc"])


@pytest.mark.parametrize("name", GOLDEN)
def test_golden_pagerank(name, oracle):
    gd = load_golden(name)
    with cg.Graph.from_csr(gd["offsets"], gd["dest"], gd["weight"]) as g:
        for iters in (1, 20):
            got, _ = g.run(PR, iters)
            pr_close(got, oracle.pagerank(gd["offsets"], gd["dest"], iters))


def test_device_generator_matches_oracle_twin(oracle):
    for scale, sym in ((12, False), (12, True), (14, False)):
        with cg.Graph.rmat(scale, 16, seed=3, symmetrise=sym) as g:
            off, dst, w = g.download()
            o2, d2, w2 = oracle.rmat_graph(scale, 16, seed=3, symmetrise=sym)
            np.testing.assert_array_equal(off, o2)
            np.testing.assert_array_equal(dst, d2)
            np.testing.assert_array_equal(w, w2)
            assert g.symmetric == (1 if sym else -1)
    with cg.Graph.grid(40, 50, seed=9) as g:
        off, dst, w = g.download()
        o2, d2, w2 = oracle.grid_graph(40, 50, seed=9)
        np.testing.assert_array_equal(off, o2)
        np.testing.assert_array_equal(dst, d2)
        np.testing.assert_array_equal(w, w2)


@pytest.mark.parametrize("sym", [False, True])
def test_rmat16_all_algorithms(oracle, sym):
    off, dst, w = oracle.rmat_graph(16, 16, seed=21, symmetrise=sym)
    deg = np.diff(off.astype(np.int64))
    roots = [int(deg.argmax()), int(np.nonzero(deg)[0][7]), 0]
    with cg.Graph.from_csr(off, dst, w) as g:
        for r in roots:
            exp_b = oracle.bfs(off, dst, r)
            for sname, mk in SCHEDULES.items():
                got, _ = g.run(BFS, r, mk() if mk else None)
                np.testing.assert_array_equal(got, exp_b, err_msg=f"BFS {r} {sname}")
            got, _ = g.run(SSSP, r)
            np.testing.assert_array_equal(got, oracle.sssp(off, dst, w, r))
            for delta in (1, 7, 500):
                got, _ = g.run(SSSP, r, cg.make_options(sssp_delta=delta))
                np.testing.assert_array_equal(got, oracle.sssp(off, dst, w, r), err_msg=f"delta {delta}")
        got, _ = g.run(CC)
        np.testing.assert_array_equal(got, oracle.cc(off, dst))
        assert g.stats().cc_path == (0 if sym else 1)
        got, _ = g.run(PR, 20)
        pr_close(got, oracle.pagerank(off, dst, 20))


def test_grid_high_diameter(oracle):
    off, dst, w = oracle.grid_graph(60, 90, seed=4)
    with cg.Graph.from_csr(off, dst, w) as g:
        for r in (0, 2711):
            got, _ = g.run(BFS, r)
            np.testing.assert_array_equal(got, oracle.bfs(off, dst, r))
            got, _ = g.run(SSSP, r)
            np.testing.assert_array_equal(got, oracle.sssp(off, dst, w, r))
        got, _ = g.run(CC)
        np.testing.assert_array_equal(got, oracle.cc(off, dst))


def test_graph_reference_driver(oracle, tmp_path):
    """main_partition-style driver: runs, trimmed mean, result, checkBinResult."""
    gd = load_golden("rmat10_s7")
    csr = cg.CSR_Result_type(int(gd["offsets"].size - 1), int(gd["dest"].size), gd["offsets"], gd["dest"],
                             gd["weight"])
    r = int(gd["roots"][0])
    res = cg.main_partition(csr, cg.Algorithm_type.SSSP, root=r, runs=4)
    assert len(res["times"]) == 4 and res["total_run_time_ms"] > 0
    golden = tmp_path / f"rmat10_SSSP_{r}.bin"
    gd[f"sssp_{r}"].tofile(golden)
    cg.checkBinResult(str(golden), res["vertexValue"], csr.vertexNum)
    # root outside [0, V): nothing runs (main_partition.hpp:330)
    res = cg.main_partition(csr, cg.Algorithm_type.BFS, root=csr.vertexNum)
    assert res["times"] == []


def test_graphb200_adapter_surface(oracle):
    gd = load_golden("toy_0")
    csr = cg.CSR_Result_type(12, 26, gd["offsets"], gd["dest"], gd["weight"])
    eng = cg.GraphB200(csr, cg.Algorithm_type.BFS)
    ms = eng.graphProcess_device(cg.Algorithm_type.BFS, 0)
    assert ms >= 0
    eng.result_D2H()
    assert eng.vertexValue.tolist() == [0, 1, 4, 1, 4, 2, 2, 1, 3, 2, 999999999, 3]
    eng.graphProcess_device(cg.Algorithm_type.PR, 20)
    eng.result_D2H()
    assert eng.vertexValue.dtype == np.float64
    pr_close(eng.vertexValue, oracle.pagerank(gd["offsets"], gd["dest"], 20))
    eng.close()


def test_batch_equals_single_runs(oracle):
    off, dst, w = oracle.rmat_graph(13, 16, seed=2)
    roots = [0, 5, 17, 99, 1234]
    with cg.Graph.from_csr(off, dst, w) as g:
        for alg in (BFS, SSSP):
            out, ms = g.run_batch(alg, roots)
            for i, r in enumerate(roots):
                exp = oracle.bfs(off, dst, r) if alg == BFS else oracle.sssp(off, dst, w, r)
                np.testing.assert_array_equal(out[i], exp)
