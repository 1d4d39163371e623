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


@pytest.mark.parametrize("sym", [False, True])
def test_chunglu_generator_and_algorithms(oracle, sym):
    """Chung-Lu power-law graph (non-power-of-two V): the device generator
    equals its CPU twin bit for bit, and all four algorithms match the oracle."""
    V, n, i0 = 20011, 300000, 5
    off, dst, w = oracle.chunglu_graph(V, n, i0, seed=11, symmetrise=sym)
    with cg.Graph.chunglu(V, n, i0, seed=11, symmetrise=sym) as g:
        o2, d2, w2 = g.download()
        np.testing.assert_array_equal(o2, off)
        np.testing.assert_array_equal(d2, dst)
        np.testing.assert_array_equal(w2, w)
        deg = np.diff(off.astype(np.int64))
        for r in (int(deg.argmax()), int(np.nonzero(deg)[0][5])):
            np.testing.assert_array_equal(g.run(BFS, r)[0], oracle.bfs(off, dst, r))
            np.testing.assert_array_equal(g.run(SSSP, r)[0], oracle.sssp(off, dst, w, r))
        np.testing.assert_array_equal(g.run(CC)[0], oracle.cc(off, dst))
        pr_close(g.run(PR, 20)[0], oracle.pagerank(off, dst, 20))


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


def test_multi_root_bfs_passes(oracle):
    """Bit-packed multi-root BFS: 70 roots (two passes of <= 64), duplicates,
    a root without out-edges, device-resident output."""
    import torch
    off, dst, w = oracle.rmat_graph(14, 16, seed=12)
    deg = np.diff(off.astype(np.int64))
    rng = np.random.default_rng(5)
    roots = [int(x) for x in rng.choice(off.size - 1, 68, replace=False)]
    roots += [roots[3], int(np.nonzero(deg == 0)[0][0])]
    with cg.Graph.from_csr(off, dst, w) as g:
        out, ms = g.run_batch(BFS, roots)
        assert ms > 0
        for i, r in enumerate(roots):
            np.testing.assert_array_equal(out[i], oracle.bfs(off, dst, r), err_msg=f"root {i}")
        d_out = torch.empty((len(roots), off.size - 1), dtype=torch.int32, device="cuda")
        g.run_batch(BFS, roots, out=d_out)
        np.testing.assert_array_equal(d_out.cpu().numpy().view(np.uint32), out)
        assert g.stats().traversed_edges == sum(int(deg[out[i] != 999999999].sum()) for i in range(len(roots)))



@pytest.mark.parametrize("weighted", [True, False])
def test_multi_root_sssp_passes(oracle, weighted):
    """Multi-root SSSP: 70 roots (passes of 64 and 6), a duplicate root, a
    root without out-edges, several bucket widths, device-resident output,
    and the one-by-one path giving the same distances."""
    import torch
    off, dst, w = oracle.rmat_graph(14, 16, seed=13)
    if not weighted:
        w = None
    deg = np.diff(off.astype(np.int64))
    rng = np.random.default_rng(6)
    roots = [int(x) for x in rng.choice(off.size - 1, 68, replace=False)]
    roots += [roots[5], int(np.nonzero(deg == 0)[0][0])]
    w_or = w if weighted else np.ones_like(dst)
    exp = np.stack([oracle.sssp(off, dst, w_or, r) for r in roots])
    with cg.Graph.from_csr(off, dst, w) as g:
        out, ms = g.run_batch(SSSP, roots)
        assert ms > 0
        np.testing.assert_array_equal(out, exp)
        assert g.stats().traversed_edges == sum(int(deg[exp[i] != 999999999].sum()) for i in range(len(roots)))
        for delta in (1, 13, 100000):
            out, _ = g.run_batch(SSSP, roots[:64], cg.make_options(sssp_delta=delta))
            np.testing.assert_array_equal(out, exp[:64], err_msg=f"delta {delta}")
        d_out = torch.empty((len(roots), off.size - 1), dtype=torch.int32, device="cuda")
        g.run_batch(SSSP, roots, out=d_out)
        np.testing.assert_array_equal(d_out.cpu().numpy().view(np.uint32), exp)
        seq, _ = g.run_batch(SSSP, roots[:5], cg.make_options(flags=L.FLAG_BATCH_SEQUENTIAL))
        np.testing.assert_array_equal(seq, exp[:5])

def _batch_graphs(oracle):
    """Uneven graphs: RMAT of scales 8-12 (directed and symmetric), grids,
    a graph without edges, one with a single vertex."""
    gs = []
    for i, scale in enumerate((8, 9, 10, 11, 12, 10, 9)):
        gs.append(oracle.rmat_graph(scale, 8 + 2 * i, seed=40 + i, symmetrise=bool(i % 2)))
    gs.append(oracle.grid_graph(17, 23, seed=3))
    gs.append(oracle.grid_graph(1, 40, seed=4))
    gs.append((np.zeros(6, np.uint32), np.zeros(0, np.uint32), np.zeros(0, np.uint32)))
    gs.append((np.zeros(2, np.uint32), np.zeros(0, np.uint32), np.zeros(0, np.uint32)))
    return gs


def test_graph_batch_matches_oracle(oracle):
    gs = _batch_graphs(oracle)
    rng = np.random.default_rng(8)
    with cg.Batch(gs) as b:
        V, E, _ = b.info()
        assert V == sum(o.size - 1 for o, _, _ in gs) and E == sum(d.size for _, d, _ in gs)
        for trial in range(3):
            roots = [int(rng.integers(0, o.size - 1)) for o, _, _ in gs]
            outs, ms = b.run(BFS, roots)
            assert ms > 0
            for i, (o, d, w) in enumerate(gs):
                np.testing.assert_array_equal(outs[i], oracle.bfs(o, d, roots[i]), err_msg=f"BFS graph {i}")
            outs, _ = b.run(SSSP, roots)
            for i, (o, d, w) in enumerate(gs):
                np.testing.assert_array_equal(outs[i], oracle.sssp(o, d, w, roots[i]), err_msg=f"SSSP graph {i}")
        assert b.info()[2] in (0, 1, 2, 3)
        outs, _ = b.run(CC)
        for i, (o, d, w) in enumerate(gs):
            np.testing.assert_array_equal(outs[i], oracle.cc(o, d), err_msg=f"CC graph {i}")
        st = b.stats()
        assert st.traversed_edges == E


def test_graph_batch_symmetric_cc_and_device_out(oracle):
    """All-symmetric batch takes the Afforest CC path; results land in a
    device buffer."""
    import torch
    gs = [oracle.rmat_graph(s, 8, seed=60 + s, symmetrise=True) for s in (9, 10, 11, 12)]
    gs.append(oracle.grid_graph(30, 31, seed=1))
    with cg.Batch(gs) as b:
        V = b.info()[0]
        d_out = torch.empty(V, dtype=torch.int32, device="cuda")
        b.run(CC, out=d_out)
        flat = d_out.cpu().numpy().view(np.uint32)
        assert b.stats().cc_path == 0
        for i, (o, d, w) in enumerate(gs):
            np.testing.assert_array_equal(flat[b.bases[i]:b.bases[i + 1]], oracle.cc(o, d))


def test_graph_batch_rejects_bad_graph():
    ok = (np.array([0, 1, 2], np.uint32), np.array([1, 0], np.uint32), None)
    bad_dest = (np.array([0, 1, 2], np.uint32), np.array([1, 2], np.uint32), None)
    bad_off = (np.array([0, 2, 1], np.uint32), np.array([1, 0], np.uint32), None)
    for bad in (bad_dest, bad_off):
        with pytest.raises(cg.CgbError):
            cg.Batch([ok, bad])
    with cg.Batch([ok, ok]) as b:
        with pytest.raises(cg.CgbError):
            b.run(BFS, [0, 2])
