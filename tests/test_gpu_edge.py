"""Edge cases through the C ABI: empty and tiny graphs, unsorted lists (sorted
by the engine as nbrSort_taskSteal does), invariant violations (status codes,
never a fault), hubs that take the split-hub paths, self-loops, reordered
zero-out-degree tails, missing weights, distance overflow, iteration budget."""
import numpy as np
import pytest

import cggraph_b200 as cg
from cggraph_b200 import CgbError
from cggraph_b200 import _lib as L

pytestmark = pytest.mark.gpu

BFS, SSSP, CC, PR = 0, 1, 2, 3
VMAX = 999999999


def csr_from_edges(V, edges, weights=None):
    edges = sorted(set(edges)) if weights is None else edges
    off = np.zeros(V + 1, np.uint32)
    for u, _ in edges:
        off[u + 1] += 1
    off = np.cumsum(off).astype(np.uint32)
    dst = np.array([v for _, v in edges], np.uint32)
    w = None if weights is None else np.array(weights, np.uint32)
    return off, dst, w


def check_all(oracle, off, dst, w, roots, **kw):
    wt = w if w is not None else np.ones(dst.size, np.uint32)
    with cg.Graph.from_csr(off, dst, w, **kw) as g:
        for r in roots:
            np.testing.assert_array_equal(g.run(BFS, r)[0], oracle.bfs(off, dst, r))
            np.testing.assert_array_equal(g.run(SSSP, r)[0], oracle.sssp(off, dst, wt, r))
        np.testing.assert_array_equal(g.run(CC)[0], oracle.cc(off, dst))
        exp = oracle.pagerank(off, dst, 20)
        got = g.run(PR, 20)[0]
        assert np.max(np.abs(got - exp) / exp) <= 1e-6


def test_no_edges(oracle):
    off = np.zeros(6, np.uint32)
    dst = np.zeros(0, np.uint32)
    with cg.Graph.from_csr(off, dst, None) as g:
        assert g.run(BFS, 2)[0].tolist() == [VMAX, VMAX, 0, VMAX, VMAX]
        assert g.run(SSSP, 4)[0].tolist() == [VMAX, VMAX, VMAX, VMAX, 0]
        assert g.run(CC)[0].tolist() == [0, 1, 2, 3, 4]
        np.testing.assert_allclose(g.run(PR, 20)[0], np.full(5, 0.15 / 5), rtol=1e-15)
    with cg.Graph.from_csr(np.zeros(2, np.uint32), dst, None) as g:
        assert g.run(BFS, 0)[0].tolist() == [0]
        assert g.run(CC)[0].tolist() == [0]


def test_unsorted_lists_are_sorted_with_weights(oracle):
    off, dst, w = oracle.rmat_graph(11, 16, seed=8)
    rng = np.random.default_rng(0)
    d2, w2 = dst.copy(), w.copy()
    for v in range(off.size - 1):
        s, e = int(off[v]), int(off[v + 1])
        p = rng.permutation(e - s)
        d2[s:e] = dst[s:e][p]
        w2[s:e] = w[s:e][p]
    with cg.Graph.from_csr(off, d2, w2) as g:
        o3, d3, w3 = g.download()
        np.testing.assert_array_equal(d3, dst)
        np.testing.assert_array_equal(w3, w)
        r = int(np.diff(off.astype(np.int64)).argmax())
        np.testing.assert_array_equal(g.run(SSSP, r)[0], oracle.sssp(off, dst, w, r))


@pytest.mark.parametrize("case", ["dup", "off0", "offV", "nonmono", "idV"])
def test_invalid_csr_is_rejected(case):
    off = np.array([0, 2, 3, 4], np.uint32)
    dst = np.array([1, 2, 0, 1], np.uint32)
    if case == "dup":
        dst = np.array([1, 1, 0, 1], np.uint32)
    elif case == "off0":
        off = np.array([1, 2, 3, 4], np.uint32)
    elif case == "offV":
        off = np.array([0, 2, 3, 3], np.uint32)
    elif case == "nonmono":
        off = np.array([0, 3, 2, 4], np.uint32)
    elif case == "idV":
        dst = np.array([1, 3, 0, 1], np.uint32)
    with pytest.raises(CgbError) as ei:
        cg.Graph.from_csr(off, dst, None, vertexNum=3, edgeNum=4)
    assert ei.value.status == L.EFORMAT


def test_bad_root_and_algorithm():
    off = np.array([0, 1, 1], np.uint32)
    with cg.Graph.from_csr(off, np.array([1], np.uint32), None) as g:
        with pytest.raises(CgbError) as ei:
            g.run(BFS, 2)
        assert ei.value.status == L.EINVAL
        with pytest.raises(CgbError):
            g.run(7, 0)
        assert g.run(BFS, 0)[0].tolist() == [0, 1]  # still usable


def test_hubs_take_split_paths(oracle):
    """A 40000-leaf out-hub (split across CTAs), a 3000-neighbour vertex (CTA
    tier), a 100-neighbour vertex (warp tier) and a 20000-in-edge sink (whole-CTA
    PageRank row)."""
    V = 60000
    edges = [(0, v) for v in range(1, 40001)]
    edges += [(1, v) for v in range(40001, 43001)]
    edges += [(2, v) for v in range(43001, 43101)]
    edges += [(v, 59999) for v in range(20000, 40000)]
    edges += [(59999, 3)]
    off, dst, _ = csr_from_edges(V, edges)
    w = (np.arange(dst.size) % 50 + 1).astype(np.uint32)
    check_all(oracle, off, dst, w, [0, 1, 20001])
    # symmetrised: the hook-and-compress CC path splits the hub's list too
    off, dst, _ = csr_from_edges(V, edges + [(v, u) for u, v in edges])
    w = (np.arange(dst.size) % 50 + 1).astype(np.uint32)
    check_all(oracle, off, dst, w, [0, 59999])


def test_self_loops_and_zero_weights(oracle):
    edges = [(0, 0), (0, 1), (1, 1), (1, 2), (2, 0), (3, 3)]
    off, dst, _ = csr_from_edges(4, edges)
    w = np.array([5, 0, 3, 0, 1, 9], np.uint32)
    check_all(oracle, off, dst, w, [0, 3])


def test_symmetry_check_when_cc_runs_first(oracle):
    """With CC as the first run, symmetry is decided without a transpose: the
    upper-triangle edges sorted by destination against the lower triangle.
    Graphs whose lower and upper counts agree while their edges do not mirror
    must take label propagation (cc_path 1), symmetric ones hooking (0)."""
    # symmetric, with self-loops and an isolated vertex
    sym = [(0, 0), (0, 2), (2, 0), (1, 3), (3, 1), (3, 3), (2, 3), (3, 2)]
    # one lower and one upper edge that are not mirrors: 0 -> 1, 2 -> 0
    skew = [(0, 1), (2, 0)]
    cases = [(5, sym, 0), (3, skew, 1)]
    # a symmetric RMAT graph, then the same with one mirror (v, u), u < v,
    # moved to (v, u') for a u' < v outside v's list: every count is kept
    off, dst, _ = oracle.rmat_graph(10, 8, seed=5, symmetrise=True)
    V = off.size - 1
    edges = [(u, int(dst[e])) for u in range(V) for e in range(int(off[u]), int(off[u + 1]))]
    cases.append((V, edges, 0))
    es = set(edges)
    v = next(x for x in range(V - 1, 0, -1) if any(d < x for (s, d) in edges if s == x))
    u = next(d for (s, d) in edges if s == v and d < v)
    u2 = next(y for y in range(v) if (v, y) not in es)
    moved = sorted((es - {(v, u)}) | {(v, u2)})
    cases.append((V, moved, 1))
    for V, edges, path in cases:
        off, dst, _ = csr_from_edges(V, edges)
        with cg.Graph.from_csr(off, dst, None) as g:
            np.testing.assert_array_equal(g.run(CC)[0], oracle.cc(off, dst))
            assert g.stats().cc_path == path
            assert g.symmetric == (1 if path == 0 else 0)
            r = int(np.argmax(np.diff(off.astype(np.int64))))
            np.testing.assert_array_equal(g.run(BFS, r)[0], oracle.bfs(off, dst, r))


def test_weights_attached_after_create(oracle):
    """cgb_graph_set_weights: unit weights until weights arrive, the given
    weights after, replacements honoured, and an upload from another thread
    while BFS and PageRank run leaves every result unchanged."""
    import threading
    off, dst, w = oracle.rmat_graph(14, 16, seed=12)
    w2 = (w[::-1] % 50 + 1).astype(np.uint32)
    deg = np.diff(off.astype(np.int64))
    r = int(deg.argmax())
    exp_bfs = oracle.bfs(off, dst, r)
    exp_pr = oracle.pagerank(off, dst, 20)
    with cg.Graph.from_csr(off, dst, None) as g:
        np.testing.assert_array_equal(g.run(SSSP, r)[0], exp_bfs)  # no weights yet: unit weights
        g.set_weights(w)
        np.testing.assert_array_equal(g.run(SSSP, r)[0], oracle.sssp(off, dst, w, r))
        g.set_weights(w2)
        np.testing.assert_array_equal(g.run(SSSP, r)[0], oracle.sssp(off, dst, w2, r))
    with cg.Graph.from_csr(off, dst, None) as g:
        err = []

        def upload():
            try:
                g.set_weights(w)
            except Exception as e:  # reported on the main thread
                err.append(e)

        th = threading.Thread(target=upload)
        th.start()
        for _ in range(3):
            np.testing.assert_array_equal(g.run(BFS, r)[0], exp_bfs)
            got = g.run(PR, 20)[0]
            assert np.max(np.abs(got - exp_pr) / exp_pr) <= 1e-6
        th.join()
        assert not err, err
        np.testing.assert_array_equal(g.run(SSSP, r)[0], oracle.sssp(off, dst, w, r))
    # lists that create had to sort: the weights' order is unknown, so refused
    d2 = dst.copy()
    for v in range(off.size - 1):
        d2[off[v]:off[v + 1]] = d2[off[v]:off[v + 1]][::-1]
    with cg.Graph.from_csr(off, d2, None) as g:
        with pytest.raises(CgbError) as ei:
            g.set_weights(w)
        assert ei.value.status == L.EINVAL


def test_edge_list_input(oracle, tmp_path):
    """The reference's other input format: packed (src, dst, weight) records,
    in any order, in memory or as a .bin file.  The CSR built on the device
    equals the oracle's restatement of the reference's reader; self-loops,
    ids >= V and duplicates are CGB_EFORMAT; a trailing partial record is
    ignored, as the reference's reader ignores it."""
    off, dst, w = oracle.rmat_graph(13, 16, seed=9)
    V = off.size - 1
    rec = oracle.csr_to_edge_list(off, dst, w, seed=4)
    o2, d2, w2 = oracle.edge_list_to_csr(rec, V)
    path = tmp_path / "edges.bin"
    rec.tofile(path)
    for make in (lambda: cg.Graph.from_edges(rec, V), lambda: cg.Graph.load_edge_file(str(path), V)):
        with make() as g:
            o3, d3, w3 = g.download()
            np.testing.assert_array_equal(o3, o2)
            np.testing.assert_array_equal(d3, d2)
            np.testing.assert_array_equal(w3, w2)
            r = int(np.diff(off.astype(np.int64)).argmax())
            np.testing.assert_array_equal(g.run(SSSP, r)[0], oracle.sssp(off, dst, w, r))
    with cg.Graph.from_edges(np.zeros((0, 3), np.uint32), 7) as g:
        assert g.run(BFS, 3)[0].tolist() == [VMAX, VMAX, VMAX, 0, VMAX, VMAX, VMAX]
    for bad in ([[5, 5, 1]], [[0, V, 1]], [[1, 2, 3], [1, 2, 4]]):
        with pytest.raises(CgbError) as ei:
            cg.Graph.from_edges(np.array(bad, np.uint32), V)
        assert ei.value.status == L.EFORMAT
    ragged = tmp_path / "ragged.bin"
    rec.tofile(ragged)
    with open(ragged, "ab") as f:
        f.write(b"\1" * 7)
    with cg.Graph.load_edge_file(str(ragged), V) as g:
        o3, d3, w3 = g.download()
        np.testing.assert_array_equal(o3, o2)
        np.testing.assert_array_equal(d3, d2)
        np.testing.assert_array_equal(w3, w2)


def test_edge_list_reference_fixtures():
    """The device edge-list loader on the records of the fixtures the
    reference's own reader (GraphBinReader) produced: the same CSR, and
    CGB_EFORMAT where the reader's assertions stop it."""
    import os

    from conftest import GOLDEN_DIR

    d = os.path.join(GOLDEN_DIR, "edgelist")
    for f in sorted(os.listdir(d)):
        g = dict(np.load(os.path.join(d, f)))
        V = int(g["V"][0])
        if g["rejected"][0]:
            with pytest.raises(CgbError) as ei:
                cg.Graph.from_edges(g["records"], V)
            assert ei.value.status == L.EFORMAT, f
            continue
        with cg.Graph.from_edges(g["records"], V) as h:
            o, dd, w = h.download()
            np.testing.assert_array_equal(o, g["offsets"], err_msg=f)
            np.testing.assert_array_equal(dd, g["dest"], err_msg=f)
            np.testing.assert_array_equal(w, g["weight"], err_msg=f)


def test_neighbour_sort_reference_fixtures():
    """cgb_graph_create on CSRs with shuffled lists gives the lists the
    reference driver's nbrSort_taskSteal makes of them (fixtures made with the
    reference), and CGB_EFORMAT where its strictly-ascending check fails."""
    import os

    from conftest import GOLDEN_DIR

    d = os.path.join(GOLDEN_DIR, "sortnbr")
    for f in sorted(os.listdir(d)):
        g = dict(np.load(os.path.join(d, f)))
        if g["rejected"][0]:
            with pytest.raises(CgbError) as ei:
                cg.Graph.from_csr(g["offsets"], g["dest"], g["weight"])
            assert ei.value.status == L.EFORMAT, f
            continue
        with cg.Graph.from_csr(g["offsets"], g["dest"], g["weight"]) as h:
            o, dd, w = h.download()
            np.testing.assert_array_equal(o, g["sorted_offsets"], err_msg=f)
            np.testing.assert_array_equal(dd, g["sorted_dest"], err_msg=f)
            np.testing.assert_array_equal(w, g["sorted_weight"], err_msg=f)


def test_reorder_degree_orders(oracle):
    """cgb_graph_reorder: IN_DEGREE_DEC and NORMAL_OUTDEGREE_DEC relabel the
    graph exactly as the oracle's restatement of the reference's Reorder
    (CSR, old2new, noZeroOutDegreeNum); BFS, SSSP and CC on the relabelled
    graph from old2new[root] give the original results under old2new
    (rootTranfer), CC matches the oracle on the relabelled graph, and other
    order methods are CGB_EUNSUPPORTED."""
    off, dst, w = oracle.rmat_graph(13, 16, seed=14)
    deg = np.diff(off.astype(np.int64))
    r = int(deg.argmax())
    exp = {BFS: oracle.bfs(off, dst, r), SSSP: oracle.sssp(off, dst, w, r)}
    with cg.Graph.from_csr(off, dst, w) as g:
        for method in (cg.OrderMethod.NORMAL_OUTDEGREE_DEC, cg.OrderMethod.IN_DEGREE_DEC):
            o2, d2, w2, m2, nz2 = oracle.reorder(off, dst, w, int(method))
            h, old2new, nz = g.reorder(method)
            with h:
                np.testing.assert_array_equal(old2new, m2)
                assert nz == nz2
                o3, d3, w3 = h.download()
                np.testing.assert_array_equal(o3, o2)
                np.testing.assert_array_equal(d3, d2)
                np.testing.assert_array_equal(w3, w2)
                for alg in (BFS, SSSP):
                    np.testing.assert_array_equal(h.run(alg, int(old2new[r]))[0][old2new], exp[alg])
                # CC labels are minimum ids (on this directed graph, of the vertices that
                # reach each one), so they depend on the ids: parity on the relabelled graph
                np.testing.assert_array_equal(h.run(CC)[0], oracle.cc(o2, d2))
        for method in (cg.OrderMethod.RCM, cg.OrderMethod.MY_IMAX_BFS_OUT):
            with pytest.raises(CgbError) as ei:
                g.reorder(method)
            assert ei.value.status == L.EUNSUPPORTED


def bfs_order_graphs(oracle):
    """The reference-pinned fixtures, then graphs with long lists (ties among
    many children), many small trees, no edges, and unreached vertices."""
    import os

    from conftest import GOLDEN_DIR

    d = os.path.join(GOLDEN_DIR, "reorder")
    for f in sorted(os.listdir(d)):
        g = np.load(os.path.join(d, f))
        yield f[:-4], g["offsets"], g["dest"], g["weight"]
    yield ("rmat13_s14",) + oracle.rmat_graph(13, 16, seed=14)
    yield ("rmat17_s2",) + oracle.rmat_graph(17, 16, seed=2)
    yield ("rmat12_s3_sym",) + oracle.rmat_graph(12, 8, seed=3, symmetrise=True)
    rng = np.random.default_rng(5)
    V = 5000
    edges = {(int(u), int(v)) for u, v in rng.integers(0, V, (6000, 2)) if u != v}
    off, dst, _ = csr_from_edges(V, sorted(edges))
    yield "sparse_forest", off, dst, rng.integers(1, 64, dst.size).astype(np.uint32)
    yield "no_edges", np.zeros(65, np.uint32), np.zeros(0, np.uint32), np.zeros(0, np.uint32)
    yield ("grid40x50",) + oracle.grid_graph(40, 50)


def test_reorder_bfs_orders(oracle):
    """cgb_graph_reorder for MY_BFS_OUT, MY_BFS_IN, MY_BFS_OUT_IN and
    MY_IMAX_BFS_IN: old2new, the relabelled CSR and noZeroOutDegreeNum equal
    the oracle's restatement of the reference's Reorder (itself pinned to the
    reference on the fixtures); BFS and SSSP on the relabelled graph from
    old2new[root] give the original results under old2new."""
    for name, off, dst, w in bfs_order_graphs(oracle):
        V = off.size - 1
        with cg.Graph.from_csr(off, dst, w) as g:
            for method in oracle.BFS_ORDERS:
                o2, d2, w2, m2, nz2 = oracle.reorder(off, dst, w, method)
                h, old2new, nz = g.reorder(method)
                with h:
                    np.testing.assert_array_equal(old2new, m2, err_msg=f"{name} method {method}")
                    assert nz == nz2, (name, method)
                    o3, d3, w3 = h.download()
                    np.testing.assert_array_equal(o3, o2)
                    np.testing.assert_array_equal(d3, d2)
                    np.testing.assert_array_equal(w3, w2)
                    if method == 16 and dst.size:
                        r = int(np.diff(off.astype(np.int64)).argmax())
                        np.testing.assert_array_equal(h.run(BFS, int(old2new[r]))[0][old2new], oracle.bfs(off, dst, r))
                        np.testing.assert_array_equal(h.run(SSSP, int(old2new[r]))[0][old2new],
                                                      oracle.sssp(off, dst, w, r))


def test_zero_out_degree_tail(oracle):
    """noZeroOutDegreeNum < V (the reordered layout whose last vertices have no
    out-edges, main_partition.hpp:78-103)."""
    rng = np.random.default_rng(1)
    V, nz = 3000, 2000
    edges = set()
    for _ in range(20000):
        u = int(rng.integers(0, nz))
        v = int(rng.integers(0, V))
        if u != v:
            edges.add((u, v))
    off, dst, _ = csr_from_edges(V, sorted(edges))
    w = rng.integers(1, 64, dst.size).astype(np.uint32)
    assert off[nz] == dst.size
    check_all(oracle, off, dst, w, [0, 1999], noZeroOutDegreeNum=nz)
    # edges at or above noZeroOutDegreeNum are refused, as the driver's check refuses them
    with pytest.raises(CgbError) as ei:
        cg.Graph.from_csr(off, dst, w, noZeroOutDegreeNum=1000)
    assert ei.value.status == L.EFORMAT


def test_missing_weights_mean_unit_weights(oracle):
    off, dst, _ = oracle.rmat_graph(11, 8, seed=4)
    with cg.Graph.from_csr(off, dst, None) as g:
        for r in (0, 9):
            np.testing.assert_array_equal(g.run(SSSP, r)[0], oracle.bfs(off, dst, r))


def test_distance_overflow_stays_unreachable(oracle):
    # 0 -> 1 -> 2 -> 3 with weights 4e8: dist(3) = 1.2e9 >= VertexValue_MAX
    off, dst, _ = csr_from_edges(4, [(0, 1), (1, 2), (2, 3)])
    w = np.array([400000000] * 3, np.uint32)
    with cg.Graph.from_csr(off, dst, w) as g:
        got = g.run(SSSP, 0)[0]
    assert got.tolist() == [0, 400000000, 800000000, VMAX]
    np.testing.assert_array_equal(got, oracle.sssp(off, dst, w, 0))


def test_iteration_budget_is_a_status(oracle):
    off, dst, w = oracle.grid_graph(1, 50)  # a path: 49 levels
    with cg.Graph.from_csr(off, dst, w) as g:
        with pytest.raises(CgbError) as ei:
            g.run(BFS, 0, cg.make_options(max_iterations=5))
        assert ei.value.status == L.ETIMEOUT
        np.testing.assert_array_equal(g.run(BFS, 0)[0], oracle.bfs(off, dst, 0))


def test_device_buffers_in_and_out(oracle):
    import torch
    off, dst, w = oracle.rmat_graph(10, 16, seed=5)
    t_off = torch.from_numpy(off.view(np.int32)).cuda()
    t_dst = torch.from_numpy(dst.view(np.int32)).cuda()
    t_w = torch.from_numpy(w.view(np.int32)).cuda()
    with cg.Graph.from_csr(t_off, t_dst, t_w, vertexNum=off.size - 1, edgeNum=dst.size) as g:
        out = torch.empty(off.size - 1, dtype=torch.int32, device="cuda")
        g.run(SSSP, 3, out=out)
        np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), oracle.sssp(off, dst, w, 3))
        pin = torch.empty(off.size - 1, dtype=torch.int32).pin_memory()
        g.run(BFS, 3, out=pin)
        np.testing.assert_array_equal(pin.numpy().view(np.uint32), oracle.bfs(off, dst, 3))


def test_memory_pool_reuse_and_trim(oracle):
    """Graph buffers come from a caching pool: graphs created after others
    are destroyed, and after the pool is trimmed, still compute correctly."""
    from cggraph_b200 import _lib as L
    off, dst, w = oracle.rmat_graph(12, 8, seed=4)
    exp = oracle.bfs(off, dst, 3)
    import ctypes
    reserved, used = ctypes.c_uint64(), ctypes.c_uint64()
    for trim in (False, True, False):
        with cg.Graph.from_csr(off, dst, w) as g:
            np.testing.assert_array_equal(g.run(0, 3)[0], exp)
            L.check(L.lib().cgb_memory_info(0, ctypes.byref(reserved), ctypes.byref(used)))
            assert used.value >= 4 * (off.size + 2 * dst.size) and reserved.value >= used.value
        if trim:
            L.check(L.lib().cgb_memory_trim(0))
    # an explicit reservation holds at least what was asked, and graphs still work
    r0, _ = cg.memory_info()
    cg.memory_reserve(r0 + (256 << 20))
    r1, _ = cg.memory_info()
    assert r1 >= r0 + (256 << 20)
    with cg.Graph.from_csr(off, dst, w) as g:
        np.testing.assert_array_equal(g.run(0, 3)[0], exp)
    cg.memory_trim()


def test_two_level_partition(oracle):
    """cgb_graph_partition equals the restatement of the reference's
    TwoLevelPartition: segment order, edges, buckets, owners and per-GPU
    counts, for room enough and for GPUs that fill up part way, with a
    zero-out-degree tail, for BFS and SSSP."""
    off, dst, w = oracle.rmat_graph(16, 16, seed=9)
    V = off.size - 1
    with cg.Graph.from_csr(off, dst, w) as g0:
        h, old2new, nz = g0.reorder(cg.OrderMethod.NORMAL_OUTDEGREE_DEC)
    o2, d2, w2 = h.download()
    h.close()
    cases = [(off, dst, w, V), (o2, d2, w2, nz)]
    off_g, dst_g, w_g = oracle.grid_graph(100, 130)
    cases.append((off_g, dst_g, w_g, off_g.size - 1))
    for o, d, ww, n in cases:
        Vc = o.size - 1
        base = Vc * 4 + (n + 1) * 4 + (1 << 30)
        with cg.Graph.from_csr(o, d, ww, noZeroOutDegreeNum=n) as g:
            for alg in (BFS, SSSP):
                for mem in ([1 << 40], [1 << 40] * 3, [base + d.size, base + d.size // 3],
                            [base + 2 * d.size, base + d.size, base + 5]):
                    got = g.partition(alg, len(mem), mem)
                    exp = oracle.two_level_partition(o, n, alg, mem)
                    for k in ("segment_num", "bucket_start", "can_hold_all", "reached_bucket"):
                        assert got[k] == exp[k], (k, alg, mem)
                    for k in ("seg_order", "seg_edges", "seg_owner", "device_segments"):
                        np.testing.assert_array_equal(got[k], exp[k], err_msg=f"{k} {alg} {mem}")
            got = g.partition(BFS, 1)  # the device's own memory: everything fits
            assert got["can_hold_all"] and np.all(got["seg_owner"] == 0)


def test_device_barrier_gives_up_and_context_survives(oracle):
    """The device-resident loops' grid barrier waits a bounded number of
    polls.  cgb_check_barrier_timeout runs such a loop in which one CTA never
    arrives: the others give up after the limit, the call reports
    CGB_ETIMEOUT, and a normal run right after still works."""
    import ctypes
    lib = L.lib()
    f = lib.cgb_check_barrier_timeout
    f.argtypes = [ctypes.c_int, ctypes.c_uint32]
    f.restype = ctypes.c_int
    assert f(0, 1 << 12) == L.ETIMEOUT
    assert f(0, 0) == L.EINVAL
    off, dst, w = oracle.rmat_graph(10, 8, seed=3)
    root = int(np.diff(off.astype(np.int64)).argmax())
    with cg.Graph.from_csr(off, dst, w) as g:
        np.testing.assert_array_equal(g.run(BFS, root)[0], oracle.bfs(off, dst, root))
        np.testing.assert_array_equal(g.run(SSSP, root)[0], oracle.sssp(off, dst, w, root))
