"""The oracle (serial C restatement) pinned against the reference's own
engine: the toy known answers and the golden fixtures that
tests/golden/make_golden.py produced with Graph_Numa."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, GOLDEN_DIR, load_golden

VMAX = 999999999


def test_toy0_known_answers(oracle):
    g = load_golden("toy_0")
    off, dst, w = g["offsets"], g["dest"], g["weight"]
    assert oracle.bfs(off, dst, 0).tolist() == [0, 1, 4, 1, 4, 2, 2, 1, 3, 2, VMAX, 3]
    assert oracle.sssp(off, dst, w, 0).tolist() == [0, 1, 19, 3, 21, 6, 9, 7, 17, 10, VMAX, 17]
    assert oracle.cc(off, dst).tolist() == [0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 10, 0]


@pytest.mark.parametrize("name", GOLDEN)
def test_oracle_matches_reference_golden(oracle, name):
    g = load_golden(name)
    off, dst, w = g["offsets"], g["dest"], g["weight"]
    for r in g["roots"].tolist():
        np.testing.assert_array_equal(oracle.bfs(off, dst, r), g[f"bfs_{r}"])
        np.testing.assert_array_equal(oracle.sssp(off, dst, w, r), g[f"sssp_{r}"])
    np.testing.assert_array_equal(oracle.cc(off, dst), g["cc"])


def test_unionfind_equals_labelprop_on_symmetric(oracle):
    g = load_golden("rmat10_s11_sym")
    a = oracle.cc(g["offsets"], g["dest"])
    b = oracle.wcc_unionfind(g["offsets"], g["dest"])
    np.testing.assert_array_equal(a, b)


def test_pagerank_push_equals_pull(oracle):
    g = load_golden("rmat10_s7")
    off, dst = g["offsets"], g["dest"]
    p1 = oracle.pagerank(off, dst, 20)
    io, isrc = oracle.csc(off, dst)
    p2 = oracle.pagerank_pull_omp(off, io, isrc, 20, threads=2)
    assert np.max(np.abs(p1 - p2) / p1) < 1e-12
    # one more hand-checked property: with no in-edges pr = 0.15/N
    indeg = np.bincount(dst, minlength=off.size - 1)
    N = off.size - 1
    assert np.allclose(p1[indeg == 0], 0.15 / N)


def test_pagerank_tiny_by_hand(oracle):
    # 0 -> 1, 1 -> 0, 1 -> 2 ; N = 3
    off = np.array([0, 1, 3, 3], np.uint32)
    dst = np.array([1, 0, 2], np.uint32)
    pr = np.full(3, 1 / 3)
    for _ in range(5):
        new = np.full(3, 0.15 / 3)
        new[1] += 0.85 * pr[0]
        new[0] += 0.85 * pr[1] / 2
        new[2] += 0.85 * pr[1] / 2
        pr = new
    np.testing.assert_allclose(oracle.pagerank(off, dst, 5), pr, rtol=1e-15)


def test_reference_live_on_new_seed(oracle):
    """The reference engine itself, run here on a graph no fixture holds."""
    if not oracle.ref_available():
        pytest.skip("reference oracle binary not built (needs the reference sources)")
    off, dst, w = oracle.rmat_graph(12, 8, seed=123)
    root = int(np.diff(off.astype(np.int64)).argmax())
    for alg, mine in ((0, oracle.bfs(off, dst, root)), (1, oracle.sssp(off, dst, w, root)), (2, oracle.cc(off, dst))):
        ref, ms, threads = oracle.ref_run(off, dst, w, alg, root, threads=2)
        np.testing.assert_array_equal(mine, ref)


def test_generator_twin_properties(oracle):
    for sym in (False, True):
        off, dst, w = oracle.rmat_graph(11, 16, seed=5, symmetrise=sym)
        V = off.size - 1
        assert off[0] == 0 and off[-1] == dst.size and np.all(np.diff(off.astype(np.int64)) >= 0)
        src = np.repeat(np.arange(V), np.diff(off.astype(np.int64)))
        assert np.all(src != dst), "self-loop"
        key = src.astype(np.int64) * V + dst
        assert np.all(np.diff(key) > 0), "not sorted / duplicate"
        assert w.min() >= 1 and w.max() <= 64
        if sym:
            rk = dst.astype(np.int64) * V + src
            order = np.argsort(rk)
            np.testing.assert_array_equal(rk[order], key)
            np.testing.assert_array_equal(w[order], w)
    off, dst, w = oracle.grid_graph(5, 7)
    assert off.size == 36 and dst.size == 2 * (5 * 6 + 4 * 7)


def test_chunglu_twin_properties(oracle):
    """The CPU twin of the Chung-Lu generator: deterministic for a seed,
    sorted self-loop-free lists, and a largest degree near the expected
    draws / (i0 ln((V + i0) / i0))."""
    import math
    V, n, i0 = 20011, 300000, 5
    off, dst, w = oracle.chunglu_graph(V, n, i0, seed=7)
    off2, dst2, w2 = oracle.chunglu_graph(V, n, i0, seed=7)
    assert np.array_equal(off, off2) and np.array_equal(dst, dst2) and np.array_equal(w, w2)
    deg = np.diff(off.astype(np.int64))
    src = np.repeat(np.arange(V), deg)
    assert (src != dst).all()
    key = src * V + dst
    assert (np.diff(key) > 0).all()
    expect = n / (i0 * math.log((V + i0) / i0))
    assert expect / 4 < deg.max() < expect * 1.5  # duplicates to in-hubs are removed
    assert w.min() >= 1 and w.max() <= 64
    offs, dsts, _ = oracle.chunglu_graph(V, n, i0, seed=7, symmetrise=True)
    assert dsts.size >= dst.size


def test_edge_list_oracle_round_trip(oracle):
    """The edge-list reader restatement: a CSR turned into shuffled records
    comes back unchanged; self-loops, ids >= V and duplicates are rejected."""
    off, dst, w = oracle.rmat_graph(10, 8, seed=3)
    rec = oracle.csr_to_edge_list(off, dst, w, seed=1)
    o2, d2, w2 = oracle.edge_list_to_csr(rec, off.size - 1)
    np.testing.assert_array_equal(o2, off)
    np.testing.assert_array_equal(d2, dst)
    np.testing.assert_array_equal(w2, w)
    V = off.size - 1
    for bad in ([[5, 5, 1]], [[0, V, 1]], [[1, 2, 3], [1, 2, 4]]):
        with pytest.raises(oracle.EdgeListError):
            oracle.edge_list_to_csr(np.array(bad, np.uint32), V)


def test_reorder_oracle_properties(oracle):
    """The degree orders: a permutation, degrees non-increasing along the new
    ids, vertices without out-edges last for NORMAL_OUTDEGREE_DEC, and the
    relabelled graph is the old one with its ids mapped."""
    off, dst, w = oracle.rmat_graph(10, 8, seed=6)
    V = off.size - 1
    for method in (12, 21):
        o2, d2, w2, old2new, nz = oracle.reorder(off, dst, w, method)
        assert sorted(old2new.tolist()) == list(range(V))
        deg = np.bincount(dst, minlength=V) if method == 21 else np.diff(off.astype(np.int64))
        new_deg = np.empty(V, np.int64)
        new_deg[old2new] = deg
        assert np.all(np.diff(new_deg) <= 0)
        if method == 12:
            assert nz == np.count_nonzero(deg) and np.all(np.diff(o2.astype(np.int64))[nz:] == 0)
        src = np.repeat(np.arange(V), np.diff(off.astype(np.int64)))
        old = sorted(zip(old2new[src].tolist(), old2new[dst].tolist(), w.tolist()))
        s2 = np.repeat(np.arange(V), np.diff(o2.astype(np.int64)))
        assert old == sorted(zip(s2.tolist(), d2.tolist(), w2.tolist()))


REORDER_DIR = os.path.join(GOLDEN_DIR, "reorder")
REORDER_GOLDEN = sorted(f[:-4] for f in os.listdir(REORDER_DIR) if f.endswith(".npz"))


def sort_rows(off, dst, w):
    """Every list sorted by destination, weights following."""
    off = off.astype(np.int64)
    src = np.repeat(np.arange(off.size - 1), np.diff(off))
    k = np.lexsort((dst, src))
    return dst[k], w[k]


@pytest.mark.parametrize("name", REORDER_GOLDEN)
def test_bfs_order_oracle_matches_reference_golden(oracle, name):
    """The BFS-based orders and IN_DEGREE_DEC of the reference's Reorder
    (fixtures made by tests/golden/make_golden.py with the reference itself):
    the oracle's order is the reference's, and its relabelled CSR is the
    reference's with every list sorted by new id."""
    g = dict(np.load(os.path.join(REORDER_DIR, name + ".npz")))
    off, dst, w = g["offsets"], g["dest"], g["weight"]
    nz_ref = int(np.count_nonzero(np.diff(off.astype(np.int64))))
    for m in oracle.BFS_ORDERS:
        order, nz = oracle.bfs_order(off, dst, m)
        np.testing.assert_array_equal(order, g[f"order_{m}"], err_msg=f"method {m}")
        assert nz == nz_ref
    _, _, _, old2new_in, _ = oracle.reorder(off, dst, w, 21)  # IN_DEGREE_DEC
    np.testing.assert_array_equal(np.argsort(old2new_in), g["order_21"])
    o2, d2, w2, old2new, nz = oracle.reorder(off, dst, w, 16)
    np.testing.assert_array_equal(o2, g["csr_offset_16"])
    rd, rw = sort_rows(g["csr_offset_16"], g["csr_dest_16"], g["csr_weight_16"])
    np.testing.assert_array_equal(d2, rd)
    np.testing.assert_array_equal(w2, rw)
    np.testing.assert_array_equal(old2new[g["order_16"]], np.arange(off.size - 1))


def test_bfs_order_reference_live(oracle):
    """The reference's Reorder itself on graphs no fixture holds: the same
    IN_DEGREE_DEC order, and the same BFS orders on lists of at most 16
    entries."""
    if not oracle.ref_available():
        pytest.skip("reference oracle binary not built (needs the reference sources)")
    off, dst, w = oracle.rmat_graph(11, 16, seed=23)  # IN_DEGREE_DEC: a total order, any list length
    ref, _ = oracle.ref_reorder(off, dst, w, 21)
    np.testing.assert_array_equal(np.argsort(oracle.reorder(off, dst, w, 21)[3]), ref)
    for seed in (21, 22):
        off, dst, w = oracle.cap_lists(*oracle.rmat_graph(11, 8, seed=seed), 16)
        for m in oracle.BFS_ORDERS:
            ref, _ = oracle.ref_reorder(off, dst, w, m)
            np.testing.assert_array_equal(oracle.bfs_order(off, dst, m)[0], ref)


def test_bfs_order_oracle_properties(oracle):
    """On lists of any length: a permutation with the vertices with out-edges
    first; trees rooted in start-list order; every other vertex with
    out-edges after its parent (the first-placed vertex listing it), parents
    in queue order and each parent's children by degree, largest first."""
    off, dst, w = oracle.rmat_graph(11, 16, seed=8)
    V = off.size - 1
    outdeg = np.diff(off.astype(np.int64))
    indeg = np.bincount(dst, minlength=V)
    src = np.repeat(np.arange(V), outdeg)
    for m in oracle.BFS_ORDERS:
        order, nz = oracle.bfs_order(off, dst, m)
        assert sorted(order.tolist()) == list(range(V))
        assert nz == np.count_nonzero(outdeg)
        assert np.all(outdeg[order[:nz]] > 0) and np.all(outdeg[order[nz:]] == 0)
        pos = np.empty(V, np.int64)
        pos[order] = np.arange(V)
        first_in = np.full(V, V, np.int64)
        np.minimum.at(first_in, dst, pos[src])
        v = order[:nz]
        parent = first_in[v]
        root = parent > np.arange(nz)
        start_deg = indeg if m == 20 else outdeg
        rk = np.lexsort((np.arange(V), -start_deg))
        rank = np.empty(V, np.int64)
        rank[rk] = np.arange(V)
        assert np.all(np.diff(rank[v[root]]) > 0)
        pp = parent[~root]
        assert np.all(np.diff(pp) >= 0)
        child_deg = {16: outdeg, 18: outdeg + indeg}.get(m, indeg)[v[~root]]
        same = np.diff(pp) == 0
        assert np.all(np.diff(child_deg)[same] <= 0)


EDGELIST_DIR = os.path.join(GOLDEN_DIR, "edgelist")
EDGELIST_GOLDEN = sorted(f[:-4] for f in os.listdir(EDGELIST_DIR) if f.endswith(".npz"))


@pytest.mark.parametrize("name", EDGELIST_GOLDEN)
def test_edge_list_oracle_matches_reference_golden(oracle, name):
    """The edge-list restatement against the reference's own reader
    (fixtures made by tests/golden/make_golden.py with GraphBinReader): the
    same CSR, and a rejection exactly where the reader's assertions stop it."""
    g = dict(np.load(os.path.join(EDGELIST_DIR, name + ".npz")))
    V = int(g["V"][0])
    if g["rejected"][0]:
        with pytest.raises(oracle.EdgeListError):
            oracle.edge_list_to_csr(g["records"], V)
        return
    off, dst, w = oracle.edge_list_to_csr(g["records"], V)
    np.testing.assert_array_equal(off, g["offsets"])
    np.testing.assert_array_equal(dst, g["dest"])
    np.testing.assert_array_equal(w, g["weight"])


def test_edge_list_reference_live(oracle):
    """The reference's reader itself on records no fixture holds."""
    if not oracle.ref_available():
        pytest.skip("reference oracle binary not built (needs the reference sources)")
    off, dst, w = oracle.rmat_graph(11, 8, seed=31)
    rec = oracle.csr_to_edge_list(off, dst, w, seed=5)
    ref = oracle.ref_edge_list(rec, off.size - 1)
    for a, b in zip(oracle.edge_list_to_csr(rec, off.size - 1), ref):
        np.testing.assert_array_equal(a, b)


SORTNBR_DIR = os.path.join(GOLDEN_DIR, "sortnbr")
SORTNBR_GOLDEN = sorted(f[:-4] for f in os.listdir(SORTNBR_DIR) if f.endswith(".npz"))


@pytest.mark.parametrize("name", SORTNBR_GOLDEN)
def test_neighbour_sort_oracle_matches_reference_golden(oracle, name):
    """The neighbour-sort restatement against the reference driver's
    nbrSort_taskSteal (fixtures made with the reference itself): the same
    sorted CSR, and a rejection where its check stops it."""
    g = dict(np.load(os.path.join(SORTNBR_DIR, name + ".npz")))
    if g["rejected"][0]:
        with pytest.raises(oracle.EdgeListError):
            oracle.sort_neighbours(g["offsets"], g["dest"], g["weight"])
        return
    for a, b in zip(oracle.sort_neighbours(g["offsets"], g["dest"], g["weight"]),
                    (g["sorted_offsets"], g["sorted_dest"], g["sorted_weight"])):
        np.testing.assert_array_equal(a, b)


def test_two_level_partition_oracle_by_hand(oracle):
    """The partition restatement on a graph worked by hand: 3 segments over
    nz = 2100 vertices of degrees 1, 40 and 300 (segment 2 has 52 vertices),
    two GPUs with room for exactly the first two segments' edges."""
    V, nz = 2200, 2100
    deg = np.zeros(V, np.int64)
    deg[0:1024] = 1
    deg[1024:2048] = 40
    deg[2048:2100] = 300
    off = np.concatenate([[0], np.cumsum(deg)])
    r = oracle.two_level_partition(off, nz, 0, [1 << 40, 1 << 40])
    assert r["segment_num"] == 3 and r["bucket_start"] == [0, 1, 1, 2, 3]
    assert r["seg_order"].tolist() == [0, 1, 2] and r["seg_edges"].tolist() == [1024, 40960, 15600]
    # bucket 0: j = 0 -> GPU 0; bucket 2: j = 0 -> GPU 0; bucket 3: j = 0 -> GPU 0
    assert r["seg_owner"].tolist() == [0, 0, 0] and r["can_hold_all"] and r["reached_bucket"] == 3
    base = V * 4 + (nz + 1) * 4 + (1 << 30)
    r = oracle.two_level_partition(off, nz, 0, [base + 4 * (1024 + 40960) + 1, base])
    assert r["seg_owner"].tolist() == [0, 0, -1] and not r["can_hold_all"] and r["reached_bucket"] == 3
    r = oracle.two_level_partition(off, nz, 1, [base + 4 * (1024 + 40960) + 1, base])  # SSSP: 8 bytes per edge
    assert r["seg_owner"].tolist() == [0, -1, -1] and r["reached_bucket"] == 2
    assert r["device_segments"].tolist() == [1, 0]


def test_two_level_partition_oracle_round_robin(oracle):
    """With room for everything, each bucket is dealt as (j + j // n) % n."""
    off, dst, w = oracle.rmat_graph(14, 16, seed=2)
    V = off.size - 1
    r = oracle.two_level_partition(off, V, 0, [1 << 45] * 3)
    assert r["can_hold_all"] and np.all(r["seg_owner"] >= 0)
    for b in range(4):
        ids = r["seg_order"][r["bucket_start"][b]:r["bucket_start"][b + 1]]
        j = np.arange(ids.size)
        np.testing.assert_array_equal(r["seg_owner"][ids], (j + j // 3) % 3)
    assert int(r["seg_edges"].astype(np.int64).sum()) == dst.size


def overflow_graph():
    """Distances that cross VertexValue_MAX: a path of weight 4e8 steps, a
    detour ending exactly below MAX, and an edge of weight 4e9."""
    edges = sorted([(0, 1, 400000000), (1, 2, 400000000), (2, 3, 400000000), (3, 4, 5), (0, 5, 999999998),
                    (5, 4, 1), (0, 4, 4000000000)])
    off = np.zeros(7, np.int64)
    for u, _, _ in edges:
        off[u + 1] += 1
    return (np.cumsum(off).astype(np.uint32), np.array([e[1] for e in edges], np.uint32),
            np.array([e[2] for e in edges], np.uint32))


def test_sssp_overflow_rule_known_answer(oracle):
    """SSSP lowers a distance only below 999999999: vertex 3 (1.2e9 away),
    vertex 4 (999999999 via the detour, 4e9 direct) keep 999999999.  The
    expected values are the reference engine's output on this graph
    (Graph_Numa through the harness), rerun below when it is built."""
    off, dst, w = overflow_graph()
    expect = [0, 400000000, 800000000, VMAX, VMAX, 999999998]
    assert oracle.sssp(off, dst, w, 0).tolist() == expect
    if oracle.ref_available():
        assert oracle.ref_run(off, dst, w, 1, 0)[0].tolist() == expect


def test_toy0_other_roots_known_answers(oracle):
    """toy_0 from a root without out-edges (2), a root no vertex reaches (10)
    and one whose reach is partial (11): the reference engine's BFS and SSSP
    outputs (Graph_Numa through the harness), rerun below when it is built."""
    g = load_golden("toy_0")
    off, dst, w = g["offsets"], g["dest"], g["weight"]
    M = VMAX
    expect = {
        (2, 0): [M, M, 0, M, M, M, M, M, M, M, M, M],
        (2, 1): [M, M, 0, M, M, M, M, M, M, M, M, M],
        (10, 0): [2, 3, 1, 3, 2, 3, 4, 3, 1, 2, 0, 2],
        (10, 1): [8, 9, 2, 11, 12, 14, 17, 15, 8, 17, 0, 19],
        (11, 0): [M, M, 1, M, M, 1, M, 2, M, 2, M, 0],
        (11, 1): [M, M, 2, M, M, 5, M, 12, M, 14, M, 0],
    }
    for (r, alg), e in expect.items():
        got = oracle.bfs(off, dst, r) if alg == 0 else oracle.sssp(off, dst, w, r)
        assert got.tolist() == e, (r, alg)
        if oracle.ref_available():
            assert oracle.ref_run(off, dst, w, alg, r)[0].tolist() == e, (r, alg)
