"""Oracle bindings (TEST INFRASTRUCTURE ONLY).

Two independent checkers for the engine's results, never used by the engine:

* ``liboracle.so`` -- the serial C restatement in ``cgb_oracle.c`` (queue BFS,
  Dijkstra, reference-semantics CC, union-find WCC, FP64 PageRank) plus the CPU
  twin of the synthetic-graph generators;
* ``_ref/cgref_oracle`` -- the reference's own MULTI_CORE engine
  (Graph_Numa, my_project/CGgraph/GraphNuma.cuh:9-698) built from the reference
  sources by ``build_ref.sh``; it reads the CSR as the three raw files of
  load_binFile (Basic/Other/IO.hpp:44-92).  Its other modes run the
  reference's Reorder, edge-list reader and neighbour sort.

The numpy restatements of preprocessing (edge list, neighbour sort, vertex
orders) are pinned to those modes by fixtures under tests/golden/.  One
restatement is not: ``two_level_partition`` (parity unpinned), since the
reference's partitioner needs GPUs to be constructed.

Only tests/, the smoke check and the benchmark's CPU-baseline leg import this.
"""
from __future__ import annotations

import ctypes
import signal
import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_BIN = os.path.join(HERE, "_ref", "cgref_oracle")
VALUE_MAX = 999999999

_u32p = ctypes.POINTER(ctypes.c_uint32)
_f64p = ctypes.POINTER(ctypes.c_double)


def build(force: bool = False) -> str:
    """Compile cgb_oracle.c into liboracle.so (gcc + OpenMP)."""
    src = os.path.join(HERE, "cgb_oracle.c")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        tmp = LIB_PATH + ".tmp"
        subprocess.check_call(["gcc", "-O2", "-fopenmp", "-shared", "-fPIC", src, "-o", tmp])
        os.replace(tmp, LIB_PATH)
    return LIB_PATH


def build_ref(reference_root: str | None = None) -> str | None:
    """Build the reference CPU engine harness when the reference sources are
    present (build_ref.sh finds them: its argument, else
    $CGGRAPH_REFERENCE_ROOT, else its default location; it keeps any
    prebuilt harness when they are absent)."""
    script = os.path.join(HERE, "build_ref.sh")
    subprocess.check_call(["bash", script] + ([reference_root] if reference_root else []))
    return REF_BIN if os.path.exists(REF_BIN) else None


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.ora_bfs.argtypes = [ctypes.c_uint32, _u32p, _u32p, ctypes.c_uint32, _u32p]
        L.ora_sssp.argtypes = [ctypes.c_uint32, _u32p, _u32p, _u32p, ctypes.c_uint32, _u32p]
        L.ora_cc.argtypes = [ctypes.c_uint32, _u32p, _u32p, _u32p]
        L.ora_wcc_unionfind.argtypes = [ctypes.c_uint32, _u32p, _u32p, _u32p]
        L.ora_pagerank.argtypes = [ctypes.c_uint32, _u32p, _u32p, ctypes.c_uint32, _f64p]
        L.ora_pagerank_pull_omp.argtypes = [ctypes.c_uint32, _u32p, _u32p, _u32p, ctypes.c_uint32,
                                            ctypes.c_int, _f64p]
        L.ora_num_threads.restype = ctypes.c_int
        L.ora_csc.argtypes = [ctypes.c_uint32, _u32p, _u32p, _u32p, _u32p]
        L.ora_csc.restype = ctypes.c_int
        L.ora_rmat_edges.argtypes = [ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64,
                                     ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, _u32p, _u32p]
        L.ora_build_csr.argtypes = [ctypes.c_uint32, ctypes.c_uint64, _u32p, _u32p, ctypes.c_int, _u32p, _u32p]
        L.ora_chunglu_edges.argtypes = [ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint64, _u32p,
                                        _u32p]
        L.ora_chunglu_edges.restype = ctypes.c_int
        L.ora_build_csr.restype = ctypes.c_int64
        L.ora_edge_weights.argtypes = [ctypes.c_uint32, _u32p, _u32p, ctypes.c_uint64, ctypes.c_uint32,
                                       ctypes.c_int, _u32p]
        L.ora_grid_csr.argtypes = [ctypes.c_uint32, ctypes.c_uint32, _u32p, _u32p]
        L.ora_grid_csr.restype = ctypes.c_int64
        L.ora_bfs_order.argtypes = [ctypes.c_uint32, _u32p, _u32p, ctypes.c_int, _u32p]
        L.ora_bfs_order.restype = ctypes.c_int64
        for f in (L.ora_bfs, L.ora_sssp, L.ora_cc, L.ora_wcc_unionfind, L.ora_pagerank, L.ora_pagerank_pull_omp):
            f.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a, t=_u32p):
    return a.ctypes.data_as(t)


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def bfs(off, dst, root):
    off, dst = _u32(off), _u32(dst)
    V = off.size - 1
    out = np.empty(V, np.uint32)
    assert lib().ora_bfs(V, _p(off), _p(dst), root, _p(out)) == 0
    return out


def sssp(off, dst, w, root):
    off, dst, w = _u32(off), _u32(dst), _u32(w)
    V = off.size - 1
    out = np.empty(V, np.uint32)
    assert lib().ora_sssp(V, _p(off), _p(dst), _p(w), root, _p(out)) == 0
    return out


def cc(off, dst):
    off, dst = _u32(off), _u32(dst)
    V = off.size - 1
    out = np.empty(V, np.uint32)
    assert lib().ora_cc(V, _p(off), _p(dst), _p(out)) == 0
    return out


def wcc_unionfind(off, dst):
    off, dst = _u32(off), _u32(dst)
    V = off.size - 1
    out = np.empty(V, np.uint32)
    assert lib().ora_wcc_unionfind(V, _p(off), _p(dst), _p(out)) == 0
    return out


def pagerank(off, dst, iters=20):
    off, dst = _u32(off), _u32(dst)
    V = off.size - 1
    out = np.empty(V, np.float64)
    assert lib().ora_pagerank(V, _p(off), _p(dst), iters, _p(out, _f64p)) == 0
    return out


def csc(off, dst):
    """In-edge CSC (in_off, in_src) with ascending sources, by counting sort."""
    off, dst = _u32(off), _u32(dst)
    V = off.size - 1
    in_off = np.empty(V + 1, np.uint32)
    in_src = np.empty(max(1, dst.size), np.uint32)
    assert lib().ora_csc(V, _p(off), _p(dst), _p(in_off), _p(in_src)) == 0
    return in_off, in_src[:dst.size].copy()


def pagerank_pull_omp(off, in_off, in_src, iters=20, threads=0):
    off, in_off, in_src = _u32(off), _u32(in_off), _u32(in_src)
    V = off.size - 1
    out = np.empty(V, np.float64)
    assert lib().ora_pagerank_pull_omp(V, _p(off), _p(in_off), _p(in_src), iters, threads, _p(out, _f64p)) == 0
    return out


def num_threads() -> int:
    return int(lib().ora_num_threads())


# ------------------------------------------------------------ generator twin
RMAT_ABC = (0.57, 0.19, 0.19)


class EdgeListError(ValueError):
    """A record set the reference's edge-list reader rejects."""


def edge_list_to_csr(records, V):
    """CSR (offsets, dest, weight) from packed (src, dst, weight) uint32
    records, as the reference's reader builds it: self-loops rejected
    (Basic/Graph/graphBinReader.hpp:150), lists grouped by source
    (:159-190), each sorted by destination (sort_nbr, :213-227) and required
    strictly ascending (check_sortNbr, :238-254), offsets from the
    out-degrees (build_csr, :286-322).  numpy, not the engine's method."""
    rec = np.asarray(records, dtype=np.uint32).reshape(-1, 3)
    src, dst, w = rec[:, 0].astype(np.int64), rec[:, 1].astype(np.int64), rec[:, 2]
    if np.any(src == dst):
        raise EdgeListError("self-loop")
    if rec.size and (src.max() >= V or dst.max() >= V):
        raise EdgeListError("id >= V")
    order = np.lexsort((dst, src))
    src, dst, w = src[order], dst[order], w[order]
    if np.any((src[1:] == src[:-1]) & (dst[1:] == dst[:-1])):
        raise EdgeListError("duplicate edge")
    off = np.zeros(V + 1, np.int64)
    np.add.at(off, src + 1, 1)
    return np.cumsum(off).astype(np.uint32), dst.astype(np.uint32), w.astype(np.uint32)


def csr_to_edge_list(off, dst, w, seed=0):
    """Packed (src, dst, weight) records of a CSR, in a seeded random order."""
    off = np.asarray(off, dtype=np.int64)
    src = np.repeat(np.arange(off.size - 1, dtype=np.uint32), np.diff(off))
    rec = np.stack([src, np.asarray(dst, np.uint32), np.asarray(w, np.uint32)], axis=1)
    return rec[np.random.default_rng(seed).permutation(len(rec))].copy()


def reorder(off, dst, w, method):
    """Relabelled CSR of the deterministic degree orders of the reference's
    Reorder: vertices by degree, largest first, ties by ascending id
    (my_project/CGgraph/Reorder.hpp:251-292); method 21 = IN_DEGREE_DEC (in-
    degree, :211-240), 12 = NORMAL_OUTDEGREE_DEC (out-degree: the vertices
    without out-edges last, noZeroOutDegreeNum before them).  Rows list their
    neighbours by new id, weights following.  The BFS-based orders
    (BFS_ORDERS) come from ``bfs_order``.  Returns (off, dst, w, old2new,
    noZeroOutDegreeNum).  numpy, not the engine's method."""
    off = np.asarray(off, dtype=np.int64)
    dst = np.asarray(dst, dtype=np.int64)
    V = off.size - 1
    outdeg = np.diff(off)
    if method in BFS_ORDERS:
        order, nz = bfs_order(off, dst, method)
    else:
        deg = np.bincount(dst, minlength=V) if method == 21 else outdeg
        order = np.lexsort((np.arange(V), -deg))
        nz = V if method == 21 else int(np.count_nonzero(outdeg))
    old2new = np.empty(V, np.int64)
    old2new[order] = np.arange(V)
    src = np.repeat(np.arange(V), outdeg)
    ns, nd = old2new[src], old2new[dst]
    k = np.lexsort((nd, ns))
    noff = np.zeros(V + 1, np.int64)
    np.add.at(noff, ns + 1, 1)
    nw = None if w is None else np.asarray(w, np.uint32)[k]
    return (np.cumsum(noff).astype(np.uint32), nd[k].astype(np.uint32), nw, old2new.astype(np.uint32), nz)


# MY_BFS_OUT, MY_BFS_IN, MY_BFS_OUT_IN, MY_IMAX_BFS_IN
# (OrderMethod, Basic/Graph/basic_struct.hpp:41-76)
BFS_ORDERS = (16, 17, 18, 20)


def bfs_order(off, dst, method):
    """The reference's MY_BFS_* vertex order (my_project/CGgraph/Reorder.hpp:
    294-535) by the serial C restatement: returns (order, number of vertices
    with out-edges); order[i] = old id of new vertex i.  Children of equal
    degree keep their list order (the reference's std::sort does so for
    lists of at most 16 entries)."""
    off, dst = _u32(off), _u32(dst)
    V = off.size - 1
    order = np.empty(V, np.uint32)
    nz = lib().ora_bfs_order(V, _p(off), _p(dst), int(method), _p(order))
    if nz < 0:
        raise ValueError(f"bfs_order: method {method} ({nz})")
    return order, int(nz)


def cap_lists(off, dst, w, k):
    """The CSR keeping the first k entries of every list."""
    off = np.asarray(off, dtype=np.int64)
    V = off.size - 1
    src = np.repeat(np.arange(V), np.diff(off))
    keep = (np.arange(dst.size) - off[src]) < k
    noff = np.zeros(V + 1, np.int64)
    np.add.at(noff, src[keep] + 1, 1)
    return np.cumsum(noff).astype(np.uint32), dst[keep].copy(), w[keep].copy()


def two_level_partition(off, nz, algorithm, device_mem_bytes):
    """The reference's TwoLevelPartition plan (my_project/CGgraph/
    Two-level_partition.cuh), restated line by line in Python: segments of
    1024 vertices over [0, nz) with edges and integer degree edges / vertices
    (get_SegmentInfo, :213-259); sorted by (degree, id) and cut at the first
    degree >= 17, 33 and 257 (partition_buckets, :267-342); dealt bucket by
    bucket to GPU (j + j // n) % n while that GPU's memory, less 4 V +
    4 (nz + 1) bytes and 2^30 reserved, stays above zero after taking 4 bytes
    per edge (8 for SSSP) (partition_GPU, :350-444).  Parity unpinned: the
    reference's partitioner queries and fills the GPUs in its constructor, so
    it does not run without them; this follows its source."""
    off = np.asarray(off, dtype=np.int64)
    V = off.size - 1
    n_dev = len(device_mem_bytes)
    nseg = (nz + 1023) // 1024
    seg = []
    for s in range(nseg):
        b, e = s * 1024, min((s + 1) * 1024, nz)
        m = int(off[e] - off[b])
        seg.append((m // (e - b), s, m))
    seg.sort(key=lambda t: (t[0], t[1]))
    degs = [t[0] for t in seg]
    import bisect
    bucket = [0] + [bisect.bisect_left(degs, x) for x in (17, 33, 257)] + [nseg]
    cap = [int(m) - (V * 4 + (nz + 1) * 4 + (1 << 30)) for m in device_mem_bytes]
    per_edge = 8 if algorithm == 1 else 4
    owner = [-1] * nseg
    count = [0] * n_dev
    all_fit, reached = True, 0
    for b in range(4):
        if not all_fit:
            break
        reached = b
        for j in range(bucket[b + 1] - bucket[b]):
            dev = (j + j // n_dev) % n_dev
            _, sid, m = seg[bucket[b] + j]
            cap[dev] -= m * per_edge
            if cap[dev] <= 0:
                cap[dev] += m * per_edge
                all_fit = False
                break
            owner[sid] = dev
            count[dev] += 1
    edges = [0] * nseg
    for _, sid, m in seg:
        edges[sid] = m
    return {"segment_num": nseg, "bucket_start": bucket, "can_hold_all": all_fit, "reached_bucket": reached,
            "seg_order": np.array([t[1] for t in seg], np.uint32), "seg_edges": np.array(edges, np.uint32),
            "seg_owner": np.array(owner, np.int32), "device_segments": np.array(count, np.uint32)}


def rmat_thresholds(a=0.57, b=0.19, c=0.19):
    """Quadrant thresholds in units of 2^-32 (floor), shared with the engine."""
    t1 = int(a * 2**32)
    t2 = int((a + b) * 2**32)
    t3 = int((a + b + c) * 2**32)
    return t1, t2, t3


def rmat_edges(scale, edge_factor, seed, scramble=True, abc=RMAT_ABC):
    n = edge_factor << scale
    src = np.empty(n, np.uint32)
    dst = np.empty(n, np.uint32)
    t1, t2, t3 = rmat_thresholds(*abc)
    lib().ora_rmat_edges(scale, n, seed, t1, t2, t3, int(scramble), _p(src), _p(dst))
    return src, dst


def build_csr(V, src, dst, symmetrise=False):
    src, dst = _u32(src), _u32(dst)
    off = np.empty(V + 1, np.uint32)
    out = np.empty(max(1, (2 if symmetrise else 1) * src.size), np.uint32)
    E = lib().ora_build_csr(V, src.size, _p(src), _p(dst), int(symmetrise), _p(off), _p(out))
    assert E >= 0
    return off, out[:E].copy()


def edge_weights(off, dst, seed, wmax=64, sym_key=False):
    """Seeded weights in [1, wmax]; None when wmax is 0 (an unweighted graph)."""
    if not wmax:
        return None
    off, dst = _u32(off), _u32(dst)
    w = np.empty(dst.size, np.uint32)
    lib().ora_edge_weights(off.size - 1, _p(off), _p(dst), seed, wmax, int(sym_key), _p(w))
    return w


def rmat_graph(scale, edge_factor=16, seed=1, symmetrise=False, wmax=64, scramble=True):
    """(off, dst, w) of the seeded RMAT graph, exactly as the engine builds it."""
    src, dst = rmat_edges(scale, edge_factor, seed, scramble)
    off, d = build_csr(1 << scale, src, dst, symmetrise)
    w = edge_weights(off, d, seed, wmax, sym_key=symmetrise)
    return off, d, w


def chunglu_graph(V, draws, weight_offset, seed=1, symmetrise=False, wmax=64):
    """(off, dst, w) of the seeded Chung-Lu graph, exactly as the engine
    builds it (cggraph_b200/csrc/gen.cu gen_chunglu)."""
    src = np.empty(draws, np.uint32)
    dst = np.empty(draws, np.uint32)
    assert lib().ora_chunglu_edges(V, draws, weight_offset, seed, _p(src), _p(dst)) == 0
    off, d = build_csr(V, src, dst, symmetrise)
    w = edge_weights(off, d, seed, wmax, sym_key=symmetrise)
    return off, d, w


def grid_graph(rows, cols, seed=1, wmax=1000):
    V = rows * cols
    off = np.empty(V + 1, np.uint32)
    dst = np.empty(max(1, 4 * V), np.uint32)
    E = lib().ora_grid_csr(rows, cols, _p(off), _p(dst))
    dst = dst[:E].copy()
    w = edge_weights(off, dst, seed, wmax, sym_key=True)
    return off, dst, w


# ------------------------------------------------- reference engine runner
def ref_run_files(paths, V, E, alg, roots, runs, threads=0):
    """Like ref_run on CSR files already written (offsets, dest, weight or
    None); returns the harness's JSON (ms, edges, threads)."""
    if not ref_available():
        raise RuntimeError("reference oracle binary not built (oracle/build_ref.sh)")
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "out.bin")
        args = [REF_BIN, str(alg), str(V), str(E), paths[0], paths[1], paths[2] or "-",
                ",".join(str(int(r)) for r in roots), out, str(runs), str(threads)]
        r = subprocess.run(args, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"cgref_oracle failed ({r.returncode}): {r.stderr[-2000:]}")
        line = [l for l in r.stdout.splitlines() if l.startswith("{")][-1]
        return json.loads(line)


def ref_reorder(off, dst, w, method, tmpdir=None):
    """Run the reference's Reorder (my_project/CGgraph/Reorder.hpp:58-241) in
    its toy-graph mode on a CSR.  Returns (order, (off, dst, w)): order[i] =
    old id of new vertex i, and the relabelled CSR the reference builds, each
    list in the old list order with new ids (Reorder.hpp:538-620)."""
    if not ref_available():
        raise RuntimeError("reference oracle binary not built (oracle/build_ref.sh)")
    off, dst = _u32(off), _u32(dst)
    V, E = off.size - 1, dst.size
    with tempfile.TemporaryDirectory(dir=tmpdir) as d:
        paths = [os.path.join(d, n) for n in ("off.bin", "dst.bin", "w.bin")]
        off.tofile(paths[0])
        dst.tofile(paths[1])
        if w is not None:
            _u32(w).tofile(paths[2])
        args = [REF_BIN, "reorder", str(int(method)), str(V), str(E), paths[0], paths[1],
                paths[2] if w is not None else "-"]
        r = subprocess.run(args, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"cgref_oracle reorder failed ({r.returncode}): {r.stderr[-2000:]}")
    lines = {}
    for l in r.stdout.splitlines():
        for key in ("old:", "csr_offset:", "csr_dest:", "csr_weight:"):
            if l.startswith(key):
                lines[key] = np.array(l[len(key):].split(), dtype=np.uint64).astype(np.uint32)
    return lines["old:"], (lines["csr_offset:"], lines["csr_dest:"], lines["csr_weight:"])


def ref_edge_list(records, V, tmpdir=None):
    """Run the reference's edge-list reader (GraphBinReader,
    Basic/Graph/graphBinReader.hpp:89-325) on packed (src, dst, weight)
    records.  Returns (off, dst, w), or None when the reader rejects the
    input: a self-loop fails its assert_msg (exit status 1,
    graphBinReader.hpp:160), a duplicate edge its assert on strictly
    ascending lists (SIGABRT, :272).  Ids >= V are outside what the reader
    checks; they are not passed."""
    if not ref_available():
        raise RuntimeError("reference oracle binary not built (oracle/build_ref.sh)")
    rec = np.ascontiguousarray(records, dtype=np.uint32).reshape(-1, 3)
    if rec.size and int(rec[:, :2].max()) >= V:
        raise ValueError("ids >= V are not passed to the reference reader")
    with tempfile.TemporaryDirectory(dir=tmpdir) as d:
        path = os.path.join(d, "edges.bin")
        rec.tofile(path)
        r = subprocess.run([REF_BIN, "edges", str(int(V)), path], capture_output=True, text=True)
    if r.returncode in (1, -signal.SIGABRT):
        return None
    if r.returncode != 0:
        raise RuntimeError(f"cgref_oracle edges failed ({r.returncode}): {r.stderr[-2000:]}")
    lines = {}
    for l in r.stdout.splitlines():
        for key in ("csr_offset:", "csr_dest:", "csr_weight:"):
            if l.startswith(key):
                lines[key] = np.array(l[len(key):].split(), dtype=np.uint64).astype(np.uint32)
    return lines["csr_offset:"], lines["csr_dest:"], lines["csr_weight:"]


def _csr_lines(stdout, keys=("csr_offset:", "csr_dest:", "csr_weight:")):
    lines = {}
    for l in stdout.splitlines():
        for key in keys:
            if l.startswith(key):
                lines[key] = np.array(l[len(key):].split(), dtype=np.uint64).astype(np.uint32)
    return [lines[k] for k in keys]


def ref_sort_neighbours(off, dst, w, tmpdir=None):
    """Run the reference's nbrSort_taskSteal (my_project/CGgraph/sortNbr.hpp:
    8-99) on a CSR.  Returns the sorted (off, dst, w), or None when its
    strictly-ascending check fails (a repeated destination; exit status 1)."""
    if not ref_available():
        raise RuntimeError("reference oracle binary not built (oracle/build_ref.sh)")
    off, dst, w = _u32(off), _u32(dst), _u32(w)
    with tempfile.TemporaryDirectory(dir=tmpdir) as d:
        paths = [os.path.join(d, n) for n in ("off.bin", "dst.bin", "w.bin")]
        for a, pth in zip((off, dst, w), paths):
            a.tofile(pth)
        r = subprocess.run([REF_BIN, "sortnbr", str(off.size - 1), str(dst.size)] + paths,
                           capture_output=True, text=True)
    if r.returncode == 1:
        return None
    if r.returncode != 0:
        raise RuntimeError(f"cgref_oracle sortnbr failed ({r.returncode}): {r.stderr[-2000:]}")
    return tuple(_csr_lines(r.stdout))


def sort_neighbours(off, dst, w):
    """Every list sorted by destination, weights following, as the reference
    driver's nbrSort_taskSteal does (my_project/CGgraph/sortNbr.hpp:8-99);
    a repeated destination in a list raises EdgeListError (its assert_msg,
    :88-93).  numpy, not the engine's method."""
    off = np.asarray(off, dtype=np.int64)
    dst = np.asarray(dst, dtype=np.uint32)
    src = np.repeat(np.arange(off.size - 1), np.diff(off))
    k = np.lexsort((dst, src))
    d2 = dst[k]
    if np.any((src[1:] == src[:-1]) & (d2[1:] == d2[:-1])):
        raise EdgeListError("repeated destination in a list")
    return off.astype(np.uint32), d2, np.asarray(w, np.uint32)[k]


def ref_available() -> bool:
    return os.path.exists(REF_BIN)


def ref_run(off, dst, w, alg, root=0, runs=1, threads=0, tmpdir=None, info_out=None):
    """Run the reference's Graph_Numa (alg 0=BFS, 1=SSSP, 2=CC) on a CSR.

    `root` may be a list (run i uses root i mod len).  Returns (values
    uint32[V] of the last run, list of per-run ms as measured by the
    reference's own timer, threads used); `info_out` (a dict) also receives
    the per-run traversed-edge counts."""
    if not ref_available():
        raise RuntimeError("reference oracle binary not built (oracle/build_ref.sh)")
    off, dst = _u32(off), _u32(dst)
    V, E = off.size - 1, dst.size
    with tempfile.TemporaryDirectory(dir=tmpdir) as d:
        paths = [os.path.join(d, n) for n in ("off.bin", "dst.bin", "w.bin", "out.bin")]
        off.tofile(paths[0])
        dst.tofile(paths[1])
        if w is not None:
            _u32(w).tofile(paths[2])
        roots = ",".join(str(int(r)) for r in (root if isinstance(root, (list, tuple)) else [root]))
        args = [REF_BIN, str(alg), str(V), str(E), paths[0], paths[1], paths[2] if w is not None else "-",
                roots, paths[3], str(runs), str(threads)]
        r = subprocess.run(args, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"cgref_oracle failed ({r.returncode}): {r.stderr[-2000:]}")
        line = [l for l in r.stdout.splitlines() if l.startswith("{")][-1]
        info = json.loads(line)
        vals = np.fromfile(paths[3], np.uint32)
        if info_out is not None:
            info_out.update(info)
    return vals, info["ms"], info["threads"]
