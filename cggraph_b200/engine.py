"""Host-side mirror of the reference's interface for the SINGLE_GPU path.

Reference (PengBo410/CGgraph, paths under CGgraph/):

* enums ``Algorithm_type``, ``Engine_type``, ``OrderMethod`` and the
  ``CSR_Result_type`` struct -- Basic/Graph/basic_struct.hpp:7-16,41-76,144-178;
* ``load_binFile`` / ``save_binArray`` -- Basic/Other/IO.hpp:44-113;
* ``GraphDeviceWorklist`` (constructor, ``graphProcess_device``,
  ``result_D2H``, ``vertexValue``) -- my_project/CGgraph/GraphDevice.cuh:9-269;
  its replacement here is ``GraphB200``, which runs the sm_100a engine of
  libcgb200.so through the C ABI;
* the SINGLE_GPU branch of ``main_partition()`` (root range check,
  ``rootTranfer`` through ``old2new``, ``runs``, trimmed mean) --
  my_project/CGgraph/main_partition.hpp:319-383,141-144;
* ``checkBinResult`` (exact compare, ``old2new`` remap) -- Basic/Graph/util.cuh:59-118.

Errors are raised as ``CgbError`` carrying the C status code where the
reference aborts (``assert_msg``) or exits (``CUDA_CHECK``).
"""
from __future__ import annotations

import ctypes
import enum
import os
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _lib as L
from ._lib import CgbError, check

VertexValue_MAX = L.VALUE_MAX


class Algorithm_type(enum.IntEnum):
    """Basic/Graph/basic_struct.hpp:144-151."""
    BFS = 0
    SSSP = 1
    CC = 2
    PR = 3
    UNDEFINE = 4


class Engine_type(enum.IntEnum):
    """Basic/Graph/basic_struct.hpp:165-178."""
    COORDINATION = 0
    COOPERATION = 1
    SINGLE_CORE = 2
    MULTI_CORE = 3
    SINGLE_GPU = 4
    BLOCK_2D = 5
    COMPUTE_INDEGREE = 6
    REORDER = 7
    ACTIVEBLOCK = 8


class OrderMethod(enum.IntEnum):
    """Basic/Graph/basic_struct.hpp:41-76."""
    NATIVE = 0
    OUTDEGREE_NODE = 1
    OUTDEGREE_SOCKET = 2
    OUTDEGREE_THREAD = 3
    GORDER = 4
    RCM = 5
    RCM_LAST_ZERO_OUTDEGREE = 6
    RCM_LAST_ONE_ZERO_DEGREE = 7
    OUTDEGREE_NODE_dec = 8
    DEGREE_NODE = 9
    RCM_INDEGREE = 10
    RCM_OUTDEGREE = 11
    NORMAL_OUTDEGREE_DEC = 12
    UnDirected_NATIVE = 13
    UnDirected_RCM = 14
    UnDirected_RCM_LAST_ZERO_OUTDEGREE = 15
    MY_BFS_OUT = 16
    MY_BFS_IN = 17
    MY_BFS_OUT_IN = 18
    MY_IMAX_BFS_OUT = 19
    MY_IMAX_BFS_IN = 20
    IN_DEGREE_DEC = 21


@dataclass
class CSR_Result_type:
    """Basic/Graph/basic_struct.hpp:7-16 (arrays are numpy uint32)."""
    vertexNum: int
    edgeNum: int
    csr_offset: np.ndarray
    csr_dest: np.ndarray
    csr_weight: Optional[np.ndarray]
    noZeroOutDegreeNum: int = 0


def load_binFile(path: str, length: int, dtype=np.uint32) -> np.ndarray:
    """Reads a raw little-endian array of `length` whole elements, requiring
    file bytes // itemsize == length; trailing bytes short of an element are
    ignored (Basic/Other/IO.hpp:44-92, which asserts the same quotient)."""
    if not os.path.exists(path):
        raise CgbError(L.EIO, f"Bin File [{path}] Not Exist")
    itemsize = np.dtype(dtype).itemsize
    if os.path.getsize(path) // itemsize != length:
        raise CgbError(L.EIO, f"(total_bytes / utilSize != length) In Function load_binFile({path})")
    return np.fromfile(path, dtype=dtype, count=length)


def save_binArray(path: str, array) -> None:
    """Basic/Other/IO.hpp:97-113."""
    np.ascontiguousarray(array).tofile(path)


def _ptr(a) -> Optional[int]:
    """Data pointer of a numpy array or a torch tensor (host, pinned or CUDA)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("array must be contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return a.data_ptr()
    raise TypeError(f"unsupported buffer type {type(a)}")


def _u32(a):
    if a is None or not isinstance(a, np.ndarray):
        return a
    return np.ascontiguousarray(a, dtype=np.uint32)


def chunglu_weight_offset(vertices: int, draws: int, max_degree: int) -> int:
    """Weight offset i0 of cgb_gen_chunglu whose top vertex has about
    max_degree distinct out-neighbours.  Its draws D0 = draws * p0 land on
    targets j with probability p_j (p proportional to 1 / (j + i0)), so the
    expected distinct count is sum_j 1 - (1 - p_j)^D0; it falls as i0 grows,
    and i0 is found by bisection."""
    # ranks in geometric bins (p_j varies slowly inside one), the first 4096 one by one
    edges = np.unique(np.concatenate([np.arange(min(4096, vertices)),
                                      np.geomspace(min(4096, vertices), vertices, 4000).astype(np.int64),
                                      [vertices]]))
    mid = (edges[:-1] + edges[1:] - 1) / 2.0
    width = np.diff(edges).astype(np.float64)

    def distinct(i0):
        total = float(np.sum(width / (mid + i0)))  # sum of the weights 1 / (j + i0)
        p = 1.0 / (mid + i0) / total
        d0 = draws * (1.0 / i0) / total
        return float(np.sum(width * -np.expm1(d0 * np.log1p(-p))))

    lo, hi = 1, 4096
    if distinct(lo) <= max_degree:
        return lo
    while hi - lo > 1:
        m = (lo + hi) // 2
        if distinct(m) > max_degree:
            lo = m
        else:
            hi = m
    return lo if abs(distinct(lo) - max_degree) < abs(distinct(hi) - max_degree) else hi


def chunglu_expected_edges(vertices: int, draws: int, weight_offset: int) -> float:
    """Expected distinct edges of cgb_gen_chunglu.  Source and target ranks
    are drawn independently with p_j proportional to 1 / (j + i0), so pair
    (x, y) is present with probability 1 - exp(-draws * p_x * p_y); summed
    over rank bins (the first 4096 ranks one by one, then 1000 geometric
    bins).  Self-loops, which the builder drops, are a negligible share."""
    lead = min(4096, vertices)
    edges = np.unique(np.concatenate([np.arange(lead),
                                      np.geomspace(max(lead, 1), vertices, 1000).astype(np.int64),
                                      [vertices]]))
    mid = (edges[:-1] + edges[1:] - 1) / 2.0
    width = np.diff(edges).astype(np.float64)
    p = 1.0 / (mid + weight_offset)
    p /= float(np.sum(width * p))
    s = 0.0
    for k in range(0, len(p), 1024):
        s += float(np.sum(width[k:k + 1024, None] * width[None, :]
                          * -np.expm1(-float(draws) * p[k:k + 1024, None] * p[None, :])))
    return s


def chunglu_draws_for_edges(vertices: int, edges: int, max_degree: int) -> tuple:
    """(draws, weight offset) of a Chung-Lu graph with about `edges`
    distinct edges whose top vertex has about max_degree out-neighbours:
    bisection on the draw count, the offset re-fitted at each step
    (duplicates grow with the draws, so more draws than edges are needed)."""
    lo, hi = int(edges), int(edges)
    while chunglu_expected_edges(vertices, hi, chunglu_weight_offset(vertices, hi, max_degree)) < edges:
        lo, hi = hi, hi * 2
    while hi - lo > max(1, edges // 2000):
        m = (lo + hi) // 2
        if chunglu_expected_edges(vertices, m, chunglu_weight_offset(vertices, m, max_degree)) < edges:
            lo = m
        else:
            hi = m
    return hi, chunglu_weight_offset(vertices, hi, max_degree)


DEFAULT_TUNING = {"push_big_deg": 512, "push_chunk": 1024, "push_ctas_per_sm": 8, "persist_enter": 1 << 15,
                  "persist_deg": 2048, "ms_edges": 256, "pr_unroll": 16, "pr_ctas_per_sm": 128, "persist_ctas": 0,
                  "sssp_pull_alpha": 0, "cluster_enter": 8192,
                  "sssp_dense_alpha": 4, "push_block": 256}


def _count(a) -> int:
    """Element count of a numpy array or a torch tensor."""
    return int(a.size if isinstance(a, np.ndarray) else a.numel())


def memory_info(device: int = 0):
    """(reserved, used) bytes of the engine's memory pool on `device`."""
    r, u = ctypes.c_uint64(), ctypes.c_uint64()
    check(L.lib().cgb_memory_info(device, ctypes.byref(r), ctypes.byref(u)))
    return r.value, u.value


def memory_reserve(nbytes: int, device: int = 0) -> None:
    """Grow the memory pool to at least `nbytes` reserved (cgb_memory_reserve)."""
    check(L.lib().cgb_memory_reserve(device, int(nbytes)))


def memory_trim(device: int = 0) -> None:
    """Return the pool's cached memory to the driver (cgb_memory_trim)."""
    check(L.lib().cgb_memory_trim(device))


def make_options(schedule: int = L.SCHED_HEURISTIC, variant: int = L.VAR_AUTO, sssp_delta: int = 0,
                 bfs_alpha: float = 0.0, bfs_beta: float = 0.0, max_iterations: int = 0, flags: int = 0) -> L.Options:
    o = L.Options()
    o.struct_size = ctypes.sizeof(L.Options)
    o.schedule = schedule
    o.variant = variant
    o.sssp_delta = sssp_delta
    o.bfs_alpha = bfs_alpha
    o.bfs_beta = bfs_beta
    o.max_iterations = max_iterations
    o.flags = flags
    return o


class Graph:
    """A graph resident in HBM (a ``cgb_graph`` handle)."""

    def __init__(self, handle: int):
        self._h = ctypes.c_void_p(handle)
        V, E, sym = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_int32()
        check(L.lib().cgb_graph_info(self._h, ctypes.byref(V), ctypes.byref(E), ctypes.byref(sym)))
        self.vertexNum = V.value
        self.edgeNum = E.value

    # ---- constructors
    @classmethod
    def from_csr(cls, offsets, dest, weight=None, vertexNum: Optional[int] = None, edgeNum: Optional[int] = None,
                 noZeroOutDegreeNum: int = 0, device: int = 0) -> "Graph":
        offsets, dest, weight = _u32(offsets), _u32(dest), _u32(weight)
        V = vertexNum if vertexNum is not None else len(offsets) - 1
        E = edgeNum if edgeNum is not None else len(dest)
        h = ctypes.c_void_p()
        check(L.lib().cgb_graph_create(_ptr(offsets), _ptr(dest) if E else None, _ptr(weight) if E else None,
                                       V, E, noZeroOutDegreeNum, device, ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def from_result(cls, csr: CSR_Result_type, device: int = 0) -> "Graph":
        return cls.from_csr(csr.csr_offset, csr.csr_dest, csr.csr_weight, csr.vertexNum, csr.edgeNum,
                            csr.noZeroOutDegreeNum, device)

    @classmethod
    def from_files(cls, offsets_path: str, dest_path: str, weight_path: Optional[str], vertexNum: int,
                   edgeNum: int, device: int = 0) -> "Graph":
        h = ctypes.c_void_p()
        enc = lambda p: p.encode() if p is not None else None  # noqa: E731
        check(L.lib().cgb_graph_load_files(enc(offsets_path), enc(dest_path), enc(weight_path), vertexNum, edgeNum,
                                           device, ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def from_edges(cls, records, vertexNum: int, device: int = 0) -> "Graph":
        """Graph from an edge list: packed uint32 (source, destination, weight)
        records, shape (E, 3) or flat, host or device memory
        (cgb_graph_create_from_edges)."""
        records = _u32(records)
        n = records.size // 3 if isinstance(records, np.ndarray) else records.numel() // 3
        h = ctypes.c_void_p()
        check(L.lib().cgb_graph_create_from_edges(_ptr(records) if n else None, n, vertexNum, device,
                                                  ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def load_edge_file(cls, path: str, vertexNum: int, device: int = 0) -> "Graph":
        """Graph from the reference's binary edge-list file: 12-byte records
        (source, destination, weight) (cgb_graph_load_edge_file)."""
        h = ctypes.c_void_p()
        check(L.lib().cgb_graph_load_edge_file(path.encode(), vertexNum, device, ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def rmat(cls, scale: int, edge_factor: int = 16, seed: int = 1, a: float = 0.57, b: float = 0.19,
             c: float = 0.19, scramble: bool = True, symmetrise: bool = False, wmax: int = 64,
             device: int = 0) -> "Graph":
        h = ctypes.c_void_p()
        check(L.lib().cgb_gen_rmat(scale, edge_factor, seed, a, b, c, int(scramble), int(symmetrise), wmax, device,
                                   ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def grid(cls, rows: int, cols: int, seed: int = 1, wmax: int = 1000, device: int = 0) -> "Graph":
        h = ctypes.c_void_p()
        check(L.lib().cgb_gen_grid(rows, cols, seed, wmax, device, ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def chunglu(cls, vertices: int, draws: int, weight_offset: int, seed: int = 1, symmetrise: bool = False,
                wmax: int = 64, device: int = 0) -> "Graph":
        """Seeded Chung-Lu power-law graph (cgb_gen_chunglu)."""
        h = ctypes.c_void_p()
        check(L.lib().cgb_gen_chunglu(vertices, draws, weight_offset, seed, int(symmetrise), wmax, device,
                                      ctypes.byref(h)))
        return cls(h.value)

    # ---- queries
    @property
    def handle(self):
        return self._h

    @property
    def symmetric(self) -> int:
        sym = ctypes.c_int32()
        check(L.lib().cgb_graph_info(self._h, None, None, ctypes.byref(sym)))
        return sym.value

    def set_stream(self, stream) -> None:
        """Run this graph's work on `stream` (a torch.cuda.Stream, a raw
        cudaStream_t as int, or None for the graph's own stream)."""
        ptr = None
        if stream is not None:
            ptr = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
        check(L.lib().cgb_graph_set_stream(self._h, ptr))

    def set_weights(self, weight) -> None:
        """Attach (or replace) the edge weights, E values in CSR order
        (cgb_graph_set_weights); safe to call from another thread while a
        BFS, CC or PageRank run uses the graph; refused while a Server is
        attached to it."""
        weight = _u32(weight)
        check(L.lib().cgb_graph_set_weights(self._h, _ptr(weight)))

    def reorder(self, order_method: int):
        """Relabelled copy in one of the reference's vertex orders
        (cgb_graph_reorder: IN_DEGREE_DEC, NORMAL_OUTDEGREE_DEC, MY_BFS_OUT,
        MY_BFS_IN, MY_BFS_OUT_IN, MY_IMAX_BFS_IN): (graph, old2new uint32[V],
        noZeroOutDegreeNum)."""
        old2new = np.empty(self.vertexNum, np.uint32)
        nz = ctypes.c_uint32()
        h = ctypes.c_void_p()
        check(L.lib().cgb_graph_reorder(self._h, int(order_method), _ptr(old2new), ctypes.byref(nz),
                                        ctypes.byref(h)))
        return Graph(h.value), old2new, nz.value

    def partition(self, algorithm: int, num_devices: int, device_mem_bytes=None) -> dict:
        """The reference's two-level segment partition over GPUs
        (cgb_graph_partition, TwoLevelPartition): segments of 1024 vertices
        sorted by degree into four buckets and dealt to the GPUs while their
        memory holds them.  Returns segment_num, bucket_start, can_hold_all,
        reached_bucket, seg_order, seg_edges, seg_owner (-1 = host) and
        device_segments."""
        info = L.PartitionInfo()
        n = (self.vertexNum + 1023) // 1024  # noZeroOutDegreeNum <= V
        order = np.empty(max(1, n), np.uint32)
        edges = np.empty(max(1, n), np.uint32)
        owner = np.empty(max(1, n), np.int32)
        per_dev = np.empty(num_devices, np.uint32)
        mem = None if device_mem_bytes is None else np.ascontiguousarray(device_mem_bytes, np.uint64)
        check(L.lib().cgb_graph_partition(self._h, int(algorithm), int(num_devices), _ptr(mem), _ptr(order),
                                          _ptr(edges), _ptr(owner), _ptr(per_dev), ctypes.byref(info)))
        n = info.segment_num
        return {"segment_num": n, "bucket_start": list(info.bucket_start), "can_hold_all": bool(info.can_hold_all),
                "reached_bucket": info.reached_bucket, "seg_order": order[:n], "seg_edges": edges[:n],
                "seg_owner": owner[:n], "device_segments": per_dev}

    def download(self, with_weight: bool = True):
        off = np.empty(self.vertexNum + 1, np.uint32)
        dst = np.empty(max(1, self.edgeNum), np.uint32)
        w = np.empty(max(1, self.edgeNum), np.uint32) if with_weight else None
        check(L.lib().cgb_graph_download(self._h, _ptr(off), _ptr(dst), _ptr(w)))
        return off, dst[: self.edgeNum], (w[: self.edgeNum] if w is not None else None)

    def device_csr(self):
        o, d, w = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        check(L.lib().cgb_graph_device_csr(self._h, ctypes.byref(o), ctypes.byref(d), ctypes.byref(w)))
        return o.value, d.value, w.value

    def result_device_ptr(self) -> int:
        p = ctypes.c_void_p()
        check(L.lib().cgb_graph_result_device(self._h, ctypes.byref(p)))
        return p.value

    # ---- runs
    def run(self, algorithm: int, root_or_iters: int = 0, options: Optional[L.Options] = None, out=None,
            to_host: bool = True):
        """One run.  Returns (values, ms).  ``out`` may be a numpy array or a
        torch tensor (host, pinned or CUDA); with ``to_host=False`` and no
        ``out`` the result stays on the device and values is None."""
        alg = int(algorithm)
        if out is None and to_host:
            out = np.empty(self.vertexNum, np.float64 if alg == Algorithm_type.PR else np.uint32)
        ms = ctypes.c_double()
        p = _ptr(out)
        check(L.lib().cgb_run(self._h, alg, int(root_or_iters), ctypes.byref(options) if options else None,
                              p if alg != Algorithm_type.PR else None, p if alg == Algorithm_type.PR else None,
                              ctypes.byref(ms)))
        return out, ms.value

    def run_batch(self, algorithm: int, roots: Sequence[int], options: Optional[L.Options] = None, out=None):
        roots = np.ascontiguousarray(roots, dtype=np.uint32)
        if out is None:
            out = np.empty((len(roots), self.vertexNum), np.uint32)
        ms = ctypes.c_double()
        check(L.lib().cgb_run_batch(self._h, int(algorithm), _ptr(roots), len(roots),
                                    ctypes.byref(options) if options else None, _ptr(out), ctypes.byref(ms)))
        return out, ms.value

    def stats(self) -> L.RunStats:
        s = L.RunStats()
        check(L.lib().cgb_run_stats_get(self._h, ctypes.byref(s)))
        return s

    def get_tuning(self, algorithm: int = 0) -> dict:
        """An algorithm's launch parameters (cgb_tuning; speed only)."""
        t = L.Tuning()
        check(L.lib().cgb_tuning_get(self._h, int(algorithm), ctypes.byref(t)))
        return {f: getattr(t, f) for f in L.TUNING_FIELDS}

    def set_tuning(self, values: dict, algorithm: int = -1) -> None:
        """Changes the given fields of an algorithm's tuning (-1: of every
        algorithm, starting from BFS's)."""
        t = L.Tuning()
        check(L.lib().cgb_tuning_get(self._h, max(0, int(algorithm)), ctypes.byref(t)))
        for k, v in values.items():
            if k not in L.TUNING_FIELDS:
                raise KeyError(k)
            setattr(t, k, int(v))
        t.struct_size = ctypes.sizeof(L.Tuning)
        check(L.lib().cgb_tuning_set(self._h, int(algorithm), ctypes.byref(t)))

    def autotune(self, algorithm: int, roots: Sequence[int], batch: bool = False, keep: bool = True,
                 cc_weak: bool = False):
        """Coordinate-descent search of the launch parameters for `algorithm`
        from `roots` (one run per root, or multi-root passes with batch=True;
        CC as weak components with cc_weak=True).  Returns (best tuning, best
        ms, starting ms); the best tuning stays on the graph unless
        keep=False."""
        r = np.ascontiguousarray(roots, dtype=np.uint32)
        best, bms, sms = L.Tuning(), ctypes.c_double(), ctypes.c_double()
        flags = (L.TUNE_BATCH if batch else 0) | (0 if keep else L.TUNE_KEEP_DEFAULT) | \
            (L.TUNE_CC_WEAK if cc_weak else 0)
        check(L.lib().cgb_autotune(self._h, int(algorithm), _ptr(r), r.size, flags, ctypes.byref(best),
                                   ctypes.byref(bms), ctypes.byref(sms)))
        return {f: getattr(best, f) for f in L.TUNING_FIELDS}, bms.value, sms.value

    def trace(self):
        n = ctypes.c_uint32()
        check(L.lib().cgb_trace_get(self._h, None, 0, ctypes.byref(n)))
        arr = (L.IterTrace * max(1, n.value))()
        check(L.lib().cgb_trace_get(self._h, arr, n.value, ctypes.byref(n)))
        return [arr[i] for i in range(n.value)]

    def close(self) -> None:
        if self._h is not None and self._h.value:
            check(L.lib().cgb_graph_destroy(self._h))
        self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many independent graphs solved together (no counterpart in the
    reference, whose engines take one graph at a time).

    ``Batch(graphs)`` takes a list of ``(offsets, dest, weight)`` CSRs
    (``weight`` may be None) and concatenates them into one disjoint-union
    graph in HBM.  ``run(BFS|SSSP, roots)`` traverses every graph from its own
    root (``roots[i]`` is a local id of graph i) in one cooperative launch,
    captured into a CUDA graph on first use; ``run(CC)`` labels every graph.
    Results come back as a list of per-graph arrays in local ids, equal to
    separate ``Graph.run`` calls.
    """

    def __init__(self, graphs, device: int = 0):
        self._h = ctypes.c_void_p()
        arrs = [(_u32(o), _u32(d), _u32(w)) for o, d, w in graphs]
        n = len(arrs)
        if n == 0:
            raise ValueError("a batch needs at least one graph")
        self._keep = arrs  # the pointer tables reference these
        P = ctypes.c_void_p * n
        offs = P(*[_ptr(o) for o, _, _ in arrs])
        dsts = P(*[_ptr(d) if _count(d) else None for _, d, _ in arrs])
        wts = P(*[_ptr(w) if w is not None and _count(w) else None for _, _, w in arrs])
        self.vertex_counts = np.array([_count(o) - 1 for o, _, _ in arrs], np.uint32)
        self.edge_counts = np.array([_count(d) for _, d, _ in arrs], np.uint32)
        any_w = any(w is not None for _, _, w in arrs)
        check(L.lib().cgb_batch_create(n, offs, dsts, wts if any_w else None, _ptr(self.vertex_counts),
                                       _ptr(self.edge_counts), device, ctypes.byref(self._h)))
        self._keep = None
        self.n = n
        self.bases = np.concatenate([[0], np.cumsum(self.vertex_counts.astype(np.int64))])

    def run(self, algorithm: int, roots: Optional[Sequence[int]] = None, out=None):
        """Returns (list of per-graph results, ms); ``out`` may be a host or
        device buffer of sum(V) uint32 to receive the concatenation instead."""
        r = None if roots is None else np.ascontiguousarray(roots, dtype=np.uint32)
        if r is not None and r.size != self.n:
            raise ValueError("one root per graph")
        flat = np.empty(int(self.bases[-1]), np.uint32) if out is None else out
        ms = ctypes.c_double()
        check(L.lib().cgb_batch_run(self._h, int(algorithm), _ptr(r), _ptr(flat), ctypes.byref(ms)))
        if out is not None:
            return out, ms.value
        return [flat[self.bases[i]:self.bases[i + 1]] for i in range(self.n)], ms.value

    def info(self):
        """(total vertices, total edges, captured-launch bits: 1 BFS, 2 SSSP)."""
        v, e, c = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_int32()
        check(L.lib().cgb_batch_info(self._h, ctypes.byref(v), ctypes.byref(e), ctypes.byref(c)))
        return v.value, e.value, c.value

    def stats(self) -> L.RunStats:
        s = L.RunStats()
        check(L.lib().cgb_batch_stats(self._h, ctypes.byref(s)))
        return s

    def close(self) -> None:
        if self._h is not None and self._h.value:
            check(L.lib().cgb_batch_destroy(self._h))
        self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching request server on one resident graph (no
    counterpart in the reference, whose drivers run one root at a time).

    ``submit(alg, root, arrival_us, out)`` queues a BFS or SSSP query that
    becomes eligible ``arrival_us`` after ``start()``; admitted queries of an
    algorithm share each traversal (up to 64 per algorithm, capped by
    ``memory_budget`` bytes of result regions), and a finished query's slot
    goes to the next arrival.  ``wait()`` blocks until all have ended;
    ``poll()`` returns their records (times in microseconds from start).
    Each result equals ``Graph.run`` of the same query.
    """

    def __init__(self, graph: "Graph", bfs_slots: int = 0, sssp_slots: int = 0, sssp_delta: int = 0,
                 memory_budget: int = 0, flags: int = 0):
        cfg = L.ServerConfig()
        cfg.struct_size = ctypes.sizeof(L.ServerConfig)
        cfg.bfs_slots, cfg.sssp_slots, cfg.sssp_delta = bfs_slots, sssp_slots, sssp_delta
        cfg.memory_budget, cfg.flags = memory_budget, flags
        self._h = ctypes.c_void_p()
        self._graph = graph  # the server borrows the graph
        check(L.lib().cgb_server_create(graph._h, ctypes.byref(cfg), ctypes.byref(self._h)))
        self._outs = {}

    def submit(self, algorithm: int, root: int, arrival_us: float = 0.0, out=None) -> int:
        rid = ctypes.c_uint64()
        check(L.lib().cgb_server_submit(self._h, int(algorithm), int(root), float(arrival_us), _ptr(out),
                                        ctypes.byref(rid)))
        if out is not None:
            self._outs[rid.value] = out
        return rid.value

    def start(self) -> None:
        check(L.lib().cgb_server_start(self._h))

    def wait(self, timeout_ms: float = 600000.0) -> int:
        pending = ctypes.c_uint32()
        check(L.lib().cgb_server_wait(self._h, float(timeout_ms), ctypes.byref(pending)))
        return pending.value

    def poll(self):
        n = ctypes.c_uint32()
        check(L.lib().cgb_server_poll(self._h, None, 0, ctypes.byref(n)))
        arr = (L.RequestInfo * max(1, n.value))()
        check(L.lib().cgb_server_poll(self._h, arr, n.value, ctypes.byref(n)))
        recs = []
        for i in range(n.value):
            r = arr[i]
            recs.append({f: getattr(r, f) for f, _ in L.RequestInfo._fields_})
            self._outs.pop(r.id, None)
        return recs

    def stats(self):
        t, b, s_, busy = ctypes.c_uint64(), ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_double()
        check(L.lib().cgb_server_stats(self._h, ctypes.byref(t), ctypes.byref(b), ctypes.byref(s_),
                                       ctypes.byref(busy)))
        return {"ticks": t.value, "bfs_slots": b.value, "sssp_slots": s_.value, "busy_ms": busy.value}

    def close(self) -> None:
        if self._h is not None and self._h.value:
            check(L.lib().cgb_server_destroy(self._h))
        self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GraphB200:
    """Drop-in for ``GraphDeviceWorklist`` (my_project/CGgraph/GraphDevice.cuh:9-269).

    ``GraphB200(csr_result, algorithm)`` uploads the CSR once (the reference's
    constructor + ``csrToDevice``); ``graphProcess_device(algorithm, root)``
    runs one traversal and returns its device time in ms (for PageRank
    ``root`` is the iteration count, GraphDevice.cuh:159-162);
    ``result_D2H()`` fills ``vertexValue`` (uint32[V], or float64[V] for
    PageRank, which the reference computes in uint32 and so cannot produce).
    """

    def __init__(self, csr_result: CSR_Result_type, algorithm: Algorithm_type, device: int = 0,
                 options: Optional[L.Options] = None):
        self.vertexNum = csr_result.vertexNum
        self.edgeNum = csr_result.edgeNum
        self.noZeroOutDegreeNum = csr_result.noZeroOutDegreeNum or csr_result.vertexNum
        self.zeroOutDegreeNum = self.vertexNum - self.noZeroOutDegreeNum
        self.algorithm = Algorithm_type(algorithm)
        self.options = options
        self.graph = Graph.from_result(csr_result, device)
        self.vertexValue = None
        self._last_alg = None

    def graphProcess_device(self, algorithm: Algorithm_type, root: int = 0) -> float:
        _, ms = self.graph.run(int(algorithm), int(root), self.options, out=None, to_host=False)
        self._last_alg = Algorithm_type(algorithm)
        return ms

    def result_D2H(self) -> None:
        if self._last_alg is None:
            raise CgbError(L.EINVAL, "result_D2H before any graphProcess_device")
        is_pr = self._last_alg == Algorithm_type.PR
        out = np.empty(self.vertexNum, np.float64 if is_pr else np.uint32)
        check(L.lib().cgb_graph_result_download(self.graph.handle, _ptr(out)))
        self.vertexValue = out

    def close(self):
        self.graph.close()


def trimmed_mean_ms(times: Sequence[float]) -> float:
    """main_partition.hpp:347-365: sort, drop min and max when runs > 2."""
    t = sorted(times)
    if len(t) > 2:
        t = t[1:-1]
    return sum(t) / len(t)


def reorder_graph(csr_result: CSR_Result_type, orderMethod: OrderMethod, files: Optional[dict] = None,
                  device: int = 0) -> dict:
    """Reorder::generateReorderGraphFile (my_project/CGgraph/Reorder.hpp:58-241)
    over cgb_graph_reorder: the relabelled CSR (lists sorted by new id), old2new
    and the number of vertices without out-edges.  With ``files`` (keys
    "offsets", "dest", "weight", "old2new", "addition" -> paths) it writes the
    five files saveCSR_reorderFile writes (:538-700): the addition file holds
    that count, and is empty for IN_DEGREE_DEC, whose order keeps no
    zero-out-degree tail."""
    with Graph.from_csr(csr_result.csr_offset, csr_result.csr_dest, csr_result.csr_weight, device=device) as g:
        h, old2new, nz = g.reorder(orderMethod)
        with h:
            off, dst, w = h.download(with_weight=csr_result.csr_weight is not None)
    V = csr_result.vertexNum
    zero = V - nz
    if files:
        save_binArray(files["offsets"], off)
        save_binArray(files["dest"], dst)
        if w is not None:
            save_binArray(files["weight"], w)
        save_binArray(files["old2new"], old2new)
        extra = np.zeros(0, np.uint32) if orderMethod == OrderMethod.IN_DEGREE_DEC else np.array([zero], np.uint32)
        save_binArray(files["addition"], extra)
    csr = CSR_Result_type(V, csr_result.edgeNum, off, dst, w, nz)
    return {"csr": csr, "old2new": old2new, "zeroOutDegreeNum": zero}


def main_partition(csr_result: CSR_Result_type, algorithm: Algorithm_type, root: int = 0, runs: int = 1,
                   engine_type: Engine_type = Engine_type.SINGLE_GPU, orderMethod: OrderMethod = OrderMethod.NATIVE,
                   rootTranfer: bool = True, old2new: Optional[np.ndarray] = None, device: int = 0,
                   options: Optional[L.Options] = None, reorder_files: Optional[dict] = None) -> dict:
    """The SINGLE_GPU branch of main_partition() (main_partition.hpp:319-383).

    Returns {"times": per-run ms, "total_run_time_ms": trimmed mean,
    "vertexValue": result} -- the printed ``[Total Run Time]`` and the array
    the reference then hands to checkBinResult.  A root outside [0, V)
    returns without running, as the reference's ``do { if (root < 0 ||
    root >= vertices) break; ... } while (0)`` does.

    Engine_type.REORDER is the preprocessing branch (:466-487): the graph in
    IN_DEGREE_DEC order, written to ``reorder_files`` when given; it returns
    reorder_graph's result.  Engine_type.COMPUTE_INDEGREE (:459-464) returns
    the degrees and the 100 vertices of largest in-degree."""
    if engine_type == Engine_type.REORDER:
        return reorder_graph(csr_result, OrderMethod.IN_DEGREE_DEC, reorder_files, device)
    if engine_type == Engine_type.COMPUTE_INDEGREE:
        # Compute_indegree (Compute_indegree.cuh:114-195): the degrees, and the
        # 100 vertices of largest in-degree it prints (ties here by id; the
        # reference's std::sort leaves their order open)
        off = np.asarray(csr_result.csr_offset, np.int64)
        outdeg = np.diff(off).astype(np.uint32)
        indeg = np.bincount(np.asarray(csr_result.csr_dest)[: csr_result.edgeNum],
                            minlength=csr_result.vertexNum).astype(np.uint32)
        top = np.lexsort((np.arange(csr_result.vertexNum), -indeg.astype(np.int64)))[:100]
        return {"inDegree": indeg, "outDegree": outdeg, "top": [(int(v), int(indeg[v])) for v in top]}
    if engine_type != Engine_type.SINGLE_GPU:
        raise CgbError(L.EUNSUPPORTED, f"Engine_type {Engine_type(engine_type).name} is not provided by this engine "
                                       "(only the SINGLE_GPU path and the REORDER / COMPUTE_INDEGREE preprocessing are rebuilt)")
    engine = GraphB200(csr_result, algorithm, device=device, options=options)
    try:
        times = []
        if 0 <= root < csr_result.vertexNum:
            switch_root = root
            if orderMethod != OrderMethod.NATIVE and rootTranfer and algorithm != Algorithm_type.PR:
                if old2new is None:
                    raise CgbError(L.EINVAL, "rootTranfer needs old2new")
                switch_root = int(old2new[root])
            for _ in range(runs):
                times.append(engine.graphProcess_device(algorithm, switch_root))
            engine.result_D2H()
        return {"times": times, "total_run_time_ms": trimmed_mean_ms(times) if times else None,
                "vertexValue": engine.vertexValue}
    finally:
        engine.close()


def checkBinResult(golden, current_array: np.ndarray, length: int, orderMethod: OrderMethod = OrderMethod.NATIVE,
                   old2new: Optional[np.ndarray] = None) -> None:
    """Exact element-wise compare (Basic/Graph/util.cuh:59-118); ``golden`` is
    a result-file path or an array.  With a reordered graph the current array
    is indexed through old2new.  Raises AssertionError naming the first
    mismatch, as assert_msg does."""
    ref = load_binFile(golden, length, current_array.dtype) if isinstance(golden, str) else np.asarray(golden)
    cur = np.asarray(current_array)
    if orderMethod == OrderMethod.NATIVE:
        bad = np.nonzero(cur[:length] != ref[:length])[0]
    else:
        bad = np.nonzero(cur[np.asarray(old2new)[:length]] != ref[:length])[0]
    if bad.size:
        i = int(bad[0])
        got = cur[i] if orderMethod == OrderMethod.NATIVE else cur[int(old2new[i])]
        raise AssertionError(f"error: current_array[{i}] = {got}, resultArray[{i}] = {ref[i]}")
