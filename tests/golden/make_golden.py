"""Generates tests/golden/*.npz from the reference's own CPU engine.

Run in a container where the reference is mounted (it builds
oracle/_ref/cgref_oracle from the reference sources with
oracle/build_ref.sh).  Each fixture holds a CSR and the uint32 results the
reference's Graph_Numa engine (my_project/CGgraph/GraphNuma.cuh) produced on
it: BFS and SSSP from a few roots, CC.  The toy graphs are the reference's own
fixtures (Basic/Graph/graphFileList.hpp:514-568); the others are seeded
synthetic graphs built by the oracle's generator twin.

The fixtures under reorder/ hold the vertex orders of the reference's
Reorder (my_project/CGgraph/Reorder.hpp) for its BFS-based methods and
IN_DEGREE_DEC on graphs whose lists have at most 16 entries, where the
reference's child sort is stable and so fully determined (order_<method>,
order[i] = old id of new vertex i), and the relabelled CSR the reference
builds for MY_BFS_OUT (csr_offset_16, csr_dest_16, csr_weight_16; lists in
old list order).

The fixtures under edgelist/ hold packed (src, dst, weight) records and the
CSR the reference's edge-list reader (Basic/Graph/graphBinReader.hpp,
GraphBinReader) builds from them, or rejected = 1 where the reader's
assertions stop it (a self-loop, a duplicate edge).

The fixtures under sortnbr/ hold CSRs with shuffled lists and what the
reference driver's neighbour sort (nbrSort_taskSteal,
my_project/CGgraph/sortNbr.hpp) makes of them, or rejected = 1 where its
strictly-ascending check stops it (a repeated destination).

usage: python tests/golden/make_golden.py [reference root]
                                          [--reorder-only | --edgelist-only | --sortnbr-only]
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

# The reference's toy CSRs (Basic/Graph/graphFileList.hpp:514-568).
TOY = {
    "toy_0": (
        [0, 3, 6, 6, 8, 8, 11, 15, 16, 21, 22, 24, 26],
        [1, 3, 7, 3, 5, 9, 5, 6, 7, 9, 11, 0, 5, 8, 9, 5, 0, 2, 4, 9, 11, 5, 2, 8, 2, 5],
        [1, 3, 7, 3, 5, 9, 5, 6, 7, 9, 11, 0, 5, 8, 9, 5, 0, 2, 4, 9, 11, 5, 2, 8, 2, 5],
    ),
    "toy_1": (
        [0, 3, 6, 6, 8, 8, 11, 16, 17, 21, 24, 26, 28],
        [1, 3, 7, 3, 5, 9, 5, 6, 7, 9, 11, 0, 5, 8, 9, 10, 5, 0, 4, 9, 11, 5, 6, 8, 2, 8, 2, 5],
        [1, 3, 7, 3, 5, 9, 5, 6, 7, 9, 11, 0, 5, 8, 9, 5, 0, 2, 4, 9, 11, 5, 2, 8, 2, 5, 2, 5],
    ),
}


def graphs():
    for name, (off, dst, w) in TOY.items():
        yield name, np.array(off, np.uint32), np.array(dst, np.uint32), np.array(w, np.uint32), [0, 6, 8]
    off, dst, w = O.rmat_graph(10, 16, seed=7)
    deg = np.diff(off.astype(np.int64))
    yield "rmat10_s7", off, dst, w, [int(deg.argmax()), 1, 77]
    off, dst, w = O.rmat_graph(10, 16, seed=11, symmetrise=True)
    deg = np.diff(off.astype(np.int64))
    yield "rmat10_s11_sym", off, dst, w, [int(deg.argmax()), 5]
    off, dst, w = O.grid_graph(16, 24, seed=3)
    yield "grid16x24_s3", off, dst, w, [0, 200]


# MY_BFS_OUT, MY_BFS_IN, MY_BFS_OUT_IN, MY_IMAX_BFS_IN, IN_DEGREE_DEC
REORDER_METHODS = (16, 17, 18, 20, 21)


def reorder_graphs():
    for name, (off, dst, w) in TOY.items():
        yield name, np.array(off, np.uint32), np.array(dst, np.uint32), np.array(w, np.uint32)
    yield ("rmat10_s7_cap16",) + O.cap_lists(*O.rmat_graph(10, 16, seed=7), 16)
    yield ("rmat11_s9_cap16",) + O.cap_lists(*O.rmat_graph(11, 4, seed=9), 16)
    yield ("grid16x24_s3",) + O.grid_graph(16, 24, seed=3)


def make_reorder():
    d = os.path.join(HERE, "reorder")
    os.makedirs(d, exist_ok=True)
    for name, off, dst, w in reorder_graphs():
        assert np.diff(off.astype(np.int64)).max() <= 16
        out = {"offsets": off, "dest": dst, "weight": w}
        for m in REORDER_METHODS:
            order, csr = O.ref_reorder(off, dst, w, m)
            out[f"order_{m}"] = order
            if m == 16:
                out["csr_offset_16"], out["csr_dest_16"], out["csr_weight_16"] = csr
        np.savez_compressed(os.path.join(d, f"{name}.npz"), **out)
        print("reorder", name, off.size - 1, dst.size)


def edge_list_cases():
    off, dst, w = O.rmat_graph(10, 8, seed=3)
    yield "rmat10_s3", O.csr_to_edge_list(off, dst, w, seed=1), off.size - 1
    off, dst, w = O.grid_graph(12, 9, seed=2)
    yield "grid12x9_s2", O.csr_to_edge_list(off, dst, w, seed=2), off.size - 1
    yield "toy0_records", O.csr_to_edge_list(*(np.array(a, np.uint32) for a in TOY["toy_0"]), seed=3), 12
    yield "empty", np.zeros((0, 3), np.uint32), 5
    yield "self_loop", np.array([[0, 1, 4], [2, 2, 1], [1, 0, 3]], np.uint32), 3
    yield "duplicate", np.array([[0, 1, 4], [1, 2, 1], [0, 1, 3]], np.uint32), 3


def make_edge_lists():
    d = os.path.join(HERE, "edgelist")
    os.makedirs(d, exist_ok=True)
    for name, rec, V in edge_list_cases():
        out = {"records": rec, "V": np.array([V], np.uint32)}
        r = O.ref_edge_list(rec, V)
        out["rejected"] = np.array([r is None], np.uint8)
        if r is not None:
            out["offsets"], out["dest"], out["weight"] = r
        np.savez_compressed(os.path.join(d, f"{name}.npz"), **out)
        print("edgelist", name, V, len(rec), "rejected" if r is None else "")


def shuffled_lists(off, dst, w, seed):
    rng = np.random.default_rng(seed)
    d, ww = dst.copy(), w.copy()
    for v in range(off.size - 1):
        a, b = int(off[v]), int(off[v + 1])
        p = rng.permutation(b - a)
        d[a:b], ww[a:b] = d[a:b][p], ww[a:b][p]
    return off, d, ww


def sortnbr_cases():
    yield ("rmat10_s3_shuffled",) + shuffled_lists(*O.rmat_graph(10, 8, seed=3), seed=1)
    yield ("rmat9_s5_sym_shuffled",) + shuffled_lists(*O.rmat_graph(9, 16, seed=5, symmetrise=True), seed=2)
    off, dst, w = O.rmat_graph(9, 8, seed=6)
    v = int(np.argmax(np.diff(off.astype(np.int64)) >= 3))
    d = dst.copy()
    d[off[v] + 1] = d[off[v]]
    yield "repeated_destination", off, d, w


def make_sortnbr():
    d = os.path.join(HERE, "sortnbr")
    os.makedirs(d, exist_ok=True)
    for name, off, dst, w in sortnbr_cases():
        out = {"offsets": off, "dest": dst, "weight": w}
        r = O.ref_sort_neighbours(off, dst, w)
        out["rejected"] = np.array([r is None], np.uint8)
        if r is not None:
            out["sorted_offsets"], out["sorted_dest"], out["sorted_weight"] = r
        np.savez_compressed(os.path.join(d, f"{name}.npz"), **out)
        print("sortnbr", name, off.size - 1, dst.size, "rejected" if r is None else "")


def main():
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    ref_root = args[0] if args else os.environ.get("CGGRAPH_REFERENCE_ROOT", "/root/reference")
    O.build()
    if O.build_ref(ref_root) is None:
        raise SystemExit("reference oracle unavailable")
    only = [a for a in sys.argv if a.endswith("-only")]
    if not only or "--reorder-only" in only:
        make_reorder()
    if not only or "--edgelist-only" in only:
        make_edge_lists()
    if not only or "--sortnbr-only" in only:
        make_sortnbr()
    if only:
        return
    for name, off, dst, w, roots in graphs():
        out = {"offsets": off, "dest": dst, "weight": w, "roots": np.array(roots, np.uint32)}
        for r in roots:
            out[f"bfs_{r}"], _, _ = O.ref_run(off, dst, w, 0, r, threads=2)
            out[f"sssp_{r}"], _, _ = O.ref_run(off, dst, w, 1, r, threads=2)
        out["cc"], _, _ = O.ref_run(off, dst, w, 2, 0, threads=2)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, off.size - 1, dst.size, roots)


if __name__ == "__main__":
    main()
