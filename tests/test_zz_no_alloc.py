"""cgb_bfs_noalloc: BFS for callers that cannot allocate device memory.

Such a caller -- for example a framework whose caching allocator already owns
the device's memory, or a serving loop that forbids cudaMalloc after start-up
-- passes its own device CSR and output buffer; the entry point keeps its
frontier queues and bitmap in a static device array instead of allocating.
These tests call it through the C ABI twice in a row on each graph and check
each result against the allocating entry point (cgb_run, BFS) and the
oracle's queue BFS, bit for bit, and that the second call leaves the device's
free memory unchanged.  The graphs cover the sizes where the scratch layout
matters: the largest accepted vertex count (a 1024 x 1024 grid, exactly
CGB_NOALLOC_MAX_VERTICES vertices), a single vertex, and a root without
out-edges.  Malformed CSRs (an id >= V, decreasing offsets, offsets[V] != E)
must come back as CGB_EFORMAT with nothing written past the caller's level
buffer.  The file runs last so that a failure here never hides the other
tests, and it must pass both alone in a fresh process and after the rest of
the suite.
"""
import ctypes

import numpy as np
import pytest

import cggraph_b200 as cg
from cggraph_b200 import _lib as L

pytestmark = pytest.mark.gpu

MAX_V = 1 << 20  # CGB_NOALLOC_MAX_VERTICES
GUARD = 64       # words after the level buffer that must stay untouched


def _noalloc(lib):
    f = lib.cgb_bfs_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                  ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _graph(name, oracle):
    if name == "rmat16":
        off, dst, w = oracle.rmat_graph(16, 16, seed=77)
        deg = np.diff(off.astype(np.int64))
        return off, dst, w, [int(deg.argmax()), int(np.nonzero(deg)[0][3])]
    if name == "grid1024_maxv":
        off, dst, w = oracle.grid_graph(1024, 1024, seed=5)
        assert off.size - 1 == MAX_V
        return off, dst, w, [0, MAX_V - 1]
    if name == "single_vertex":
        return np.array([0, 0], np.uint32), np.zeros(0, np.uint32), None, [0, 0]
    if name == "root_without_out_edges":
        # 0 -> 1 -> 2, and vertex 3 with in-edges only
        off = np.array([0, 2, 3, 3, 3], np.uint32)
        dst = np.array([1, 3, 2], np.uint32)
        return off, dst, None, [3, 2]
    raise ValueError(name)


def _device(a, torch):
    if a.size == 0:
        return torch.empty(1, dtype=torch.int32, device="cuda")
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


@pytest.mark.parametrize("name", ["rmat16", "grid1024_maxv", "single_vertex", "root_without_out_edges"])
def test_noalloc_bfs_matches_allocating_entry_point(oracle, name):
    import torch
    lib = L.lib()
    bfs_noalloc = _noalloc(lib)
    off, dst, w, roots = _graph(name, oracle)
    V, E = off.size - 1, dst.size
    d_off, d_dst = _device(off, torch), _device(dst, torch)
    # levels followed by a guard region that must stay as it was
    d_lvl = torch.full((V + GUARD,), 0x5A5A5A5A, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    with cg.Graph.from_csr(off, dst, w) as g:
        expected = [g.run(0, r)[0] for r in roots]
    torch.cuda.synchronize()
    free_after_first = None
    for i, r in enumerate(roots):
        np.testing.assert_array_equal(expected[i], oracle.bfs(off, dst, r), err_msg=f"cgb_run vs oracle, root {r}")
        st = bfs_noalloc(d_off.data_ptr(), d_dst.data_ptr(), V, E, r, d_lvl.data_ptr(), stream.cuda_stream)
        assert st == L.OK, lib.cgb_last_error_string()
        torch.cuda.synchronize()
        got = d_lvl.cpu().numpy().view(np.uint32)
        np.testing.assert_array_equal(got[:V], expected[i], err_msg=f"{name}: call {i + 1}, root {r}")
        assert np.all(got[V:] == 0x5A5A5A5A), "written past the level buffer"
        free_now = torch.cuda.mem_get_info()[0]
        if i == 0:
            free_after_first = free_now
        else:
            assert free_now == free_after_first, "the second call changed the device's free memory"


@pytest.mark.parametrize("case", ["dest_id_out_of_range", "offsets_decrease", "offsets_end_not_E",
                                  "offsets_start_not_zero"])
def test_noalloc_rejects_malformed_csr(oracle, case):
    """Each malformed CSR is caught by the entry point's own checks (offsets
    before the BFS starts, ids where they are read) and returns CGB_EFORMAT;
    the level buffer's guard region stays untouched, and a valid call right
    after succeeds."""
    import torch
    lib = L.lib()
    bfs_noalloc = _noalloc(lib)
    off, dst, _ = oracle.rmat_graph(10, 8, seed=3)
    off, dst = off.copy(), dst.copy()
    V, E = off.size - 1, dst.size
    deg = np.diff(off.astype(np.int64))
    root = int(deg.argmax())
    bad_off, bad_dst, bad_E = off.copy(), dst.copy(), E
    if case == "dest_id_out_of_range":
        # an id far past V in the root's own list, so the first level reads it
        bad_dst[off[root]] = V + 12345
    elif case == "offsets_decrease":
        v = int(np.nonzero(deg)[0][5])
        assert off[v] > 0
        bad_off[v + 1] = off[v] - 1  # offsets[v + 1] < offsets[v]
    elif case == "offsets_end_not_E":
        bad_E = E - 1
    elif case == "offsets_start_not_zero":
        bad_off[0] = 1
    d_off, d_dst = _device(bad_off, torch), _device(bad_dst, torch)
    d_lvl = torch.full((V + GUARD,), 0x5A5A5A5A, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    st = bfs_noalloc(d_off.data_ptr(), d_dst.data_ptr(), V, bad_E, root, d_lvl.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    assert st == L.EFORMAT, (case, st, lib.cgb_last_error_string())
    assert np.all(d_lvl.cpu().numpy().view(np.uint32)[V:] == 0x5A5A5A5A)
    # the shared scratch is usable again at once
    g_off, g_dst = _device(off, torch), _device(dst, torch)
    st = bfs_noalloc(g_off.data_ptr(), g_dst.data_ptr(), V, E, root, d_lvl.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    assert st == L.OK, lib.cgb_last_error_string()
    np.testing.assert_array_equal(d_lvl.cpu().numpy().view(np.uint32)[:V], oracle.bfs(off, dst, root))


def test_noalloc_rejects_graphs_over_its_limit():
    lib = L.lib()
    bfs_noalloc = _noalloc(lib)
    too_many = MAX_V + 1
    # Size checks come before any device access, so dummy pointers are never read.
    st = bfs_noalloc(ctypes.c_void_p(16), ctypes.c_void_p(16), too_many, 1, 0, ctypes.c_void_p(16), None)
    assert st == L.EINVAL
    assert b"CGB_NOALLOC_MAX_VERTICES" in lib.cgb_last_error_string()
