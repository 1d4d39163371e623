"""cgb_bfs_noalloc: BFS for callers that cannot allocate device memory.

Such a caller -- for example a framework whose caching allocator already owns
the device's memory, or a serving loop that forbids cudaMalloc after start-up
-- passes its own device CSR and output buffer; the entry point keeps its
frontier queues and bitmap in a static device array instead of allocating.
This test calls it through the C ABI twice in a row and checks each result
against the allocating entry point (cgb_run, BFS), bit for bit, and that the
second call leaves the device's free memory unchanged.  It runs last so that
a failure here never hides the other tests, and it must pass both alone in a
fresh process and after the rest of the suite.
"""
import ctypes

import numpy as np
import pytest

import cggraph_b200 as cg
from cggraph_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _noalloc(lib):
    f = lib.cgb_bfs_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                  ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def test_noalloc_bfs_matches_allocating_entry_point(oracle):
    import torch
    lib = L.lib()
    bfs_noalloc = _noalloc(lib)
    off, dst, w = oracle.rmat_graph(16, 16, seed=77)
    V, E = off.size - 1, dst.size
    d_off = torch.from_numpy(off.view(np.int32)).cuda()
    d_dst = torch.from_numpy(dst.view(np.int32)).cuda()
    d_lvl = torch.empty(V, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    deg = np.diff(off.astype(np.int64))
    roots = [int(deg.argmax()), int(np.nonzero(deg)[0][3])]
    with cg.Graph.from_csr(off, dst, w) as g:
        expected = [g.run(0, r)[0] for r in roots]
    torch.cuda.synchronize()
    free_after_first = None
    for i, r in enumerate(roots):
        st = bfs_noalloc(d_off.data_ptr(), d_dst.data_ptr(), V, E, r, d_lvl.data_ptr(), stream.cuda_stream)
        assert st == L.OK, lib.cgb_last_error_string()
        torch.cuda.synchronize()
        got = d_lvl.cpu().numpy().view(np.uint32)
        np.testing.assert_array_equal(got, expected[i], err_msg=f"call {i + 1}, root {r}")
        free_now = torch.cuda.mem_get_info()[0]
        if i == 0:
            free_after_first = free_now
        else:
            assert free_now == free_after_first, "the second call changed the device's free memory"


def test_noalloc_rejects_graphs_over_its_limit():
    lib = L.lib()
    bfs_noalloc = _noalloc(lib)
    too_many = (1 << 20) + 1
    # Size checks come before any device access, so dummy pointers are never read.
    st = bfs_noalloc(ctypes.c_void_p(16), ctypes.c_void_p(16), too_many, 1, 0, ctypes.c_void_p(16), None)
    assert st == L.EINVAL
    assert b"CGB_NOALLOC_MAX_VERTICES" in lib.cgb_last_error_string()
