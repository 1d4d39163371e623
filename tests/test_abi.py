"""The C-ABI library loads and exports every symbol include/*.h declares;
argument errors come back as status codes (no GPU needed)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            text = open(os.path.join(inc, f)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(cgb_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    from cggraph_b200 import build
    build.build()
    from cggraph_b200 import _lib
    return _lib.lib()


def test_library_exports_every_declared_symbol(lib):
    syms = declared_symbols()
    assert len(syms) >= 15
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_binding_list_matches_headers():
    from cggraph_b200 import _lib
    assert sorted(_lib.EXPORTS) == declared_symbols()


def test_argument_errors_are_status_codes(lib):
    from cggraph_b200 import _lib
    assert lib.cgb_abi_version() == 1
    assert lib.cgb_graph_create(None, None, None, 4, 0, 0, 0, None) == _lib.EINVAL
    h = ctypes.c_void_p()
    assert lib.cgb_graph_create(None, None, None, 4, 0, 0, 0, ctypes.byref(h)) == _lib.EINVAL
    assert b"offsets" in lib.cgb_last_error_string()
    assert lib.cgb_run(None, 0, 0, None, None, None, None) == _lib.EINVAL
    assert lib.cgb_status_string(_lib.EFORMAT) == b"invalid CSR"
    # sizes beyond 2^32 - 2^24 are refused before any array is read
    one = (ctypes.c_uint32 * 2)()
    for V, E in ((0xFF000001, 0), (4, 0xFF000001)):
        assert lib.cgb_graph_create(one, one, None, V, E, 0, 0, ctypes.byref(h)) == _lib.EUNSUPPORTED
        assert b"2^32 - 2^24" in lib.cgb_last_error_string()


def test_file_sizes_follow_the_reference(lib, tmp_path):
    """load_binFile takes a file of total_bytes / 4 == length elements and
    ignores trailing bytes short of one; the edge-list reader takes
    total_bytes / 12 records and ignores a trailing partial one.  Accepted
    files get past the size check (CGB_ECUDA without a GPU); the reference's
    own loaders accept and reject the same files when its harness is built."""
    import subprocess
    import numpy as np
    from cggraph_b200 import _lib
    from oracle import oracle as O
    off, dst, w = O.rmat_graph(8, 8, seed=1)
    V, E = off.size - 1, dst.size
    po, pd, pw = (tmp_path / n for n in ("off.bin", "dst.bin", "w.bin"))
    off.tofile(po)
    w.tofile(pw)
    h = ctypes.c_void_p()
    for extra, accepted in ((b"", True), (b"\7\7", True), (b"\7\7\7\7", False)):
        pd.write_bytes(dst.tobytes() + extra)
        st = lib.cgb_graph_load_files(str(po).encode(), str(pd).encode(), str(pw).encode(), V, E, 0,
                                      ctypes.byref(h))
        assert (st != _lib.EIO) == accepted, (extra, st)
        if st == _lib.OK:
            lib.cgb_graph_destroy(h)
        if O.ref_available():
            r = subprocess.run([O.REF_BIN, "0", str(V), str(E), str(po), str(pd), str(pw), "0", "-"],
                               capture_output=True)
            assert (r.returncode == 0) == accepted, (extra, r.returncode)
    rec = O.csr_to_edge_list(off, dst, w, seed=2)
    pe = tmp_path / "edges.bin"
    for extra in (b"", b"\1" * 5, b"\1" * 11):
        pe.write_bytes(rec.tobytes() + extra)
        st = lib.cgb_graph_load_edge_file(str(pe).encode(), V, 0, ctypes.byref(h))
        assert st != _lib.EIO, (extra, st)
        if st == _lib.OK:
            lib.cgb_graph_destroy(h)
        if O.ref_available():
            ref = O._csr_lines(subprocess.run([O.REF_BIN, "edges", str(V), str(pe)], capture_output=True,
                                              text=True).stdout)
            for a, b in zip(ref, (off, dst, w)):
                np.testing.assert_array_equal(a, b)


def test_load_files_size_check(lib, tmp_path):
    """load_binFile's size assertion becomes CGB_EIO (Basic/Other/IO.hpp:50-52)."""
    import numpy as np
    from cggraph_b200 import _lib
    off = tmp_path / "off.bin"
    dst = tmp_path / "dst.bin"
    np.array([0, 1, 1], np.uint32).tofile(off)
    np.array([1, 0], np.uint32).tofile(dst)  # two entries where E = 1 is claimed
    h = ctypes.c_void_p()
    st = lib.cgb_graph_load_files(str(off).encode(), str(dst).encode(), None, 2, 1, 0, ctypes.byref(h))
    assert st == _lib.EIO
    st = lib.cgb_graph_load_files(str(tmp_path / "nope").encode(), str(dst).encode(), None, 2, 1, 0,
                                  ctypes.byref(h))
    assert st == _lib.EIO


def run_cpp_adapter(tmp_path):
    """Compiles a main_partition-style driver against include/cgb200.hpp and
    returns its output."""
    import subprocess
    src = tmp_path / "adapter.cpp"
    src.write_text(r'''
#include "cgb200.hpp"
#include <cstdio>
struct CSR_Result_type { uint32_t vertexNum, edgeNum; uint32_t *csr_offset, *csr_dest, *csr_weight;
                         uint32_t noZeroOutDegreeNum; };
int main() {
    uint32_t off[4] = {0, 1, 2, 2}, dst[2] = {1, 2}, w[2] = {5, 7};
    CSR_Result_type csr{3, 2, off, dst, w, 3};
    try {
        cgb200::GraphB200<CSR_Result_type> g(csr, CGB_SSSP);
        g.graphProcess_device(CGB_SSSP, 0);
        g.result_D2H();
        std::printf("%u %u %u\n", g.vertexValue[0], g.vertexValue[1], g.vertexValue[2]);
    } catch (const cgb200::error& e) {
        std::printf("status %d\n", (int)e.status);
    }
    try {
        cgb200::ReorderB200<CSR_Result_type> reorder(csr);
        reorder.generateReorderGraphFile(CGB_ORDER_MY_BFS_OUT, std::string(EDGE_FILE) + ".off");
        CSR_Result_type r = reorder.get_CSR_reorder();
        std::printf("%u %u %u %u\n", reorder.old2new[0], reorder.old2new[2], r.noZeroOutDegreeNum,
                    r.csr_offset[3]);
    } catch (const cgb200::error& e) {
        std::printf("status %d\n", (int)e.status);
    }
    try {
        cgb200::GraphB200<CSR_Result_type> g(std::string(EDGE_FILE), 3, CGB_SSSP);
        uint32_t w2[2] = {5, 7};
        g.setWeights(w2);
        g.graphProcess_device(CGB_SSSP, 0);
        g.result_D2H();
        std::printf("%u %u %u\n", g.vertexValue[0], g.vertexValue[1], g.vertexValue[2]);
    } catch (const cgb200::error& e) {
        std::printf("status %d\n", (int)e.status);
    }
    return 0;
}
''')
    edges = tmp_path / "edges.bin"
    import struct
    edges.write_bytes(struct.pack("<6I", 1, 2, 1, 0, 1, 1))  # (src, dst, w) records; weights replaced later
    exe = tmp_path / "adapter"
    libdir = os.path.join(ROOT, "cggraph_b200")
    subprocess.check_call(["g++", "-std=c++17", "-O1", f'-DEDGE_FILE="{edges}"', str(src), "-I",
                           os.path.join(ROOT, "include"), "-L", libdir,
                           "-lcgb200", f"-Wl,-rpath,{libdir}", "-o", str(exe)])
    return subprocess.run([str(exe)], capture_output=True, text=True, timeout=120).stdout.strip()


# SSSP on the path 0 -> 1 -> 2 (weights 5, 7); its MY_BFS_OUT order is 0, 1,
# then 2 (no out-edges) last; SSSP again from the edge-list file.
ADAPTER_GPU_OUT = "0 5 12\n0 2 2 2\n0 5 12"


def test_cpp_adapter_compiles_and_reports_status(tmp_path, lib):
    """include/cgb200.hpp (the GraphDeviceWorklist- and Reorder-shaped
    adapters) compiles against a CSR_Result_type-like struct and links;
    without a GPU the constructors throw cgb200::error with CGB_ECUDA."""
    import torch
    out = run_cpp_adapter(tmp_path)
    assert out == (ADAPTER_GPU_OUT if torch.cuda.is_available() else "status 5\nstatus 5\nstatus 5"), out


@pytest.mark.gpu
def test_cpp_adapter_runs(tmp_path, lib):
    """The adapters on a GPU: SSSP from the CSR and from an edge-list file
    given its weights later, and the relabelling of the Reorder adapter."""
    assert run_cpp_adapter(tmp_path) == ADAPTER_GPU_OUT


def test_struct_layouts_match_header(tmp_path):
    """The ctypes mirrors of the public structs have the C header's sizes
    and field offsets."""
    import subprocess
    from cggraph_b200 import _lib
    structs = {"cgb_options": _lib.Options, "cgb_run_stats": _lib.RunStats, "cgb_iter_trace": _lib.IterTrace,
               "cgb_server_config": _lib.ServerConfig, "cgb_request_info": _lib.RequestInfo,
               "cgb_tuning": _lib.Tuning, "cgb_partition_info": _lib.PartitionInfo}
    lines = ['#include "cgb200.h"', "#include <stdio.h>", "#include <stddef.h>", "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(line.rsplit(" ", 1) for line in subprocess.run([str(exe)], check=True, capture_output=True,
                                                              text=True).stdout.split("\n") if line)
    for cname, py in structs.items():
        assert int(got[cname]) == ctypes.sizeof(py), cname
        for f, _ in py._fields_:
            assert int(got[f"{cname}.{f}"]) == getattr(py, f).offset, f"{cname}.{f}"


def test_flag_constants_match_header():
    """Every CGB_ flag and limit #define of the header that the Python
    mirror names has the header's value (server, run, tuning flags...)."""
    import re
    from cggraph_b200 import _lib
    text = open(os.path.join(ROOT, "include", "cgb200.h")).read()
    defs = re.findall(r"#define CGB_(\w+)\s+(0x[0-9a-fA-F]+|\d+)u?\b", text)
    named = [(n, int(v, 0)) for n, v in defs if hasattr(_lib, n)]
    assert len(named) >= 20
    for n, v in named:
        assert getattr(_lib, n) == v, n
    for n in ("SERVER_NO_BFS", "SERVER_NO_SSSP", "SERVER_HOST_TICKS", "SERVER_BATCH_ONLY", "SERVER_ADMIT_ANY_SLOT",
              "FLAG_CC_WEAK", "TUNE_CC_WEAK"):
        assert any(m == n for m, _ in named), n
