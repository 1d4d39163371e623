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
