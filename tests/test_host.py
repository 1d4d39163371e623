"""Host-side mirror of the reference interface (no GPU needed)."""
import numpy as np
import pytest

import cggraph_b200 as cg
from cggraph_b200 import CgbError


def test_enum_values_match_reference():
    # Basic/Graph/basic_struct.hpp:144-151,165-178
    assert [int(a) for a in (cg.Algorithm_type.BFS, cg.Algorithm_type.SSSP, cg.Algorithm_type.CC,
                             cg.Algorithm_type.PR)] == [0, 1, 2, 3]
    assert int(cg.Engine_type.SINGLE_GPU) == 4 and int(cg.Engine_type.MULTI_CORE) == 3
    assert int(cg.OrderMethod.RCM_LAST_ZERO_OUTDEGREE) == 6 and int(cg.OrderMethod.IN_DEGREE_DEC) == 21
    assert cg.VertexValue_MAX == 999999999


def test_load_bin_file_checks_size(tmp_path):
    p = tmp_path / "a.bin"
    np.arange(5, dtype=np.uint32).tofile(p)
    np.testing.assert_array_equal(cg.load_binFile(str(p), 5), np.arange(5))
    with pytest.raises(CgbError):
        cg.load_binFile(str(p), 4)
    with pytest.raises(CgbError):
        cg.load_binFile(str(tmp_path / "missing.bin"), 4)
    cg.save_binArray(str(tmp_path / "b.bin"), np.arange(3, dtype=np.uint32))
    assert (tmp_path / "b.bin").stat().st_size == 12


def test_trimmed_mean():
    # main_partition.hpp:347-365
    assert cg.trimmed_mean_ms([5.0, 1.0, 3.0, 100.0]) == 4.0
    assert cg.trimmed_mean_ms([2.0, 4.0]) == 3.0
    assert cg.trimmed_mean_ms([7.0]) == 7.0


def test_check_bin_result(tmp_path):
    ref = np.array([0, 1, 2, 999999999], np.uint32)
    cg.checkBinResult(ref, ref.copy(), 4)
    p = tmp_path / "g.bin"
    ref.tofile(p)
    cg.checkBinResult(str(p), ref.copy(), 4)
    bad = ref.copy()
    bad[2] = 5
    with pytest.raises(AssertionError, match=r"current_array\[2\]"):
        cg.checkBinResult(ref, bad, 4)
    # reordered graph: current array indexed through old2new (util.cuh:88-112)
    old2new = np.array([3, 2, 1, 0])
    cg.checkBinResult(ref, ref[::-1].copy(), 4, cg.OrderMethod.RCM, old2new)


def test_only_single_gpu_engine_is_provided():
    csr = cg.CSR_Result_type(2, 1, np.array([0, 1, 1], np.uint32), np.array([1], np.uint32), None)
    with pytest.raises(CgbError, match="SINGLE_GPU"):
        cg.main_partition(csr, cg.Algorithm_type.BFS, 0, engine_type=cg.Engine_type.COORDINATION)


def test_chunglu_weight_offset_matches_twin(oracle):
    """The offset helper's distinct-degree estimate against the CPU twin's
    actual largest out-degree."""
    import numpy as np
    import cggraph_b200 as cg
    V, n = 20011, 300000
    i0 = cg.chunglu_weight_offset(V, n, 3000)
    off, _, _ = oracle.chunglu_graph(V, n, i0, seed=3)
    top = int(np.diff(off.astype(np.int64)).max())
    assert 0.8 * 3000 < top < 1.25 * 3000
    assert cg.chunglu_weight_offset(V, n, 100) > cg.chunglu_weight_offset(V, n, 3000)


def test_chunglu_draws_for_edges_matches_twin(oracle):
    """The draw-count solver: the CPU twin, given the solved draws and
    offset, keeps the requested number of distinct edges (to 1 %), and the
    expected-edge estimate tracks the twin's count at another draw count."""
    import numpy as np
    import cggraph_b200 as cg
    V, want = 200003, 3_000_000
    draws, i0 = cg.chunglu_draws_for_edges(V, want, 20000)
    assert draws > want
    off, _, _ = oracle.chunglu_graph(V, draws, i0, seed=5)
    assert abs(int(off[-1]) - want) < 0.01 * want
    off, _, _ = oracle.chunglu_graph(V, want, 7, seed=6)
    est = cg.chunglu_expected_edges(V, want, 7)
    assert abs(int(off[-1]) - est) < 0.01 * est


def test_reorder_engine_type_writes_the_reference_files(tmp_path, monkeypatch):
    """main_partition(Engine_type.REORDER) is the reference's preprocessing
    branch (main_partition.hpp:466-487): the IN_DEGREE_DEC relabelling, written
    as saveCSR_reorderFile's five files.  The device call is replaced by the
    oracle's restatement here, so only the host logic is under test."""
    import cggraph_b200.engine as E
    from oracle import oracle as O

    off, dst, w = O.rmat_graph(9, 8, seed=4)
    V = off.size - 1

    class FakeReordered:
        def __init__(self, method):
            self.o, self.d, self.w, self.m, self.nz = O.reorder(off, dst, w, int(method))

        def __enter__(self):
            return self

        def __exit__(self, *exc):
            return False

        def download(self, with_weight=True):
            return self.o, self.d, (self.w if with_weight else None)

    class FakeGraph:
        @classmethod
        def from_csr(cls, o, d, ww=None, device=0):
            assert o is off and d is dst and ww is w
            return cls()

        def __enter__(self):
            return self

        def __exit__(self, *exc):
            return False

        def reorder(self, method):
            h = FakeReordered(method)
            return h, h.m, h.nz

    monkeypatch.setattr(E, "Graph", FakeGraph)
    files = {k: str(tmp_path / f"{k}.bin") for k in ("offsets", "dest", "weight", "old2new", "addition")}
    csr = cg.CSR_Result_type(V, dst.size, off, dst, w)
    r = cg.main_partition(csr, cg.Algorithm_type.BFS, engine_type=cg.Engine_type.REORDER, reorder_files=files)
    o2, d2, w2, m2, nz = O.reorder(off, dst, w, 21)
    np.testing.assert_array_equal(np.fromfile(files["offsets"], np.uint32), o2)
    np.testing.assert_array_equal(np.fromfile(files["dest"], np.uint32), d2)
    np.testing.assert_array_equal(np.fromfile(files["weight"], np.uint32), w2)
    np.testing.assert_array_equal(np.fromfile(files["old2new"], np.uint32), m2)
    assert np.fromfile(files["addition"], np.uint32).size == 0  # IN_DEGREE_DEC keeps no zero tail
    assert r["zeroOutDegreeNum"] == V - nz and r["csr"].noZeroOutDegreeNum == nz
    r = cg.reorder_graph(csr, cg.OrderMethod.MY_BFS_OUT, files)
    o2, d2, w2, m2, nz = O.reorder(off, dst, w, 16)
    np.testing.assert_array_equal(np.fromfile(files["old2new"], np.uint32), m2)
    assert np.fromfile(files["addition"], np.uint32).tolist() == [V - nz]


def test_compute_indegree_engine_type():
    """main_partition(Engine_type.COMPUTE_INDEGREE): the degrees and the
    vertices of largest in-degree (Compute_indegree.cuh:114-195)."""
    off = np.array([0, 2, 3, 5, 5], np.uint32)
    dst = np.array([1, 3, 3, 0, 3], np.uint32)
    csr = cg.CSR_Result_type(4, 5, off, dst, None)
    r = cg.main_partition(csr, cg.Algorithm_type.BFS, engine_type=cg.Engine_type.COMPUTE_INDEGREE)
    assert r["inDegree"].tolist() == [1, 1, 0, 3] and r["outDegree"].tolist() == [2, 1, 2, 0]
    assert r["top"] == [(3, 3), (0, 1), (1, 1), (2, 0)]


def test_bench_refuses_gpus_without_one_process_per_gpu():
    """bench.py --gpus N without torchrun's WORLD_SIZE=N stops with a message
    naming the launch it needs, before any device work."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--gpus", "2", "--steps", "1"],
                       capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode != 0
    assert "torch.distributed.run --nproc-per-node 2" in r.stderr + r.stdout
