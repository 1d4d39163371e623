"""Request server on the GPU: queries that arrive while others run are
admitted into freed slots, and every result equals a lone run of the same
query (bit-exact for BFS levels and SSSP distances)."""
import numpy as np
import pytest

import cggraph_b200 as cg
from cggraph_b200 import _lib as L

pytestmark = pytest.mark.gpu

BFS, SSSP = 0, 1


def _poisson_arrivals(n, rate_per_s, seed):
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1e6 / rate_per_s, n))


def _serve_and_check(g, queries, arrivals, **cfg):
    V = g.vertexNum
    outs = [np.full(V, 7, np.uint32) for _ in queries]
    with cg.Server(g, **cfg) as srv:
        ids = [srv.submit(a, r, t, out=o) for (a, r), t, o in zip(queries, arrivals, outs)]
        srv.start()
        assert srv.wait(120000) == 0
        recs = {r["id"]: r for r in srv.poll()}
        st = srv.stats()
    assert sorted(recs) == sorted(ids)
    for i, ((alg, root), rid) in enumerate(zip(queries, ids)):
        rec = recs[rid]
        assert rec["status"] == 0
        assert rec["arrival_us"] <= rec["admit_us"] <= rec["done_us"]
        lone, _ = g.run(alg, root)
        np.testing.assert_array_equal(outs[i], lone, err_msg=f"query {i} alg {alg} root {root}")
        off = g._host_off
        deg = np.diff(off.astype(np.int64))
        assert rec["traversed_edges"] == int(deg[lone != L.VALUE_MAX].sum())
        assert rec["reached"] == int((lone != L.VALUE_MAX).sum())
    return recs, st


@pytest.mark.parametrize("flags", [0, L.SERVER_HOST_TICKS, L.SERVER_BATCH_ONLY, L.SERVER_ADMIT_ANY_SLOT])
def test_server_mix_equals_lone_runs(oracle, flags):
    """RMAT-14 (weights 1..64): 120 BFS/SSSP queries with Poisson arrivals,
    8 slots per algorithm so that slots are reused while other queries run;
    BFS levels in the device-resident loop (default) or one host tick per
    level; queries that find their group idle on the single-root engine
    (default) or batched like the rest."""
    off, dst, w = oracle.rmat_graph(14, 16, seed=31)
    rng = np.random.default_rng(4)
    V = off.size - 1
    queries = [(int(rng.integers(0, 2)), int(rng.integers(0, V))) for _ in range(120)]
    queries[5] = (BFS, queries[3][1])  # repeated roots
    queries[6] = (SSSP, queries[3][1])
    arrivals = _poisson_arrivals(len(queries), 20000, 9)
    with cg.Graph.from_csr(off, dst, w) as g:
        g._host_off = off
        recs, st = _serve_and_check(g, queries, arrivals, bfs_slots=8, sssp_slots=8, flags=flags)
        assert st["bfs_slots"] == 8 and st["sssp_slots"] == 8
        # slots were reused: more queries than slots per algorithm
        assert max(r["slot"] for r in recs.values()) < 8


@pytest.mark.parametrize("flags", [0, L.SERVER_HOST_TICKS, L.SERVER_BATCH_ONLY])
def test_server_high_diameter_grid(oracle, flags):
    """A grid keeps SSSP queries alive for hundreds of rounds while short
    BFS queries come and go; per-slot buckets keep late arrivals exact; BFS
    levels run many per launch in the device-resident loop (default)."""
    off, dst, w = oracle.grid_graph(40, 60, seed=5)
    rng = np.random.default_rng(2)
    V = off.size - 1
    queries = [(int(rng.integers(0, 2)), int(rng.integers(0, V))) for _ in range(40)]
    arrivals = _poisson_arrivals(len(queries), 5000, 3)
    with cg.Graph.from_csr(off, dst, w) as g:
        g._host_off = off
        _serve_and_check(g, queries, arrivals, bfs_slots=4, sssp_slots=4, sssp_delta=300, flags=flags)


@pytest.mark.parametrize("seed", [11, 12, 13, 14])
def test_server_loop_and_tick_switches(oracle, seed):
    """Default flags on the grid with both algorithms in the mix: the SSSP
    group runs its device-resident loop while the BFS group is idle and host
    ticks while it is not, so one traversal switches between the two many
    times; thresholds advanced on the device must reach the host ticks (a
    stale threshold once dropped vertices from a late query's far list)."""
    off, dst, w = oracle.grid_graph(40, 60, seed=5)
    rng = np.random.default_rng(seed)
    V = off.size - 1
    queries = [(int(rng.integers(0, 2)), int(rng.integers(0, V))) for _ in range(48)]
    arrivals = _poisson_arrivals(len(queries), 2000 * (seed - 10), seed)
    with cg.Graph.from_csr(off, dst, w) as g:
        g._host_off = off
        _serve_and_check(g, queries, arrivals, bfs_slots=4, sssp_slots=4, sssp_delta=300)


def test_server_sparse_arrivals_run_alone(oracle):
    """Below capacity (20 req/s against queries of well under a
    millisecond) each query finds its group idle and runs on the
    single-root engine: results exact, and each query's latency close to
    a lone run's (admitted on arrival, done within 50 ms)."""
    off, dst, w = oracle.rmat_graph(14, 16, seed=7)
    rng = np.random.default_rng(8)
    V = off.size - 1
    queries = [(int(rng.integers(0, 2)), int(rng.integers(0, V))) for _ in range(12)]
    arrivals = 50000.0 * np.arange(1, len(queries) + 1)
    with cg.Graph.from_csr(off, dst, w) as g:
        g._host_off = off
        recs, _ = _serve_and_check(g, queries, arrivals)
        for r in recs.values():
            assert r["admit_us"] - r["arrival_us"] < 10000
            assert r["done_us"] - r["arrival_us"] < 50000


def test_weights_fixed_while_a_server_is_attached(oracle):
    """The SSSP group and its second engine context read the weights without
    the graph's lock, so replacing them is refused while a server exists,
    and allowed again once it is gone."""
    off, dst, w = oracle.rmat_graph(12, 8, seed=3)
    with cg.Graph.from_csr(off, dst, w) as g:
        srv = cg.Server(g)
        with pytest.raises(cg.CgbError):
            g.set_weights(w)
        srv.close()
        g.set_weights(w[::-1].copy())
        lone, _ = g.run(SSSP, 1)
        g.set_weights(w)
        np.testing.assert_array_equal(g.run(SSSP, 1)[0], oracle.sssp(off, dst, w, 1))


def test_server_memory_budget_caps_slots(oracle):
    off, dst, w = oracle.rmat_graph(12, 8, seed=2)
    V = off.size - 1
    with cg.Graph.from_csr(off, dst, w) as g:
        g._host_off = off
        with cg.Server(g, memory_budget=3 * 4 * V) as srv:
            st = srv.stats()
            assert st["bfs_slots"] + st["sssp_slots"] == 3
        queries = [(BFS, 1), (SSSP, 2), (BFS, 3), (SSSP, 4), (BFS, 5), (SSSP, 6), (BFS, 7)]
        _serve_and_check(g, queries, [0.0] * len(queries), memory_budget=3 * 4 * V)
        with pytest.raises(cg.CgbError):
            cg.Server(g, memory_budget=4 * V - 1)
        with cg.Server(g, flags=L.SERVER_NO_SSSP) as srv:
            with pytest.raises(cg.CgbError):
                srv.submit(SSSP, 0)
            with pytest.raises(cg.CgbError):
                srv.submit(BFS, V)
