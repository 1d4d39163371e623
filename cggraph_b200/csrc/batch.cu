// Batches of independent graphs solved together.
//
// The n graphs are concatenated into one disjoint-union graph (graph i's
// vertex v becomes base[i] + v).  Components never cross graphs, so
//   BFS / SSSP from one root per graph = one multi-source run on the union
//     with every root at distance 0, done by one cooperative device-resident
//     launch (k_bfs_persistent without exit thresholds, k_sssp_device),
//     captured once into a CUDA graph and replayed for later batches;
//   CC = CC of the union with each label taken relative to its graph's base.
// Results are written per graph in local ids, concatenated in graph order.
#include <vector>

#include "../../include/cgb200.h"
#include "engine.cuh"
#include "persist.cuh"

struct cgb_batch {
    uint32_t n = 0;
    std::vector<uint32_t> base;  // n + 1 vertex offsets
    uint32_t* d_base = nullptr;
    uint32_t* d_roots = nullptr;
    cgb_graph* g = nullptr;
    cudaGraphExec_t exec[2] = {nullptr, nullptr};  // BFS, SSSP
    bool captured[2] = {false, false};
    bool capture_failed[2] = {false, false};
    cgb::PersistSssp* sx = nullptr;
    uint32_t delta = 1;
};

namespace cgb {

// Graph i's offsets shifted by the edges before it; its own invariants
// (off[0] == 0, off[Vi] == Ei, non-decreasing) are checked here because the
// union's check cannot see a graph boundary.
__global__ void k_union_off(const uint32_t* __restrict__ off, uint32_t Vi, uint32_t Ei, uint32_t ebase, uint32_t* uoff,
                            uint32_t* bad)
{
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < Vi; j += gridDim.x * blockDim.x) {
        uoff[j] = off[j] + ebase;
        if (off[j] > off[j + 1]) atomicOr(bad, 1u);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && (off[0] != 0 || off[Vi] != Ei)) atomicOr(bad, 1u);
}

__global__ void k_union_dst(const uint32_t* __restrict__ dst, uint32_t Ei, uint32_t Vi, uint32_t vbase, uint32_t* udst,
                            uint32_t* bad)
{
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < Ei; e += gridDim.x * blockDim.x) {
        const uint32_t d = dst[e];
        if (d >= Vi) atomicOr(bad, 2u);
        udst[e] = min(d, Vi - 1) + vbase;
    }
}

__global__ void k_fill_ones(uint32_t n, uint32_t* a)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = 1;
}

// Values MAX, visited 0; for SSSP also the far bitmap and the near bitmap
// of slot 1 (the first round's; the kernel zeroes the others ahead of use).
__global__ void k_batch_init(uint32_t V, uint32_t* val, uint32_t* visited, uint32_t words, uint32_t* far_bm,
                             uint32_t* near_bm1)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += stride) val[i] = kValueMax;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < words; i += stride) {
        visited[i] = 0;
        if (far_bm) {
            far_bm[i] = 0;
            near_bm1[i] = 0;
        }
    }
}

__global__ void k_batch_roots(const uint32_t* roots, const uint32_t* base, uint32_t n, uint32_t nz, uint32_t* val,
                              uint32_t* visited, uint32_t* q, PersistState* st, PersistSssp* sx, uint32_t delta)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    uint32_t len = 0;
    for (uint32_t i = 0; i < n; i++) {
        const uint32_t r = base[i] + roots[i];
        if (val[r] == 0) continue;
        val[r] = 0;
        visited[r >> 5] |= 1u << (r & 31u);
        if (r < nz) q[len++] = r;
    }
    st->qlen[0] = len;
    if (sx) {
        sx->bucket_lo = 0;
        sx->thr[0] = delta;
        for (int k = 0; k < 3; k++) {
            sx->min_far[k] = kValueMax;
            sx->far_delta[k] = 0;
            sx->kept[k] = 0;
            sx->split[k] = 0;
        }
    }
}

// CC labels of the union relative to each vertex's graph.
__global__ void k_batch_local_labels(uint32_t V, const uint32_t* __restrict__ base, uint32_t n, uint32_t* lab)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = n;  // graph i with base[i] <= v < base[i+1]
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (base[mid] <= v) lo = mid;
            else hi = mid;
        }
        lab[v] -= base[lo];
    }
}

}  // namespace cgb

using namespace cgb;

template <typename F>
static cgb_status bguard(F&& f)
{
    try {
        f();
        return CGB_OK;
    } catch (const Error& e) {
        set_error(e.msg);
        return e.code;
    } catch (const std::exception& e) {
        set_error(e.what());
        return CGB_ECUDA;
    }
}

// Queues one whole multi-source run (BFS alg 0 / SSSP alg 1) on the stream.
static void enqueue_batch_run(cgb_batch* b, int alg)
{
    cgb_graph* g = b->g;
    const uint32_t V = g->V, words = g->words();
    PersistState* st = static_cast<PersistState*>(g->persist);
    uint32_t* far_bm = alg == 1 ? g->front_bm : nullptr;
    CGB_CUDA_TRY(cudaMemsetAsync(st, 0, sizeof(PersistState), g->stream));
    k_batch_init<<<grid_for(V, kBlock, num_sms() * 8), kBlock, 0, g->stream>>>(V, g->value, g->visited, words, far_bm,
                                                                             g->aux_bm + words);
    k_batch_roots<<<1, 1, 0, g->stream>>>(b->d_roots, b->d_base, b->n, g->nz, g->value, g->visited, g->q[0], st,
                                          alg == 1 ? b->sx : nullptr, b->delta);
    if (alg == 0) launch_bfs_unbounded(g, st);
    else launch_sssp_device(g, far_bm, b->delta, st, b->sx);
}

extern "C" {

cgb_status cgb_batch_create(uint32_t n, const uint32_t* const* offsets, const uint32_t* const* dests,
                            const uint32_t* const* weights, const uint32_t* Vs, const uint32_t* Es, int device,
                            cgb_batch** out)
{
    return bguard([&] {
        CGB_REQUIRE(out && offsets && dests && Vs && Es && n >= 1, CGB_EINVAL, "bad batch arguments");
        *out = nullptr;
        uint64_t Vt = 0, Et = 0;
        bool any_w = false;
        for (uint32_t i = 0; i < n; i++) {
            CGB_REQUIRE(Vs[i] >= 1 && offsets[i] && (Es[i] == 0 || dests[i]), CGB_EINVAL, "bad graph in batch");
            Vt += Vs[i];
            Et += Es[i];
            any_w |= weights && weights[i];
        }
        CGB_REQUIRE(Vt <= kMaxGraphSize && Et <= kMaxGraphSize, CGB_EUNSUPPORTED,
                    "batch exceeds 2^32 - 2^24 vertices or edges");
        cgb_batch* b = new cgb_batch();
        try {
            b->n = n;
            b->g = graph_alloc((uint32_t)Vt, (uint32_t)Et, (uint32_t)Vt, device, any_w);
            cgb_graph* g = b->g;
            b->base.assign(n + 1, 0);
            uint32_t* tmp = nullptr;
            size_t tmp_cap = 0;
            uint64_t vb = 0, eb = 0;
            CGB_CUDA_TRY(cudaMalloc((void**)&b->d_roots, 4 * std::max<uint32_t>(n, 1)));
            uint32_t* bad = b->d_roots;  // used as the check flag until the roots are needed
            CGB_CUDA_TRY(cudaMemsetAsync(bad, 0, 4, g->stream));
            for (uint32_t i = 0; i < n; i++) {
                const size_t need = std::max<size_t>((size_t)Vs[i] + 1, Es[i]) * 4;
                if (need > tmp_cap) {
                    if (tmp) cudaFree(tmp);
                    CGB_CUDA_TRY(cudaMalloc((void**)&tmp, need));
                    tmp_cap = need;
                }
                CGB_CUDA_TRY(cudaMemcpyAsync(tmp, offsets[i], ((size_t)Vs[i] + 1) * 4, cudaMemcpyDefault, g->stream));
                k_union_off<<<grid_for(Vs[i], kBlock, num_sms() * 4), kBlock, 0, g->stream>>>(tmp, Vs[i], Es[i], (uint32_t)eb,
                                                                                           g->off + vb, bad);
                if (Es[i]) {
                    CGB_CUDA_TRY(cudaMemcpyAsync(tmp, dests[i], (size_t)Es[i] * 4, cudaMemcpyDefault, g->stream));
                    k_union_dst<<<grid_for(Es[i], kBlock, num_sms() * 4), kBlock, 0, g->stream>>>(tmp, Es[i], Vs[i],
                                                                                                (uint32_t)vb,
                                                                                                g->dst + eb, bad);
                    if (g->w) {
                        if (weights && weights[i])
                            CGB_CUDA_TRY(cudaMemcpyAsync(g->w + eb, weights[i], (size_t)Es[i] * 4, cudaMemcpyDefault,
                                                         g->stream));
                        else
                            k_fill_ones<<<grid_for(Es[i], kBlock, num_sms() * 4), kBlock, 0, g->stream>>>(Es[i], g->w + eb);
                    }
                }
                CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));  // tmp is reused
                b->base[i] = (uint32_t)vb;
                vb += Vs[i];
                eb += Es[i];
            }
            b->base[n] = (uint32_t)vb;
            const uint32_t Etot = (uint32_t)Et;
            CGB_CUDA_TRY(cudaMemcpy(g->off + Vt, &Etot, 4, cudaMemcpyHostToDevice));
            if (tmp) cudaFree(tmp);
            uint32_t hbad = 0;
            CGB_CUDA_TRY(cudaMemcpy(&hbad, bad, 4, cudaMemcpyDeviceToHost));
            CGB_REQUIRE(!(hbad & 1u), CGB_EFORMAT, "a batch graph's offsets violate offsets[0]==0, offsets[V]==E, order");
            CGB_REQUIRE(!(hbad & 2u), CGB_EFORMAT, "a batch graph's dest holds an id >= its V");
            validate_and_sort(g);  // sorts each list; a graph's ids stay inside its own range
            compute_weight_sum(g);
            CGB_CUDA_TRY(cudaMalloc((void**)&b->d_base, (n + 1) * 4ull));
            CGB_CUDA_TRY(cudaMemcpy(b->d_base, b->base.data(), (n + 1) * 4ull, cudaMemcpyHostToDevice));
            CGB_CUDA_TRY(cudaMalloc((void**)&b->sx, sizeof(PersistSssp)));
            ensure_frontier(g);
            if (!g->persist) g->persist = pool_alloc(sizeof(PersistBlock), g->stream);
            b->delta = sssp_delta_for(g, 8.0);
        } catch (...) {
            if (b->g) graph_free(b->g);
            if (b->d_base) cudaFree(b->d_base);
            if (b->d_roots) cudaFree(b->d_roots);
            if (b->sx) cudaFree(b->sx);
            delete b;
            throw;
        }
        *out = b;
    });
}

cgb_status cgb_batch_destroy(cgb_batch* b)
{
    return bguard([&] {
        if (!b) return;
        cudaSetDevice(b->g->device);
        for (int i = 0; i < 2; i++)
            if (b->exec[i]) cudaGraphExecDestroy(b->exec[i]);
        cudaFree(b->d_base);
        cudaFree(b->d_roots);
        cudaFree(b->sx);
        graph_free(b->g);
        delete b;
    });
}

cgb_status cgb_batch_info(const cgb_batch* b, uint32_t* total_vertices, uint32_t* total_edges, int32_t* one_launch)
{
    return bguard([&] {
        CGB_REQUIRE(b != nullptr, CGB_EINVAL, "batch is NULL");
        if (total_vertices) *total_vertices = b->g->V;
        if (total_edges) *total_edges = b->g->E;
        if (one_launch) *one_launch = (b->captured[0] ? 1 : 0) | (b->captured[1] ? 2 : 0);
    });
}

cgb_status cgb_batch_run(cgb_batch* b, int algorithm, const uint32_t* roots, uint32_t* out_u32, double* out_ms)
{
    return bguard([&] {
        CGB_REQUIRE(b != nullptr, CGB_EINVAL, "batch is NULL");
        CGB_REQUIRE(algorithm == CGB_BFS || algorithm == CGB_SSSP || algorithm == CGB_CC, CGB_EINVAL,
                    "batch runs are BFS, SSSP or CC");
        cgb_graph* g = b->g;
        std::lock_guard<GraphMutex> lock(g->mu);
        CGB_CUDA_TRY(cudaSetDevice(g->device));
        g->stats = cgb_run_stats{};
        if (algorithm == CGB_CC) {
            cgb_options o{};
            o.struct_size = sizeof(o);
            CGB_CUDA_TRY(cudaMemsetAsync(g->ctr, 0, sizeof(DevCounters), g->stream));
            run_cc(g, o);  // records ev_start itself
            k_batch_local_labels<<<grid_for(g->V, kBlock, num_sms() * 8), kBlock, 0, g->stream>>>(g->V, b->d_base, b->n,
                                                                                                g->value);
        } else {
            CGB_REQUIRE(roots != nullptr, CGB_EINVAL, "roots is NULL");
            for (uint32_t i = 0; i < b->n; i++)
                CGB_REQUIRE(roots[i] < b->base[i + 1] - b->base[i], CGB_EINVAL, "root outside its graph");
            const int a = algorithm == CGB_BFS ? 0 : 1;
            CGB_CUDA_TRY(cudaMemcpyAsync(b->d_roots, roots, b->n * 4ull, cudaMemcpyHostToDevice, g->stream));
            if (!b->captured[a] && !b->capture_failed[a]) {
                // capture the whole run once: memset + 2 kernels + one cooperative launch
                CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
                cudaGraph_t graph = nullptr;
                bool ok = cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
                if (ok) {
                    try {
                        enqueue_batch_run(b, a);
                    } catch (...) {
                        ok = false;
                    }
                    ok = (cudaStreamEndCapture(g->stream, &graph) == cudaSuccess) && ok;
                }
                if (ok) ok = cudaGraphInstantiate(&b->exec[a], graph, 0) == cudaSuccess;
                if (graph) cudaGraphDestroy(graph);
                cudaGetLastError();  // a refused capture leaves its error behind
                b->captured[a] = ok;
                b->capture_failed[a] = !ok;
            }
            CGB_CUDA_TRY(cudaEventRecord(g->ev_start, g->stream));
            if (b->captured[a]) CGB_CUDA_TRY(cudaGraphLaunch(b->exec[a], g->stream));
            else enqueue_batch_run(b, a);
            CGB_CUDA_TRY(cudaEventRecord(g->ev_stop, g->stream));
            PersistState h;
            CGB_CUDA_TRY(cudaMemcpyAsync(&h, g->persist, sizeof(h), cudaMemcpyDeviceToHost, g->stream));
            CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
            CGB_REQUIRE(!(h.status & 2u), CGB_EOVERFLOW, "batch run: queue overflow");
            CGB_REQUIRE(!(h.status & 1u), CGB_ETIMEOUT, "batch run: grid barrier gave up");
            g->stats.iterations = h.levels;
            g->stats.launches = b->captured[a] ? 1 : 4;
        }
        CGB_CUDA_TRY(cudaEventRecord(g->ev_stop, g->stream));
        CGB_CUDA_TRY(cudaEventSynchronize(g->ev_stop));
        float ms = 0.f;
        CGB_CUDA_TRY(cudaEventElapsedTime(&ms, g->ev_start, g->ev_stop));
        g->stats.ms = ms;
        if (algorithm != CGB_CC) {
            count_reached(g);
            const uint64_t per_edge = algorithm == CGB_BFS ? 8 : (g->w ? 12 : 8);
            g->stats.alg_bytes = per_edge * g->stats.traversed_edges + 12ull * g->V;
        } else {
            g->stats.traversed_edges = g->E;
            g->stats.reached = g->V;
            g->stats.alg_bytes = 8ull * g->E + 20ull * g->V;
        }
        g->result = g->value;
        g->result_alg = algorithm;
        if (out_u32) {
            CGB_CUDA_TRY(cudaMemcpyAsync(out_u32, g->value, (size_t)g->V * 4, cudaMemcpyDefault, g->stream));
            CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
        }
        if (out_ms) *out_ms = ms;
    });
}

cgb_status cgb_batch_stats(const cgb_batch* b, cgb_run_stats* out)
{
    return bguard([&] {
        CGB_REQUIRE(b != nullptr && out != nullptr, CGB_EINVAL, "NULL argument");
        *out = b->g->stats;
    });
}

}  // extern "C"
