// Multi-root SSSP: up to 64 roots per pass, one distance per (vertex, root)
// and bit-packed per-vertex root masks.
//
// Layout: dist[v * 64 + k] (vertex-major), so the 64 distances of a vertex
// are one 256-byte run; a warp relaxes an edge (v, u) for every root at once,
// lane k handling roots k and k + 32, with two coalesced 128-byte loads of
// dist[u][*].  Per vertex two 64-bit masks record which roots still need
// work: pend (improved below the current threshold: expand next round) and
// farm (improved at or above it: kept for a later bucket).
//
// Delta-stepping with one threshold shared by all roots: rounds expand the
// near work (pend) until none is left, then a split moves the far pairs of
// the next bucket [lo, hi) into pend (jumping to the bucket of the smallest
// far distance when a bucket is empty).  The relaxation is label-correcting
// (atomicMin; a pair is re-expanded whenever it improves), so the result is
// the exact shortest-path distance of every pair whatever the order -- equal
// to n separate cgb_run(CGB_SSSP) results.
//
// Work of a round: the queue of vertices with pend != 0 is cut into
// descriptors of at most cgb_tuning.ms_edges edges (hub lists are spread
// over many warps); a warp takes one descriptor, reads its 32 next edges' targets and
// weights coalesced, and walks them with shuffles.
#include "mssp.cuh"

namespace cgb {

__global__ void k_mssp_init(uint32_t V, uint4* dist4, unsigned long long* pend, unsigned long long* farm)
{
    const uint64_t n4 = (uint64_t)V * (kMsRoots / 4);
    const uint4 mx = make_uint4(kValueMax, kValueMax, kValueMax, kValueMax);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += (uint64_t)gridDim.x * blockDim.x)
        dist4[i] = mx;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        pend[v] = 0;
        farm[v] = 0;
    }
}

// Roots at distance 0 and queued once each (one thread).
__global__ void k_mssp_roots(const uint32_t* roots, uint32_t n, uint32_t* dist, unsigned long long* pend, uint32_t* q,
                             MsspCounters* c)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    uint32_t len = 0;
    for (uint32_t k = 0; k < n; k++) {
        const uint32_t r = roots[k];
        dist[(size_t)r * kMsRoots + k] = 0;
        if (pend[r] == 0) q[len++] = r;
        pend[r] |= 1ull << k;
    }
    c->nq_out = len;
}

__global__ void __launch_bounds__(kBlock) k_mssp_desc(const uint32_t* __restrict__ q, const uint32_t* nq_ptr,
                                                      const uint32_t* __restrict__ off, unsigned long long* pend,
                                                      unsigned long long* maskq, uint4* desc, uint64_t cap,
                                                      MsspCounters* c, uint32_t ms_edges)
{
    mssp_desc_body(q, nq_ptr, off, pend, maskq, desc, cap, c, ms_edges);
}

template <bool kHasW>
__global__ void __launch_bounds__(kBlock) k_mssp_expand(const uint4* __restrict__ desc, const MsspCounters* cc,
                                                        const unsigned long long* __restrict__ maskq,
                                                        const uint32_t* __restrict__ dst,
                                                        const uint32_t* __restrict__ w, uint32_t* dist,
                                                        unsigned long long* pend, unsigned long long* farm,
                                                        uint32_t* qout, uint32_t* qout_len, uint32_t* far_out,
                                                        uint32_t* far_len, uint32_t cap, uint32_t thr,
                                                        const uint32_t* thr_slot, unsigned long long* alive,
                                                        MsspCounters* c)
{
    mssp_expand_body<kHasW>(desc, cc, maskq, dst, w, dist, pend, farm, qout, qout_len, far_out, far_len, cap, thr,
                            thr_slot, alive, c);
}

__global__ void __launch_bounds__(kBlock) k_mssp_split(const uint32_t* __restrict__ far_in, const uint32_t* nfar_ptr,
                                                       const uint32_t* __restrict__ dist, unsigned long long* pend,
                                                       unsigned long long* farm, uint32_t* q, uint32_t* q_len,
                                                       uint32_t* far_out, uint32_t* far_out_len, uint32_t cap,
                                                       uint32_t lo, uint32_t hi, const uint32_t* lo_slot,
                                                       const uint32_t* hi_slot, unsigned long long adv,
                                                       uint32_t* min_far_slot, unsigned long long* far_alive,
                                                       MsspCounters* c)
{
    mssp_split_body(far_in, nfar_ptr, dist, pend, farm, q, q_len, far_out, far_out_len, cap, lo, hi, lo_slot, hi_slot,
                    adv, min_far_slot, far_alive, c);
}

// dist (vertex-major, 64 slots) -> out[k * V + v] for k < n, through a
// 32-vertex x 64-root shared tile.
__global__ void __launch_bounds__(kBlock) k_mssp_out(const uint32_t* __restrict__ dist, uint32_t V, uint32_t n,
                                                     uint32_t* out)
{
    __shared__ uint32_t tile[32][kMsRoots + 1];
    const uint32_t tiles = (V + 31) / 32;
    for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        const uint32_t v0 = t * 32;
        for (uint32_t i = threadIdx.x; i < 32 * kMsRoots; i += blockDim.x) {
            const uint32_t r = i / kMsRoots, k = i % kMsRoots;
            if (v0 + r < V) tile[r][k] = dist[(size_t)(v0 + r) * kMsRoots + k];
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < 32 * n; i += blockDim.x) {
            const uint32_t k = i / 32, r = i % 32;
            if (v0 + r < V) out[(size_t)k * V + v0 + r] = tile[r][k];
        }
        __syncthreads();
    }
}

void mssp_expand(bool weighted, uint32_t grid, cudaStream_t st, const uint4* desc, const MsspCounters* cc,
                 const unsigned long long* maskq, const uint32_t* dst, const uint32_t* w, uint32_t* dist,
                 unsigned long long* pend, unsigned long long* farm, uint32_t* qout, uint32_t* qout_len,
                 uint32_t* far_out, uint32_t* far_len, uint32_t cap, uint32_t thr, const uint32_t* thr_slot,
                 unsigned long long* alive)
{
    MsspCounters* c = const_cast<MsspCounters*>(cc);
    if (weighted)
        k_mssp_expand<true><<<grid, kBlock, 0, st>>>(desc, cc, maskq, dst, w, dist, pend, farm, qout, qout_len, far_out,
                                                     far_len, cap, thr, thr_slot, alive, c);
    else
        k_mssp_expand<false><<<grid, kBlock, 0, st>>>(desc, cc, maskq, dst, w, dist, pend, farm, qout, qout_len,
                                                      far_out, far_len, cap, thr, thr_slot, alive, c);
    CGB_CUDA_TRY(cudaGetLastError());
}

MsspBuffers* mssp_buffers_alloc(uint32_t V, uint64_t E)
{
    auto* b = new MsspBuffers();
    try {
        CGB_CUDA_TRY(cudaMalloc((void**)&b->dist, (size_t)V * kMsRoots * 4));
        CGB_CUDA_TRY(cudaMalloc((void**)&b->pend, (size_t)V * 8));
        CGB_CUDA_TRY(cudaMalloc((void**)&b->farm, (size_t)V * 8));
        CGB_CUDA_TRY(cudaMalloc((void**)&b->maskq, (size_t)V * 8));
        CGB_CUDA_TRY(cudaMalloc((void**)&b->far_list[0], (size_t)V * 4));
        CGB_CUDA_TRY(cudaMalloc((void**)&b->far_list[1], (size_t)V * 4));
        b->desc_cap = (uint64_t)V + E / kMinMsEdges + 1;  // any descriptor size cgb_tuning_set allows
        CGB_CUDA_TRY(cudaMalloc((void**)&b->desc, b->desc_cap * sizeof(uint4)));
        CGB_CUDA_TRY(cudaMalloc((void**)&b->c, sizeof(MsspCounters)));
        CGB_CUDA_TRY(cudaMallocHost((void**)&b->h, sizeof(MsspCounters)));
    } catch (...) {
        mssp_buffers_free(b);
        throw;
    }
    return b;
}

void mssp_buffers_free(MsspBuffers* b)
{
    if (!b) return;
    cudaFree(b->dist);
    cudaFree(b->pend);
    cudaFree(b->farm);
    cudaFree(b->maskq);
    cudaFree(b->far_list[0]);
    cudaFree(b->far_list[1]);
    cudaFree(b->desc);
    cudaFree(b->c);
    if (b->h) cudaFreeHost(b->h);
    delete b;
}

static void mssp_alloc(cgb_graph* g)
{
    if (!g->mssp) g->mssp = mssp_buffers_alloc(g->V, g->E);
}

void free_mssp(cgb_graph* g)
{
    mssp_buffers_free(g->mssp);
    g->mssp = nullptr;
}

static MsspCounters mssp_sync(cgb_graph* g)
{
    MsspBuffers& b = *g->mssp;
    CGB_CUDA_TRY(cudaMemcpyAsync(b.h, b.c, sizeof(MsspCounters), cudaMemcpyDeviceToHost, g->stream));
    CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    CGB_REQUIRE(!b.h->overflow, CGB_EOVERFLOW, "multi-root SSSP queue overflow");
    return *b.h;
}

__global__ void k_mssp_set(uint32_t* a, uint32_t value) { *a = value; }

uint32_t mssp_default_delta(cgb_graph* g)
{
    if (g->w && g->sum_w == 0) compute_weight_sum(g);
    // a round serves up to 64 roots (on RMAT-22/24 its rounds stop shrinking
    // beyond 64 x the unit); at least 8
    return std::max<uint32_t>(8u, sssp_delta_for(g, 64.0));
}

void run_mssp(cgb_graph* g, const uint32_t* d_roots, uint32_t n, uint32_t* out, uint32_t delta)
{
    CGB_REQUIRE(n >= 1 && n <= kMsRoots, CGB_EINVAL, "multi-root SSSP takes 1..64 roots per pass");
    ensure_frontier(g);
    mssp_alloc(g);
    MsspBuffers& b = *g->mssp;
    const uint32_t V = g->V;
    if (delta == 0) delta = 1;
    CGB_CUDA_TRY(cudaMemsetAsync(b.c, 0, sizeof(MsspCounters), g->stream));
    ++g->stats.launches;
    k_mssp_init<<<num_sms() * 8, kBlock, 0, g->stream>>>(V, reinterpret_cast<uint4*>(b.dist), b.pend, b.farm);
    ++g->stats.launches;
    k_mssp_roots<<<1, 1, 0, g->stream>>>(d_roots, n, b.dist, b.pend, g->q[0], b.c);
    uint32_t nq = mssp_sync(g).nq_out, nfar = 0;
    CGB_CUDA_TRY(cudaMemcpyAsync(&b.c->nq_in, &b.c->nq_out, 4, cudaMemcpyDeviceToDevice, g->stream));
    int cur = 0, fcur = 0;  // near queue / far list holding the live entries
    uint64_t thr = delta;
    bool last_split_empty = false;
    uint32_t min_far = kValueMax;
    uint64_t rounds = 0;
    while (nq > 0 || nfar > 0) {
        CGB_REQUIRE(++rounds <= 4ull * V + 64, CGB_ETIMEOUT, "multi-root SSSP round bound exceeded");
        const int nxt = cur ^ 1;
        CGB_CUDA_TRY(cudaMemsetAsync(&b.c->nq_out, 0, 4, g->stream));
        if (nq > 0) {
            // near round at threshold thr: q[cur] -> q[nxt]
            const uint32_t t32 = (uint32_t)std::min<uint64_t>(thr, 0xFFFFFFFFull);
            CGB_CUDA_TRY(cudaMemsetAsync(&b.c->ndesc, 0, 4, g->stream));
            ++g->stats.launches;
            k_mssp_desc<<<grid_for(nq, kBlock, num_sms() * 8), kBlock, 0, g->stream>>>(g->q[cur], &b.c->nq_in, g->off,
                                                                                    b.pend, b.maskq, b.desc,
                                                                                    b.desc_cap, b.c,
                                                                                    g->tune.ms_edges);
            ++g->stats.launches;
            mssp_expand(g->w != nullptr, num_sms() * 8, g->stream, b.desc, b.c, b.maskq, g->dst, g->w, b.dist, b.pend,
                        b.farm, g->q[nxt], &b.c->nq_out, b.far_list[fcur], &b.c->nfar_live, V, t32, nullptr,
                        nullptr);
            const MsspCounters h = mssp_sync(g);
            nq = h.nq_out;
            nfar = h.nfar_live;
            last_split_empty = false;
            g->stats.pushes_td++;
        } else {
            // split of the far list at the next bucket [thr, hi): far_list[fcur] -> q[nxt] + far_list[fcur ^ 1]
            uint64_t hi = thr + delta;
            if (last_split_empty && min_far != kValueMax)
                hi = std::max<uint64_t>(hi, ((uint64_t)min_far / delta + 1) * delta);
            const uint32_t lo32 = (uint32_t)std::min<uint64_t>(thr, 0xFFFFFFFFull);
            const uint32_t hi32 = (uint32_t)std::min<uint64_t>(hi, 0xFFFFFFFFull);
            k_mssp_set<<<1, 1, 0, g->stream>>>(&b.c->min_far, kValueMax);
            CGB_CUDA_TRY(cudaMemsetAsync(&b.c->nfar_next, 0, 4, g->stream));
            ++g->stats.launches;
            k_mssp_split<<<grid_for(nfar, kBlock / 32, num_sms() * 8), kBlock, 0, g->stream>>>(
                b.far_list[fcur], &b.c->nfar_live, b.dist, b.pend, b.farm, g->q[nxt], &b.c->nq_out,
                b.far_list[fcur ^ 1], &b.c->nfar_next, V, lo32, hi32, nullptr, nullptr, ~0ull, nullptr, nullptr, b.c);
            const MsspCounters h = mssp_sync(g);
            nq = h.nq_out;
            nfar = h.nfar_next;
            min_far = h.min_far;
            fcur ^= 1;
            k_mssp_set<<<1, 1, 0, g->stream>>>(&b.c->nfar_live, nfar);
            thr = hi;
            last_split_empty = nq == 0;
        }
        cur = nxt;
        CGB_CUDA_TRY(cudaMemcpyAsync(&b.c->nq_in, &b.c->nq_out, 4, cudaMemcpyDeviceToDevice, g->stream));
    }
    ++g->stats.launches;
    k_mssp_out<<<num_sms() * 16, kBlock, 0, g->stream>>>(b.dist, V, n, out);
    g->stats.iterations = rounds;
    g->stats.sssp_delta = delta;
}

}  // namespace cgb
