// Pull-based FP64 PageRank.
//
// The reference's formula (my_project/CGgraph/GraphNuma.cuh:233-244,545-554,
// device_algorithm.cuh:538-545): pr0 = 1/N and per iteration
//     pr'[v] = 0.15/N + 0.85 * sum_{u -> v} pr[u] / outdeg[u],
// with no redistribution of dangling mass.  The reference evaluates it by
// pushing in uint32 (so every value truncates to 0) into the wrong slot; this
// engine evaluates the formula in FP64 by pulling over the in-edge CSC, which
// needs no atomics and gives the same result on every run.
//
// Layout (built once per graph, graph.cu ensure_pr): vertices are relabelled
// by a stable sort on (out-degree bucket floor(log2 outdeg), largest first
// and zero out-degree last; then in-degree, largest first).  Every
// contribution that is ever gathered (vertices with out-edges) then lies in
// one dense prefix of contrib[] (RMAT-24: 7.4 M of 16.8 M vertices, 59 MB,
// L2-resident), and consecutive rows have nearly equal in-degrees.  Rows are
// the relabelled vertices in order, so pr'/contrib' writes are coalesced;
// one last pass maps the result back to the caller's vertex ids.
//
// One launch of k_pr_pull per iteration reads contrib[u] = pr[u]/outdeg[u]
// of the previous iteration and writes pr' and contrib' (the division is
// fused into the epilogue).  Rows below kPrHuge in-edges are stored as a
// sliced ELL (SELL-32: 32 consecutive rows per slice, edge j of lane l at
// slice base + 32j + l, padded to the slice's longest row); ordering rows by
// in-degree inside each out-degree bucket keeps the padding under 1 % on
// RMAT.  A warp sums one slice, one row per lane (k_pr_pull).  Rows of
// kPrHuge or more in-edges are cut into kPrChunk-edge chunks summed by
// separate CTAs (k_pr_hub_chunks, on a second stream beside the pull) and
// combined in chunk order (k_pr_hub_finish).
// Every summation order is fixed by the graph alone, so results are
// bit-reproducible.
#include "engine.cuh"

namespace cgb {

__global__ void k_pr_init(uint32_t V, const uint32_t* __restrict__ outdeg, double* pr, double* contrib)
{
    const double p0 = 1.0 / (double)V;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        const uint32_t deg = outdeg[v];
        pr[v] = p0;
        contrib[v] = deg ? p0 / (double)deg : 0.0;
    }
}

// On skewed graphs (kHint) the gathers of the hottest contributions carry an
// L2 evict-last policy and the rest evict-first.  The layout puts vertices in
// descending out-degree buckets, so contributions [0, kPrHot) are the most
// gathered ones; 6.5 M doubles (52 MB) stay in L2 beside the streamed column
// indices while the long tail passes through (Chung-Lu, 330 MB of
// contributions: 7.3 -> 6.8 ms per iteration; RMAT-24: 0.847 -> 0.817 ms;
// same results).  Graphs without hubs (meshes) keep plain loads: their
// contributions are reused by nearby rows, which evict-first cut short (the
// 4800 x 5000 grid: 6.5 -> 7.5 ms per run with the hints).
constexpr uint32_t kPrHot = 6500000;
constexpr uint32_t kPrHintMinDeg = 64;  // largest out-degree from which a graph counts as skewed

__device__ __forceinline__ double ld_f64_l2hint(const double* p, uint64_t policy)
{
    double v;
    asm volatile("ld.global.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(policy));
    return v;
}

// One warp per 32-row slice of the sliced ELL: in step j every lane loads
// its row's j-th source (one coalesced 128-byte load per warp) and gathers
// that contribution; kU steps (cgb_tuning.pr_unroll) are issued before they
// are summed, in j order, so each lane keeps kU gathers in flight.  Padding slots name
// vertex V, whose contribution is 0.  Hub rows (bit set in hub_bm) are
// finished by k_pr_hub_finish.  The slice stream and the outputs use
// evict-first accesses so that L2 keeps the gathered contributions.
template <int kU, bool kHint>
__global__ void __launch_bounds__(kBlock) k_pr_pull(uint32_t V, const uint64_t* __restrict__ slice_ptr,
                                                    const uint32_t* __restrict__ slice_len,
                                                    const uint32_t* __restrict__ col,
                                                    const uint32_t* __restrict__ hub_bm,
                                                    const uint32_t* __restrict__ outdeg,
                                                    const double* __restrict__ contrib, double* __restrict__ pr_out,
                                                    double* __restrict__ contrib_out, double base, double damp)
{
    const uint32_t lane = lane_id();
    const uint32_t nslices = (V + 31) / 32;
    const uint32_t nwarps = gridDim.x * (kBlock / 32);
    uint64_t pol_hot, pol_cold;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol_hot));
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol_cold));
    for (uint32_t s = blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5); s < nslices; s += nwarps) {
        const uint32_t len = slice_len[s];
        const uint32_t* c = col + slice_ptr[s] + lane;
        double acc = 0.0;
        // kU steps per batch: all their gathers in flight, then summed in
        // step order; the last batch is predicated (masked steps add
        // contrib[V] = +0.0, which leaves the sum and its order unchanged)
        for (uint32_t j = 0; j < len; j += kU) {
            uint32_t u[kU];
#pragma unroll
            for (int t = 0; t < kU; t++) u[t] = j + t < len ? __ldcs(c + 32u * (j + t)) : V;  // read once
            double x[kU];
#pragma unroll
            for (int t = 0; t < kU; t++)
                x[t] = kHint ? ld_f64_l2hint(contrib + u[t], u[t] < kPrHot ? pol_hot : pol_cold) : contrib[u[t]];
#pragma unroll
            for (int t = 0; t < kU; t++) acc += x[t];
        }
        const uint32_t r = s * 32 + lane;
        const bool hub = (hub_bm[s] >> lane) & 1u;
        if (r < V && !hub) {
            const double p = base + damp * acc;
            const uint32_t od = __ldcs(outdeg + r);
            __stcs(pr_out + r, p);  // not read again this iteration: keep L2 for the gathers
            __stcs(contrib_out + r, od ? p / (double)od : 0.0);
        }
    }
}

// One CTA per kPrChunk-edge chunk of a hub row: fixed-order partial sum.
__global__ void __launch_bounds__(kBlock) k_pr_hub_chunks(const uint2* __restrict__ chunks, uint32_t n,
                                                          const uint32_t* __restrict__ in_off,
                                                          const uint32_t* __restrict__ in_src,
                                                          const double* __restrict__ contrib, double* part)
{
    __shared__ double s_part[kBlock / 32];
    for (uint32_t c = blockIdx.x; c < n; c += gridDim.x) {
        const uint2 ch = chunks[c];
        const uint32_t e1 = min(in_off[ch.x + 1], ch.y + kPrChunk);
        double sum = 0.0;
        uint32_t k = ch.y + threadIdx.x;
        for (; k + 3 * kBlock < e1; k += 4 * kBlock) {
            const uint32_t u0 = in_src[k], u1 = in_src[k + kBlock];
            const uint32_t u2 = in_src[k + 2 * kBlock], u3 = in_src[k + 3 * kBlock];
            const double c0 = contrib[u0], c1 = contrib[u1], c2 = contrib[u2], c3 = contrib[u3];
            sum += c0;
            sum += c1;
            sum += c2;
            sum += c3;
        }
        for (; k < e1; k += kBlock) sum += contrib[in_src[k]];
        sum = warp_sum(sum);
        if (lane_id() == 0) s_part[threadIdx.x >> 5] = sum;
        __syncthreads();
        if (threadIdx.x < 32) {
            double t = threadIdx.x < kBlock / 32 ? s_part[threadIdx.x] : 0.0;
            t = warp_sum(t);
            if (threadIdx.x == 0) part[c] = t;
        }
        __syncthreads();
    }
}

// Hub rows: sum their chunk partials in chunk order, then the epilogue.
__global__ void k_pr_hub_finish(const uint32_t* __restrict__ rows, uint32_t n, const uint32_t* __restrict__ base_idx,
                                const double* __restrict__ part, const uint32_t* __restrict__ outdeg, double* pr_out,
                                double* contrib_out, double base, double damp)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double t = 0.0;
        for (uint32_t c = base_idx[i]; c < base_idx[i + 1]; c++) t += part[c];
        const uint32_t r = rows[i];
        const double p = base + damp * t;
        const uint32_t od = outdeg[r];
        pr_out[r] = p;
        contrib_out[r] = od ? p / (double)od : 0.0;
    }
}

// Back to the caller's vertex ids: out[v] = pr[rank[v]].
__global__ void k_pr_unpermute(uint32_t V, const uint32_t* __restrict__ rank, const double* __restrict__ pr,
                               double* out)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) out[v] = pr[rank[v]];
}

void run_pr(cgb_graph* g, uint32_t iters, const cgb_options& o)
{
    (void)o;
    ensure_pr(g);
    ensure_max_degree(g);
    const bool timing = g->flags & CGB_FLAG_KERNEL_TIMING;
    const uint32_t V = g->V;
    const double base = 0.15 / (double)V;
    const double damp = 0.85;
    if (iters == 0) iters = 1;  // graphProcess_device runs at least one iteration
    CGB_CUDA_TRY(cudaEventRecord(g->ev_start, g->stream));
    if (timing) ktimer_begin(g, CGB_K_INIT);
    ++g->stats.launches;
    k_pr_init<<<grid_for(V, kBlock, num_sms() * 8), kBlock, 0, g->stream>>>(V, g->pr_outdeg, g->pr[0], g->contrib[0]);
    if (timing) ktimer_end(g);
    const uint32_t grid = grid_for(div_up(V, 32), kBlock / 32, num_sms() * g->tune.pr_ctas_per_sm);
    const uint32_t unroll = g->tune.pr_unroll;
    // hub chunks on a second stream, beside the pull (they read the same
    // contributions and write only the chunk partials); joined before the
    // hub rows are finished
    const bool fork = g->n_pr_chunks > 0;
    if (fork && !g->aux_stream) {
        CGB_CUDA_TRY(cudaStreamCreateWithFlags(&g->aux_stream, cudaStreamNonBlocking));
        CGB_CUDA_TRY(cudaEventCreateWithFlags(&g->ev_fork, cudaEventDisableTiming));
        CGB_CUDA_TRY(cudaEventCreateWithFlags(&g->ev_join, cudaEventDisableTiming));
    }
    int cur = 0;
    for (uint32_t it = 0; it < iters; it++) {
        const int out = cur ^ 1;
        if (timing) ktimer_begin(g, CGB_K_PR);
        if (fork) {
            ++g->stats.launches;
            CGB_CUDA_TRY(cudaEventRecord(g->ev_fork, g->stream));
            CGB_CUDA_TRY(cudaStreamWaitEvent(g->aux_stream, g->ev_fork, 0));
            k_pr_hub_chunks<<<std::min<uint32_t>(g->n_pr_chunks, num_sms() * 8), kBlock, 0, g->aux_stream>>>(
                g->pr_chunks, g->n_pr_chunks, g->pr_off, g->pr_src, g->contrib[cur], g->pr_part);
            CGB_CUDA_TRY(cudaEventRecord(g->ev_join, g->aux_stream));
        }
        ++g->stats.launches;
        const bool hint = g->max_degree >= kPrHintMinDeg;
        auto pull = unroll == 4 ? (hint ? k_pr_pull<4, true> : k_pr_pull<4, false>)
                    : unroll == 16 ? (hint ? k_pr_pull<16, true> : k_pr_pull<16, false>)
                                   : (hint ? k_pr_pull<8, true> : k_pr_pull<8, false>);
        pull<<<grid, kBlock, 0, g->stream>>>(V, g->pr_slice_ptr, g->pr_slice_len, g->pr_col, g->pr_hub_bm,
                                             g->pr_outdeg, g->contrib[cur], g->pr[out], g->contrib[out], base, damp);
        if (fork) CGB_CUDA_TRY(cudaStreamWaitEvent(g->stream, g->ev_join, 0));
        if (g->n_pr_huge) {
            ++g->stats.launches;
            k_pr_hub_finish<<<grid_for(g->n_pr_huge, kBlock, num_sms()), kBlock, 0, g->stream>>>(
                g->pr_huge_rows, g->n_pr_huge, g->pr_chunk_base, g->pr_part, g->pr_outdeg, g->pr[out],
                g->contrib[out], base, damp);
        }
        if (timing) ktimer_end(g);
        cur = out;
    }
    // the other pr buffer receives the result in the caller's ids
    ++g->stats.launches;
    k_pr_unpermute<<<grid_for(V, kBlock, num_sms() * 8), kBlock, 0, g->stream>>>(V, g->pr_rank, g->pr[cur],
                                                                               g->pr[cur ^ 1]);
    CGB_CUDA_TRY(cudaEventRecord(g->ev_stop, g->stream));
    g->result = g->pr[cur ^ 1];
    g->stats.iterations = iters;
}

}  // namespace cgb
