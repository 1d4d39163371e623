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
// One launch per iteration reads contrib[u] = pr[u]/outdeg[u] of the previous
// iteration and writes both pr' and contrib' (the division is fused into the
// epilogue), so an iteration streams in_src (4 B/edge), gathers contrib
// (8 B/edge), and writes 16 B/vertex.
//
// Work split (rows = destination vertices, in natural order so pr' writes are
// coalesced): a warp owns 32 consecutive rows.
//   in-degree >= kPrHuge      a whole CTA per row, in k_pr_huge_rows;
//   32 <= in-degree < kPrHuge the warp walks the row (ballot election) and
//                             reduces with a fixed shuffle tree;
//   in-degree < 32            the warp gathers the concatenated short rows 32
//                             edges at a time: each lane finds its row by a
//                             5-step shuffle binary search over the warp's
//                             inclusive degree scan, then a segmented shuffle
//                             scan sums each row's run and the run's last lane
//                             adds it to the row's shared-memory accumulator.
// Every reduction order is fixed by the graph alone, so results are
// bit-reproducible.
#include "engine.cuh"

namespace cgb {

__global__ void k_pr_init(uint32_t V, const uint32_t* __restrict__ off, double* pr, double* contrib)
{
    const double p0 = 1.0 / (double)V;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        const uint32_t deg = off[v + 1] - off[v];
        pr[v] = p0;
        contrib[v] = deg ? p0 / (double)deg : 0.0;
    }
}

__device__ __forceinline__ double shfl_d(double x, int src)
{
    return __shfl_sync(0xffffffffu, x, src);
}

__global__ void __launch_bounds__(kBlock) k_pr_pull(uint32_t V, const uint32_t* __restrict__ in_off,
                                                    const uint32_t* __restrict__ in_src,
                                                    const uint32_t* __restrict__ off,
                                                    const double* __restrict__ contrib, double* __restrict__ pr_out,
                                                    double* __restrict__ contrib_out, double base, double damp)
{
    __shared__ double s_acc[kBlock];
    const uint32_t lane = lane_id();
    const uint32_t wib = threadIdx.x >> 5;
    double* acc_w = s_acc + wib * 32;
    const uint32_t nwarps = gridDim.x * (kBlock / 32);
    for (uint32_t grp = blockIdx.x * (kBlock / 32) + wib; grp * 32u < V; grp += nwarps) {
        const uint32_t r = grp * 32 + lane;
        uint32_t s = 0, d = 0;
        if (r < V) {
            s = in_off[r];
            d = in_off[r + 1] - s;
        }
        double acc = 0.0;
        // long rows, one at a time
        uint32_t lmask = __ballot_sync(0xffffffffu, d >= 32 && d < kPrHuge);
        while (lmask) {
            const uint32_t leader = __ffs(lmask) - 1;
            lmask &= lmask - 1;
            const uint32_t st = __shfl_sync(0xffffffffu, s, leader);
            const uint32_t dg = __shfl_sync(0xffffffffu, d, leader);
            double sum = 0.0;
            for (uint32_t k = lane; k < dg; k += 32) sum += contrib[in_src[st + k]];
            sum = warp_sum(sum);
            if (lane == leader) acc = sum;
        }
        // short rows, segmented
        const uint32_t sd = d < 32 ? d : 0;
        const uint32_t incl = warp_incl_scan(sd);
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        acc_w[lane] = 0.0;
        __syncwarp();
        for (uint32_t base_k = 0; base_k < total; base_k += 32) {
            const uint32_t k = base_k + lane;
            const bool valid = k < total;
            // owner = number of lanes whose inclusive scan is <= k
            uint32_t j = 0;
#pragma unroll
            for (uint32_t b = 16; b > 0; b >>= 1) {
                const uint32_t probe = __shfl_sync(0xffffffffu, incl, j + b - 1);
                if (probe <= k) j += b;
            }
            const uint32_t own_incl = __shfl_sync(0xffffffffu, incl, j);
            const uint32_t own_sd = __shfl_sync(0xffffffffu, sd, j);
            const uint32_t own_s = __shfl_sync(0xffffffffu, s, j);
            double val = 0.0;
            if (valid) val = contrib[in_src[own_s + (k - (own_incl - own_sd))]];
            // segmented inclusive scan over runs of equal owner
#pragma unroll
            for (uint32_t o = 1; o < 32; o <<= 1) {
                const double nv = shfl_d(val, (int)(lane >= o ? lane - o : lane));
                const uint32_t no = __shfl_sync(0xffffffffu, j, lane >= o ? lane - o : lane);
                if (lane >= o && no == j) val += nv;
            }
            const uint32_t next_j = __shfl_sync(0xffffffffu, j, lane < 31 ? lane + 1 : lane);
            const bool next_valid = __shfl_sync(0xffffffffu, (uint32_t)valid, lane < 31 ? lane + 1 : lane);
            const bool tail = valid && (lane == 31 || !next_valid || next_j != j);
            if (tail) acc_w[j] += val;
            __syncwarp();
        }
        if (sd) acc = acc_w[lane];
        __syncwarp();
        if (r < V && d < kPrHuge) {
            const double p = base + damp * acc;
            const uint32_t od = off[r + 1] - off[r];
            pr_out[r] = p;
            contrib_out[r] = od ? p / (double)od : 0.0;
        }
    }
}

// Rows with in-degree >= kPrHuge: one CTA per row, fixed reduction tree.
__global__ void __launch_bounds__(kBlock) k_pr_huge_rows(const uint32_t* __restrict__ rows, uint32_t n,
                                                         const uint32_t* __restrict__ in_off,
                                                         const uint32_t* __restrict__ in_src,
                                                         const uint32_t* __restrict__ off,
                                                         const double* __restrict__ contrib, double* pr_out,
                                                         double* contrib_out, double base, double damp)
{
    __shared__ double s_part[kBlock / 32];
    for (uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
        const uint32_t r = rows[i];
        const uint32_t s = in_off[r], e = in_off[r + 1];
        double sum = 0.0;
        for (uint32_t k = s + threadIdx.x; k < e; k += kBlock) sum += contrib[in_src[k]];
        sum = warp_sum(sum);
        if (lane_id() == 0) s_part[threadIdx.x >> 5] = sum;
        __syncthreads();
        if (threadIdx.x < 32) {
            double t = threadIdx.x < kBlock / 32 ? s_part[threadIdx.x] : 0.0;
            t = warp_sum(t);
            if (threadIdx.x == 0) {
                const double p = base + damp * t;
                const uint32_t od = off[r + 1] - off[r];
                pr_out[r] = p;
                contrib_out[r] = od ? p / (double)od : 0.0;
            }
        }
        __syncthreads();
    }
}

void run_pr(cgb_graph* g, uint32_t iters, const cgb_options& o)
{
    (void)o;
    ensure_pr(g);
    const bool timing = g->flags & CGB_FLAG_KERNEL_TIMING;
    const uint32_t V = g->V;
    const double base = 0.15 / (double)V;
    const double damp = 0.85;
    if (iters == 0) iters = 1;  // graphProcess_device runs at least one iteration
    CGB_CUDA_TRY(cudaEventRecord(g->ev_start, g->stream));
    if (timing) ktimer_begin(g, CGB_K_INIT);
    ++g->stats.launches;
    k_pr_init<<<grid_for(V, kBlock, kNumSMs * 8), kBlock, 0, g->stream>>>(V, g->off, g->pr[0], g->contrib[0]);
    if (timing) ktimer_end(g);
    const uint32_t grid = grid_for(div_up(V, 32), kBlock / 32, kNumSMs * 16);
    int cur = 0;
    for (uint32_t it = 0; it < iters; it++) {
        const int out = cur ^ 1;
        if (timing) ktimer_begin(g, CGB_K_PR);
        ++g->stats.launches;
        k_pr_pull<<<grid, kBlock, 0, g->stream>>>(V, g->in_off, g->in_src, g->off, g->contrib[cur], g->pr[out],
                                                  g->contrib[out], base, damp);
        if (g->n_pr_huge) {
            ++g->stats.launches;
            k_pr_huge_rows<<<std::min<uint32_t>(g->n_pr_huge, kNumSMs * 8), kBlock, 0, g->stream>>>(
                g->pr_huge_rows, g->n_pr_huge, g->in_off, g->in_src, g->off, g->contrib[cur], g->pr[out],
                g->contrib[out], base, damp);
        }
        if (timing) ktimer_end(g);
        cur = out;
    }
    CGB_CUDA_TRY(cudaEventRecord(g->ev_stop, g->stream));
    g->result = g->pr[cur];
    g->stats.iterations = iters;
}

}  // namespace cgb
