// Delta-stepping SSSP (near/far piles) with atomicMin relaxation.
//
// Result semantics follow the reference's SSSP: dist[root] = 0, relaxation
// dist[d] = min(dist[d], dist[u] + w) applied only when it lowers the value
// (my_project/CGgraph/device_algorithm.cuh:293-329, host_algorithm.hpp:277-300),
// unreachable vertices keep 999999999; a candidate >= 999999999 never lowers
// a value, exactly as in the reference's uint32 comparison.  The reference
// re-relaxes Bellman-Ford style from a worklist; any order of monotone
// atomicMin relaxations reaches the same fixpoint, so the result is
// bit-identical.
//
// Schedule: vertices whose tentative distance is below the current threshold
// form the near queue, which is expanded round after round with the
// degree-binned push of push.cuh; improvements at or above the threshold go
// to the far pile as (vertex, distance) pairs.  When the near queue empties
// the threshold advances by delta and the far pile is split: entries whose
// distance is stale are dropped, those below the new threshold become the
// near queue.  A per-vertex stamp keeps each vertex at most once per round.
#include "engine.cuh"
#include "policy.cuh"
#include "push.cuh"

namespace cgb {

template <bool kHasW>
struct SsspOp {
    const uint32_t* __restrict__ off;
    const uint32_t* __restrict__ dst;
    const uint32_t* __restrict__ w;
    uint32_t* dist;
    uint32_t* stamp;
    uint32_t it;
    uint32_t thr;
    uint32_t nz;
    uint32_t* near_out;
    uint32_t* near_len;
    uint32_t cap;
    uint2* far_out;
    uint32_t* far_len;
    uint32_t far_cap;
    DevCounters* ctr;

    __device__ __forceinline__ bool load(uint32_t v, uint32_t& s, uint32_t& d, uint32_t& m) const
    {
        s = off[v];
        d = off[v + 1] - s;
        m = dist[v];
        return m < kValueMax;
    }
    __device__ __forceinline__ void edge(bool valid, uint32_t e, uint32_t du) const
    {
        bool to_near = false, to_far = false;
        uint32_t d = 0, nd = 0;
        if (valid) {
            d = dst[e];
            const uint64_t cand = (uint64_t)du + (kHasW ? (uint64_t)w[e] : 1ull);
            if (cand < kValueMax) {
                nd = (uint32_t)cand;
                if (nd < dist[d]) {
                    const uint32_t old = atomicMin(dist + d, nd);
                    if (nd < old && d < nz) {
                        if (nd < thr) to_near = atomicExch(stamp + d, it) != it;
                        else to_far = true;
                    }
                }
            }
        }
        warp_append(to_near, d, near_out, near_len, cap, &ctr->overflow);
        warp_append2(to_far, make_uint2(d, nd), far_out, far_len, far_cap, &ctr->overflow);
    }
};

__global__ void k_sssp_init(uint32_t V, uint32_t* dist, uint32_t* stamp)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) {
        dist[i] = kValueMax;
        stamp[i] = 0;
    }
}

__global__ void k_sssp_root(uint32_t* dist, uint32_t root, uint32_t* q0)
{
    dist[root] = 0;
    q0[0] = root;
}

// Splits the far pile at threshold thr (see file comment).
__global__ void __launch_bounds__(kBlock) k_sssp_split(const uint2* __restrict__ far_in, uint32_t n,
                                                       const uint32_t* dist, uint32_t thr, uint32_t* stamp,
                                                       uint32_t it, uint32_t* near_out, uint32_t* near_len,
                                                       uint32_t cap, uint2* far_out, uint32_t* far_len,
                                                       uint32_t far_cap, DevCounters* ctr)
{
    uint32_t mn = kValueMax;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t n_round = (n + 31u) & ~31u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_round; i += stride) {
        bool to_near = false, to_far = false;
        uint2 ent = make_uint2(0, 0);
        if (i < n) {
            ent = far_in[i];
            if (dist[ent.x] == ent.y) {
                if (ent.y < thr) to_near = atomicExch(stamp + ent.x, it) != it;
                else {
                    to_far = true;
                    mn = min(mn, ent.y);
                }
            }
        }
        warp_append(to_near, ent.x, near_out, near_len, cap, &ctr->overflow);
        warp_append2(to_far, ent, far_out, far_len, far_cap, &ctr->overflow);
    }
    mn = __reduce_min_sync(0xffffffffu, mn);
    if (lane_id() == 0 && mn != kValueMax) atomicMin(&ctr->min_far, mn);
}

template <bool kHasW>
static void sssp_loop(cgb_graph* g, uint32_t root, uint32_t delta, const cgb_options& o)
{
    const bool timing = g->flags & CGB_FLAG_KERNEL_TIMING;
    const bool tracing = g->flags & CGB_FLAG_TRACE;
    const uint32_t V = g->V;
    const uint64_t max_iters = o.max_iterations ? o.max_iterations : ~0ull;
    Policy* pol = (o.schedule == CGB_SCHED_LEARNED) ? policy_get() : nullptr;
    const uint32_t base_delta = delta;

    CGB_CUDA_TRY(cudaEventRecord(g->ev_start, g->stream));
    if (timing) ktimer_begin(g, CGB_K_INIT);
    ++g->stats.launches;
    k_sssp_init<<<kNumSMs * 4, kBlock, 0, g->stream>>>(V, g->value, g->stamp);
    ++g->stats.launches;
    k_sssp_root<<<1, 1, 0, g->stream>>>(g->value, root, g->q[0]);
    CGB_CUDA_TRY(cudaMemsetAsync(g->ctr, 0, sizeof(DevCounters), g->stream));
    if (timing) ktimer_end(g);

    int cur = 0, fcur = 0;
    uint64_t nnear = root < g->nz ? 1 : 0;
    uint64_t nfar = 0;
    uint64_t thr = delta;
    uint32_t it = 1;
    uint64_t iters = 0;
    uint64_t settled_guess = 0;

    for (;;) {
        while (nnear > 0) {
            CGB_REQUIRE(iters < max_iters, CGB_ETIMEOUT, "SSSP iteration budget exhausted");
            it++;
            const int out = cur ^ 1;
            CGB_CUDA_TRY(cudaMemsetAsync(&g->ctr->qlen[out], 0, sizeof(uint32_t), g->stream));
            CGB_CUDA_TRY(cudaMemsetAsync(&g->ctr->huge_len, 0, sizeof(uint32_t), g->stream));
            if (tracing) CGB_CUDA_TRY(cudaEventRecord(g->ev_iter[0], g->stream));
            if (timing) ktimer_begin(g, CGB_K_PUSH);
            SsspOp<kHasW> op{g->off, g->dst, g->w, g->value, g->stamp, it, (uint32_t)std::min<uint64_t>(thr, kValueMax),
                             g->nz, g->q[out], &g->ctr->qlen[out], V, g->far[fcur], &g->ctr->far_len[fcur],
                             g->far_cap, g->ctr};
            launch_push_twc(g, g->q[cur], (uint32_t)nnear, op, false);
            if (timing) ktimer_end(g);
            if (tracing) CGB_CUDA_TRY(cudaEventRecord(g->ev_iter[1], g->stream));
            sync_counters(g);
            CGB_REQUIRE(!g->h_ctr->overflow, CGB_EOVERFLOW, "SSSP queue overflow");
            if (tracing) {
                float ms = 0.f;
                CGB_CUDA_TRY(cudaEventElapsedTime(&ms, g->ev_iter[0], g->ev_iter[1]));
                cgb_iter_trace t{};
                t.iteration = (uint32_t)iters;
                t.algorithm = CGB_SSSP;
                t.frontier_vertices = nnear;
                t.unvisited_vertices = nfar;
                t.variant = CGB_VAR_TWC;
                t.delta = delta;
                t.ms = ms;
                g->trace.push_back(t);
            }
            settled_guess += nnear;
            nnear = g->h_ctr->qlen[out];
            nfar = g->h_ctr->far_len[fcur];
            cur = out;
            iters++;
        }
        if (nfar == 0) break;
        if (pol) {
            float feat[kPolicyFeatures];
            policy_features(feat, CGB_SSSP, g, nnear, 0, (uint64_t)V - std::min<uint64_t>(settled_guess, V), nfar, 0,
                            (uint32_t)iters, 0, delta);
            const int k = policy_choose_delta(pol, feat);
            if (k >= 0) {
                static const float scale[5] = {0.25f, 0.5f, 1.f, 2.f, 4.f};
                delta = std::max<uint32_t>(1u, (uint32_t)(base_delta * scale[k]));
            }
        }
        thr += delta;
        // split the far pile until the near queue is non-empty or the pile is gone
        for (;;) {
            CGB_REQUIRE(iters < max_iters, CGB_ETIMEOUT, "SSSP iteration budget exhausted");
            it++;
            const int out = cur ^ 1;
            const int fout = fcur ^ 1;
            CGB_CUDA_TRY(cudaMemsetAsync(&g->ctr->qlen[out], 0, sizeof(uint32_t), g->stream));
            CGB_CUDA_TRY(cudaMemsetAsync(&g->ctr->far_len[fout], 0, sizeof(uint32_t), g->stream));
            CGB_CUDA_TRY(cudaMemsetAsync(&g->ctr->min_far, 0xff, sizeof(uint32_t), g->stream));
            if (timing) ktimer_begin(g, CGB_K_FRONTIER);
            ++g->stats.launches;
            k_sssp_split<<<grid_for(nfar, kBlock, kNumSMs * 8), kBlock, 0, g->stream>>>(
                g->far[fcur], (uint32_t)nfar, g->value, (uint32_t)std::min<uint64_t>(thr, kValueMax), g->stamp, it,
                g->q[out], &g->ctr->qlen[out], V, g->far[fout], &g->ctr->far_len[fout], g->far_cap, g->ctr);
            if (timing) ktimer_end(g);
            sync_counters(g);
            CGB_REQUIRE(!g->h_ctr->overflow, CGB_EOVERFLOW, "SSSP far pile overflow");
            nnear = g->h_ctr->qlen[out];
            nfar = g->h_ctr->far_len[fout];
            cur = out;
            fcur = fout;
            iters++;
            if (nnear > 0 || nfar == 0) break;
            // every remaining entry is at or above thr: jump to the bucket of the smallest
            const uint64_t mn = g->h_ctr->min_far;
            thr = (mn / delta + 1) * (uint64_t)delta;
        }
        // the next near rounds append to the pile the split just wrote
        if (nnear == 0 && nfar == 0) break;
    }
    CGB_CUDA_TRY(cudaEventRecord(g->ev_stop, g->stream));
    g->stats.iterations = iters;
    g->stats.sssp_delta = delta;
}

uint32_t sssp_default_delta(const cgb_graph* g)
{
    if (g->E == 0 || g->V == 0) return 1;
    const double mean_w = g->w ? (double)g->sum_w / (double)g->E : 1.0;
    const double mean_deg = (double)g->E / (double)g->V;
    double d = 32.0 * mean_w / std::max(1.0, mean_deg);
    if (d < 1.0) d = 1.0;
    if (d > 1e8) d = 1e8;
    return (uint32_t)d;
}

void run_sssp(cgb_graph* g, uint32_t root, const cgb_options& o)
{
    ensure_frontier(g);
    ensure_sssp(g);
    const uint32_t delta = o.sssp_delta ? o.sssp_delta : sssp_default_delta(g);
    if (g->w) sssp_loop<true>(g, root, delta, o);
    else sssp_loop<false>(g, root, delta, o);
}

}  // namespace cgb
