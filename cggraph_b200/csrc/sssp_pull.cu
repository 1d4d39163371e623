// Pull rounds of delta-stepping SSSP (direction optimisation).
//
// A push round relaxes the out-edges of the near set N (vertices improved
// below the threshold): one returning atomicMin per improving edge, plus a
// bitmap atomic, scattered over the whole distance array -- the heavy middle
// rounds of a power-law graph, where N's out-edges are a large share of E,
// are bound by those atomics.  A pull round computes the same relaxation
// from the other side: every vertex v that can still improve (dist[v] > lo,
// the bucket's lower bound, which every member of N is at or above) scans
// its in-edges (u, w) and takes the minimum of dist[u] + w over the sources
// u in N, read from a bitmap of N.  One thread owns each v, so dist[v] is
// written without atomics, and the in-edge arrays stream in order.  The
// relaxation is label-correcting either way (any value read for dist[u] is
// a real path length, and a lowered u joins the next near set), so push and
// pull rounds can be mixed freely and the result is the exact distance.
//
// Lists are binned by in-degree as in the multi-root bottom-up (msbfs.cu):
// a CTA packs the first kPullLight in-edges of its vertices edge-parallel;
// longer lists finish on a warp, hub lists on chunks spread over the grid
// whose minima meet in `acc` by atomicMin before one thread settles them.
#include "engine.cuh"

namespace cgb {

constexpr uint32_t kPullLight = 32;
constexpr uint32_t kPullChunk = 4096;

struct PullArgs {
    uint32_t V;
    const uint32_t* in_off;
    const uint32_t* in_src;
    const uint32_t* in_w;  // NULL: unit weights
    uint32_t* dist;
    const uint32_t* near_set;  // bitmap of N
    uint32_t lo, thr, nz;
    uint32_t* qout;
    uint32_t* qout_len;
    uint32_t cap;
    uint32_t* far_bm;
    uint32_t* acc;       // partial minima of listed vertices
    uint32_t* heavy_w;   // vertices finished by a warp (capacity V)
    uint32_t* heavy_b;   // vertices finished by chunks (capacity cap_b)
    uint32_t* heavy_w_len;
    uint32_t* heavy_b_len;
    uint32_t cap_b;
    const uint32_t* off;  // out-offsets: degree sums of the next near set
    DevCounters* ctr;
};

__device__ __forceinline__ bool in_near(const uint32_t* bm, uint32_t u) { return (bm[u >> 5] >> (u & 31u)) & 1u; }

__device__ __forceinline__ uint32_t relax_cand(uint32_t du, uint32_t w)
{
    const uint64_t c = (uint64_t)du + w;
    return c < kValueMax ? (uint32_t)c : kValueMax;
}

// v's new distance `best` (< dv): to the next near set below thr, to the far
// bitmap otherwise (counted when its bit is new).  Returns the out-degree
// the next near set gains.
__device__ __forceinline__ void pull_settle(const PullArgs& a, uint32_t v, uint32_t best, bool& to_near,
                                            uint32_t& deg, uint32_t& new_far)
{
    a.dist[v] = best;
    if (v >= a.nz) return;
    if (best < a.thr) {
        to_near = true;
        deg = a.off[v + 1] - a.off[v];
    } else {
        const uint32_t bit = 1u << (v & 31u);
        uint32_t* wp = a.far_bm + (v >> 5);
        if (!(*wp & bit) && !(atomicOr(wp, bit) & bit)) new_far = 1;
    }
}

__device__ __forceinline__ void pull_publish(const PullArgs& a, bool to_near, uint32_t v, uint32_t deg,
                                             uint32_t new_far)
{
    warp_append(to_near, v, a.qout, a.qout_len, a.cap, &a.ctr->overflow);
    const unsigned long long ds = warp_sum((unsigned long long)deg);
    const uint32_t nf = warp_sum(new_far);
    if (lane_id() == 0) {
        if (ds) atomicAdd(&a.ctr->medges, ds);
        if (nf) atomicAdd(&a.ctr->far_len[0], nf);
    }
}

__global__ void __launch_bounds__(kBlock) k_sp_pull_light(PullArgs a)
{
    __shared__ uint32_t s_scan[kBlock / 32 + 1];
    __shared__ uint32_t s_edge[kBlock];
    __shared__ uint32_t s_owner[kBlock];
    __shared__ uint32_t s_best[kBlock];
    const uint32_t tid = threadIdx.x;
    for (uint32_t base = blockIdx.x * kBlock; base < a.V; base += gridDim.x * kBlock) {
        const uint32_t v = base + tid;
        uint32_t dv = 0, e0 = 0, deg = 0, cnt = 0;
        if (v < a.V) {
            dv = a.dist[v];
            if (dv > a.lo) {
                e0 = a.in_off[v];
                deg = a.in_off[v + 1] - e0;
                cnt = min(deg, kPullLight);
            }
        }
        s_best[tid] = kValueMax;
        uint32_t total;
        const uint32_t rank = block_excl_scan(cnt, total, s_scan);
        uint32_t consumed = 0;
        for (uint32_t done = 0; done < total; done += kBlock) {
            while (consumed < cnt && rank + consumed < done + kBlock) {
                s_edge[rank + consumed - done] = e0 + consumed;
                s_owner[rank + consumed - done] = tid;
                consumed++;
            }
            __syncthreads();
            if (tid < min((uint32_t)kBlock, total - done)) {
                const uint32_t e = s_edge[tid];
                const uint32_t u = __ldcs(a.in_src + e);
                if (in_near(a.near_set, u)) {
                    const uint32_t c = relax_cand(a.dist[u], a.in_w ? __ldcs(a.in_w + e) : 1u);
                    if (c < s_best[s_owner[tid]]) atomicMin(&s_best[s_owner[tid]], c);
                }
            }
            __syncthreads();
        }
        bool to_near = false, to_warp = false, to_block = false;
        uint32_t ndeg = 0, new_far = 0;
        if (cnt) {
            const uint32_t best = s_best[tid];
            if (deg > kPullLight) {
                a.acc[v] = best;
                to_block = deg - kPullLight >= kPullChunk;
                to_warp = !to_block;
            } else if (best < dv) {
                pull_settle(a, v, best, to_near, ndeg, new_far);
            }
        }
        pull_publish(a, to_near, v, ndeg, new_far);
        warp_append(to_warp, v, a.heavy_w, a.heavy_w_len, a.cap, &a.ctr->overflow);
        warp_append(to_block, v, a.heavy_b, a.heavy_b_len, a.cap_b, &a.ctr->overflow);
        __syncthreads();  // s_best is rewritten by the next batch
    }
}

__global__ void __launch_bounds__(kBlock) k_sp_pull_warp(PullArgs a)
{
    const uint32_t n = min(*a.heavy_w_len, a.cap);
    const uint32_t lane = lane_id();
    const uint32_t n_round = (n + 31u) & ~31u;
    // a warp per listed vertex; lane 0 keeps the result, published per 32 vertices
    for (uint32_t i0 = (blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5)) * 32; i0 < n_round;
         i0 += gridDim.x * kBlock) {
        bool to_near = false;
        uint32_t my_v = 0, my_deg = 0, my_far = 0;
        for (uint32_t j = 0; j < 32 && i0 + j < n; j++) {
            const uint32_t v = a.heavy_w[i0 + j];
            uint32_t best = a.acc[v];
            const uint32_t e1 = a.in_off[v + 1];
            for (uint32_t e = a.in_off[v] + kPullLight; e < e1; e += 128) {
                uint32_t src[4], wt[4];
#pragma unroll
                for (int t = 0; t < 4; t++) {
                    const uint32_t k = e + 32 * t + lane;
                    src[t] = k < e1 ? __ldcs(a.in_src + k) : 0xFFFFFFFFu;
                    wt[t] = (k < e1 && a.in_w) ? __ldcs(a.in_w + k) : 1u;
                }
                uint32_t m = kValueMax;
#pragma unroll
                for (int t = 0; t < 4; t++)
                    if (src[t] != 0xFFFFFFFFu && in_near(a.near_set, src[t]))
                        m = min(m, relax_cand(a.dist[src[t]], wt[t]));
                best = min(best, __reduce_min_sync(0xffffffffu, m));
            }
            if (lane == j) {
                my_v = v;
                const uint32_t dv = a.dist[v];
                if (best < dv) pull_settle(a, v, best, to_near, my_deg, my_far);
            }
        }
        pull_publish(a, to_near, my_v, my_deg, my_far);
    }
}

// Hub lists: kPullChunk-edge chunks dealt round-robin over the CTAs; each
// CTA's minimum meets the vertex's others in acc[v] by atomicMin.
__global__ void __launch_bounds__(kBlock) k_sp_pull_chunks(PullArgs a)
{
    __shared__ uint32_t s_min;
    const uint32_t n = min(*a.heavy_b_len, a.cap_b);
    uint64_t chunk_base = 0;
    for (uint32_t i = 0; i < n; i++) {
        const uint32_t v = a.heavy_b[i];
        const uint32_t b0 = a.in_off[v] + kPullLight, e1 = a.in_off[v + 1];
        const uint32_t nch = (e1 - b0 + kPullChunk - 1) / kPullChunk;
        const uint32_t first = (uint32_t)((blockIdx.x + gridDim.x - (chunk_base % gridDim.x)) % gridDim.x);
        chunk_base += nch;
        for (uint32_t c = first; c < nch; c += gridDim.x) {
            const uint32_t cs = b0 + c * kPullChunk, ce = min(e1, cs + kPullChunk);
            uint32_t m = kValueMax;
            for (uint32_t e = cs + threadIdx.x; e < ce; e += 4 * kBlock) {
                uint32_t src[4], wt[4];
#pragma unroll
                for (int t = 0; t < 4; t++) {
                    const uint32_t k = e + t * kBlock;
                    src[t] = k < ce ? __ldcs(a.in_src + k) : 0xFFFFFFFFu;
                    wt[t] = (k < ce && a.in_w) ? __ldcs(a.in_w + k) : 1u;
                }
#pragma unroll
                for (int t = 0; t < 4; t++)
                    if (src[t] != 0xFFFFFFFFu && in_near(a.near_set, src[t]))
                        m = min(m, relax_cand(a.dist[src[t]], wt[t]));
            }
            m = __reduce_min_sync(0xffffffffu, m);
            if (threadIdx.x == 0) s_min = kValueMax;
            __syncthreads();
            if (lane_id() == 0 && m < s_min) atomicMin(&s_min, m);
            __syncthreads();
            if (threadIdx.x == 0 && s_min < a.acc[v]) atomicMin(a.acc + v, s_min);
            __syncthreads();
        }
    }
}

__global__ void __launch_bounds__(kBlock) k_sp_pull_settle(PullArgs a)
{
    const uint32_t n = min(*a.heavy_b_len, a.cap_b);
    const uint32_t n_round = (n + 31u) & ~31u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_round; i += gridDim.x * blockDim.x) {
        bool to_near = false;
        uint32_t v = 0, deg = 0, nf = 0;
        if (i < n) {
            v = a.heavy_b[i];
            const uint32_t best = a.acc[v], dv = a.dist[v];
            if (best < dv) pull_settle(a, v, best, to_near, deg, nf);
        }
        pull_publish(a, to_near, v, deg, nf);
    }
}

__global__ void k_sp_near_bitmap(const uint32_t* __restrict__ q, uint32_t n, uint32_t* bm)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t u = q[i];
        atomicOr(bm + (u >> 5), 1u << (u & 31u));
    }
}

void sssp_pull_round(cgb_graph* g, const uint32_t* q_in, uint32_t nin, uint32_t lo, uint32_t thr, uint32_t* qout,
                     uint32_t* qout_len, uint32_t* far_bm, uint32_t* near_set)
{
    const uint32_t words = g->words();
    CGB_CUDA_TRY(cudaMemsetAsync(near_set, 0, (size_t)words * 4, g->stream));
    k_sp_near_bitmap<<<grid_for(nin, kBlock, num_sms() * 8), kBlock, 0, g->stream>>>(q_in, nin, near_set);
    CGB_CUDA_TRY(cudaMemsetAsync(&g->ctr->huge_len, 0, 4, g->stream));
    CGB_CUDA_TRY(cudaMemsetAsync(&g->ctr->found, 0, 4, g->stream));
    PullArgs a{};
    a.V = g->V;
    a.in_off = g->in_off;
    a.in_src = g->in_src;
    a.in_w = g->in_w;
    a.dist = g->value;
    a.near_set = near_set;
    a.lo = lo;
    a.thr = thr;
    a.nz = g->nz;
    a.qout = qout;
    a.qout_len = qout_len;
    a.cap = g->V;
    a.far_bm = far_bm;
    a.acc = g->stamp;
    a.heavy_w = const_cast<uint32_t*>(q_in);  // the near set lives in the bitmap from here on
    a.heavy_b = reinterpret_cast<uint32_t*>(g->chunk_q);
    a.heavy_w_len = &g->ctr->huge_len;
    a.heavy_b_len = &g->ctr->found;
    a.cap_b = (uint32_t)std::min<uint64_t>(2ull * g->chunk_cap, (uint64_t)g->E / kPullChunk + 2);
    a.off = g->off;
    a.ctr = g->ctr;
    g->stats.launches += 5;
    k_sp_pull_light<<<grid_for(g->V, kBlock, num_sms() * 8), kBlock, 0, g->stream>>>(a);
    k_sp_pull_warp<<<num_sms() * 4, kBlock, 0, g->stream>>>(a);
    k_sp_pull_chunks<<<num_sms() * 4, kBlock, 0, g->stream>>>(a);
    k_sp_pull_settle<<<num_sms(), kBlock, 0, g->stream>>>(a);
}

}  // namespace cgb
