// Multi-root SSSP state and kernels shared by the batch path (mssp.cu) and
// the request server (serve.cu).  See mssp.cu for the algorithm.
#pragma once

#include "engine.cuh"

namespace cgb {

constexpr uint32_t kMsRoots = 64;   // distance slots per vertex

struct MsspCounters {
    uint32_t nq_in;        // entries of the near queue being expanded
    uint32_t nq_out;       // entries of the near queue being built
    uint32_t nfar_live;    // entries of the live far list (expansion rounds append)
    uint32_t nfar_next;    // entries kept by a split in the other far list
    uint32_t ndesc;        // descriptors of the round
    uint32_t min_far;      // smallest far distance >= hi seen by a split
    uint32_t overflow;
    unsigned long long relax;  // successful relaxations
};

struct MsspBuffers {
    uint32_t* dist = nullptr;               // V * 64
    unsigned long long* pend = nullptr;     // V
    unsigned long long* farm = nullptr;     // V
    unsigned long long* maskq = nullptr;    // V: pend of each queue entry, taken by the descriptor pass
    uint32_t* far_list[2] = {nullptr, nullptr};  // V each
    uint4* desc = nullptr;                  // {v, edge begin, edge end, queue index}
    uint64_t desc_cap = 0;
    MsspCounters* c = nullptr;
    MsspCounters* h = nullptr;              // pinned host copy
};

MsspBuffers* mssp_buffers_alloc(uint32_t V, uint64_t E);

// The bodies of the round kernels (k_mssp_desc, k_mssp_expand, k_mssp_split):
// warp-level, striding over the grid's warps with no CTA barrier, so a
// device-resident loop of kBlock-thread CTAs can run them as its phases.

// Takes (and clears) the pend mask of every queued vertex and cuts its list
// into descriptors of at most ms_edges edges.
__device__ __forceinline__ void mssp_desc_body(const uint32_t* __restrict__ q, const uint32_t* nq_ptr,
                                                      const uint32_t* __restrict__ off, unsigned long long* pend,
                                                      unsigned long long* maskq, uint4* desc, uint64_t cap,
                                                      MsspCounters* c, uint32_t ms_edges)
{
    const uint32_t nq = *nq_ptr;
    const uint32_t n_round = (nq + 31u) & ~31u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_round; i += gridDim.x * blockDim.x) {
        uint32_t v = 0, s = 0, d = 0, nd = 0;
        if (i < nq) {
            v = q[i];
            maskq[i] = pend[v];
            pend[v] = 0;
            s = off[v];
            d = off[v + 1] - s;
            nd = (d + ms_edges - 1) / ms_edges;
        }
        // warp-inclusive scan of the descriptor counts, one atomic per warp
        uint32_t incl = nd;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane_id() >= (uint32_t)o) incl += t;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        uint32_t base = 0;
        if (lane_id() == 31 && total) base = atomicAdd(&c->ndesc, total);
        base = __shfl_sync(0xffffffffu, base, 31);
        const uint64_t pos = (uint64_t)base + incl - nd;
        for (uint32_t j = 0; j < nd; j++) {
            if (pos + j < cap) {
                const uint32_t eb = s + j * ms_edges;
                desc[pos + j] = make_uint4(v, eb, min(eb + ms_edges, s + d), i);
            } else {
                atomicOr(&c->overflow, 1u);
            }
        }
    }
}

// One near round: relaxes every descriptor's edges for the roots of its
// vertex's mask.  Pairs improved below their root's threshold (thr, or
// thr_slot[k] per root) go to pend (their vertex queued in qout on the
// 0 -> non-zero transition), the others to farm (vertex listed in far_out
// on the same transition).  alive (optional) collects the roots that got
// near work ([0]) and far work ([1]).
template <bool kHasW>
__device__ __forceinline__ void mssp_expand_body(const uint4* __restrict__ desc, const MsspCounters* cc,
                                                        const unsigned long long* __restrict__ maskq,
                                                        const uint32_t* __restrict__ dst,
                                                        const uint32_t* __restrict__ w, uint32_t* dist,
                                                        unsigned long long* pend, unsigned long long* farm,
                                                        uint32_t* qout, uint32_t* qout_len, uint32_t* far_out,
                                                        uint32_t* far_len, uint32_t cap, uint32_t thr,
                                                        const uint32_t* thr_slot, unsigned long long* alive,
                                                        MsspCounters* c)
{
    const uint32_t ndesc = min((uint64_t)cc->ndesc, (uint64_t)0xFFFFFFFFu);
    const uint32_t lane = lane_id();
    const uint32_t warps = gridDim.x * (kBlock / 32);
    const uint32_t thr0 = thr_slot ? thr_slot[lane] : thr, thr1 = thr_slot ? thr_slot[lane + 32] : thr;
    unsigned long long relax = 0, near_live = 0, far_live = 0;
    for (uint32_t j = blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5); j < ndesc; j += warps) {
        const uint4 d = desc[j];
        const unsigned long long m = maskq[d.w];
        const bool a0 = (m >> lane) & 1ull, a1 = (m >> (lane + 32)) & 1ull;
        const uint32_t* dv_row = dist + (size_t)d.x * kMsRoots;
        const uint32_t dv0 = a0 ? dv_row[lane] : kValueMax;
        const uint32_t dv1 = a1 ? dv_row[lane + 32] : kValueMax;
        const bool s0 = dv0 < kValueMax, s1 = dv1 < kValueMax;
        for (uint32_t e0 = d.y; e0 < d.z; e0 += 32) {
            const uint32_t cnt = min(32u, d.z - e0);
            uint32_t my_u = 0, my_w = 1;
            if (lane < cnt) {
                my_u = dst[e0 + lane];
                if (kHasW) my_w = w[e0 + lane];
            }
            // lane t collects the root masks improved through edge t, then
            // every lane publishes its own edge's masks (32 atomics at once)
            unsigned long long my_nb = 0, my_fb = 0;
            for (uint32_t t0 = 0; t0 < cnt; t0 += 4) {
                uint32_t u[4], wt[4], x0[4], x1[4];
#pragma unroll
                for (int i = 0; i < 4; i++) {  // loads first: four targets in flight
                    const uint32_t t = min(t0 + i, cnt - 1);
                    u[i] = __shfl_sync(0xffffffffu, my_u, t);
                    wt[i] = __shfl_sync(0xffffffffu, my_w, t);
                    const uint32_t* du = dist + (size_t)u[i] * kMsRoots;
                    x0[i] = s0 ? du[lane] : 0u;
                    x1[i] = s1 ? du[lane + 32] : 0u;
                }
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const uint32_t t = t0 + i;
                    if (t >= cnt) break;  // warp-uniform
                    uint32_t* du = dist + (size_t)u[i] * kMsRoots;
                    bool m0 = false, m1 = false, n0 = false, n1 = false;
                    const uint64_t c0 = (uint64_t)dv0 + wt[i], c1 = (uint64_t)dv1 + wt[i];
                    if (s0 && c0 < kValueMax && (uint32_t)c0 < x0[i]) {
                        m0 = (uint32_t)c0 < atomicMin(du + lane, (uint32_t)c0);
                        n0 = m0 && (uint32_t)c0 < thr0;
                    }
                    if (s1 && c1 < kValueMax && (uint32_t)c1 < x1[i]) {
                        m1 = (uint32_t)c1 < atomicMin(du + lane + 32, (uint32_t)c1);
                        n1 = m1 && (uint32_t)c1 < thr1;
                    }
                    // improved roots; their near / far split only when there are any
                    const unsigned long long mb = (unsigned long long)__ballot_sync(0xffffffffu, m0) |
                                                  ((unsigned long long)__ballot_sync(0xffffffffu, m1) << 32);
                    if (mb) {
                        relax += (m0 ? 1 : 0) + (m1 ? 1 : 0);
                        const unsigned long long nb = (unsigned long long)__ballot_sync(0xffffffffu, n0) |
                                                      ((unsigned long long)__ballot_sync(0xffffffffu, n1) << 32);
                        if (lane == t) {
                            my_nb = nb;
                            my_fb = mb & ~nb;
                        }
                    }
                }
            }
            const bool qn = my_nb && atomicOr(pend + my_u, my_nb) == 0ull;
            const bool qf = my_fb && atomicOr(farm + my_u, my_fb) == 0ull;
            near_live |= my_nb;
            far_live |= my_fb;
            warp_append(qn, my_u, qout, qout_len, cap, &c->overflow);
            warp_append(qf, my_u, far_out, far_len, cap, &c->overflow);
        }
    }
    relax = warp_sum(relax);
    if (lane == 0 && relax) atomicAdd(&c->relax, relax);
    if (alive) {
        near_live = warp_or(near_live);
        far_live = warp_or(far_live);
        if (lane == 0 && near_live) atomicOr(alive, near_live);
        if (lane == 0 && far_live) atomicOr(alive + 1, far_live);
    }
}

// Split: for every vertex of the far list and every root k of `adv` (the
// roots whose near work is done), the far pairs with lo_k <= dist < hi_k go
// to pend (vertex queued in q on pend's 0 -> non-zero transition), those
// below lo_k were expanded already and are dropped, and the rest stay far;
// vertices with far pairs left are written to far_out.  The smallest kept
// distance >= hi_k is reported per root (min_far_slot) or overall
// (c->min_far); far_alive (optional) receives the roots with far pairs left.
// lo_slot / hi_slot (per root) may be NULL for one range [lo, hi).
__device__ __forceinline__ void mssp_split_body(const uint32_t* __restrict__ far_in, const uint32_t* nfar_ptr,
                                                       const uint32_t* __restrict__ dist, unsigned long long* pend,
                                                       unsigned long long* farm, uint32_t* q, uint32_t* q_len,
                                                       uint32_t* far_out, uint32_t* far_out_len, uint32_t cap,
                                                       uint32_t lo, uint32_t hi, const uint32_t* lo_slot,
                                                       const uint32_t* hi_slot, unsigned long long adv,
                                                       uint32_t* min_far_slot, unsigned long long* far_alive,
                                                       MsspCounters* c)
{
    const uint32_t nfar = *nfar_ptr;
    const uint32_t lane = lane_id();
    const uint32_t warps = gridDim.x * (kBlock / 32);
    const uint32_t lo0 = lo_slot ? lo_slot[lane] : lo, lo1 = lo_slot ? lo_slot[lane + 32] : lo;
    const uint32_t hi0 = hi_slot ? hi_slot[lane] : hi, hi1 = hi_slot ? hi_slot[lane + 32] : hi;
    const bool adv0 = (adv >> lane) & 1ull, adv1 = (adv >> (lane + 32)) & 1ull;
    uint32_t mn0 = kValueMax, mn1 = kValueMax;
    unsigned long long live = 0;
    // a warp takes 32 far vertices; those with no pair of an advancing root
    // stay far untouched (one aggregated append), the others are processed
    // one at a time with the lanes over the roots
    const uint32_t n_round = (nfar + 31u) & ~31u;
    for (uint32_t base = (blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5)) * 32; base < n_round;
         base += warps * 32) {
        const uint32_t i = base + lane;
        const uint32_t my_v = i < nfar ? far_in[i] : 0;
        const unsigned long long my_m = i < nfar ? farm[my_v] : 0ull;
        const bool hit = (my_m & adv) != 0ull;
        if (i < nfar && !hit) live |= my_m;
        warp_append(i < nfar && !hit, my_v, far_out, far_out_len, cap, &c->overflow);
        for (uint32_t hits = __ballot_sync(0xffffffffu, hit); hits; hits &= hits - 1) {
            const uint32_t src = __ffs(hits) - 1;
            const uint32_t v = __shfl_sync(0xffffffffu, my_v, src);
            const unsigned long long m = __shfl_sync(0xffffffffu, my_m, src);
            const bool a0 = adv0 && ((m >> lane) & 1ull), a1 = adv1 && ((m >> (lane + 32)) & 1ull);
            const uint32_t* row = dist + (size_t)v * kMsRoots;
            const uint32_t d0 = a0 ? row[lane] : kValueMax, d1 = a1 ? row[lane + 32] : kValueMax;
            const bool mv0 = a0 && d0 < hi0, mv1 = a1 && d1 < hi1;
            const bool nr0 = mv0 && d0 >= lo0, nr1 = mv1 && d1 >= lo1;
            if (a0 && !mv0) mn0 = min(mn0, d0);
            if (a1 && !mv1) mn1 = min(mn1, d1);
            const unsigned long long moved = (unsigned long long)__ballot_sync(0xffffffffu, mv0) |
                                             ((unsigned long long)__ballot_sync(0xffffffffu, mv1) << 32);
            const unsigned long long nearb = (unsigned long long)__ballot_sync(0xffffffffu, nr0) |
                                             ((unsigned long long)__ballot_sync(0xffffffffu, nr1) << 32);
            const unsigned long long keep = m & ~moved;
            if (lane == 0) {
                live |= keep;
                if (moved) farm[v] = keep;  // no expansion runs during a split: v's far mask is this warp's
                if (nearb && atomicOr(pend + v, nearb) == 0ull) {
                    const uint32_t p = atomicAdd(q_len, 1u);
                    if (p < cap) q[p] = v;
                    else atomicOr(&c->overflow, 1u);
                }
                if (keep) {
                    const uint32_t p = atomicAdd(far_out_len, 1u);
                    if (p < cap) far_out[p] = v;
                    else atomicOr(&c->overflow, 1u);
                }
            }
        }
    }
    if (min_far_slot) {
        // per root: mn0 is root lane's, mn1 root lane + 32's, each reduced over the warp's vertices
        if (mn0 != kValueMax) atomicMin(min_far_slot + lane, mn0);
        if (mn1 != kValueMax) atomicMin(min_far_slot + lane + 32, mn1);
    } else {
        const uint32_t mn = __reduce_min_sync(0xffffffffu, min(mn0, mn1));
        if (lane == 0 && mn != kValueMax) atomicMin(&c->min_far, mn);
    }
    if (far_alive) {
        live = warp_or(live);
        if (lane == 0 && live) atomicOr(far_alive, live);
    }
}


void mssp_buffers_free(MsspBuffers* b);

__global__ void k_mssp_desc(const uint32_t* __restrict__ q, const uint32_t* nq_ptr, const uint32_t* __restrict__ off,
                            unsigned long long* pend, unsigned long long* maskq, uint4* desc, uint64_t cap,
                            MsspCounters* c, uint32_t ms_edges);
__global__ void k_mssp_split(const uint32_t* __restrict__ far_in, const uint32_t* nfar_ptr,
                             const uint32_t* __restrict__ dist, unsigned long long* pend, unsigned long long* farm,
                             uint32_t* q, uint32_t* q_len, uint32_t* far_out, uint32_t* far_out_len, uint32_t cap,
                             uint32_t lo, uint32_t hi, const uint32_t* lo_slot, const uint32_t* hi_slot,
                             unsigned long long adv, uint32_t* min_far_slot, unsigned long long* far_alive,
                             MsspCounters* c);
// Launches k_mssp_expand (weighted or unit weights) on stream st.
void mssp_expand(bool weighted, uint32_t grid, cudaStream_t st, const uint4* desc, const MsspCounters* cc,
                 const unsigned long long* maskq, const uint32_t* dst, const uint32_t* w, uint32_t* dist,
                 unsigned long long* pend, unsigned long long* farm, uint32_t* qout, uint32_t* qout_len,
                 uint32_t* far_out, uint32_t* far_len, uint32_t cap, uint32_t thr, const uint32_t* thr_slot,
                 unsigned long long* alive);

}  // namespace cgb
