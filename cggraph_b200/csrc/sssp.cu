// Delta-stepping SSSP (near queue, far bitmap) with atomicMin relaxation.
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
// T form the near queue, which is expanded round after round with the
// degree-binned push of push.cuh; a vertex improved to a distance >= T sets
// its bit in the far bitmap (V/32 words, L2-resident).  When the near queue
// empties, the bitmap is split at [T, T + delta): those vertices become the
// near queue, vertices below T are dropped (any improvement below T was
// pushed to the near queue and has been expanded), the rest stay.  A near
// bitmap, cleared before each round, keeps each vertex at most once in a
// round's queue.
#include "engine.cuh"
#include "persist.cuh"
#include "policy.cuh"
#include "push.cuh"

namespace cgb {

__shared__ uint32_t s_sssp_newfar;  // per-CTA count of vertices newly set in the far bitmap
__shared__ unsigned long long s_sssp_medges;  // per-CTA out-degree sum of the next near queue
__shared__ uint32_t s_sssp_touched;  // per-CTA count of vertices reached for the first time

template <bool kHasW>
struct SsspOp {
    const uint32_t* __restrict__ off;
    const uint32_t* __restrict__ dst;
    const uint32_t* __restrict__ w;
    uint32_t* dist;
    uint32_t* near_bm;  // dedup of this round's near queue (cleared before the round)
    uint32_t thr;
    uint32_t nz;
    uint32_t* near_out;
    uint32_t* near_len;
    uint32_t cap;
    uint32_t* far_bm;
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
        bool to_near = false, new_far = false, first = false;
        uint32_t d = 0;
        if (valid) {
            // the edge arrays stream through once: evict first, so L2 keeps dist[] and the bitmaps
            d = __ldcs(dst + e);
            const uint64_t cand = (uint64_t)du + (kHasW ? (uint64_t)__ldcs(w + e) : 1ull);
            if (cand < kValueMax) {
                const uint32_t nd = (uint32_t)cand;
                if (nd < dist[d]) {
                    const uint32_t old = atomicMin(dist + d, nd);
                    first = old == kValueMax;
                    if (nd < old && d < nz) {
                        if (nd < thr) {
                            const uint32_t bit = 1u << (d & 31u);
                            uint32_t* wp = near_bm + (d >> 5);
                            to_near = !(*wp & bit) && !(atomicOr(wp, bit) & bit);
                        } else {
                            const uint32_t bit = 1u << (d & 31u);
                            uint32_t* wp = far_bm + (d >> 5);
                            new_far = !(*wp & bit) && !(atomicOr(wp, bit) & bit);
                        }
                    }
                }
            }
        }
        warp_append(to_near, d, near_out, near_len, cap, &ctr->overflow);
        const uint32_t nf = __popc(__ballot_sync(0xffffffffu, new_far));
        if (nf && lane_id() == 0) atomicAdd(&s_sssp_newfar, nf);
        const uint32_t nt = __popc(__ballot_sync(0xffffffffu, first));
        if (nt && lane_id() == 0) atomicAdd(&s_sssp_touched, nt);
        if (__any_sync(0xffffffffu, to_near)) {
            // out-edges of the next near queue: the next round's push / pull choice
            const unsigned long long dg = warp_sum((unsigned long long)(to_near ? off[d + 1] - off[d] : 0u));
            if (dg && lane_id() == 0) atomicAdd(&s_sssp_medges, dg);
        }
    }
    __device__ __forceinline__ void block_begin() const
    {
        if (threadIdx.x == 0) {
            s_sssp_newfar = 0;
            s_sssp_medges = 0;
            s_sssp_touched = 0;
        }
    }
    __device__ __forceinline__ void block_end() const
    {
        if (threadIdx.x == 0 && s_sssp_newfar) atomicAdd(&ctr->far_len[0], s_sssp_newfar);
        if (threadIdx.x == 0 && s_sssp_medges) atomicAdd(&ctr->medges, s_sssp_medges);
        if (threadIdx.x == 0 && s_sssp_touched) atomicAdd(&ctr->touched, s_sssp_touched);
    }
};

// Dense-frontier relaxation: the near set's out-edges lower dist[] with
// fire-and-forget atomicMin (the result is unused, so it issues as a
// reduction) and enqueue nothing; k_sssp_dense_scan then finds the improved
// vertices by comparing dist[] with its snapshot from before the round.
template <bool kHasW>
struct SsspDenseOp {
    const uint32_t* __restrict__ off;
    const uint32_t* __restrict__ dst;
    const uint32_t* __restrict__ w;
    uint32_t* dist;

    __device__ __forceinline__ bool load(uint32_t v, uint32_t& s, uint32_t& d, uint32_t& m) const
    {
        s = off[v];
        d = off[v + 1] - s;
        m = dist[v];
        return m < kValueMax;
    }
    __device__ __forceinline__ void edge(bool valid, uint32_t e, uint32_t du) const
    {
        if (!valid) return;
        const uint32_t d = __ldcs(dst + e);
        const uint64_t cand = (uint64_t)du + (kHasW ? (uint64_t)__ldcs(w + e) : 1ull);
        if (cand < kValueMax && (uint32_t)cand < dist[d]) atomicMin(dist + d, (uint32_t)cand);
    }
    __device__ __forceinline__ void block_begin() const {}
    __device__ __forceinline__ void block_end() const {}
};

// After a dense round: every vertex whose distance dropped below its snapshot
// joins the next near queue (below thr) or the far bitmap.  A warp owns one
// 32-vertex bitmap word, so far bits are set without atomics; the next
// queue's out-edges and the new far bits are counted.
__global__ void __launch_bounds__(kBlock) k_sssp_dense_scan(uint32_t V, const uint32_t* __restrict__ dist,
                                                            const uint32_t* __restrict__ snap, uint32_t thr,
                                                            uint32_t nz, const uint32_t* __restrict__ off,
                                                            uint32_t* far_bm, uint32_t* near_out, uint32_t* near_len,
                                                            uint32_t cap, DevCounters* ctr)
{
    const uint32_t n_round = (V + 31u) & ~31u;
    unsigned long long deg_sum = 0;
    uint32_t new_far = 0, touched = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n_round; v += gridDim.x * blockDim.x) {
        bool to_near = false, to_far = false;
        if (v < V) {
            const uint32_t dv = dist[v], sv = snap[v];
            touched += (sv == kValueMax && dv < kValueMax) ? 1u : 0u;
            if (v < nz && dv < sv) {
                to_near = dv < thr;
                to_far = !to_near;
                if (to_near) deg_sum += off[v + 1] - off[v];
            }
        }
        warp_append(to_near, v, near_out, near_len, cap, &ctr->overflow);
        const uint32_t fm = __ballot_sync(0xffffffffu, to_far);
        if (fm && lane_id() == 0) {
            const uint32_t old = far_bm[v >> 5];
            if (fm & ~old) {
                far_bm[v >> 5] = old | fm;
                new_far += __popc(fm & ~old);
            }
        }
    }
    deg_sum = warp_sum(deg_sum);
    touched = warp_sum(touched);
    if (lane_id() == 0) {
        if (deg_sum) atomicAdd(&ctr->medges, deg_sum);
        if (new_far) atomicAdd(&ctr->far_len[0], new_far);
        if (touched) atomicAdd(&ctr->touched, touched);
    }
}

// Counters of the next round (and, for a push round, the near-dedup bitmap)
// reset by one launch instead of one memset each: rounds are short, and a
// run has dozens of them.
__global__ void k_sssp_round_reset(DevCounters* ctr, int out, uint32_t* bm, uint32_t words)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ctr->qlen[out] = 0;
        ctr->chunk_len = 0;
        ctr->medges = 0;
    }
    if (bm)
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < words; i += gridDim.x * blockDim.x) bm[i] = 0;
}

// The same before a bucket split: next queue, far count, smallest far distance.
__global__ void k_sssp_split_reset(DevCounters* ctr, int out)
{
    ctr->qlen[out] = 0;
    ctr->far_len[0] = 0;
    ctr->min_far = 0xFFFFFFFFu;
    ctr->medges = 0;
}

__global__ void k_sssp_init(uint32_t V, uint32_t* dist, uint32_t* far_bm, uint32_t words)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += stride) dist[i] = kValueMax;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < words; i += stride) far_bm[i] = 0;
}

__global__ void k_sssp_root(uint32_t* dist, uint32_t root, uint32_t* q0)
{
    dist[root] = 0;
    q0[0] = root;
}

// Splits the far bitmap at [lo, hi) (see file comment).  One lane per bitmap
// word; far_len[0] receives the number of vertices left in the bitmap and
// min_far the smallest distance among them.
__global__ void __launch_bounds__(kBlock) k_sssp_split(uint32_t words, uint32_t* far_bm, const uint32_t* dist,
                                                       uint32_t lo, uint32_t hi, uint32_t* near_out,
                                                       uint32_t* near_len, uint32_t cap, DevCounters* ctr,
                                                       const uint32_t* __restrict__ off)
{
    uint32_t mn = kValueMax, left = 0;
    unsigned long long dg = 0;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t words_round = (words + 31u) & ~31u;
    for (uint32_t wi = blockIdx.x * blockDim.x + threadIdx.x; wi < words_round; wi += stride) {
        uint32_t word = wi < words ? far_bm[wi] : 0u;
        uint32_t keep = word;
        // at most 32 near candidates per lane: append them one bit position at a time
        while (__any_sync(0xffffffffu, word != 0)) {
            bool to_near = false;
            uint32_t v = 0;
            if (word) {
                const uint32_t b = __ffs(word) - 1;
                word &= word - 1;
                v = wi * 32 + b;
                const uint32_t dv = dist[v];
                if (dv < hi) {
                    keep &= ~(1u << b);
                    to_near = dv >= lo;
                    if (to_near) dg += off[v + 1] - off[v];
                } else {
                    mn = min(mn, dv);
                }
            }
            warp_append(to_near, v, near_out, near_len, cap, &ctr->overflow);
        }
        if (wi < words) {
            if (keep != far_bm[wi]) far_bm[wi] = keep;
            left += __popc(keep);
        }
    }
    mn = __reduce_min_sync(0xffffffffu, mn);
    left = warp_sum(left);
    dg = warp_sum(dg);
    if (lane_id() == 0) {
        if (mn != kValueMax) atomicMin(&ctr->min_far, mn);
        if (left) atomicAdd(&ctr->far_len[0], left);
        if (dg) atomicAdd(&ctr->medges, dg);
    }
}

template <bool kHasW>
static void sssp_loop(cgb_graph* g, uint32_t root, uint32_t delta, const cgb_options& o)
{
    const bool timing = g->flags & CGB_FLAG_KERNEL_TIMING;
    const bool tracing = g->flags & CGB_FLAG_TRACE;
    const uint32_t V = g->V;
    const uint32_t words = g->words();
    uint32_t* far_bm = g->front_bm;  // the BFS bitmaps are free during SSSP
    uint32_t* near_bm = g->visited;
    const uint64_t max_iters = o.max_iterations ? o.max_iterations : ~0ull;
    Policy* pol = (o.schedule == CGB_SCHED_LEARNED) ? policy_get() : nullptr;
    PolicySamples* collect = g->collect;
    const uint32_t base_delta = delta;

    CGB_CUDA_TRY(cudaEventRecord(g->ev_start, g->stream));
    if (timing) ktimer_begin(g, CGB_K_INIT);
    ++g->stats.launches;
    k_sssp_init<<<num_sms() * 4, kBlock, 0, g->stream>>>(V, g->value, far_bm, words);
    ++g->stats.launches;
    k_sssp_root<<<1, 1, 0, g->stream>>>(g->value, root, g->q[0]);
    if (timing) ktimer_end(g);

    int cur = 0;
    uint64_t nnear = root < g->nz ? 1 : 0;
    uint64_t nfar = 0;
    uint64_t thr = delta;
    uint64_t bucket_lo = 0;      // the current bucket is [bucket_lo, thr): every near vertex is in it
    uint64_t near_edges = 0;     // out-edges of the near queue (0 = unknown: push)
    double touch_rate = 0.0;     // vertices reached for the first time per edge, last push or dense round
    uint64_t touched_seen = 0;   // ctr->touched after that round
    // pull rounds need the in-edges (and their weights in CSC order)
    const bool pull_ok = o.schedule != CGB_SCHED_FIXED && g->tune.sssp_pull_alpha > 0;
    uint64_t iters = 0;
    uint64_t expanded = 0;

    // Near rounds at threshold thr until the near queue is empty.
    const bool persist_ok = !tracing && o.schedule != CGB_SCHED_FIXED && g->max_degree < g->tune.persist_deg;
    auto near_rounds = [&]() {
        while (nnear > 0) {
            CGB_REQUIRE(iters < max_iters, CGB_ETIMEOUT, "SSSP iteration budget exhausted");
            if (persist_ok && nnear <= g->tune.persist_enter) {
                // small near queue: run the rounds on the device
                if (timing) ktimer_begin(g, CGB_K_PUSH);
                const PersistResult r =
                    sssp_persistent(g, cur, (uint32_t)nnear, (uint32_t)std::min<uint64_t>(thr, kValueMax), far_bm,
                                    g->tune.persist_enter, (uint32_t)std::min<uint64_t>(max_iters - iters, 1u << 20));
                if (timing) ktimer_end(g);
                sync_counters(g);
                iters += r.levels;
                expanded += r.added;
                nnear = r.nf;
                nfar = g->h_ctr->far_len[0];
                near_edges = 0;  // not counted by the device-resident rounds: push next
                cur = r.cur;
                if (r.levels > 0) continue;
            }
            const int out = cur ^ 1;
            // direction: pull when the near set's out-edges times alpha exceed the graph's edges;
            // else a dense frontier when they are many for what the round will change.  A push
            // round pays an atomic with a returned value and a queue append per improvement, a
            // dense round a reduction per edge plus one pass over V.  While the search reaches
            // new territory nearly every edge improves its target, so the out-edges are weighted
            // by the previous round's first touches per edge, floored at 1/8 for the rounds that
            // mostly lower known distances
            const bool pull = pull_ok && (double)near_edges * g->tune.sssp_pull_alpha > (double)g->E;
            const bool dense = !pull && o.schedule != CGB_SCHED_FIXED && g->tune.sssp_dense_alpha > 0 &&
                               (double)near_edges * g->tune.sssp_dense_alpha * std::max(touch_rate, 0.125) >
                                   (double)V;
            if (pull) {
                ensure_csc(g);
                ensure_csc_weights(g);
            }
            ++g->stats.launches;
            k_sssp_round_reset<<<(!pull && !dense) ? num_sms() * 2 : 1, kBlock, 0, g->stream>>>(
                g->ctr, out, (!pull && !dense) ? near_bm : nullptr, words);
            if (tracing) CGB_CUDA_TRY(cudaEventRecord(g->ev_iter[0], g->stream));
            if (timing) ktimer_begin(g, pull ? CGB_K_PULL : CGB_K_PUSH);
            if (pull) {
                sssp_pull_round(g, g->q[cur], (uint32_t)nnear, (uint32_t)std::min<uint64_t>(bucket_lo, kValueMax),
                                (uint32_t)std::min<uint64_t>(thr, kValueMax), g->q[out], &g->ctr->qlen[out], far_bm,
                                g->aux_bm);
                g->stats.pulls_bu++;
            } else if (dense) {
                CGB_CUDA_TRY(cudaMemcpyAsync(g->stamp, g->value, (size_t)V * 4, cudaMemcpyDeviceToDevice, g->stream));
                SsspDenseOp<kHasW> op{g->off, g->dst, g->w, g->value};
                launch_push(g, g->q[cur], (uint32_t)nnear, op, false);
                ++g->stats.launches;
                k_sssp_dense_scan<<<grid_for(V, kBlock, num_sms() * 8), kBlock, 0, g->stream>>>(
                    V, g->value, g->stamp, (uint32_t)std::min<uint64_t>(thr, kValueMax), g->nz, g->off, far_bm,
                    g->q[out], &g->ctr->qlen[out], V, g->ctr);
                g->stats.pushes_td++;
            } else {
                SsspOp<kHasW> op{g->off, g->dst, g->w, g->value, near_bm,
                                 (uint32_t)std::min<uint64_t>(thr, kValueMax), g->nz, g->q[out], &g->ctr->qlen[out],
                                 V, far_bm, g->ctr};
                launch_push(g, g->q[cur], (uint32_t)nnear, op, false);
                g->stats.pushes_td++;
            }
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
                t.unvisited_vertices = g->h_ctr->far_len[0];
                t.variant = pull ? CGB_VAR_PULL : dense ? CGB_VAR_DENSE : CGB_VAR_TWC;
                t.frontier_edges = near_edges;
                t.delta = delta;
                t.ms = ms;
                g->trace.push_back(t);
            }
            expanded += nnear;
            if (!pull && near_edges > 0) {
                touch_rate = (double)(g->h_ctr->touched - touched_seen) / (double)near_edges;
                touched_seen = g->h_ctr->touched;
            }
            nnear = g->h_ctr->qlen[out];
            nfar = g->h_ctr->far_len[0];
            near_edges = g->h_ctr->medges;
            cur = out;
            iters++;
        }
    };
    // Next bucket [thr, thr + d): split the far bitmap (jumping over empty
    // buckets) until the near queue is non-empty or the bitmap is empty.
    auto advance = [&](uint32_t d) {
        uint64_t lo = thr;
        thr += d;
        for (;;) {
            CGB_REQUIRE(iters < max_iters, CGB_ETIMEOUT, "SSSP iteration budget exhausted");
            const int out = cur ^ 1;
            ++g->stats.launches;
            k_sssp_split_reset<<<1, 1, 0, g->stream>>>(g->ctr, out);
            if (timing) ktimer_begin(g, CGB_K_FRONTIER);
            ++g->stats.launches;
            k_sssp_split<<<grid_for(words, kBlock, num_sms() * 4), kBlock, 0, g->stream>>>(
                words, far_bm, g->value, (uint32_t)std::min<uint64_t>(lo, kValueMax),
                (uint32_t)std::min<uint64_t>(thr, kValueMax), g->q[out], &g->ctr->qlen[out], V, g->ctr, g->off);
            if (timing) ktimer_end(g);
            sync_counters(g);
            CGB_REQUIRE(!g->h_ctr->overflow, CGB_EOVERFLOW, "SSSP queue overflow");
            nnear = g->h_ctr->qlen[out];
            nfar = g->h_ctr->far_len[0];
            near_edges = g->h_ctr->medges;
            cur = out;
            iters++;
            bucket_lo = lo;
            if (nnear > 0 || nfar == 0) break;
            // every vertex left is at or above thr: jump to the bucket of the smallest
            const uint64_t mn = g->h_ctr->min_far;
            lo = thr;
            thr = (mn / d + 1) * (uint64_t)d;
        }
    };
    auto state_now = [&]() {
        FeatIn in{};
        in.alg = CGB_SSSP;
        in.iteration = (uint32_t)iters;
        in.symmetric = g->symmetric == 1;
        in.V = V;
        in.E = g->E;
        in.nf = (double)nnear;
        in.unvisited_v = (double)V - (double)std::min<uint64_t>(expanded, V);
        in.delta = delta;
        in.base_delta = base_delta;
        in.far_count = (double)nfar;
        in.settled = (double)std::min<uint64_t>(expanded, V);
        return in;
    };

    near_rounds();
    while (nfar > 0) {
        uint32_t d = delta;
        if (collect) {
            // counterfactual: one bucket phase per delta choice from the same state
            const size_t vbytes = (size_t)V * 4, wbytes = (size_t)words * 4;
            CGB_CUDA_TRY(cudaMemcpyAsync(collect->save_value, g->value, vbytes, cudaMemcpyDeviceToDevice, g->stream));
            CGB_CUDA_TRY(cudaMemcpyAsync(collect->save_bm0, far_bm, wbytes, cudaMemcpyDeviceToDevice, g->stream));
            const uint64_t s_thr = thr, s_iters = iters, s_exp = expanded, s_far = nfar;
            const int s_cur = cur;
            float ms[kPolicyOutputs] = {};
            bool have[kPolicyOutputs] = {};
            int best = kDeltaUnit;
            for (int k = 0; k < kNumDeltaChoices; k++) {
                const uint32_t dk = std::max<uint32_t>(1u, (uint32_t)(base_delta * delta_scale(k)));
                CGB_CUDA_TRY(cudaEventRecord(g->ev_iter[0], g->stream));
                advance(dk);
                near_rounds();
                CGB_CUDA_TRY(cudaEventRecord(g->ev_iter[1], g->stream));
                CGB_CUDA_TRY(cudaEventSynchronize(g->ev_iter[1]));
                float t = 0.f;
                CGB_CUDA_TRY(cudaEventElapsedTime(&t, g->ev_iter[0], g->ev_iter[1]));
                // cost per unit of distance the phase covers (delta x scale)
                ms[kOutDelta0 + k] = t / delta_scale(k);
                have[kOutDelta0 + k] = true;
                if (ms[kOutDelta0 + k] < ms[kOutDelta0 + best]) best = k;
                CGB_CUDA_TRY(cudaMemcpyAsync(g->value, collect->save_value, vbytes, cudaMemcpyDeviceToDevice,
                                             g->stream));
                CGB_CUDA_TRY(cudaMemcpyAsync(far_bm, collect->save_bm0, wbytes, cudaMemcpyDeviceToDevice, g->stream));
                thr = s_thr;
                iters = s_iters;
                expanded = s_exp;
                nfar = s_far;
                nnear = 0;
                cur = s_cur;
            }
            policy_log_sample(g, state_now(), ms, have);
            d = std::max<uint32_t>(1u, (uint32_t)(base_delta * delta_scale(best)));
        } else if (pol) {
            policy_enqueue(pol, g, state_now(), false, false, 0);
            sync_counters(g);
            const int k = policy_pick_delta(g->h_ctr->policy_out);
            if (k >= 0) d = std::max<uint32_t>(1u, (uint32_t)(base_delta * delta_scale(k)));
        }
        delta = d;
        advance(d);
        near_rounds();
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
    double d = 8.0 * mean_w / std::max(1.0, mean_deg);
    if (d < 1.0) d = 1.0;
    if (d > 1e8) d = 1e8;
    return (uint32_t)d;
}

void run_sssp(cgb_graph* g, uint32_t root, const cgb_options& o)
{
    ensure_frontier(g);
    if (g->w && g->sum_w == 0) compute_weight_sum(g);
    const uint32_t delta = o.sssp_delta ? o.sssp_delta : sssp_default_delta(g);
    if (g->w) sssp_loop<true>(g, root, delta, o);
    else sssp_loop<false>(g, root, delta, o);
}

}  // namespace cgb
