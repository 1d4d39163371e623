// Direction-optimising BFS.
//
// Result semantics follow the reference's BFS: level[root] = 0, a vertex's
// level is its parent's + 1, unreachable vertices keep 999999999
// (my_project/CGgraph/GraphDevice.cuh:224-235, device_algorithm.cuh:85-119).
// The reference pushes with atomicMin until no value changes; this engine
// runs level-synchronously, which reaches the same fixpoint:
//   top-down  -- push from a vertex queue with the degree-binned expansion of
//                push.cuh; a visited bitmap (V/32 words, L2-resident) filters
//                before one atomicOr claims a vertex, so each vertex is
//                written and enqueued exactly once;
//   bottom-up -- every unvisited vertex scans its in-edges (the CSC) until it
//                finds a parent in the frontier bitmap; one warp owns 32
//                consecutive vertices = one bitmap word, so visited and next-
//                frontier words are written without atomics.
// The direction switch is Beamer's (alpha = 15, beta = 18) unless the
// schedule says otherwise.
#include "engine.cuh"
#include "persist.cuh"
#include "policy.cuh"
#include "push.cuh"

namespace cgb {

// Per-CTA accumulators of the top-down op (flushed once per CTA).
__shared__ unsigned long long s_td_medges;
__shared__ uint32_t s_td_maxdeg;

struct BfsTdOp {
    const uint32_t* __restrict__ off;
    const uint32_t* __restrict__ dst;
    uint32_t* level;
    uint32_t* visited;
    uint32_t next_level;
    uint32_t nz;
    uint32_t* qout;
    uint32_t* qlen;
    uint32_t cap;
    DevCounters* ctr;
    static constexpr int kBatch = 4;  // edge slots per lane visited together (push.cuh)

    __device__ __forceinline__ bool load(uint32_t v, uint32_t& s, uint32_t& d, uint32_t& m) const
    {
        s = off[v];
        d = off[v + 1] - s;
        m = 0;
        return true;
    }
    template <int N>
    __device__ __forceinline__ void edges(const bool (&valid)[N], const uint32_t (&e)[N], const uint32_t (&)[N]) const
    {
        uint32_t d[N], word[N], bit[N], lo[N], hi[N];
        bool win[N], enq[N];
#pragma unroll
        for (int i = 0; i < N; i++) d[i] = valid[i] ? __ldcs(dst + e[i]) : 0u;  // streamed once: evict first
#pragma unroll
        for (int i = 0; i < N; i++) {
            bit[i] = 1u << (d[i] & 31u);
            word[i] = valid[i] ? visited[d[i] >> 5] : ~0u;
        }
#pragma unroll
        for (int i = 0; i < N; i++) {
            win[i] = false;
            if (!(word[i] & bit[i])) win[i] = !(atomicOr(visited + (d[i] >> 5), bit[i]) & bit[i]);
        }
#pragma unroll
        for (int i = 0; i < N; i++) {
            if (win[i]) level[d[i]] = next_level;
            enq[i] = win[i] && d[i] < nz;
            lo[i] = enq[i] ? off[d[i]] : 0u;
            hi[i] = enq[i] ? off[d[i] + 1] : 0u;
        }
        warp_append_n<N>(enq, d, qout, qlen, cap, &ctr->overflow);
        bool any = false;
#pragma unroll
        for (int i = 0; i < N; i++) any |= enq[i];
        if (__any_sync(0xffffffffu, any)) {
            unsigned long long sum = 0;
            uint32_t mx = 0;
#pragma unroll
            for (int i = 0; i < N; i++) {
                sum += hi[i] - lo[i];
                mx = max(mx, hi[i] - lo[i]);
            }
            sum = warp_sum(sum);
            mx = warp_max(mx);
            if (lane_id() == 0) {
                atomicAdd(&s_td_medges, sum);
                atomicMax(&s_td_maxdeg, mx);
            }
        }
    }
    __device__ __forceinline__ void edge(bool valid, uint32_t e, uint32_t m) const
    {
        const bool v[1] = {valid};
        const uint32_t ee[1] = {e}, mm[1] = {m};
        edges<1>(v, ee, mm);
    }
    __device__ __forceinline__ void block_begin() const
    {
        if (threadIdx.x == 0) {
            s_td_medges = 0;
            s_td_maxdeg = 0;
        }
    }
    __device__ __forceinline__ void block_end() const
    {
        if (threadIdx.x == 0 && s_td_medges) {
            atomicAdd(&ctr->medges, s_td_medges);
            atomicMax(&ctr->max_deg, s_td_maxdeg);
        }
    }
};

__global__ void k_bfs_init(uint32_t V, uint32_t* level, uint32_t* visited, uint32_t words)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += stride) level[i] = kValueMax;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < words; i += stride) visited[i] = 0;
}

__global__ void k_bfs_root(uint32_t* level, uint32_t* visited, uint32_t root, uint32_t* q0)
{
    level[root] = 0;
    visited[root >> 5] = 1u << (root & 31u);
    q0[0] = root;
}

// Queue -> frontier bitmap (bitmap cleared beforehand).
__global__ void k_q2bm(const uint32_t* __restrict__ q, uint32_t n, uint32_t* bm)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t v = q[i];
        atomicOr(bm + (v >> 5), 1u << (v & 31u));
    }
}

// One bottom-up level.  Reads front (current frontier bitmap), writes
// next (all words, so it needs no clearing) and the next queue.  Each lane
// scans its vertex's in-list four entries at a time: four source loads,
// then their four frontier words, are in flight together, and the scan
// stops after the group that holds a parent.  A CTA takes kBlock / 32
// consecutive bitmap words per step (one per warp) and appends the step's
// found vertices with one atomic.
__global__ void __launch_bounds__(kBlock) k_bfs_bu(uint32_t V, const uint32_t* __restrict__ in_off,
                                                   const uint32_t* __restrict__ in_src,
                                                   const uint32_t* __restrict__ off, uint32_t* level,
                                                   uint32_t* visited, const uint32_t* __restrict__ front,
                                                   uint32_t* next, uint32_t next_level, uint32_t nz, uint32_t* qout,
                                                   uint32_t* qlen, uint32_t cap, DevCounters* ctr)
{
    const uint32_t words = (V + 31) / 32;
    constexpr uint32_t kWarps = kBlock / 32;
    unsigned long long medges = 0;
    uint32_t found_cnt = 0, mx = 0;
    for (uint32_t base = blockIdx.x * kWarps; base < words; base += gridDim.x * kWarps) {
        const uint32_t wi = base + (threadIdx.x >> 5);
        const uint32_t v = wi * 32 + lane_id();
        bool enq = false;
        if (wi < words) {  // uniform across the warp
            const uint32_t vis = visited[wi];
            bool found = false;
            if (v < V && !((vis >> lane_id()) & 1u)) {
                const uint32_t e1 = in_off[v + 1];
                for (uint32_t e = in_off[v]; e < e1 && !found; e += 4) {
                    uint32_t u[4], f[4];
#pragma unroll
                    for (int k = 0; k < 4; k++) u[k] = e + k < e1 ? in_src[e + k] : in_src[e];
#pragma unroll
                    for (int k = 0; k < 4; k++) f[k] = front[u[k] >> 5] >> (u[k] & 31u);
#pragma unroll
                    for (int k = 0; k < 4; k++) found |= (f[k] & 1u) != 0;
                }
            }
            const uint32_t fm = __ballot_sync(0xffffffffu, found);
            if (found) level[v] = next_level;
            if (lane_id() == 0) {
                next[wi] = fm;
                if (fm) visited[wi] = vis | fm;
            }
            enq = found && v < nz;
            uint32_t deg = 0;
            if (enq) deg = off[v + 1] - off[v];
            medges += deg;
            found_cnt += enq;
            mx = max(mx, deg);
        }
        const bool p[1] = {enq};
        const uint32_t it[1] = {v};
        block_append_n<1>(p, it, qout, qlen, cap, &ctr->overflow);
    }
    medges = warp_sum(medges);
    found_cnt = warp_sum(found_cnt);
    mx = warp_max(mx);
    if (lane_id() == 0 && found_cnt) {
        atomicAdd(&ctr->medges, medges);
        atomicAdd(&ctr->found, found_cnt);
        atomicMax(&ctr->max_deg, mx);
    }
}

__global__ void k_level_reset(DevCounters* ctr, int out)
{
    ctr->qlen[out] = 0;
    ctr->chunk_len = 0;
    ctr->medges = 0;
    ctr->found = 0;
    ctr->max_deg = 0;
}

// qlen[out], chunk_len, medges, found, max_deg: one launch, not five memsets
static void reset_level_counters(cgb_graph* g, int out)
{
    ++g->stats.launches;
    k_level_reset<<<1, 1, 0, g->stream>>>(g->ctr, out);
}

void run_bfs(cgb_graph* g, uint32_t root, const cgb_options& o)
{
    ensure_frontier(g);
    const bool want_pull = !(o.schedule == CGB_SCHED_FIXED && o.variant != CGB_VAR_PULL && o.variant != CGB_VAR_AUTO);
    const bool force_pull = (o.schedule == CGB_SCHED_FIXED && o.variant == CGB_VAR_PULL);
    if (want_pull) ensure_csc(g);
    const double alpha = o.bfs_alpha > 0 ? o.bfs_alpha : 15.0;
    const double beta = o.bfs_beta > 0 ? o.bfs_beta : 18.0;
    const uint32_t V = g->V;
    const uint32_t words = g->words();
    const bool timing = g->flags & CGB_FLAG_KERNEL_TIMING;
    const bool tracing = g->flags & CGB_FLAG_TRACE;
    PolicySamples* collect = want_pull && !force_pull ? g->collect : nullptr;
    Policy* pol = (o.schedule == CGB_SCHED_LEARNED && want_pull && !force_pull) ? policy_for(g) : nullptr;

    PinnedArray<uint32_t> host_root_deg(2);  // pinned: see pinned_acquire
    CGB_CUDA_TRY(cudaMemcpyAsync(host_root_deg.data(), g->off + root, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                 g->stream));
    CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    CGB_CUDA_TRY(cudaEventRecord(g->ev_start, g->stream));
    if (timing) ktimer_begin(g, CGB_K_INIT);
    ++g->stats.launches;
    k_bfs_init<<<num_sms() * 4, kBlock, 0, g->stream>>>(V, g->value, g->visited, words);
    ++g->stats.launches;
    k_bfs_root<<<1, 1, 0, g->stream>>>(g->value, g->visited, root, g->q[0]);
    if (timing) ktimer_end(g);

    uint32_t cur = 0;  // queue holding the current frontier
    uint64_t nf = (root < g->nz) ? 1 : 0;
    uint64_t prev_nf = 0;
    uint64_t scout = host_root_deg[1] - host_root_deg[0];
    int64_t edges_to_check = (int64_t)g->E;
    uint32_t maxdeg = (uint32_t)scout;
    uint64_t visited_cnt = 1;
    uint32_t level = 0;
    bool bottom_up = false;
    bool have_policy_out = false;
    uint64_t awake = 0, old_awake = 0;
    uint32_t* front = g->front_bm;
    uint32_t* next = g->front_bm + words;
    uint64_t iters = 0;
    const uint64_t max_iters = o.max_iterations ? o.max_iterations : (uint64_t)V + 2;

    // Queues one level in the given direction (frontier in q[cur] and, when
    // the last level was pulled, in `front`; next frontier to q[out] / next);
    // a push level with the given expansion variant (PushExpand).
    auto do_level = [&](bool pull, int out, int expand) {
        reset_level_counters(g, out);
        if (pull) {
            if (!bottom_up) {
                // entering bottom-up: frontier queue -> bitmap
                if (timing) ktimer_begin(g, CGB_K_FRONTIER);
                CGB_CUDA_TRY(cudaMemsetAsync(front, 0, words * sizeof(uint32_t), g->stream));
                ++g->stats.launches;
                k_q2bm<<<grid_for(nf, kBlock, num_sms() * 8), kBlock, 0, g->stream>>>(g->q[cur], (uint32_t)nf, front);
                if (timing) ktimer_end(g);
            }
            if (timing) ktimer_begin(g, CGB_K_PULL);
            const uint32_t grid = grid_for((uint64_t)words * 32, kBlock, num_sms() * 16);
            ++g->stats.launches;
            k_bfs_bu<<<grid, kBlock, 0, g->stream>>>(V, g->in_off, g->in_src, g->off, g->value, g->visited, front,
                                                     next, level + 1, g->nz, g->q[out], &g->ctr->qlen[out], V,
                                                     g->ctr);
            if (timing) ktimer_end(g);
        } else {
            if (timing) ktimer_begin(g, CGB_K_PUSH);
            BfsTdOp op{g->off, g->dst, g->value, g->visited, level + 1, g->nz, g->q[out], &g->ctr->qlen[out], V, g->ctr};
            launch_push(g, g->q[cur], (uint32_t)nf, op, false, expand);
            if (timing) ktimer_end(g);
        }
    };
    auto state_now = [&]() {
        FeatIn in{};
        in.alg = CGB_BFS;
        in.iteration = level;
        in.prev_dir = bottom_up ? 1 : 0;
        in.symmetric = g->symmetric == 1;
        in.V = V;
        in.E = g->E;
        in.nf = (double)nf;
        in.mf = (double)scout;
        in.unvisited_v = (double)V - (double)visited_cnt;
        in.unvisited_e = (double)std::max<int64_t>(edges_to_check, 0);
        in.max_deg = maxdeg;
        in.prev_nf = (double)prev_nf;
        return in;
    };

    // device-resident levels for small frontiers (not while collecting
    // samples, which time each level's variants on the host)
    const bool persist_ok = !tracing && !collect && o.schedule != CGB_SCHED_FIXED;
    while (nf > 0) {
        CGB_REQUIRE(iters < max_iters, CGB_ETIMEOUT, "BFS iteration budget exhausted");
        // ----- direction decision
        const bool heur = bottom_up ? (awake >= old_awake) || ((double)awake > (double)V / beta)
                                    : (double)scout > (double)edges_to_check / alpha;
        // small frontiers far from the switch point: run levels on the device
        if (persist_ok && !heur && nf <= g->tune.persist_enter && maxdeg < g->tune.persist_deg &&
            (double)scout * alpha * 4.0 <= (double)edges_to_check) {
            if (timing) ktimer_begin(g, CGB_K_PUSH);
            const unsigned long long scout_exit = (unsigned long long)((double)edges_to_check / alpha / 4.0);
            const PersistResult r =
                bfs_persistent(g, cur, (uint32_t)nf, scout, maxdeg, level, g->tune.persist_enter, scout_exit, g->tune.persist_deg,
                               (uint32_t)std::min<uint64_t>(max_iters - iters, 1u << 20));
            if (timing) ktimer_end(g);
            if (r.levels > 0) {
                visited_cnt += r.added - nf + r.nf;
                edges_to_check -= (int64_t)r.scouts;
                iters += r.levels;
                level += r.levels;
                g->stats.pushes_td += r.levels;
                prev_nf = nf;
                nf = r.nf;
                scout = r.scout;
                maxdeg = r.max_deg;
                cur = r.cur;
                bottom_up = false;
                have_policy_out = false;
                continue;
            }
        }
        const int out = cur ^ 1;
        // the heuristic's expansion of a push level: every list of 32 edges or
        // more chunked for small frontiers, else the degree-binned tiers
        const int heur_expand = nf <= kSmallFrontier ? kExpandChunked : kExpandBinned;
        bool go_pull;
        int expand = heur_expand;
        if (force_pull) go_pull = true;
        else if (!want_pull) go_pull = false;
        else if (collect) {
            // counterfactual: time the three level variants from the same state
            const size_t vbytes = (size_t)V * 4, wbytes = (size_t)words * 4;
            CGB_CUDA_TRY(cudaMemcpyAsync(collect->save_value, g->value, vbytes, cudaMemcpyDeviceToDevice, g->stream));
            CGB_CUDA_TRY(cudaMemcpyAsync(collect->save_bm0, g->visited, wbytes, cudaMemcpyDeviceToDevice, g->stream));
            float ms[kPolicyOutputs] = {};
            bool have[kPolicyOutputs] = {};
            const int outs[3] = {kOutPush, kOutPull, kOutPushChunked};
            // every trial starts right after a restore, the first one too: after
            // the snapshot copy alone the levels array is colder in L2, and the
            // first variant timed slower than it runs (a bias toward the others)
            CGB_CUDA_TRY(cudaMemcpyAsync(g->value, collect->save_value, vbytes, cudaMemcpyDeviceToDevice, g->stream));
            CGB_CUDA_TRY(cudaMemcpyAsync(g->visited, collect->save_bm0, wbytes, cudaMemcpyDeviceToDevice, g->stream));
            for (int d = 0; d < 3; d++) {
                CGB_CUDA_TRY(cudaEventRecord(g->ev_iter[0], g->stream));
                do_level(d == 1, out, d == 2 ? kExpandChunked : kExpandBinned);
                CGB_CUDA_TRY(cudaEventRecord(g->ev_iter[1], g->stream));
                sync_counters(g);
                CGB_CUDA_TRY(cudaEventElapsedTime(&ms[outs[d]], g->ev_iter[0], g->ev_iter[1]));
                have[outs[d]] = true;
                CGB_CUDA_TRY(cudaMemcpyAsync(g->value, collect->save_value, vbytes, cudaMemcpyDeviceToDevice,
                                             g->stream));
                CGB_CUDA_TRY(cudaMemcpyAsync(g->visited, collect->save_bm0, wbytes, cudaMemcpyDeviceToDevice,
                                             g->stream));
            }
            policy_log_sample(g, state_now(), ms, have);
            int best = 0;
            for (int d = 1; d < 3; d++)
                if (ms[outs[d]] < ms[outs[best]]) best = d;
            go_pull = best == 1;
            expand = best == 2 ? kExpandChunked : kExpandBinned;
        } else if (pol && have_policy_out) {
            const int hc = heur ? 1 : (heur_expand == kExpandChunked ? 2 : 0);
            const int choice = policy_pick_bfs_level(g->h_ctr->policy_out, hc);
            go_pull = choice < 0 ? heur : choice == 1;
            if (choice == 0) expand = kExpandBinned;
            if (choice == 2) expand = kExpandChunked;
        } else {
            go_pull = heur;
        }

        float it_ms = 0.f;
        if (tracing) CGB_CUDA_TRY(cudaEventRecord(g->ev_iter[0], g->stream));
        const FeatIn before = state_now();
        do_level(go_pull, out, expand);
        if (go_pull) {
            if (!bottom_up) {
                awake = nf;
                old_awake = 0;
            }
            std::swap(front, next);
            g->stats.pulls_bu++;
        } else {
            g->stats.pushes_td++;
        }
        if (tracing) CGB_CUDA_TRY(cudaEventRecord(g->ev_iter[1], g->stream));
        // inference for the next level, fused before the counter read-back;
        // skipped while both Beamer ratios are far (64x) from their
        // thresholds, where the choice is not in doubt
        const double r_alpha = (double)scout * alpha / (double)std::max<int64_t>(edges_to_check, 1);
        const double r_beta = (double)nf * beta / (double)V;
        const bool near_boundary = (r_alpha > 1.0 / 64 && r_alpha < 64.0) || (r_beta > 1.0 / 64 && r_beta < 64.0);
        const bool infer = kPolicyLevels && pol && near_boundary;
        if (infer) {
            FeatIn in = before;
            in.unvisited_e = (double)std::max<int64_t>(edges_to_check - (int64_t)scout, 0);
            policy_enqueue(pol, g, in, 1, go_pull, out);
        }
        sync_counters(g);
        have_policy_out = infer;
        if (tracing) {
            CGB_CUDA_TRY(cudaEventElapsedTime(&it_ms, g->ev_iter[0], g->ev_iter[1]));
            cgb_iter_trace t{};
            t.iteration = (uint32_t)iters;
            t.algorithm = CGB_BFS;
            t.frontier_vertices = nf;
            t.frontier_edges = scout;
            t.unvisited_vertices = (uint64_t)V - visited_cnt;
            t.unvisited_edges = (uint64_t)std::max<int64_t>(edges_to_check, 0);
            t.max_frontier_degree = maxdeg;
            t.variant = go_pull ? CGB_VAR_PULL : CGB_VAR_TWC;
            t.ms = it_ms;
            g->trace.push_back(t);
        }
        CGB_REQUIRE(!g->h_ctr->overflow, CGB_EOVERFLOW, "BFS frontier queue overflow");
        const uint64_t n_next = g->h_ctr->qlen[out];
        const uint64_t m_next = g->h_ctr->medges;
        if (go_pull) {
            old_awake = awake;
            awake = g->h_ctr->found;
            visited_cnt += g->h_ctr->found;
        } else {
            visited_cnt += n_next;  // upper bound when nz < V; only steers the schedule
        }
        bottom_up = go_pull;
        edges_to_check -= (int64_t)scout;
        scout = m_next;
        maxdeg = g->h_ctr->max_deg;
        prev_nf = nf;
        nf = n_next;
        cur = out;
        level++;
        iters++;
    }
    CGB_CUDA_TRY(cudaEventRecord(g->ev_stop, g->stream));
    g->stats.iterations = iters;
}

}  // namespace cgb
