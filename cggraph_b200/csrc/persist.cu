// Device-resident BFS levels and SSSP near rounds (see persist.cuh).
#include <cooperative_groups.h>

#include "persist.cuh"

namespace cgb {

// Shared expansion of one frontier held in qin[0, nf): a warp takes 32
// frontier vertices; lists of 32 or more edges are walked by the whole warp
// (ballot election), shorter ones lane by lane.  Visit(valid, e, msg) is
// warp-collective.
template <int kWarps = kBlock / 32, class Visit, class Load>
__device__ __forceinline__ void expand_small(const uint32_t* __restrict__ qin, uint32_t nf, const Load& load,
                                             const Visit& visit)
{
    const uint32_t lane = lane_id();
    const uint32_t nwarps = gridDim.x * kWarps;
    for (uint32_t base = (blockIdx.x * kWarps + (threadIdx.x >> 5)) * 32; base < nf; base += nwarps * 32) {
        const uint32_t i = base + lane;
        uint32_t start = 0, deg = 0, msg = 0;
        if (i < nf) load(qin[i], start, deg, msg);
        uint32_t wmask;
        while ((wmask = __ballot_sync(0xffffffffu, deg >= 32)) != 0) {
            const uint32_t leader = __ffs(wmask) - 1;
            const uint32_t st = __shfl_sync(0xffffffffu, start, leader);
            const uint32_t dg = __shfl_sync(0xffffffffu, deg, leader);
            const uint32_t m = __shfl_sync(0xffffffffu, msg, leader);
            if (lane == leader) deg = 0;
            for (uint32_t k = 0; k < dg; k += 32) visit(k + lane < dg, st + k + lane, m);
        }
        for (uint32_t j = 0; __any_sync(0xffffffffu, j < deg); j++) visit(j < deg, start + j, msg);
    }
}

__global__ void __launch_bounds__(kBlock) k_bfs_persistent(const uint32_t* __restrict__ off,
                                                           const uint32_t* __restrict__ dst, uint32_t* level,
                                                           uint32_t* visited, uint32_t* q0, uint32_t* q1, uint32_t cap,
                                                           uint32_t nz, uint32_t start_level, uint32_t cur,
                                                           uint32_t nf_exit, unsigned long long scout_exit,
                                                           uint32_t deg_exit, uint32_t max_levels, PersistState* st)
{
    uint32_t it = 0;
    for (; it < max_levels; it++) {
        const uint32_t s_cur = it % 3, s_next = (it + 1) % 3, s_zero = (it + 2) % 3;
        const uint32_t nf = *(volatile uint32_t*)&st->qlen[s_cur];
        const unsigned long long scout = *(volatile unsigned long long*)&st->medges[s_cur];
        const uint32_t mdeg = *(volatile uint32_t*)&st->max_deg[s_cur];
        if (nf == 0 || nf > nf_exit || scout > scout_exit || mdeg > deg_exit) break;
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            st->qlen[s_zero] = 0;
            st->medges[s_zero] = 0;
            st->max_deg[s_zero] = 0;
            st->added += nf;
            st->scouts += scout;
        }
        const uint32_t* qin = cur ? q1 : q0;
        uint32_t* qout = cur ? q0 : q1;
        const uint32_t next_level = start_level + it + 1;
        auto load = [&](uint32_t v, uint32_t& s, uint32_t& d, uint32_t& m) {
            s = off[v];
            d = off[v + 1] - s;
            m = 0;
        };
        auto visit = [&](bool valid, uint32_t e, uint32_t) {
            bool win = false;
            uint32_t d = 0;
            if (valid) {
                d = dst[e];
                const uint32_t bit = 1u << (d & 31u);
                uint32_t* wp = visited + (d >> 5);
                if (!(*wp & bit) && !(atomicOr(wp, bit) & bit)) {
                    win = true;
                    level[d] = next_level;
                }
            }
            const bool enq = win && d < nz;
            uint32_t deg = 0;
            if (enq) deg = off[d + 1] - off[d];
            append(enq, d, qout, &st->qlen[s_next], cap, st);
            if (__any_sync(0xffffffffu, enq)) {
                const unsigned long long sum = warp_sum((unsigned long long)deg);
                const uint32_t mx = warp_max(deg);
                if (lane_id() == 0) {
                    atomicAdd(&st->medges[s_next], sum);
                    atomicMax(&st->max_deg[s_next], mx);
                }
            }
        };
        expand_small(qin, nf, load, visit);
        if (!grid_barrier(st)) break;
        cur ^= 1;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->levels = it;
        st->cur = cur;
        st->nf = st->qlen[it % 3];
    }
}

// The same BFS level loop as one thread-block cluster (kThreads per CTA,
// up to 16 CTAs): levels are separated by the cluster's hardware barrier,
// which also orders the global-memory counters and bitmaps at cluster scope,
// instead of the grid barrier's global-memory round trip.  For frontiers of
// up to a few thousand vertices (a road-like grid's whole run), where the
// barrier is most of a level's time.  Every exit decision is read after the
// barrier from the same counter, so all threads leave together.
template <int kThreads>
__global__ void __launch_bounds__(kThreads, 1) k_bfs_cluster(const uint32_t* __restrict__ off,
                                                             const uint32_t* __restrict__ dst, uint32_t* level,
                                                             uint32_t* visited, uint32_t* q0, uint32_t* q1,
                                                             uint32_t cap, uint32_t nz, uint32_t start_level,
                                                             uint32_t cur, uint32_t nf_exit,
                                                             unsigned long long scout_exit, uint32_t deg_exit,
                                                             uint32_t max_levels, PersistState* st)
{
    cooperative_groups::cluster_group cluster = cooperative_groups::this_cluster();
    uint32_t it = 0;
    for (; it < max_levels; it++) {
        const uint32_t s_cur = it % 3, s_next = (it + 1) % 3, s_zero = (it + 2) % 3;
        const uint32_t nf = *(volatile uint32_t*)&st->qlen[s_cur];
        const unsigned long long scout = *(volatile unsigned long long*)&st->medges[s_cur];
        const uint32_t mdeg = *(volatile uint32_t*)&st->max_deg[s_cur];
        if (nf == 0 || nf > nf_exit || scout > scout_exit || mdeg > deg_exit) break;
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            st->qlen[s_zero] = 0;
            st->medges[s_zero] = 0;
            st->max_deg[s_zero] = 0;
            st->added += nf;
            st->scouts += scout;
        }
        const uint32_t* qin = cur ? q1 : q0;
        uint32_t* qout = cur ? q0 : q1;
        const uint32_t next_level = start_level + it + 1;
        auto load = [&](uint32_t v, uint32_t& s, uint32_t& d, uint32_t& m) {
            s = off[v];
            d = off[v + 1] - s;
            m = 0;
        };
        auto visit = [&](bool valid, uint32_t e, uint32_t) {
            bool win = false;
            uint32_t d = 0;
            if (valid) {
                d = dst[e];
                const uint32_t bit = 1u << (d & 31u);
                uint32_t* wp = visited + (d >> 5);
                if (!(*wp & bit) && !(atomicOr(wp, bit) & bit)) {
                    win = true;
                    level[d] = next_level;
                }
            }
            const bool enq = win && d < nz;
            uint32_t deg = 0;
            if (enq) deg = off[d + 1] - off[d];
            append(enq, d, qout, &st->qlen[s_next], cap, st);
            if (__any_sync(0xffffffffu, enq)) {
                const unsigned long long sum = warp_sum((unsigned long long)deg);
                const uint32_t mx = warp_max(deg);
                if (lane_id() == 0) {
                    atomicAdd(&st->medges[s_next], sum);
                    atomicMax(&st->max_deg[s_next], mx);
                }
            }
        };
        expand_small<kThreads / 32>(qin, nf, load, visit);
        cluster.sync();
        cur ^= 1;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->levels = it;
        st->cur = cur;
        st->nf = st->qlen[it % 3];
    }
}

// Whole delta-stepping SSSP on the device (graph batches, whose frontiers
// are small, and the tail of a single run once its frontiers are): each
// round either expands the near queue at the current threshold or, when it
// is empty and far vertices remain, splits the far bitmap at the next bucket
// [lo, hi) into a new near queue.  The thresholds, the smallest far
// distance, the change of the far count and the longest list of the next
// frontier rotate over the same three slots as the queue lengths; every CTA
// keeps the running far count itself by adding the previous round's change,
// so all CTAs take the same decision each round.  The loop leaves before a
// round whose frontier exceeds nf_exit vertices or holds a list of deg_exit
// edges or more (the host loop's binned kernels take those), and sx
// receives the far count and bucket bound the host continues from; the far
// count is also written to *far_len_out (the host loop's counter) when it is
// given.  Each split recounts the far bitmap's population rather than
// subtracting what it cleared, so a count that was off (it only decides
// when the run ends) is corrected at the next split.
template <bool kHasW>
__global__ void __launch_bounds__(kBlock) k_sssp_device(const uint32_t* __restrict__ off,
                                                        const uint32_t* __restrict__ dst,
                                                        const uint32_t* __restrict__ w, uint32_t* dist,
                                                        uint32_t* near_bm3, uint32_t words, uint32_t* far_bm,
                                                        uint32_t* q0, uint32_t* q1, uint32_t cap, uint32_t nz,
                                                        uint32_t delta, uint32_t max_rounds, uint32_t nf_exit,
                                                        uint32_t deg_exit, uint32_t cur, PersistState* st,
                                                        PersistSssp* sx, uint32_t* far_len_out)
{
    uint32_t it = 0, far = 0, far_now = 0;
    uint64_t bucket_lo = *(volatile unsigned long long*)&sx->bucket_lo;
    const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x, gthreads = gridDim.x * blockDim.x;
    const uint32_t lane = lane_id();
    for (; it < max_rounds; it++) {
        const uint32_t s_cur = it % 3, s_next = (it + 1) % 3, s_zero = (it + 2) % 3;
        const uint32_t nf = *(volatile uint32_t*)&st->qlen[s_cur];
        far_now = *(volatile uint32_t*)&sx->split[s_cur] ? *(volatile uint32_t*)&sx->kept[s_cur]
                                                          : far + *(volatile uint32_t*)&sx->far_delta[s_cur];
        const uint64_t thr = *(volatile unsigned long long*)&sx->thr[s_cur];
        const uint32_t min_far = *(volatile uint32_t*)&sx->min_far[s_cur];
        const uint32_t mdeg = *(volatile uint32_t*)&st->max_deg[s_cur];
        if (nf == 0 && far_now == 0) break;
        if (nf > nf_exit || mdeg >= deg_exit) break;
        far = far_now;
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            st->qlen[s_zero] = 0;
            st->max_deg[s_zero] = 0;
            sx->min_far[s_zero] = kValueMax;
            sx->far_delta[s_zero] = 0;
            sx->kept[s_zero] = 0;
            sx->split[s_zero] = 0;
            st->added += nf;
        }
        uint32_t* zero_bm = near_bm3 + (size_t)s_zero * words;
        for (uint32_t i = gtid; i < words; i += gthreads) zero_bm[i] = 0;
        const uint32_t* qin = cur ? q1 : q0;
        uint32_t* qout = cur ? q0 : q1;
        uint32_t mx = 0;  // longest list this thread appended to the next frontier
        if (nf > 0) {
            // expansion round at threshold thr
            if (blockIdx.x == 0 && threadIdx.x == 0) sx->thr[s_next] = thr;
            uint32_t* nbm = near_bm3 + (size_t)s_next * words;
            const uint32_t t = (uint32_t)(thr < kValueMax ? thr : kValueMax);
            auto load = [&](uint32_t v, uint32_t& s, uint32_t& d, uint32_t& m) {
                s = off[v];
                d = off[v + 1] - s;
                m = dist[v];
            };
            auto visit = [&](bool valid, uint32_t e, uint32_t du) {
                bool to_near = false, new_far = false;
                uint32_t d = 0;
                if (valid && du < kValueMax) {
                    d = dst[e];
                    const uint64_t cand = (uint64_t)du + (kHasW ? (uint64_t)w[e] : 1ull);
                    if (cand < kValueMax) {
                        const uint32_t nd = (uint32_t)cand;
                        if (nd < dist[d]) {
                            const uint32_t old = atomicMin(dist + d, nd);
                            if (nd < old && d < nz) {
                                const uint32_t bit = 1u << (d & 31u);
                                uint32_t* wp = (nd < t ? nbm : far_bm) + (d >> 5);
                                const bool fresh = !(*wp & bit) && !(atomicOr(wp, bit) & bit);
                                to_near = fresh && nd < t;
                                new_far = fresh && nd >= t;
                            }
                        }
                    }
                }
                append(to_near, d, qout, &st->qlen[s_next], cap, st);
                if (to_near) mx = max(mx, off[d + 1] - off[d]);
                const uint32_t nfar = __popc(__ballot_sync(0xffffffffu, new_far));
                if (nfar && lane_id() == 0) atomicAdd(&sx->far_delta[s_next], nfar);
            };
            expand_small(qin, nf, load, visit);
        } else {
            // split round: next bucket [lo, hi); after a split that found
            // nothing, jump straight to the bucket of the smallest far distance
            const uint64_t lo = thr;
            uint64_t hi = thr + delta;
            if (min_far != kValueMax) {
                const uint64_t j = ((uint64_t)min_far / delta + 1) * (uint64_t)delta;
                if (j > hi) hi = j;
            }
            bucket_lo = lo;
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                sx->thr[s_next] = hi;
                sx->split[s_next] = 1;
            }
            const uint32_t lo32 = (uint32_t)(lo < kValueMax ? lo : kValueMax);
            const uint32_t hi32 = (uint32_t)(hi < kValueMax ? hi : kValueMax);
            uint32_t mn = kValueMax, kept = 0;
            // a warp takes 4 x 32 words with four coalesced loads in flight
            // (the far bitmap is mostly empty on high-diameter graphs, so the
            // scan itself is most of a split); lane b of word j reads the
            // distance of vertex 32 j + b (coalesced); the warp owns its
            // words, so it writes back what stays without atomics
            const uint32_t gw = gtid / 32, nwarps = gthreads / 32;
            for (uint32_t w4 = gw * 128; w4 < words; w4 += nwarps * 128) {
                uint32_t mine[4];
#pragma unroll
                for (int k = 0; k < 4; k++) mine[k] = w4 + 32 * k + lane < words ? far_bm[w4 + 32 * k + lane] : 0u;
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const uint32_t w0 = w4 + 32 * k;
                    uint32_t todo = __ballot_sync(0xffffffffu, mine[k] != 0);
                    while (todo) {
                        const uint32_t j = __ffs(todo) - 1;
                        todo &= todo - 1;
                        const uint32_t bits = __shfl_sync(0xffffffffu, mine[k], j);
                        const uint32_t v = (w0 + j) * 32 + lane;
                        const bool in = (bits >> lane) & 1u;
                        const uint32_t dv = in ? dist[v] : 0u;
                        const bool leave = in && dv < hi32;
                        const bool to_near = leave && dv >= lo32;
                        const bool keep = in && !leave;
                        if (keep) mn = min(mn, dv);
                        const uint32_t km = __ballot_sync(0xffffffffu, keep);
                        if (lane == 0) {
                            if (km != bits) far_bm[w0 + j] = km;
                            kept += __popc(km);
                        }
                        if (to_near) mx = max(mx, off[v + 1] - off[v]);
                        append(to_near, v, qout, &st->qlen[s_next], cap, st);
                    }
                }
            }
            mn = __reduce_min_sync(0xffffffffu, mn);
            kept = warp_sum(kept);
            if (lane == 0) {
                if (mn != kValueMax) atomicMin(&sx->min_far[s_next], mn);
                if (kept) atomicAdd(&sx->kept[s_next], kept);
            }
        }
        mx = warp_max(mx);
        if (mx && lane == 0) atomicMax(&st->max_deg[s_next], mx);
        if (!grid_barrier(st)) break;
        cur ^= 1;  // both kinds of round wrote the other queue
    }
    if (it == max_rounds)
        far_now = *(volatile uint32_t*)&sx->split[it % 3] ? *(volatile uint32_t*)&sx->kept[it % 3]
                                                           : far + *(volatile uint32_t*)&sx->far_delta[it % 3];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->levels = it;
        st->cur = cur;
        st->nf = st->qlen[it % 3];
        sx->far_left = far_now;
        sx->bucket_lo = bucket_lo;
        if (far_len_out) *far_len_out = far_now;
    }
}

// ----------------------------------------------------------------- host
void launch_bfs_unbounded(cgb_graph* g, PersistState* st)
{
    uint32_t cap = g->V, nz = g->nz, lvl = 0, cur = 0, nf_exit = 0xFFFFFFFFu, deg_exit = 0xFFFFFFFFu;
    uint32_t max_levels = g->V + 2;
    unsigned long long scout_exit = ~0ull;
    void* args[] = {&g->off, &g->dst, &g->value, &g->visited, &g->q[0], &g->q[1], &cap, &nz, &lvl, &cur, &nf_exit,
                    &scout_exit, &deg_exit, &max_levels, &st};
    CGB_CUDA_TRY(cudaLaunchCooperativeKernel((void*)k_bfs_persistent, num_sms(), kBlock, args, 0, g->stream));
}

void launch_sssp_device(cgb_graph* g, uint32_t* far_bm, uint32_t delta, PersistState* st, PersistSssp* sx)
{
    uint32_t cap = g->V, nz = g->nz, words = g->words(), rounds = 0xFFFFFFF0u;
    uint32_t nf_exit = 0xFFFFFFFFu, deg_exit = 0xFFFFFFFFu, cur = 0;
    uint32_t* nbm = g->aux_bm;
    uint32_t* far_len_out = nullptr;
    void* args[] = {&g->off, &g->dst, &g->w, &g->value, &nbm, &words, &far_bm, &g->q[0], &g->q[1], &cap, &nz, &delta,
                    &rounds, &nf_exit, &deg_exit, &cur, &st, &sx, &far_len_out};
    if (g->w)
        CGB_CUDA_TRY(cudaLaunchCooperativeKernel((void*)k_sssp_device<true>, num_sms(), kBlock, args, 0, g->stream));
    else
        CGB_CUDA_TRY(cudaLaunchCooperativeKernel((void*)k_sssp_device<false>, num_sms(), kBlock, args, 0, g->stream));
}

static PersistBlock* persist_block(cgb_graph* g)
{
    if (!g->persist) g->persist = pool_alloc(sizeof(PersistBlock), g->stream);
    return static_cast<PersistBlock*>(g->persist);
}

static PersistState* persist_state(cgb_graph* g) { return &persist_block(g)->st; }

// The graph's pinned host block for the state (pinned: a pageable copy waits
// for other threads' pageable copies, see pinned_acquire).
static PersistBlock* host_block(cgb_graph* g)
{
    if (!g->h_persist) {
        g->h_persist = pinned_acquire(sizeof(PersistBlock));
        g->h_persist_bytes = sizeof(PersistBlock);
    }
    return static_cast<PersistBlock*>(g->h_persist);
}

static PersistState* host_state(cgb_graph* g) { return &host_block(g)->st; }

// Host copy of the state after a launch (synchronises the stream).
static PersistState read_state(cgb_graph* g)
{
    PersistState* hp = host_state(g);
    CGB_CUDA_TRY(cudaMemcpyAsync(hp, g->persist, sizeof(PersistState), cudaMemcpyDeviceToHost, g->stream));
    CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    const PersistState h = *hp;
    CGB_REQUIRE(!(h.status & 2u), CGB_EOVERFLOW, "device-resident loop: queue overflow");
    CGB_REQUIRE(!(h.status & 1u), CGB_ETIMEOUT, "device-resident loop: grid barrier gave up");
    return h;
}

static void init_state(cgb_graph* g, uint32_t nf, unsigned long long scout, uint32_t max_deg)
{
    // the graph's pinned state block: its previous copy has completed, since
    // every launch is followed by read_state (a synchronisation)
    PersistState& h = *host_state(g);
    h = PersistState{};
    h.qlen[0] = nf;
    h.medges[0] = scout;
    h.max_deg[0] = max_deg;
    static_assert(sizeof(PersistState) % 4 == 0, "copied as words");
    h2d_small(g->persist, &h, sizeof(PersistState), g->stream);
}

// CTAs of the level-loop cluster: 16 when the device schedules such a
// cluster of kClusterThreads-thread CTAs (a non-portable size), else 8, else
// 0 (no cluster path).  Decided once per process.
static uint32_t cluster_size()
{
    static int size = -1;
    if (size >= 0) return (uint32_t)size;
    size = 0;
    auto kern = k_bfs_cluster<kClusterThreads>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
    }
    for (int c : {16, 8}) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(c);
        cfg.blockDim = dim3(kClusterThreads);
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = c;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) == cudaSuccess && n > 0) {
            size = c;
            break;
        }
        cudaGetLastError();
    }
    return (uint32_t)size;
}

PersistResult bfs_persistent(cgb_graph* g, uint32_t cur, uint32_t nf, unsigned long long scout, uint32_t max_deg,
                             uint32_t level, uint32_t nf_exit, unsigned long long scout_exit, uint32_t deg_exit,
                             uint32_t max_levels)
{
    PersistState* st = persist_state(g);
    init_state(g, nf, scout, max_deg);
    uint32_t cap = g->V, nz = g->nz;
    ++g->stats.launches;
    const uint32_t csize = cluster_size();
    if (csize && nf <= g->tune.cluster_enter) {
        // small frontier: one cluster, hardware barrier between levels; back to
        // the caller when the frontier outgrows twice the entry size
        const uint32_t c_exit = std::min(nf_exit, 2 * g->tune.cluster_enter);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(csize);
        cfg.blockDim = dim3(kClusterThreads);
        cfg.stream = g->stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = csize;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        CGB_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_bfs_cluster<kClusterThreads>, g->off, g->dst, g->value, g->visited,
                                        g->q[0], g->q[1], cap, nz, level, cur, c_exit, scout_exit, deg_exit,
                                        max_levels, st));
    } else {
        static uint32_t full = 0;
        if (!full) full = cooperative_grid(k_bfs_persistent);
        const uint32_t grid = g->tune.persist_ctas ? std::min(g->tune.persist_ctas, full) : full;
        void* args[] = {&g->off, &g->dst, &g->value, &g->visited, &g->q[0], &g->q[1], &cap, &nz, &level, &cur,
                        &nf_exit, &scout_exit, &deg_exit, &max_levels, &st};
        CGB_CUDA_TRY(cudaLaunchCooperativeKernel((void*)k_bfs_persistent, grid, kBlock, args, 0, g->stream));
    }
    const PersistState h = read_state(g);
    PersistResult r;
    r.levels = h.levels;
    r.cur = h.cur;
    r.nf = h.nf;
    r.scout = h.medges[h.levels % 3];
    r.max_deg = h.max_deg[h.levels % 3];
    r.added = h.added;
    r.scouts = h.scouts;
    return r;
}

SsspTail sssp_device_tail(cgb_graph* g, uint32_t cur, uint32_t nf, uint32_t max_deg, uint64_t thr, uint32_t nfar,
                          uint64_t bucket_lo, uint32_t* far_bm, uint32_t delta, uint32_t nf_exit, uint32_t deg_exit,
                          uint32_t max_rounds)
{
    PersistBlock* blk = persist_block(g);
    PersistState* st = &blk->st;
    PersistSssp* sx = &blk->sx;
    // the pinned host block: its previous copy has completed, since every
    // launch is followed by a synchronising read-back
    PersistBlock& h = *host_block(g);
    h = PersistBlock{};
    h.st.qlen[0] = nf;
    h.st.max_deg[0] = max_deg;
    h.sx.thr[0] = thr;
    for (int k = 0; k < 3; k++) h.sx.min_far[k] = kValueMax;
    h.sx.far_delta[0] = nfar;
    h.sx.bucket_lo = bucket_lo;
    static_assert(sizeof(PersistBlock) % 4 == 0, "copied as words");
    h2d_small(blk, &h, sizeof(PersistBlock), g->stream);
    const uint32_t words = g->words();
    // round 0 appends against near bitmap slot 1; slot 2 is zeroed by round 0
    CGB_CUDA_TRY(cudaMemsetAsync(g->aux_bm + (size_t)words, 0, (size_t)words * 4, g->stream));
    uint32_t cap = g->V, nz = g->nz;
    uint32_t* nbm = g->aux_bm;
    uint32_t* far_len_out = &g->ctr->far_len[0];  // the host loop's far count continues from the tail's
    void* args[] = {&g->off, &g->dst, &g->w, &g->value, &nbm, (void*)&words, &far_bm, &g->q[0], &g->q[1], &cap, &nz,
                    &delta, &max_rounds, &nf_exit, &deg_exit, &cur, &st, &sx, &far_len_out};
    ++g->stats.launches;
    if (g->w) {
        static uint32_t full = 0;
        if (!full) full = cooperative_grid(k_sssp_device<true>);
        const uint32_t grid = g->tune.persist_ctas ? std::min(g->tune.persist_ctas, full) : full;
        CGB_CUDA_TRY(cudaLaunchCooperativeKernel((void*)k_sssp_device<true>, grid, kBlock, args, 0, g->stream));
    } else {
        static uint32_t full = 0;
        if (!full) full = cooperative_grid(k_sssp_device<false>);
        const uint32_t grid = g->tune.persist_ctas ? std::min(g->tune.persist_ctas, full) : full;
        CGB_CUDA_TRY(cudaLaunchCooperativeKernel((void*)k_sssp_device<false>, grid, kBlock, args, 0, g->stream));
    }
    CGB_CUDA_TRY(cudaMemcpyAsync(&h.sx, sx, sizeof(PersistSssp), cudaMemcpyDeviceToHost, g->stream));
    const PersistState hs = read_state(g);  // synchronises
    SsspTail t;
    t.r.levels = hs.levels;
    t.r.cur = hs.cur;
    t.r.nf = hs.nf;
    t.r.max_deg = hs.max_deg[hs.levels % 3];
    t.r.added = hs.added;
    t.thr = h.sx.thr[hs.levels % 3];
    t.nfar = h.sx.far_left;
    t.bucket_lo = h.sx.bucket_lo;
    return t;
}

// CTA 0 leaves at once; the others wait at the barrier for a release that
// never comes and give up after spin_limit polls.
__global__ void k_barrier_timeout(PersistState* st, uint32_t spin_limit)
{
    if (blockIdx.x == 0) return;
    grid_barrier(st, spin_limit);
}

cgb_status barrier_timeout_check(uint32_t spin_limit)
{
    PersistState* st = nullptr;
    CGB_CUDA_TRY(cudaMalloc((void**)&st, sizeof(PersistState)));
    cudaStream_t s = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    PersistState h{};
    if (e == cudaSuccess) e = cudaMemsetAsync(st, 0, sizeof(PersistState), s);
    if (e == cudaSuccess) {
        const uint32_t grid = cooperative_grid(k_barrier_timeout);
        void* args[] = {&st, &spin_limit};
        e = cudaLaunchCooperativeKernel((void*)k_barrier_timeout, grid, kBlock, args, 0, s);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, st, sizeof(PersistState), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (s) cudaStreamDestroy(s);
    cudaFree(st);
    CGB_CUDA_TRY(e);
    return (h.status & 1u) ? CGB_ETIMEOUT : CGB_OK;
}

}  // namespace cgb
