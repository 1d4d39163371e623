// Multi-root BFS with bit-packed per-root masks (up to 64 roots per pass).
//
// Every vertex carries three 64-bit masks: seen (roots that reached it),
// frontier (roots for which it is on the current level) and next (roots that
// reach it on the next level).  One traversal of an edge serves every root
// whose bit rides on it (the multi-source BFS of Then et al., VLDB 2014),
// so a batch of 64 roots costs a small multiple of one BFS instead of 64.
//   top-down  -- for each vertex of the active queue and each out-edge (v,u):
//                next[u] |= frontier[v] & ~seen[u] (atomicOr; the first
//                setter queues u), then a finalise pass moves next into
//                seen/frontier and writes the level of every new (root, u);
//   bottom-up -- every vertex not seen by all roots ORs the frontier masks of
//                its in-neighbours restricted to its missing roots, stopping
//                as soon as none is missing; one thread owns the vertex, so
//                its masks are written without atomics.
// Levels go to out[k * V + u] (root-major, 999999999 = unreachable), the
// layout of cgb_run_batch; they equal k separate cgb_run(CGB_BFS) results.
#include "msbfs.cuh"
#include "push.cuh"

namespace cgb {

__global__ void k_ms_init(uint32_t V, unsigned long long* seen, unsigned long long* f0, unsigned long long* next)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        seen[v] = 0;
        f0[v] = 0;
        next[v] = 0;
    }
}

__global__ void k_ms_fill(uint64_t n, uint32_t* a, uint32_t value)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        a[i] = value;
}

// Roots: seen/frontier bits, level 0, and the first active queue (a root
// listed twice still gets one queue entry).
__global__ void k_ms_roots(const uint32_t* roots, uint32_t n, uint32_t V, unsigned long long* seen,
                           unsigned long long* f0, uint32_t* level_out, uint32_t* q, uint32_t* qlen, uint32_t nz,
                           unsigned long long* alive)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (uint32_t k = 0; k < n; k++) {
        const uint32_t r = roots[k];
        if (!seen[r] && r < nz) q[(*qlen)++] = r;
        seen[r] |= 1ull << k;
        if (r < nz) {
            f0[r] |= 1ull << k;  // only vertices with out-edges are ever read as frontier
            *alive |= 1ull << k;
        }
        level_out[(size_t)k * V + r] = 0;
    }
}

// Moves next into seen / the new frontier for the queued vertices, writes
// their levels, and keeps those with new roots (and out-edges) active.
__global__ void __launch_bounds__(kBlock) k_ms_finalize(const uint32_t* __restrict__ q, uint32_t n,
                                                        const uint32_t* n_ptr, unsigned long long* seen, unsigned long long* next,
                                                        unsigned long long* fnext, uint32_t* level_out, uint32_t V,
                                                        uint32_t lvl, uint32_t nz, uint32_t* qact, uint32_t* qact_len,
                                                        uint32_t cap, DevCounters* ctr, const uint32_t* start,
                                                        unsigned long long* alive)
{
    if (n_ptr) n = *n_ptr;
    const uint32_t n_round = (n + 31u) & ~31u;
    unsigned long long live = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_round; i += gridDim.x * blockDim.x) {
        bool act = false;
        uint32_t u = 0;
        if (i < n) {
            u = q[i];
            const unsigned long long x = next[u] & ~seen[u];
            next[u] = 0;
            if (x) {
                seen[u] |= x;
                for (unsigned long long m = x; m; m &= m - 1) {
                    const uint32_t k = __ffsll(m) - 1;
                    level_out[(size_t)k * V + u] = start ? lvl - start[k] : lvl;
                }
                act = u < nz;
                if (act) {
                    fnext[u] = x;
                    live |= x;
                }
            }
        }
        warp_append(act, u, qact, qact_len, cap, &ctr->overflow);
    }
    if (alive) {
        live = warp_or(live);
        if (lane_id() == 0 && live) atomicOr(alive, live);
    }
}

// Clears the frontier masks of the vertices of a queue.
__global__ void k_ms_clear(const uint32_t* __restrict__ q, uint32_t n, unsigned long long* f)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) f[q[i]] = 0;
}

// Bottom-up levels, binned by in-degree.  A vertex is done when every root
// it still misses (among the roots with a frontier, `full`) has been found
// in its in-neighbours' frontier masks -- rare while the roots sit at
// different depths, so lists are often walked to the end.  Walking a hub's
// list on one thread would make the hub the whole kernel's time, so:
//   k_ms_bu_light  -- the first kMsLight in-edges of every vertex, packed
//                     edge-parallel per CTA;
//                     vertices left unfinished go to a warp list (or, with
//                     at least kMsBlockDeg edges left, a CTA list) with the
//                     roots found so far parked in `acc` (the top-down
//                     scratch mask, zero between levels);
//   k_ms_bu_warp   -- a warp per listed vertex, lanes striding the list;
//   k_ms_bu_chunks -- hub lists cut into chunks over all CTAs, merged into
//                     acc by atomicOr; k_ms_bu_settle then finishes them.
// Each vertex has one owner at a time, so its masks and levels are written
// without atomics; new vertices with out-edges join the next queue.
constexpr uint32_t kMsLight = 32;
constexpr uint32_t kMsBlockDeg = 4096;

__device__ __forceinline__ unsigned long long warp_or64(unsigned long long v)
{
    const uint32_t lo = __reduce_or_sync(0xffffffffu, (uint32_t)v);
    const uint32_t hi = __reduce_or_sync(0xffffffffu, (uint32_t)(v >> 32));
    return ((unsigned long long)hi << 32) | lo;
}

// Records the roots `got` newly found for vertex u (its owner only).
__device__ __forceinline__ bool ms_bu_settle(uint32_t u, unsigned long long s, unsigned long long got,
                                             unsigned long long* seen, unsigned long long* fnext,
                                             uint32_t* level_out, uint32_t V, uint32_t lvl, uint32_t nz,
                                             const uint32_t* start)
{
    seen[u] = s | got;
    for (unsigned long long m = got; m; m &= m - 1) {
        const uint32_t k = __ffsll(m) - 1;
        level_out[(size_t)k * V + u] = start ? lvl - start[k] : lvl;
    }
    if (u < nz) fnext[u] = got;
    return u < nz;
}

__global__ void __launch_bounds__(kBlock) k_ms_bu_light(MsBuArgs a)
{
    // A CTA takes kBlock consecutive vertices; a CTA-wide exclusive scan
    // packs the first kMsLight in-edges of each into shared memory, one edge
    // per thread (coalesced reads of in_src), and the finds are ORed into
    // the owner's shared mask.
    __shared__ uint32_t s_scan[kBlock / 32 + 1];
    __shared__ uint32_t s_edge[kBlock];
    __shared__ uint32_t s_owner[kBlock];
    __shared__ unsigned long long s_acc[kBlock];
    __shared__ unsigned long long s_pend[kBlock];
    const uint32_t V = a.V, tid = threadIdx.x;
    unsigned long long live = 0;
    for (uint32_t base = blockIdx.x * kBlock; base < V; base += gridDim.x * kBlock) {
        const uint32_t u = base + tid;
        unsigned long long s = 0, pending = 0;
        uint32_t e0 = 0, deg = 0, cnt = 0;
        if (u < V) {
            s = a.seen[u];
            pending = a.full & ~s;
            if (pending) {
                e0 = a.in_off[u];
                deg = a.in_off[u + 1] - e0;
                cnt = min(deg, kMsLight);
            }
        }
        s_acc[tid] = 0;
        s_pend[tid] = pending;
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
                const uint32_t o = s_owner[tid];
                const unsigned long long x = a.front[a.in_src[s_edge[tid]]] & s_pend[o];
                if (x) atomicOr(&s_acc[o], x);
            }
            __syncthreads();
        }
        bool act = false, to_warp = false, to_block = false;
        if (pending) {
            const unsigned long long got = s_acc[tid];
            if (got != pending && deg > kMsLight) {
                a.acc[u] = got;  // finish on a warp or on hub chunks
                to_block = deg - kMsLight >= kMsBlockDeg;
                to_warp = !to_block;
            } else if (got) {
                act = ms_bu_settle(u, s, got, a.seen, a.fnext, a.level_out, V, a.lvl, a.nz, a.start);
                if (act) live |= got;
            }
        }
        warp_append(act, u, a.qact, a.qact_len, a.cap, &a.ctr->overflow);
        warp_append(to_warp, u, a.heavy_w, a.heavy_len, a.cap, &a.ctr->overflow);
        warp_append(to_block, u, a.heavy_b, a.heavy_len + 1, a.cap_b, &a.ctr->overflow);
        __syncthreads();  // s_acc / s_pend are rewritten by the next batch
    }
    if (a.alive) {
        live = warp_or(live);
        if (lane_id() == 0 && live) atomicOr(a.alive, live);
    }
}

__global__ void __launch_bounds__(kBlock) k_ms_bu_warp(MsBuArgs a)
{
    const uint32_t n = min(a.heavy_len[0], a.cap);
    const uint32_t lane = lane_id();
    unsigned long long live = 0;
    for (uint32_t i = blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5); i < n; i += gridDim.x * (kBlock / 32)) {
        const uint32_t u = a.heavy_w[i];
        const unsigned long long s = a.seen[u];
        const unsigned long long pending = a.full & ~s;
        unsigned long long got = a.acc[u];
        const uint32_t e1 = a.in_off[u + 1];
        for (uint32_t e = a.in_off[u] + kMsLight; e < e1 && got != pending; e += 128) {
            uint32_t src[4];
#pragma unroll
            for (int j = 0; j < 4; j++) src[j] = e + 32 * j + lane < e1 ? a.in_src[e + 32 * j + lane] : 0xFFFFFFFFu;
            unsigned long long x = 0;
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (src[j] != 0xFFFFFFFFu) x |= a.front[src[j]];
            got |= warp_or64(x & pending);
        }
        bool act = false;
        if (got) {
            // the new roots' levels: lane l writes roots l and l + 32
#pragma unroll
            for (uint32_t k = lane; k < 64; k += 32)
                if ((got >> k) & 1ull) a.level_out[(size_t)k * a.V + u] = a.start ? a.lvl - a.start[k] : a.lvl;
        }
        if (lane == 0) {
            a.acc[u] = 0;
            if (got) {
                a.seen[u] = s | got;
                act = u < a.nz;
                if (act) {
                    a.fnext[u] = got;
                    live |= got;
                }
            }
        }
        warp_append(act, u, a.qact, a.qact_len, a.cap, &a.ctr->overflow);
    }
    if (a.alive) {
        live = warp_or(live);
        if (lane == 0 && live) atomicOr(a.alive, live);
    }
}

// Hub lists: the rest of every listed vertex's list is cut into
// kMsBlockDeg-edge chunks dealt round-robin over the CTAs (a hub's chunks
// run on different SMs); each CTA ORs its chunk's finds into acc[u] and
// skips chunks of vertices already complete.
__global__ void __launch_bounds__(kBlock) k_ms_bu_chunks(MsBuArgs a)
{
    __shared__ unsigned long long s_got;
    const uint32_t n = min(a.heavy_len[1], a.cap_b);
    uint64_t chunk_base = 0;
    for (uint32_t i = 0; i < n; i++) {
        const uint32_t u = a.heavy_b[i];
        const uint32_t b0 = a.in_off[u] + kMsLight, e1 = a.in_off[u + 1];
        const uint32_t nch = (e1 - b0 + kMsBlockDeg - 1) / kMsBlockDeg;
        const unsigned long long pending = a.full & ~a.seen[u];
        const uint32_t first = (uint32_t)((blockIdx.x + gridDim.x - (chunk_base % gridDim.x)) % gridDim.x);
        chunk_base += nch;
        for (uint32_t c = first; c < nch; c += gridDim.x) {
            // complete already?  (one read, shared, so the whole CTA takes the same branch)
            __syncthreads();
            if (threadIdx.x == 0) s_got = *(volatile unsigned long long*)(a.acc + u);
            __syncthreads();
            if (s_got == pending) break;
            const uint32_t cs = b0 + c * kMsBlockDeg, ce = min(e1, cs + kMsBlockDeg);
            unsigned long long got = 0;
            for (uint32_t e = cs + threadIdx.x; e < ce; e += 4 * kBlock) {
                uint32_t src[4];
#pragma unroll
                for (int j = 0; j < 4; j++) src[j] = e + j * kBlock < ce ? a.in_src[e + j * kBlock] : 0xFFFFFFFFu;
#pragma unroll
                for (int j = 0; j < 4; j++)
                    if (src[j] != 0xFFFFFFFFu) got |= a.front[src[j]];
            }
            got = warp_or64(got & pending);
            if (threadIdx.x == 0) s_got = 0;
            __syncthreads();
            if (lane_id() == 0 && got) atomicOr(&s_got, got);
            __syncthreads();
            if (threadIdx.x == 0 && (s_got & ~*(volatile unsigned long long*)(a.acc + u))) atomicOr(a.acc + u, s_got);
            __syncthreads();
        }
    }
}

// Settles the listed hub vertices from their merged masks.
__global__ void __launch_bounds__(kBlock) k_ms_bu_settle(MsBuArgs a)
{
    const uint32_t n = min(a.heavy_len[1], a.cap_b);
    const uint32_t n_round = (n + 31u) & ~31u;
    unsigned long long live = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_round; i += gridDim.x * blockDim.x) {
        bool act = false;
        uint32_t u = 0;
        if (i < n) {
            u = a.heavy_b[i];
            const unsigned long long s = a.seen[u];
            const unsigned long long got = a.acc[u] & (a.full & ~s);
            a.acc[u] = 0;
            if (got) {
                act = ms_bu_settle(u, s, got, a.seen, a.fnext, a.level_out, a.V, a.lvl, a.nz, a.start);
                if (act) live |= got;
            }
        }
        warp_append(act, u, a.qact, a.qact_len, a.cap, &a.ctr->overflow);
    }
    if (a.alive) {
        live = warp_or(live);
        if (lane_id() == 0 && live) atomicOr(a.alive, live);
    }
}

void ms_bottom_up(const MsBuArgs& a, cudaStream_t st, uint64_t* launches)
{
    CGB_CUDA_TRY(cudaMemsetAsync(a.heavy_len, 0, 8, st));
    k_ms_bu_light<<<grid_for(a.V, kBlock, num_sms() * 8), kBlock, 0, st>>>(a);
    k_ms_bu_warp<<<num_sms() * 8, kBlock, 0, st>>>(a);
    k_ms_bu_chunks<<<num_sms() * 4, kBlock, 0, st>>>(a);
    k_ms_bu_settle<<<num_sms(), kBlock, 0, st>>>(a);
    if (launches) *launches += 4;
}

__global__ void k_ms_degree_sum(const uint32_t* __restrict__ q, uint32_t n, const uint32_t* n_ptr,
                                const uint32_t* __restrict__ off, DevCounters* ctr)
{
    if (n_ptr) n = *n_ptr;
    unsigned long long s = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t v = q[i];
        s += off[v + 1] - off[v];
    }
    s = warp_sum(s);
    if (lane_id() == 0 && s) atomicAdd(&ctr->medges, s);
}

unsigned long long* ms_alloc(size_t n)
{
    void* p = nullptr;
    CGB_CUDA_TRY(cudaMalloc(&p, (n ? n : 1) * 8));
    return (unsigned long long*)p;
}

// Runs one pass of up to 64 roots; level_out (device) receives n * V levels.
void run_msbfs(cgb_graph* g, const uint32_t* d_roots, uint32_t n, uint32_t* level_out, double alpha)
{
    CGB_REQUIRE(n >= 1 && n <= 64, CGB_EINVAL, "multi-root BFS takes 1..64 roots per pass");
    ensure_frontier(g);
    ensure_csc(g);
    const uint32_t V = g->V;
    if (!g->ms) g->ms = ms_buffers_alloc(V, g->E);
    MsBuffers& b = *g->ms;
    // Invariant at the start of a level: front[cur] is non-zero only at the
    // vertices of the active queue q[cur]; front[cur ^ 1] and next are zero.
    const unsigned long long full = n == 64 ? ~0ull : ((1ull << n) - 1);
    const uint32_t gridV = grid_for(V, kBlock, num_sms() * 8);
    ++g->stats.launches;
    k_ms_init<<<gridV, kBlock, 0, g->stream>>>(V, b.seen, b.front[0], b.next);
    CGB_CUDA_TRY(cudaMemsetAsync(b.front[1], 0, (size_t)V * 8, g->stream));
    ++g->stats.launches;
    k_ms_fill<<<num_sms() * 8, kBlock, 0, g->stream>>>((uint64_t)n * V, level_out, kValueMax);
    CGB_CUDA_TRY(cudaMemsetAsync(g->ctr, 0, sizeof(DevCounters), g->stream));
    ++g->stats.launches;
    k_ms_roots<<<1, 1, 0, g->stream>>>(d_roots, n, V, b.seen, b.front[0], level_out, g->q[0], &g->ctr->qlen[0], g->nz,
                                       &g->ctr->alive);
    sync_counters(g);
    uint64_t nact = g->h_ctr->qlen[0];
    // Roots with vertices in the current frontier.  Bottom-up looks only
    // for these: a root whose traversal has ended (a small component) would
    // otherwise keep every vertex scanning its whole in-list.
    unsigned long long live = g->h_ctr->alive & full;
    int cur = 0;
    uint32_t lvl = 0;
    while (nact > 0) {
        CGB_REQUIRE(lvl <= V, CGB_ETIMEOUT, "multi-root BFS level bound exceeded");
        // direction: out-edges of the active vertices against the graph's edges
        CGB_CUDA_TRY(cudaMemsetAsync(&g->ctr->medges, 0, 8, g->stream));
        ++g->stats.launches;
        k_ms_degree_sum<<<grid_for(nact, kBlock, num_sms() * 8), kBlock, 0, g->stream>>>(g->q[cur], (uint32_t)nact,
                                                                                      nullptr, g->off, g->ctr);
        sync_counters(g);
        const bool pull = (double)g->h_ctr->medges * alpha > (double)g->E;
        const bool tracing = (g->flags & CGB_FLAG_TRACE) != 0;
        const uint64_t level_edges = g->h_ctr->medges;
        if (tracing) CGB_CUDA_TRY(cudaEventRecord(g->ev_iter[0], g->stream));
        const int nxt = cur ^ 1;
        unsigned long long* fcur = b.front[cur];
        unsigned long long* fnxt = b.front[nxt];
        CGB_CUDA_TRY(cudaMemsetAsync(&g->ctr->qlen[nxt], 0, 4, g->stream));
        CGB_CUDA_TRY(cudaMemsetAsync(&g->ctr->alive, 0, 8, g->stream));
        if (pull) {
            MsBuArgs ba{V, g->in_off, g->in_src, fcur, b.seen, fnxt, b.next, live, level_out, lvl + 1, g->nz,
                        g->q[nxt], &g->ctr->qlen[nxt], V, g->ctr, nullptr, &g->ctr->alive, b.heavy_w, b.heavy_b,
                        b.heavy_len, b.cap_b};
            ms_bottom_up(ba, g->stream, &g->stats.launches);
            g->stats.pulls_bu++;
        } else {
            // expansion into next[]: touched vertices are queued once in stamp[]
            CGB_CUDA_TRY(cudaMemsetAsync(&g->ctr->found, 0, 4, g->stream));
            CGB_CUDA_TRY(cudaMemsetAsync(&g->ctr->chunk_len, 0, 4, g->stream));
            MsTdOp op{g->off, g->dst, fcur, b.seen, b.next, g->stamp, &g->ctr->found, V, g->ctr};
            launch_push(g, g->q[cur], (uint32_t)nact, op, false);
            sync_counters(g);
            CGB_REQUIRE(!g->h_ctr->overflow, CGB_EOVERFLOW, "multi-root BFS queue overflow");
            const uint32_t touched = g->h_ctr->found;
            if (touched) {
                ++g->stats.launches;
                k_ms_finalize<<<grid_for(touched, kBlock, num_sms() * 8), kBlock, 0, g->stream>>>(
                    g->stamp, touched, nullptr, b.seen, b.next, fnxt, level_out, V, lvl + 1, g->nz, g->q[nxt],
                    &g->ctr->qlen[nxt], V, g->ctr, nullptr, &g->ctr->alive);
            }
            g->stats.pushes_td++;
        }
        ++g->stats.launches;
        k_ms_clear<<<grid_for(nact, kBlock, num_sms() * 8), kBlock, 0, g->stream>>>(g->q[cur], (uint32_t)nact, fcur);
        sync_counters(g);
        CGB_REQUIRE(!g->h_ctr->overflow, CGB_EOVERFLOW, "multi-root BFS queue overflow");
        if (tracing) {
            CGB_CUDA_TRY(cudaEventRecord(g->ev_iter[1], g->stream));
            CGB_CUDA_TRY(cudaEventSynchronize(g->ev_iter[1]));
            cgb_iter_trace t{};
            t.iteration = lvl;
            t.algorithm = CGB_BFS;
            t.frontier_vertices = nact;
            t.frontier_edges = level_edges;
            t.variant = pull ? CGB_VAR_PULL : CGB_VAR_TWC;
            CGB_CUDA_TRY(cudaEventElapsedTime(&t.ms, g->ev_iter[0], g->ev_iter[1]));
            g->trace.push_back(t);
        }
        nact = g->h_ctr->qlen[nxt];
        live = g->h_ctr->alive;
        cur = nxt;
        lvl++;
    }
    g->stats.iterations = lvl;
}

MsBuffers* ms_buffers_alloc(uint32_t V, uint64_t E)
{
    auto* b = new MsBuffers();
    try {
        b->seen = ms_alloc(V);
        b->front[0] = ms_alloc(V);
        b->front[1] = ms_alloc(V);
        b->next = ms_alloc(V);
        CGB_CUDA_TRY(cudaMemset(b->next, 0, (size_t)V * 8));  // zero between levels (bottom-up parks masks here)
        CGB_CUDA_TRY(cudaMalloc((void**)&b->heavy_w, (size_t)V * 4));
        b->cap_b = (uint32_t)std::min<uint64_t>(E / kMsBlockDeg + 2, V);
        CGB_CUDA_TRY(cudaMalloc((void**)&b->heavy_b, (size_t)b->cap_b * 4));
        CGB_CUDA_TRY(cudaMalloc((void**)&b->heavy_len, 8));
    } catch (...) {
        ms_buffers_free(b);
        throw;
    }
    return b;
}

void ms_buffers_free(MsBuffers* b)
{
    if (!b) return;
    cudaFree(b->seen);
    cudaFree(b->front[0]);
    cudaFree(b->front[1]);
    cudaFree(b->next);
    cudaFree(b->heavy_w);
    cudaFree(b->heavy_b);
    cudaFree(b->heavy_len);
    delete b;
}

void free_msbfs(cgb_graph* g)
{
    ms_buffers_free(g->ms);
    g->ms = nullptr;
}

}  // namespace cgb
