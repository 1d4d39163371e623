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
                           unsigned long long* f0, uint32_t* level_out, uint32_t* q, uint32_t* qlen, uint32_t nz)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (uint32_t k = 0; k < n; k++) {
        const uint32_t r = roots[k];
        if (!seen[r] && r < nz) q[(*qlen)++] = r;
        seen[r] |= 1ull << k;
        if (r < nz) f0[r] |= 1ull << k;  // only vertices with out-edges are ever read as frontier
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

// One bottom-up level over all vertices.
__global__ void __launch_bounds__(kBlock) k_ms_bu(uint32_t V, const uint32_t* __restrict__ in_off,
                                                  const uint32_t* __restrict__ in_src,
                                                  const unsigned long long* __restrict__ front,
                                                  unsigned long long* seen, unsigned long long* fnext,
                                                  unsigned long long full, uint32_t* level_out, uint32_t lvl,
                                                  uint32_t nz, uint32_t* qact, uint32_t* qact_len, uint32_t cap,
                                                  DevCounters* ctr, const uint32_t* start, unsigned long long* alive)
{
    const uint32_t n_round = (V + 31u) & ~31u;
    unsigned long long live = 0;
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n_round; u += gridDim.x * blockDim.x) {
        bool act = false;
        if (u < V) {
            const unsigned long long s = seen[u];
            const unsigned long long pending = full & ~s;
            if (pending) {
                unsigned long long got = 0;
                const uint32_t e1 = in_off[u + 1];
                for (uint32_t e = in_off[u]; e < e1; e++) {
                    got |= front[in_src[e]] & pending;
                    if (got == pending) break;
                }
                if (got) {
                    seen[u] = s | got;
                    for (unsigned long long m = got; m; m &= m - 1) {
                        const uint32_t k = __ffsll(m) - 1;
                        level_out[(size_t)k * V + u] = start ? lvl - start[k] : lvl;
                    }
                    act = u < nz;
                    if (act) {
                        fnext[u] = got;
                        live |= got;
                    }
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
void run_msbfs(cgb_graph* g, const uint32_t* d_roots, uint32_t n, uint32_t* level_out)
{
    CGB_REQUIRE(n >= 1 && n <= 64, CGB_EINVAL, "multi-root BFS takes 1..64 roots per pass");
    ensure_frontier(g);
    ensure_csc(g);
    const uint32_t V = g->V;
    if (!g->ms) {
        g->ms = new MsBuffers();
        g->ms->seen = ms_alloc(V);
        g->ms->front[0] = ms_alloc(V);
        g->ms->front[1] = ms_alloc(V);
        g->ms->next = ms_alloc(V);
    }
    MsBuffers& b = *g->ms;
    // Invariant at the start of a level: front[cur] is non-zero only at the
    // vertices of the active queue q[cur]; front[cur ^ 1] and next are zero.
    const unsigned long long full = n == 64 ? ~0ull : ((1ull << n) - 1);
    const uint32_t gridV = grid_for(V, kBlock, kNumSMs * 8);
    ++g->stats.launches;
    k_ms_init<<<gridV, kBlock, 0, g->stream>>>(V, b.seen, b.front[0], b.next);
    CGB_CUDA_TRY(cudaMemsetAsync(b.front[1], 0, (size_t)V * 8, g->stream));
    ++g->stats.launches;
    k_ms_fill<<<kNumSMs * 8, kBlock, 0, g->stream>>>((uint64_t)n * V, level_out, kValueMax);
    CGB_CUDA_TRY(cudaMemsetAsync(g->ctr, 0, sizeof(DevCounters), g->stream));
    ++g->stats.launches;
    k_ms_roots<<<1, 1, 0, g->stream>>>(d_roots, n, V, b.seen, b.front[0], level_out, g->q[0], &g->ctr->qlen[0], g->nz);
    sync_counters(g);
    uint64_t nact = g->h_ctr->qlen[0];
    int cur = 0;
    uint32_t lvl = 0;
    const double alpha = 15.0;
    while (nact > 0) {
        CGB_REQUIRE(lvl <= V, CGB_ETIMEOUT, "multi-root BFS level bound exceeded");
        // direction: out-edges of the active vertices against the graph's edges
        CGB_CUDA_TRY(cudaMemsetAsync(&g->ctr->medges, 0, 8, g->stream));
        ++g->stats.launches;
        k_ms_degree_sum<<<grid_for(nact, kBlock, kNumSMs * 8), kBlock, 0, g->stream>>>(g->q[cur], (uint32_t)nact,
                                                                                      nullptr, g->off, g->ctr);
        sync_counters(g);
        const bool pull = (double)g->h_ctr->medges * alpha > (double)g->E;
        const int nxt = cur ^ 1;
        unsigned long long* fcur = b.front[cur];
        unsigned long long* fnxt = b.front[nxt];
        CGB_CUDA_TRY(cudaMemsetAsync(&g->ctr->qlen[nxt], 0, 4, g->stream));
        if (pull) {
            ++g->stats.launches;
            k_ms_bu<<<grid_for(V, kBlock, kNumSMs * 16), kBlock, 0, g->stream>>>(
                V, g->in_off, g->in_src, fcur, b.seen, fnxt, full, level_out, lvl + 1, g->nz, g->q[nxt],
                &g->ctr->qlen[nxt], V, g->ctr, nullptr, nullptr);
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
                k_ms_finalize<<<grid_for(touched, kBlock, kNumSMs * 8), kBlock, 0, g->stream>>>(
                    g->stamp, touched, nullptr, b.seen, b.next, fnxt, level_out, V, lvl + 1, g->nz, g->q[nxt],
                    &g->ctr->qlen[nxt], V, g->ctr, nullptr, nullptr);
            }
            g->stats.pushes_td++;
        }
        ++g->stats.launches;
        k_ms_clear<<<grid_for(nact, kBlock, kNumSMs * 8), kBlock, 0, g->stream>>>(g->q[cur], (uint32_t)nact, fcur);
        sync_counters(g);
        CGB_REQUIRE(!g->h_ctr->overflow, CGB_EOVERFLOW, "multi-root BFS queue overflow");
        nact = g->h_ctr->qlen[nxt];
        cur = nxt;
        lvl++;
    }
    g->stats.iterations = lvl;
}

void free_msbfs(cgb_graph* g)
{
    if (!g->ms) return;
    cudaFree(g->ms->seen);
    cudaFree(g->ms->front[0]);
    cudaFree(g->ms->front[1]);
    cudaFree(g->ms->next);
    delete g->ms;
    g->ms = nullptr;
}

}  // namespace cgb
