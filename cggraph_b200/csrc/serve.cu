// Request server: BFS and SSSP root queries against one resident graph with
// continuous batching (no counterpart in the reference, whose drivers run
// one root at a time, my_project/CGgraph/main_partition.hpp:188-227).
//
// Each algorithm has a group of up to 64 slots that share one traversal
// with bit-packed per-vertex root masks (the multi-root engines of
// msbfs.cu / mssp.cu).  The server thread runs ticks; a tick
//   1. admits requests whose arrival time has passed into free slots (a
//      slot is free once the previous occupant's result has been copied
//      out, and the slots of a group are capped so that their result
//      regions fit the memory budget);
//   2. advances every active slot by one BFS level / one SSSP round, all
//      slots of a group in the same kernels; each group has its own host
//      thread and stream (the BFS group the graph's), so the two overlap on
//      the device and short BFS levels never wait for SSSP rounds;
//   3. retires the slots whose traversal ended (no frontier bits left for
//      them), copying their results out and freeing the slot.
// A request admitted while others run starts at its own level 0 (BFS
// levels are written as tick - start[slot]) and keeps its own delta-stepping
// buckets (SSSP thresholds per slot), so its result equals a lone cgb_run.
// All traversal state stays in HBM; the host only decides admissions and
// reads a few counters per tick.
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>
#include <vector>

#include "../../include/cgb200.h"
#include "engine.cuh"
#include "msbfs.cuh"
#include "mssp.cuh"
#include "persist.cuh"
#include "push.cuh"

namespace cgb {

// One run of the single-root engine (capi.cu), with the graph's lock held.
void run_one(cgb_graph* g, int alg, uint32_t root_or_iters, const cgb_options& o);

constexpr uint32_t kSrvSlots = 64;

// ---------------------------------------------------------------- kernels

// Clears the bits of `mask` from every vertex's seen mask (slots reused).
__global__ void k_srv_clear_bits(uint32_t V, unsigned long long* seen, unsigned long long mask)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x)
        if (seen[v] & mask) seen[v] &= ~mask;
}

// BFS admissions: n pairs (slot, root); roots with out-edges join the
// current frontier at q[qpos + j] (j = rank among them, computed on the host).
__global__ void k_srv_bfs_admit(uint32_t n, const uint32_t* __restrict__ slots, const uint32_t* __restrict__ roots,
                                const uint32_t* __restrict__ qidx, uint32_t V, uint32_t* region,
                                unsigned long long* seen, unsigned long long* front, uint32_t* q)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t k = slots[i], r = roots[i];
    region[(size_t)k * V + r] = 0;
    atomicOr(seen + r, 1ull << k);
    if (qidx[i] != 0xFFFFFFFFu) {
        atomicOr(front + r, 1ull << k);
        q[qidx[i]] = r;
    }
}

// Per finished slot (bit k of mask): traversed edges (out-degrees of the
// reached vertices), reached vertices and the largest finite value of
// region k.
__global__ void __launch_bounds__(kBlock) k_srv_stats(const uint32_t* __restrict__ region, uint32_t V,
                                                      const uint32_t* __restrict__ off, unsigned long long mask,
                                                      unsigned long long* edges, uint32_t* reached, uint32_t* depth)
{
    const uint32_t n_round = (V + 31u) & ~31u;
    for (unsigned long long m = mask; m; m &= m - 1) {
        const uint32_t k = __ffsll(m) - 1;
        const uint32_t* r = region + (size_t)k * V;
        unsigned long long e = 0;
        uint32_t cnt = 0, mx = 0;
        for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n_round; v += gridDim.x * blockDim.x) {
            if (v < V) {
                const uint32_t x = r[v];
                if (x != kValueMax) {
                    e += off[v + 1] - off[v];
                    cnt++;
                    mx = max(mx, x);
                }
            }
        }
        e = warp_sum(e);
        cnt = warp_sum(cnt);
        mx = warp_max(mx);
        if (lane_id() == 0) {
            if (e) atomicAdd(edges + k, e);
            if (cnt) atomicAdd(reached + k, cnt);
            if (mx) atomicMax(depth + k, mx);
        }
    }
}

// SSSP: distances of the slots in mask back to MAX (slots reused), a warp
// per vertex with lanes over slots.
__global__ void k_srv_sp_reset(uint32_t V, uint32_t* dist, unsigned long long mask)
{
    const uint32_t lane = lane_id();
    const bool m0 = (mask >> lane) & 1ull, m1 = (mask >> (lane + 32)) & 1ull;
    for (uint32_t v = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); v < V; v += gridDim.x * (blockDim.x / 32)) {
        uint32_t* row = dist + (size_t)v * kMsRoots;
        if (m0) row[lane] = kValueMax;
        if (m1) row[lane + 32] = kValueMax;
    }
}

// SSSP admissions: dist[root][slot] = 0 and the root queued (once) in q.
__global__ void k_srv_sp_admit(uint32_t n, const uint32_t* __restrict__ slots, const uint32_t* __restrict__ roots,
                               uint32_t* dist, unsigned long long* pend, uint32_t* q, uint32_t* q_len, uint32_t cap,
                               MsspCounters* c)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t k = slots[i], r = roots[i];
    dist[(size_t)r * kMsRoots + k] = 0;
    if (atomicOr(pend + r, 1ull << k) == 0ull) {
        const uint32_t p = atomicAdd(q_len, 1u);
        if (p < cap) q[p] = r;
        else atomicOr(&c->overflow, 1u);
    }
}

// SSSP results of the slots in mask: region[k * V + v] = dist[v][k],
// through a 32-vertex x 64-slot shared tile.
__global__ void __launch_bounds__(kBlock) k_srv_sp_extract(const uint32_t* __restrict__ dist, uint32_t V,
                                                           unsigned long long mask, uint32_t* region)
{
    __shared__ uint32_t tile[32][kMsRoots + 1];
    __shared__ uint8_t ks[kMsRoots];
    uint32_t n = 0;
    for (unsigned long long m = mask; m; m &= m - 1) {
        if (threadIdx.x == 0) ks[n] = (uint8_t)(__ffsll(m) - 1);
        n++;
    }
    __syncthreads();
    const uint32_t tiles = (V + 31) / 32;
    for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        const uint32_t v0 = t * 32;
        for (uint32_t i = threadIdx.x; i < 32 * kMsRoots; i += blockDim.x) {
            const uint32_t r = i / kMsRoots, k = i % kMsRoots;
            if (v0 + r < V) tile[r][k] = dist[(size_t)(v0 + r) * kMsRoots + k];
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < 32 * n; i += blockDim.x) {
            const uint32_t k = ks[i / 32], r = i % 32;
            if (v0 + r < V) region[(size_t)k * V + v0 + r] = tile[r][k];
        }
        __syncthreads();
    }
}

// The same for a few finished slots (ks[0..n)): reads only their columns (one
// 32-byte sector per vertex and slot) instead of whole 256-byte rows.
__global__ void k_srv_sp_extract_cols(const uint32_t* __restrict__ dist, uint32_t V, uint4 ks, uint32_t n,
                                      uint32_t* region)
{
    const uint32_t k[4] = {ks.x, ks.y, ks.z, ks.w};
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        const uint32_t* row = dist + (size_t)v * kMsRoots;
#pragma unroll
        for (uint32_t i = 0; i < 4; i++)
            if (i < n) region[(size_t)k[i] * V + v] = row[k[i]];
    }
}

__global__ void k_srv_copy_u32(const uint32_t* src, uint32_t* dst) { *dst = *src; }

// ------------------------------------------------ device-resident BFS levels
//
// The BFS group's levels run on the device, many per launch: one
// cooperative kernel (one CTA per SM) separates the phases of a level with
// the bounded grid barrier of persist.cuh and keeps going until
//   - a slot's traversal ended (its result can be copied out: the host
//     retires it),
//   - the host raised the pinned mailbox (a query waits for a free slot:
//     the host admits it), checked after every level,
//   - the time budget ran out, or
//   - the frontier outgrew the loop (more than nf_exit vertices, or enough
//     out-edges that a bottom-up level is cheaper: the host loop's kernels
//     take those levels).
// A level is the top-down multi-root step of msbfs.cu: every frontier
// vertex v offers its roots front[v] & ~seen[u] to each out-neighbour u
// (atomicOr into next[u]; the first setter lists u), lists of kLoopHub
// edges or more are cut into kLoopChunk-edge chunks that every warp takes
// part in, then the listed vertices keep their new roots, write their
// levels (level - start[slot]) and form the next frontier.

constexpr uint32_t kLoopHub = 2048;    // lists at least this long are chunked across the grid
constexpr uint32_t kLoopChunk = 1024;

struct SrvBfsLoopState {
    PersistState ps;               // barrier, rotating qlen / medges
    uint32_t touched_len[3];       // vertices listed in next[] this level
    uint32_t chunk_len[3];         // hub chunks this level
    unsigned long long alive[3];   // slots given next-frontier vertices
    uint32_t stop[3];              // block 0's decision to leave before the level
    // on exit
    uint32_t ticks, cur, nf, reason;
    unsigned long long alive_out, finished, medges_out;
};

struct SrvBfsLoopArgs {
    const uint32_t* off;
    const uint32_t* dst;
    unsigned long long* seen;
    unsigned long long* front[2];
    unsigned long long* next;
    uint32_t* q[2];
    uint32_t* touched;
    uint32_t* region;
    const uint32_t* start;
    uint2* chunk_q;
    uint32_t chunk_cap;
    uint32_t V, nz, cap;
    uint64_t E;
    uint32_t cur, tick0;
    unsigned long long active;
    uint32_t nf_exit, max_ticks;
    unsigned long long budget_ns;
    const uint32_t* mailbox;  // pinned host word: non-zero asks the loop to return
    SrvBfsLoopState* st;
};

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// One edge v -> u of a top-down level (warp-collective).
__device__ __forceinline__ void srv_td_edge(const SrvBfsLoopArgs& a, const unsigned long long* fcur, bool valid,
                                            uint32_t e, uint32_t v, uint32_t* tlen)
{
    bool first = false;
    uint32_t u = 0;
    if (valid) {
        u = a.dst[e];
        const unsigned long long add = fcur[v] & ~a.seen[u];
        if (add && (a.next[u] & add) != add) first = atomicOr(a.next + u, add) == 0ull;
    }
    append(first, u, a.touched, tlen, a.V, &a.st->ps);
}

__global__ void __launch_bounds__(kBlock) k_srv_bfs_loop(SrvBfsLoopArgs a)
{
    SrvBfsLoopState* st = a.st;
    PersistState* ps = &st->ps;
    const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x, gthreads = gridDim.x * blockDim.x;
    const uint32_t lane = lane_id(), gw = gtid / 32, nwarps = gthreads / 32;
    const unsigned long long t0 = global_ns();
    uint32_t cur = a.cur, it = 0;
    for (; it < a.max_ticks; it++) {
        const uint32_t s_cur = it % 3, s_next = (it + 1) % 3, s_zero = (it + 2) % 3;
        const uint32_t nf = *(volatile uint32_t*)&ps->qlen[s_cur];
        const unsigned long long mf = *(volatile unsigned long long*)&ps->medges[s_cur];
        if (*(volatile uint32_t*)&st->stop[s_cur] || nf == 0 || nf > a.nf_exit || (double)mf * 15.0 > (double)a.E)
            break;
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            ps->qlen[s_zero] = 0;
            ps->medges[s_zero] = 0;
            st->touched_len[s_zero] = 0;
            st->chunk_len[s_zero] = 0;
            st->alive[s_zero] = 0;
            st->stop[s_zero] = 0;
        }
        const uint32_t* qin = a.q[cur];
        uint32_t* qout = a.q[cur ^ 1];
        const unsigned long long* fcur = a.front[cur];
        unsigned long long* fnxt = a.front[cur ^ 1];
        uint32_t* tlen = &st->touched_len[s_cur];
        // expansion: short lists lane by lane, medium lists by one warp, hub lists as chunks
        for (uint32_t base = gw * 32; base < nf; base += nwarps * 32) {
            const uint32_t i = base + lane;
            uint32_t v = 0, s0 = 0, d = 0;
            if (i < nf) {
                v = qin[i];
                s0 = a.off[v];
                d = a.off[v + 1] - s0;
            }
            uint32_t hub = __ballot_sync(0xffffffffu, d >= kLoopHub);
            while (hub) {
                const uint32_t l = __ffs(hub) - 1;
                hub &= hub - 1;
                const uint32_t hv = __shfl_sync(0xffffffffu, v, l), hd = __shfl_sync(0xffffffffu, d, l);
                const uint32_t nch = (hd + kLoopChunk - 1) / kLoopChunk;
                uint32_t slot = 0;
                if (lane == 0) slot = atomicAdd(&st->chunk_len[s_cur], nch);
                slot = __shfl_sync(0xffffffffu, slot, 0);
                for (uint32_t c = lane; c < nch; c += 32) {
                    if (slot + c < a.chunk_cap) a.chunk_q[slot + c] = make_uint2(hv, c);
                    else atomicOr(&ps->status, 2u);
                }
                if (lane == l) d = 0;
            }
            uint32_t wm;
            while ((wm = __ballot_sync(0xffffffffu, d >= 32)) != 0) {
                const uint32_t l = __ffs(wm) - 1;
                const uint32_t wv = __shfl_sync(0xffffffffu, v, l), ws = __shfl_sync(0xffffffffu, s0, l);
                const uint32_t wd = __shfl_sync(0xffffffffu, d, l);
                if (lane == l) d = 0;
                for (uint32_t k = 0; k < wd; k += 32) srv_td_edge(a, fcur, k + lane < wd, ws + k + lane, wv, tlen);
            }
            for (uint32_t j = 0; __any_sync(0xffffffffu, j < d); j++) srv_td_edge(a, fcur, j < d, s0 + j, v, tlen);
        }
        if (!grid_barrier(ps)) break;
        const uint32_t nch = min(*(volatile uint32_t*)&st->chunk_len[s_cur], a.chunk_cap);
        for (uint32_t c = gw; c < nch; c += nwarps) {
            const uint2 dsc = a.chunk_q[c];
            const uint32_t s0 = a.off[dsc.x], e1 = a.off[dsc.x + 1];
            const uint32_t cs = s0 + dsc.y * kLoopChunk, ce = min(e1, cs + kLoopChunk);
            for (uint32_t k = cs; k < ce; k += 32) srv_td_edge(a, fcur, k + lane < ce, k + lane, dsc.x, tlen);
        }
        if (!grid_barrier(ps)) break;
        // the listed vertices keep their new roots and form the next frontier
        const uint32_t nt = *(volatile uint32_t*)tlen;
        const uint32_t lvl = a.tick0 + it + 1;
        unsigned long long live = 0, medges = 0;
        for (uint32_t b = gw * 32; b < nt; b += nwarps * 32) {
            const uint32_t i = b + lane;
            bool act = false;
            uint32_t u = 0;
            if (i < nt) {
                u = a.touched[i];
                const unsigned long long x = a.next[u] & ~a.seen[u];
                a.next[u] = 0;
                if (x) {
                    a.seen[u] |= x;
                    for (unsigned long long m = x; m; m &= m - 1) {
                        const uint32_t k = __ffsll(m) - 1;
                        a.region[(size_t)k * a.V + u] = lvl - a.start[k];
                    }
                    act = u < a.nz;
                    if (act) {
                        fnxt[u] = x;
                        live |= x;
                        medges += a.off[u + 1] - a.off[u];
                    }
                }
            }
            append(act, u, qout, &ps->qlen[s_next], a.cap, ps);
        }
        for (uint32_t i = gtid; i < nf; i += gthreads) a.front[cur][qin[i]] = 0;
        live = warp_or(live);
        medges = warp_sum(medges);
        if (lane == 0) {
            if (live) atomicOr(&st->alive[s_next], live);
            if (medges) atomicAdd(&ps->medges[s_next], medges);
        }
        if (!grid_barrier(ps)) break;
        // block 0 decides whether the next level runs here
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            const unsigned long long alive = *(volatile unsigned long long*)&st->alive[s_next];
            const bool fin = (a.active & ~alive) != 0ull;
            const bool mail = *(volatile const uint32_t*)a.mailbox != 0u;
            const bool late = global_ns() - t0 > a.budget_ns;
            st->stop[s_next] = (fin || mail || late) ? 1u : 0u;
            st->reason = fin ? 1u : mail ? 2u : late ? 3u : 0u;
        }
        if (!grid_barrier(ps)) break;
        cur ^= 1;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->ticks = it;
        st->cur = cur;
        st->nf = ps->qlen[it % 3];
        st->medges_out = ps->medges[it % 3];
        const unsigned long long alive = it > 0 ? st->alive[it % 3] : a.active;
        st->alive_out = alive;
        st->finished = it > 0 ? (a.active & ~alive) : 0ull;
    }
}

// ----------------------------------------------- device-resident SSSP rounds
//
// The SSSP group's rounds on the device, many per launch: one cooperative
// kernel runs the tick of the host loop (sp_issue) as grid phases separated
// by the bounded grid barrier -- plan (per-slot bucket advances, by the
// slots' near / far liveness of the previous round), split of the far list
// for the advancing slots, descriptors, expansion -- using the bodies of the
// multi-root kernels of mssp.cu, until a slot's query ended, the host
// raised the pinned mailbox (a query waits for a free slot), or the time
// budget ran out.  Per-slot thresholds, smallest far distances and
// liveness live in the loop state between launches; the host loads them
// before a launch and reads them back after it.

struct SrvSpLoopState {
    PersistState ps;                   // barrier and status
    unsigned long long thr[kSrvSlots]; // per-slot threshold
    uint32_t thr32[kSrvSlots];         // the same, clamped (expansion)
    uint32_t lo[kSrvSlots], hi[kSrvSlots];  // bucket being split in (split)
    uint32_t min_far[kSrvSlots];       // smallest far distance the slot's last split kept
    uint32_t min_far_new[kSrvSlots];   // ... reported by this round's split
    uint32_t last_empty[kSrvSlots];    // the slot's last split found no near pair
    unsigned long long near_alive, far_alive, adv, active;
    unsigned long long alive_round[2]; // this round: [0] near work, [1] far work
    uint32_t cur, fcur, stop, reason;
    uint32_t ticks;
    unsigned long long finished;
};

struct SrvSpLoopArgs {
    const uint32_t* off;
    const uint32_t* dst;
    const uint32_t* w;
    uint32_t* dist;
    unsigned long long* pend;
    unsigned long long* farm;
    unsigned long long* maskq;
    uint32_t* far_list[2];
    uint4* desc;
    uint64_t desc_cap;
    MsspCounters* c;
    uint32_t* q[2];
    uint32_t V, ms_edges, delta, max_ticks;
    unsigned long long budget_ns;
    const uint32_t* mailbox;
    SrvSpLoopState* st;
};

template <bool kHasW>
__global__ void __launch_bounds__(kBlock) k_srv_sssp_loop(SrvSpLoopArgs a)
{
    SrvSpLoopState* st = a.st;
    PersistState* ps = &st->ps;
    MsspCounters* c = a.c;
    const unsigned long long t0 = global_ns();
    uint32_t it = 0;
    for (; it < a.max_ticks; it++) {
        // plan (block 0): slots whose near work ran out but which keep far pairs advance a bucket
        if (blockIdx.x == 0 && threadIdx.x < kSrvSlots) {
            const uint32_t k = threadIdx.x;
            const unsigned long long adv = st->active & ~st->near_alive & st->far_alive;
            if ((adv >> k) & 1ull) {
                const uint64_t t = st->thr[k];
                uint64_t hi = t + a.delta;
                if (st->last_empty[k] && st->min_far[k] != kValueMax)
                    hi = std::max<uint64_t>(hi, ((uint64_t)st->min_far[k] / a.delta + 1) * (uint64_t)a.delta);
                st->lo[k] = t < 0xFFFFFFFFull ? (uint32_t)t : 0xFFFFFFFFu;
                st->hi[k] = hi < 0xFFFFFFFFull ? (uint32_t)hi : 0xFFFFFFFFu;
                st->thr[k] = hi;
                st->min_far_new[k] = kValueMax;
            }
            st->thr32[k] = st->thr[k] < 0xFFFFFFFFull ? (uint32_t)st->thr[k] : 0xFFFFFFFFu;
            if (k == 0) {
                st->adv = adv;
                c->nfar_next = 0;
                c->nq_out = 0;
                c->ndesc = 0;
                st->alive_round[0] = 0;
                if (adv) st->alive_round[1] = 0;  // recomputed by the split
            }
        }
        if (!grid_barrier(ps)) break;
        const unsigned long long adv = *(volatile unsigned long long*)&st->adv;
        const uint32_t cur = *(volatile uint32_t*)&st->cur;
        uint32_t fcur = *(volatile uint32_t*)&st->fcur;
        if (adv) {
            mssp_split_body(a.far_list[fcur], &c->nfar_live, a.dist, a.pend, a.farm, a.q[cur], &c->nq_in,
                            a.far_list[fcur ^ 1], &c->nfar_next, a.V, 0, 0, st->lo, st->hi, adv, st->min_far_new,
                            &st->alive_round[1], c);
            if (!grid_barrier(ps)) break;
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                c->nfar_live = c->nfar_next;
                st->fcur = fcur ^ 1;
            }
            fcur ^= 1;
        }
        mssp_desc_body(a.q[cur], &c->nq_in, a.off, a.pend, a.maskq, a.desc, a.desc_cap, c, a.ms_edges);
        if (!grid_barrier(ps)) break;
        mssp_expand_body<kHasW>(a.desc, c, a.maskq, a.dst, a.w, a.dist, a.pend, a.farm, a.q[cur ^ 1], &c->nq_out,
                                a.far_list[fcur], &c->nfar_live, a.V, 0, st->thr32, st->alive_round, c);
        if (!grid_barrier(ps)) break;
        // round's end (block 0): liveness, the split slots' far minima, the decision to go on
        if (blockIdx.x == 0 && threadIdx.x < kSrvSlots) {
            const uint32_t k = threadIdx.x;
            const unsigned long long near = st->alive_round[0], far = st->alive_round[1];
            if ((st->adv >> k) & 1ull) {
                st->min_far[k] = st->min_far_new[k];
                st->last_empty[k] = ((near >> k) & 1ull) ? 0u : 1u;
            }
            __syncwarp(0xffffffffu);
            if (k == 0) {
                c->nq_in = c->nq_out;
                st->cur = cur ^ 1;
                st->near_alive = near;
                st->far_alive = far;
                const unsigned long long fin = st->active & ~(near | far);
                const bool mail = *(volatile const uint32_t*)a.mailbox != 0u;
                const bool late = global_ns() - t0 > a.budget_ns;
                st->finished = fin;
                st->stop = (fin || mail || late || c->overflow) ? 1u : 0u;
                st->reason = fin ? 1u : mail ? 2u : late ? 3u : 0u;
            }
        }
        if (!grid_barrier(ps)) break;
        if (*(volatile uint32_t*)&st->stop) {
            it++;
            break;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) st->ticks = it;
}

// ------------------------------------------------------------------ state

using Clock = std::chrono::steady_clock;

struct SrvReq {
    cgb_request_info info{};
    uint32_t* out = nullptr;
};

enum class SlotState { kFree, kActive };

// Per-slot statistics block (device) and its pinned mirror.
struct SlotStats {
    unsigned long long edges[kSrvSlots];
    uint32_t reached[kSrvSlots];
    uint32_t depth[kSrvSlots];
    unsigned long long alive[2];  // BFS: [0] next-frontier slots; SSSP: [0] near work, [1] far work
    uint32_t min_far[kSrvSlots];
};

// Host-visible upload block for a tick's admissions and per-slot thresholds.
struct SlotUpload {
    uint32_t slots[kSrvSlots];
    uint32_t roots[kSrvSlots];
    uint32_t qidx[kSrvSlots];
    uint32_t start[kSrvSlots];  // BFS: tick of admission
    uint32_t thr[kSrvSlots];    // SSSP: near threshold per slot
    uint32_t lo[kSrvSlots];     // SSSP: bucket being split in
    uint32_t hi[kSrvSlots];
    uint32_t min_far[kSrvSlots];
};

struct Group {
    int alg = CGB_BFS;
    uint32_t nslots = 0;
    SlotState state[kSrvSlots];
    int64_t req[kSrvSlots];
    bool used[kSrvSlots] = {};
    uint32_t* region = nullptr;  // nslots * V results
    SlotStats* d_stats = nullptr;
    SlotStats* h_stats = nullptr;
    SlotUpload* d_up = nullptr;
    SlotUpload* h_up = nullptr;
    cudaStream_t stream = nullptr;
    unsigned long long active = 0;
    unsigned long long live = 0;  // BFS: slots with vertices in the current frontier
    uint32_t root[kSrvSlots];
    uint32_t* out[kSrvSlots];  // where the slot's result goes (host / device / NULL)
    std::vector<uint32_t> admit;  // slots admitted this tick (root / out filled under the server lock)
    // BFS
    SrvBfsLoopState* loop = nullptr;    // device-resident levels (null: host ticks only)
    SrvBfsLoopState* h_loop = nullptr;  // pinned mirror
    uint32_t* mailbox = nullptr;        // pinned word the loop polls: non-zero = return to the host
    cudaEvent_t ev_loop = nullptr;
    uint64_t loop_levels = 0, loop_launches = 0;
    MsBuffers* mb = nullptr;
    uint32_t* q[2] = {nullptr, nullptr};
    uint32_t* touched = nullptr;
    uint32_t nact = 0, cur = 0, tick = 0;
    unsigned long long medges = 0;
    // SSSP
    SrvSpLoopState* sp_loop = nullptr;    // device-resident rounds (null: host ticks only)
    SrvSpLoopState* h_sp_loop = nullptr;  // pinned mirror
    MsspBuffers* sp = nullptr;
    uint32_t delta = 1, fcur = 0;
    unsigned long long near_alive = 0, far_alive = 0, split_mask = 0;
    uint64_t thr[kSrvSlots] = {};
    uint32_t min_far[kSrvSlots];
    bool last_empty[kSrvSlots] = {};
};

}  // namespace cgb

using namespace cgb;

struct cgb_server {
    cgb_graph* g = nullptr;
    // a second single-root engine context over g's CSR for the SSSP group's
    // single-root runs, so that they do not hold g, which BFS ticks and BFS
    // single-root runs need
    cgb_graph* shadow = nullptr;
    uint32_t flags = 0;  // cgb_server_config.flags
    // The groups' device-resident loops are cooperative launches whose CTAs wait
    // for each other at grid barriers; two of them resident at once could each
    // hold SMs the other waits for, so one runs at a time.
    std::mutex coop_mu;
    std::atomic<int> coop_waiters{0};  // threads waiting for coop_mu: a running loop returns for them
    Group grp[2];  // [0] BFS, [1] SSSP
    std::vector<SrvReq> reqs;
    std::deque<int64_t> waiting[2];    // submitted, not admitted (arrival order of submission)
    std::vector<cgb_request_info> done;
    std::mutex mu;
    std::condition_variable cv;
    std::thread th[2];
    std::atomic<bool> stop{false};
    bool started = false;
    Clock::time_point t0;
    uint64_t ticks[2] = {0, 0}, completed = 0;
    double busy_ms[2] = {0, 0};
    double lone_est_us[2] = {0, 0};   // running mean of single-root run times
    // running mean of batched queries' admission-to-result times; until a batched
    // query has finished, unknown (infinite): due queries go the single-root way
    // (at most kLoneMaxDue at a time), since a zero start let the first two queries
    // due together start a batch that later arrivals joined
    double batch_est_us[2] = {1e300, 1e300};
    uint64_t lone_runs[2] = {0, 0}, batch_runs[2] = {0, 0};
    cgb_status error = CGB_OK;
    std::string error_msg;
};

namespace cgb {

static double us_since(const cgb_server* s, Clock::time_point t)
{
    return std::chrono::duration<double, std::micro>(t - s->t0).count();
}

static void group_alloc(cgb_server* s, Group& G, int alg, uint32_t nslots)
{
    cgb_graph* g = s->g;
    const uint32_t V = g->V;
    G.alg = alg;
    G.nslots = nslots;
    for (uint32_t k = 0; k < kSrvSlots; k++) {
        G.state[k] = SlotState::kFree;
        G.req[k] = -1;
        G.min_far[k] = kValueMax;
    }
    if (nslots == 0) return;
    CGB_CUDA_TRY(cudaMalloc((void**)&G.region, (size_t)nslots * V * 4));
    CGB_CUDA_TRY(cudaMalloc((void**)&G.d_stats, sizeof(SlotStats)));
    CGB_CUDA_TRY(cudaMallocHost((void**)&G.h_stats, sizeof(SlotStats)));
    CGB_CUDA_TRY(cudaMalloc((void**)&G.d_up, sizeof(SlotUpload)));
    CGB_CUDA_TRY(cudaMallocHost((void**)&G.h_up, sizeof(SlotUpload)));
    CGB_CUDA_TRY(cudaMemset(G.d_stats, 0, sizeof(SlotStats)));
    CGB_CUDA_TRY(cudaMemset(G.d_up, 0, sizeof(SlotUpload)));
    memset(G.h_stats, 0, sizeof(SlotStats));
    memset(G.h_up, 0, sizeof(SlotUpload));
    if (alg == CGB_BFS) {
        G.stream = g->stream;  // the binned push expansion runs on the graph's stream
        G.mb = ms_buffers_alloc(V, g->E);
        if (!(s->flags & CGB_SERVER_HOST_TICKS)) {
            CGB_CUDA_TRY(cudaMalloc((void**)&G.loop, sizeof(SrvBfsLoopState)));
            CGB_CUDA_TRY(cudaMallocHost((void**)&G.h_loop, sizeof(SrvBfsLoopState)));
            CGB_CUDA_TRY(cudaMallocHost((void**)&G.mailbox, sizeof(uint32_t)));
            *G.mailbox = 0;
            CGB_CUDA_TRY(cudaEventCreateWithFlags(&G.ev_loop, cudaEventDisableTiming));
        }
        CGB_CUDA_TRY(cudaMemset(G.mb->seen, 0, (size_t)V * 8));
        CGB_CUDA_TRY(cudaMemset(G.mb->front[0], 0, (size_t)V * 8));
        CGB_CUDA_TRY(cudaMemset(G.mb->front[1], 0, (size_t)V * 8));
        CGB_CUDA_TRY(cudaMemset(G.mb->next, 0, (size_t)V * 8));
        CGB_CUDA_TRY(cudaMalloc((void**)&G.q[0], (size_t)V * 4));
        CGB_CUDA_TRY(cudaMalloc((void**)&G.q[1], (size_t)V * 4));
        CGB_CUDA_TRY(cudaMalloc((void**)&G.touched, (size_t)V * 4));
    } else {
        CGB_CUDA_TRY(cudaStreamCreateWithFlags(&G.stream, cudaStreamNonBlocking));
        G.sp = mssp_buffers_alloc(V, g->E);
        if (!(s->flags & CGB_SERVER_HOST_TICKS)) {
            CGB_CUDA_TRY(cudaMalloc((void**)&G.sp_loop, sizeof(SrvSpLoopState)));
            CGB_CUDA_TRY(cudaMallocHost((void**)&G.h_sp_loop, sizeof(SrvSpLoopState)));
            CGB_CUDA_TRY(cudaMallocHost((void**)&G.mailbox, sizeof(uint32_t)));
            *G.mailbox = 0;
            CGB_CUDA_TRY(cudaEventCreateWithFlags(&G.ev_loop, cudaEventDisableTiming));
        }
        CGB_CUDA_TRY(cudaMalloc((void**)&G.q[0], (size_t)V * 4));
        CGB_CUDA_TRY(cudaMalloc((void**)&G.q[1], (size_t)V * 4));
        CGB_CUDA_TRY(cudaMemset(G.sp->c, 0, sizeof(MsspCounters)));
        CGB_CUDA_TRY(cudaMemset(G.sp->pend, 0, (size_t)V * 8));
        CGB_CUDA_TRY(cudaMemset(G.sp->farm, 0, (size_t)V * 8));
        k_ms_fill<<<num_sms() * 8, kBlock>>>((uint64_t)V * kMsRoots, G.sp->dist, kValueMax);  // reused slots reset on admission
        CGB_CUDA_TRY(cudaGetLastError());
    }
}

static void group_free(cgb_server* s, Group& G)
{
    cudaFree(G.region);
    cudaFree(G.d_stats);
    if (G.h_stats) cudaFreeHost(G.h_stats);
    cudaFree(G.d_up);
    if (G.h_up) cudaFreeHost(G.h_up);
    ms_buffers_free(G.mb);
    cudaFree(G.loop);
    if (G.h_loop) cudaFreeHost(G.h_loop);
    cudaFree(G.sp_loop);
    if (G.h_sp_loop) cudaFreeHost(G.h_sp_loop);
    if (G.mailbox) cudaFreeHost(G.mailbox);
    if (G.ev_loop) cudaEventDestroy(G.ev_loop);
    cudaFree(G.q[0]);
    cudaFree(G.q[1]);
    cudaFree(G.touched);
    if (G.sp) mssp_buffers_free(G.sp);
    if (G.stream && G.stream != s->g->stream) cudaStreamDestroy(G.stream);
    G = Group();
}

// ---- BFS group: this tick's admissions (no host sync)
static void bfs_admit(cgb_server* s, Group& G)
{
    cgb_graph* g = s->g;
    const uint32_t V = g->V;
    cudaStream_t st = G.stream;
    const uint32_t cur = G.cur;
    if (!G.admit.empty()) {
        unsigned long long reuse = 0;
        uint32_t n = 0, qpos = G.nact;
        for (const uint32_t k : G.admit) {
            const uint32_t root = G.root[k];
            if (G.used[k]) reuse |= 1ull << k;
            G.used[k] = true;
            G.h_up->slots[n] = k;
            G.h_up->roots[n] = root;
            G.h_up->qidx[n] = root < g->nz ? qpos++ : 0xFFFFFFFFu;
            if (root < g->nz) G.live |= 1ull << k;
            G.h_up->start[k] = G.tick;
            n++;
        }
        G.nact = qpos;
        if (reuse)
            k_srv_clear_bits<<<num_sms() * 8, kBlock, 0, st>>>(V, G.mb->seen, reuse);
        for (const uint32_t k : G.admit)
            k_ms_fill<<<num_sms() * 4, kBlock, 0, st>>>((uint64_t)V, G.region + (size_t)k * V, kValueMax);
        CGB_CUDA_TRY(cudaMemcpyAsync(G.d_up, G.h_up, sizeof(SlotUpload), cudaMemcpyHostToDevice, st));
        k_srv_bfs_admit<<<1, kSrvSlots, 0, st>>>(n, G.d_up->slots, G.d_up->roots, G.d_up->qidx, V, G.region,
                                                 G.mb->seen, G.mb->front[cur], G.q[cur]);
        G.admit.clear();
    }
}

// ---- BFS group: issue one level for every active slot (no host sync)
static void bfs_issue(cgb_server* s, Group& G)
{
    cgb_graph* g = s->g;
    const uint32_t V = g->V;
    cudaStream_t st = G.stream;
    const uint32_t cur = G.cur, nxt = cur ^ 1;
    bfs_admit(s, G);
    CGB_CUDA_TRY(cudaMemsetAsync(&G.d_stats->alive[0], 0, 8, st));
    CGB_CUDA_TRY(cudaMemsetAsync(&g->ctr->qlen[nxt], 0, 4, st));
    CGB_CUDA_TRY(cudaMemsetAsync(&g->ctr->medges, 0, 8, st));
    CGB_CUDA_TRY(cudaMemsetAsync(&g->ctr->overflow, 0, 4, st));
    if (G.nact == 0) return;
    const uint32_t lvl = G.tick + 1;
    const bool pull = (double)G.medges * 15.0 > (double)g->E;
    if (pull) {
        MsBuArgs ba{V, g->in_off, g->in_src, G.mb->front[cur], G.mb->seen, G.mb->front[nxt], G.mb->next, G.live,
                    G.region, lvl, g->nz, G.q[nxt], &g->ctr->qlen[nxt], V, g->ctr, G.d_up->start,
                    &G.d_stats->alive[0], G.mb->heavy_w, G.mb->heavy_b, G.mb->heavy_len, G.mb->cap_b};
        ms_bottom_up(ba, st, nullptr);
    } else {
        CGB_CUDA_TRY(cudaMemsetAsync(&g->ctr->found, 0, 4, st));
        CGB_CUDA_TRY(cudaMemsetAsync(&g->ctr->chunk_len, 0, 4, st));
        MsTdOp op{g->off, g->dst, G.mb->front[cur], G.mb->seen, G.mb->next, G.touched, &g->ctr->found, V, g->ctr};
        launch_push(g, G.q[cur], G.nact, op, false);
        k_ms_finalize<<<num_sms() * 8, kBlock, 0, st>>>(G.touched, 0, &g->ctr->found, G.mb->seen, G.mb->next,
                                                     G.mb->front[nxt], G.region, V, lvl, g->nz, G.q[nxt],
                                                     &g->ctr->qlen[nxt], V, g->ctr, G.d_up->start,
                                                     &G.d_stats->alive[0]);
    }
    k_ms_clear<<<grid_for(G.nact, kBlock, num_sms() * 8), kBlock, 0, st>>>(G.q[cur], G.nact, G.mb->front[cur]);
    k_ms_degree_sum<<<num_sms() * 4, kBlock, 0, st>>>(G.q[nxt], 0, &g->ctr->qlen[nxt], g->off, g->ctr);
}

// ---- SSSP group: admissions, per-slot bucket splits, one near round
// ---- SSSP group: this tick's admissions (no host sync)
static void sp_admit(cgb_server* s, Group& G)
{
    cgb_graph* g = s->g;
    const uint32_t V = g->V;
    cudaStream_t st = G.stream;
    MsspBuffers& b = *G.sp;
    const uint32_t cur = G.cur;
    if (!G.admit.empty()) {
        unsigned long long reuse = 0;
        uint32_t n = 0;
        for (const uint32_t k : G.admit) {
            if (G.used[k]) reuse |= 1ull << k;
            G.used[k] = true;
            G.h_up->slots[n] = k;
            G.h_up->roots[n] = G.root[k];
            G.thr[k] = G.delta;
            G.last_empty[k] = false;
            G.min_far[k] = kValueMax;
            n++;
        }
        if (reuse) k_srv_sp_reset<<<num_sms() * 8, kBlock, 0, st>>>(V, b.dist, reuse);
        for (uint32_t k = 0; k < kSrvSlots; k++) G.h_up->thr[k] = (uint32_t)std::min<uint64_t>(G.thr[k], 0xFFFFFFFFu);
        CGB_CUDA_TRY(cudaMemcpyAsync(G.d_up, G.h_up, sizeof(SlotUpload), cudaMemcpyHostToDevice, st));
        k_srv_sp_admit<<<1, kSrvSlots, 0, st>>>(n, G.d_up->slots, G.d_up->roots, b.dist, b.pend, G.q[cur],
                                                &b.c->nq_in, V, b.c);
        G.admit.clear();
    }
}

// ---- SSSP group: per-slot bucket splits and one near round (no host sync)
static void sp_issue(cgb_server* s, Group& G)
{
    cgb_graph* g = s->g;
    const uint32_t V = g->V;
    cudaStream_t st = G.stream;
    MsspBuffers& b = *G.sp;
    const uint32_t cur = G.cur, nxt = cur ^ 1;
    sp_admit(s, G);
    // slots whose near work ran out but which still have far pairs move to their
    // next bucket (a slot admitted this tick, or free, has neither bit)
    const unsigned long long adv = G.active & ~G.near_alive & G.far_alive;
    G.split_mask = adv;
    if (adv) {
        for (uint32_t k = 0; k < kSrvSlots; k++) {
            if (!((adv >> k) & 1ull)) continue;
            uint64_t hi = G.thr[k] + G.delta;
            if (G.last_empty[k] && G.min_far[k] != kValueMax)
                hi = std::max<uint64_t>(hi, ((uint64_t)G.min_far[k] / G.delta + 1) * G.delta);
            G.h_up->lo[k] = (uint32_t)std::min<uint64_t>(G.thr[k], 0xFFFFFFFFu);
            G.h_up->hi[k] = (uint32_t)std::min<uint64_t>(hi, 0xFFFFFFFFu);
            G.thr[k] = hi;
            G.h_up->min_far[k] = kValueMax;
        }
        for (uint32_t k = 0; k < kSrvSlots; k++) G.h_up->thr[k] = (uint32_t)std::min<uint64_t>(G.thr[k], 0xFFFFFFFFu);
        CGB_CUDA_TRY(cudaMemcpyAsync(G.d_up, G.h_up, sizeof(SlotUpload), cudaMemcpyHostToDevice, st));
        CGB_CUDA_TRY(cudaMemcpyAsync(G.d_stats->min_far, G.h_up->min_far, sizeof(G.h_up->min_far),
                                     cudaMemcpyHostToDevice, st));
        CGB_CUDA_TRY(cudaMemsetAsync(&b.c->nfar_next, 0, 4, st));
        CGB_CUDA_TRY(cudaMemsetAsync(&G.d_stats->alive[1], 0, 8, st));
        k_mssp_split<<<num_sms() * 8, kBlock, 0, st>>>(b.far_list[G.fcur], &b.c->nfar_live, b.dist, b.pend, b.farm,
                                                     G.q[cur], &b.c->nq_in, b.far_list[G.fcur ^ 1], &b.c->nfar_next,
                                                     V, 0, 0, G.d_up->lo, G.d_up->hi, adv, G.d_stats->min_far,
                                                     &G.d_stats->alive[1], b.c);
        k_srv_copy_u32<<<1, 1, 0, st>>>(&b.c->nfar_next, &b.c->nfar_live);
        G.fcur ^= 1;
    }
    CGB_CUDA_TRY(cudaMemsetAsync(&G.d_stats->alive[0], 0, 8, st));
    CGB_CUDA_TRY(cudaMemsetAsync(&b.c->nq_out, 0, 4, st));
    CGB_CUDA_TRY(cudaMemsetAsync(&b.c->ndesc, 0, 4, st));
    k_mssp_desc<<<num_sms() * 8, kBlock, 0, st>>>(G.q[cur], &b.c->nq_in, g->off, b.pend, b.maskq, b.desc, b.desc_cap,
                                                b.c, g->tune_alg[CGB_SSSP].ms_edges);
    mssp_expand(g->w != nullptr, num_sms() * 8, st, b.desc, b.c, b.maskq, g->dst, g->w, b.dist, b.pend, b.farm,
                G.q[nxt], &b.c->nq_out, b.far_list[G.fcur], &b.c->nfar_live, V, 0, G.d_up->thr, G.d_stats->alive);
    k_srv_copy_u32<<<1, 1, 0, st>>>(&b.c->nq_out, &b.c->nq_in);
    CGB_CUDA_TRY(cudaMemcpyAsync(&G.h_stats->alive, &G.d_stats->alive, sizeof(G.h_stats->alive),
                                 cudaMemcpyDeviceToHost, st));
    CGB_CUDA_TRY(cudaMemcpyAsync(G.h_stats->min_far, G.d_stats->min_far, sizeof(G.h_stats->min_far),
                                 cudaMemcpyDeviceToHost, st));
    CGB_CUDA_TRY(cudaMemcpyAsync(b.h, b.c, sizeof(MsspCounters), cudaMemcpyDeviceToHost, st));
}

// A query waits whose arrival time has passed, and a slot is free for it.
static bool admission_due(cgb_server* s, const Group& G, int a)
{
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->waiting[a].empty()) return false;
    if (s->reqs[s->waiting[a].front()].info.arrival_us > us_since(s, Clock::now())) return false;
    if (!(s->flags & CGB_SERVER_ADMIT_ANY_SLOT) && G.active != 0 &&
        2u * (uint32_t)__builtin_popcountll(G.active) > G.nslots)
        return false;
    for (uint32_t k = 0; k < G.nslots; k++)
        if (G.state[k] == SlotState::kFree) return true;
    return false;
}

// Levels of the BFS group on the device (k_srv_bfs_loop) from its current
// frontier; returns the slots whose traversal ended.  While the loop runs,
// this thread raises the pinned mailbox as soon as a waiting query could be
// admitted, and the loop returns after the level in progress.
constexpr unsigned long long kLoopBudgetNs = 4000000;  // a launch returns after 4 ms at most
static unsigned long long bfs_device_levels(cgb_server* s, Group& G, uint32_t nf_exit)
{
    cgb_graph* g = s->g;
    SrvBfsLoopState& h = *G.h_loop;
    h = SrvBfsLoopState{};
    h.ps.qlen[0] = G.nact;
    h.ps.medges[0] = G.medges;
    static_assert(sizeof(SrvBfsLoopState) % 4 == 0, "copied as words");
    h2d_small(G.loop, &h, sizeof(SrvBfsLoopState), G.stream);
    *reinterpret_cast<volatile uint32_t*>(G.mailbox) = 0;
    SrvBfsLoopArgs args{};
    args.off = g->off;
    args.dst = g->dst;
    args.seen = G.mb->seen;
    args.front[0] = G.mb->front[0];
    args.front[1] = G.mb->front[1];
    args.next = G.mb->next;
    args.q[0] = G.q[0];
    args.q[1] = G.q[1];
    args.touched = G.touched;
    args.region = G.region;
    args.start = G.d_up->start;
    args.chunk_q = g->chunk_q;
    args.chunk_cap = g->chunk_cap;
    args.V = g->V;
    args.nz = g->nz;
    args.cap = g->V;
    args.E = g->E;
    args.cur = G.cur;
    args.tick0 = G.tick;
    args.active = G.active;
    args.nf_exit = nf_exit;
    args.max_ticks = g->V + 2;
    args.budget_ns = kLoopBudgetNs;
    args.mailbox = G.mailbox;
    args.st = G.loop;
    static uint32_t grid = 0;
    if (!grid) grid = cooperative_grid(k_srv_bfs_loop);
    void* kargs[] = {&args};
    s->coop_waiters++;
    std::lock_guard<std::mutex> coop(s->coop_mu);
    s->coop_waiters--;
    CGB_CUDA_TRY(cudaLaunchCooperativeKernel((void*)k_srv_bfs_loop, grid, kBlock, kargs, 0, G.stream));
    CGB_CUDA_TRY(cudaMemcpyAsync(&h, G.loop, sizeof(SrvBfsLoopState), cudaMemcpyDeviceToHost, G.stream));
    CGB_CUDA_TRY(cudaEventRecord(G.ev_loop, G.stream));
    for (;;) {
        const cudaError_t e = cudaEventQuery(G.ev_loop);
        if (e == cudaSuccess) break;
        if (e != cudaErrorNotReady) CGB_CUDA_TRY(e);
        if (admission_due(s, G, 0) || s->coop_waiters.load() > 0)
            *reinterpret_cast<volatile uint32_t*>(G.mailbox) = 1;
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
    CGB_REQUIRE(!(h.ps.status & 2u), CGB_EOVERFLOW, "server BFS loop: queue overflow");
    CGB_REQUIRE(!(h.ps.status & 1u), CGB_ETIMEOUT, "server BFS loop: grid barrier gave up");
    G.cur = h.cur;
    G.nact = h.nf;
    G.tick += h.ticks;
    G.live = h.alive_out;
    G.medges = h.medges_out;
    G.loop_levels += h.ticks;
    G.loop_launches++;
    return h.finished;
}

// Cooperative grid of `kernel` with up to `per_sm` kBlock-thread CTAs per SM
// (as many as are resident at once).
template <typename K>
static uint32_t cooperative_grid_n(K kernel, int per_sm)
{
    int dev = 0, occ = 0;
    CGB_CUDA_TRY(cudaGetDevice(&dev));
    CGB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, kBlock, 0));
    CGB_REQUIRE(occ >= 1, CGB_EUNSUPPORTED, "device-resident loop does not fit on an SM");
    return (uint32_t)num_sms() * (uint32_t)std::min(occ, per_sm);
}

// Rounds of the SSSP group on the device (k_srv_sssp_loop) from its current
// state; returns the slots whose query ended.  The host raises the pinned
// mailbox as for the BFS loop.
static unsigned long long sp_device_ticks(cgb_server* s, Group& G)
{
    cgb_graph* g = s->g;
    MsspBuffers& b = *G.sp;
    SrvSpLoopState& h = *G.h_sp_loop;
    h = SrvSpLoopState{};
    for (uint32_t k = 0; k < kSrvSlots; k++) {
        h.thr[k] = G.thr[k];
        h.min_far[k] = G.min_far[k];
        h.last_empty[k] = G.last_empty[k] ? 1u : 0u;
    }
    h.near_alive = G.near_alive;
    h.far_alive = G.far_alive;
    h.alive_round[1] = G.far_alive;
    h.active = G.active;
    h.cur = G.cur;
    h.fcur = G.fcur;
    static_assert(sizeof(SrvSpLoopState) % 4 == 0, "copied as words");
    h2d_small(G.sp_loop, &h, sizeof(SrvSpLoopState), G.stream);
    *reinterpret_cast<volatile uint32_t*>(G.mailbox) = 0;
    SrvSpLoopArgs args{};
    args.off = g->off;
    args.dst = g->dst;
    args.w = g->w;
    args.dist = b.dist;
    args.pend = b.pend;
    args.farm = b.farm;
    args.maskq = b.maskq;
    args.far_list[0] = b.far_list[0];
    args.far_list[1] = b.far_list[1];
    args.desc = b.desc;
    args.desc_cap = b.desc_cap;
    args.c = b.c;
    args.q[0] = G.q[0];
    args.q[1] = G.q[1];
    args.V = g->V;
    args.ms_edges = g->tune_alg[CGB_SSSP].ms_edges;
    args.delta = G.delta;
    args.max_ticks = 4u * g->V + 64u;
    args.budget_ns = kLoopBudgetNs;
    args.mailbox = G.mailbox;
    args.st = G.sp_loop;
    void* kargs[] = {&args};
    s->coop_waiters++;
    std::lock_guard<std::mutex> coop(s->coop_mu);
    s->coop_waiters--;
    if (g->w) {
        static uint32_t grid = 0;
        if (!grid) grid = cooperative_grid_n(k_srv_sssp_loop<true>, 4);
        CGB_CUDA_TRY(cudaLaunchCooperativeKernel((void*)k_srv_sssp_loop<true>, grid, kBlock, kargs, 0, G.stream));
    } else {
        static uint32_t grid = 0;
        if (!grid) grid = cooperative_grid_n(k_srv_sssp_loop<false>, 4);
        CGB_CUDA_TRY(cudaLaunchCooperativeKernel((void*)k_srv_sssp_loop<false>, grid, kBlock, kargs, 0, G.stream));
    }
    CGB_CUDA_TRY(cudaMemcpyAsync(&h, G.sp_loop, sizeof(SrvSpLoopState), cudaMemcpyDeviceToHost, G.stream));
    CGB_CUDA_TRY(cudaMemcpyAsync(b.h, b.c, sizeof(MsspCounters), cudaMemcpyDeviceToHost, G.stream));
    CGB_CUDA_TRY(cudaEventRecord(G.ev_loop, G.stream));
    for (;;) {
        const cudaError_t e = cudaEventQuery(G.ev_loop);
        if (e == cudaSuccess) break;
        if (e != cudaErrorNotReady) CGB_CUDA_TRY(e);
        if (admission_due(s, G, 1) || s->coop_waiters.load() > 0)
            *reinterpret_cast<volatile uint32_t*>(G.mailbox) = 1;
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
    CGB_REQUIRE(!b.h->overflow, CGB_EOVERFLOW, "server SSSP loop: queue overflow");
    CGB_REQUIRE(!(h.ps.status & 1u), CGB_ETIMEOUT, "server SSSP loop: grid barrier gave up");
    for (uint32_t k = 0; k < kSrvSlots; k++) {
        G.thr[k] = h.thr[k];
        G.min_far[k] = h.min_far[k];
        G.last_empty[k] = h.last_empty[k] != 0;
    }
    G.near_alive = h.near_alive;
    G.far_alive = h.far_alive;
    G.cur = h.cur;
    G.fcur = h.fcur;
    G.tick += h.ticks;
    G.loop_levels += h.ticks;
    if (h.ticks) {
        // the host ticks' expansions read the thresholds from d_up: they moved on
        // the device, so the next host tick must not classify with the old ones
        // (a vertex improved into [old, new) would go to the far list and be
        // dropped by the next split, which starts at the new threshold)
        for (uint32_t k = 0; k < kSrvSlots; k++)
            G.h_up->thr[k] = (uint32_t)std::min<uint64_t>(G.thr[k], 0xFFFFFFFFu);
        CGB_CUDA_TRY(cudaMemcpyAsync(G.d_up->thr, G.h_up->thr, sizeof(G.h_up->thr), cudaMemcpyHostToDevice, G.stream));
    }
    G.loop_launches++;
    return h.ticks ? h.finished : 0ull;
}

// After the tick's kernels completed: slots whose traversal ended.
static unsigned long long group_finished(cgb_server* s, Group& G)
{
    cgb_graph* g = s->g;
    if (G.alg == CGB_BFS) {
        G.nact = g->h_ctr->qlen[G.cur ^ 1];
        G.medges = g->h_ctr->medges;
        CGB_REQUIRE(!g->h_ctr->overflow, CGB_EOVERFLOW, "server BFS queue overflow");
        const unsigned long long alive = G.h_stats->alive[0];
        G.live = alive;
        G.cur ^= 1;
        G.tick++;
        return G.active & ~alive;
    }
    CGB_REQUIRE(!G.sp->h->overflow, CGB_EOVERFLOW, "server SSSP queue overflow");
    G.near_alive = G.h_stats->alive[0];
    G.far_alive = G.h_stats->alive[1];
    for (uint32_t k = 0; k < kSrvSlots; k++) {
        if (!((G.split_mask >> k) & 1ull)) continue;
        G.min_far[k] = G.h_stats->min_far[k];
        G.last_empty[k] = !((G.near_alive >> k) & 1ull);
    }
    G.cur ^= 1;
    G.tick++;
    return G.active & ~(G.near_alive | G.far_alive);
}

// Results of the finished slots: statistics, copy to the request's buffer.
// `lone`: slots whose result region already holds a single-root run's result.
static void group_retire(cgb_server* s, Group& G, unsigned long long fin, unsigned long long lone = 0)
{
    if (!fin) return;
    cgb_graph* g = s->g;
    const uint32_t V = g->V;
    cudaStream_t st = G.stream;
    const unsigned long long ext = fin & ~lone;
    if (G.alg == CGB_SSSP && ext) {
        if (__builtin_popcountll(ext) <= 4) {
            uint32_t k[4] = {0, 0, 0, 0}, n = 0;
            for (unsigned long long m = ext; m; m &= m - 1) k[n++] = __builtin_ctzll(m);
            k_srv_sp_extract_cols<<<num_sms() * 8, kBlock, 0, st>>>(G.sp->dist, V, make_uint4(k[0], k[1], k[2], k[3]), n,
                                                                  G.region);
        } else {
            k_srv_sp_extract<<<num_sms() * 8, kBlock, 0, st>>>(G.sp->dist, V, ext, G.region);
        }
    }
    CGB_CUDA_TRY(cudaMemsetAsync(G.d_stats, 0, offsetof(SlotStats, alive), st));
    k_srv_stats<<<num_sms() * 4, kBlock, 0, st>>>(G.region, V, g->off, fin, G.d_stats->edges, G.d_stats->reached,
                                                G.d_stats->depth);
    for (unsigned long long m = fin; m; m &= m - 1) {
        const uint32_t k = __builtin_ctzll(m);
        if (G.out[k])
            CGB_CUDA_TRY(cudaMemcpyAsync(G.out[k], G.region + (size_t)k * V, (size_t)V * 4, cudaMemcpyDefault, st));
    }
    CGB_CUDA_TRY(cudaMemcpyAsync(G.h_stats, G.d_stats, offsetof(SlotStats, alive), cudaMemcpyDeviceToHost, st));
    CGB_CUDA_TRY(cudaStreamSynchronize(st));
    const double now = us_since(s, Clock::now());
    std::lock_guard<std::mutex> lk(s->mu);
    for (unsigned long long m = fin; m; m &= m - 1) {
        const uint32_t k = __builtin_ctzll(m);
        SrvReq& R = s->reqs[G.req[k]];
        R.info.traversed_edges = G.h_stats->edges[k];
        R.info.reached = G.h_stats->reached[k];
        R.info.depth = G.h_stats->depth[k];
        R.info.done_us = now;
        R.info.status = CGB_OK;
        if (!((lone >> k) & 1ull)) {
            const uint64_t n = ++s->batch_runs[G.alg == CGB_BFS ? 0 : 1];
            double& e = s->batch_est_us[G.alg == CGB_BFS ? 0 : 1];
            e += (now - R.info.admit_us - e) / (double)std::min<uint64_t>(n, 16);
        }
        s->done.push_back(R.info);
        s->completed++;
        G.state[k] = SlotState::kFree;
        G.req[k] = -1;
    }
    G.active &= ~fin;
    s->cv.notify_all();
}

// A query served alone on the single-root engine (the latency of a lone
// cgb_run).  Its result region gets the engine's result, and the slot
// retires as a batched one does.
constexpr uint32_t kLoneMaxDue = 4;

static void lone_run(cgb_server* s, Group& G, int a, uint32_t k)
{
    cgb_graph* g = (a == 1 && s->shadow) ? s->shadow : s->g;
    // the engine's device-resident loops are cooperative launches, as the
    // groups' are, so a run that may start one takes the cooperative-launch
    // lock: any BFS run (its small-frontier levels), and an SSSP run only
    // where its device-resident tail can run (no list of persist_deg edges or
    // more; on power-law graphs it never does, and SSSP runs then overlap
    // BFS runs and ticks)
    const cgb_tuning& t = g->tune_alg[CGB_SSSP];
    const bool coop_needed = a == 0 || (t.persist_enter > 0 && g->max_degree < t.persist_deg);
    Clock::time_point t0;
    {
        std::lock_guard<GraphMutex> glk(g->mu);
        std::unique_lock<std::mutex> coop(s->coop_mu, std::defer_lock);
        if (coop_needed) {
            s->coop_waiters++;
            coop.lock();
            s->coop_waiters--;
        }
        t0 = Clock::now();  // the run's own time, not the wait for the graph
        cgb_options o;
        memset(&o, 0, sizeof(o));
        o.struct_size = sizeof(o);
        run_one(g, G.alg, G.root[k], o);
        CGB_CUDA_TRY(cudaMemcpyAsync(G.region + (size_t)k * g->V, g->value, (size_t)g->V * 4,
                                     cudaMemcpyDeviceToDevice, g->stream));
        CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    }
    const double us = std::chrono::duration<double, std::micro>(Clock::now() - t0).count();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        const uint64_t n = ++s->lone_runs[a];
        s->lone_est_us[a] += (us - s->lone_est_us[a]) / (double)std::min<uint64_t>(n, 8);
    }
    group_retire(s, G, 1ull << k, 1ull << k);
}

// Pairs free slots with requests whose arrival time has passed.
static void pick_admissions(cgb_server* s, Group& G, std::deque<int64_t>& waiting, double now_us, uint32_t max_n)
{
    G.admit.clear();
    uint32_t k = 0;
    while (!waiting.empty() && G.admit.size() < max_n) {
        SrvReq& R = s->reqs[waiting.front()];
        if (R.info.arrival_us > now_us) break;
        while (k < G.nslots && G.state[k] != SlotState::kFree) k++;
        if (k >= G.nslots) break;
        G.state[k] = SlotState::kActive;
        G.req[k] = waiting.front();
        G.root[k] = R.info.root;
        G.out[k] = R.out;
        G.active |= 1ull << k;
        R.info.slot = k;
        R.info.admit_us = now_us;
        G.admit.push_back(k);
        waiting.pop_front();
    }
}

// The serving loop of one group (a = 0 BFS, 1 SSSP); each group has its
// own thread and stream, so short BFS levels never wait for SSSP rounds.
// The BFS group uses the graph's shared scratch (counters, chunk queue) and
// holds the graph's lock for each tick; the SSSP group touches only its own
// buffers and the read-only CSR.
static void group_loop(cgb_server* s, int a)
{
    cgb_graph* g = s->g;
    Group& G = s->grp[a];
    int lone_k = -1;         // slot admitted this tick for the single-root engine
    bool other_idle = true;  // the other group had no query at this tick's admission
    try {
        CGB_CUDA_TRY(cudaSetDevice(g->device));
        while (!s->stop.load()) {
            {
                std::unique_lock<std::mutex> lk(s->mu);
                if (s->error != CGB_OK) break;
                const double now = us_since(s, Clock::now());
                // up to kLoneMaxDue due queries are served one by one on the
                // single-root engine while that ends them sooner than a batch
                // would (running means of both services), else they are batched.
                // This holds while the group's batch runs too (a single-root run
                // then comes between two of its ticks): otherwise one batched query
                // at moderate load made every later arrival join a slow batch of a
                // few.  The cap bounds how long single-root runs, which hold the
                // graph, keep the other group's ticks waiting; and under load a
                // batch serves many more queries per second.
                bool lone = false;
                if (!(s->flags & CGB_SERVER_BATCH_ONLY)) {
                    uint32_t due = 0;
                    for (const int64_t r : s->waiting[a]) {
                        if (s->reqs[r].info.arrival_us > now || due > kLoneMaxDue) break;
                        due++;
                    }
                    lone = due > 0 && due <= kLoneMaxDue &&
                           (double)due * s->lone_est_us[a] <= std::max(s->batch_est_us[a], s->lone_est_us[a]);
                }
                // a running group takes new queries only while at least half of
                // its slots are free (unless CGB_SERVER_ADMIT_ANY_SLOT), so that
                // admitted queries share more of their dense levels
                const bool hold = !(s->flags & CGB_SERVER_ADMIT_ANY_SLOT) && G.active != 0 &&
                                  2u * (uint32_t)__builtin_popcountll(G.active) > G.nslots;
                // the device-resident loops run only while the other group is idle:
                // they take turns on the cooperative-launch lock, whereas ticks of
                // both groups overlap on their two streams
                other_idle = s->grp[a ^ 1].active == 0;
                if (lone) pick_admissions(s, G, s->waiting[a], now, 1u);  // needs a free slot, not a batch
                else if (!hold) pick_admissions(s, G, s->waiting[a], now, kSrvSlots);
                else G.admit.clear();
                if (lone && G.admit.size() == 1) {
                    lone_k = (int)G.admit[0];
                    G.admit.clear();
                }
                if (!G.active) {
                    if (s->waiting[a].empty()) {
                        s->cv.wait_for(lk, std::chrono::milliseconds(5));
                    } else {
                        const double t = s->reqs[s->waiting[a].front()].info.arrival_us;
                        if (t > now) s->cv.wait_for(lk, std::chrono::microseconds((int64_t)(t - now) + 1));
                    }
                    continue;
                }
            }
            const auto t_tick = Clock::now();
            unsigned long long fin;
            if (lone_k >= 0) {
                lone_run(s, G, a, (uint32_t)lone_k);
                lone_k = -1;
            } else if (a == 0) {
                std::lock_guard<GraphMutex> glk(g->mu);
                g->tune = g->tune_alg[CGB_BFS];
                bfs_admit(s, G);
                // small frontiers whose levels push: on the device, many levels per launch
                const uint32_t nf_exit = std::max<uint32_t>(g->tune.persist_enter, 1u);
                const bool pull = (double)G.medges * 15.0 > (double)g->E;
                uint64_t before = G.loop_levels;
                fin = 0;
                if (G.loop && other_idle && G.nact > 0 && G.nact <= nf_exit && !pull)
                    fin = bfs_device_levels(s, G, nf_exit);
                if (G.loop_levels == before) {
                    bfs_issue(s, G);
                    CGB_CUDA_TRY(cudaMemcpyAsync(G.h_stats->alive, G.d_stats->alive, sizeof(G.h_stats->alive),
                                                 cudaMemcpyDeviceToHost, G.stream));
                    CGB_CUDA_TRY(cudaMemcpyAsync(g->h_ctr, g->ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost,
                                                 G.stream));
                    CGB_CUDA_TRY(cudaStreamSynchronize(G.stream));
                    fin = group_finished(s, G);
                }
                group_retire(s, G, fin);
            } else {
                uint64_t before = G.loop_levels;
                fin = 0;
                if (G.sp_loop && other_idle) {
                    sp_admit(s, G);
                    fin = sp_device_ticks(s, G);
                }
                if (G.loop_levels == before) {
                    sp_issue(s, G);
                    CGB_CUDA_TRY(cudaStreamSynchronize(G.stream));
                    fin = group_finished(s, G);
                }
                group_retire(s, G, fin);
            }
            std::lock_guard<std::mutex> lk(s->mu);
            s->ticks[a]++;
            s->busy_ms[a] += std::chrono::duration<double, std::milli>(Clock::now() - t_tick).count();
        }
    } catch (const Error& e) {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->error == CGB_OK) {
            s->error = e.code;
            s->error_msg = e.msg;
        }
    } catch (const std::exception& e) {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->error == CGB_OK) {
            s->error = CGB_ECUDA;
            s->error_msg = e.what();
        }
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->error != CGB_OK) {
        // requests still admitted or waiting end with the error
        for (auto& R : s->reqs)
            if (R.info.done_us == 0 && R.info.status == CGB_OK) {
                R.info.status = s->error;
                R.info.done_us = us_since(s, Clock::now());
                s->done.push_back(R.info);
                s->completed++;
            }
        for (int k = 0; k < 2; k++) s->waiting[k].clear();
    }
    s->cv.notify_all();
}

}  // namespace cgb

template <typename F>
static cgb_status sguard(F&& f)
{
    try {
        f();
        return CGB_OK;
    } catch (const Error& e) {
        set_error(e.msg);
        return e.code;
    } catch (const std::exception& e) {
        set_error(e.what());
        return CGB_ECUDA;
    }
}

extern "C" {

cgb_status cgb_server_create(cgb_graph* g, const cgb_server_config* cfg, cgb_server** out)
{
    return sguard([&] {
        CGB_REQUIRE(g != nullptr && out != nullptr, CGB_EINVAL, "NULL argument");
        *out = nullptr;
        cgb_server_config c{};
        c.struct_size = sizeof(c);
        if (cfg) {
            CGB_REQUIRE(cfg->struct_size >= sizeof(c), CGB_EINVAL, "cgb_server_config.struct_size too small");
            c = *cfg;
        }
        uint32_t nb = c.bfs_slots ? std::min(c.bfs_slots, kSrvSlots) : kSrvSlots;
        uint32_t ns = c.sssp_slots ? std::min(c.sssp_slots, kSrvSlots) : kSrvSlots;
        if (c.flags & CGB_SERVER_NO_BFS) nb = 0;
        if (c.flags & CGB_SERVER_NO_SSSP) ns = 0;
        const uint64_t per_slot = 4ull * g->V;  // one result region per slot
        if (c.memory_budget) {
            const uint64_t fit = c.memory_budget / per_slot;
            CGB_REQUIRE(fit >= (uint64_t)((nb ? 1 : 0) + (ns ? 1 : 0)), CGB_ENOMEM,
                        "memory budget holds no result region");
            // split the regions that fit between the groups in proportion to their slot requests
            while ((uint64_t)nb + ns > fit) {
                if (nb >= ns && nb > 1) nb--;
                else if (ns > 1) ns--;
                else break;
            }
        }
        std::lock_guard<GraphMutex> lock(g->mu);
        CGB_CUDA_TRY(cudaSetDevice(g->device));
        ensure_frontier(g);
        if (nb) ensure_csc(g);
        if (ns && g->w && g->sum_w == 0) compute_weight_sum(g);
        cgb_server* s = new cgb_server();
        s->g = g;
        s->flags = c.flags;
        try {
            group_alloc(s, s->grp[0], CGB_BFS, nb);
            group_alloc(s, s->grp[1], CGB_SSSP, ns);
            s->grp[1].delta = c.sssp_delta ? c.sssp_delta : mssp_default_delta(g);
            if (ns && !(c.flags & CGB_SERVER_BATCH_ONLY)) s->shadow = graph_shadow(g);
            CGB_CUDA_TRY(cudaDeviceSynchronize());
        } catch (...) {
            group_free(s, s->grp[0]);
            group_free(s, s->grp[1]);
            graph_shadow_free(s->shadow);
            delete s;
            throw;
        }
        g->servers++;
        *out = s;
    });
}

cgb_status cgb_server_submit(cgb_server* s, int algorithm, uint32_t root, double arrival_us, uint32_t* out_u32,
                             uint64_t* id)
{
    return sguard([&] {
        CGB_REQUIRE(s != nullptr, CGB_EINVAL, "server is NULL");
        CGB_REQUIRE(algorithm == CGB_BFS || algorithm == CGB_SSSP, CGB_EINVAL, "server requests are BFS or SSSP");
        CGB_REQUIRE(root < s->g->V, CGB_EINVAL, "root >= vertexNum");
        const int a = algorithm == CGB_BFS ? 0 : 1;
        CGB_REQUIRE(s->grp[a].nslots > 0, CGB_EUNSUPPORTED, "server has no slots for this algorithm");
        std::lock_guard<std::mutex> lk(s->mu);
        CGB_REQUIRE(s->error == CGB_OK, s->error, "server stopped after an error");
        SrvReq R;
        R.info.id = s->reqs.size();
        R.info.algorithm = algorithm;
        R.info.root = root;
        R.info.arrival_us = arrival_us;
        R.info.status = CGB_OK;
        R.out = out_u32;
        // keep each queue ordered by arrival time
        auto& wq = s->waiting[a];
        s->reqs.push_back(R);
        const int64_t idx = (int64_t)s->reqs.size() - 1;
        auto it = wq.end();
        while (it != wq.begin() && s->reqs[*(it - 1)].info.arrival_us > arrival_us) --it;
        wq.insert(it, idx);
        if (id) *id = R.info.id;
        s->cv.notify_all();
    });
}

cgb_status cgb_server_start(cgb_server* s)
{
    return sguard([&] {
        CGB_REQUIRE(s != nullptr, CGB_EINVAL, "server is NULL");
        CGB_REQUIRE(!s->started, CGB_EINVAL, "server already started");
        s->t0 = Clock::now();
        s->started = true;
        for (int a = 0; a < 2; a++)
            if (s->grp[a].nslots) s->th[a] = std::thread(group_loop, s, a);
    });
}

cgb_status cgb_server_wait(cgb_server* s, double timeout_ms, uint32_t* pending)
{
    return sguard([&] {
        CGB_REQUIRE(s != nullptr, CGB_EINVAL, "server is NULL");
        std::unique_lock<std::mutex> lk(s->mu);
        const auto until = Clock::now() + std::chrono::microseconds((int64_t)(timeout_ms * 1000.0));
        while (s->completed < s->reqs.size() && s->error == CGB_OK) {
            if (s->cv.wait_until(lk, until) == std::cv_status::timeout) break;
        }
        if (pending) *pending = (uint32_t)(s->reqs.size() - s->completed);
        CGB_REQUIRE(s->error == CGB_OK, s->error, s->error_msg);
    });
}

cgb_status cgb_server_poll(cgb_server* s, cgb_request_info* out, uint32_t cap, uint32_t* n)
{
    return sguard([&] {
        CGB_REQUIRE(s != nullptr && n != nullptr, CGB_EINVAL, "NULL argument");
        std::lock_guard<std::mutex> lk(s->mu);
        const uint32_t k = (uint32_t)std::min<size_t>(cap, s->done.size());
        if (out) {
            std::copy(s->done.begin(), s->done.begin() + k, out);
            s->done.erase(s->done.begin(), s->done.begin() + k);
        }
        *n = out ? k : (uint32_t)s->done.size();
    });
}

cgb_status cgb_server_stats(const cgb_server* s, uint64_t* ticks, uint32_t* bfs_slots, uint32_t* sssp_slots,
                            double* busy_ms)
{
    return sguard([&] {
        CGB_REQUIRE(s != nullptr, CGB_EINVAL, "server is NULL");
        if (ticks) *ticks = s->ticks[0] + s->ticks[1];
        if (bfs_slots) *bfs_slots = s->grp[0].nslots;
        if (sssp_slots) *sssp_slots = s->grp[1].nslots;
        if (busy_ms) *busy_ms = s->busy_ms[0] + s->busy_ms[1];
    });
}

cgb_status cgb_server_destroy(cgb_server* s)
{
    return sguard([&] {
        if (!s) return;
        s->stop.store(true);
        s->cv.notify_all();
        for (int a = 0; a < 2; a++)
            if (s->th[a].joinable()) s->th[a].join();
        cudaSetDevice(s->g->device);
        group_free(s, s->grp[0]);
        group_free(s, s->grp[1]);
        graph_shadow_free(s->shadow);
        s->g->servers--;
        delete s;
    });
}

}  // extern "C"
