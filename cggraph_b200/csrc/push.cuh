// Degree-binned push expansion over a vertex frontier.
//
// Replaces the reference's per-thread load balancers WarpDonate::schedule
// (my_project/CGgraph/device_warpDonate.cuh:42-388) and CTA::schedule
// (my_project/CGgraph/device_CTA.cuh:28-112), which run one frontier vertex
// per thread and hand large lists to the warp or CTA with __syncthreads
// loops, serialising a hub's whole list on one CTA.  Here each frontier
// vertex is binned by out-degree:
//   deg >= kHugeDeg          deferred to k_push_huge, which splits the list
//                            into kHugeChunk-edge chunks across every CTA;
//   kCtaDeg <= deg < kHuge   the whole CTA walks the list (owner election);
//   32 <= deg < kCtaDeg      one warp walks the list (ballot election);
//   deg < 32                 fine-grained gather: a CTA-wide exclusive scan of
//                            the remaining degrees packs the small lists
//                            into shared memory, one edge per thread.
// Every edge visit is warp-collective (Op::edge is called by all 32 lanes,
// with `valid` false on idle lanes) so that the ops can aggregate their
// queue appends with one ballot and one atomic per warp.
#pragma once

#include <type_traits>

#include "common.cuh"
#include "engine.cuh"

namespace cgb {

// Batched edge visits.  An op that declares `static constexpr int kBatch = N`
// also provides
//   template <int M> __device__ void edges(const bool (&valid)[M],
//                                          const uint32_t (&e)[M],
//                                          const uint32_t (&msg)[M]) const;
// (warp-collective, like edge) which visits M edge slots per lane at once:
// every load of the M slots is issued before any of them is used, so a lane
// keeps M gathers in flight instead of one dependent chain per edge.  The
// expansion loops below hand such ops N slots per lane (32 * N edges per
// warp step); other ops are called edge by edge.
template <class T, class = void>
struct op_batch {
    static constexpr int value = 1;
};
template <class T>
struct op_batch<T, std::void_t<decltype(T::kBatch)>> {
    static constexpr int value = T::kBatch;
};

template <class Op, int N>
__device__ __forceinline__ void visit_n(const Op& op, const bool (&valid)[N], const uint32_t (&e)[N],
                                        const uint32_t (&m)[N])
{
    if constexpr (op_batch<Op>::value == 1) {
#pragma unroll
        for (int i = 0; i < N; i++) op.edge(valid[i], e[i], m[i]);
    } else {
        op.template edges<N>(valid, e, m);
    }
}

// Edges [first, end) of one list walked by the calling warp (all lanes call
// it with the same arguments), op_batch<Op> slots per lane at a time.
template <class Op>
__device__ __forceinline__ void warp_range(const Op& op, uint32_t first, uint32_t end, uint32_t m)
{
    constexpr int N = op_batch<Op>::value;
    const uint32_t lane = lane_id();
    for (uint32_t k = first; k < end; k += 32 * N) {
        bool valid[N];
        uint32_t e[N], mm[N];
#pragma unroll
        for (int i = 0; i < N; i++) {
            const uint32_t idx = k + 32 * i + lane;
            valid[i] = idx < end;
            e[i] = valid[i] ? idx : 0u;
            mm[i] = m;
        }
        visit_n<Op, N>(op, valid, e, mm);
    }
}

// The same for a whole CTA of kBlk threads (every thread calls it with the
// same arguments).
template <class Op, int kBlk>
__device__ __forceinline__ void cta_range(const Op& op, uint32_t first, uint32_t end, uint32_t m)
{
    constexpr int N = op_batch<Op>::value;
    for (uint32_t k = first; k < end; k += kBlk * N) {
        bool valid[N];
        uint32_t e[N], mm[N];
#pragma unroll
        for (int i = 0; i < N; i++) {
            const uint32_t idx = k + kBlk * i + threadIdx.x;
            valid[i] = idx < end;
            e[i] = valid[i] ? idx : 0u;
            mm[i] = m;
        }
        visit_n<Op, N>(op, valid, e, mm);
    }
}

// Warp-aggregated append of up to N items per lane (pred[i] selects item
// i): one atomic per warp.  Every lane of the warp must call it.  Items past
// `cap` are not written and raise *overflow.
template <int N>
__device__ __forceinline__ void warp_append_n(const bool (&pred)[N], const uint32_t (&item)[N], uint32_t* q,
                                              uint32_t* ctr, uint32_t cap, uint32_t* overflow)
{
    uint32_t cnt = 0;
#pragma unroll
    for (int i = 0; i < N; i++) cnt += pred[i] ? 1u : 0u;
    const uint32_t incl = warp_incl_scan(cnt);
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    if (total == 0) return;
    uint32_t base = 0;
    if (lane_id() == 0) base = atomicAdd(ctr, total);
    uint32_t idx = __shfl_sync(0xffffffffu, base, 0) + incl - cnt;
#pragma unroll
    for (int i = 0; i < N; i++) {
        if (pred[i]) {
            if (idx < cap) q[idx] = item[i];
            else atomicOr(overflow, 1u);
            idx++;
        }
    }
}

// CTA-aggregated append of up to N items per thread: one atomic per CTA of
// kBlock threads instead of one per warp (a queue counter that every warp of
// a full-graph scan hits serialises at its L2 slice).  Every thread of the
// CTA must call it: it synchronises the CTA.
template <int N>
__device__ __forceinline__ void block_append_n(const bool (&pred)[N], const uint32_t (&item)[N], uint32_t* q,
                                               uint32_t* ctr, uint32_t cap, uint32_t* overflow)
{
    __shared__ uint32_t s_scan[kBlock / 32 + 1];
    __shared__ uint32_t s_base;
    uint32_t cnt = 0;
#pragma unroll
    for (int i = 0; i < N; i++) cnt += pred[i] ? 1u : 0u;
    uint32_t total;
    const uint32_t excl = block_excl_scan(cnt, total, s_scan);
    if (total == 0) return;  // uniform across the CTA
    if (threadIdx.x == 0) s_base = atomicAdd(ctr, total);
    __syncthreads();
    uint32_t idx = s_base + excl;
#pragma unroll
    for (int i = 0; i < N; i++) {
        if (pred[i]) {
            if (idx < cap) q[idx] = item[i];
            else atomicOr(overflow, 1u);
            idx++;
        }
    }
    __syncthreads();  // s_base is rewritten by the next call
}

// Fine-grained tier: a CTA-wide exclusive scan of the (small) remaining
// degrees packs the lists into shared memory, one edge per thread per round.
// Every thread of the CTA must call it.
template <class Op>
__device__ __forceinline__ void fine_tier(const Op& op, uint32_t start, uint32_t deg, uint32_t msg, uint32_t* s_scan,
                                          uint32_t* s_edge, uint32_t* s_emsg)
{
    const uint32_t tid = threadIdx.x;
    uint32_t total;
    const uint32_t rank = block_excl_scan(deg, total, s_scan);
    uint32_t consumed = 0;
    for (uint32_t done = 0; done < total; done += kBlock) {
        while (consumed < deg && rank + consumed < done + kBlock) {
            s_edge[rank + consumed - done] = start + consumed;
            s_emsg[rank + consumed - done] = msg;
            consumed++;
        }
        __syncthreads();
        const uint32_t n = min((uint32_t)kBlock, total - done);
        const bool valid = tid < n;
        op.edge(valid, valid ? s_edge[tid] : 0u, valid ? s_emsg[tid] : 0u);
        __syncthreads();
    }
}

// Fine-grained tier of one warp (no CTA barriers): a warp-inclusive scan of
// the lanes' remaining degrees (each below 32) packs their lists into rounds
// of 32 edges; in each round every lane takes one edge and finds the lane
// that owns it -- the last lane whose exclusive prefix is <= the edge's
// position -- by a 5-step shuffle search.  Batched ops take op_batch<Op>
// rounds at once.  Called by all 32 lanes.
template <class Op>
__device__ __forceinline__ void fine_tier_warp(const Op& op, uint32_t start, uint32_t deg, uint32_t msg)
{
    constexpr int N = op_batch<Op>::value;
    const uint32_t lane = lane_id();
    uint32_t incl = deg;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += t;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    const uint32_t excl = incl - deg;
    for (uint32_t base = 0; base < total; base += 32 * N) {
        bool valid[N];
        uint32_t e[N], mm[N];
#pragma unroll
        for (int i = 0; i < N; i++) {
            const uint32_t idx = base + 32 * i + lane;
            uint32_t o = 0;
#pragma unroll
            for (uint32_t step = 16; step >= 1; step >>= 1) {
                const uint32_t ex = __shfl_sync(0xffffffffu, excl, o + step);
                if (ex <= idx) o += step;
            }
            const uint32_t st = __shfl_sync(0xffffffffu, start, o);
            const uint32_t ex = __shfl_sync(0xffffffffu, excl, o);
            mm[i] = __shfl_sync(0xffffffffu, msg, o);
            valid[i] = idx < total;
            e[i] = valid[i] ? st + (idx - ex) : 0u;
        }
        visit_n<Op, N>(op, valid, e, mm);
    }
}

// Op interface:
//   __device__ bool load(uint32_t v, uint32_t& start, uint32_t& deg, uint32_t& msg) const;
//   __device__ void edge(bool valid, uint32_t e, uint32_t msg) const;   // warp-collective
// and, for the engine's kernels (k_push_binned, k_push_chunks), per-CTA hooks
// around all of a CTA's work, each followed / preceded by a CTA barrier:
//   __device__ void block_begin() const;   // e.g. zero shared accumulators
//   __device__ void block_end() const;     // e.g. flush them with one atomic
template <class Op, bool kIdentity>
__global__ void __launch_bounds__(kBlock) k_push_twc(const uint32_t* __restrict__ qin, uint32_t nin, Op op,
                                                     uint32_t* __restrict__ huge_q, uint32_t* huge_len,
                                                     uint32_t huge_cap)
{
    __shared__ uint32_t s_scan[kBlock / 32 + 1];
    __shared__ uint32_t s_owner, s_start, s_deg, s_msg;
    __shared__ uint32_t s_edge[kBlock];
    __shared__ uint32_t s_emsg[kBlock];
    const uint32_t tid = threadIdx.x;

    for (uint32_t base = blockIdx.x * kBlock; base < nin; base += gridDim.x * kBlock) {
        uint32_t i = base + tid;
        uint32_t start = 0, deg = 0, msg = 0;
        if (i < nin) {
            uint32_t v = kIdentity ? i : qin[i];
            if (!op.load(v, start, deg, msg)) deg = 0;
            if (deg >= kHugeDeg) {
                // capacity V: each vertex appears at most once per frontier
                const uint32_t slot = atomicAdd(huge_len, 1u);
                if (slot < huge_cap) huge_q[slot] = v;
                deg = 0;
            }
        }
        // CTA tier
        while (__syncthreads_or(deg >= kCtaDeg)) {
            if (deg >= kCtaDeg) s_owner = tid;
            __syncthreads();
            if (s_owner == tid) {
                s_start = start;
                s_deg = deg;
                s_msg = msg;
                deg = 0;
            }
            __syncthreads();
            const uint32_t st = s_start, dg = s_deg, m = s_msg;
            for (uint32_t k = 0; k < dg; k += kBlock) op.edge(k + tid < dg, st + k + tid, m);
            __syncthreads();
        }
        // warp tier
        uint32_t wmask;
        while ((wmask = __ballot_sync(0xffffffffu, deg >= 32)) != 0) {
            const uint32_t leader = __ffs(wmask) - 1;
            const uint32_t st = __shfl_sync(0xffffffffu, start, leader);
            const uint32_t dg = __shfl_sync(0xffffffffu, deg, leader);
            const uint32_t m = __shfl_sync(0xffffffffu, msg, leader);
            if (lane_id() == leader) deg = 0;
            for (uint32_t k = 0; k < dg; k += 32) op.edge(k + lane_id() < dg, st + k + lane_id(), m);
        }
        fine_tier(op, start, deg, msg, s_scan, s_edge, s_emsg);
    }
}

// Hubs deferred by k_push_twc: the concatenated chunk list of all deferred
// vertices is dealt round-robin to the CTAs of the grid.
template <class Op>
__global__ void __launch_bounds__(kBlock) k_push_huge(const uint32_t* __restrict__ huge_q, const uint32_t* huge_len,
                                                      uint32_t huge_cap, Op op)
{
    const uint32_t n = min(*huge_len, huge_cap);
    uint64_t chunk_base = 0;
    for (uint32_t h = 0; h < n; h++) {
        const uint32_t v = huge_q[h];
        uint32_t start, deg, msg;
        if (!op.load(v, start, deg, msg)) continue;
        const uint32_t nch = (deg + kHugeChunk - 1) / kHugeChunk;
        const uint32_t first = (uint32_t)((blockIdx.x + gridDim.x - (chunk_base % gridDim.x)) % gridDim.x);
        for (uint32_t c = first; c < nch; c += gridDim.x) {
            const uint32_t cs = c * kHugeChunk;
            const uint32_t ce = min(deg, cs + kHugeChunk);
            for (uint32_t k = cs; k < ce; k += kBlock) op.edge(k + threadIdx.x < ce, start + k + threadIdx.x, msg);
        }
        chunk_base += nch;
    }
}

// Binned expansion used by the engine.  Lists of at least big_deg edges are
// cut into chunk-edge pieces whose descriptors (vertex, chunk index) go to a
// chunk queue; k_push_chunks then deals the chunks across the whole grid, so
// a frontier of a few hubs keeps every SM busy however few vertices it has.
// Lists of 32..big_deg-1 edges are walked by one warp, shorter ones by the
// warp's fine-grained tier (fine_tier_warp).  Chunk-queue capacity
// E/chunk + E/big_deg + 64 bounds any frontier in which each vertex appears
// once; the queue is sized for the smallest chunk and big_deg launch_push
// uses (kMinChunk and 32).
template <class Op, bool kIdentity, int kBlk>
__global__ void __launch_bounds__(kBlk) k_push_binned(const uint32_t* __restrict__ qin, uint32_t nin, Op op,
                                                        uint2* __restrict__ chunk_q, uint32_t* chunk_len,
                                                        uint32_t chunk_cap, uint32_t* overflow, uint32_t big_deg,
                                                        uint32_t chunk)
{
    op.block_begin();
    __syncthreads();
    for (uint32_t base = blockIdx.x * kBlk; base < nin; base += gridDim.x * kBlk) {
        const uint32_t i = base + threadIdx.x;
        uint32_t v = 0, start = 0, deg = 0, msg = 0;
        if (i < nin) {
            v = kIdentity ? i : qin[i];
            if (!op.load(v, start, deg, msg)) deg = 0;
        }
        // big lists: the warp writes their chunk descriptors together
        uint32_t bmask;
        while ((bmask = __ballot_sync(0xffffffffu, deg >= big_deg)) != 0) {
            const uint32_t leader = __ffs(bmask) - 1;
            const uint32_t bv = __shfl_sync(0xffffffffu, v, leader);
            const uint32_t nch = (__shfl_sync(0xffffffffu, deg, leader) + chunk - 1) / chunk;
            uint32_t slot = 0;
            if (lane_id() == 0) slot = atomicAdd(chunk_len, nch);
            slot = __shfl_sync(0xffffffffu, slot, 0);
            for (uint32_t c = lane_id(); c < nch; c += 32) {
                if (slot + c < chunk_cap) chunk_q[slot + c] = make_uint2(bv, c);
                else atomicOr(overflow, 1u);
            }
            if (lane_id() == leader) deg = 0;
        }
        // warp tier
        uint32_t wmask;
        while ((wmask = __ballot_sync(0xffffffffu, deg >= 32)) != 0) {
            const uint32_t leader = __ffs(wmask) - 1;
            const uint32_t st = __shfl_sync(0xffffffffu, start, leader);
            const uint32_t dg = __shfl_sync(0xffffffffu, deg, leader);
            const uint32_t m = __shfl_sync(0xffffffffu, msg, leader);
            if (lane_id() == leader) deg = 0;
            warp_range(op, st, st + dg, m);
        }
        fine_tier_warp(op, start, deg, msg);
    }
    __syncthreads();
    op.block_end();
}

// One CTA per chunk descriptor, grid-stride over the chunk queue.
template <class Op, int kBlk>
__global__ void __launch_bounds__(kBlk) k_push_chunks(const uint2* __restrict__ chunk_q, const uint32_t* chunk_len,
                                                        uint32_t chunk_cap, Op op, uint32_t chunk)
{
    const uint32_t n = min(*chunk_len, chunk_cap);
    if (blockIdx.x >= n) return;
    op.block_begin();
    __syncthreads();
    for (uint32_t c = blockIdx.x; c < n; c += gridDim.x) {
        const uint2 d = chunk_q[c];
        uint32_t start, deg, msg;
        if (!op.load(d.x, start, deg, msg)) continue;
        const uint32_t cs = d.y * chunk;
        const uint32_t ce = min(deg, cs + chunk);
        cta_range<Op, kBlk>(op, start + cs, start + ce, msg);
    }
    __syncthreads();
    op.block_end();
}

// Frontiers of at most this many vertices cut every list of 32 edges or
// more into kMinChunk-edge chunks: with few vertices per thread, a warp
// walking a long list alone would leave most of the grid idle.
constexpr uint32_t kSmallFrontier = 32768;

template <class Op, int kBlk>
inline void launch_push_blk(cgb_graph* g, const uint32_t* qin, uint32_t nin, const Op& op, bool identity,
                            uint32_t ctas, uint32_t big_deg, uint32_t chunk)
{
    const uint32_t grid = grid_for(nin, kBlk, ctas);
    if (identity)
        k_push_binned<Op, true, kBlk><<<grid, kBlk, 0, g->stream>>>(qin, nin, op, g->chunk_q, &g->ctr->chunk_len,
                                                                     g->chunk_cap, &g->ctr->overflow, big_deg, chunk);
    else
        k_push_binned<Op, false, kBlk><<<grid, kBlk, 0, g->stream>>>(qin, nin, op, g->chunk_q, &g->ctr->chunk_len,
                                                                      g->chunk_cap, &g->ctr->overflow, big_deg, chunk);
    k_push_chunks<Op, kBlk><<<ctas, kBlk, 0, g->stream>>>(g->chunk_q, &g->ctr->chunk_len, g->chunk_cap, op, chunk);
}

// Expansion variants of launch_push: the size rule (chunk every list of 32
// edges or more for frontiers of at most kSmallFrontier vertices, else only
// lists of push_big_deg edges or more), or either tier forced.
enum PushExpand { kExpandAuto = 0, kExpandBinned = 1, kExpandChunked = 2 };

// Launches the binned expansion (plus the chunk kernel) of a queue whose
// length the host knows, with the graph's tuned CTA size (push_block) and
// grid.  The chunk-queue length must be zero beforehand.
template <class Op>
inline void launch_push(cgb_graph* g, const uint32_t* qin, uint32_t nin, const Op& op, bool identity,
                        int expand = kExpandAuto)
{
    if (nin == 0) return;
    const cgb_tuning& t = g->tune;
    const uint32_t ctas = num_sms() * t.push_ctas_per_sm;
    const bool small = expand == kExpandAuto ? nin <= kSmallFrontier : expand == kExpandChunked;
    const uint32_t big_deg = small ? 32u : t.push_big_deg;
    const uint32_t chunk = small ? kMinChunk : t.push_chunk;
    g->stats.launches += 2;
    if (t.push_block == 128) launch_push_blk<Op, 128>(g, qin, nin, op, identity, ctas, big_deg, chunk);
    else if (t.push_block == 512) launch_push_blk<Op, 512>(g, qin, nin, op, identity, ctas, big_deg, chunk);
    else launch_push_blk<Op, 256>(g, qin, nin, op, identity, ctas, big_deg, chunk);
}

}  // namespace cgb
