// Connected components with the reference's result semantics.
//
// The reference initialises label[v] = v and pushes labels along out-edges
// with atomicMin until nothing changes (my_project/CGgraph/GraphNuma.cuh:539-544,
// host_algorithm.hpp:412-433, device_algorithm.cuh:430-465).  The fixpoint is
// label[v] = min{u : u reaches v}; on a symmetric graph that is the minimum
// vertex id of v's connected component.
//
// Symmetric graphs (checked once per graph): min-label hooking with pointer
// jumping, in the sampling order of Afforest (Sutton, Ben-Nun, Barak 2018):
//   1. comp[v] = min(v, first neighbour) -- lists are sorted, so that is the
//      smallest neighbour; every pointer goes to a smaller vertex along an
//      edge, so this is already a valid forest, built without atomics (the
//      initialisation of ECL-CC, Jaiganesh and Burtscher 2018);
//   2. one round that links v with its second neighbour, and with its first
//      one where step 1 left it pointing at itself (first neighbour larger);
//      every find halves the path it walks, so no separate compress pass
//      runs before step 5;
//   3. find the roots of 1024 hashed vertices and take the most frequent
//      one as the giant component c;
//   4. link every remaining edge of each vertex whose root is not c (the
//      giant component's own edges can be skipped because every edge leaving
//      it is seen again from its other, non-giant endpoint), with the
//      degree-binned expansion of push.cuh so hubs are split across CTAs;
//   5. compress.
// Linking always hooks the larger root under the smaller one, so comp[x] <= x
// holds throughout and each final root is its component's minimum id.
//
// Directed graphs: the reference's own label propagation, frontier-driven.
#include "engine.cuh"
#include "push.cuh"

namespace cgb {

constexpr uint32_t kLinkRetries = 1u << 20;

__device__ __forceinline__ uint32_t ld_comp(const uint32_t* comp, uint32_t i)
{
    return *((volatile const uint32_t*)comp + i);
}

// Hooks the trees of u and v, larger root under smaller root.
// Root of x with path halving: each visited vertex is pointed at its
// grandparent on the way up.  Concurrent halving is benign: a vertex only
// ever moves to one of its own ancestors, so every pointer still goes to a
// smaller vertex of the same tree.
__device__ __forceinline__ uint32_t find_halve(uint32_t x, uint32_t* comp)
{
    uint32_t p = ld_comp(comp, x);
    for (uint32_t steps = 0; p != x && steps < kLinkRetries; steps++) {
        const uint32_t gp = ld_comp(comp, p);
        if (gp != p) *((volatile uint32_t*)comp + x) = gp;
        x = gp;
        p = ld_comp(comp, x);
    }
    return x;
}

__device__ __forceinline__ void link(uint32_t u, uint32_t v, uint32_t* comp, DevCounters* ctr)
{
    uint32_t p1 = find_halve(u, comp), p2 = find_halve(v, comp);
    for (uint32_t tries = 0; p1 != p2; tries++) {
        if (tries >= kLinkRetries) {
            atomicOr(&ctr->link_giveup, 1u);
            return;
        }
        const uint32_t high = max(p1, p2), low = min(p1, p2);
        // hook the larger root under the smaller one; on failure another
        // thread hooked `high` first: retry from both roots' new roots
        if (atomicCAS(comp + high, high, low) == high) return;
        p1 = find_halve(high, comp);
        p2 = find_halve(low, comp);
    }
}

__global__ void k_cc_init(uint32_t V, uint32_t* comp)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) comp[i] = i;
}

// comp[v] = min(v, smallest neighbour) (symmetric graphs, sorted lists).
__global__ void k_cc_init_min_nbr(uint32_t V, const uint32_t* __restrict__ off, const uint32_t* __restrict__ dst,
                                  uint32_t* comp)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        const uint32_t s = off[v];
        comp[v] = (off[v + 1] > s) ? min(v, dst[s]) : v;
    }
}

// Links v with its r-th neighbour; with `first_up` also with its first
// neighbour when that one is larger than v (the min-neighbour
// initialisation only covered edge 0 when it pointed down).
__global__ void k_cc_link_round(uint32_t V, const uint32_t* __restrict__ off, const uint32_t* __restrict__ dst,
                                uint32_t* comp, uint32_t r, int first_up, DevCounters* ctr)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        const uint32_t s = off[v], d = off[v + 1] - s;
        if (first_up && d > 0 && dst[s] > v) link(v, dst[s], comp, ctr);
        if (d > r) link(v, dst[s + r], comp, ctr);
    }
}

// Points every vertex at its root (path halving on the way, which shortens
// the chains that other threads are still walking).
__global__ void k_cc_compress(uint32_t V, uint32_t* comp)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        const uint32_t r = find_halve(v, comp);
        if (ld_comp(comp, v) != r) comp[v] = r;
    }
}

__global__ void k_cc_sample(uint32_t V, uint32_t* comp, uint32_t* out, uint32_t n, uint64_t seed)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t v = (uint32_t)(mix64(seed ^ i) % V);
        out[i] = find_halve(v, comp);
    }
}

struct CcLinkOp {
    const uint32_t* __restrict__ off;
    const uint32_t* __restrict__ dst;
    uint32_t* comp;
    uint32_t giant;
    uint32_t skip;  // neighbours already linked by the sampling rounds
    DevCounters* ctr;

    __device__ __forceinline__ bool load(uint32_t v, uint32_t& s, uint32_t& d, uint32_t& m) const
    {
        s = off[v];
        d = off[v + 1] - s;
        m = v;
        if (d <= skip || find_halve(v, comp) == giant) return false;
        s += skip;
        d -= skip;
        return true;
    }
    __device__ __forceinline__ void edge(bool valid, uint32_t e, uint32_t v) const
    {
        if (valid) link(v, dst[e], comp, ctr);
    }
    __device__ __forceinline__ void block_begin() const {}
    __device__ __forceinline__ void block_end() const {}
};

struct CcPropOp {
    const uint32_t* __restrict__ off;
    const uint32_t* __restrict__ dst;
    uint32_t* label;
    uint32_t* stamp;
    uint32_t it;
    uint32_t nz;
    uint32_t* qout;
    uint32_t* qlen;
    uint32_t cap;
    DevCounters* ctr;

    __device__ __forceinline__ bool load(uint32_t v, uint32_t& s, uint32_t& d, uint32_t& m) const
    {
        s = off[v];
        d = off[v + 1] - s;
        m = label[v];
        return true;
    }
    __device__ __forceinline__ void edge(bool valid, uint32_t e, uint32_t m) const
    {
        bool enq = false;
        uint32_t d = 0;
        if (valid) {
            d = __ldcs(dst + e);  // streamed once: evict first
            if (m < label[d]) {
                const uint32_t old = atomicMin(label + d, m);
                if (m < old && d < nz) enq = atomicExch(stamp + d, it) != it;
            }
        }
        warp_append(enq, d, qout, qlen, cap, &ctr->overflow);
    }
    __device__ __forceinline__ void block_begin() const {}
    __device__ __forceinline__ void block_end() const {}
};

__global__ void k_zero(uint32_t n, uint32_t* a)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = 0;
}

static void cc_afforest(cgb_graph* g)
{
    const bool timing = g->flags & CGB_FLAG_KERNEL_TIMING;
    const uint32_t V = g->V;
    const uint32_t grid = div_up(V, kBlock);  // one vertex per thread: many CAS chains in flight
    constexpr uint32_t kRounds = 2;
    constexpr uint32_t kSamples = 1024;

    if (timing) ktimer_begin(g, CGB_K_INIT);
    ++g->stats.launches;
    k_cc_init_min_nbr<<<grid, kBlock, 0, g->stream>>>(V, g->off, g->dst, g->value);
    CGB_CUDA_TRY(cudaMemsetAsync(g->ctr, 0, sizeof(DevCounters), g->stream));
    if (timing) ktimer_end(g);
    // no compress here: the link round's finds halve the init forest's paths
    for (uint32_t r = 1; r < kRounds; r++) {
        if (timing) ktimer_begin(g, CGB_K_HOOK);
        ++g->stats.launches;
        k_cc_link_round<<<grid, kBlock, 0, g->stream>>>(V, g->off, g->dst, g->value, r, r == 1, g->ctr);
        if (timing) ktimer_end(g);
    }
    // no compress here either: sampling and the final link find roots themselves
    if (timing) ktimer_begin(g, CGB_K_OTHER);
    ++g->stats.launches;
    k_cc_sample<<<4, kBlock, 0, g->stream>>>(V, g->value, g->sample, kSamples, 0xAFF0E57ull);
    if (timing) ktimer_end(g);
    std::vector<uint32_t> h(kSamples);
    CGB_CUDA_TRY(cudaMemcpyAsync(h.data(), g->sample, kSamples * sizeof(uint32_t), cudaMemcpyDeviceToHost, g->stream));
    CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    std::sort(h.begin(), h.end());
    uint32_t giant = h[0], best = 0;
    for (uint32_t i = 0; i < kSamples;) {
        uint32_t j = i;
        while (j < kSamples && h[j] == h[i]) j++;
        if (j - i > best) {
            best = j - i;
            giant = h[i];
        }
        i = j;
    }
    CGB_CUDA_TRY(cudaMemsetAsync(&g->ctr->chunk_len, 0, sizeof(uint32_t), g->stream));
    if (timing) ktimer_begin(g, CGB_K_HOOK);
    CcLinkOp op{g->off, g->dst, g->value, giant, kRounds, g->ctr};
    launch_push(g, nullptr, V, op, true);
    if (timing) ktimer_end(g);
    if (timing) ktimer_begin(g, CGB_K_COMPRESS);
    ++g->stats.launches;
    k_cc_compress<<<grid, kBlock, 0, g->stream>>>(V, g->value);
    if (timing) ktimer_end(g);
    sync_counters(g);
    CGB_REQUIRE(!g->h_ctr->link_giveup, CGB_ETIMEOUT, "CC link retry bound exceeded");
    g->stats.iterations = kRounds + 1;
    g->stats.cc_path = 0;
}

static void cc_propagate(cgb_graph* g, const cgb_options& o)
{
    const bool timing = g->flags & CGB_FLAG_KERNEL_TIMING;
    const uint32_t V = g->V;
    const uint32_t grid = grid_for(V, kBlock, kNumSMs * 8);
    const uint64_t max_iters = o.max_iterations ? o.max_iterations : (uint64_t)V + 2;
    if (timing) ktimer_begin(g, CGB_K_INIT);
    ++g->stats.launches;
    k_cc_init<<<grid, kBlock, 0, g->stream>>>(V, g->value);
    ++g->stats.launches;
    k_zero<<<grid, kBlock, 0, g->stream>>>(V, g->stamp);
    CGB_CUDA_TRY(cudaMemsetAsync(g->ctr, 0, sizeof(DevCounters), g->stream));
    if (timing) ktimer_end(g);
    uint64_t n = V;
    int cur = 0;
    uint32_t it = 0;
    bool identity = true;
    uint64_t iters = 0;
    while (n > 0) {
        CGB_REQUIRE(iters < max_iters, CGB_ETIMEOUT, "CC iteration budget exhausted");
        it++;
        const int out = cur ^ 1;
        CGB_CUDA_TRY(cudaMemsetAsync(&g->ctr->qlen[out], 0, sizeof(uint32_t), g->stream));
        CGB_CUDA_TRY(cudaMemsetAsync(&g->ctr->chunk_len, 0, sizeof(uint32_t), g->stream));
        if (timing) ktimer_begin(g, CGB_K_PUSH);
        CcPropOp op{g->off, g->dst, g->value, g->stamp, it, g->nz, g->q[out], &g->ctr->qlen[out], V, g->ctr};
        launch_push(g, identity ? nullptr : g->q[cur], (uint32_t)n, op, identity);
        if (timing) ktimer_end(g);
        sync_counters(g);
        CGB_REQUIRE(!g->h_ctr->overflow, CGB_EOVERFLOW, "CC queue overflow");
        n = g->h_ctr->qlen[out];
        cur = out;
        identity = false;
        iters++;
    }
    g->stats.iterations = iters;
    g->stats.cc_path = 1;
}

void run_cc(cgb_graph* g, const cgb_options& o)
{
    ensure_frontier(g);
    ensure_symmetry_known(g);
    CGB_CUDA_TRY(cudaEventRecord(g->ev_start, g->stream));
    if (g->symmetric == 1) cc_afforest(g);
    else cc_propagate(g, o);
    CGB_CUDA_TRY(cudaEventRecord(g->ev_stop, g->stream));
}

}  // namespace cgb
