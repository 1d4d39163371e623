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
//
// Weak components (CGB_FLAG_CC_WEAK): the same hooking over the edges taken
// as undirected, read from both the CSR (out-lists) and the CSC (in-lists),
// both sorted.  The labels equal the reference's CC run on the symmetrised
// graph, without a symmetrised copy of the graph: step 1 points v at the
// smallest of its first out- and in-neighbour, step 2 links v with the first
// two of each list, step 4 links the remaining out- and in-edges of every
// vertex outside the giant component.  An edge u -> v is skipped only when
// both u (its out-list) and v (its in-list) were found in the giant
// component, and then it joins nothing new.
#include "engine.cuh"
#include "push.cuh"

namespace cgb {

constexpr uint32_t kLinkRetries = 1u << 20;
constexpr int kCompressVerts = 4;  // vertices per thread in the compress pass

// Two kinds of access to the forest.  Strong accesses (volatile: no L1,
// always the current value at L2) and weak ones (plain: may be served from
// this SM's L1, so possibly stale).  Nearly every path ends at the giant
// component's root, and strong loads of that one word all queue at one L2
// slice; weak loads hit L1 instead.  A stale value is still a vertex that
// was an ancestor once, and pointers only ever move to smaller ancestors,
// so a weak walk ends at an ancestor of its start: two walks that meet are
// in one tree, and a vertex it took for a root but is not fails the hooking
// CAS (which is at L2), after which the roots are found again with strong
// loads.
template <bool kStrong>
__device__ __forceinline__ uint32_t ld_comp(const uint32_t* comp, uint32_t i)
{
    if constexpr (kStrong) return *((volatile const uint32_t*)comp + i);
    else return comp[i];
}

template <bool kStrong>
__device__ __forceinline__ void st_comp(uint32_t* comp, uint32_t i, uint32_t v)
{
    if constexpr (kStrong) *((volatile uint32_t*)comp + i) = v;
    else comp[i] = v;
}

// Roots of x[0..N-1] with path halving: each visited vertex is pointed at
// its grandparent on the way up.  Concurrent halving is benign: a vertex
// only ever moves to one of its own ancestors, so every pointer still goes
// to a smaller vertex of the same tree.  All N paths are walked in one loop
// (the N loads of a step are independent).
template <bool kStrong, int N>
__device__ __forceinline__ void find_roots(uint32_t (&x)[N], uint32_t* comp)
{
    uint32_t p[N];
#pragma unroll
    for (int i = 0; i < N; i++) p[i] = ld_comp<kStrong>(comp, x[i]);
    for (uint32_t steps = 0; steps < kLinkRetries; steps++) {
        bool more = false;
#pragma unroll
        for (int i = 0; i < N; i++) more |= p[i] != x[i];
        if (!more) return;
        uint32_t gp[N];
#pragma unroll
        for (int i = 0; i < N; i++) gp[i] = p[i] != x[i] ? ld_comp<kStrong>(comp, p[i]) : x[i];
#pragma unroll
        for (int i = 0; i < N; i++) {
            if (p[i] != x[i]) {
                if (gp[i] != p[i]) st_comp<kStrong>(comp, x[i], gp[i]);
                x[i] = gp[i];
                p[i] = ld_comp<kStrong>(comp, x[i]);
            }
        }
    }
}

template <bool kStrong>
__device__ __forceinline__ uint32_t find_halve(uint32_t x, uint32_t* comp)
{
    uint32_t r[1] = {x};
    find_roots<kStrong, 1>(r, comp);
    return r[0];
}

// Hooks the trees whose roots were a and b (found a moment ago, possibly by
// weak loads, so possibly no longer roots): the larger goes under the
// smaller one.  The CAS succeeds only on a current root; a failed CAS means
// another thread hooked `high` first (or the walk saw a stale root), and
// both roots are found again with strong loads.
__device__ __forceinline__ void hook_roots(uint32_t a, uint32_t b, uint32_t* comp, DevCounters* ctr)
{
    for (uint32_t tries = 0; a != b; tries++) {
        if (tries >= kLinkRetries) {
            atomicOr(&ctr->link_giveup, 1u);
            return;
        }
        const uint32_t high = max(a, b), low = min(a, b);
        if (atomicCAS(comp + high, high, low) == high) return;
        uint32_t r[2] = {high, low};
        find_roots<true, 2>(r, comp);
        a = r[0];
        b = r[1];
    }
}

// Hooks the trees of u and v, larger root under smaller root.
__device__ __forceinline__ void link(uint32_t u, uint32_t v, uint32_t* comp, DevCounters* ctr)
{
    uint32_t r[2] = {u, v};
    find_roots<false, 2>(r, comp);
    hook_roots(r[0], r[1], comp, ctr);
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

// Weak components: comp[v] = min(v, smallest out-neighbour, smallest
// in-neighbour).
__global__ void k_cc_init_min_nbr_weak(uint32_t V, const uint32_t* __restrict__ off,
                                       const uint32_t* __restrict__ dst, const uint32_t* __restrict__ in_off,
                                       const uint32_t* __restrict__ in_src, uint32_t* comp)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        const uint32_t s = off[v], is = in_off[v];
        uint32_t c = v;
        if (off[v + 1] > s) c = min(c, dst[s]);
        if (in_off[v + 1] > is) c = min(c, in_src[is]);
        comp[v] = c;
    }
}

// Weak components: links v with the first two entries of its out- and
// in-list, except the one k_cc_init_min_nbr_weak already pointed it at.
__global__ void k_cc_link_round_weak(uint32_t V, const uint32_t* __restrict__ off, const uint32_t* __restrict__ dst,
                                     const uint32_t* __restrict__ in_off, const uint32_t* __restrict__ in_src,
                                     uint32_t* comp, DevCounters* ctr)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        const uint32_t s = off[v], d = off[v + 1] - s;
        const uint32_t is = in_off[v], id = in_off[v + 1] - is;
        const uint32_t o0 = d > 0 ? dst[s] : v, i0 = id > 0 ? in_src[is] : v;
        const uint32_t init = min(v, min(o0, i0));
        if (o0 != init) link(v, o0, comp, ctr);
        if (i0 != init && i0 != o0) link(v, i0, comp, ctr);
        if (d > 1) link(v, dst[s + 1], comp, ctr);
        if (id > 1) link(v, in_src[is + 1], comp, ctr);
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
// the chains that other threads are still walking).  Each thread walks the
// paths of kN vertices, kN x (grid threads) apart, in one loop.  No hooking
// runs during this pass, so the set of roots is fixed and weak loads are
// exact about which vertex is a root (L1 holds nothing from before the
// launch).
template <int kN>
__global__ void k_cc_compress(uint32_t V, uint32_t* comp)
{
    const uint64_t T = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v0 < V; v0 += kN * T) {
        uint32_t x[kN];
#pragma unroll
        for (int i = 0; i < kN; i++) x[i] = (uint32_t)(v0 + i * T < V ? v0 + i * T : v0);
        find_roots<false, kN>(x, comp);
#pragma unroll
        for (int i = 0; i < kN; i++) {
            const uint64_t v = v0 + i * T;
            if (v < V && ld_comp<false>(comp, (uint32_t)v) != x[i]) comp[v] = x[i];
        }
    }
}

__global__ void k_cc_sample(uint32_t V, uint32_t* comp, uint32_t* out, uint32_t n, uint64_t seed)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t v = (uint32_t)(mix64(seed ^ i) % V);
        out[i] = find_halve<true>(v, comp);
    }
}

// Steps from n sampled vertices towards their roots in the init forest,
// each walk cut at max_steps (read only).
__global__ void k_cc_depth(uint32_t V, const uint32_t* __restrict__ comp, uint32_t n, uint64_t seed,
                           uint32_t max_steps, unsigned long long* steps)
{
    unsigned long long t = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t v = (uint32_t)(mix64(seed ^ i) % V);
        for (uint32_t k = 0; k < max_steps; k++) {
            const uint32_t p = comp[v];
            if (p == v) break;
            v = p;
            t++;
        }
    }
    t = warp_sum(t);
    if (lane_id() == 0 && t) atomicAdd(steps, t);
}

// One pointer-jumping pass, comp[v] = comp[comp[v]] (an ancestor replaces
// the parent, so a concurrent update only shortens a walk); raises *changed
// when some pointer moved.
__global__ void k_cc_jump(uint32_t V, uint32_t* comp, uint32_t* changed)
{
    bool ch = false;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        const uint32_t p = comp[v];
        const uint32_t pp = comp[p];
        if (pp != p) {
            comp[v] = pp;
            ch = true;
        }
    }
    if (__any_sync(0xffffffffu, ch) && lane_id() == 0) *changed = 1u;
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
        if (d <= skip || find_halve<false>(v, comp) == giant) return false;
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

// Afforest over the out-lists (symmetric graphs), or over the out- and
// in-lists (weak components of any graph).
static void cc_afforest(cgb_graph* g, bool weak)
{
    const bool timing = g->flags & CGB_FLAG_KERNEL_TIMING;
    const uint32_t V = g->V;
    const uint32_t grid = div_up(V, kBlock);  // one vertex per thread: many CAS chains in flight
    constexpr uint32_t kRounds = 2;
    constexpr uint32_t kSamples = 1024;

    if (timing) ktimer_begin(g, CGB_K_INIT);
    ++g->stats.launches;
    if (weak)
        k_cc_init_min_nbr_weak<<<grid, kBlock, 0, g->stream>>>(V, g->off, g->dst, g->in_off, g->in_src, g->value);
    else
        k_cc_init_min_nbr<<<grid, kBlock, 0, g->stream>>>(V, g->off, g->dst, g->value);
    CGB_CUDA_TRY(cudaMemsetAsync(g->ctr, 0, sizeof(DevCounters), g->stream));
    if (timing) ktimer_end(g);
    // The init forest is shallow on skewed graphs, and the link round's finds
    // halve its paths.  On meshes it is deep: on a grid numbered row by row,
    // each vertex's smallest neighbour is the one above it, so the trees are
    // whole columns (4800 levels on the 4800 x 5000 grid) and every find of
    // the link rounds walks one.  A probe measures the mean depth of 1024
    // sampled vertices; above kDeepForest the forest is flattened by
    // pointer jumping first (each pass halves every path).  The probe's
    // walks stop after 4 x kDeepForest steps.  Graphs with a vertex of
    // kProbeMaxDeg or more out-edges skip the probe (and its host
    // synchronisation): their hubs give shallow init forests.
    constexpr uint32_t kProbeMaxDeg = 64;
    if (g->max_degree < kProbeMaxDeg) {
        constexpr uint32_t kProbe = 1024;
        constexpr double kDeepForest = 8.0;
        if (timing) ktimer_begin(g, CGB_K_COMPRESS);
        ++g->stats.launches;
        k_cc_depth<<<4, kBlock, 0, g->stream>>>(V, g->value, kProbe, 0xDE9741ull, (uint32_t)(4 * kDeepForest),
                                                &g->ctr->reached_edges);
        sync_counters(g);
        if ((double)g->h_ctr->reached_edges / kProbe > kDeepForest) {
            // four passes per read-back; only the last pass of each group raises
            // the flag, so a clear flag means that pass moved nothing
            const uint32_t jgrid = grid_for(V, kBlock, num_sms() * 8);
            for (uint32_t group = 0;; group++) {
                CGB_REQUIRE(group < 12, CGB_ETIMEOUT, "CC pointer jumping did not converge");
                for (int k = 0; k < 4; k++) {
                    if (k == 3) CGB_CUDA_TRY(cudaMemsetAsync(&g->ctr->found, 0, sizeof(uint32_t), g->stream));
                    ++g->stats.launches;
                    k_cc_jump<<<jgrid, kBlock, 0, g->stream>>>(V, g->value, &g->ctr->found);
                }
                sync_counters(g);
                if (!g->h_ctr->found) break;
            }
        }
        CGB_CUDA_TRY(cudaMemsetAsync(g->ctr, 0, sizeof(DevCounters), g->stream));
        if (timing) ktimer_end(g);
    }
    for (uint32_t r = 1; r < kRounds; r++) {
        if (timing) ktimer_begin(g, CGB_K_HOOK);
        ++g->stats.launches;
        if (weak)
            k_cc_link_round_weak<<<grid, kBlock, 0, g->stream>>>(V, g->off, g->dst, g->in_off, g->in_src, g->value,
                                                                 g->ctr);
        else
            k_cc_link_round<<<grid, kBlock, 0, g->stream>>>(V, g->off, g->dst, g->value, r, r == 1, g->ctr);
        if (timing) ktimer_end(g);
    }
    // no compress here either: sampling and the final link find roots themselves
    if (timing) ktimer_begin(g, CGB_K_OTHER);
    ++g->stats.launches;
    k_cc_sample<<<4, kBlock, 0, g->stream>>>(V, g->value, g->sample, kSamples, 0xAFF0E57ull);
    if (timing) ktimer_end(g);
    PinnedArray<uint32_t> h(kSamples);  // pinned: a pageable copy would wait on other threads' copies
    CGB_CUDA_TRY(cudaMemcpyAsync(h.data(), g->sample, kSamples * sizeof(uint32_t), cudaMemcpyDeviceToHost, g->stream));
    CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    std::sort(h.data(), h.data() + kSamples);
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
    if (weak) {
        CGB_CUDA_TRY(cudaMemsetAsync(&g->ctr->chunk_len, 0, sizeof(uint32_t), g->stream));
        CcLinkOp iop{g->in_off, g->in_src, g->value, giant, kRounds, g->ctr};
        launch_push(g, nullptr, V, iop, true);
    }
    if (timing) ktimer_end(g);
    if (timing) ktimer_begin(g, CGB_K_COMPRESS);
    ++g->stats.launches;
    k_cc_compress<kCompressVerts><<<div_up(V, kBlock * kCompressVerts), kBlock, 0, g->stream>>>(V, g->value);
    if (timing) ktimer_end(g);
    sync_counters(g);
    CGB_REQUIRE(!g->h_ctr->link_giveup, CGB_ETIMEOUT, "CC link retry bound exceeded");
    g->stats.iterations = kRounds + 1;
    g->stats.cc_path = weak ? 2 : 0;
}

static void cc_propagate(cgb_graph* g, const cgb_options& o)
{
    const bool timing = g->flags & CGB_FLAG_KERNEL_TIMING;
    const uint32_t V = g->V;
    const uint32_t grid = grid_for(V, kBlock, num_sms() * 8);
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
    const bool weak = o.flags & CGB_FLAG_CC_WEAK;
    // weak components read the in-lists (the CSR itself when the graph is
    // known to be symmetric); no symmetry check is needed for them
    if (weak) ensure_csc(g);
    else ensure_symmetry_known(g);
    CGB_CUDA_TRY(cudaEventRecord(g->ev_start, g->stream));
    if (weak) cc_afforest(g, g->in_off != g->off);
    else if (g->symmetric == 1) cc_afforest(g, false);
    else cc_propagate(g, o);
    CGB_CUDA_TRY(cudaEventRecord(g->ev_stop, g->stream));
}

}  // namespace cgb
