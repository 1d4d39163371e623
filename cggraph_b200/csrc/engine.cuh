// Internal state of a resident graph and the per-algorithm drivers.
#pragma once

#include <algorithm>
#include <atomic>
#include <mutex>
#include <vector>

#include "common.cuh"

// Device counters shared by the frontier kernels of one graph.
struct DevCounters {
    uint32_t qlen[2];         // lengths of the two alternating vertex queues
    uint32_t huge_len;        // vertices deferred to the split-hub kernel (allocation-free BFS)
    uint32_t far_len[2];      // SSSP: vertices pending in the far bitmap (index 0)
    uint32_t overflow;        // a queue ran out of capacity
    uint32_t link_giveup;     // a CC link loop hit its retry bound
    uint32_t found;           // BFS bottom-up: vertices found this level
    unsigned long long medges;    // sum of out-degrees of the next frontier
    unsigned long long reached_edges;
    uint32_t reached;
    uint32_t touched;         // SSSP: vertices whose distance left infinity this run (root excluded)
    uint32_t min_far;         // SSSP: smallest distance left in the far bitmap
    uint32_t max_deg;         // max degree of the next frontier
    uint32_t chunk_len;       // chunk descriptors queued by k_push_binned
    unsigned long long alive; // multi-root BFS: roots with vertices in the next frontier
    float policy_out[CGB_POLICY_OUTPUTS];  // learned scheduler: predicted log-costs
};

// Destination of counterfactual training samples (cgb_policy_collect).
struct PolicySamples {
    float* features;   // max * CGB_POLICY_FEATURES
    float* targets;    // max * CGB_POLICY_OUTPUTS
    uint8_t* mask;     // max * CGB_POLICY_OUTPUTS
    uint32_t max;
    uint32_t count;
    // state snapshots for the trials
    uint32_t* save_value = nullptr;
    uint32_t* save_bm0 = nullptr;
    uint32_t* save_bm1 = nullptr;
    uint32_t* save_q = nullptr;
    DevCounters* save_ctr = nullptr;
};

namespace cgb {
struct MsBuffers;
struct MsspBuffers;
}

// A graph's lock.  Taking it also swaps in weights that
// cgb_graph_set_weights uploaded while the graph was busy, so they take
// effect at the next entry point that uses the graph.
struct GraphMutex {
    std::mutex m;
    struct cgb_graph* owner = nullptr;
    void lock();
    bool try_lock();
    void unlock() { m.unlock(); }
};

// Launch parameters a graph starts with (cgb_tuning in the C ABI).
inline cgb_tuning default_tuning()
{
    cgb_tuning t{};
    t.struct_size = sizeof(cgb_tuning);
    t.push_big_deg = 512;
    t.push_chunk = 1024;
    t.push_ctas_per_sm = 8;
    t.persist_enter = 1u << 15;
    t.persist_deg = 2048;
    t.ms_edges = 256;
    t.pr_unroll = 16;
    t.pr_ctas_per_sm = 128;
    t.sssp_pull_alpha = 0;
    t.cluster_enter = 8192;
    t.sssp_dense_alpha = 4;
    t.push_block = 256;
    return t;
}

// Ranges accepted by cgb_tuning_set; buffer capacities are sized for the
// smallest chunk / descriptor sizes allowed here.
constexpr uint32_t kMinBigDeg = 128, kMinChunk = 256, kMinMsEdges = 64;

struct cgb_graph {
    int device = 0;
    uint32_t V = 0, E = 0, nz = 0;  // nz = noZeroOutDegreeNum
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    GraphMutex mu;
    // weights uploaded by cgb_graph_set_weights while the graph was busy
    std::mutex pending_mu;
    uint32_t* pending_w = nullptr;
    uint64_t pending_sum_w = 0;

    // CSR (always resident)
    uint32_t* off = nullptr;
    uint32_t* dst = nullptr;
    uint32_t* w = nullptr;  // may be null: unit weights
    uint64_t sum_w = 0;     // sum of weights (delta heuristic)
    uint32_t max_degree = 0;  // longest neighbour list (ensure_frontier)
    cgb_tuning tune_alg[4] = {default_tuning(), default_tuning(), default_tuning(), default_tuning()};
    cgb_tuning tune = default_tuning();  // active launch parameters: tune_alg of the running algorithm

    // in-edge CSC (built on first need; aliases the CSR when symmetric)
    uint32_t* in_off = nullptr;
    uint32_t* in_src = nullptr;
    bool csc_owned = false;
    uint32_t* in_w = nullptr;  // weights in CSC order (SSSP pull rounds); may alias w
    bool in_w_owned = false;
    bool lists_resorted = false;
    void* h_persist = nullptr;  // pinned host copy of the device-resident loop state
    size_t h_persist_bytes = 0;  // create sorted the neighbour lists (weights follow that order)
    int symmetric = -1;

    // PageRank layout: vertices relabelled by out-degree bucket (stable; zero
    // out-degree last), in-edge CSC over the new ids, out-degree by new id
    uint32_t* pr_rank = nullptr;     // old id -> new id
    uint32_t* pr_off = nullptr;      // V+1
    uint32_t* pr_src = nullptr;      // E
    uint32_t* pr_outdeg = nullptr;   // V
    uint2* pr_chunks = nullptr;      // hub rows: (row, first edge) of each kPrChunk-edge chunk
    uint32_t* pr_chunk_base = nullptr;  // per hub row: index of its first chunk (n_pr_huge + 1)
    uint32_t* pr_huge_rows = nullptr;   // hub rows (new ids)
    double* pr_part = nullptr;       // per-chunk partial sums
    uint32_t n_pr_huge = 0, n_pr_chunks = 0;
    // sliced ELL (32 rows per slice) of the non-hub rows: edge j of row
    // 32*s + l at col[slice_ptr[s] + 32*j + l]; padding points at vertex V,
    // whose contribution is kept at 0
    uint64_t* pr_slice_ptr = nullptr;   // nslices + 1
    uint32_t* pr_slice_len = nullptr;   // nslices
    uint32_t* pr_col = nullptr;
    uint32_t* pr_hub_bm = nullptr;      // bitmap of hub rows
    uint64_t pr_sell_size = 0;
    bool pr_ready = false;

    // results / algorithm state
    uint32_t* value = nullptr;  // uint32[V]
    double* pr[2] = {nullptr, nullptr};
    double* contrib[2] = {nullptr, nullptr};
    const void* result = nullptr;
    int result_alg = -1;

    // frontier workspace
    uint32_t* q[2] = {nullptr, nullptr};  // capacity V each
    uint2* chunk_q = nullptr;             // (vertex, chunk) descriptors of big lists
    uint32_t chunk_cap = 0;
    uint32_t* visited = nullptr;          // bitmap, words = V/32 + 1
    uint32_t* front_bm = nullptr;
    uint32_t* stamp = nullptr;            // uint32[V]
    uint32_t* sample = nullptr;           // CC sampling buffer
    uint32_t* aux_bm = nullptr;           // 3 bitmaps: device-resident SSSP near dedup
    void* persist = nullptr;              // state of the device-resident loops
    cgb::MsBuffers* ms = nullptr;         // multi-root BFS masks
    cgb::MsspBuffers* mssp = nullptr;     // multi-root SSSP distances and masks

    DevCounters* ctr = nullptr;       // device
    DevCounters* h_ctr = nullptr;     // pinned host mirror

    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    cudaEvent_t ev_iter[2] = {nullptr, nullptr};
    // PageRank hub chunks run beside the sliced pull: a second stream forked
    // from and joined to `stream` by these events (created on first use)
    cudaStream_t aux_stream = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    std::vector<cudaEvent_t> kev;     // per-launch timing events (pairs)
    size_t kev_used = 0;
    std::vector<int> kev_class;

    cgb_run_stats stats{};
    std::vector<cgb_iter_trace> trace;
    PolicySamples* collect = nullptr;   // set while cgb_policy_collect runs
    uint32_t flags = 0;

    // request servers attached (cgb_server_create): their SSSP groups and
    // second engine context read w without the graph's lock, so the weights
    // cannot be replaced meanwhile
    std::atomic<int> servers{0};

    uint32_t words() const { return V / 32 + 1; }
    cgb_graph() { mu.owner = this; }
};

namespace cgb {

constexpr uint32_t kPrHuge = 4096;   // PageRank rows split into chunks across CTAs
constexpr uint32_t kPrChunk = 4096;  // edges per PageRank hub chunk
constexpr uint32_t kHugeDeg = 16384; // push: hubs split across CTAs
constexpr uint32_t kCtaDeg = 1024;   // push: CTA-per-vertex tier
constexpr uint32_t kHugeChunk = 4096;

// graph lifetime and preparation (graph.cu)
cgb_graph* graph_alloc(uint32_t V, uint32_t E, uint32_t nz, int device, bool with_weight);
void graph_free(cgb_graph* g);
// Attaches or replaces the edge weights (cgb_graph_set_weights).
void graph_set_weights(cgb_graph* g, const uint32_t* weight);
void validate_and_sort(cgb_graph* g);
void compute_weight_sum(cgb_graph* g);
uint32_t sssp_default_delta(const cgb_graph* g);           // single-root runs
void ensure_max_degree(cgb_graph* g);                      // g->max_degree, computed once
// A second single-root engine context over g's CSR (borrowed, not copied):
// own stream, counters, distances and frontier scratch.  Freed with
// graph_shadow_free, which leaves g's arrays alone.
cgb_graph* graph_shadow(cgb_graph* g);
void graph_shadow_free(cgb_graph* sh);
uint32_t sssp_delta_for(const cgb_graph* g, double c);     // c x mean weight / mean out-degree

// workspace management (graph.cu)
void ensure_frontier(cgb_graph* g);
void ensure_csc(cgb_graph* g);
void ensure_symmetry_known(cgb_graph* g);
void ensure_pr(cgb_graph* g);
void sync_counters(cgb_graph* g);

// timing helpers (graph.cu)
void ktimer_begin(cgb_graph* g, int cls);
void ktimer_end(cgb_graph* g);
void ktimer_collect(cgb_graph* g);

// drivers
void run_bfs(cgb_graph* g, uint32_t root, const cgb_options& o);
void run_sssp(cgb_graph* g, uint32_t root, const cgb_options& o);
void run_cc(cgb_graph* g, const cgb_options& o);
void run_pr(cgb_graph* g, uint32_t iters, const cgb_options& o);
void count_reached(cgb_graph* g);  // fills stats.reached / traversed_edges for BFS/SSSP
// Multi-root BFS of n <= 64 roots; a level pulls (bottom-up) when the
// frontier's out-edges times alpha exceed the graph's edges.
void run_msbfs(cgb_graph* g, const uint32_t* d_roots, uint32_t n, uint32_t* level_out, double alpha);
constexpr double kMsAlpha = 15.0;  // default alpha of multi-root passes
void free_msbfs(cgb_graph* g);
// Multi-root SSSP of n <= 64 roots (device array); out (device) receives
// n * V distances, root-major.
void run_mssp(cgb_graph* g, const uint32_t* d_roots, uint32_t n, uint32_t* out, uint32_t delta);
void free_mssp(cgb_graph* g);
// Pinned host blocks of at most 256 bytes from process-lifetime slabs.
// Device memory from the engine's pool, allocated in the order of stream s
// (and complete on return); released with the graph (graph_free).
void* pool_alloc(size_t bytes, cudaStream_t s);
// Releases pool memory in the order of stream s.
void pool_free(void* p, cudaStream_t s);
// A graph from an edge list of packed (source, destination, weight) u32
// records in host or device memory (cgb_graph_create_from_edges).
cgb_graph* graph_from_edges(const uint32_t* records, uint64_t E, uint32_t V, int device);
// Relabelled copy of g in one of the reference's vertex orders (cgb_graph_reorder).
cgb_graph* graph_reorder(cgb_graph* g, int method, uint32_t* old2new_out, uint32_t* nz_out);
// The reference's two-level segment partition over GPUs (cgb_graph_partition).
void graph_partition(cgb_graph* g, int algorithm, uint32_t ndev, const uint64_t* mem_bytes, uint32_t* seg_order,
                     uint32_t* seg_edges, int32_t* seg_owner, uint32_t* device_segments, cgb_partition_info* info);
void* pinned_small_alloc(size_t bytes);
// Pinned host memory for small transfers, from a process-wide pool.
void* pinned_acquire(size_t bytes);
void pinned_release(void* p, size_t bytes);
// A small transfer from pinned host memory by a kernel (no copy engine).
void h2d_small(void* dst, const void* pinned_src, size_t bytes, cudaStream_t s);

// n values of T in pinned host memory for the scope of a transfer (the
// stream must be synchronised before the block goes out of scope).
template <typename T>
struct PinnedArray {
    T* p;
    size_t n;
    explicit PinnedArray(size_t count) : p(static_cast<T*>(pinned_acquire(count * sizeof(T)))), n(count) {}
    ~PinnedArray() { pinned_release(p, n * sizeof(T)); }
    PinnedArray(const PinnedArray&) = delete;
    PinnedArray& operator=(const PinnedArray&) = delete;
    T& operator[](size_t i) { return p[i]; }
    T* data() { return p; }
};
void pinned_small_free(void* p);
// Weights in CSC order (in_w); needs the graph's weights.
void ensure_csc_weights(cgb_graph* g);
// One pull round of SSSP over the near set q_in[0, nin) at bucket [lo, thr):
// next near set to qout, new far vertices to far_bm; near_set is a scratch
// bitmap (words()).  q_in is scratch afterwards.
void sssp_pull_round(cgb_graph* g, const uint32_t* q_in, uint32_t nin, uint32_t lo, uint32_t thr, uint32_t* qout,
                     uint32_t* qout_len, uint32_t* far_bm, uint32_t* near_set);
uint32_t mssp_default_delta(cgb_graph* g);

}  // namespace cgb
