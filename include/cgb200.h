/*
 * cgb200 -- a B200 (sm_100a) graph engine for BFS, SSSP, CC and PageRank
 * behind the selection interface of CGgraph (PengBo410/CGgraph).
 *
 * Plain C ABI: no C++ or framework types cross it.  Every call returns a
 * cgb_status; cgb_last_error_string() describes the last failure on the
 * calling thread.  Host and device pointers are both accepted wherever a
 * buffer is passed (the copy direction is inferred from the pointer).
 *
 * Reference interfaces replaced (paths under CGgraph/ of the reference):
 *   - CSR_Result_type {vertexNum, edgeNum, csr_offset, csr_dest, csr_weight,
 *     noZeroOutDegreeNum}                    Basic/Graph/basic_struct.hpp:7-16
 *   - load_binFile<T>(path, length)          Basic/Other/IO.hpp:44-92
 *   - nbrSort_taskSteal(csr) (sort + strict-ascending check)
 *                                            my_project/CGgraph/sortNbr.hpp:8-99
 *   - GraphDeviceWorklist(csr, alg)          my_project/CGgraph/GraphDevice.cuh:48-71
 *   - GraphDeviceWorklist::graphProcess_device(alg, root) -> ms
 *                                            my_project/CGgraph/GraphDevice.cuh:92-176
 *   - GraphDeviceWorklist::result_D2H() / vertexValue
 *                                            my_project/CGgraph/GraphDevice.cuh:21,259-262
 *   - Algorithm_type {BFS, SSSP, CC, PR}     Basic/Graph/basic_struct.hpp:144-151
 *   - VertexValue_MAX = 999999999            Basic/Graph/basic_def.hpp:18
 */
#ifndef CGB200_H
#define CGB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CGB_VALUE_MAX 999999999u /* VertexValue_MAX, Basic/Graph/basic_def.hpp:18 */
#define CGB_ABI_VERSION 1

typedef enum cgb_status {
    CGB_OK = 0,
    CGB_EINVAL = 1,    /* bad argument (null pointer, root >= V, unknown algorithm) */
    CGB_EFORMAT = 2,   /* CSR violates the reference's invariants (offsets, ids, duplicates) */
    CGB_EIO = 3,       /* file missing or of the wrong size (load_binFile's checks) */
    CGB_ENOMEM = 4,    /* device or host allocation failed */
    CGB_ECUDA = 5,     /* CUDA runtime error (replaces CUDA_CHECK's exit(1)) */
    CGB_ETIMEOUT = 6,  /* a device-side wait or the iteration budget ran out */
    CGB_EOVERFLOW = 7, /* a work queue overflowed its capacity */
    CGB_EUNSUPPORTED = 8
} cgb_status;

/* Algorithm_type values, Basic/Graph/basic_struct.hpp:144-151. */
typedef enum cgb_algorithm { CGB_BFS = 0, CGB_SSSP = 1, CGB_CC = 2, CGB_PR = 3 } cgb_algorithm;

/* Per-iteration schedule choice.  Every schedule computes the same result. */
typedef enum cgb_schedule {
    CGB_SCHED_HEURISTIC = 0, /* Beamer direction switch, fixed SSSP delta */
    CGB_SCHED_LEARNED = 1,   /* MLP policy (cgb_policy_*), heuristic fallback */
    CGB_SCHED_FIXED = 2      /* the variant / direction given in cgb_options */
} cgb_schedule;

/* Push-expansion variants (cgb_options.variant for CGB_SCHED_FIXED). */
typedef enum cgb_variant {
    CGB_VAR_AUTO = 0,
    CGB_VAR_TWC = 1,      /* degree-binned thread / warp / CTA expansion */
    CGB_VAR_PULL = 2,     /* pull over the in-edges (BFS bottom-up; SSSP pull round) */
    CGB_VAR_PUSH = 3,     /* top-down push (BFS: forbid the pull direction) */
    CGB_VAR_DENSE = 4     /* SSSP round with a dense frontier: relax without enqueueing, then
                             find the improved vertices by one pass over all of them (trace only) */
} cgb_variant;

typedef struct cgb_options {
    uint32_t struct_size;   /* sizeof(cgb_options); 0 = all defaults */
    int32_t schedule;       /* cgb_schedule */
    int32_t variant;        /* cgb_variant, for CGB_SCHED_FIXED */
    uint32_t sssp_delta;    /* 0 = heuristic: 128 * mean weight / mean degree (64 x for multi-root passes) */
    double bfs_alpha;       /* Beamer alpha, 0 = 15 */
    double bfs_beta;        /* Beamer beta, 0 = 18 */
    uint64_t max_iterations;/* 0 = unlimited (V + 1 levels bound BFS anyway) */
    uint32_t flags;         /* CGB_FLAG_* */
    uint32_t reserved[7];
} cgb_options;

#define CGB_FLAG_KERNEL_TIMING 0x1u /* record per-kernel CUDA-event times (cgb_run_stats) */
#define CGB_FLAG_TRACE 0x2u         /* log one cgb_iter_trace per iteration */
#define CGB_FLAG_BATCH_SEQUENTIAL 0x4u /* cgb_run_batch: one cgb_run per root instead of multi-root passes */
#define CGB_FLAG_CC_WEAK 0x8u /* CC over the edges taken as undirected (weak components): labels equal the
                                 reference's CC on the symmetrised graph, with no symmetrised copy; on a
                                 directed graph without it CC is the reference's label propagation along
                                 out-edges */

typedef struct cgb_graph cgb_graph;

/* Per-run statistics of the last cgb_run on a graph. */
typedef struct cgb_run_stats {
    double ms;                /* device time of the run (CUDA events around it) */
    uint64_t iterations;      /* levels / relaxation rounds / PageRank iterations */
    uint64_t traversed_edges; /* TEPS numerator: BFS/SSSP sum of outdeg of reached vertices,
                                 CC edges of the graph, PR E * iterations */
    uint64_t reached;         /* vertices with a value != CGB_VALUE_MAX */
    uint64_t alg_bytes;       /* algorithmic HBM bytes of the run (lower bound) */
    double kernel_ms[8];      /* per kernel class, with CGB_FLAG_KERNEL_TIMING */
    uint64_t kernel_launches[8];
    uint64_t pushes_td, pulls_bu; /* BFS: levels run top-down / bottom-up */
    uint32_t sssp_delta;      /* delta used */
    int32_t cc_path;          /* 0 = hook+compress (symmetric), 1 = label propagation,
                                 2 = hook+compress over out- and in-lists (CGB_FLAG_CC_WEAK) */
    uint64_t launches;        /* kernels launched by the run */
} cgb_run_stats;

/* Kernel classes indexing kernel_ms / kernel_launches. */
#define CGB_K_PUSH 0   /* push expansion (BFS top-down, SSSP, CC label propagation) */
#define CGB_K_PULL 1   /* BFS bottom-up */
#define CGB_K_PR 2     /* PageRank pull iteration */
#define CGB_K_HOOK 3   /* CC hooking */
#define CGB_K_COMPRESS 4
#define CGB_K_FRONTIER 5 /* frontier conversion / bucket split */
#define CGB_K_INIT 6
#define CGB_K_OTHER 7

/* One entry per iteration when CGB_FLAG_TRACE is set (features the learned
 * scheduler is trained on). */
typedef struct cgb_iter_trace {
    uint32_t iteration;
    uint32_t algorithm;
    uint64_t frontier_vertices;
    uint64_t frontier_edges;
    uint64_t unvisited_vertices;
    uint64_t unvisited_edges;
    uint32_t max_frontier_degree;
    int32_t variant;       /* cgb_variant actually run */
    uint32_t delta;        /* SSSP delta in force */
    float ms;              /* measured device time of the iteration */
} cgb_iter_trace;

/* --------------------------------------------------------------- graph */

/* Copies a CSR (host or device pointers) into HBM and checks the invariants
 * the reference asserts: offsets[0] == 0, offsets non-decreasing,
 * offsets[V] == E, dest[e] < V; neighbour lists are sorted by dest on the
 * device (weights follow, as nbrSort_taskSteal does) and must then be
 * strictly ascending (no duplicate edges).  weight may be NULL (SSSP then
 * uses weight 1).  no_zero_out_degree_num = 0 means V; the vertices from it
 * on must have no out-edges, offsets[no_zero_out_degree_num] == E (the
 * driver's RCM_LAST_ZERO_OUTDEGREE_check, main_partition.hpp:88-101), else
 * CGB_EFORMAT.  V and E are at
 * most 2^32 - 2^24 (CGB_EUNSUPPORTED beyond; the reference's uint32 count types
 * end at 2^32 - 1).  The caller keeps ownership of its arrays.  Replaces GraphDeviceWorklist's constructor and
 * csrToDevice() (GraphDevice.cuh:48-71,208-221). */
cgb_status cgb_graph_create(const uint32_t* offsets, const uint32_t* dest, const uint32_t* weight,
                            uint32_t V, uint32_t E, uint32_t no_zero_out_degree_num, int device,
                            cgb_graph** out);

/* Loads the three raw little-endian arrays with load_binFile's size check
 * (file bytes == length * 4, Basic/Other/IO.hpp:50-52), then as
 * cgb_graph_create.  weight_path may be NULL. */
cgb_status cgb_graph_load_files(const char* offsets_path, const char* dest_path, const char* weight_path,
                                uint32_t V, uint32_t E, int device, cgb_graph** out);

/* Builds the graph from an edge list: num_edges packed records of three
 * uint32 {source, destination, weight} (host or device memory), in any
 * order. The CSR is built on the device: lists grouped by source and sorted
 * by destination, weights following. CGB_EFORMAT for a self-loop, an id >= V
 * or a duplicate edge, as the reference's reader asserts. Replaces
 * GraphBinReader::group_load_directedGraph + sort_nbr + getStruct_csrResult
 * (Basic/Graph/graphBinReader.hpp:89-208,213-227,286-322). */
cgb_status cgb_graph_create_from_edges(const uint32_t* records, uint64_t num_edges, uint32_t V, int device,
                                       cgb_graph** out);

/* The same from a binary edge-list file (the reference's has_csrFile = 0
 * input, main_partition.hpp:105-116): the edge count is the file size / 12,
 * rounded down; trailing bytes short of a record are ignored, as the
 * reference's reader ignores them. */
cgb_status cgb_graph_load_edge_file(const char* path, uint32_t V, int device, cgb_graph** out);

/* OrderMethod values (Basic/Graph/basic_struct.hpp:41-76) that cgb_graph_reorder builds. */
#define CGB_ORDER_NATIVE 0
#define CGB_ORDER_NORMAL_OUTDEGREE_DEC 12
#define CGB_ORDER_MY_BFS_OUT 16
#define CGB_ORDER_MY_BFS_IN 17
#define CGB_ORDER_MY_BFS_OUT_IN 18
#define CGB_ORDER_MY_IMAX_BFS_IN 20
#define CGB_ORDER_IN_DEGREE_DEC 21

/* A relabelled copy of g (on g's device): vertices sorted by degree,
 * largest first, ties by ascending id, as the reference's Reorder sorts them
 * (my_project/CGgraph/Reorder.hpp:251-292). CGB_ORDER_IN_DEGREE_DEC sorts by
 * in-degree (Reorder.hpp:211-240); CGB_ORDER_NORMAL_OUTDEGREE_DEC by
 * out-degree, so the vertices without out-edges come last and the new
 * graph's noZeroOutDegreeNum is their start. old2new (V entries, host or
 * device memory, may be NULL) receives the new id of every vertex, for
 * rootTranfer and checkBinResult; *no_zero_out_degree_num (may be NULL) the
 * new graph's noZeroOutDegreeNum.
 * The BFS orders (Reorder.hpp:294-535) list the vertices with out-edges in
 * the order of queue BFSs started from them by degree, largest first
 * (out-degree; in-degree for CGB_ORDER_MY_IMAX_BFS_IN), each vertex queueing
 * its unvisited neighbours by degree, largest first (out-degree for
 * MY_BFS_OUT, in-degree for MY_BFS_IN and MY_IMAX_BFS_IN, their sum for
 * MY_BFS_OUT_IN; equal degrees in list order), followed by the vertices
 * without out-edges in the order the BFSs meet them; noZeroOutDegreeNum is
 * their start. Other order methods (RCM, GORDER, MY_IMAX_BFS_OUT, which the
 * reference leaves undefined) are CGB_EUNSUPPORTED. The relabelled lists are
 * sorted by new id, as the reference's driver sorts them after loading
 * (main_partition.hpp:146). */
cgb_status cgb_graph_reorder(cgb_graph* g, int order_method, uint32_t* old2new,
                             uint32_t* no_zero_out_degree_num, cgb_graph** out);

/* The reference's two-level partition of a graph over GPUs
 * (my_project/CGgraph/Two-level_partition.cuh:213-444), the plan its
 * CPU+GPU co-execution engine runs on. The vertices with out-edges,
 * [0, noZeroOutDegreeNum), are cut into segments of CGB_SEGMENT_SIZE
 * vertices; segments are sorted by average degree (edges / vertices, an
 * integer quotient; ties by segment id) and cut into four buckets (degree up
 * to 16, up to 32, up to 256, above); then dealt to num_devices GPUs bucket
 * by bucket, segment j of a bucket to GPU (j + j / num_devices) %
 * num_devices, each GPU taking 4 bytes per edge (8 for CGB_SSSP) out of its
 * memory less 4 V + 4 (noZeroOutDegreeNum + 1) bytes and a 1 GiB reserve,
 * until a GPU would reach zero; that segment and all after it stay with the
 * host (owner -1). device_mem_bytes (num_devices entries) may be NULL: the
 * total memory of devices 0 .. num_devices - 1. Output arrays may be NULL:
 * seg_order (segment_num entries) the segment ids in sorted order,
 * seg_edges and seg_owner (segment_num, by segment id), device_segments
 * (num_devices) the segments each GPU takes. The per-GPU CSR copies the
 * reference then builds are not made. */
#define CGB_SEGMENT_SIZE 1024
typedef struct cgb_partition_info {
    uint32_t segment_num;     /* ceil(noZeroOutDegreeNum / CGB_SEGMENT_SIZE) */
    uint32_t bucket_start[5]; /* bucket b = sorted positions [bucket_start[b], bucket_start[b + 1]) */
    int32_t can_hold_all;     /* canHoldAllSegment: every segment went to a GPU */
    uint32_t reached_bucket;  /* the last bucket the deal entered */
} cgb_partition_info;

cgb_status cgb_graph_partition(cgb_graph* g, int algorithm, uint32_t num_devices, const uint64_t* device_mem_bytes,
                               uint32_t* seg_order, uint32_t* seg_edges, int32_t* seg_owner,
                               uint32_t* device_segments, cgb_partition_info* info);

/* CGB_EINVAL while a request server is attached to the graph (destroy the
 * server first). */
cgb_status cgb_graph_destroy(cgb_graph* g);

/* Runs all later work of this graph on `stream` (a cudaStream_t of the
 * graph's device; NULL restores the graph's own stream).  Lets a caller
 * order the engine's kernels with its own work and time them with events on
 * its stream. */
/* CGB_EINVAL while a request server is attached to the graph (its BFS group
 * runs on the graph's stream). */
cgb_status cgb_graph_set_stream(cgb_graph* g, void* stream);

/* Attaches edge weights to a graph created without them, or replaces its
 * weights: E values in the graph's CSR order, in host or device memory. Only
 * SSSP reads weights, so a caller can upload them while BFS, CC or PageRank
 * run on the same graph from another thread: the upload does not wait for
 * the graph. When it returns, the weights are in effect for every later
 * call on the graph (a run already in progress finishes with the old ones;
 * SSSP without weights uses unit weights). CGB_EINVAL while a request
 * server is attached to the graph, and when cgb_graph_create had to sort the neighbour
 * lists (give the weights to create then). Engine-specific (no reference
 * counterpart). */
cgb_status cgb_graph_set_weights(cgb_graph* g, const uint32_t* weight);

/* V, E and whether the graph is symmetric (-1 = not yet known). */
cgb_status cgb_graph_info(const cgb_graph* g, uint32_t* V, uint32_t* E, int32_t* symmetric);

/* Device pointers of the resident CSR and of the last run's result
 * (uint32[V] for BFS/SSSP/CC, double[V] for PR). */
cgb_status cgb_graph_device_csr(const cgb_graph* g, const uint32_t** offsets, const uint32_t** dest,
                                const uint32_t** weight);
cgb_status cgb_graph_result_device(const cgb_graph* g, const void** values);

/* Copies the last run's result (V uint32, or V double after PageRank) to a
 * host or device buffer.  Replaces GraphDeviceWorklist::result_D2H()
 * (GraphDevice.cuh:259-262). */
cgb_status cgb_graph_result_download(const cgb_graph* g, void* values);

/* ----------------------------------------------------------------- run */

/* One run of `algorithm` (cgb_algorithm).  For BFS/SSSP root_or_iters is the
 * root (< V); for CC it is ignored; for PR it is the iteration count, as in
 * graphProcess_device (GraphDevice.cuh:159-162: at least one iteration).
 * Results: out_u32 (V entries, BFS/SSSP/CC; CGB_VALUE_MAX = unreachable) or
 * out_f64 (V entries, PR); either may be NULL to keep the result on the
 * device only.  out_ms (may be NULL) receives the device time of the run,
 * the quantity graphProcess_device returns.  Calls on one graph serialise. */
cgb_status cgb_run(cgb_graph* g, int algorithm, uint32_t root_or_iters, const cgb_options* opt,
                   uint32_t* out_u32, double* out_f64, double* out_ms);

/* Several roots of BFS or SSSP in one call (no counterpart in the reference,
 * whose drivers loop over roots); out_u32 (host or device) holds nroots * V
 * values, root-major.  Roots run in passes of up to 64 sharing one
 * traversal with bit-packed per-vertex root masks (CGB_FLAG_BATCH_SEQUENTIAL:
 * one cgb_run per root instead).  Results equal nroots separate cgb_run
 * calls; out_ms and the statistics cover all passes. */
cgb_status cgb_run_batch(cgb_graph* g, int algorithm, const uint32_t* roots, uint32_t nroots,
                         const cgb_options* opt, uint32_t* out_u32, double* out_ms);

cgb_status cgb_run_stats_get(const cgb_graph* g, cgb_run_stats* out);

/* Copies up to max_entries trace entries of the last traced run; *count
 * receives the number available. */
cgb_status cgb_trace_get(const cgb_graph* g, cgb_iter_trace* out, uint32_t max_entries, uint32_t* count);

/* Graph buffers come from a per-device memory pool that keeps freed memory
 * for the next graph; this returns the cached memory to the driver. */
cgb_status cgb_memory_trim(int device);

/* The pool's size on a device: *reserved bytes held from the driver and
 * *used bytes handed out to live allocations (either pointer may be NULL).
 * Engine-specific (no reference counterpart): for monitoring the pool. */
cgb_status cgb_memory_info(int device, uint64_t* reserved, uint64_t* used);

/* Grows the pool to at least `bytes` reserved (no-op when it holds that much
 * already). Growing the pool costs driver time; a process that creates and
 * destroys graphs repeatedly can pay it once, up front. Engine-specific (no
 * reference counterpart). */
cgb_status cgb_memory_reserve(int device, uint64_t bytes);

/* ------------------------------------------------------------ tuning */

/* Launch parameters of a graph's kernels, one set per algorithm.  They
 * change only speed: every setting gives the same results.  cgb_graph_create
 * starts from the defaults below; cgb_autotune searches them for one graph
 * and algorithm. */
typedef struct {
    uint32_t struct_size;      /* sizeof(cgb_tuning) */
    uint32_t push_big_deg;     /* lists of at least this many edges are cut into chunks (128..65536, default 512) */
    uint32_t push_chunk;       /* edges per chunk (a power of two, 256..65536, default 1024) */
    uint32_t push_ctas_per_sm; /* grid of the push kernels, CTAs per SM (1..32, default 8) */
    uint32_t persist_enter;    /* device-resident loops take frontiers up to this size (0 = never, default 32768) */
    uint32_t persist_deg;      /* ... whose lists are all shorter than this (64..65536, default 2048) */
    uint32_t ms_edges;         /* multi-root SSSP: edges per work descriptor (64..4096, default 256) */
    uint32_t pr_unroll;        /* PageRank pull: gathers in flight per lane (4, 8 or 16, default 16) */
    uint32_t pr_ctas_per_sm;   /* PageRank pull grid, CTAs per SM (1..1024, capped at one 32-row slice
                                  per warp; default 128) */
    uint32_t persist_ctas;     /* CTAs of the device-resident loops (0 = one per SM, else 1..that;
                                  fewer CTAs make each level's grid barrier cheaper) */
    uint32_t sssp_pull_alpha;  /* SSSP rounds pull (scan in-edges of unsettled vertices) when the near
                                  set's out-edges times this exceed E; 0 = always push (default; on
                                  RMAT-24 the pull kernels lose to the push, the autotuner may pick it) */
    uint32_t cluster_enter;    /* BFS frontiers up to this size run their levels in one thread-block
                                  cluster with a hardware barrier (0 = never, default 8192) */
    uint32_t sssp_dense_alpha; /* SSSP rounds use a dense frontier when the near set's out-edges times
                                  this times max(first touches per edge in the previous round, 1/8)
                                  exceed V (0 = never, default 4) */
    uint32_t push_block;       /* threads per CTA of the push expansion kernels: 128, 256 or 512
                                  (0 = 256, the default); the reference fixes 256 (BLOCKSIZE,
                                  Basic/Graph/basic_def.hpp:8) */
    uint32_t reserved[2];
} cgb_tuning;

cgb_status cgb_tuning_get(const cgb_graph* g, int algorithm, cgb_tuning* out);
/* algorithm -1 sets every algorithm's tuning.  Rejects out-of-range values
 * with CGB_EINVAL and leaves the tuning unchanged. */
cgb_status cgb_tuning_set(cgb_graph* g, int algorithm, const cgb_tuning* t);

#define CGB_TUNE_BATCH 0x1u /* tune cgb_run_batch passes of the roots (else one cgb_run per root) */
#define CGB_TUNE_KEEP_DEFAULT 0x2u /* report the best tuning but leave the graph's tuning unchanged */
#define CGB_TUNE_CC_WEAK 0x4u /* tune CC runs with CGB_FLAG_CC_WEAK (weak components) */

/* Project-written autotuner (no counterpart in the reference, whose
 * thresholds are compile-time constants, device_warpDonate.cuh / device_CTA.cuh):
 * coordinate descent over the cgb_tuning fields that `algorithm` uses (BFS
 * or SSSP runs or multi-root passes from the roots; CC runs, one per entry
 * of `roots`, whose values are then ignored; PageRank runs of roots[i]
 * iterations), starting from the algorithm's current tuning, scoring each
 * candidate by the summed device time of the runs (best of two).
 * Sets the best tuning on the graph (unless CGB_TUNE_KEEP_DEFAULT) and
 * reports it with its time and the starting time. */
cgb_status cgb_autotune(cgb_graph* g, int algorithm, const uint32_t* roots, uint32_t nroots, uint32_t flags,
                        cgb_tuning* best, double* best_ms, double* start_ms);

/* ------------------------------------------------------- graph batches */

/* Many independent graphs solved together (no counterpart in the
 * reference, whose engines take one graph).  The n CSRs (host or device
 * pointers; weights may be NULL, or an array with NULL entries meaning unit
 * weights) are concatenated into one disjoint-union graph in HBM; each
 * graph's invariants are checked as cgb_graph_create checks them. */
typedef struct cgb_batch cgb_batch;
cgb_status cgb_batch_create(uint32_t n, const uint32_t* const* offsets, const uint32_t* const* dests,
                            const uint32_t* const* weights, const uint32_t* vertex_counts,
                            const uint32_t* edge_counts, int device, cgb_batch** out);
cgb_status cgb_batch_destroy(cgb_batch* b);

/* BFS or SSSP from roots[i] (a local id of graph i) in every graph at once,
 * or CC of every graph (roots ignored).  out_u32 receives the concatenated
 * per-graph results in local ids (sum of V entries), equal to separate
 * cgb_run calls.  BFS and SSSP run as one cooperative launch, captured into
 * a CUDA graph on first use and replayed afterwards. */
cgb_status cgb_batch_run(cgb_batch* b, int algorithm, const uint32_t* roots, uint32_t* out_u32, double* out_ms);

/* Totals of the union, and which runs replay a captured CUDA graph
 * (bit 0 BFS, bit 1 SSSP). */
cgb_status cgb_batch_info(const cgb_batch* b, uint32_t* total_vertices, uint32_t* total_edges, int32_t* one_launch);
cgb_status cgb_batch_stats(const cgb_batch* b, cgb_run_stats* out);

/* ----------------------------------------------------------- serving */

/* A request server on one resident graph (no counterpart in the reference,
 * whose drivers run one root at a time): BFS and SSSP root queries are
 * admitted as they arrive into up to 64 slots per algorithm, and all
 * admitted queries of an algorithm advance together, one level / round per
 * tick, sharing each edge traversal through bit-packed per-vertex masks;
 * a query that ends frees its slot for the next arrival (continuous
 * batching).  Each result equals a lone cgb_run of the same query. */
typedef struct cgb_server cgb_server;

typedef struct {
    uint32_t struct_size;    /* sizeof(cgb_server_config) */
    uint32_t bfs_slots;      /* concurrent BFS queries, <= 64 (0 = 64) */
    uint32_t sssp_slots;     /* concurrent SSSP queries, <= 64 (0 = 64) */
    uint32_t sssp_delta;     /* bucket width, 0 = the multi-root default of cgb_run_batch */
    uint64_t memory_budget;  /* bytes for per-query result regions (4 * V each); slots are
                                capped to fit; 0 = no cap */
    uint32_t flags;          /* CGB_SERVER_* */
    uint32_t reserved[5];
} cgb_server_config;

#define CGB_SERVER_NO_BFS 0x1u  /* no BFS slots (saves their masks) */
#define CGB_SERVER_NO_SSSP 0x2u /* no SSSP slots (saves the 256 B per vertex of distances) */
#define CGB_SERVER_HOST_TICKS 0x4u /* advance every level from the host thread (one synchronisation per
                                      level) instead of the device-resident level loop */
#define CGB_SERVER_BATCH_ONLY 0x8u /* every query joins its multi-root group.  By default a group
                                      serves its n <= 4 due queries one at a time on the single-root
                                      engine of cgb_run (between two ticks of its batch, if one runs)
                                      while n x (mean single-root time) <= (mean admission-to-result
                                      time of batched queries; unknown = infinite), and batches them
                                      otherwise */
#define CGB_SERVER_ADMIT_ANY_SLOT 0x10u /* a running group admits a due query into any free slot; by
                                           default only while at least half of its slots are free, so
                                           that admitted queries share more of their dense levels */

typedef struct {
    uint64_t id;
    int32_t algorithm;
    uint32_t root;
    double arrival_us;        /* times relative to cgb_server_start */
    double admit_us;
    double done_us;           /* result complete (and copied to out_u32) */
    uint64_t traversed_edges; /* out-degrees of the reached vertices */
    uint32_t reached;         /* vertices with a finite result */
    uint32_t depth;           /* BFS: deepest level; SSSP: largest finite distance */
    int32_t status;           /* CGB_OK or the error that ended the query */
    uint32_t slot;
} cgb_request_info;

cgb_status cgb_server_create(cgb_graph* g, const cgb_server_config* cfg, cgb_server** out);
/* Queues a query that becomes eligible arrival_us after cgb_server_start
 * (past times: at once).  out_u32 (host or device, V entries, or NULL)
 * receives the result when the query ends; it must stay valid until then. */
cgb_status cgb_server_submit(cgb_server* s, int algorithm, uint32_t root, double arrival_us, uint32_t* out_u32,
                             uint64_t* id);
/* Starts the clock and the serving thread. */
cgb_status cgb_server_start(cgb_server* s);
/* Waits until every submitted query has ended or timeout_ms passed;
 * pending receives the number still open. */
cgb_status cgb_server_wait(cgb_server* s, double timeout_ms, uint32_t* pending);
/* Moves up to cap records of ended queries into out (out NULL: n = how many
 * are waiting). */
cgb_status cgb_server_poll(cgb_server* s, cgb_request_info* out, uint32_t cap, uint32_t* n);
cgb_status cgb_server_stats(const cgb_server* s, uint64_t* ticks, uint32_t* bfs_slots, uint32_t* sssp_slots,
                            double* busy_ms);
/* Stops the serving thread and frees the server (the graph stays). */
cgb_status cgb_server_destroy(cgb_server* s);

/* --------------------------------------------------- allocation-free BFS */

/* Largest vertex count cgb_bfs_noalloc accepts. */
#define CGB_NOALLOC_MAX_VERTICES (1u << 20)

/* BFS levels for callers that cannot allocate device memory (a framework
 * whose caching allocator owns the device's memory, or a serving loop that
 * forbids cudaMalloc/cudaFree after start-up because they synchronise the
 * device).  No counterpart in the reference: it is an addition of this
 * engine.  The caller passes the CSR (device pointers offsets[V+1],
 * dest[E]), the root and the output levels[V] (device pointer), and a
 * cudaStream_t (NULL = default stream); results equal cgb_run(CGB_BFS).
 * Scratch (frontier queues, visited bitmap, counters) lives in one static
 * device array of about 12.7 MB that every GPU loading the library keeps
 * until exit; V > CGB_NOALLOC_MAX_VERTICES is rejected with CGB_EINVAL.
 * The first call on a device looks up the array's device address.  All
 * calls share the array: calls that overlap on the GPU race and must be
 * serialised by the caller.  Allocates nothing: no cudaMalloc, cudaFree or
 * allocating library routine. */
cgb_status cgb_bfs_noalloc(const uint32_t* offsets, const uint32_t* dest, uint32_t V, uint32_t E, uint32_t root,
                           uint32_t* levels, void* stream);

/* -------------------------------------------------------- learned policy */

/* The per-iteration scheduler (CGB_SCHED_LEARNED) is an FP32 MLP
 * CGB_POLICY_FEATURES -> 64 -> 64 -> CGB_POLICY_OUTPUTS whose outputs predict
 * the log-cost of each choice:
 *   [0] BFS next level pushed (degree-binned expansion), [1] pulled
 *       (bottom-up over a dense frontier bitmap), [9] pushed with every list
 *       of 32 edges or more cut into chunks dealt across the grid;
 *   [2..8] SSSP delta x {1/4, 1/2, 1, 2, 4, 8, 16} for the rest of the run,
 *       chosen once at the first bucket boundary (the cost of the remainder);
 *   [10..13] SSSP next near round as a sparse frontier (queue) with the
 *       degree-binned expansion, a sparse frontier with every list of 32
 *       edges or more chunked, a dense frontier (relax, then scan all
 *       vertices), or a pull over the in-edges.
 * Parameters are CGB_POLICY_PARAMS floats: W1[24][64] b1[64] W2[64][64]
 * b2[64] W3[64][14] b3[14] (row-major, input index first).  The reference
 * has no scheduler; these entry points have no counterpart in it. */
#define CGB_POLICY_FEATURES 24
#define CGB_POLICY_OUTPUTS 14
#define CGB_POLICY_PARAMS 6670

/* Makes `params` the policy of the current device (NULL unloads it: the
 * heuristic decides). */
cgb_status cgb_policy_load(const float* params);

/* Per-iteration training samples of one run: at every decision point the
 * engine snapshots its state, runs each choice (BFS level: the three
 * variants; SSSP bucket: all seven deltas; SSSP near round: the four round
 * variants), times it with CUDA events, restores, and continues with the
 * fastest.  features: max * 24 floats; targets: max * 14 log-costs; mask:
 * max * 14 (1 where measured).  The run's result equals a plain cgb_run. */
cgb_status cgb_policy_collect(cgb_graph* g, int algorithm, uint32_t root, const cgb_options* opt, float* features,
                              float* targets, uint8_t* mask, uint32_t max, uint32_t* count);

/* Trains the network on the GPU (hand-written forward, backward and Adam
 * kernels) with masked mean-squared error on the log-costs.  init may be
 * NULL (seeded initialisation).  Writes the trained parameters and the
 * final epoch's mean loss. */
cgb_status cgb_policy_train(const float* features, const float* targets, const uint8_t* mask, uint32_t n,
                            uint32_t epochs, uint32_t batch, float lr, uint64_t seed, const float* init,
                            float* params_out, float* final_loss);

/* Forward pass of `params` on n samples (outputs n * 9), and the masked MSE
 * loss with its full parameter gradient, both on the GPU (for checks). */
cgb_status cgb_policy_forward(const float* params, const float* features, uint32_t n, float* outputs);
cgb_status cgb_policy_loss_grad(const float* params, const float* features, const float* targets,
                                const uint8_t* mask, uint32_t n, float* loss, float* grad);

/* ---------------------------------------------------------------- misc */

/* Self-check of the engine's device-side timeout path (no counterpart in
 * the reference).  The device-resident loops separate their levels with a
 * grid barrier whose wait is bounded: a CTA that polls it more than a limit
 * sets a status flag and leaves, and the run returns CGB_ETIMEOUT instead of
 * hanging.  This launches one such loop on `device` in which one CTA never
 * arrives, with the given limit (1 .. 2^24 polls), and returns CGB_ETIMEOUT
 * when the others gave up as they should (the context stays usable). */
cgb_status cgb_check_barrier_timeout(int device, uint32_t spin_limit);

const char* cgb_last_error_string(void);
const char* cgb_status_string(cgb_status s);
int cgb_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* CGB200_H */
