// C ABI of the engine (include/cgb200.h, include/cgb200_gen.h).
#include <sys/stat.h>

#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/cgb200.h"
#include "../../include/cgb200_gen.h"
#include "engine.cuh"
#include "persist.cuh"

namespace cgb {
cgb_graph* gen_rmat(uint32_t scale, uint32_t ef, uint64_t seed, double a, double b, double c, int scr, int sym,
                    uint32_t wmax, int device);
cgb_graph* gen_grid(uint32_t rows, uint32_t cols, uint64_t seed, uint32_t wmax, int device);
cgb_graph* gen_chunglu(uint32_t V, uint64_t draws, uint32_t i0, uint64_t seed, int sym, uint32_t wmax, int device);
void memory_trim(int device);
void memory_info(int device, uint64_t* reserved, uint64_t* used);
void memory_reserve(int device, uint64_t bytes);
}  // namespace cgb

using namespace cgb;

template <typename F>
static cgb_status guarded(F&& f)
{
    try {
        f();
        return CGB_OK;
    } catch (const Error& e) {
        set_error(e.msg);
        return e.code;
    } catch (const std::bad_alloc&) {
        set_error("host allocation failed");
        return CGB_ENOMEM;
    } catch (const std::exception& e) {
        set_error(e.what());
        return CGB_ECUDA;
    }
}

static cgb_options effective_options(const cgb_options* o)
{
    cgb_options r;
    std::memset(&r, 0, sizeof(r));
    r.struct_size = sizeof(r);
    if (o && o->struct_size) std::memcpy(&r, o, std::min<size_t>(o->struct_size, sizeof(r)));
    return r;
}

// Copies n elements from a host or device buffer (direction from the pointer).
static void copy_any(void* dst, const void* src, size_t bytes, cudaStream_t s)
{
    if (!bytes) return;
    CGB_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, s));
}

extern "C" {

int cgb_abi_version(void) { return CGB_ABI_VERSION; }

cgb_status cgb_check_barrier_timeout(int device, uint32_t spin_limit)
{
    return guarded([&] {
        CGB_REQUIRE(spin_limit >= 1 && spin_limit <= (1u << 24), CGB_EINVAL, "spin_limit must be in [1, 2^24]");
        CGB_CUDA_TRY(cudaSetDevice(device));
        const cgb_status st = barrier_timeout_check(spin_limit);
        if (st != CGB_OK) throw Error{st, "grid barrier gave up after spin_limit polls (the expected outcome)"};
    });
}

const char* cgb_last_error_string(void) { return last_error().c_str(); }

const char* cgb_status_string(cgb_status s)
{
    switch (s) {
    case CGB_OK: return "ok";
    case CGB_EINVAL: return "invalid argument";
    case CGB_EFORMAT: return "invalid CSR";
    case CGB_EIO: return "I/O error";
    case CGB_ENOMEM: return "out of memory";
    case CGB_ECUDA: return "CUDA error";
    case CGB_ETIMEOUT: return "timeout";
    case CGB_EOVERFLOW: return "queue overflow";
    case CGB_EUNSUPPORTED: return "unsupported";
    }
    return "unknown status";
}

cgb_status cgb_graph_create(const uint32_t* offsets, const uint32_t* dest, const uint32_t* weight, uint32_t V,
                            uint32_t E, uint32_t nz, int device, cgb_graph** out)
{
    return guarded([&] {
        CGB_REQUIRE(out != nullptr, CGB_EINVAL, "out is NULL");
        *out = nullptr;
        CGB_REQUIRE(offsets != nullptr, CGB_EINVAL, "offsets is NULL");
        CGB_REQUIRE(E == 0 || dest != nullptr, CGB_EINVAL, "dest is NULL");
        CGB_REQUIRE(V >= 1, CGB_EINVAL, "V must be >= 1");
        CGB_REQUIRE(V <= kMaxGraphSize && E <= kMaxGraphSize, CGB_EUNSUPPORTED, "V and E must be at most 2^32 - 2^24");
        cgb_graph* g = graph_alloc(V, E, nz, device, weight != nullptr && E > 0);
        try {
            copy_any(g->off, offsets, ((size_t)V + 1) * 4, g->stream);
            copy_any(g->dst, dest, (size_t)E * 4, g->stream);
            if (g->w) copy_any(g->w, weight, (size_t)E * 4, g->stream);
            CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
            validate_and_sort(g);
            compute_weight_sum(g);
        } catch (...) {
            graph_free(g);
            throw;
        }
        *out = g;
    });
}

// The first `length` words of a file that holds at least that many.
static std::vector<uint32_t> read_words(const char* path, uint64_t length)
{
    std::vector<uint32_t> a(length);
    FILE* f = std::fopen(path, "rb");
    if (!f) throw Error{CGB_EIO, std::string("cannot open ") + path};
    size_t got = length ? std::fread(a.data(), 4, length, f) : 0;
    std::fclose(f);
    if (got != length) throw Error{CGB_EIO, std::string("short read on ") + path};
    return a;
}

static uint64_t file_bytes(const char* path)
{
    struct stat st;
    CGB_REQUIRE(path != nullptr, CGB_EINVAL, "path is NULL");
    if (stat(path, &st) != 0) throw Error{CGB_EIO, std::string("Bin File [") + path + "] Not Exist"};
    return (uint64_t)st.st_size;
}

// load_binFile (Basic/Other/IO.hpp:44-92): the file must hold `length`
// whole elements, total_bytes / 4 == length; trailing bytes short of an
// element are ignored, as there.
static std::vector<uint32_t> load_array(const char* path, uint64_t length)
{
    if (file_bytes(path) / 4 != length)
        throw Error{CGB_EIO, std::string("(total_bytes / utilSize != length) for ") + path};
    return read_words(path, length);
}

cgb_status cgb_graph_load_files(const char* off_path, const char* dst_path, const char* w_path, uint32_t V,
                                uint32_t E, int device, cgb_graph** out)
{
    cgb_status st = CGB_OK;
    std::vector<uint32_t> off, dst, w;
    cgb_status ls = guarded([&] {
        CGB_REQUIRE(out != nullptr, CGB_EINVAL, "out is NULL");
        *out = nullptr;
        off = load_array(off_path, (uint64_t)V + 1);
        dst = load_array(dst_path, E);
        if (w_path) w = load_array(w_path, E);
    });
    if (ls != CGB_OK) return ls;
    st = cgb_graph_create(off.data(), dst.data(), w_path ? w.data() : nullptr, V, E, 0, device, out);
    return st;
}

cgb_status cgb_graph_create_from_edges(const uint32_t* records, uint64_t num_edges, uint32_t V, int device,
                                       cgb_graph** out)
{
    return guarded([&] {
        CGB_REQUIRE(out != nullptr, CGB_EINVAL, "out is NULL");
        *out = nullptr;
        *out = graph_from_edges(records, num_edges, V, device);
    });
}

cgb_status cgb_graph_load_edge_file(const char* path, uint32_t V, int device, cgb_graph** out)
{
    return guarded([&] {
        CGB_REQUIRE(out != nullptr, CGB_EINVAL, "out is NULL");
        *out = nullptr;
        // the reader takes total_bytes / 12 records and ignores a trailing
        // partial one (graphBinReader.hpp:92-93,152)
        const uint64_t E = file_bytes(path) / 12;
        const std::vector<uint32_t> rec = read_words(path, E * 3);
        *out = graph_from_edges(rec.data(), E, V, device);
    });
}

cgb_status cgb_graph_reorder(cgb_graph* g, int order_method, uint32_t* old2new, uint32_t* no_zero_out_degree_num,
                             cgb_graph** out)
{
    return guarded([&] {
        CGB_REQUIRE(out != nullptr, CGB_EINVAL, "out is NULL");
        *out = nullptr;
        CGB_REQUIRE(g != nullptr, CGB_EINVAL, "graph is NULL");
        std::lock_guard<GraphMutex> lock(g->mu);
        CGB_CUDA_TRY(cudaSetDevice(g->device));
        *out = graph_reorder(g, order_method, old2new, no_zero_out_degree_num);
    });
}

cgb_status cgb_graph_partition(cgb_graph* g, int algorithm, uint32_t num_devices, const uint64_t* device_mem_bytes,
                               uint32_t* seg_order, uint32_t* seg_edges, int32_t* seg_owner,
                               uint32_t* device_segments, cgb_partition_info* info)
{
    return guarded([&] {
        CGB_REQUIRE(g != nullptr && info != nullptr, CGB_EINVAL, "graph or info is NULL");
        CGB_REQUIRE(num_devices >= 1, CGB_EINVAL, "num_devices must be >= 1");
        CGB_REQUIRE(algorithm >= CGB_BFS && algorithm <= CGB_PR, CGB_EINVAL, "unknown algorithm");
        if (!device_mem_bytes) {
            int n = 0;
            CGB_CUDA_TRY(cudaGetDeviceCount(&n));
            CGB_REQUIRE(num_devices <= (uint32_t)n, CGB_EINVAL, "num_devices exceeds the visible devices");
        }
        std::lock_guard<GraphMutex> lock(g->mu);
        CGB_CUDA_TRY(cudaSetDevice(g->device));
        graph_partition(g, algorithm, num_devices, device_mem_bytes, seg_order, seg_edges, seg_owner,
                        device_segments, info);
    });
}

cgb_status cgb_graph_destroy(cgb_graph* g)
{
    return guarded([&] {
        CGB_REQUIRE(!g || g->servers.load() == 0, CGB_EINVAL, "a request server is attached to the graph");
        graph_free(g);
    });
}

cgb_status cgb_graph_set_stream(cgb_graph* g, void* stream)
{
    return guarded([&] {
        CGB_REQUIRE(g != nullptr, CGB_EINVAL, "graph is NULL");
        CGB_REQUIRE(g->servers.load() == 0, CGB_EINVAL, "a request server is attached to the graph");
        std::lock_guard<GraphMutex> lock(g->mu);
        CGB_CUDA_TRY(cudaSetDevice(g->device));
        CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
        g->stream = stream ? (cudaStream_t)stream : g->own_stream;
    });
}

cgb_status cgb_graph_set_weights(cgb_graph* g, const uint32_t* weight)
{
    return guarded([&] {
        CGB_REQUIRE(g != nullptr, CGB_EINVAL, "graph is NULL");
        CGB_REQUIRE(weight != nullptr || g->E == 0, CGB_EINVAL, "weight is NULL");
        graph_set_weights(g, weight);
    });
}

cgb_status cgb_graph_info(const cgb_graph* g, uint32_t* V, uint32_t* E, int32_t* symmetric)
{
    return guarded([&] {
        CGB_REQUIRE(g != nullptr, CGB_EINVAL, "graph is NULL");
        if (V) *V = g->V;
        if (E) *E = g->E;
        if (symmetric) *symmetric = g->symmetric;
    });
}

cgb_status cgb_graph_device_csr(const cgb_graph* g, const uint32_t** offsets, const uint32_t** dest,
                                const uint32_t** weight)
{
    return guarded([&] {
        CGB_REQUIRE(g != nullptr, CGB_EINVAL, "graph is NULL");
        if (offsets) *offsets = g->off;
        if (dest) *dest = g->dst;
        if (weight) *weight = g->w;
    });
}

cgb_status cgb_graph_result_device(const cgb_graph* g, const void** values)
{
    return guarded([&] {
        CGB_REQUIRE(g != nullptr && values != nullptr, CGB_EINVAL, "NULL argument");
        CGB_REQUIRE(g->result != nullptr, CGB_EINVAL, "no run has completed on this graph");
        *values = g->result;
    });
}

cgb_status cgb_graph_result_download(const cgb_graph* g, void* values)
{
    return guarded([&] {
        CGB_REQUIRE(g != nullptr && values != nullptr, CGB_EINVAL, "NULL argument");
        CGB_REQUIRE(g->result != nullptr, CGB_EINVAL, "no run has completed on this graph");
        CGB_CUDA_TRY(cudaSetDevice(g->device));
        const size_t bytes = (size_t)g->V * (g->result_alg == CGB_PR ? 8 : 4);
        copy_any(values, g->result, bytes, g->stream);
        CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    });
}

}  // extern "C"

// One run of the single-root engine; the caller holds the graph's lock.
namespace cgb {
void run_one(cgb_graph* g, int alg, uint32_t root_or_iters, const cgb_options& o)
{
    g->tune = g->tune_alg[alg];
    g->stats = cgb_run_stats{};
    g->trace.clear();
    g->flags = o.flags;
    g->kev_class.clear();
    g->kev_used = 0;
    g->result = nullptr;
    CGB_CUDA_TRY(cudaMemsetAsync(g->ctr, 0, sizeof(DevCounters), g->stream));
    switch (alg) {
    case CGB_BFS:
        run_bfs(g, root_or_iters, o);
        break;
    case CGB_SSSP:
        run_sssp(g, root_or_iters, o);
        break;
    case CGB_CC:
        run_cc(g, o);
        break;
    case CGB_PR:
        run_pr(g, root_or_iters, o);
        break;
    }
    CGB_CUDA_TRY(cudaEventSynchronize(g->ev_stop));
    CGB_CUDA_TRY(cudaGetLastError());
    float ms = 0.f;
    CGB_CUDA_TRY(cudaEventElapsedTime(&ms, g->ev_start, g->ev_stop));
    g->stats.ms = ms;
    if (o.flags & CGB_FLAG_KERNEL_TIMING) ktimer_collect(g);
    const uint64_t V = g->V, E = g->E;
    if (alg == CGB_BFS || alg == CGB_SSSP) {
        count_reached(g);
        const uint64_t per_edge = alg == CGB_BFS ? 8 : (g->w ? 12 : 8);
        g->stats.alg_bytes = per_edge * g->stats.traversed_edges + 12 * V;
    } else if (alg == CGB_CC) {
        g->stats.traversed_edges = E;
        g->stats.reached = V;
        g->stats.alg_bytes = 8 * E + 20 * V;
    } else {
        g->stats.traversed_edges = E * g->stats.iterations;
        g->stats.reached = V;
        g->stats.alg_bytes = (12 * E + 20 * V + 4) * g->stats.iterations;
    }
    if (alg != CGB_PR) g->result = g->value;
    g->result_alg = alg;
}
}  // namespace cgb

extern "C" {

cgb_status cgb_run(cgb_graph* g, int algorithm, uint32_t root_or_iters, const cgb_options* opt, uint32_t* out_u32,
                   double* out_f64, double* out_ms)
{
    return guarded([&] {
        CGB_REQUIRE(g != nullptr, CGB_EINVAL, "graph is NULL");
        CGB_REQUIRE(algorithm >= CGB_BFS && algorithm <= CGB_PR, CGB_EINVAL, "unknown Algorithm_type");
        if (algorithm == CGB_BFS || algorithm == CGB_SSSP)
            CGB_REQUIRE(root_or_iters < g->V, CGB_EINVAL, "root >= vertexNum");
        const cgb_options o = effective_options(opt);
        std::lock_guard<GraphMutex> lock(g->mu);
        CGB_CUDA_TRY(cudaSetDevice(g->device));
        run_one(g, algorithm, root_or_iters, o);
        if (algorithm == CGB_PR) {
            if (out_f64) copy_any(out_f64, g->result, (size_t)g->V * 8, g->stream);
        } else if (out_u32) {
            copy_any(out_u32, g->result, (size_t)g->V * 4, g->stream);
        }
        CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
        if (out_ms) *out_ms = g->stats.ms;
    });
}

// Sum of out-degrees of the reached vertices of n root-major level arrays.
__global__ void k_batch_reached(uint64_t n, uint32_t V, const uint32_t* __restrict__ val,
                                const uint32_t* __restrict__ off, DevCounters* ctr)
{
    unsigned long long edges = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        if (val[i] != kValueMax) {
            const uint32_t v = (uint32_t)(i % V);
            edges += off[v + 1] - off[v];
        }
    }
    edges = warp_sum(edges);
    if (lane_id() == 0 && edges) atomicAdd(&ctr->reached_edges, edges);
}

static bool is_device_ptr(const void* p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

cgb_status cgb_run_batch(cgb_graph* g, int algorithm, const uint32_t* roots, uint32_t nroots, const cgb_options* opt,
                         uint32_t* out_u32, double* out_ms)
{
    return guarded([&] {
        CGB_REQUIRE(g != nullptr && roots != nullptr, CGB_EINVAL, "NULL argument");
        CGB_REQUIRE(algorithm == CGB_BFS || algorithm == CGB_SSSP, CGB_EINVAL, "batch runs are BFS or SSSP");
        for (uint32_t i = 0; i < nroots; i++) CGB_REQUIRE(roots[i] < g->V, CGB_EINVAL, "root >= vertexNum");
        const cgb_options o = effective_options(opt);
        std::lock_guard<GraphMutex> lock(g->mu);
        CGB_CUDA_TRY(cudaSetDevice(g->device));
        const uint64_t V = g->V;
        if ((o.flags & CGB_FLAG_BATCH_SEQUENTIAL) || nroots == 1) {
            double total = 0;
            uint64_t edges = 0, launches = 0;
            for (uint32_t i = 0; i < nroots; i++) {
                run_one(g, algorithm, roots[i], o);
                total += g->stats.ms;
                edges += g->stats.traversed_edges;
                launches += g->stats.launches;
                if (out_u32) copy_any(out_u32 + (size_t)i * V, g->result, (size_t)V * 4, g->stream);
            }
            CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
            g->stats.ms = total;
            g->stats.traversed_edges = edges;
            g->stats.launches = launches;
            if (out_ms) *out_ms = total;
            return;
        }
        // multi-root passes of up to 64 roots
        g->tune = g->tune_alg[algorithm];
        g->stats = cgb_run_stats{};
        g->trace.clear();
        g->flags = o.flags;
        const bool dev_out = out_u32 && is_device_ptr(out_u32);
        const uint32_t per = 64;
        uint32_t* d_roots = nullptr;
        uint32_t* tmp = nullptr;
        try {
            // pool memory, ordered on the graph's stream (cudaMalloc / cudaFree of the
            // result staging, up to 64 x V words, cost a device-wide synchronisation)
            d_roots = static_cast<uint32_t*>(pool_alloc((size_t)per * 4, g->stream));
            if (!dev_out) tmp = static_cast<uint32_t*>(pool_alloc((size_t)std::min(per, nroots) * V * 4, g->stream));
            PinnedArray<uint32_t> h_roots(per);
            double total = 0;
            uint64_t edges = 0, iters = 0, launches = 0;
            for (uint32_t s0 = 0; s0 < nroots; s0 += per) {
                const uint32_t n = std::min(per, nroots - s0);
                uint32_t* lv = dev_out ? out_u32 + (size_t)s0 * V : tmp;
                std::copy(roots + s0, roots + s0 + n, h_roots.data());
                h2d_small(d_roots, h_roots.data(), (size_t)n * 4, g->stream);
                g->stats.launches = 0;
                CGB_CUDA_TRY(cudaEventRecord(g->ev_start, g->stream));
                if (algorithm == CGB_BFS) run_msbfs(g, d_roots, n, lv, o.bfs_alpha > 0 ? o.bfs_alpha : kMsAlpha);
                else run_mssp(g, d_roots, n, lv, o.sssp_delta ? o.sssp_delta : mssp_default_delta(g));
                CGB_CUDA_TRY(cudaEventRecord(g->ev_stop, g->stream));
                CGB_CUDA_TRY(cudaEventSynchronize(g->ev_stop));
                float ms = 0.f;
                CGB_CUDA_TRY(cudaEventElapsedTime(&ms, g->ev_start, g->ev_stop));
                total += ms;
                iters += g->stats.iterations;
                launches += g->stats.launches;
                CGB_CUDA_TRY(cudaMemsetAsync(&g->ctr->reached_edges, 0, 8, g->stream));
                k_batch_reached<<<num_sms() * 8, kBlock, 0, g->stream>>>((uint64_t)n * V, (uint32_t)V, lv, g->off, g->ctr);
                sync_counters(g);
                edges += g->h_ctr->reached_edges;
                if (out_u32 && !dev_out)
                    CGB_CUDA_TRY(cudaMemcpyAsync(out_u32 + (size_t)s0 * V, lv, (size_t)n * V * 4, cudaMemcpyDeviceToHost,
                                                 g->stream));
            }
            CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
            g->stats.ms = total;
            g->stats.iterations = iters;
            g->stats.launches = launches;
            g->stats.traversed_edges = edges;
            g->stats.alg_bytes = (algorithm == CGB_BFS ? 8 : (g->w ? 12 : 8)) * edges + 12ull * V * nroots;
            if (out_ms) *out_ms = total;
        } catch (...) {
            cudaStreamSynchronize(g->stream);
            pool_free(d_roots, g->stream);
            pool_free(tmp, g->stream);
            throw;
        }
        pool_free(d_roots, g->stream);
        pool_free(tmp, g->stream);
    });
}

cgb_status cgb_policy_collect(cgb_graph* g, int algorithm, uint32_t root, const cgb_options* opt, float* features,
                              float* targets, uint8_t* mask, uint32_t max, uint32_t* count)
{
    PolicySamples ps{features, targets, mask, max, 0};
    cgb_status st = guarded([&] {
        CGB_REQUIRE(g != nullptr && features && targets && mask, CGB_EINVAL, "NULL argument");
        CGB_REQUIRE(algorithm == CGB_BFS || algorithm == CGB_SSSP, CGB_EINVAL, "samples come from BFS or SSSP runs");
        CGB_REQUIRE(root < g->V, CGB_EINVAL, "root >= vertexNum");
        cgb_options o = effective_options(opt);
        if (o.schedule == CGB_SCHED_FIXED) o.schedule = CGB_SCHED_HEURISTIC;
        std::lock_guard<GraphMutex> lock(g->mu);
        CGB_CUDA_TRY(cudaSetDevice(g->device));
        CGB_CUDA_TRY(cudaMalloc((void**)&ps.save_value, (size_t)g->V * 4));
        CGB_CUDA_TRY(cudaMalloc((void**)&ps.save_bm0, (size_t)g->words() * 4));
        CGB_CUDA_TRY(cudaMalloc((void**)&ps.save_q, (size_t)g->V * 4));
        CGB_CUDA_TRY(cudaMalloc((void**)&ps.save_ctr, sizeof(DevCounters)));
        g->collect = &ps;
        try {
            run_one(g, algorithm, root, o);
        } catch (...) {
            g->collect = nullptr;
            throw;
        }
        g->collect = nullptr;
    });
    if (ps.save_value) cudaFree(ps.save_value);
    if (ps.save_bm0) cudaFree(ps.save_bm0);
    if (ps.save_q) cudaFree(ps.save_q);
    if (ps.save_ctr) cudaFree(ps.save_ctr);
    if (count) *count = ps.count;
    return st;
}

cgb_status cgb_run_stats_get(const cgb_graph* g, cgb_run_stats* out)
{
    return guarded([&] {
        CGB_REQUIRE(g != nullptr && out != nullptr, CGB_EINVAL, "NULL argument");
        *out = g->stats;
    });
}

cgb_status cgb_trace_get(const cgb_graph* g, cgb_iter_trace* out, uint32_t max_entries, uint32_t* count)
{
    return guarded([&] {
        CGB_REQUIRE(g != nullptr, CGB_EINVAL, "graph is NULL");
        if (count) *count = (uint32_t)g->trace.size();
        if (out)
            for (uint32_t i = 0; i < max_entries && i < g->trace.size(); i++) out[i] = g->trace[i];
    });
}

cgb_status cgb_gen_rmat(uint32_t scale, uint32_t edge_factor, uint64_t seed, double a, double b, double c,
                        int scramble, int symmetrise, uint32_t wmax, int device, cgb_graph** out)
{
    return guarded([&] {
        CGB_REQUIRE(out != nullptr, CGB_EINVAL, "out is NULL");
        *out = gen_rmat(scale, edge_factor, seed, a, b, c, scramble, symmetrise, wmax, device);
    });
}

cgb_status cgb_gen_grid(uint32_t rows, uint32_t cols, uint64_t seed, uint32_t wmax, int device, cgb_graph** out)
{
    return guarded([&] {
        CGB_REQUIRE(out != nullptr, CGB_EINVAL, "out is NULL");
        *out = gen_grid(rows, cols, seed, wmax, device);
    });
}

cgb_status cgb_memory_trim(int device)
{
    return guarded([&] { memory_trim(device); });
}

cgb_status cgb_memory_info(int device, uint64_t* reserved, uint64_t* used)
{
    return guarded([&] { memory_info(device, reserved, used); });
}

cgb_status cgb_memory_reserve(int device, uint64_t bytes)
{
    return guarded([&] { memory_reserve(device, bytes); });
}

cgb_status cgb_gen_chunglu(uint32_t vertices, uint64_t draws, uint32_t weight_offset, uint64_t seed, int symmetrise,
                           uint32_t wmax, int device, cgb_graph** out)
{
    return guarded([&] {
        CGB_REQUIRE(out != nullptr, CGB_EINVAL, "out is NULL");
        *out = gen_chunglu(vertices, draws, weight_offset, seed, symmetrise, wmax, device);
    });
}

cgb_status cgb_graph_download(const cgb_graph* g, uint32_t* offsets, uint32_t* dest, uint32_t* weight)
{
    return guarded([&] {
        CGB_REQUIRE(g != nullptr, CGB_EINVAL, "graph is NULL");
        CGB_CUDA_TRY(cudaSetDevice(g->device));
        if (offsets) copy_any(offsets, g->off, ((size_t)g->V + 1) * 4, g->stream);
        if (dest) copy_any(dest, g->dst, (size_t)g->E * 4, g->stream);
        if (weight && g->w) copy_any(weight, g->w, (size_t)g->E * 4, g->stream);
        CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    });
}

}  // extern "C"
