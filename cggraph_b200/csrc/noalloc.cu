// BFS for callers that cannot allocate device memory.
//
// Some callers may not call cudaMalloc: a framework whose caching allocator
// has already reserved the device's memory and must stay its only owner, or
// a serving loop that forbids allocation after start-up because
// cudaMalloc/cudaFree synchronise the device and can fail under memory
// pressure.  cgb_bfs_noalloc gives them the engine's top-down BFS with every
// scratch buffer (two frontier queues, the hub queue, the visited bitmap and
// the counters) carved out of one file-scope device array, g_noalloc_scratch.
//
// Input checks: the caller's CSR is checked on the device like
// cgb_graph_create checks it, with no allocation.  The offsets are checked
// first (offsets[0] == 0, non-decreasing, offsets[V] == E), and the BFS
// starts only once they pass, so every list read stays inside dest[0, E).
// Each destination id is checked where it is read: an id >= V sets an error
// word and is skipped, so neither the bitmap nor levels[] is touched outside
// its bounds; the host reads that word after every level and returns
// CGB_EFORMAT.  (The lists need not be sorted: BFS levels do not depend on
// the order of a list.)
//
// Limits and sharing: the array is sized for CGB_NOALLOC_MAX_VERTICES
// vertices (about 12.7 MB, held by every GPU that loads this library until
// the process exits); larger graphs are rejected with CGB_EINVAL.  All calls
// share the one array: each call clears what must start at zero, and calls
// whose work overlaps on the GPU (concurrent calls on different streams of
// one device) race on it and must be serialised by the caller.  A call
// synchronises its stream once per BFS level to read the next frontier's
// length.
//
// Set-up: host code cannot use the array's name as a device address (in host
// code it names a host-side stand-in), so the first call on each device,
// with that device current, asks cudaGetSymbolAddress for the array's device
// address and caches it.  The cached address belongs to the device's primary
// context: calling cudaDeviceReset while this library is loaded is not
// supported.  Nothing here calls cudaMalloc, cudaFree, cudaMallocHost or any
// other allocating routine.
#include <mutex>

#include "../../include/cgb200.h"
#include "engine.cuh"
#include "push.cuh"

namespace cgb {

constexpr uint32_t kNaMaxV = CGB_NOALLOC_MAX_VERTICES;
constexpr size_t kNaCtrBytes = 256;                                  // NaCounters, padded
constexpr size_t kNaQueueWords = kNaMaxV;                            // per queue
constexpr size_t kNaBitmapWords = kNaMaxV / 32 + 8;
constexpr size_t kNaWords = kNaCtrBytes / 4 + 3 * kNaQueueWords + kNaBitmapWords;
// Counters of a call: the engine's frontier counters plus the input-check
// word (1: offsets decrease, 2: offsets[0] != 0, 4: offsets[V] != E,
// 8: a destination id >= V).
struct NaCounters {
    DevCounters ctr;
    uint32_t bad;
};
static_assert(sizeof(NaCounters) <= kNaCtrBytes, "counters do not fit their slot");

static __device__ __align__(256) uint32_t g_noalloc_scratch[kNaWords];

struct NaLayout {
    DevCounters* ctr;
    uint32_t* bad;
    uint32_t* q[2];
    uint32_t* huge_q;
    uint32_t* visited;
};

static NaLayout layout_of(uint32_t* base)
{
    NaLayout l;
    NaCounters* c = reinterpret_cast<NaCounters*>(base);
    l.ctr = &c->ctr;
    l.bad = &c->bad;
    uint32_t* p = base + kNaCtrBytes / 4;
    l.q[0] = p;
    l.q[1] = p + kNaQueueWords;
    l.huge_q = p + 2 * kNaQueueWords;
    l.visited = p + 3 * kNaQueueWords;
    return l;
}

// Per-device cache of the array's device address (set-up on first use).
static std::mutex g_na_mu;
static uint32_t* g_na_ptr[256];

static uint32_t* scratch_for_current_device()
{
    int dev = 0;
    CGB_CUDA_TRY(cudaGetDevice(&dev));
    CGB_REQUIRE(dev >= 0 && dev < 256, CGB_EUNSUPPORTED, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_na_mu);
    if (!g_na_ptr[dev]) {
        void* ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || ptr == nullptr)
            throw Error{CGB_ECUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e)};
        g_na_ptr[dev] = static_cast<uint32_t*>(ptr);
    }
    return g_na_ptr[dev];
}

// Top-down visit: claim an unvisited destination with one atomicOr on the
// visited bitmap, write its level, append it to the next queue.  A
// destination id >= V sets bit 8 of *bad and is skipped before any access
// that it indexes.
struct NaBfsOp {
    const uint32_t* __restrict__ off;
    const uint32_t* __restrict__ dst;
    uint32_t V;
    uint32_t* bad;
    uint32_t* level;
    uint32_t* visited;
    uint32_t next_level;
    uint32_t* qout;
    uint32_t* qlen;
    uint32_t cap;
    uint32_t* overflow;

    __device__ __forceinline__ bool load(uint32_t v, uint32_t& s, uint32_t& d, uint32_t& m) const
    {
        s = off[v];
        d = off[v + 1] - s;
        m = 0;
        return true;
    }
    __device__ __forceinline__ void edge(bool valid, uint32_t e, uint32_t) const
    {
        bool win = false;
        uint32_t d = 0;
        if (valid) d = dst[e];
        if (valid && d >= V) {
            atomicOr(bad, 8u);
            d = 0;
        } else if (valid) {
            const uint32_t bit = 1u << (d & 31u);
            uint32_t* wp = visited + (d >> 5);
            if (!(*wp & bit) && !(atomicOr(wp, bit) & bit)) {
                win = true;
                level[d] = next_level;
            }
        }
        warp_append(win, d, qout, qlen, cap, overflow);
    }
};

// Checks the offsets (bits of *bad as in NaCounters); the BFS is launched
// only when *bad stays 0.
__global__ void k_na_check(uint32_t V, uint32_t E, const uint32_t* __restrict__ off, uint32_t* bad)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t b = 0;
    for (uint32_t v = tid; v < V; v += stride) b |= off[v] > off[v + 1] ? 1u : 0u;
    if (tid == 0) {
        b |= off[0] != 0 ? 2u : 0u;
        b |= off[V] != E ? 4u : 0u;
    }
    if (b) atomicOr(bad, b);
}

__global__ void k_na_init(uint32_t V, uint32_t* level, uint32_t* visited, uint32_t words, uint32_t root,
                          uint32_t* q0)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    for (uint32_t i = tid; i < V; i += stride) level[i] = (i == root) ? 0u : kValueMax;
    for (uint32_t i = tid; i < words; i += stride) visited[i] = (i == (root >> 5)) ? (1u << (root & 31u)) : 0u;
    if (tid == 0) q0[0] = root;
}

__global__ void k_na_reset(DevCounters* ctr, int out)
{
    ctr->qlen[out] = 0;
    ctr->huge_len = 0;
}

static void throw_bad_input(uint32_t bad)
{
    if (bad & 2u) throw Error{CGB_EFORMAT, "cgb_bfs_noalloc: offsets[0] != 0"};
    if (bad & 4u) throw Error{CGB_EFORMAT, "cgb_bfs_noalloc: offsets[V] != E"};
    if (bad & 1u) throw Error{CGB_EFORMAT, "cgb_bfs_noalloc: offsets are not non-decreasing"};
    throw Error{CGB_EFORMAT, "cgb_bfs_noalloc: dest holds a vertex id >= V"};
}

// Level-synchronous top-down BFS over the degree-binned expansion of
// push.cuh, scratch in g_noalloc_scratch.  Results equal cgb_run(CGB_BFS).
static void bfs_noalloc(const uint32_t* off, const uint32_t* dst, uint32_t V, uint32_t E, uint32_t root,
                        uint32_t* level, cudaStream_t st)
{
    uint32_t* base = scratch_for_current_device();
    const NaLayout l = layout_of(base);
    const uint32_t words = V / 32 + 1;
    uint32_t h[3] = {0, 0, 0};  // next queue length, overflow flag, input-check word (stack memory)
    // counters to zero, then the offsets check; nothing reads dest before it passes
    CGB_CUDA_TRY(cudaMemsetAsync(base, 0, kNaCtrBytes, st));
    k_na_check<<<grid_for(V, kBlock, num_sms() * 4), kBlock, 0, st>>>(V, E, off, l.bad);
    CGB_CUDA_TRY(cudaGetLastError());
    CGB_CUDA_TRY(cudaMemcpyAsync(&h[2], l.bad, 4, cudaMemcpyDeviceToHost, st));
    CGB_CUDA_TRY(cudaStreamSynchronize(st));
    if (h[2]) throw_bad_input(h[2]);
    k_na_init<<<num_sms() * 4, kBlock, 0, st>>>(V, level, l.visited, words, root, l.q[0]);
    CGB_CUDA_TRY(cudaGetLastError());
    uint32_t nf = 1;
    int cur = 0;
    for (uint32_t lvl = 0; nf > 0; lvl++) {
        CGB_REQUIRE(lvl <= V, CGB_ETIMEOUT, "BFS level bound exceeded");
        const int out = cur ^ 1;
        k_na_reset<<<1, 1, 0, st>>>(l.ctr, out);
        NaBfsOp op{off, dst, V, l.bad, level, l.visited, lvl + 1, l.q[out], &l.ctr->qlen[out], V, &l.ctr->overflow};
        const uint32_t grid = grid_for(nf, kBlock, num_sms() * 8);
        k_push_twc<NaBfsOp, false><<<grid, kBlock, 0, st>>>(l.q[cur], nf, op, l.huge_q, &l.ctr->huge_len, V);
        k_push_huge<NaBfsOp><<<num_sms() * 4, kBlock, 0, st>>>(l.huge_q, &l.ctr->huge_len, V, op);
        CGB_CUDA_TRY(cudaGetLastError());
        CGB_CUDA_TRY(cudaMemcpyAsync(&h[0], &l.ctr->qlen[out], 4, cudaMemcpyDeviceToHost, st));
        CGB_CUDA_TRY(cudaMemcpyAsync(&h[1], &l.ctr->overflow, 4, cudaMemcpyDeviceToHost, st));
        CGB_CUDA_TRY(cudaMemcpyAsync(&h[2], l.bad, 4, cudaMemcpyDeviceToHost, st));
        CGB_CUDA_TRY(cudaStreamSynchronize(st));
        if (h[2]) throw_bad_input(h[2]);
        CGB_REQUIRE(!h[1], CGB_EOVERFLOW, "BFS frontier queue overflow");
        nf = h[0];
        cur = out;
    }
}

}  // namespace cgb

extern "C" cgb_status cgb_bfs_noalloc(const uint32_t* offsets, const uint32_t* dest, uint32_t V, uint32_t E,
                                      uint32_t root, uint32_t* levels, void* stream)
{
    using namespace cgb;
    try {
        CGB_REQUIRE(offsets != nullptr && levels != nullptr && (E == 0 || dest != nullptr), CGB_EINVAL,
                    "cgb_bfs_noalloc: NULL pointer");
        CGB_REQUIRE(V >= 1, CGB_EINVAL, "cgb_bfs_noalloc: V must be >= 1");
        if (V > kNaMaxV)
            throw Error{CGB_EINVAL, "cgb_bfs_noalloc: V = " + std::to_string(V) +
                                        " exceeds the static scratch limit CGB_NOALLOC_MAX_VERTICES = " +
                                        std::to_string(kNaMaxV) + "; use cgb_run for larger graphs"};
        CGB_REQUIRE(root < V, CGB_EINVAL, "cgb_bfs_noalloc: root >= V");
        bfs_noalloc(offsets, dest, V, E, root, levels, static_cast<cudaStream_t>(stream));
        return CGB_OK;
    } catch (const Error& e) {
        set_error(e.msg);
        return e.code;
    } catch (const std::exception& e) {
        set_error(e.what());
        return CGB_ECUDA;
    }
}
