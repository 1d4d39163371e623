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
// Limits and sharing: the array is sized for CGB_NOALLOC_MAX_VERTICES
// vertices (about 12.7 MB, held by every GPU that loads this library until
// the process exits); larger graphs are rejected with CGB_EINVAL.  All calls
// share the one array: each call clears what must start at zero, and calls
// whose work overlaps on the GPU (concurrent calls on different streams of
// one device) race on it and must be serialised by the caller.
//
// Set-up: host code cannot use the array's name as a device address (in host
// code it names a host-side stand-in), so the first call on each device,
// with that device current, asks cudaGetSymbolAddress for the array's device
// address and caches it; that first call should therefore come before any
// stream capture.  Nothing here calls cudaMalloc, cudaFree, cudaMallocHost
// or any other allocating routine.
#include <mutex>

#include "../../include/cgb200.h"
#include "engine.cuh"
#include "push.cuh"

namespace cgb {

constexpr uint32_t kNaMaxV = CGB_NOALLOC_MAX_VERTICES;
constexpr size_t kNaCtrBytes = 256;                                  // DevCounters, padded
constexpr size_t kNaQueueWords = kNaMaxV;                            // per queue
constexpr size_t kNaBitmapWords = kNaMaxV / 32 + 8;
constexpr size_t kNaWords = kNaCtrBytes / 4 + 3 * kNaQueueWords + kNaBitmapWords;
static_assert(sizeof(DevCounters) <= kNaCtrBytes, "counters do not fit their slot");

static __device__ __align__(256) uint32_t g_noalloc_scratch[kNaWords];

struct NaLayout {
    DevCounters* ctr;
    uint32_t* q[2];
    uint32_t* huge_q;
    uint32_t* visited;
};

static NaLayout layout_of(uint32_t* base)
{
    NaLayout l;
    l.ctr = reinterpret_cast<DevCounters*>(base);
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
// visited bitmap, write its level, append it to the next queue.
struct NaBfsOp {
    const uint32_t* __restrict__ off;
    const uint32_t* __restrict__ dst;
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
        if (valid) {
            d = dst[e];
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

__global__ void k_na_init(uint32_t V, uint32_t* level, uint32_t* visited, uint32_t words, DevCounters* ctr,
                          uint32_t root, uint32_t* q0)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    for (uint32_t i = tid; i < V; i += stride) level[i] = (i == root) ? 0u : kValueMax;
    for (uint32_t i = tid; i < words; i += stride) visited[i] = (i == (root >> 5)) ? (1u << (root & 31u)) : 0u;
    for (uint32_t i = tid; i < sizeof(DevCounters) / 4; i += stride) reinterpret_cast<uint32_t*>(ctr)[i] = 0;
    if (tid == 0) q0[0] = root;
}

__global__ void k_na_reset(DevCounters* ctr, int out)
{
    ctr->qlen[out] = 0;
    ctr->huge_len = 0;
}

// Level-synchronous top-down BFS over the degree-binned expansion of
// push.cuh, scratch in g_noalloc_scratch.  Results equal cgb_run(CGB_BFS).
static void bfs_noalloc(const uint32_t* off, const uint32_t* dst, uint32_t V, uint32_t root, uint32_t* level,
                        cudaStream_t st)
{
    const NaLayout l = layout_of(scratch_for_current_device());
    const uint32_t words = V / 32 + 1;
    k_na_init<<<kNumSMs * 4, kBlock, 0, st>>>(V, level, l.visited, words, l.ctr, root, l.q[0]);
    CGB_CUDA_TRY(cudaGetLastError());
    uint32_t nf = 1;
    int cur = 0;
    for (uint32_t lvl = 0; nf > 0; lvl++) {
        CGB_REQUIRE(lvl <= V, CGB_ETIMEOUT, "BFS level bound exceeded");
        const int out = cur ^ 1;
        k_na_reset<<<1, 1, 0, st>>>(l.ctr, out);
        NaBfsOp op{off, dst, level, l.visited, lvl + 1, l.q[out], &l.ctr->qlen[out], V, &l.ctr->overflow};
        const uint32_t grid = grid_for(nf, kBlock, kNumSMs * 8);
        k_push_twc<NaBfsOp, false><<<grid, kBlock, 0, st>>>(l.q[cur], nf, op, l.huge_q, &l.ctr->huge_len, V);
        k_push_huge<NaBfsOp><<<kNumSMs * 4, kBlock, 0, st>>>(l.huge_q, &l.ctr->huge_len, V, op);
        CGB_CUDA_TRY(cudaGetLastError());
        uint32_t h[2] = {0, 0};  // next queue length, overflow flag (stack memory, no allocation)
        CGB_CUDA_TRY(cudaMemcpyAsync(&h[0], &l.ctr->qlen[out], 4, cudaMemcpyDeviceToHost, st));
        CGB_CUDA_TRY(cudaMemcpyAsync(&h[1], &l.ctr->overflow, 4, cudaMemcpyDeviceToHost, st));
        CGB_CUDA_TRY(cudaStreamSynchronize(st));
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
        bfs_noalloc(offsets, dest, V, root, levels, static_cast<cudaStream_t>(stream));
        return CGB_OK;
    } catch (const Error& e) {
        set_error(e.msg);
        return e.code;
    } catch (const std::exception& e) {
        set_error(e.what());
        return CGB_ECUDA;
    }
}
