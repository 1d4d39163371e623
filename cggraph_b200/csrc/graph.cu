// Resident graph: upload, validation, neighbour sort, in-edge CSC, symmetry
// check, workspaces and kernel timers.
#include <atomic>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <vector>

#include "engine.cuh"

namespace cgb {

int num_sms()
{
    constexpr int kMaxDevices = 64;
    static std::atomic<int> cache[kMaxDevices];
    int dev = 0;
    CGB_CUDA_TRY(cudaGetDevice(&dev));
    CGB_REQUIRE(dev >= 0 && dev < kMaxDevices, CGB_EUNSUPPORTED, "device ordinal out of range");
    int v = cache[dev].load(std::memory_order_relaxed);
    if (v == 0) {
        CGB_CUDA_TRY(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev));
        CGB_REQUIRE(v > 0, CGB_ECUDA, "device reports no multiprocessors");
        cache[dev].store(v, std::memory_order_relaxed);
    }
    return v;
}


// ------------------------------------------------------------------ errors
static thread_local std::string t_last_error;
void set_error(const std::string& msg) { t_last_error = msg; }
const std::string& last_error() { return t_last_error; }

// --------------------------------------------------------------- allocation
// Graph buffers come from one stream-ordered memory pool per device that
// keeps freed memory cached (release threshold: never), so creating a graph
// after destroying another reuses the same pages: plain cudaFree of tens of
// GB returns them to the driver and can stall for hundreds of milliseconds.
// dalloc and dfree are ordered on the stream that uses the block (the
// graph's stream for everything here): a block freed on a stream is reused
// at once by the next allocation on it, and neither call waits for the
// device.  A block freed on another graph's stream is reused only once that
// free has happened (the allocation never waits for the other stream);
// otherwise the pool grows, and keeps what it grew by for later graphs.
// graph_alloc completes the graph's own buffers before returning, so they
// are usable on every stream.
namespace {
struct DevicePool {
    cudaMemPool_t pool = nullptr;
};
std::mutex g_pool_mu;
DevicePool g_pools[64];

DevicePool& device_pool()
{
    int dev = 0;
    CGB_CUDA_TRY(cudaGetDevice(&dev));
    CGB_REQUIRE(dev >= 0 && dev < 64, CGB_EUNSUPPORTED, "device index >= 64");
    std::lock_guard<std::mutex> lock(g_pool_mu);
    DevicePool& p = g_pools[dev];
    if (!p.pool) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        CGB_CUDA_TRY(cudaMemPoolCreate(&p.pool, &props));
        uint64_t keep = ~0ull;
        CGB_CUDA_TRY(cudaMemPoolSetAttribute(p.pool, cudaMemPoolAttrReleaseThreshold, &keep));
        // a block freed on one graph's stream is reused only once that free
        // has happened (never by making the allocation wait for that stream)
        int no = 0;
        CGB_CUDA_TRY(cudaMemPoolSetAttribute(p.pool, cudaMemPoolReuseAllowInternalDependencies, &no));
    }
    return p;
}
}  // namespace

template <typename T>
static T* dalloc(size_t n, cudaStream_t s)
{
    void* p = nullptr;
    if (n == 0) n = 1;
    CGB_CUDA_TRY(cudaMallocFromPoolAsync(&p, n * sizeof(T), device_pool().pool, s));
    return (T*)p;
}

static void dfree(void* p, cudaStream_t s)
{
    if (!p) return;
    cudaFreeAsync(p, s);
}

void pool_free(void* p, cudaStream_t s) { dfree(p, s); }

void* pool_alloc(size_t bytes, cudaStream_t s)
{
    void* p = dalloc<char>(bytes, s);
    CGB_CUDA_TRY(cudaStreamSynchronize(s));
    return p;
}

// Small pinned host blocks (each graph's counter mirror) come from slabs that
// live as long as the process: cudaMallocHost / cudaFreeHost per graph cost
// a driver call each, and freeing pinned memory has stalled for milliseconds.
namespace {
constexpr size_t kPinnedSlot = 256, kPinnedSlab = 256 * 1024;
std::mutex g_pinned_mu;
std::vector<void*> g_pinned_free;
}  // namespace

void* pinned_small_alloc(size_t bytes)
{
    CGB_REQUIRE(bytes <= kPinnedSlot, CGB_EINVAL, "pinned block too large");
    std::lock_guard<std::mutex> lock(g_pinned_mu);
    if (g_pinned_free.empty()) {
        char* slab = nullptr;
        CGB_CUDA_TRY(cudaMallocHost((void**)&slab, kPinnedSlab));
        for (size_t o = 0; o < kPinnedSlab; o += kPinnedSlot) g_pinned_free.push_back(slab + o);
    }
    void* p = g_pinned_free.back();
    g_pinned_free.pop_back();
    return p;
}

void pinned_small_free(void* p)
{
    if (!p) return;
    std::lock_guard<std::mutex> lock(g_pinned_mu);
    g_pinned_free.push_back(p);
}

// Pinned host blocks for the engine's own small transfers (flags, counts,
// samples, hub-row tables), by power-of-two size class, reused and kept
// until exit.  A copy to or from pageable memory is staged by the driver
// and waits for everything queued before it on its stream; while it waits,
// other threads' pageable copies wait too (a counter read behind a 2 GB
// upload held another graph's PageRank layout for 45 ms).
namespace {
std::mutex g_pinned_big_mu;
std::vector<void*> g_pinned_big_free[40];
int pinned_class(size_t bytes)
{
    int c = 9;  // 512 bytes
    while (((size_t)1 << c) < bytes) c++;
    return c;
}
}  // namespace

void* pinned_acquire(size_t bytes)
{
    if (bytes <= kPinnedSlot) return pinned_small_alloc(kPinnedSlot);
    const int c = pinned_class(bytes);
    CGB_REQUIRE(c < 40, CGB_EINVAL, "pinned block too large");
    {
        std::lock_guard<std::mutex> lock(g_pinned_big_mu);
        if (!g_pinned_big_free[c].empty()) {
            void* p = g_pinned_big_free[c].back();
            g_pinned_big_free[c].pop_back();
            return p;
        }
    }
    void* p = nullptr;
    CGB_CUDA_TRY(cudaMallocHost(&p, (size_t)1 << c));
    return p;
}

void pinned_release(void* p, size_t bytes)
{
    if (!p) return;
    if (bytes <= kPinnedSlot) {
        pinned_small_free(p);
        return;
    }
    std::lock_guard<std::mutex> lock(g_pinned_big_mu);
    g_pinned_big_free[pinned_class(bytes)].push_back(p);
}

// Small host-to-device transfers by a kernel that reads the pinned source
// through its device mapping, not by a copy engine: a copy engine works in
// order, and a small copy queued behind another graph's multi-GB upload
// waited for all of it (about 40 ms).  `src` must come from pinned_acquire
// (or another cudaMallocHost block); `bytes` is a multiple of 4.
__global__ void k_copy_words_from_host(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst, uint64_t n)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

void h2d_small(void* dst, const void* pinned_src, size_t bytes, cudaStream_t s)
{
    const uint64_t n = bytes / 4;
    if (!n) return;
    k_copy_words_from_host<<<grid_for(n, kBlock, num_sms()), kBlock, 0, s>>>(static_cast<const uint32_t*>(pinned_src),
                                                                           static_cast<uint32_t*>(dst), n);
    CGB_CUDA_TRY(cudaGetLastError());
}

void memory_trim(int device)
{
    CGB_CUDA_TRY(cudaSetDevice(device));
    DevicePool& dp = device_pool();
    CGB_CUDA_TRY(cudaDeviceSynchronize());  // every pending free has happened
    CGB_CUDA_TRY(cudaMemPoolTrimTo(dp.pool, 0));
}

// Grows the pool to at least `bytes` reserved: allocations of at most
// kReserveChunk each that bring the used amount up to `bytes` (the pool
// reserves at least what is in use), freed again; the pool keeps them
// (release threshold: never) for later allocations.  One block of many GB
// is avoided: buffers placed in such a block ran PageRank 2.6x slower here.
constexpr uint64_t kReserveChunk = 1ull << 30;

void memory_reserve(int device, uint64_t bytes)
{
    CGB_CUDA_TRY(cudaSetDevice(device));
    DevicePool& dp = device_pool();
    uint64_t r = 0, u = 0;
    CGB_CUDA_TRY(cudaMemPoolGetAttribute(dp.pool, cudaMemPoolAttrReservedMemCurrent, &r));
    CGB_CUDA_TRY(cudaMemPoolGetAttribute(dp.pool, cudaMemPoolAttrUsedMemCurrent, &u));
    if (r >= bytes) return;
    cudaStream_t s = nullptr;
    CGB_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    std::vector<void*> blocks;
    cudaError_t err = cudaSuccess;
    for (uint64_t need = bytes - u; need > 0 && err == cudaSuccess;) {
        const uint64_t n = std::min(need, kReserveChunk);
        void* p = nullptr;
        err = cudaMallocFromPoolAsync(&p, n, dp.pool, s);
        if (err == cudaSuccess) blocks.push_back(p);
        need -= n;
    }
    for (void* p : blocks) cudaFreeAsync(p, s);
    cudaError_t err2 = cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    CGB_CUDA_TRY(err);
    CGB_CUDA_TRY(err2);
}

void memory_info(int device, uint64_t* reserved, uint64_t* used)
{
    CGB_CUDA_TRY(cudaSetDevice(device));
    DevicePool& dp = device_pool();
    uint64_t r = 0, u = 0;
    CGB_CUDA_TRY(cudaMemPoolGetAttribute(dp.pool, cudaMemPoolAttrReservedMemCurrent, &r));
    CGB_CUDA_TRY(cudaMemPoolGetAttribute(dp.pool, cudaMemPoolAttrUsedMemCurrent, &u));
    if (reserved) *reserved = r;
    if (used) *used = u;
}

static uint32_t bits_for(uint64_t n)  // bits to represent values < n
{
    uint32_t b = 1;
    while (b < 64 && (1ull << b) < n) b++;
    return b;
}

// ------------------------------------------------------------- validation
__global__ void k_check_offsets(uint32_t V, uint32_t E, const uint32_t* __restrict__ off, uint32_t* bad)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        if (off[v] > off[v + 1]) atomicOr(bad, 1u);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (off[0] != 0) atomicOr(bad, 2u);
        if (off[V] != E) atomicOr(bad, 4u);
    }
}

// Marks the first edge of every non-empty neighbour list in a bitmap over
// edge indices (E/32 + 1 words).
__global__ void k_mark_heads(uint32_t V, const uint32_t* __restrict__ off, uint32_t* heads)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        const uint32_t s = off[v];
        if (off[v + 1] > s) atomicOr(heads + (s >> 5), 1u << (s & 31u));
    }
}

// bad |= 8 for an id >= V; unsorted |= 1 where a list is not strictly
// ascending; dup |= 1 where it has equal neighbours.  A warp reads 32 x 8
// consecutive entries with independent loads and takes each entry's
// successor from the next lane (the last lane reads one entry more).
constexpr uint32_t kCheckRuns = 8;

__global__ void k_check_edges(uint32_t V, uint32_t E, const uint32_t* __restrict__ dst,
                              const uint32_t* __restrict__ heads, uint32_t* flags)
{
    const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / 32;
    const uint32_t lane = lane_id();
    uint32_t bad = 0, unsorted = 0, dup = 0;
    for (uint64_t base = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32 * 32 * kCheckRuns; base < E;
         base += warps * 32 * kCheckRuns) {
        uint32_t d[kCheckRuns], nx[kCheckRuns], hw[kCheckRuns];
#pragma unroll
        for (uint32_t k = 0; k < kCheckRuns; k++) {
            const uint64_t e = base + k * 32 + lane;
            d[k] = e < E ? dst[e] : 0;
            nx[k] = (lane == 31 && e + 1 < E) ? dst[e + 1] : 0;
            hw[k] = e + 1 < E ? heads[(e + 1) >> 5] : 0;
        }
#pragma unroll
        for (uint32_t k = 0; k < kCheckRuns; k++) {
            const uint64_t e = base + k * 32 + lane;
            const uint32_t down = __shfl_down_sync(0xffffffffu, d[k], 1);
            const uint32_t next = lane == 31 ? nx[k] : down;
            if (e < E) {
                bad |= d[k] >= V;
                if (e + 1 < E && !((hw[k] >> ((e + 1) & 31u)) & 1u)) {
                    unsorted |= d[k] > next;
                    dup |= d[k] == next;
                }
            }
        }
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(flags, 8u);
    if (__any_sync(0xffffffffu, unsorted) && lane == 0) atomicOr(flags + 1, 1u);
    if (__any_sync(0xffffffffu, dup) && lane == 0) atomicOr(flags + 2, 1u);
}

// Source vertex of edge e: last v with off[v] <= e (skipping empty lists).
__device__ __forceinline__ uint32_t edge_source(const uint32_t* __restrict__ off, uint32_t V, uint32_t e)
{
    uint32_t lo = 0, hi = V;  // invariant: off[lo] <= e < off[hi]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (off[mid] <= e) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Every edge with its row, tile by tile.  trow[t] is the row of tile t's
// first edge (trow[ntiles] that of the last edge), found for all tiles at
// once by k_tile_rows.  A CTA stages off[trow[t] .. trow[t + 1] + 1] in
// shared memory and marks the first edge of every row that starts inside
// the tile with that row's index; each warp then takes 32 edges at a time
// and gives each the last mark at or before it (a max-scan across the
// lanes, carried from round to round), starting from the row of its first
// edge.  For every edge e of the tile, r being the non-empty row with beg =
// off[r] <= e < end = off[r + 1], it calls f.store(e, r, beg, end,
// f.load(e, r, beg, end)) with the warp's lanes on consecutive edges; the
// loads of F::kBatch rounds are issued before their stores, so a functor's
// gathers can be in flight together (a larger batch holds more registers:
// worth it for a long chain of dependent gathers, not for one or two).  A tile spanning kRowStage rows or
// more (long runs of empty rows) searches off in global memory per edge
// instead.  Each thread works on its own copy of f; f.tile_end() runs on
// every thread after each tile (the warp still converged), and f.stop() is
// asked before each tile (a functor that has found its answer ends the
// pass).
constexpr uint32_t kRowTile = 4096;        // edges per tile
constexpr uint32_t kRowStage = 4096 + 64;  // staged offsets per CTA: a tile of one-edge rows fits

__global__ void k_tile_rows(uint32_t V, uint32_t E, const uint32_t* __restrict__ off, uint32_t ntiles, uint32_t* trow)
{
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t <= ntiles; t += gridDim.x * blockDim.x) {
        const uint64_t e = (uint64_t)t * kRowTile;
        trow[t] = edge_source(off, V, (uint32_t)(e < E ? e : E - 1));
    }
}

template <class F>
__global__ void __launch_bounds__(kBlock) k_edges_by_row(uint32_t E, const uint32_t* __restrict__ off,
                                                         const uint32_t* __restrict__ trow, F fp)
{
    F f = fp;
    constexpr uint32_t kSeg = kRowTile / (kBlock / 32);  // edges per warp and tile
    constexpr uint32_t kRounds = kSeg / 32;
    constexpr uint32_t kBatch = F::kBatch;  // rounds whose loads are issued before their stores
    __shared__ uint32_t s_off[kRowStage];
    __shared__ uint16_t s_mark[kRowTile];  // 1 + row index at a row's first edge, else 0
    __shared__ uint32_t s_r[2];
    __shared__ bool s_stop;
    const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
    for (uint64_t t0 = (uint64_t)blockIdx.x * kRowTile; t0 < E; t0 += (uint64_t)gridDim.x * kRowTile) {
        const uint32_t e0 = (uint32_t)t0;
        const uint32_t e1 = (uint32_t)(t0 + kRowTile < E ? t0 + kRowTile : E);
        if (threadIdx.x == 0) s_stop = f.stop();  // one read, so the whole CTA agrees
        if (threadIdx.x < 2) s_r[threadIdx.x] = trow[t0 / kRowTile + threadIdx.x];
        for (uint32_t i = threadIdx.x; i < kRowTile; i += blockDim.x) s_mark[i] = 0;
        __syncthreads();
        if (s_stop) return;
        const uint32_t r0 = s_r[0], n = s_r[1] - s_r[0] + 1;  // rows r0 .. r0 + n - 1 cover the tile
        if (n < kRowStage) {
            for (uint32_t i = threadIdx.x; i <= n; i += blockDim.x) s_off[i] = off[r0 + i];
            __syncthreads();
            // rows after r0 (which holds e0) that start inside the tile
            for (uint32_t i = 1 + threadIdx.x; i < n; i += blockDim.x) {
                const uint32_t b = s_off[i];
                if (s_off[i + 1] > b && b < e1) s_mark[b - e0] = (uint16_t)(i + 1);
            }
            __syncthreads();
            const uint32_t sb = e0 + warp * kSeg;
            if (sb < e1) {
                uint32_t lo = 0, hi = n;  // the row of sb: s_off[lo] <= sb < s_off[hi]
                while (hi - lo > 1) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (s_off[mid] <= sb) lo = mid;
                    else hi = mid;
                }
                // rows of all rounds first, then the calls: their loads are
                // independent of one another and can be in flight together
                uint32_t carry = lo, rel[kRounds];
#pragma unroll
                for (uint32_t k = 0; k < kRounds; k++) {
                    const uint32_t x = s_mark[warp * kSeg + k * 32 + lane];  // 0 past e1
                    // the last marked lane at or below this one names the row
                    const uint32_t below = __ballot_sync(0xffffffffu, x != 0) & (0xffffffffu >> (31 - lane));
                    const uint32_t y = __shfl_sync(0xffffffffu, x, below ? 31 - __clz(below) : 0);
                    rel[k] = below ? y - 1 : carry;
                    carry = __shfl_sync(0xffffffffu, rel[k], 31);
                }
#pragma unroll
                for (uint32_t k0 = 0; k0 < kRounds; k0 += kBatch) {
                    typename F::Val v[kBatch];
#pragma unroll
                    for (uint32_t k = 0; k < kBatch; k++) {
                        const uint32_t e = sb + (k0 + k) * 32 + lane, q = rel[k0 + k];
                        if (e < e1) v[k] = f.load(e, r0 + q, s_off[q], s_off[q + 1]);
                    }
#pragma unroll
                    for (uint32_t k = 0; k < kBatch; k++) {
                        const uint32_t e = sb + (k0 + k) * 32 + lane, q = rel[k0 + k];
                        if (e < e1) f.store(e, r0 + q, s_off[q], s_off[q + 1], v[k]);
                    }
                }
            }
        } else {
            for (uint32_t e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
                uint32_t lo = r0, hi = r0 + n;  // off[lo] <= e < off[hi]
                while (hi - lo > 1) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (off[mid] <= e) lo = mid;
                    else hi = mid;
                }
                f.store(e, lo, off[lo], off[lo + 1], f.load(e, lo, off[lo], off[lo + 1]));
            }
        }
        f.tile_end();
        __syncthreads();
    }
}

template <class F>
static void launch_edges_by_row(cgb_graph* g, uint32_t V, uint32_t E, const uint32_t* off, const F& f)
{
    if (E == 0) return;
    const uint32_t tiles = div_up(E, kRowTile);
    uint32_t* trow = dalloc<uint32_t>((size_t)tiles + 1, g->stream);
    k_tile_rows<<<grid_for((uint64_t)tiles + 1, kBlock, num_sms() * 8), kBlock, 0, g->stream>>>(V, E, off, tiles, trow);
    k_edges_by_row<<<min(tiles, num_sms() * 8), kBlock, 0, g->stream>>>(E, off, trow, f);  // 24 KB each
    dfree(trow, g->stream);
}

// key = row << b | dst (b = bits for V): sorting the keys sorts every list
struct RowKeysF {
    static constexpr uint32_t kBatch = 1;
    __device__ __forceinline__ bool stop() const { return false; }
    __device__ __forceinline__ void tile_end() {}
    const uint32_t* __restrict__ dst;
    uint32_t b;
    uint64_t* __restrict__ keys;
    using Val = uint32_t;
    __device__ __forceinline__ Val load(uint32_t e, uint32_t, uint32_t, uint32_t) const { return __ldg(dst + e); }
    __device__ __forceinline__ void store(uint32_t e, uint32_t r, uint32_t, uint32_t, Val d)
    {
        keys[e] = ((uint64_t)r << b) | d;
    }
};

// the source of every edge, in CSR order
struct RowOutF {
    static constexpr uint32_t kBatch = 1;
    __device__ __forceinline__ bool stop() const { return false; }
    __device__ __forceinline__ void tile_end() {}
    uint32_t* __restrict__ rows;
    using Val = uint32_t;
    __device__ __forceinline__ Val load(uint32_t, uint32_t, uint32_t, uint32_t) const { return 0; }
    __device__ __forceinline__ void store(uint32_t e, uint32_t r, uint32_t, uint32_t, Val) { rows[e] = r; }
};

__global__ void k_split_keys(uint32_t E, const uint64_t* __restrict__ keys, uint32_t b, uint32_t* low)
{
    const uint64_t mask = (1ull << b) - 1;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x)
        low[e] = (uint32_t)(keys[e] & mask);
}

__global__ void k_widen(uint32_t n, const uint32_t* __restrict__ a, uint64_t* o)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) o[i] = a[i];
}

__global__ void k_narrow(uint32_t n, const uint64_t* __restrict__ a, uint32_t* o)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) o[i] = (uint32_t)a[i];
}

__global__ void k_max_degree(uint32_t V, const uint32_t* __restrict__ off, uint32_t* out)
{
    uint32_t m = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x)
        m = max(m, off[v + 1] - off[v]);
    m = warp_max(m);
    if (lane_id() == 0 && m) atomicMax(out, m);
}

__global__ void k_sum_u32(uint32_t n, const uint32_t* __restrict__ a, unsigned long long* out)
{
    unsigned long long s = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += a[i];
    s = warp_sum(s);
    if (lane_id() == 0 && s) atomicAdd(out, s);
}

__global__ void k_collect_heavy_rows(uint32_t V, const uint32_t* __restrict__ in_off, uint32_t th, uint32_t* rows,
                                     uint32_t* n)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        if (in_off[v + 1] - in_off[v] >= th) rows[atomicAdd(n, 1u)] = v;
    }
}

__global__ void k_count_reached(uint32_t V, const uint32_t* __restrict__ value, const uint32_t* __restrict__ off,
                                DevCounters* ctr)
{
    unsigned long long edges = 0;
    uint32_t cnt = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        if (value[v] != kValueMax) {
            cnt++;
            edges += off[v + 1] - off[v];
        }
    }
    edges = warp_sum(edges);
    cnt = warp_sum(cnt);
    if (lane_id() == 0 && cnt) {
        atomicAdd(&ctr->reached_edges, edges);
        atomicAdd(&ctr->reached, cnt);
    }
}

// -------------------------------------------------------------- graph ops
void sync_counters(cgb_graph* g)
{
    CGB_CUDA_TRY(cudaMemcpyAsync(g->h_ctr, g->ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, g->stream));
    CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
}

static void radix_sort_u64(cgb_graph* g, uint64_t*& keys, uint64_t*& alt, uint64_t n, int end_bit)
{
    cub::DoubleBuffer<uint64_t> db(keys, alt);
    size_t temp_bytes = 0;
    CGB_CUDA_TRY(cub::DeviceRadixSort::SortKeys(nullptr, temp_bytes, db, n, 0, end_bit, g->stream));
    void* temp = dalloc<char>(temp_bytes, g->stream);
    cudaError_t err = cub::DeviceRadixSort::SortKeys(temp, temp_bytes, db, n, 0, end_bit, g->stream);
    CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    dfree(temp, g->stream);
    CGB_CUDA_TRY(err);
    if (db.Current() != keys) std::swap(keys, alt);
}

// Sorts every neighbour list by destination, weights following
// (nbrSort_taskSteal, my_project/CGgraph/sortNbr.hpp:8-99).
static void sort_neighbours(cgb_graph* g)
{
    const uint32_t V = g->V, E = g->E;
    const uint32_t b = bits_for(V);
    uint64_t* keys = dalloc<uint64_t>(E, g->stream);
    uint64_t* alt = dalloc<uint64_t>(E, g->stream);
    const uint32_t grid = grid_for(E, kBlock, num_sms() * 16);
    if (g->w) {
        uint64_t* vals = dalloc<uint64_t>(E, g->stream);
        uint64_t* valt = dalloc<uint64_t>(E, g->stream);
        launch_edges_by_row(g, V, E, g->off, RowKeysF{g->dst, b, keys});
        k_widen<<<grid, kBlock, 0, g->stream>>>(E, g->w, vals);
        cub::DoubleBuffer<uint64_t> kb(keys, alt), vb(vals, valt);
        size_t temp_bytes = 0;
        CGB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, kb, vb, (uint64_t)E, 0, 2 * b, g->stream));
        void* temp = dalloc<char>(temp_bytes, g->stream);
        cudaError_t err = cub::DeviceRadixSort::SortPairs(temp, temp_bytes, kb, vb, (uint64_t)E, 0, 2 * b, g->stream);
        CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
        dfree(temp, g->stream);
        CGB_CUDA_TRY(err);
        k_split_keys<<<grid, kBlock, 0, g->stream>>>(E, kb.Current(), b, g->dst);
        k_narrow<<<grid, kBlock, 0, g->stream>>>(E, vb.Current(), g->w);
        CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
        dfree(vals, g->stream);
        dfree(valt, g->stream);
    } else {
        launch_edges_by_row(g, V, E, g->off, RowKeysF{g->dst, b, keys});
        radix_sort_u64(g, keys, alt, E, 2 * b);
        k_split_keys<<<grid, kBlock, 0, g->stream>>>(E, keys, b, g->dst);
        CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    }
    dfree(keys, g->stream);
    dfree(alt, g->stream);
}

void validate_and_sort(cgb_graph* g)
{
    const uint32_t V = g->V, E = g->E;
    uint32_t* flags = dalloc<uint32_t>(4, g->stream);
    CGB_CUDA_TRY(cudaMemsetAsync(flags, 0, 4 * sizeof(uint32_t), g->stream));
    k_check_offsets<<<grid_for(V, kBlock, num_sms() * 8), kBlock, 0, g->stream>>>(V, E, g->off, flags);
    PinnedArray<uint32_t> h(4);
    CGB_CUDA_TRY(cudaMemcpyAsync(h.data(), flags, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, g->stream));
    CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    if (h[0]) {
        dfree(flags, g->stream);
        if (h[0] & 2u) throw Error{CGB_EFORMAT, "csr_offset[0] != 0"};
        if (h[0] & 4u) throw Error{CGB_EFORMAT, "csr_offset[V] != E"};
        throw Error{CGB_EFORMAT, "csr_offset is not non-decreasing"};
    }
    // the vertices from noZeroOutDegreeNum on hold no edges: csr_offset[nz] == E
    // (the driver's RCM_LAST_ZERO_OUTDEGREE_check, main_partition.hpp:88-101)
    if (g->nz < V) {
        CGB_CUDA_TRY(cudaMemcpyAsync(h.data(), g->off + g->nz, sizeof(uint32_t), cudaMemcpyDeviceToHost, g->stream));
        CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
        if (h[0] != E) {
            dfree(flags, g->stream);
            throw Error{CGB_EFORMAT, "a vertex at or above noZeroOutDegreeNum has out-edges (csr_offset[noZeroOutDegreeNum] != E)"};
        }
    }
    if (E == 0) {
        dfree(flags, g->stream);
        return;
    }
    const uint32_t hw = E / 32 + 2;
    uint32_t* heads = dalloc<uint32_t>(hw, g->stream);
    for (int pass = 0; pass < 2; pass++) {
        CGB_CUDA_TRY(cudaMemsetAsync(heads, 0, hw * sizeof(uint32_t), g->stream));
        CGB_CUDA_TRY(cudaMemsetAsync(flags, 0, 4 * sizeof(uint32_t), g->stream));
        k_mark_heads<<<grid_for(V, kBlock, num_sms() * 8), kBlock, 0, g->stream>>>(V, g->off, heads);
        k_check_edges<<<grid_for(E, kBlock, num_sms() * 16), kBlock, 0, g->stream>>>(V, E, g->dst, heads, flags);
        CGB_CUDA_TRY(cudaMemcpyAsync(h.data(), flags, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, g->stream));
        CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
        if (h[0] & 8u) {
            dfree(heads, g->stream);
            dfree(flags, g->stream);
            throw Error{CGB_EFORMAT, "csr_dest holds a vertex id >= V"};
        }
        if (pass == 0 && h[1]) {
            sort_neighbours(g);
            g->lists_resorted = true;
            continue;
        }
        if (h[1] || h[2]) {
            dfree(heads, g->stream);
            dfree(flags, g->stream);
            throw Error{CGB_EFORMAT, "neighbour list not strictly ascending after sorting (duplicate edge)"};
        }
        break;
    }
    dfree(heads, g->stream);
    dfree(flags, g->stream);
}

void compute_weight_sum(cgb_graph* g)
{
    if (!g->w || g->E == 0) return;
    unsigned long long* d = dalloc<unsigned long long>(1, g->stream);
    CGB_CUDA_TRY(cudaMemsetAsync(d, 0, sizeof(unsigned long long), g->stream));
    k_sum_u32<<<grid_for(g->E, kBlock, num_sms() * 8), kBlock, 0, g->stream>>>(g->E, g->w, d);
    PinnedArray<unsigned long long> h(1);
    CGB_CUDA_TRY(cudaMemcpyAsync(h.data(), d, sizeof(unsigned long long), cudaMemcpyDeviceToHost, g->stream));
    CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    dfree(d, g->stream);
    g->sum_w = h[0];
}

// differ = 1 when a and b differ somewhere.  Warps walk the arrays in
// lockstep; the first warp that sees a difference sets the flag with one
// atomic, and every warp looks at the flag each 16 steps to stop early.
// Weights given after create (cgb_graph_set_weights) are uploaded and summed
// on a private stream without holding the graph, then left pending; whoever
// takes the graph's lock next swaps them in (GraphMutex::lock), at once if
// the graph is idle.  Weights in CSC order are rebuilt on their next use.
static void swap_in_pending_weights(cgb_graph* g) noexcept
{
    uint32_t* w = nullptr;
    uint64_t sum = 0;
    {
        std::lock_guard<std::mutex> pl(g->pending_mu);
        w = g->pending_w;
        sum = g->pending_sum_w;
        g->pending_w = nullptr;
    }
    if (!w) return;
    cudaSetDevice(g->device);
    // stream-ordered frees: after every earlier use of the old weights
    if (g->in_w_owned) dfree(g->in_w, g->stream);
    g->in_w = nullptr;
    g->in_w_owned = false;
    if (g->w) dfree(g->w, g->stream);
    g->w = w;
    g->sum_w = sum;
}

void graph_set_weights(cgb_graph* g, const uint32_t* weight)
{
    CGB_REQUIRE(!g->lists_resorted, CGB_EINVAL,
                "weights must be given to cgb_graph_create when it had to sort the neighbour lists");
    CGB_REQUIRE(g->servers.load() == 0, CGB_EINVAL, "weights cannot change while a server is attached to the graph");
    const uint32_t E = g->E;
    if (E == 0) return;
    CGB_CUDA_TRY(cudaSetDevice(g->device));
    cudaStream_t s = nullptr;
    CGB_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    uint32_t* w = nullptr;
    unsigned long long* sum = nullptr;
    PinnedArray<unsigned long long> hs(1);
    try {
        w = dalloc<uint32_t>(E, s);
        sum = dalloc<unsigned long long>(1, s);
        CGB_CUDA_TRY(cudaMemcpyAsync(w, weight, (size_t)E * 4, cudaMemcpyDefault, s));
        CGB_CUDA_TRY(cudaMemsetAsync(sum, 0, sizeof(unsigned long long), s));
        k_sum_u32<<<grid_for(E, kBlock, num_sms() * 8), kBlock, 0, s>>>(E, w, sum);
        CGB_CUDA_TRY(cudaMemcpyAsync(hs.data(), sum, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
        CGB_CUDA_TRY(cudaStreamSynchronize(s));
    } catch (...) {
        dfree(w, s);
        dfree(sum, s);
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
        throw;
    }
    dfree(sum, s);
    CGB_CUDA_TRY(cudaStreamSynchronize(s));
    CGB_CUDA_TRY(cudaStreamDestroy(s));
    uint32_t* replaced = nullptr;
    {
        std::lock_guard<std::mutex> pl(g->pending_mu);
        replaced = g->pending_w;  // weights set twice while the graph stayed busy
        g->pending_w = w;
        g->pending_sum_w = hs[0];
    }
    if (replaced) dfree(replaced, g->stream);
    if (g->mu.try_lock()) g->mu.unlock();  // idle graph: swapped in now
}

__global__ void k_compare_u32(uint64_t n, const uint32_t* __restrict__ a, const uint32_t* __restrict__ b,
                              uint32_t* differ)
{
    const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / 32;
    const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32;
    uint32_t k = 0;
    for (uint64_t base = w * 32; base < n; base += warps * 32, k++) {
        if ((k & 15u) == 0 && *(volatile uint32_t*)differ) return;
        const uint64_t i = base + lane_id();
        if (__any_sync(0xffffffffu, i < n && a[i] != b[i])) {
            if (lane_id() == 0) atomicOr(differ, 1u);
            return;
        }
    }
}

// off[v] = min{j : key[j] >= v} over keys sorted ascending, for v in
// [0, V] (off[V] = n): one lower-bound search per vertex.
__global__ void k_offsets_from_u32(uint32_t V, uint32_t n, const uint32_t* __restrict__ key, uint32_t* off)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v <= V; v += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = n;
        while (lo < hi) {
            const uint32_t mid = lo + (hi - lo) / 2;
            if (key[mid] < v) lo = mid + 1;
            else hi = mid;
        }
        off[v] = lo;
    }
}

__global__ void k_pack_u32x2(uint32_t n, const uint32_t* __restrict__ hi, const uint32_t* __restrict__ lo,
                             uint64_t* out)
{
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
        out[j] = ((uint64_t)hi[j] << 32) | lo[j];
}

__global__ void k_unpack_u32x2(uint32_t n, const uint64_t* __restrict__ in, uint32_t* hi, uint32_t* lo)
{
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const uint64_t x = in[j];
        hi[j] = (uint32_t)(x >> 32);
        lo[j] = (uint32_t)x;
    }
}

// Stable sort of (key, value) pairs by the key's low `bits` bits: vals_out
// receives the values in key order, keys_out the keys.
static void stable_sort_u32(cgb_graph* g, const uint32_t* keys_in, uint32_t* keys_out, const uint32_t* vals_in,
                            uint32_t* vals_out, uint32_t n, int bits)
{
    size_t tb = 0;
    CGB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys_in, keys_out, vals_in, vals_out, (uint64_t)n, 0,
                                                 bits, g->stream));
    void* temp = dalloc<char>(tb, g->stream);
    cudaError_t err = cub::DeviceRadixSort::SortPairs(temp, tb, keys_in, keys_out, vals_in, vals_out, (uint64_t)n, 0,
                                                      bits, g->stream);
    CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    dfree(temp, g->stream);
    CGB_CUDA_TRY(err);
}

// The transpose's source and (optionally) weight arrays: the CSR lists
// edges by ascending source, so a stable sort on the destination alone
// (32-bit keys over bits_for(V) bits) orders each in-list by source.
// dst_sorted receives the destinations in CSC order.
static void transpose_arrays(cgb_graph* g, uint32_t* dst_sorted, uint32_t* in_src, uint32_t* in_w)
{
    const uint32_t E = g->E, V = g->V;
    const uint32_t grid = grid_for(E, kBlock, num_sms() * 16);
    uint32_t* src = dalloc<uint32_t>(E, g->stream);
    launch_edges_by_row(g, V, E, g->off, RowOutF{src});
    if (!in_w) {
        stable_sort_u32(g, g->dst, dst_sorted, src, in_src, E, (int)bits_for(V));
    } else {
        // (source, weight) ride together as one 64-bit value: no gathers afterwards
        uint64_t* sw = dalloc<uint64_t>(E, g->stream);
        uint64_t* sw_sorted = dalloc<uint64_t>(E, g->stream);
        k_pack_u32x2<<<grid, kBlock, 0, g->stream>>>(E, src, g->w, sw);
        size_t tb = 0;
        CGB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tb, g->dst, dst_sorted, sw, sw_sorted, (uint64_t)E, 0,
                                                     (int)bits_for(V), g->stream));
        void* temp = dalloc<char>(tb, g->stream);
        cudaError_t err = cub::DeviceRadixSort::SortPairs(temp, tb, g->dst, dst_sorted, sw, sw_sorted, (uint64_t)E, 0,
                                                          (int)bits_for(V), g->stream);
        k_unpack_u32x2<<<grid, kBlock, 0, g->stream>>>(E, sw_sorted, in_src, in_w);
        CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
        dfree(temp, g->stream);
        dfree(sw, g->stream);
        dfree(sw_sorted, g->stream);
        CGB_CUDA_TRY(err);
    }
    CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    dfree(src, g->stream);
}

static void exclusive_sum_u32(cgb_graph* g, const uint32_t* in, uint32_t* out, uint64_t n)
{
    size_t tb = 0;
    CGB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, in, out, n, g->stream));
    void* temp = dalloc<char>(tb, g->stream);
    cudaError_t err = cub::DeviceScan::ExclusiveSum(temp, tb, in, out, n, g->stream);
    dfree(temp, g->stream);
    CGB_CUDA_TRY(err);
}

// Symmetry without a full transpose.  Lists are strictly ascending, so the
// entries of v below v are a prefix of its list and those above v a suffix;
// the lower triangle in CSR order is sorted by (v, u).  The graph is
// symmetric exactly when the upper-triangle edges (u, v), u < v, stably
// sorted by v, are the lower triangle: the same pairs (v, u) in the same
// order (a self-loop is its own mirror).  Only those edges are sorted.
__global__ void k_sym_counts(uint32_t V, const uint32_t* __restrict__ off, const uint32_t* __restrict__ dst,
                             uint32_t* lower, uint32_t* upper)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        const uint32_t beg = off[v], end = off[v + 1];
        uint32_t lo = beg, hi = end;  // first entry >= v
        while (lo < hi) {
            const uint32_t mid = lo + (hi - lo) / 2;
            if (dst[mid] < v) lo = mid + 1;
            else hi = mid;
        }
        lower[v] = lo - beg;
        upper[v] = end - lo - ((lo < end && dst[lo] == v) ? 1u : 0u);
    }
}

// The upper-triangle edges in CSR order: key = v, value = u; u's entries
// above u are the last upper[u] = uoff[u + 1] - uoff[u] of its list.
struct SymUpperF {
    static constexpr uint32_t kBatch = 1;
    __device__ __forceinline__ bool stop() const { return false; }
    __device__ __forceinline__ void tile_end() {}
    const uint32_t* __restrict__ dst;
    const uint32_t* __restrict__ uoff;
    uint32_t* __restrict__ key;
    uint32_t* __restrict__ val;
    struct Val {
        uint32_t d, pos;
    };
    __device__ __forceinline__ Val load(uint32_t e, uint32_t u, uint32_t, uint32_t end) const
    {
        const uint32_t a = __ldg(uoff + u), b = __ldg(uoff + u + 1);
        return Val{__ldg(dst + e), a + (e - (end - (b - a)))};
    }
    __device__ __forceinline__ void store(uint32_t, uint32_t u, uint32_t, uint32_t, Val x)
    {
        if (x.d > u) {
            key[x.pos] = x.d;
            val[x.pos] = u;
        }
    }
};

// Lower-triangle edge (v, d), d < v, the j-th of v's list, against position
// loff[v] + j of the sorted upper-triangle edges.
struct SymCompareF {
    static constexpr uint32_t kBatch = 1;
    const uint32_t* __restrict__ dst;
    const uint32_t* __restrict__ loff;
    const uint32_t* __restrict__ skey;
    const uint32_t* __restrict__ sval;
    uint32_t* differ;
    bool bad = false;  // this thread's mismatches since the last tile end
    __device__ __forceinline__ bool stop() const { return *(volatile const uint32_t*)differ != 0; }
    using Val = bool;
    __device__ __forceinline__ Val load(uint32_t e, uint32_t v, uint32_t beg, uint32_t) const
    {
        const uint32_t d = __ldg(dst + e);
        if (d >= v) return false;
        const uint32_t i = __ldg(loff + v) + (e - beg);
        return __ldg(skey + i) != v || __ldg(sval + i) != d;
    }
    __device__ __forceinline__ void store(uint32_t, uint32_t, uint32_t, uint32_t, Val x) { bad |= x; }
    __device__ __forceinline__ void tile_end()
    {
        if (__any_sync(0xffffffffu, bad) && lane_id() == 0) atomicOr(differ, 1u);
        bad = false;
    }
};

static bool check_symmetric(cgb_graph* g)
{
    const uint32_t V = g->V, E = g->E;
    if (E == 0) return true;
    uint32_t* lower = dalloc<uint32_t>((size_t)V + 1, g->stream);
    uint32_t* upper = dalloc<uint32_t>((size_t)V + 1, g->stream);
    uint32_t* loff = dalloc<uint32_t>((size_t)V + 1, g->stream);
    uint32_t* uoff = dalloc<uint32_t>((size_t)V + 1, g->stream);
    CGB_CUDA_TRY(cudaMemsetAsync(lower + V, 0, 4, g->stream));
    CGB_CUDA_TRY(cudaMemsetAsync(upper + V, 0, 4, g->stream));
    k_sym_counts<<<grid_for(V, kBlock, num_sms() * 8), kBlock, 0, g->stream>>>(V, g->off, g->dst, lower, upper);
    exclusive_sum_u32(g, lower, loff, (uint64_t)V + 1);
    exclusive_sum_u32(g, upper, uoff, (uint64_t)V + 1);
    PinnedArray<uint32_t> tot(2);
    CGB_CUDA_TRY(cudaMemcpyAsync(&tot[0], loff + V, 4, cudaMemcpyDeviceToHost, g->stream));
    CGB_CUDA_TRY(cudaMemcpyAsync(&tot[1], uoff + V, 4, cudaMemcpyDeviceToHost, g->stream));
    CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    dfree(lower, g->stream);
    dfree(upper, g->stream);
    bool sym = tot[0] == tot[1];
    if (sym && tot[1] > 0) {
        const uint32_t n = tot[1];
        uint32_t* key = dalloc<uint32_t>(n, g->stream);
        uint32_t* val = dalloc<uint32_t>(n, g->stream);
        uint32_t* skey = dalloc<uint32_t>(n, g->stream);
        uint32_t* sval = dalloc<uint32_t>(n, g->stream);
        uint32_t* differ = dalloc<uint32_t>(1, g->stream);
        launch_edges_by_row(g, V, E, g->off, SymUpperF{g->dst, uoff, key, val});
        stable_sort_u32(g, key, skey, val, sval, n, (int)bits_for(V));
        dfree(key, g->stream);
        dfree(val, g->stream);
        CGB_CUDA_TRY(cudaMemsetAsync(differ, 0, 4, g->stream));
        launch_edges_by_row(g, V, E, g->off, SymCompareF{g->dst, loff, skey, sval, differ});
        PinnedArray<uint32_t> h(1);
        CGB_CUDA_TRY(cudaMemcpyAsync(h.data(), differ, 4, cudaMemcpyDeviceToHost, g->stream));
        CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
        sym = h[0] == 0;
        dfree(skey, g->stream);
        dfree(sval, g->stream);
        dfree(differ, g->stream);
    }
    dfree(loff, g->stream);
    dfree(uoff, g->stream);
    return sym;
}

// Builds the transpose (in-edge CSC) by a radix sort of packed (dst, src)
// keys and compares it with the CSR: equal means the graph is symmetric, the
// transpose is dropped and the CSR serves both directions.
static void build_transpose(cgb_graph* g)
{
    const uint32_t V = g->V, E = g->E;
    uint32_t* in_off = dalloc<uint32_t>((size_t)V + 1, g->stream);
    uint32_t* in_src = dalloc<uint32_t>(E, g->stream);
    if (E == 0) {
        CGB_CUDA_TRY(cudaMemsetAsync(in_off, 0, ((size_t)V + 1) * sizeof(uint32_t), g->stream));
    } else {
        uint32_t* dsorted = dalloc<uint32_t>(E, g->stream);
        // weights in CSC order are built on first need (ensure_csc_weights)
        transpose_arrays(g, dsorted, in_src, nullptr);
        k_offsets_from_u32<<<grid_for((uint64_t)V + 1, kBlock, num_sms() * 16), kBlock, 0, g->stream>>>(V, E, dsorted,
                                                                                                      in_off);
        CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
        dfree(dsorted, g->stream);
    }
    uint32_t* differ = dalloc<uint32_t>(1, g->stream);
    CGB_CUDA_TRY(cudaMemsetAsync(differ, 0, sizeof(uint32_t), g->stream));
    k_compare_u32<<<num_sms() * 8, kBlock, 0, g->stream>>>((uint64_t)V + 1, in_off, g->off, differ);
    if (E) k_compare_u32<<<num_sms() * 8, kBlock, 0, g->stream>>>(E, in_src, g->dst, differ);
    PinnedArray<uint32_t> h(1);
    CGB_CUDA_TRY(cudaMemcpyAsync(h.data(), differ, 4, cudaMemcpyDeviceToHost, g->stream));
    CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    dfree(differ, g->stream);
    if (h[0]) {
        g->symmetric = 0;
        g->in_off = in_off;
        g->in_src = in_src;
        g->csc_owned = true;
    } else {
        g->symmetric = 1;
        dfree(in_off, g->stream);
        dfree(in_src, g->stream);
        g->in_off = g->off;
        g->in_src = g->dst;
        g->csc_owned = false;
    }
}

// The half-size check above; the transpose itself is built only when a run
// needs the in-edges (ensure_csc).
void ensure_symmetry_known(cgb_graph* g)
{
    if (g->symmetric >= 0) return;
    g->symmetric = check_symmetric(g) ? 1 : 0;
}

void ensure_csc(cgb_graph* g)
{
    if (g->in_off) return;
    if (g->symmetric == 1) {
        g->in_off = g->off;
        g->in_src = g->dst;
        g->csc_owned = false;
        return;
    }
    build_transpose(g);
}

void ensure_csc_weights(cgb_graph* g)
{
    if (!g->w || g->in_w) return;
    ensure_csc(g);
    // transpose the weights: a stable sort by destination lists every
    // in-list by source, the order of in_src; alias w when the result equals
    // it (a symmetric graph with symmetric weights)
    const uint32_t E = g->E;
    if (E == 0) {
        g->in_w = g->w;
        g->in_w_owned = false;
        return;
    }
    uint32_t* dsorted = dalloc<uint32_t>(E, g->stream);
    uint32_t* srcs = dalloc<uint32_t>(E, g->stream);
    uint32_t* vals = dalloc<uint32_t>(E, g->stream);
    transpose_arrays(g, dsorted, srcs, vals);
    dfree(dsorted, g->stream);
    dfree(srcs, g->stream);
    uint32_t* differ = dalloc<uint32_t>(1, g->stream);
    CGB_CUDA_TRY(cudaMemsetAsync(differ, 0, 4, g->stream));
    k_compare_u32<<<num_sms() * 8, kBlock, 0, g->stream>>>(E, vals, g->w, differ);
    PinnedArray<uint32_t> h(1);
    CGB_CUDA_TRY(cudaMemcpyAsync(h.data(), differ, 4, cudaMemcpyDeviceToHost, g->stream));
    CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    dfree(differ, g->stream);
    if (h[0]) {
        g->in_w = vals;
        g->in_w_owned = true;
    } else {
        dfree(vals, g->stream);
        g->in_w = g->w;
        g->in_w_owned = false;
    }
}

void ensure_frontier(cgb_graph* g)
{
    if (g->q[0]) return;
    const uint32_t V = g->V;
    g->q[0] = dalloc<uint32_t>(V, g->stream);
    g->q[1] = dalloc<uint32_t>(V, g->stream);
    // any frontier (each vertex once): sum over lists >= big_deg of ceil(deg / chunk)
    // <= E / chunk + E / big_deg, at the smallest sizes launch_push uses (kMinChunk;
    // big_deg 32 for small frontiers, else at least kMinBigDeg)
    g->chunk_cap = (uint32_t)std::min<uint64_t>((uint64_t)g->E / kMinChunk + g->E / 32 + 64, 0xFFFFFFF0ull);
    g->chunk_q = dalloc<uint2>(g->chunk_cap, g->stream);
    g->visited = dalloc<uint32_t>(g->words(), g->stream);
    g->front_bm = dalloc<uint32_t>(2 * (size_t)g->words(), g->stream);
    g->stamp = dalloc<uint32_t>(V, g->stream);
    g->sample = dalloc<uint32_t>(1024, g->stream);
    g->aux_bm = dalloc<uint32_t>(3 * (size_t)g->words(), g->stream);
    ensure_max_degree(g);
}

void ensure_max_degree(cgb_graph* g)
{
    if (g->max_degree || g->E == 0) return;
    uint32_t* d = dalloc<uint32_t>(1, g->stream);
    CGB_CUDA_TRY(cudaMemsetAsync(d, 0, 4, g->stream));
    k_max_degree<<<grid_for(g->V, kBlock, num_sms() * 8), kBlock, 0, g->stream>>>(g->V, g->off, d);
    PinnedArray<uint32_t> md(1);
    CGB_CUDA_TRY(cudaMemcpyAsync(md.data(), d, 4, cudaMemcpyDeviceToHost, g->stream));
    CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    g->max_degree = md[0];
    dfree(d, g->stream);
}

__global__ void k_in_degree_from_off(uint32_t V, const uint32_t* __restrict__ in_off, uint32_t* indeg)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x)
        indeg[v] = in_off[v + 1] - in_off[v];
}

// Sort key of a vertex for the PageRank layout: its out-degree bucket
// (0 for the largest lists, 32 for none) in the top 6 bits, then its
// in-degree descending (clamped to 26 bits).
__global__ void k_pr_bucket(uint32_t V, const uint32_t* __restrict__ off, const uint32_t* __restrict__ indeg,
                            uint32_t* key, uint32_t* id)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        const uint32_t od = off[v + 1] - off[v];
        const uint32_t bucket = od ? (uint32_t)__clz(od) : 32u;
        const uint32_t in = min(indeg[v], (1u << 26) - 1);
        key[v] = (bucket << 26) | ((1u << 26) - 1 - in);
        id[v] = v;
    }
}

// Slice lengths of the sliced ELL: the longest non-hub row of each slice.
__global__ void k_sell_len(uint32_t V, const uint32_t* __restrict__ off, uint32_t hub, uint32_t* len, uint64_t* width)
{
    const uint32_t nslices = (V + 31) / 32;
    for (uint32_t s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < nslices;
         s += (gridDim.x * blockDim.x) >> 5) {
        const uint32_t r = s * 32 + lane_id();
        uint32_t d = r < V ? off[r + 1] - off[r] : 0;
        if (d >= hub) d = 0;
        d = warp_max(d);
        if (lane_id() == 0) {
            len[s] = d;
            width[s] = 32ull * d;
        }
    }
}

__global__ void k_pr_rank(uint32_t V, const uint32_t* __restrict__ order, const uint32_t* __restrict__ off,
                          uint32_t* rank, uint32_t* outdeg_new)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) {
        const uint32_t v = order[i];
        rank[v] = i;
        outdeg_new[i] = off[v + 1] - off[v];
    }
}

__global__ void k_row_bounds(const uint32_t* __restrict__ rows, uint32_t n, const uint32_t* __restrict__ off,
                             uint32_t* lohi)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        lohi[i] = off[rows[i]];
        lohi[n + i] = off[rows[i] + 1];
    }
}

// Edges of the relabelled graph in new-source order: position p of the
// out-list of order[r] (r = new source, its list at [beg, end) of the
// relabelled out-offsets) gives key = new destination and value = r; a
// stable sort by key then lists each new row's sources in ascending new ids.
struct PrEdgesF {
    static constexpr uint32_t kBatch = 8;
    __device__ __forceinline__ bool stop() const { return false; }
    __device__ __forceinline__ void tile_end() {}
    const uint32_t* __restrict__ order;
    const uint32_t* __restrict__ off;
    const uint32_t* __restrict__ dst;
    const uint32_t* __restrict__ rank;
    uint32_t* __restrict__ key;
    uint32_t* __restrict__ val;
    using Val = uint32_t;
    __device__ __forceinline__ Val load(uint32_t p, uint32_t r, uint32_t beg, uint32_t) const
    {
        return __ldg(rank + __ldg(dst + __ldg(off + __ldg(order + r)) + (p - beg)));
    }
    __device__ __forceinline__ void store(uint32_t p, uint32_t r, uint32_t, uint32_t, Val k)
    {
        key[p] = k;
        val[p] = r;
    }
};

// SELL columns from the relabelled CSC, one warp per 32-row slice, lane i
// on row 32s + i: column j of the slice is 32 consecutive words, so every
// store is coalesced, and each lane reads its own row front to back.
// Positions past a row's end hold the padding target V; hub rows (hub
// in-edges or more) are summed from pr_src instead, keep only padding here
// and are marked in hub_bm (one word per slice, written whole).
__global__ void k_sell_fill(uint32_t V, const uint32_t* __restrict__ pr_off, const uint32_t* __restrict__ pr_src,
                            const uint64_t* __restrict__ slice_ptr, const uint32_t* __restrict__ slice_len,
                            uint32_t hub, uint32_t* col, uint32_t* hub_bm)
{
    const uint32_t nslices = (V + 31) / 32;
    const uint32_t lane = lane_id();
    for (uint32_t sl = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; sl < nslices;
         sl += (gridDim.x * blockDim.x) >> 5) {
        const uint32_t r = sl * 32 + lane;
        const uint32_t beg = r < V ? pr_off[r] : 0;
        const uint32_t len = r < V ? pr_off[r + 1] - beg : 0;
        const bool is_hub = len >= hub;
        const uint32_t hubs = __ballot_sync(0xffffffffu, is_hub);
        if (lane == 0) hub_bm[sl] = hubs;
        const uint32_t use = is_hub ? 0 : len;
        uint32_t* c = col + slice_ptr[sl] + lane;
        const uint32_t width = slice_len[sl];
        for (uint32_t j = 0; j < width; j++) c[32ull * j] = j < use ? pr_src[beg + j] : V;
    }
}

// Sliced ELL layout of the non-hub rows (slice lengths, offsets and the
// column array); k_sell_fill writes the columns and their padding.
static void build_sell(cgb_graph* g)
{
    const uint32_t V = g->V;
    const uint32_t nslices = (V + 31) / 32;
    g->pr_slice_len = dalloc<uint32_t>(nslices, g->stream);
    g->pr_slice_ptr = dalloc<uint64_t>((size_t)nslices + 1, g->stream);
    g->pr_hub_bm = dalloc<uint32_t>(g->words(), g->stream);
    CGB_CUDA_TRY(cudaMemsetAsync(g->pr_hub_bm, 0, (size_t)g->words() * 4, g->stream));
    uint64_t* width = dalloc<uint64_t>((size_t)nslices + 1, g->stream);
    CGB_CUDA_TRY(cudaMemsetAsync(width + nslices, 0, 8, g->stream));
    k_sell_len<<<grid_for((uint64_t)nslices * 32, kBlock, num_sms() * 8), kBlock, 0, g->stream>>>(
        V, g->pr_off, kPrHuge, g->pr_slice_len, width);
    size_t tb = 0;
    CGB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, width, g->pr_slice_ptr, (uint64_t)nslices + 1, g->stream));
    void* temp = dalloc<char>(tb, g->stream);
    cudaError_t err =
        cub::DeviceScan::ExclusiveSum(temp, tb, width, g->pr_slice_ptr, (uint64_t)nslices + 1, g->stream);
    PinnedArray<uint64_t> tp(1);
    CGB_CUDA_TRY(cudaMemcpyAsync(tp.data(), g->pr_slice_ptr + nslices, 8, cudaMemcpyDeviceToHost, g->stream));
    CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    const uint64_t total = tp[0];
    dfree(temp, g->stream);
    dfree(width, g->stream);
    CGB_CUDA_TRY(err);
    g->pr_sell_size = total;
    g->pr_col = dalloc<uint32_t>(total, g->stream);
}

// Builds the PageRank layout (see cgb_graph): the relabel keeps every
// gathered contribution (vertices with out-edges) in one dense prefix of
// the contrib array, and groups rows of similar size.
void ensure_pr(cgb_graph* g)
{
    if (g->pr_ready) return;
    const uint32_t V = g->V, E = g->E;
    for (int i = 0; i < 2; i++) {
        if (!g->pr[i]) g->pr[i] = dalloc<double>(V, g->stream);
        if (!g->contrib[i]) g->contrib[i] = dalloc<double>((size_t)V + 1, g->stream);
        CGB_CUDA_TRY(cudaMemsetAsync(g->contrib[i] + V, 0, sizeof(double), g->stream));  // padding target
    }
    g->pr_rank = dalloc<uint32_t>(V, g->stream);
    g->pr_outdeg = dalloc<uint32_t>(V, g->stream);
    g->pr_off = dalloc<uint32_t>((size_t)V + 1, g->stream);
    g->pr_src = dalloc<uint32_t>(E, g->stream);
    // 1. stable order by (out-degree bucket, in-degree descending)
    uint32_t* order = nullptr;
    {
        uint32_t* key = dalloc<uint32_t>(V, g->stream);
        uint32_t* key2 = dalloc<uint32_t>(V, g->stream);
        uint32_t* id = dalloc<uint32_t>(V, g->stream);
        uint32_t* id2 = dalloc<uint32_t>(V, g->stream);
        // in-degrees from the transpose (shared with bottom-up BFS; no atomics)
        ensure_csc(g);
        k_in_degree_from_off<<<grid_for(V, kBlock, num_sms() * 8), kBlock, 0, g->stream>>>(V, g->in_off, key2);
        k_pr_bucket<<<grid_for(V, kBlock, num_sms() * 8), kBlock, 0, g->stream>>>(V, g->off, key2, key, id);
        cub::DoubleBuffer<uint32_t> kb(key, key2), vb(id, id2);
        size_t tb = 0;
        CGB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tb, kb, vb, (uint64_t)V, 0, 32, g->stream));
        void* temp = dalloc<char>(tb, g->stream);
        cudaError_t err = cub::DeviceRadixSort::SortPairs(temp, tb, kb, vb, (uint64_t)V, 0, 32, g->stream);
        k_pr_rank<<<grid_for(V, kBlock, num_sms() * 8), kBlock, 0, g->stream>>>(V, vb.Current(), g->off, g->pr_rank,
                                                                             g->pr_outdeg);
        CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
        dfree(temp, g->stream);
        dfree(key, g->stream);
        dfree(key2, g->stream);
        CGB_CUDA_TRY(err);
        order = vb.Current();
        dfree(vb.Alternate(), g->stream);
    }
    // 2. in-edge CSC over the new ids: the edges enumerated by new source,
    //    stable-sorted by new destination (one 32-bit sort), so each row
    //    lists its sources in ascending new ids
    {
        // offsets of the new sources' out-lists: exclusive scan of the out-degrees in new order
        // (pr_outdeg has V entries; the scan of V + 1 reads a zero-padded copy)
        uint32_t* src_off = dalloc<uint32_t>((size_t)V + 1, g->stream);
        uint32_t* od = dalloc<uint32_t>((size_t)V + 1, g->stream);
        CGB_CUDA_TRY(cudaMemcpyAsync(od, g->pr_outdeg, (size_t)V * 4, cudaMemcpyDeviceToDevice, g->stream));
        CGB_CUDA_TRY(cudaMemsetAsync(od + V, 0, 4, g->stream));
        size_t tb = 0;
        CGB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, od, src_off, (uint64_t)V + 1, g->stream));
        void* temp = dalloc<char>(tb, g->stream);
        cudaError_t err = cub::DeviceScan::ExclusiveSum(temp, tb, od, src_off, (uint64_t)V + 1, g->stream);
        CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
        dfree(temp, g->stream);
        dfree(od, g->stream);
        CGB_CUDA_TRY(err);
        if (E) {
            uint32_t* key = dalloc<uint32_t>(E, g->stream);
            uint32_t* val = dalloc<uint32_t>(E, g->stream);
            uint32_t* kout = dalloc<uint32_t>(E, g->stream);
            launch_edges_by_row(g, V, E, src_off, PrEdgesF{order, g->off, g->dst, g->pr_rank, key, val});
            stable_sort_u32(g, key, kout, val, g->pr_src, E, (int)bits_for(V));
            k_offsets_from_u32<<<grid_for((uint64_t)V + 1, kBlock, num_sms() * 16), kBlock, 0, g->stream>>>(
                V, E, kout, g->pr_off);
            CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
            dfree(key, g->stream);
            dfree(val, g->stream);
            dfree(kout, g->stream);
        } else {
            CGB_CUDA_TRY(cudaMemsetAsync(g->pr_off, 0, ((size_t)V + 1) * 4, g->stream));
        }
        dfree(src_off, g->stream);
        build_sell(g);
        if (E)
            k_sell_fill<<<grid_for((uint64_t)(V + 31) / 32 * 32, kBlock, num_sms() * 16), kBlock, 0, g->stream>>>(
                V, g->pr_off, g->pr_src, g->pr_slice_ptr, g->pr_slice_len, kPrHuge, g->pr_col, g->pr_hub_bm);
        CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
        dfree(order, g->stream);
    }
    // 3. hub rows and their chunk table (host-built; few rows)
    {
        uint32_t* n = dalloc<uint32_t>(1, g->stream);
        uint32_t* rows = dalloc<uint32_t>(V, g->stream);
        CGB_CUDA_TRY(cudaMemsetAsync(n, 0, sizeof(uint32_t), g->stream));
        k_collect_heavy_rows<<<grid_for(V, kBlock, num_sms() * 8), kBlock, 0, g->stream>>>(V, g->pr_off, kPrHuge, rows,
                                                                                        n);
        PinnedArray<uint32_t> hn(1);
        CGB_CUDA_TRY(cudaMemcpyAsync(hn.data(), n, 4, cudaMemcpyDeviceToHost, g->stream));
        CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
        const uint32_t h = hn[0];
        dfree(n, g->stream);
        // pinned staging for every transfer here (see pinned_acquire, h2d_small)
        PinnedArray<uint32_t> hrows(std::max<uint32_t>(h, 1)), lohi_h(2 * (size_t)std::max<uint32_t>(h, 1));
        if (h) {
            CGB_CUDA_TRY(cudaMemcpyAsync(hrows.data(), rows, h * 4ull, cudaMemcpyDeviceToHost, g->stream));
            CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
            std::sort(hrows.data(), hrows.data() + h);
            h2d_small(rows, hrows.data(), h * 4ull, g->stream);
            uint32_t* lohi = dalloc<uint32_t>(2ull * h, g->stream);
            k_row_bounds<<<grid_for(h, kBlock, num_sms() * 8), kBlock, 0, g->stream>>>(rows, h, g->pr_off, lohi);
            CGB_CUDA_TRY(cudaMemcpyAsync(lohi_h.data(), lohi, 2ull * h * 4, cudaMemcpyDeviceToHost, g->stream));
            CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
            dfree(lohi, g->stream);
        }
        uint64_t nch = 0;
        for (uint32_t i = 0; i < h; i++) nch += (lohi_h[h + i] - lohi_h[i] + kPrChunk - 1) / kPrChunk;
        PinnedArray<uint2> chunks(std::max<uint64_t>(nch, 1));
        PinnedArray<uint32_t> base(h + 1);
        uint32_t c = 0;
        for (uint32_t i = 0; i < h; i++) {
            base[i] = c;
            for (uint32_t e = lohi_h[i]; e < lohi_h[h + i]; e += kPrChunk) chunks[c++] = make_uint2(hrows[i], e);
        }
        base[h] = c;
        g->n_pr_huge = h;
        g->n_pr_chunks = c;
        g->pr_huge_rows = rows;
        g->pr_chunk_base = dalloc<uint32_t>(h + 1, g->stream);
        h2d_small(g->pr_chunk_base, base.data(), (h + 1) * 4ull, g->stream);
        g->pr_chunks = dalloc<uint2>(c, g->stream);
        if (c)
            h2d_small(g->pr_chunks, chunks.data(), (size_t)c * sizeof(uint2), g->stream);
        CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));  // the pinned tables go out of scope
        g->pr_part = dalloc<double>(c, g->stream);
    }
    g->pr_ready = true;
}

void count_reached(cgb_graph* g)
{
    CGB_CUDA_TRY(cudaMemsetAsync(&g->ctr->reached_edges, 0, sizeof(unsigned long long), g->stream));
    CGB_CUDA_TRY(cudaMemsetAsync(&g->ctr->reached, 0, sizeof(uint32_t), g->stream));
    k_count_reached<<<grid_for(g->V, kBlock, num_sms() * 8), kBlock, 0, g->stream>>>(g->V, g->value, g->off, g->ctr);
    sync_counters(g);
    g->stats.reached = g->h_ctr->reached;
    g->stats.traversed_edges = g->h_ctr->reached_edges;
}

// --------------------------------------------------------------- timers
void ktimer_begin(cgb_graph* g, int cls)
{
    if (g->kev_used + 2 > g->kev.size()) {
        for (int i = 0; i < 64; i++) {
            cudaEvent_t e;
            CGB_CUDA_TRY(cudaEventCreate(&e));
            g->kev.push_back(e);
        }
    }
    CGB_CUDA_TRY(cudaEventRecord(g->kev[g->kev_used], g->stream));
    g->kev_class.push_back(cls);
    g->kev_used += 2;
}

void ktimer_end(cgb_graph* g) { CGB_CUDA_TRY(cudaEventRecord(g->kev[g->kev_used - 1], g->stream)); }

void ktimer_collect(cgb_graph* g)
{
    for (size_t i = 0; i < g->kev_class.size(); i++) {
        float ms = 0.f;
        CGB_CUDA_TRY(cudaEventElapsedTime(&ms, g->kev[2 * i], g->kev[2 * i + 1]));
        const int c = g->kev_class[i];
        g->stats.kernel_ms[c] += ms;
        g->stats.kernel_launches[c] += 1;
    }
    g->kev_class.clear();
    g->kev_used = 0;
}

// --------------------------------------------------------------- lifetime
cgb_graph* graph_alloc(uint32_t V, uint32_t E, uint32_t nz, int device, bool with_weight)
{
    CGB_REQUIRE(V <= kMaxGraphSize && E <= kMaxGraphSize, CGB_EUNSUPPORTED, "V and E must be at most 2^32 - 2^24");
    CGB_CUDA_TRY(cudaSetDevice(device));
    cgb_graph* g = new cgb_graph();
    g->device = device;
    g->V = V;
    g->E = E;
    g->nz = (nz == 0 || nz > V) ? V : nz;
    try {
        CGB_CUDA_TRY(cudaStreamCreateWithFlags(&g->own_stream, cudaStreamNonBlocking));
        g->stream = g->own_stream;
        CGB_CUDA_TRY(cudaEventCreate(&g->ev_start));
        CGB_CUDA_TRY(cudaEventCreate(&g->ev_stop));
        CGB_CUDA_TRY(cudaEventCreate(&g->ev_iter[0]));
        CGB_CUDA_TRY(cudaEventCreate(&g->ev_iter[1]));
        g->ctr = dalloc<DevCounters>(1, g->stream);
        g->h_ctr = static_cast<DevCounters*>(pinned_small_alloc(sizeof(DevCounters)));
        CGB_CUDA_TRY(cudaMemsetAsync(g->ctr, 0, sizeof(DevCounters), g->stream));
        g->off = dalloc<uint32_t>((size_t)V + 1, g->stream);
        g->dst = dalloc<uint32_t>(E, g->stream);
        if (with_weight) g->w = dalloc<uint32_t>(E, g->stream);
        g->value = dalloc<uint32_t>(V, g->stream);
        // the buffers are stream-ordered allocations: complete them, so the
        // graph is usable on every stream from here on
        CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    } catch (...) {
        graph_free(g);
        throw;
    }
    return g;
}

cgb_graph* graph_shadow(cgb_graph* g)
{
    CGB_CUDA_TRY(cudaSetDevice(g->device));
    cgb_graph* sh = new cgb_graph();
    sh->device = g->device;
    sh->V = g->V;
    sh->E = g->E;
    sh->nz = g->nz;
    sh->off = g->off;
    sh->dst = g->dst;
    sh->w = g->w;
    sh->sum_w = g->sum_w;
    sh->max_degree = g->max_degree;
    sh->symmetric = g->symmetric;
    sh->lists_resorted = g->lists_resorted;
    // the in-edges too, when the graph has built them (borrowed as well)
    sh->in_off = g->in_off;
    sh->in_src = g->in_src;
    sh->csc_owned = false;
    sh->in_w = g->in_w;
    sh->in_w_owned = false;
    for (int a = 0; a < 4; a++) sh->tune_alg[a] = g->tune_alg[a];
    try {
        CGB_CUDA_TRY(cudaStreamCreateWithFlags(&sh->own_stream, cudaStreamNonBlocking));
        sh->stream = sh->own_stream;
        CGB_CUDA_TRY(cudaEventCreate(&sh->ev_start));
        CGB_CUDA_TRY(cudaEventCreate(&sh->ev_stop));
        CGB_CUDA_TRY(cudaEventCreate(&sh->ev_iter[0]));
        CGB_CUDA_TRY(cudaEventCreate(&sh->ev_iter[1]));
        sh->ctr = dalloc<DevCounters>(1, sh->stream);
        sh->h_ctr = static_cast<DevCounters*>(pinned_small_alloc(sizeof(DevCounters)));
        CGB_CUDA_TRY(cudaMemsetAsync(sh->ctr, 0, sizeof(DevCounters), sh->stream));
        sh->value = dalloc<uint32_t>(sh->V, sh->stream);
        CGB_CUDA_TRY(cudaStreamSynchronize(sh->stream));
    } catch (...) {
        graph_shadow_free(sh);
        throw;
    }
    return sh;
}

void graph_shadow_free(cgb_graph* sh)
{
    if (!sh) return;
    // borrowed from the graph it shadows (a CSC it built itself stays owned)
    if (!sh->csc_owned) sh->in_off = sh->in_src = nullptr;
    if (!sh->in_w_owned) sh->in_w = nullptr;
    sh->off = sh->dst = sh->w = nullptr;
    graph_free(sh);
}

void graph_free(cgb_graph* g)
{
    if (!g) return;
    cudaSetDevice(g->device);
    if (g->stream) cudaStreamSynchronize(g->stream);
    if (g->csc_owned) {
        dfree(g->in_off, g->stream);
        dfree(g->in_src, g->stream);
    }
    if (g->in_w_owned) dfree(g->in_w, g->stream);
    if (g->pending_w) dfree(g->pending_w, g->stream);
    free_msbfs(g);
    free_mssp(g);
    void* ptrs[] = {g->off, g->dst, g->w, g->pr_huge_rows, g->pr_rank, g->pr_off, g->pr_src, g->pr_outdeg,
                    g->pr_chunks, g->pr_chunk_base, g->pr_part, g->pr_slice_ptr, g->pr_slice_len, g->pr_col,
                    g->pr_hub_bm, g->value, g->pr[0], g->pr[1], g->contrib[0],
                    g->contrib[1], g->q[0], g->q[1], g->chunk_q, g->visited, g->front_bm, g->stamp, g->sample,
                    g->aux_bm, g->persist, g->ctr};
    for (void* p : ptrs) dfree(p, g->stream);
    pinned_small_free(g->h_ctr);
    pinned_release(g->h_persist, g->h_persist_bytes);
    for (cudaEvent_t e : g->kev) cudaEventDestroy(e);
    cudaEvent_t evs[] = {g->ev_start, g->ev_stop, g->ev_iter[0], g->ev_iter[1], g->ev_fork, g->ev_join};
    for (cudaEvent_t e : evs)
        if (e) cudaEventDestroy(e);
    if (g->aux_stream) cudaStreamDestroy(g->aux_stream);
    if (g->own_stream) cudaStreamDestroy(g->own_stream);
    delete g;
}

// ------------------------------------------------------------------ reorder
// Relabelled copies of a graph, the deterministic orders of the reference's
// Reorder (my_project/CGgraph/Reorder.hpp): vertices sorted by degree,
// largest first, ties by ascending id (sortDegree, :251-292).  IN_DEGREE_DEC
// sorts by in-degree (:211-240); NORMAL_OUTDEGREE_DEC by out-degree, which
// puts the vertices without out-edges last and gives noZeroOutDegreeNum
// (main_partition.hpp:78-104 reads it for that order).  new id = rank in the
// order, old2new[v] = new id of v.  The new CSR lists every row's
// neighbours by new id, weights following.

__global__ void k_degree_desc_key(uint32_t V, const uint32_t* __restrict__ off, uint32_t* key, uint32_t* id)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        key[v] = ~(off[v + 1] - off[v]);  // ascending key = descending degree
        id[v] = v;
    }
}

__global__ void k_reorder_rows(uint32_t V, const uint32_t* __restrict__ order, const uint32_t* __restrict__ off,
                               uint32_t* old2new, uint32_t* new_deg, uint32_t* nonzero)
{
    uint32_t nz = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) {
        const uint32_t u = order[i];
        old2new[u] = i;
        const uint32_t d = off[u + 1] - off[u];
        new_deg[i] = d;
        nz += d ? 1u : 0u;
    }
    nz = warp_sum(nz);
    if (lane_id() == 0 && nz) atomicAdd(nonzero, nz);
}

// Row r of the relabelled graph is the old row order[r]: its entries with
// their ids mapped, weights alongside.
struct ReorderRowsF {
    static constexpr uint32_t kBatch = 8;
    __device__ __forceinline__ bool stop() const { return false; }
    __device__ __forceinline__ void tile_end() {}
    const uint32_t* __restrict__ order;
    const uint32_t* __restrict__ off;
    const uint32_t* __restrict__ dst;
    const uint32_t* __restrict__ w;
    const uint32_t* __restrict__ old2new;
    uint32_t* __restrict__ new_dst;
    uint32_t* __restrict__ new_w;
    struct Val {
        uint32_t d, wt;
    };
    __device__ __forceinline__ Val load(uint32_t p, uint32_t r, uint32_t beg, uint32_t) const
    {
        const uint32_t e = __ldg(off + __ldg(order + r)) + (p - beg);
        return Val{__ldg(old2new + __ldg(dst + e)), w ? __ldg(w + e) : 0u};
    }
    __device__ __forceinline__ void store(uint32_t p, uint32_t, uint32_t, uint32_t, Val x)
    {
        new_dst[p] = x.d;
        if (new_w) new_w[p] = x.wt;
    }
};

// ---------------------------------------------------------- BFS-based orders
// The reference's MY_BFS_* orders (Reorder.hpp:294-535) run one queue BFS
// after another on the CPU: start vertices in start-list order (degree
// descending, ties by id), each popped vertex queueing its unvisited
// neighbours by child degree, largest first, the vertices without out-edges
// set aside in the order they are met.  The same sequence follows from three
// data-parallel facts.
//  1. The vertices with out-edges split into BFS trees: v belongs to the tree
//     of the lowest start-list rank r that reaches v (a vertex reaching v is
//     either a root or reached by a lower-ranked one), at depth
//     dist(root, v).  label = (r << 32 | depth) is the lexicographic minimum
//     over every vertex reaching v, the fixpoint of
//     label[v] = min(label[v], label[u] + 1) over edges u -> v from
//     label[v] = rank[v] << 32: one frontier round per depth.
//  2. The queue holds the trees by rank, each level by level, and a level in
//     the order of (queue index of the first parent that lists the vertex,
//     child degree descending, list index).  So level d+1 is built from
//     level d in queue order: every child is claimed by its lowest-index
//     parent, parents emit their claimed children in list order, and a
//     stable radix sort on (parent index, ~degree) orders them.  Level
//     indices order the vertices of one tree and level as queue positions
//     do, and across trees by tree rank.
//  3. Concatenated, the levels are in (depth, level index) order; a stable
//     sort on the tree rank turns that into the queue sequence.
// The vertices without out-edges follow in the order the reference appends
// them: at the first visit of a parent that lists them (by visit position,
// then list index), or, when no parent is visited before their own turn in
// the start list, at that turn, which falls after every tree of a lower
// rank.  Equal child degrees keep list order; the reference's std::sort
// does the same for lists of at most 16 entries and may permute ties in
// longer ones.

constexpr uint64_t kNoLabel = ~0ull;  // vertices without out-edges

__global__ void k_in_degree(uint32_t E, const uint32_t* __restrict__ dst, uint32_t* indeg)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < E; e += stride)
        atomicAdd(indeg + __ldg(dst + e), 1u);
}

// Ascending keys: start degree descending (ties keep id order through the
// stable sort), child degree descending (saturated to 32 bits; only one
// vertex can have 2^32 or more incident edges).
__global__ void k_bfs_order_keys(uint32_t V, const uint32_t* __restrict__ off, const uint32_t* __restrict__ indeg,
                                 int method, uint32_t* start_key, uint32_t* id, uint32_t* child_key)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += stride) {
        const uint32_t od = off[v + 1] - off[v], in = indeg[v];
        start_key[v] = ~(method == CGB_ORDER_MY_IMAX_BFS_IN ? in : od);
        id[v] = (uint32_t)v;
        const uint64_t cd = method == CGB_ORDER_MY_BFS_OUT      ? (uint64_t)od
                            : method == CGB_ORDER_MY_BFS_OUT_IN ? (uint64_t)od + in
                                                                : (uint64_t)in;
        child_key[v] = ~(uint32_t)(cd < 0xffffffffull ? cd : 0xffffffffull);
    }
}

// label and rank from the start list; the vertices with out-edges form the
// first frontier.  ctr[0] counts it, ctr[1] is the (unreachable) overflow.
__global__ void k_bfs_order_init(uint32_t V, const uint32_t* __restrict__ off, const uint32_t* __restrict__ start_list,
                                 uint64_t* label, uint32_t* rank, uint32_t* front, uint32_t* ctr)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i0 = blockIdx.x * (uint64_t)blockDim.x; i0 < V; i0 += stride) {  // warp-uniform trip count
        const uint64_t i = i0 + threadIdx.x;
        bool nz = false;
        uint32_t v = 0;
        if (i < V) {
            v = start_list[i];
            nz = off[v + 1] > off[v];
            label[v] = nz ? (i << 32) : kNoLabel;
            rank[v] = (uint32_t)i;
        }
        warp_append(nz, v, front, ctr, V, ctr + 1);
    }
}

// One round of label[v] = min(label[v], label[u] + 1), a warp per frontier
// vertex u.  A vertex lowered in this round joins the next frontier once
// (stamp).  A stale read of label[u] only delays: u was lowered in this
// round, so it is in the next frontier too.
__global__ void k_bfs_order_relax(const uint32_t* __restrict__ off, const uint32_t* __restrict__ dst, uint64_t* label,
                                  const uint32_t* __restrict__ front, uint32_t nfront, uint32_t* next, uint32_t* ctr,
                                  uint32_t* stamp, uint32_t round, uint32_t cap)
{
    const uint32_t lane = lane_id();
    const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / 32;
    for (uint64_t w = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) / 32; w < nfront; w += warps) {
        const uint32_t u = front[w];
        const uint64_t cand = label[u] + 1;
        const uint64_t end = off[u + 1];
        for (uint64_t e0 = off[u]; e0 < end; e0 += 32) {
            bool push = false;
            uint32_t v = 0;
            if (e0 + lane < end) {
                v = __ldg(dst + e0 + lane);
                const uint64_t cur = label[v];
                if (cur != kNoLabel && cand < cur) {
                    const uint64_t old = atomicMin((unsigned long long*)(label + v), (unsigned long long)cand);
                    push = cand < old && atomicExch(stamp + v, round) != round;
                }
            }
            warp_append(push, v, next, ctr, cap, ctr + 1);
        }
    }
}

// The roots (label == rank << 32) in rank order: flags for a compaction.
__global__ void k_bfs_order_root_flags(uint32_t V, const uint32_t* __restrict__ start_list,
                                       const uint64_t* __restrict__ label, uint32_t* flag)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < V; i += stride)
        flag[i] = label[start_list[i]] == (i << 32) ? 1u : 0u;
    if (blockIdx.x == 0 && threadIdx.x == 0) flag[V] = 0;
}

__global__ void k_scatter_flagged(uint32_t n, const uint32_t* __restrict__ flag, const uint32_t* __restrict__ idx,
                                  const uint32_t* __restrict__ item, uint32_t* out)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += stride)
        if (flag[i]) out[idx[i]] = item[i];
}

// Level d+1 from level d (P[0, n) in queue order), a warp per parent.  A
// child v of parent u has label[v] == label[u] + 1: the same tree, one level
// down.  claim: the lowest parent index wins; count: children per parent;
// emit: each parent's children in list order at start[i], with the sort key
// (parent index << 32 | ~child degree).
enum class LevelPass { kClaim, kCount, kEmit };

template <LevelPass kPass>
__global__ void k_bfs_order_level(const uint32_t* __restrict__ off, const uint32_t* __restrict__ dst,
                                  const uint64_t* __restrict__ label, const uint32_t* __restrict__ P, uint32_t n,
                                  uint32_t* par, uint32_t* cnt, const uint32_t* __restrict__ start,
                                  const uint32_t* __restrict__ child_key, uint32_t* C, uint64_t* K)
{
    const uint32_t lane = lane_id();
    const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / 32;
    for (uint64_t w = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) / 32; w < n; w += warps) {
        const uint32_t i = (uint32_t)w;
        const uint32_t u = P[i];
        const uint64_t t = label[u] + 1;
        const uint64_t end = off[u + 1];
        uint32_t c = 0;
        const uint32_t base = kPass == LevelPass::kEmit ? start[i] : 0u;
        for (uint64_t e0 = off[u]; e0 < end; e0 += 32) {
            bool mine = false;
            uint32_t v = 0;
            if (e0 + lane < end) {
                v = __ldg(dst + e0 + lane);
                if (label[v] == t) {
                    if (kPass == LevelPass::kClaim) {
                        if (par[v] > i) atomicMin(par + v, i);
                    } else {
                        mine = par[v] == i;
                    }
                }
            }
            if (kPass == LevelPass::kCount) {
                c += mine ? 1u : 0u;
            } else if (kPass == LevelPass::kEmit) {
                const uint32_t b = __ballot_sync(0xffffffffu, mine);
                if (mine) {
                    const uint32_t at = base + c + __popc(b & lanemask_lt());
                    C[at] = v;
                    K[at] = ((uint64_t)i << 32) | child_key[v];
                }
                c += __popc(b);
            }
        }
        if (kPass == LevelPass::kCount) {
            c = warp_sum(c);
            if (lane == 0) cnt[i] = c;
        }
    }
}

__global__ void k_bfs_order_tree_key(uint32_t n, const uint32_t* __restrict__ lv, const uint64_t* __restrict__ label,
                                     uint32_t* key)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n; j += stride)
        key[j] = (uint32_t)(label[lv[j]] >> 32);
}

// Vertices without out-edges: zp = lowest queue position of a parent that
// lists them (first pass), zj = their index in that parent's list (second).
template <bool kIndex>
__global__ void k_bfs_order_zero_parent(const uint32_t* __restrict__ off, const uint32_t* __restrict__ dst,
                                        const uint64_t* __restrict__ label, const uint32_t* __restrict__ order,
                                        uint32_t n, uint32_t* zp, uint32_t* zj)
{
    const uint32_t lane = lane_id();
    const uint64_t warps = (uint64_t)gridDim.x * blockDim.x / 32;
    for (uint64_t w = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) / 32; w < n; w += warps) {
        const uint32_t i = (uint32_t)w;
        const uint32_t u = order[i];
        const uint64_t beg = off[u], end = off[u + 1];
        for (uint64_t e = beg + lane; e < end; e += 32) {
            const uint32_t z = __ldg(dst + e);
            if (label[z] != kNoLabel) continue;
            if (kIndex) {
                if (zp[z] == i) zj[z] = (uint32_t)(e - beg);
            } else if (zp[z] > i) {
                atomicMin(zp + z, i);
            }
        }
    }
}

__global__ void k_bfs_order_zero_list(uint32_t V, const uint64_t* __restrict__ label, uint32_t* zl, uint32_t* ctr)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v0 = blockIdx.x * (uint64_t)blockDim.x; v0 < V; v0 += stride) {
        const uint64_t v = v0 + threadIdx.x;
        warp_append(v < V && label[v] == kNoLabel, (uint32_t)v, zl, ctr, V, ctr + 1);
    }
}

// Sort keys of the vertices without out-edges, met at (visit position zp,
// list index zj) or at their own start-list turn k, which comes after the
// P(k) queue positions of the trees ranked below k: hi = 2 zp + 1, lo = zj,
// or hi = 2 P(k), lo = k.
__global__ void k_bfs_order_zero_keys(uint32_t Z, const uint32_t* __restrict__ zl, const uint32_t* __restrict__ zp,
                                      const uint32_t* __restrict__ zj, const uint32_t* __restrict__ rank,
                                      const uint32_t* __restrict__ tree_sorted, uint32_t n, uint32_t* lo, uint64_t* hi)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < Z; i += stride) {
        const uint32_t z = zl[i], k = rank[z];
        uint32_t a = 0, b = n;  // first tree_sorted entry >= k
        while (a < b) {
            const uint32_t m = a + (b - a) / 2;
            if (tree_sorted[m] < k) a = m + 1;
            else b = m;
        }
        if (zp[z] < a) {
            hi[i] = 2ull * zp[z] + 1;
            lo[i] = zj[z];
        } else {
            hi[i] = 2ull * a;
            lo[i] = k;
        }
    }
}

static void sort_pairs_u64(cgb_graph* g, const uint64_t* kin, uint64_t* kout, const uint32_t* vin, uint32_t* vout,
                           uint64_t n, int bits)
{
    size_t tb = 0;
    CGB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tb, kin, kout, vin, vout, n, 0, bits, g->stream));
    void* temp = dalloc<char>(tb, g->stream);
    cudaError_t err = cub::DeviceRadixSort::SortPairs(temp, tb, kin, kout, vin, vout, n, 0, bits, g->stream);
    CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    dfree(temp, g->stream);
    CGB_CUDA_TRY(err);
}

// Pool allocations on the graph's stream, returned when the scope ends.
struct ScopedPool {
    cudaStream_t s;
    std::vector<void*> held;
    explicit ScopedPool(cudaStream_t st) : s(st) {}
    template <typename T>
    T* get(size_t n)
    {
        T* p = dalloc<T>(n ? n : 1, s);
        held.push_back(p);
        return p;
    }
    ~ScopedPool()
    {
        cudaStreamSynchronize(s);
        for (void* p : held) dfree(p, s);
    }
};

static uint32_t read_u32(cgb_graph* g, const uint32_t* d)
{
    PinnedArray<uint32_t> h(1);
    CGB_CUDA_TRY(cudaMemcpyAsync(h.data(), d, 4, cudaMemcpyDeviceToHost, g->stream));
    CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    return h[0];
}

// order[i] = old id of new vertex i; returns the number of vertices with
// out-edges (they come first).
static uint32_t bfs_vertex_order(cgb_graph* g, int method, uint32_t* order)
{
    const uint32_t V = g->V, E = g->E;
    cudaStream_t s = g->stream;
    ScopedPool pool(s);
    const uint32_t gv = grid_for(V, kBlock, num_sms() * 8);
    const uint32_t gw = num_sms() * 16;  // warp-per-vertex kernels
    uint32_t* indeg = pool.get<uint32_t>(V);
    uint32_t* skey = pool.get<uint32_t>(V);
    uint32_t* skey2 = pool.get<uint32_t>(V);
    uint32_t* ids = pool.get<uint32_t>(V);
    uint32_t* start_list = pool.get<uint32_t>(V);
    uint32_t* child_key = pool.get<uint32_t>(V);
    uint32_t* rank = pool.get<uint32_t>(V);
    uint64_t* label = pool.get<uint64_t>(V);
    uint32_t* fa = pool.get<uint32_t>(V);
    uint32_t* fb = pool.get<uint32_t>(V);
    uint32_t* stamp = pool.get<uint32_t>(V);
    uint32_t* par = pool.get<uint32_t>(V);
    uint32_t* ctr = pool.get<uint32_t>(2);
    uint32_t* lv = pool.get<uint32_t>(V);
    uint32_t* flag = pool.get<uint32_t>((size_t)V + 1);
    uint32_t* idx = pool.get<uint32_t>((size_t)V + 1);
    uint32_t* C = pool.get<uint32_t>(V);
    uint64_t* K = pool.get<uint64_t>(V);
    uint64_t* K2 = pool.get<uint64_t>(V);
    CGB_CUDA_TRY(cudaMemsetAsync(indeg, 0, (size_t)V * 4, s));
    if (E) k_in_degree<<<grid_for(E, kBlock, num_sms() * 8), kBlock, 0, s>>>(E, g->dst, indeg);
    k_bfs_order_keys<<<gv, kBlock, 0, s>>>(V, g->off, indeg, method, skey, ids, child_key);
    stable_sort_u32(g, skey, skey2, ids, start_list, V, 32);

    // 1. labels (tree rank << 32 | depth)
    CGB_CUDA_TRY(cudaMemsetAsync(ctr, 0, 8, s));
    k_bfs_order_init<<<gv, kBlock, 0, s>>>(V, g->off, start_list, label, rank, fa, ctr);
    uint32_t nfront = read_u32(g, ctr);
    const uint32_t n_out = nfront;  // vertices with out-edges
    CGB_CUDA_TRY(cudaMemsetAsync(stamp, 0, (size_t)V * 4, s));
    for (uint32_t round = 1; nfront; round++) {
        CGB_CUDA_TRY(cudaMemsetAsync(ctr, 0, 8, s));
        k_bfs_order_relax<<<grid_for((uint64_t)nfront * 32, kBlock, gw), kBlock, 0, s>>>(
            g->off, g->dst, label, fa, nfront, fb, ctr, stamp, round, V);
        nfront = read_u32(g, ctr);
        std::swap(fa, fb);
    }

    // 2. levels in queue order, concatenated into lv; level 0 = the roots by rank
    k_bfs_order_root_flags<<<gv, kBlock, 0, s>>>(V, start_list, label, flag);
    exclusive_sum_u32(g, flag, idx, (uint64_t)V + 1);
    k_scatter_flagged<<<gv, kBlock, 0, s>>>(V, flag, idx, start_list, lv);
    uint32_t n = read_u32(g, idx + V);
    uint64_t done = 0;
    uint32_t* cnt = flag;  // reused: n + 1 <= V + 1 entries
    uint32_t* start = idx;
    CGB_CUDA_TRY(cudaMemsetAsync(par, 0xff, (size_t)V * 4, s));
    while (n) {
        const uint32_t* P = lv + done;
        const uint32_t gl = grid_for((uint64_t)n * 32, kBlock, gw);
        k_bfs_order_level<LevelPass::kClaim><<<gl, kBlock, 0, s>>>(g->off, g->dst, label, P, n, par, nullptr,
                                                                    nullptr, nullptr, nullptr, nullptr);
        k_bfs_order_level<LevelPass::kCount><<<gl, kBlock, 0, s>>>(g->off, g->dst, label, P, n, par, cnt, nullptr,
                                                                    nullptr, nullptr, nullptr);
        CGB_CUDA_TRY(cudaMemsetAsync(cnt + n, 0, 4, s));
        exclusive_sum_u32(g, cnt, start, (uint64_t)n + 1);
        const uint32_t m = read_u32(g, start + n);
        CGB_REQUIRE(done + n + m <= n_out, CGB_EOVERFLOW, "BFS order: level sizes exceed the vertices with out-edges");
        if (m) {
            k_bfs_order_level<LevelPass::kEmit><<<gl, kBlock, 0, s>>>(g->off, g->dst, label, P, n, par, nullptr,
                                                                       start, child_key, C, K);
            sort_pairs_u64(g, K, K2, C, lv + done + n, m, 32 + (int)bits_for(n));
        }
        done += n;
        n = m;
    }
    CGB_REQUIRE(done == n_out, CGB_EOVERFLOW, "BFS order: a vertex with out-edges was not placed");

    // 3. queue sequence: the levels stably sorted by tree rank
    if (n_out) {
        k_bfs_order_tree_key<<<gv, kBlock, 0, s>>>(n_out, lv, label, skey);
        stable_sort_u32(g, skey, skey2, lv, order, n_out, (int)bits_for(V));
    }
    const uint32_t* tree_sorted = skey2;

    // 4. the vertices without out-edges
    const uint32_t Z = V - n_out;
    if (Z) {
        uint32_t* zp = par;
        uint32_t* zj = stamp;
        CGB_CUDA_TRY(cudaMemsetAsync(zp, 0xff, (size_t)V * 4, s));
        if (n_out) {
            const uint32_t gz = grid_for((uint64_t)n_out * 32, kBlock, gw);
            k_bfs_order_zero_parent<false><<<gz, kBlock, 0, s>>>(g->off, g->dst, label, order, n_out, zp, zj);
            k_bfs_order_zero_parent<true><<<gz, kBlock, 0, s>>>(g->off, g->dst, label, order, n_out, zp, zj);
        }
        CGB_CUDA_TRY(cudaMemsetAsync(ctr, 0, 8, s));
        k_bfs_order_zero_list<<<gv, kBlock, 0, s>>>(V, label, fa, ctr);
        CGB_REQUIRE(read_u32(g, ctr) == Z, CGB_EOVERFLOW, "BFS order: vertex count without out-edges");
        // (hi, lo) pairs are distinct: sort by lo, then stably by hi
        k_bfs_order_zero_keys<<<gv, kBlock, 0, s>>>(Z, fa, zp, zj, rank, tree_sorted, n_out, fb, K);
        stable_sort_u32(g, fb, cnt, fa, C, Z, 32);
        k_bfs_order_zero_keys<<<gv, kBlock, 0, s>>>(Z, C, zp, zj, rank, tree_sorted, n_out, fb, K);
        sort_pairs_u64(g, K, K2, C, order + n_out, Z, (int)bits_for(2ull * n_out + 2));
    }
    CGB_CUDA_TRY(cudaStreamSynchronize(s));
    return n_out;
}

cgb_graph* graph_reorder(cgb_graph* g, int method, uint32_t* old2new_out, uint32_t* nz_out)
{
    const bool bfs = method == CGB_ORDER_MY_BFS_OUT || method == CGB_ORDER_MY_BFS_IN ||
                     method == CGB_ORDER_MY_BFS_OUT_IN || method == CGB_ORDER_MY_IMAX_BFS_IN;
    CGB_REQUIRE(method == CGB_ORDER_IN_DEGREE_DEC || method == CGB_ORDER_NORMAL_OUTDEGREE_DEC || bfs,
                CGB_EUNSUPPORTED,
                "order method: IN_DEGREE_DEC (21), NORMAL_OUTDEGREE_DEC (12) and the BFS orders "
                "MY_BFS_OUT (16), MY_BFS_IN (17), MY_BFS_OUT_IN (18), MY_IMAX_BFS_IN (20) are built");
    const uint32_t V = g->V, E = g->E;
    const bool by_in = method == CGB_ORDER_IN_DEGREE_DEC;
    if (by_in) ensure_csc(g);
    const uint32_t* deg_off = by_in ? g->in_off : g->off;
    cudaStream_t s = g->stream;
    uint32_t* key = dalloc<uint32_t>(V, s);
    uint32_t* key2 = dalloc<uint32_t>(V, s);
    uint32_t* id = dalloc<uint32_t>(V, s);
    uint32_t* order = dalloc<uint32_t>(V, s);
    uint32_t* old2new = dalloc<uint32_t>(V, s);
    uint32_t* new_deg = dalloc<uint32_t>((size_t)V + 1, s);
    uint32_t* nonzero = dalloc<uint32_t>(1, s);
    if (bfs) {
        bfs_vertex_order(g, method, order);  // vertices with out-edges first
    } else {
        k_degree_desc_key<<<grid_for(V, kBlock, num_sms() * 8), kBlock, 0, s>>>(V, deg_off, key, id);
        stable_sort_u32(g, key, key2, id, order, V, 32);
    }
    CGB_CUDA_TRY(cudaMemsetAsync(nonzero, 0, 4, s));
    CGB_CUDA_TRY(cudaMemsetAsync(new_deg + V, 0, 4, s));
    k_reorder_rows<<<grid_for(V, kBlock, num_sms() * 8), kBlock, 0, s>>>(V, order, g->off, old2new, new_deg, nonzero);
    PinnedArray<uint32_t> hn(1);
    CGB_CUDA_TRY(cudaMemcpyAsync(hn.data(), nonzero, 4, cudaMemcpyDeviceToHost, s));
    CGB_CUDA_TRY(cudaStreamSynchronize(s));
    // out-degree and BFS orders: every vertex with out-edges comes before every one without
    const uint32_t nz = by_in ? V : hn[0];
    cgb_graph* r = nullptr;
    try {
        r = graph_alloc(V, E, nz, g->device, g->w != nullptr && E > 0);
        exclusive_sum_u32(g, new_deg, r->off, (uint64_t)V + 1);
        CGB_CUDA_TRY(cudaStreamSynchronize(s));
        launch_edges_by_row(g, V, E, r->off, ReorderRowsF{order, g->off, g->dst, g->w, old2new, r->dst, r->w});
        if (old2new_out)
            CGB_CUDA_TRY(cudaMemcpyAsync(old2new_out, old2new, (size_t)V * 4, cudaMemcpyDefault, s));
        CGB_CUDA_TRY(cudaStreamSynchronize(s));
        validate_and_sort(r);  // lists sorted by new id, weights following
        compute_weight_sum(r);
    } catch (...) {
        cudaStreamSynchronize(s);
        for (void* p : {(void*)key, (void*)key2, (void*)id, (void*)order, (void*)old2new, (void*)new_deg, (void*)nonzero})
            dfree(p, s);
        if (r) graph_free(r);
        throw;
    }
    for (void* p : {(void*)key, (void*)key2, (void*)id, (void*)order, (void*)old2new, (void*)new_deg, (void*)nonzero})
        dfree(p, s);
    CGB_CUDA_TRY(cudaStreamSynchronize(s));
    if (nz_out) *nz_out = nz;
    return r;
}

}  // namespace cgb

void GraphMutex::lock()
{
    m.lock();
    cgb::swap_in_pending_weights(owner);
}

bool GraphMutex::try_lock()
{
    if (!m.try_lock()) return false;
    cgb::swap_in_pending_weights(owner);
    return true;
}
