// Seeded synthetic graphs built directly in HBM (RMAT, Chung-Lu, 2-D grid).
// The arithmetic mirrors the oracle's CPU twin exactly (integer quadrant
// thresholds, splitmix64 counters), so both build the same CSR.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>

#include "../../include/cgb200_gen.h"
#include "engine.cuh"

namespace cgb {

__device__ __forceinline__ uint32_t scramble_id(uint64_t x, uint32_t scale, uint64_t m1, uint64_t m2, uint64_t c)
{
    const uint64_t mask = (scale >= 64) ? ~0ull : ((1ull << scale) - 1);
    const uint32_t sh = scale / 2 ? scale / 2 : 1;
    x = (x * m1) & mask;
    x ^= x >> sh;
    x = (x * m2 + c) & mask;
    return (uint32_t)x;
}

constexpr uint64_t kSentinel = ~0ull;

__global__ void k_rmat_keys(uint32_t scale, uint64_t n, uint64_t s, uint64_t t1, uint64_t t2, uint64_t t3, int scr,
                            uint64_t m1, uint64_t m2, uint64_t c, int sym, uint64_t* keys)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t u = 0, v = 0;
        for (uint32_t l = 0; l < scale; l++) {
            const uint64_t r = mix64(s ^ mix64(i * 64 + l)) >> 32;
            const uint64_t bu = r >= t2;
            const uint64_t bv = (r >= t1 && r < t2) || r >= t3;
            u = (u << 1) | bu;
            v = (v << 1) | bv;
        }
        if (scr) {
            u = scramble_id(u, scale, m1, m2, c);
            v = scramble_id(v, scale, m1, m2, c);
        }
        const bool loop = u == v;
        keys[i] = loop ? kSentinel : ((u << 32) | v);
        if (sym) keys[n + i] = loop ? kSentinel : ((v << 32) | u);
    }
}

__global__ void k_keys_to_csr(uint32_t V, uint64_t m, const uint64_t* __restrict__ keys, uint32_t* off, uint32_t* dst)
{
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e <= m; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t hi = e < m ? (keys[e] >> 32) : V;
        const uint64_t lo = e == 0 ? 0 : (keys[e - 1] >> 32) + 1;
        for (uint64_t v = lo; v <= hi; v++) off[v] = (uint32_t)e;
        if (e < m) dst[e] = (uint32_t)keys[e];
    }
}

__device__ __forceinline__ uint32_t src_of(const uint32_t* __restrict__ off, uint32_t V, uint32_t e)
{
    uint32_t lo = 0, hi = V;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (off[mid] <= e) lo = mid;
        else hi = mid;
    }
    return lo;
}

__global__ void k_edge_weights(uint32_t V, uint32_t E, const uint32_t* __restrict__ off,
                               const uint32_t* __restrict__ dst, uint64_t s, uint32_t wmax, int sym_key, uint32_t* w)
{
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) {
        uint32_t a = src_of(off, V, e), b = dst[e];
        if (sym_key && b < a) {
            const uint32_t t = a;
            a = b;
            b = t;
        }
        const uint64_t h = mix64(s ^ (((uint64_t)a << 32) | b));
        w[e] = 1u + (uint32_t)(h % wmax);
    }
}

__global__ void k_grid_deg(uint32_t rows, uint32_t cols, uint32_t* deg)
{
    const uint64_t V = (uint64_t)rows * cols;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t r = (uint32_t)(v / cols), c = (uint32_t)(v % cols);
        deg[v] = (r > 0) + (c > 0) + (c + 1 < cols) + (r + 1 < rows);
    }
}

__global__ void k_grid_fill(uint32_t rows, uint32_t cols, const uint32_t* __restrict__ off, uint32_t* dst)
{
    const uint64_t V = (uint64_t)rows * cols;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t r = (uint32_t)(v / cols), c = (uint32_t)(v % cols);
        uint32_t e = off[v];
        const uint32_t x = (uint32_t)v;
        if (r > 0) dst[e++] = x - cols;
        if (c > 0) dst[e++] = x - 1;
        if (c + 1 < cols) dst[e++] = x + 1;
        if (r + 1 < rows) dst[e++] = x + cols;
    }
}

// ------------------------------------------------------------- Chung-Lu
// Vertex i (before the id permutation) has weight floor(2^40 / (i + i0)), so
// the expected degree of the rank-i vertex falls as 1 / (i + i0): a power law
// whose degree distribution has exponent 2 (Zipf rank exponent 1), with the
// largest expected degree set by i0.  Each draw picks both endpoints with
// probability proportional to weight, from the exact integer prefix sums
// (cum[j] = sum of the weights below j), so the CPU twin draws the same
// edges; the affine maps a*x+b mod V spread out-hubs and in-hubs over the
// id range independently.

__global__ void k_cl_weights(uint32_t V, uint64_t i0, uint64_t* w)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x)
        w[i] = (1ull << 40) / ((uint64_t)i + i0);
}

// Largest j < V with cum[j] <= r (cum[0] = 0 <= r < cum[V]): an analytic
// guess from the inverse of the weight integral, then an exact galloping
// and binary search against the table.
__device__ __forceinline__ uint32_t cl_pick(uint64_t r, const uint64_t* __restrict__ cum, uint32_t V, double i0)
{
    const double g = i0 * exp((double)r * (1.0 / 1099511627776.0)) - i0;
    uint32_t j = (uint32_t)fmin(fmax(g, 0.0), (double)(V - 1));
    uint32_t lo, hi;  // cum[lo] <= r < cum[hi]
    if (cum[j] <= r) {
        lo = j;
        uint32_t step = 1;
        hi = min(V, j + 1);
        while (hi < V && cum[hi] <= r) {
            lo = hi;
            step *= 2;
            hi = (uint32_t)min((uint64_t)V, (uint64_t)lo + step);
        }
    } else {
        hi = j;
        uint32_t step = 1;
        lo = j > 0 ? j - 1 : 0;
        while (lo > 0 && cum[lo] > r) {
            hi = lo;
            step *= 2;
            lo = lo > step ? lo - step : 0;
        }
    }
    while (hi - lo > 1) {
        const uint32_t mid = lo + (hi - lo) / 2;
        if (cum[mid] <= r) lo = mid;
        else hi = mid;
    }
    return lo;
}

__global__ void k_cl_keys(uint32_t V, uint64_t n, const uint64_t* __restrict__ cum, double i0, uint64_t s_out,
                          uint64_t s_in, uint64_t a_out, uint64_t b_out, uint64_t a_in, uint64_t b_in, int sym,
                          uint64_t* keys)
{
    const uint64_t W = cum[V];
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t hi = mix64(i);
        const uint64_t x = cl_pick(mix64(s_out ^ hi) % W, cum, V, i0);
        const uint64_t y = cl_pick(mix64(s_in ^ hi) % W, cum, V, i0);
        const uint64_t u = (a_out * x + b_out) % V, v = (a_in * y + b_in) % V;
        const bool loop = u == v;
        keys[i] = loop ? kSentinel : ((u << 32) | v);
        if (sym) keys[n + i] = loop ? kSentinel : ((v << 32) | u);
    }
}

static uint64_t gcd64(uint64_t a, uint64_t b)
{
    while (b) {
        const uint64_t t = a % b;
        a = b;
        b = t;
    }
    return a;
}

// Affine bijection of [0, V): multiplier coprime with V, both from the seed.
static void cl_affine(uint32_t V, uint64_t seed, uint64_t tag, uint64_t& a, uint64_t& b)
{
    a = V > 1 ? 1 + mix64(seed ^ tag) % (V - 1) : 1;
    while (gcd64(a, V) != 1) a = a % (V - 1) + 1;
    b = mix64(seed ^ (tag + 1)) % V;
}

// Scratch from the engine's pool, ordered on the generator's stream (a
// cudaFree would synchronise the whole device).
static void* galloc(size_t bytes, cudaStream_t st) { return pool_alloc(bytes ? bytes : 1, st); }

cgb_graph* gen_rmat(uint32_t scale, uint32_t ef, uint64_t seed, double a, double b, double c, int scr, int sym,
                    uint32_t wmax, int device)
{
    CGB_REQUIRE(scale >= 1 && scale <= 31, CGB_EINVAL, "RMAT scale must be in [1, 31]");
    CGB_REQUIRE(a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0, CGB_EINVAL, "bad RMAT probabilities");
    CGB_CUDA_TRY(cudaSetDevice(device));
    const uint32_t V = 1u << scale;
    const uint64_t n = (uint64_t)ef << scale;
    const uint64_t total = sym ? 2 * n : n;
    const uint64_t t1 = (uint64_t)(a * 4294967296.0);
    const uint64_t t2 = (uint64_t)((a + b) * 4294967296.0);
    const uint64_t t3 = (uint64_t)((a + b + c) * 4294967296.0);
    const uint64_t m1 = mix64(seed ^ 0x5C0A11ull) | 1ull;
    const uint64_t m2 = mix64(seed ^ 0x5C0A12ull) | 1ull;
    const uint64_t cc = mix64(seed ^ 0x5C0A13ull);
    cudaStream_t st;
    CGB_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    uint64_t* keys = (uint64_t*)galloc(total * 8, st);
    uint64_t* alt = (uint64_t*)galloc(total * 8, st);
    uint64_t* cnt = (uint64_t*)galloc(8, st);
    void* temp = nullptr;
    cgb_graph* g = nullptr;
    try {
        k_rmat_keys<<<num_sms() * 16, kBlock, 0, st>>>(scale, n, mix64(seed), t1, t2, t3, scr, m1, m2, cc, sym, keys);
        cub::DoubleBuffer<uint64_t> db(keys, alt);
        size_t tb = 0, tb2 = 0;
        CGB_CUDA_TRY(cub::DeviceRadixSort::SortKeys(nullptr, tb, db, total, 0, 32 + (int)scale, st));
        uint64_t* in_unique = nullptr;
        CGB_CUDA_TRY(cub::DeviceSelect::Unique(nullptr, tb2, keys, alt, cnt, total, st));
        temp = galloc(std::max(tb, tb2), st);
        CGB_CUDA_TRY(cub::DeviceRadixSort::SortKeys(temp, tb, db, total, 0, 32 + (int)scale, st));
        in_unique = db.Current();
        uint64_t* out_unique = db.Alternate();
        CGB_CUDA_TRY(cub::DeviceSelect::Unique(temp, tb2, in_unique, out_unique, cnt, total, st));
        PinnedArray<uint64_t> hm(2);  // pinned: see pinned_acquire
        CGB_CUDA_TRY(cudaMemcpyAsync(hm.data(), cnt, 8, cudaMemcpyDeviceToHost, st));
        CGB_CUDA_TRY(cudaStreamSynchronize(st));
        uint64_t m = hm[0];
        if (m) {
            CGB_CUDA_TRY(cudaMemcpyAsync(hm.data() + 1, out_unique + m - 1, 8, cudaMemcpyDeviceToHost, st));
            CGB_CUDA_TRY(cudaStreamSynchronize(st));
            if (hm[1] == kSentinel) m--;
        }
        CGB_REQUIRE(m < 0xFFFFFFFFull, CGB_EUNSUPPORTED, "RMAT graph has >= 2^32 edges");
        g = graph_alloc(V, (uint32_t)m, V, device, wmax > 0);
        k_keys_to_csr<<<num_sms() * 16, kBlock, 0, st>>>(V, m, out_unique, g->off, g->dst);
        if (wmax)
            k_edge_weights<<<num_sms() * 16, kBlock, 0, st>>>(V, (uint32_t)m, g->off, g->dst, mix64(seed ^ 0x77E16ull),
                                                            wmax, sym, g->w);
        CGB_CUDA_TRY(cudaStreamSynchronize(st));
        if (sym) g->symmetric = 1;
    } catch (...) {
        pool_free(keys, st);
        pool_free(alt, st);
        pool_free(cnt, st);
        if (temp) pool_free(temp, st);
        cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
        if (g) graph_free(g);
        throw;
    }
    pool_free(keys, st);
    pool_free(alt, st);
    pool_free(cnt, st);
    pool_free(temp, st);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    compute_weight_sum(g);
    return g;
}

cgb_graph* gen_chunglu(uint32_t V, uint64_t draws, uint32_t i0, uint64_t seed, int sym, uint32_t wmax, int device)
{
    CGB_REQUIRE(V >= 2 && V < 0xFFFFFFFFu && i0 >= 1, CGB_EINVAL, "Chung-Lu needs V >= 2 and weight offset >= 1");
    const uint64_t total = sym ? 2 * draws : draws;
    CGB_CUDA_TRY(cudaSetDevice(device));
    uint64_t a_out, b_out, a_in, b_in;
    cl_affine(V, seed, 0xC1A0011ull, a_out, b_out);
    cl_affine(V, seed, 0xC1A0021ull, a_in, b_in);
    uint32_t bits = 1;
    while (bits < 32 && (1ull << bits) < V) bits++;
    cudaStream_t st;
    CGB_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    uint64_t* cum = nullptr;
    uint64_t* keys = nullptr;
    uint64_t* alt = nullptr;
    uint64_t* cnt = nullptr;
    void* temp = nullptr;
    cgb_graph* g = nullptr;
    try {
        // exact integer prefix sums of the weights (cum[V] = total weight)
        cum = (uint64_t*)galloc(((size_t)V + 1) * 8, st);
        uint64_t* wts = (uint64_t*)galloc(((size_t)V + 1) * 8, st);
        k_cl_weights<<<num_sms() * 8, kBlock, 0, st>>>(V, i0, wts);
        CGB_CUDA_TRY(cudaMemsetAsync(wts + V, 0, 8, st));
        size_t tb = 0;
        CGB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, wts, cum, (uint64_t)V + 1, st));
        void* stemp = galloc(tb, st);
        CGB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(stemp, tb, wts, cum, (uint64_t)V + 1, st));
        CGB_CUDA_TRY(cudaStreamSynchronize(st));
        pool_free(stemp, st);
        pool_free(wts, st);
        keys = (uint64_t*)galloc(total * 8, st);
        k_cl_keys<<<num_sms() * 16, kBlock, 0, st>>>(V, draws, cum, (double)i0, mix64(seed ^ 0xC1A0001ull),
                                                   mix64(seed ^ 0xC1A0002ull), a_out, b_out, a_in, b_in, sym, keys);
        CGB_CUDA_TRY(cudaStreamSynchronize(st));
        pool_free(cum, st);
        cum = nullptr;
        alt = (uint64_t*)galloc(total * 8, st);
        cnt = (uint64_t*)galloc(8, st);
        cub::DoubleBuffer<uint64_t> db(keys, alt);
        size_t tb1 = 0, tb2 = 0;
        CGB_CUDA_TRY(cub::DeviceRadixSort::SortKeys(nullptr, tb1, db, total, 0, 32 + (int)bits, st));
        CGB_CUDA_TRY(cub::DeviceSelect::Unique(nullptr, tb2, keys, alt, cnt, total, st));
        temp = galloc(std::max(tb1, tb2), st);
        CGB_CUDA_TRY(cub::DeviceRadixSort::SortKeys(temp, tb1, db, total, 0, 32 + (int)bits, st));
        uint64_t* in_unique = db.Current();
        uint64_t* out_unique = db.Alternate();
        CGB_CUDA_TRY(cub::DeviceSelect::Unique(temp, tb2, in_unique, out_unique, cnt, total, st));
        PinnedArray<uint64_t> hm(2);  // pinned: see pinned_acquire
        CGB_CUDA_TRY(cudaMemcpyAsync(hm.data(), cnt, 8, cudaMemcpyDeviceToHost, st));
        CGB_CUDA_TRY(cudaStreamSynchronize(st));
        uint64_t m = hm[0];
        if (m) {
            CGB_CUDA_TRY(cudaMemcpyAsync(hm.data() + 1, out_unique + m - 1, 8, cudaMemcpyDeviceToHost, st));
            CGB_CUDA_TRY(cudaStreamSynchronize(st));
            if (hm[1] == kSentinel) m--;
        }
        CGB_REQUIRE(m < 0xFFFFFFFFull, CGB_EUNSUPPORTED, "Chung-Lu graph has >= 2^32 edges");
        g = graph_alloc(V, (uint32_t)m, V, device, wmax > 0);
        k_keys_to_csr<<<num_sms() * 16, kBlock, 0, st>>>(V, m, out_unique, g->off, g->dst);
        if (wmax)
            k_edge_weights<<<num_sms() * 16, kBlock, 0, st>>>(V, (uint32_t)m, g->off, g->dst, mix64(seed ^ 0x77E16ull),
                                                            wmax, sym, g->w);
        CGB_CUDA_TRY(cudaStreamSynchronize(st));
        if (sym) g->symmetric = 1;
    } catch (...) {
        if (cum) pool_free(cum, st);
        if (keys) pool_free(keys, st);
        if (alt) pool_free(alt, st);
        if (cnt) pool_free(cnt, st);
        if (temp) pool_free(temp, st);
        cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
        if (g) graph_free(g);
        throw;
    }
    pool_free(keys, st);
    pool_free(alt, st);
    pool_free(cnt, st);
    pool_free(temp, st);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    compute_weight_sum(g);
    return g;
}

cgb_graph* gen_grid(uint32_t rows, uint32_t cols, uint64_t seed, uint32_t wmax, int device)
{
    const uint64_t V64 = (uint64_t)rows * cols;
    CGB_REQUIRE(rows >= 1 && cols >= 1 && V64 < 0xFFFFFFFFull, CGB_EINVAL, "bad grid size");
    const uint64_t E64 = 4 * V64 - 2ull * rows - 2ull * cols;
    CGB_REQUIRE(E64 < 0xFFFFFFFFull, CGB_EUNSUPPORTED, "grid has >= 2^32 edges");
    const uint32_t V = (uint32_t)V64, E = (uint32_t)E64;
    CGB_CUDA_TRY(cudaSetDevice(device));
    cgb_graph* g = graph_alloc(V, E, V, device, wmax > 0);
    uint32_t* deg = nullptr;
    void* temp = nullptr;
    try {
        deg = (uint32_t*)galloc(((size_t)V + 1) * 4, g->stream);
        k_grid_deg<<<num_sms() * 8, kBlock, 0, g->stream>>>(rows, cols, deg);
        CGB_CUDA_TRY(cudaMemsetAsync(deg + V, 0, 4, g->stream));
        size_t tb = 0;
        CGB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, deg, g->off, (uint64_t)V + 1, g->stream));
        temp = galloc(tb, g->stream);
        CGB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(temp, tb, deg, g->off, (uint64_t)V + 1, g->stream));
        k_grid_fill<<<num_sms() * 8, kBlock, 0, g->stream>>>(rows, cols, g->off, g->dst);
        if (wmax)
            k_edge_weights<<<num_sms() * 16, kBlock, 0, g->stream>>>(V, E, g->off, g->dst, mix64(seed ^ 0x77E16ull), wmax,
                                                                   1, g->w);
        CGB_CUDA_TRY(cudaStreamSynchronize(g->stream));
    } catch (...) {
        if (deg) pool_free(deg, g->stream);
        if (temp) pool_free(temp, g->stream);
        graph_free(g);
        throw;
    }
    pool_free(deg, g->stream);
    pool_free(temp, g->stream);
    g->symmetric = 1;
    compute_weight_sum(g);
    return g;
}

}  // namespace cgb
