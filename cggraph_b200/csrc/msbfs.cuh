// Multi-root BFS state and kernels shared by the batch path (msbfs.cu) and
// the request server (serve.cu).  See msbfs.cu for the algorithm.
#pragma once

#include "engine.cuh"

namespace cgb {

struct MsBuffers {
    unsigned long long* seen = nullptr;
    unsigned long long* front[2] = {nullptr, nullptr};
    unsigned long long* next = nullptr;     // top-down scratch; bottom-up partial masks; zero between levels
    uint32_t* heavy_w = nullptr;            // bottom-up: vertices finished by a warp (V)
    uint32_t* heavy_b = nullptr;            // ... by a CTA (cap_b)
    uint32_t* heavy_len = nullptr;          // [2] lengths of the two lists
    uint32_t cap_b = 0;
};

MsBuffers* ms_buffers_alloc(uint32_t V, uint64_t E);
void ms_buffers_free(MsBuffers* b);

// One bottom-up level (three kernels, see msbfs.cu).
struct MsBuArgs {
    uint32_t V;
    const uint32_t* in_off;
    const uint32_t* in_src;
    const unsigned long long* front;  // current frontier masks
    unsigned long long* seen;
    unsigned long long* fnext;        // next frontier masks (zero on entry)
    unsigned long long* acc;          // partial masks (zero on entry and exit)
    unsigned long long full;          // roots that still have a frontier
    uint32_t* level_out;
    uint32_t lvl;
    uint32_t nz;
    uint32_t* qact;                   // next queue
    uint32_t* qact_len;
    uint32_t cap;
    DevCounters* ctr;
    const uint32_t* start;            // per-root start level (server) or NULL
    unsigned long long* alive;        // roots given new frontier vertices, or NULL
    uint32_t* heavy_w;
    uint32_t* heavy_b;
    uint32_t* heavy_len;
    uint32_t cap_b;
};
void ms_bottom_up(const MsBuArgs& a, cudaStream_t st, uint64_t* launches);

struct MsTdOp {
    const uint32_t* __restrict__ off;
    const uint32_t* __restrict__ dst;
    const unsigned long long* __restrict__ front;
    const unsigned long long* seen;
    unsigned long long* next;
    uint32_t* qout;
    uint32_t* qlen;
    uint32_t cap;
    DevCounters* ctr;

    __device__ __forceinline__ bool load(uint32_t v, uint32_t& s, uint32_t& d, uint32_t& m) const
    {
        s = off[v];
        d = off[v + 1] - s;
        m = v;
        return true;
    }
    __device__ __forceinline__ void edge(bool valid, uint32_t e, uint32_t v) const
    {
        bool first = false;
        uint32_t u = 0;
        if (valid) {
            u = dst[e];
            const unsigned long long add = front[v] & ~seen[u];
            if (add && (next[u] & add) != add) first = atomicOr(next + u, add) == 0ull;
        }
        warp_append(first, u, qout, qlen, cap, &ctr->overflow);
    }
    __device__ __forceinline__ void block_begin() const {}
    __device__ __forceinline__ void block_end() const {}
};

// n_ptr (optional) replaces n by a device-resident count.
__global__ void k_ms_finalize(const uint32_t* __restrict__ q, uint32_t n, const uint32_t* n_ptr,
                              unsigned long long* seen,
                              unsigned long long* next, unsigned long long* fnext, uint32_t* level_out, uint32_t V,
                              uint32_t lvl, uint32_t nz, uint32_t* qact, uint32_t* qact_len, uint32_t cap,
                              DevCounters* ctr, const uint32_t* start, unsigned long long* alive);
__global__ void k_ms_clear(const uint32_t* __restrict__ q, uint32_t n, unsigned long long* f);
__global__ void k_ms_fill(uint64_t n, uint32_t* a, uint32_t value);
__global__ void k_ms_degree_sum(const uint32_t* __restrict__ q, uint32_t n, const uint32_t* n_ptr,
                                const uint32_t* __restrict__ off, DevCounters* ctr);
unsigned long long* ms_alloc(size_t n);

}  // namespace cgb
