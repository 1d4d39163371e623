// Shared device/host helpers of the cgb200 engine (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/cgb200.h"

namespace cgb {

constexpr uint32_t kValueMax = CGB_VALUE_MAX;  // VertexValue_MAX, Basic/Graph/basic_def.hpp:18
constexpr int kBlock = 256;                    // threads per CTA for the frontier kernels
constexpr int kWarp = 32;
// SM count of the current device (148 on a B200), cached per device: the
// grids of the frontier kernels are sized in multiples of it.
int num_sms();
// Largest V and E of a graph.  Kernels step 32-bit indices by a grid stride
// below 2^24, so indices up to 2^32 - 2^24 never wrap.
constexpr uint32_t kMaxGraphSize = 0xFF000000u;

// Error state of the calling thread (cgb_last_error_string).
void set_error(const std::string& msg);
const std::string& last_error();

struct Error {
    cgb_status code;
    std::string msg;
};

#define CGB_CUDA_TRY(expr)                                                                       \
    do {                                                                                         \
        cudaError_t _e = (expr);                                                                 \
        if (_e != cudaSuccess) {                                                                 \
            throw ::cgb::Error{_e == cudaErrorMemoryAllocation ? CGB_ENOMEM : CGB_ECUDA,         \
                               std::string(#expr) + ": " + cudaGetErrorString(_e)};              \
        }                                                                                        \
    } while (0)

#define CGB_REQUIRE(cond, code, msg)                   \
    do {                                               \
        if (!(cond)) throw ::cgb::Error{(code), (msg)}; \
    } while (0)

// ------------------------------------------------------------ device helpers

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint32_t lanemask_lt() { return (1u << lane_id()) - 1u; }

// Warp-aggregated append: every lane of the warp must call this (pred may be
// false).  Returns nothing; writes `item` of each predicated lane into
// q[atomicAdd(ctr)...] with one atomic per warp.  Items past `cap` are not
// written and raise *overflow.
__device__ __forceinline__ void warp_append(bool pred, uint32_t item, uint32_t* q, uint32_t* ctr, uint32_t cap,
                                            uint32_t* overflow)
{
    uint32_t want = __ballot_sync(0xffffffffu, pred);
    if (!want) return;
    uint32_t leader = __ffs(want) - 1;
    uint32_t base = 0;
    if (lane_id() == leader) base = atomicAdd(ctr, (uint32_t)__popc(want));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (pred) {
        uint32_t idx = base + __popc(want & lanemask_lt());
        if (idx < cap) q[idx] = item;
        else atomicOr(overflow, 1u);
    }
}

__device__ __forceinline__ void warp_append2(bool pred, uint2 item, uint2* q, uint32_t* ctr, uint32_t cap,
                                             uint32_t* overflow)
{
    uint32_t want = __ballot_sync(0xffffffffu, pred);
    if (!want) return;
    uint32_t leader = __ffs(want) - 1;
    uint32_t base = 0;
    if (lane_id() == leader) base = atomicAdd(ctr, (uint32_t)__popc(want));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (pred) {
        uint32_t idx = base + __popc(want & lanemask_lt());
        if (idx < cap) q[idx] = item;
        else atomicOr(overflow, 1u);
    }
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ unsigned long long warp_or(unsigned long long v)
{
    for (int o = 16; o > 0; o >>= 1) v |= __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ uint32_t warp_max(uint32_t v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Inclusive warp scan.
__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v)
{
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t n = __shfl_up_sync(0xffffffffu, v, o);
        if (lane_id() >= (uint32_t)o) v += n;
    }
    return v;
}

// Exclusive block scan over kBlock threads; returns the exclusive prefix and
// the block total.  `smem` needs kBlock/32 + 1 words.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t& total, uint32_t* smem)
{
    const uint32_t warp = threadIdx.x >> 5;
    uint32_t incl = warp_incl_scan(v);
    if (lane_id() == 31) smem[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane_id() < (kBlock / 32) ? smem[lane_id()] : 0;
        uint32_t wi = warp_incl_scan(w);
        if (lane_id() < (kBlock / 32)) smem[lane_id()] = wi - w;
        if (lane_id() == (kBlock / 32) - 1) smem[kBlock / 32] = wi;
    }
    __syncthreads();
    uint32_t excl = smem[warp] + incl - v;
    total = smem[kBlock / 32];
    __syncthreads();
    return excl;
}

// splitmix64 finaliser (Steele, Lea, Flood 2014; public-domain constants),
// shared by the synthetic-graph generators on host and device.
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

inline uint32_t div_up(uint64_t a, uint64_t b) { return (uint32_t)((a + b - 1) / b); }

inline uint32_t grid_for(uint64_t items, uint32_t per_block, uint32_t max_blocks)
{
    uint64_t g = (items + per_block - 1) / per_block;
    if (g < 1) g = 1;
    if (g > max_blocks) g = max_blocks;
    return (uint32_t)g;
}

}  // namespace cgb
