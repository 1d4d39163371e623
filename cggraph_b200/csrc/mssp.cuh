// Multi-root SSSP state and kernels shared by the batch path (mssp.cu) and
// the request server (serve.cu).  See mssp.cu for the algorithm.
#pragma once

#include "engine.cuh"

namespace cgb {

constexpr uint32_t kMsRoots = 64;   // distance slots per vertex

struct MsspCounters {
    uint32_t nq_in;        // entries of the near queue being expanded
    uint32_t nq_out;       // entries of the near queue being built
    uint32_t nfar_live;    // entries of the live far list (expansion rounds append)
    uint32_t nfar_next;    // entries kept by a split in the other far list
    uint32_t ndesc;        // descriptors of the round
    uint32_t min_far;      // smallest far distance >= hi seen by a split
    uint32_t overflow;
    unsigned long long relax;  // successful relaxations
};

struct MsspBuffers {
    uint32_t* dist = nullptr;               // V * 64
    unsigned long long* pend = nullptr;     // V
    unsigned long long* farm = nullptr;     // V
    unsigned long long* maskq = nullptr;    // V: pend of each queue entry, taken by the descriptor pass
    uint32_t* far_list[2] = {nullptr, nullptr};  // V each
    uint4* desc = nullptr;                  // {v, edge begin, edge end, queue index}
    uint64_t desc_cap = 0;
    MsspCounters* c = nullptr;
    MsspCounters* h = nullptr;              // pinned host copy
};

MsspBuffers* mssp_buffers_alloc(uint32_t V, uint64_t E);
void mssp_buffers_free(MsspBuffers* b);

__global__ void k_mssp_desc(const uint32_t* __restrict__ q, const uint32_t* nq_ptr, const uint32_t* __restrict__ off,
                            unsigned long long* pend, unsigned long long* maskq, uint4* desc, uint64_t cap,
                            MsspCounters* c, uint32_t ms_edges);
__global__ void k_mssp_split(const uint32_t* __restrict__ far_in, const uint32_t* nfar_ptr,
                             const uint32_t* __restrict__ dist, unsigned long long* pend, unsigned long long* farm,
                             uint32_t* q, uint32_t* q_len, uint32_t* far_out, uint32_t* far_out_len, uint32_t cap,
                             uint32_t lo, uint32_t hi, const uint32_t* lo_slot, const uint32_t* hi_slot,
                             unsigned long long adv, uint32_t* min_far_slot, unsigned long long* far_alive,
                             MsspCounters* c);
// Launches k_mssp_expand (weighted or unit weights) on stream st.
void mssp_expand(bool weighted, uint32_t grid, cudaStream_t st, const uint4* desc, const MsspCounters* cc,
                 const unsigned long long* maskq, const uint32_t* dst, const uint32_t* w, uint32_t* dist,
                 unsigned long long* pend, unsigned long long* farm, uint32_t* qout, uint32_t* qout_len,
                 uint32_t* far_out, uint32_t* far_len, uint32_t cap, uint32_t thr, const uint32_t* thr_slot,
                 unsigned long long* alive);

}  // namespace cgb
