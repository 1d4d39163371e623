// CSR from an edge list, on the device.
//
// The reference's other input format (has_csrFile = 0) is a binary file of
// packed 12-byte records {u32 src, u32 dst, u32 weight}; the edge count is the
// file size / 12 (Basic/Graph/graphBinReader.hpp:35-39, 89-104).  Its reader
// rejects self-loops (":150"), groups the edges by source, sorts every list
// by destination (sort_nbr, ":213-227"; its check rejects equal neighbours,
// ":238-254") and lays the lists out by out-degree (build_csr, ":286-322").
//
// Here: the records are turned into 64-bit keys (source << b | destination,
// b = bits for V) carrying the weights, radix-sorted on the device (a stable
// sort, so the result does not depend on the records' order), checked for
// self-loops, ids >= V and duplicates (CGB_EFORMAT, as the reference's
// asserts), and unpacked into the graph's CSR; the offsets come from one
// lower-bound search per vertex over the sorted sources.
#include <cub/device/device_radix_sort.cuh>

#include "engine.cuh"

namespace cgb {

// flags: 1 = self-loop, 2 = id >= V, 4 = duplicate edge
__global__ void k_records_to_keys(uint64_t E, const uint32_t* __restrict__ rec, uint32_t V, uint32_t b, uint64_t* keys,
                                  uint32_t* vals, uint32_t* flags)
{
    uint32_t bad = 0;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t s = rec[3 * e], d = rec[3 * e + 1];
        bad |= (s == d) ? 1u : 0u;
        bad |= (s >= V || d >= V) ? 2u : 0u;
        keys[e] = ((uint64_t)min(s, V - 1) << b) | min(d, V - 1);
        vals[e] = rec[3 * e + 2];
    }
    if (bad) atomicOr(flags, bad);
}

__global__ void k_unpack_sorted(uint64_t E, const uint64_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                                uint32_t b, uint32_t* src, uint32_t* dst, uint32_t* w, uint32_t* flags)
{
    const uint64_t mask = (1ull << b) - 1;
    uint32_t dup = 0;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = keys[e];
        src[e] = (uint32_t)(k >> b);
        dst[e] = (uint32_t)(k & mask);
        w[e] = vals[e];
        dup |= (e > 0 && keys[e - 1] == k) ? 4u : 0u;
    }
    if (dup) atomicOr(flags, dup);
}

// off[v] = first index whose sorted source is >= v, for v in [0, V].
__global__ void k_offsets_from_sources(uint32_t V, uint64_t E, const uint32_t* __restrict__ src, uint32_t* off)
{
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v <= V; v += gridDim.x * blockDim.x) {
        uint64_t lo = 0, hi = E;
        while (lo < hi) {
            const uint64_t mid = lo + (hi - lo) / 2;
            if (src[mid] < v) lo = mid + 1;
            else hi = mid;
        }
        off[v] = (uint32_t)lo;
    }
}

static uint32_t key_bits(uint64_t n)
{
    uint32_t b = 1;
    while (b < 32 && (1ull << b) < n) b++;
    return b;
}

cgb_graph* graph_from_edges(const uint32_t* records, uint64_t E, uint32_t V, int device)
{
    CGB_REQUIRE(V >= 1, CGB_EINVAL, "V must be >= 1");
    CGB_REQUIRE(V <= kMaxGraphSize && E <= kMaxGraphSize, CGB_EUNSUPPORTED, "V and E must be at most 2^32 - 2^24");
    CGB_REQUIRE(E == 0 || records != nullptr, CGB_EINVAL, "records is NULL");
    cgb_graph* g = graph_alloc(V, (uint32_t)E, V, device, E > 0);
    cudaStream_t s = g->stream;
    std::vector<void*> tmp;
    auto alloc = [&](size_t bytes) {
        void* p = pool_alloc(bytes ? bytes : 1, s);
        tmp.push_back(p);
        return p;
    };
    try {
        if (E == 0) {
            CGB_CUDA_TRY(cudaMemsetAsync(g->off, 0, ((size_t)V + 1) * 4, s));
        } else {
            const uint32_t b = key_bits(V);
            auto* rec = static_cast<uint32_t*>(alloc(E * 12));
            auto* keys = static_cast<uint64_t*>(alloc(E * 8));
            auto* keys_out = static_cast<uint64_t*>(alloc(E * 8));
            auto* vals = static_cast<uint32_t*>(alloc(E * 4));
            auto* vals_out = static_cast<uint32_t*>(alloc(E * 4));
            auto* src = static_cast<uint32_t*>(alloc(E * 4));
            auto* flags = static_cast<uint32_t*>(alloc(4));
            CGB_CUDA_TRY(cudaMemcpyAsync(rec, records, E * 12, cudaMemcpyDefault, s));
            CGB_CUDA_TRY(cudaMemsetAsync(flags, 0, 4, s));
            const uint32_t grid = grid_for(E, kBlock, num_sms() * 16);
            k_records_to_keys<<<grid, kBlock, 0, s>>>(E, rec, V, b, keys, vals, flags);
            size_t tb = 0;
            CGB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys, keys_out, vals, vals_out, E, 0, 2 * b, s));
            void* temp = alloc(tb);
            CGB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(temp, tb, keys, keys_out, vals, vals_out, E, 0, 2 * b, s));
            k_unpack_sorted<<<grid, kBlock, 0, s>>>(E, keys_out, vals_out, b, src, g->dst, g->w, flags);
            k_offsets_from_sources<<<grid_for((uint64_t)V + 1, kBlock, num_sms() * 16), kBlock, 0, s>>>(V, E, src,
                                                                                                     g->off);
            PinnedArray<uint32_t> h(1);
            CGB_CUDA_TRY(cudaMemcpyAsync(h.data(), flags, 4, cudaMemcpyDeviceToHost, s));
            CGB_CUDA_TRY(cudaStreamSynchronize(s));
            if (h[0] & 1u) throw Error{CGB_EFORMAT, "edge list holds a self-loop (src == dst)"};
            if (h[0] & 2u) throw Error{CGB_EFORMAT, "edge list holds a vertex id >= V"};
            if (h[0] & 4u) throw Error{CGB_EFORMAT, "edge list holds a duplicate edge"};
        }
        for (void* p : tmp) pool_free(p, s);
        tmp.clear();
        CGB_CUDA_TRY(cudaStreamSynchronize(s));
        validate_and_sort(g);
        compute_weight_sum(g);
    } catch (...) {
        cudaStreamSynchronize(s);
        for (void* p : tmp) pool_free(p, s);
        graph_free(g);
        throw;
    }
    return g;
}

}  // namespace cgb
