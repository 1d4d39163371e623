// The reference's two-level partition (my_project/CGgraph/Two-level_partition.cuh):
// level 1 cuts the vertices with out-edges, [0, noZeroOutDegreeNum), into
// segments of 1024 vertices (get_SegmentInfo, :213-259); level 2 sorts the
// segments by average degree and cuts them into four buckets, degree up to
// 16, up to 32, up to 256 and above (partition_buckets, :267-342); then the
// segments are dealt to the GPUs bucket by bucket, round robin with the
// balancing offset, while each GPU's memory holds their edges
// (partition_GPU, :350-444).  The segments left over stay with the host.
//
// Here the per-segment statistics and the degree sort run on the device
// (offsets differences and one stable radix sort); the deal is a sequential
// capacity walk over at most V / 1024 segments, done on the host as the
// reference does.  The per-GPU CSR copies of build_deviceCSR (:484-720) are
// not made: the engine runs every graph whole on one GPU.
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <vector>

#include "engine.cuh"

namespace cgb {

constexpr uint32_t kSegmentSize = 1024;                    // SEGMENT_SIZE, :7
constexpr uint64_t kGpuReservedBytes = 1024ull * 1024 * 1024;  // GPU_RESERVED_MEMORY, :12
constexpr uint32_t kBucketNum = 4;                         // BUCKET_NUM, :10

// Segment s covers vertices [1024 s, min(1024 (s + 1), nz)): its edges are an
// offsets difference, its degree the integer quotient edges / vertices
// (seg_degree, :250), its sort key that degree.
__global__ void k_segment_keys(uint32_t nseg, uint32_t nz, const uint32_t* __restrict__ off, uint32_t* edges,
                               uint32_t* key, uint32_t* id)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < nseg; s += stride) {
        const uint64_t b = s * kSegmentSize;
        const uint64_t e = b + kSegmentSize < nz ? b + kSegmentSize : nz;
        const uint32_t m = off[e] - off[b];
        edges[s] = m;
        key[s] = m / (uint32_t)(e - b);
        id[s] = (uint32_t)s;
    }
}

void graph_partition(cgb_graph* g, int algorithm, uint32_t ndev, const uint64_t* mem_bytes, uint32_t* seg_order,
                     uint32_t* seg_edges, int32_t* seg_owner, uint32_t* device_segments, cgb_partition_info* info)
{
    const uint32_t V = g->V, nz = g->nz;
    const uint32_t nseg = (uint32_t)(((uint64_t)nz + kSegmentSize - 1) / kSegmentSize);
    std::vector<uint64_t> mem(ndev);
    for (uint32_t d = 0; d < ndev; d++) {
        if (mem_bytes) {
            mem[d] = mem_bytes[d];
        } else {
            cudaDeviceProp prop;
            CGB_CUDA_TRY(cudaGetDeviceProperties(&prop, (int)d));
            mem[d] = prop.totalGlobalMem;  // GPUInfo::getGlobalMem_byte
        }
    }
    cudaStream_t s = g->stream;
    std::vector<uint32_t> h_key(nseg), h_id(nseg), h_edges(nseg);
    if (nseg) {
        struct Held {  // pool blocks returned on every path
            cudaStream_t s;
            std::vector<void*> p;
            void* get(size_t bytes)
            {
                p.push_back(pool_alloc(bytes ? bytes : 1, s));
                return p.back();
            }
            ~Held()
            {
                cudaStreamSynchronize(s);
                for (void* q : p) pool_free(q, s);
            }
        } held{s, {}};
        auto* edges = static_cast<uint32_t*>(held.get((size_t)nseg * 4));
        auto* key = static_cast<uint32_t*>(held.get((size_t)nseg * 4));
        auto* key2 = static_cast<uint32_t*>(held.get((size_t)nseg * 4));
        auto* id = static_cast<uint32_t*>(held.get((size_t)nseg * 4));
        auto* id2 = static_cast<uint32_t*>(held.get((size_t)nseg * 4));
        k_segment_keys<<<grid_for(nseg, kBlock, num_sms() * 4), kBlock, 0, s>>>(nseg, nz, g->off, edges, key, id);
        size_t tb = 0;
        CGB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tb, key, key2, id, id2, (uint64_t)nseg, 0, 32, s));
        void* temp = held.get(tb);
        // stable: equal degrees keep ascending segment ids, the reference's tie order (:270-280)
        CGB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(temp, tb, key, key2, id, id2, (uint64_t)nseg, 0, 32, s));
        CGB_CUDA_TRY(cudaMemcpyAsync(h_key.data(), key2, (size_t)nseg * 4, cudaMemcpyDeviceToHost, s));
        CGB_CUDA_TRY(cudaMemcpyAsync(h_id.data(), id2, (size_t)nseg * 4, cudaMemcpyDeviceToHost, s));
        CGB_CUDA_TRY(cudaMemcpyAsync(h_edges.data(), edges, (size_t)nseg * 4, cudaMemcpyDeviceToHost, s));
        CGB_CUDA_TRY(cudaStreamSynchronize(s));
    }

    // buckets: first sorted position with degree >= 17, >= 33, >= 257 (:293-318)
    info->segment_num = nseg;
    info->bucket_start[0] = 0;
    const uint32_t bounds[3] = {17u, 33u, 257u};  // HALFWARP + 1, WARPSIZE + 1, BLOCKSIZE + 1
    for (int b = 0; b < 3; b++)
        info->bucket_start[b + 1] = (uint32_t)(std::lower_bound(h_key.begin(), h_key.end(), bounds[b]) - h_key.begin());
    info->bucket_start[kBucketNum] = nseg;

    // each GPU keeps the values, the offsets and a reserve (:363-375)
    std::vector<int64_t> cap(ndev);
    for (uint32_t d = 0; d < ndev; d++)
        cap[d] = (int64_t)mem[d] -
                 (int64_t)((uint64_t)V * 4 + ((uint64_t)nz + 1) * 4 + kGpuReservedBytes);
    const uint64_t per_edge = algorithm == CGB_SSSP ? 8 : 4;  // dest (+ weight) bytes
    std::vector<int32_t> owner(nseg, -1);
    std::vector<uint32_t> count(ndev, 0);
    bool all = true;
    uint32_t reached = 0;
    for (uint32_t b = 0; b < kBucketNum && all; b++) {
        reached = b;
        const uint32_t first = info->bucket_start[b], n = info->bucket_start[b + 1] - first;
        for (uint32_t j = 0; j < n; j++) {
            const uint32_t dev = (j + j / ndev) % ndev;  // MORE_BALANCE_PARTITION (:397-401)
            const uint32_t sid = h_id[first + j];
            const int64_t occupancy = (int64_t)(h_edges[sid] * per_edge);
            cap[dev] -= occupancy;
            if (cap[dev] <= 0) {  // this GPU is full: the walk ends here (:410-418)
                cap[dev] += occupancy;
                all = false;
                break;
            }
            owner[sid] = (int32_t)dev;
            count[dev]++;
        }
    }
    info->can_hold_all = all ? 1 : 0;
    info->reached_bucket = reached;
    if (seg_order) std::copy(h_id.begin(), h_id.end(), seg_order);
    if (seg_edges) std::copy(h_edges.begin(), h_edges.end(), seg_edges);
    if (seg_owner) std::copy(owner.begin(), owner.end(), seg_owner);
    if (device_segments) std::copy(count.begin(), count.end(), device_segments);
}

}  // namespace cgb
