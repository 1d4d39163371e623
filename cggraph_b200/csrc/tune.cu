// Launch-parameter tuning of one graph: cgb_tuning_get / cgb_tuning_set and
// the autotuner (cgb_autotune).
//
// The reference fixes its work-distribution thresholds at compile time
// (WarpDonate / CTA::schedule switch at 16 / 32 / 256 edges,
// my_project/CGgraph/device_warpDonate.cuh:42-388, device_CTA.cuh:28-112).
// Here they are per-graph parameters: the out-degree from which a list is
// cut into chunks, the chunk length, the push grid (CTAs per SM) and CTA
// size (the reference's fixed BLOCKSIZE 256, Basic/Graph/basic_def.hpp:8),
// the frontier size and list length below which the device-resident loops
// run, and the multi-root SSSP descriptor length.  None of them changes a
// result.
//
// Each algorithm has its own tuning (a run makes its algorithm's tuning the
// active one).  The autotuner is coordinate descent: starting from the
// algorithm's current tuning it tries, one field at a time, every candidate value of that field
// with the others fixed, keeps the fastest, and sweeps the fields twice.  A
// candidate's score is the summed device time of runs from the given roots
// (best of two runs per root, after one untimed run), so the starting
// tuning is always among the candidates and the result is never slower on
// that measurement.
#include <vector>

#include "../../include/cgb200.h"
#include "engine.cuh"

using namespace cgb;

namespace {

bool valid(const cgb_tuning& t)
{
    auto pow2 = [](uint32_t x) { return x && !(x & (x - 1)); };
    return t.push_big_deg >= kMinBigDeg && t.push_big_deg <= 65536 && t.push_chunk >= kMinChunk &&
           t.push_chunk <= 65536 && pow2(t.push_chunk) && t.push_ctas_per_sm >= 1 && t.push_ctas_per_sm <= 32 &&
           t.persist_deg >= 64 && t.persist_deg <= 65536 && t.ms_edges >= kMinMsEdges && t.ms_edges <= 4096 &&
           (t.pr_unroll == 4 || t.pr_unroll == 8 || t.pr_unroll == 16) && t.pr_ctas_per_sm >= 1 &&
           t.pr_ctas_per_sm <= 1024 && t.persist_ctas <= 4096 && t.sssp_pull_alpha <= 1024 &&
           t.cluster_enter <= (1u << 24) && t.sssp_dense_alpha <= 1024 &&
           (t.push_block == 128 || t.push_block == 256 || t.push_block == 512);
}

struct Field {
    uint32_t cgb_tuning::*member;
    std::vector<uint32_t> values;
    bool bfs, sssp, cc, pr, ms_bfs, ms_sssp;  // used by: one BFS / SSSP / CC / PR run; multi-root passes
};

std::vector<Field> fields()
{
    return {
        {&cgb_tuning::push_big_deg, {128, 256, 512, 1024, 2048, 4096}, true, true, true, false, true, false},
        {&cgb_tuning::push_chunk, {256, 512, 1024, 2048, 4096}, true, true, true, false, true, false},
        {&cgb_tuning::push_ctas_per_sm, {2, 4, 8, 16}, true, true, true, false, true, false},
        {&cgb_tuning::push_block, {128, 256, 512}, true, true, true, false, true, false},
        {&cgb_tuning::persist_enter, {0, 4096, 16384, 32768, 131072}, true, true, false, false, false, false},
        {&cgb_tuning::persist_deg, {256, 1024, 2048, 8192}, true, true, false, false, false, false},
        {&cgb_tuning::persist_ctas, {0, 16, 32, 64}, true, true, false, false, false, false},
        {&cgb_tuning::sssp_pull_alpha, {0, 2, 3, 5, 8}, false, true, false, false, false, false},
        {&cgb_tuning::cluster_enter, {0, 2048, 8192, 16384}, true, false, false, false, false, false},
        {&cgb_tuning::sssp_dense_alpha, {0, 2, 4, 8, 16}, false, true, false, false, false, false},
        {&cgb_tuning::ms_edges, {64, 128, 256, 512, 1024}, false, false, false, false, false, true},
        {&cgb_tuning::pr_unroll, {4, 8, 16}, false, false, false, true, false, false},
        {&cgb_tuning::pr_ctas_per_sm, {16, 32, 64, 128, 256, 1024}, false, false, false, true, false, false},
    };
}

// The batching autotuner's tiler: the reference's two-level partition
// (my_project/CGgraph/Two-level_partition.cuh:213-342, cgb_graph_partition)
// cuts the vertices into 1024-vertex segments and sorts them into four
// buckets by average out-degree (up to 16, 32, 256, above).  The bucket that
// holds the median edge sets the multi-root SSSP work tile (descriptor
// length, ms_edges): lists in segments of degree above 256 are walked in
// 1024-edge tiles, 33..256 in 256, 17..32 in 128, up to 16 in 64.  The
// search then starts from the better of that tile and the graph's current
// one.
uint32_t tile_from_partition(cgb_graph* g)
{
    cgb_partition_info info{};
    const uint32_t nseg = (uint32_t)(((uint64_t)g->nz + 1023) / 1024);
    if (nseg == 0) return 0;
    std::vector<uint32_t> order(nseg), edges(nseg);
    const uint64_t roomy = ~0ull >> 2;  // one device that holds everything: the deal is irrelevant here
    {
        std::lock_guard<GraphMutex> lock(g->mu);
        CGB_CUDA_TRY(cudaSetDevice(g->device));
        graph_partition(g, CGB_SSSP, 1, &roomy, order.data(), edges.data(), nullptr, nullptr, &info);
    }
    uint64_t per_bucket[4] = {0, 0, 0, 0}, total = 0;
    for (int b = 0; b < 4; b++)
        for (uint32_t j = info.bucket_start[b]; j < info.bucket_start[b + 1]; j++) per_bucket[b] += edges[order[j]];
    for (int b = 0; b < 4; b++) total += per_bucket[b];
    const uint32_t tiles[4] = {64, 128, 256, 1024};
    uint64_t acc = 0;
    for (int b = 0; b < 4; b++) {
        acc += per_bucket[b];
        if (2 * acc >= total) return tiles[b];
    }
    return tiles[3];
}

}  // namespace

extern "C" {

cgb_status cgb_tuning_get(const cgb_graph* g, int algorithm, cgb_tuning* out)
{
    if (!g || !out || algorithm < 0 || algorithm > CGB_PR) {
        set_error("NULL argument or unknown algorithm");
        return CGB_EINVAL;
    }
    *out = g->tune_alg[algorithm];
    return CGB_OK;
}

cgb_status cgb_tuning_set(cgb_graph* g, int algorithm, const cgb_tuning* t)
{
    if (!g || !t || algorithm < -1 || algorithm > CGB_PR) {
        set_error("NULL argument or unknown algorithm");
        return CGB_EINVAL;
    }
    if (t->struct_size < sizeof(cgb_tuning)) {
        set_error("cgb_tuning.struct_size too small");
        return CGB_EINVAL;
    }
    cgb_tuning tv = *t;
    if (tv.push_block == 0) tv.push_block = 256;
    t = &tv;
    if (!valid(*t)) {
        set_error("cgb_tuning value out of range");
        return CGB_EINVAL;
    }
    std::lock_guard<GraphMutex> lock(g->mu);
    for (int a = 0; a <= CGB_PR; a++) {
        if (algorithm != -1 && a != algorithm) continue;
        g->tune_alg[a] = *t;
        g->tune_alg[a].struct_size = sizeof(cgb_tuning);
    }
    return CGB_OK;
}

cgb_status cgb_autotune(cgb_graph* g, int algorithm, const uint32_t* roots, uint32_t nroots, uint32_t flags,
                        cgb_tuning* best, double* best_ms, double* start_ms)
{
    if (!g || !roots || nroots == 0) {
        set_error("NULL argument or no roots");
        return CGB_EINVAL;
    }
    const bool batch = (flags & CGB_TUNE_BATCH) != 0;
    if (algorithm != CGB_BFS && algorithm != CGB_SSSP && !((algorithm == CGB_CC || algorithm == CGB_PR) && !batch)) {
        set_error("cgb_autotune tunes BFS, SSSP (runs or multi-root passes), CC or PageRank (runs)");
        return CGB_EINVAL;
    }
    cgb_tuning& slot = g->tune_alg[algorithm];
    const cgb_tuning start = slot;
    cgb_options run_opt{};
    run_opt.struct_size = sizeof(cgb_options);
    run_opt.flags = (algorithm == CGB_CC && (flags & CGB_TUNE_CC_WEAK)) ? CGB_FLAG_CC_WEAK : 0u;
    // score of the graph's current tuning
    auto score = [&](double& ms) -> cgb_status {
        ms = 0;
        if (batch) {
            for (uint32_t s0 = 0; s0 < nroots; s0 += 64) {
                const uint32_t n = std::min(64u, nroots - s0);
                double best_rep = 1e300;
                for (int rep = 0; rep < 3; rep++) {
                    double t = 0;
                    const cgb_status st = cgb_run_batch(g, algorithm, roots + s0, n, nullptr, nullptr, &t);
                    if (st != CGB_OK) return st;
                    if (rep > 0) best_rep = std::min(best_rep, t);
                }
                ms += best_rep;
            }
        } else {
            for (uint32_t i = 0; i < nroots; i++) {
                double best_rep = 1e300;
                for (int rep = 0; rep < 3; rep++) {
                    double t = 0;
                    const cgb_status st =
                        cgb_run(g, algorithm, algorithm == CGB_CC ? 0 : roots[i], &run_opt, nullptr, nullptr, &t);
                    // (PageRank: roots[i] is the iteration count)
                    if (st != CGB_OK) return st;
                    if (rep > 0) best_rep = std::min(best_rep, t);
                }
                ms += best_rep;
            }
        }
        return CGB_OK;
    };
    double cur_ms = 0;
    cgb_status st = score(cur_ms);
    if (st != CGB_OK) return st;
    const double first_ms = cur_ms;
    cgb_tuning cur = start;
    if (batch && algorithm == CGB_SSSP) {
        // the partition's degree buckets propose the starting tile
        uint32_t tile = 0;
        try {
            tile = tile_from_partition(g);
        } catch (const Error& e) {
            set_error(e.msg);
            return e.code;
        }
        if (tile && tile != cur.ms_edges) {
            cgb_tuning cand = cur;
            cand.ms_edges = tile;
            if (valid(cand)) {
                {
                    std::lock_guard<GraphMutex> lock(g->mu);
                    slot = cand;
                }
                double ms = 0;
                st = score(ms);
                std::lock_guard<GraphMutex> lock(g->mu);
                if (st != CGB_OK) {
                    slot = start;
                    return st;
                }
                if (ms < cur_ms) {
                    cur_ms = ms;
                    cur = cand;
                }
                slot = cur;
            }
        }
    }
    for (int sweep = 0; sweep < 2; sweep++) {
        bool moved = false;
        for (const Field& f : fields()) {
            const bool used = algorithm == CGB_CC   ? f.cc
                              : algorithm == CGB_PR ? f.pr
                              : algorithm == CGB_BFS ? (batch ? f.ms_bfs : f.bfs)
                                                     : (batch ? f.ms_sssp : f.sssp);
            if (!used) continue;
            for (uint32_t v : f.values) {
                if (cur.*(f.member) == v) continue;
                cgb_tuning cand = cur;
                cand.*(f.member) = v;
                if (!valid(cand)) continue;
                {
                    std::lock_guard<GraphMutex> lock(g->mu);
                    slot = cand;
                }
                double ms = 0;
                st = score(ms);
                if (st != CGB_OK) {
                    std::lock_guard<GraphMutex> lock(g->mu);
                    slot = start;
                    return st;
                }
                if (ms < cur_ms) {
                    cur_ms = ms;
                    cur = cand;
                    moved = true;
                }
            }
            std::lock_guard<GraphMutex> lock(g->mu);
            slot = cur;
        }
        if (!moved) break;
    }
    {
        std::lock_guard<GraphMutex> lock(g->mu);
        slot = (flags & CGB_TUNE_KEEP_DEFAULT) ? start : cur;
    }
    if (best) *best = cur;
    if (best_ms) *best_ms = cur_ms;
    if (start_ms) *start_ms = first_ms;
    return CGB_OK;
}

}  // extern "C"
