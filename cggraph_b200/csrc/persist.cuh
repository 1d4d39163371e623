// Device-resident frontier loops for small frontiers (high-diameter graphs).
//
// A road-like grid runs thousands of BFS levels / SSSP rounds whose
// frontiers hold a few thousand vertices; a host-driven loop then pays one
// launch + one device-to-host read + one synchronisation (tens of
// microseconds) per level for a few microseconds of work.  These kernels run
// many levels in one cooperative launch, separated by a grid-wide barrier,
// and return to the host when the frontier outgrows `nf_exit` (the host
// loop's binned / bottom-up kernels then take over), when it empties, or
// after `max_levels`.
//
// Counters rotate over three slots: level L appends to slot (L+1)%3, reads
// its own size from slot L%3, and zeroes slot (L+2)%3, which nobody touches
// during level L -- so one barrier per level suffices.  The barrier's spin
// is bounded: on expiry it sets `status` and every CTA leaves the loop.
#pragma once

#include <algorithm>

#include "engine.cuh"

namespace cgb {

constexpr uint32_t kBarrierSpins = 1u << 22;  // mostly x ~64 ns: gives up after ~0.3 s
constexpr int kClusterThreads = 1024;          // threads per CTA of the cluster level loop

// Host-visible state of a device-resident loop.
struct PersistState {
    uint32_t qlen[3];          // rotating queue lengths (see file comment)
    uint32_t bar_count, bar_gen;
    uint32_t status;           // 1 = a barrier gave up, 2 = queue overflow
    uint32_t levels;           // levels run by the launch
    uint32_t cur;              // queue index holding the frontier on exit
    uint32_t nf;               // frontier size on exit
    uint32_t max_deg[3];       // rotating: max out-degree of the next frontier
    unsigned long long medges[3];  // rotating: out-edges of the next frontier
    unsigned long long added;  // sum of the frontier sizes of the levels run
    unsigned long long scouts; // sum of their out-edge counts
};

// Extra state of the whole-device SSSP (k_sssp_device).  Every field
// rotates over the three slots of the queue lengths, so that what a round
// reads is never written during that round.
struct PersistSssp {
    unsigned long long thr[3];  // threshold of the round
    uint32_t min_far[3];        // smallest far distance seen by a split
    uint32_t far_delta[3];      // change of the far-bitmap population made by an expansion round (mod 2^32)
    uint32_t kept[3];           // far-bitmap population left by a split round (a recount)
    uint32_t split[3];          // 1: the round was a split (kept holds the population)
    // on exit: vertices left in the far bitmap, and the lower bound of the
    // bucket of the last split (0 if none ran)
    uint32_t far_left;
    unsigned long long bucket_lo;
};

// A graph's device-resident loop state (g->persist): the loop counters,
// then the whole-device SSSP's bucket state.
struct PersistBlock {
    PersistState st;
    PersistSssp sx;
};

struct PersistResult {
    uint32_t levels = 0;       // levels (rounds) run
    uint32_t cur = 0;          // queue index holding the frontier on exit
    uint32_t nf = 0;           // frontier size on exit
    uint32_t max_deg = 0;      // its max out-degree (BFS)
    unsigned long long scout = 0;   // its out-edges (BFS)
    unsigned long long added = 0;   // sum of the frontier sizes run
    unsigned long long scouts = 0;  // sum of their out-edges (BFS)
};

// The host loops enter these device-resident loops for frontiers of at
// most cgb_tuning.persist_enter vertices whose lists are all shorter than
// cgb_tuning.persist_deg edges.

// Runs BFS top-down levels on the device from the frontier q[cur][0, nf)
// (level `level`, out-edges `scout`, longest list max_deg) until it empties,
// exceeds nf_exit vertices, scout_exit out-edges or a list of deg_exit
// edges, or max_levels levels have run.
PersistResult bfs_persistent(cgb_graph* g, uint32_t cur, uint32_t nf, unsigned long long scout, uint32_t max_deg,
                             uint32_t level, uint32_t nf_exit, unsigned long long scout_exit, uint32_t deg_exit,
                             uint32_t max_levels);

// One cooperative launch of k_bfs_persistent with no exit threshold, from
// the state's qlen[0] roots in q[0] (graph batches).
void launch_bfs_unbounded(cgb_graph* g, PersistState* st);
// One cooperative launch of the whole-device SSSP (graph batches).  Expects
// dist, the far bitmap, slot 1 of the near bitmaps (aux_bm) and `sx` reset,
// and the roots in q[0] (qlen[0]).
void launch_sssp_device(cgb_graph* g, uint32_t* far_bm, uint32_t delta, PersistState* st, PersistSssp* sx);

// The rest of one SSSP run on the device, from the host loop's state: the
// near queue q[cur][0, nf) (longest list max_deg) at threshold thr, nfar
// vertices in far_bm, bucket width delta.  Near rounds and bucket splits
// alternate in one cooperative launch until the run ends, a round's
// frontier exceeds nf_exit vertices or holds a list of deg_exit edges or
// more, or max_rounds rounds have run; the state the host loop continues
// from is returned (thr: the threshold of the next round; nfar; bucket_lo).
struct SsspTail {
    PersistResult r;
    uint64_t thr = 0, bucket_lo = 0;
    uint32_t nfar = 0;
};
SsspTail sssp_device_tail(cgb_graph* g, uint32_t cur, uint32_t nf, uint32_t max_deg, uint64_t thr, uint32_t nfar,
                          uint64_t bucket_lo, uint32_t* far_bm, uint32_t delta, uint32_t nf_exit, uint32_t deg_exit,
                          uint32_t max_rounds);

// Warp-aggregated append into a device-resident loop's queue (every lane
// calls it); past `cap` the loop's status records an overflow.
__device__ __forceinline__ void append(bool pred, uint32_t item, uint32_t* q, uint32_t* ctr, uint32_t cap,
                                       PersistState* st)
{
    const uint32_t want = __ballot_sync(0xffffffffu, pred);
    if (!want) return;
    const uint32_t leader = __ffs(want) - 1;
    uint32_t base = 0;
    if (lane_id() == leader) base = atomicAdd(ctr, (uint32_t)__popc(want));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (pred) {
        const uint32_t idx = base + __popc(want & lanemask_lt());
        if (idx < cap) q[idx] = item;
        else atomicOr(&st->status, 2u);
    }
}

// Grid-wide barrier (every CTA of a cooperative launch must call it).
// Returns false when the wait gave up after `spins` polls (status set by the
// CTA that gave up).
__device__ __forceinline__ bool grid_barrier(PersistState* st, uint32_t spins_max = kBarrierSpins)
{
    __shared__ uint32_t s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile uint32_t* gen = &st->bar_gen;
        const uint32_t g0 = *gen;
        __threadfence();
        const uint32_t arrived = atomicAdd(&st->bar_count, 1u);
        uint32_t ok = 1;
        if (arrived == gridDim.x - 1) {
            st->bar_count = 0;
            __threadfence();
            atomicAdd(&st->bar_gen, 1u);
        } else {
            uint32_t spins = 0;
            while (*gen == g0) {
                if (++spins > spins_max) {
                    atomicOr(&st->status, 1u);
                    ok = 0;
                    break;
                }
                if (spins > 1024) __nanosleep(64);  // spin tight first: levels are short
            }
        }
        __threadfence();
        s_ok = ok && !(*(volatile uint32_t*)&st->status);
    }
    __syncthreads();
    return s_ok;
}

// Self-check of the barrier's bounded wait: one cooperative launch (one CTA
// per SM) in which CTA 0 never arrives, so every other CTA gives up after
// spin_limit polls and sets the status; returns CGB_ETIMEOUT when they did.
// No wait in it is unbounded.
cgb_status barrier_timeout_check(uint32_t spin_limit);

// Cooperative grid of `kernel` with kBlock threads: one CTA per SM (enough
// threads for the frontiers these loops take, and the fewest arrivals per
// barrier), checked against the occupancy limit.
template <typename K>
inline uint32_t cooperative_grid(K kernel)
{
    int dev = 0, sms = 0, per_sm = 0;
    CGB_CUDA_TRY(cudaGetDevice(&dev));
    CGB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CGB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBlock, 0));
    CGB_REQUIRE(per_sm >= 1, CGB_EUNSUPPORTED, "device-resident loop does not fit on an SM");
    return (uint32_t)sms;
}

}  // namespace cgb
