// Per-iteration schedule policy: a small FP32 MLP (24 features -> 64 -> 64
// -> 14 predicted log-costs) trained on the engine's own counterfactual
// traces, with the Beamer / fixed-delta / size-threshold heuristics as
// fallback.
#pragma once

#include "engine.cuh"

namespace cgb {

constexpr int kPolicyFeatures = CGB_POLICY_FEATURES;  // 24
constexpr int kPolicyHidden = 64;
constexpr int kPolicyOutputs = CGB_POLICY_OUTPUTS;    // 14
// parameter layout: W1[24][64] b1[64] W2[64][64] b2[64] W3[64][14] b3[14]
constexpr int kPolicyParams = CGB_POLICY_PARAMS;
static_assert(kPolicyParams == kPolicyFeatures * kPolicyHidden + kPolicyHidden + kPolicyHidden * kPolicyHidden +
                                   kPolicyHidden + kPolicyHidden * kPolicyOutputs + kPolicyOutputs,
              "parameter count");

// Output heads: predicted log-cost of each choice (lower is better).
constexpr int kOutPush = 0, kOutPull = 1;  // BFS next level: binned push / bottom-up pull
constexpr int kOutPushChunked = 9;         // BFS next level: push, every list >= 32 edges chunked
constexpr int kOutDelta0 = 2;              // SSSP delta x delta_scale(i) for the rest of the run
// SSSP next near round: sparse frontier (binned push), sparse frontier with
// chunked lists, dense frontier, pull
constexpr int kOutRound0 = 10;
constexpr int kNumRoundChoices = 4;
enum RoundVariant { kRoundPush = 0, kRoundPushChunked = 1, kRoundDense = 2, kRoundPull = 3 };
constexpr int kNumDeltaChoices = 7;        // x {1/4, 1/2, 1, 2, 4, 8, 16}
constexpr int kDeltaUnit = 2;              // index of x1 (the heuristic delta)
__host__ __device__ inline float delta_scale(int i) { return 0.25f * (float)(1 << i); }

// Raw quantities at a decision point.  The same function turns them into
// features on the host (trace logging) and on the device (inference).
struct FeatIn {
    uint32_t alg;          // CGB_BFS / CGB_SSSP
    uint32_t iteration;
    int32_t prev_dir;      // BFS: last level was pull (1) or push (0)
    uint32_t symmetric;
    double V, E;
    double nf, mf;         // frontier vertices / out-edges of the frontier
    double unvisited_v, unvisited_e;
    double max_deg, prev_nf;
    double delta, base_delta;  // SSSP
    double far_count, settled; // SSSP
};

__host__ __device__ inline float lg(double x) { return (float)log1p(x > 0 ? x : 0.0); }

__host__ __device__ inline void policy_features(const FeatIn& in, float* f)
{
    const double V = in.V > 1 ? in.V : 1, E = in.E > 1 ? in.E : 1;
    const double avg = E / V;
    f[0] = lg(in.nf) / lg(V);
    f[1] = lg(in.mf) / lg(E);
    f[2] = (float)(in.nf / V);
    f[3] = (float)(in.mf / E);
    f[4] = (float)(in.unvisited_v / V);
    f[5] = (float)(in.unvisited_e / E);
    f[6] = lg(in.max_deg) / lg(E);
    f[7] = lg(in.mf / (in.nf > 1 ? in.nf : 1)) / lg(avg * 64 + 1);
    f[8] = lg(avg) / 8.f;
    f[9] = (float)(in.iteration > 256 ? 256 : in.iteration) / 64.f;
    f[10] = (float)in.prev_dir;
    f[11] = 1.f;
    f[12] = (float)(lg(in.nf) - lg(in.prev_nf)) / 8.f;
    f[13] = (float)(lg(in.mf * 15.0) - lg(in.unvisited_e)) / 8.f;  // Beamer alpha test, in logs
    f[14] = (float)(lg(in.nf * 18.0) - lg(V)) / 8.f;               // Beamer beta test, in logs
    f[15] = (float)in.symmetric;
    f[16] = in.alg == CGB_BFS ? 1.f : 0.f;
    f[17] = in.alg == CGB_SSSP ? 1.f : 0.f;
    f[18] = in.base_delta > 0 ? (float)(log(in.delta / in.base_delta) / log(4.0)) : 0.f;
    f[19] = (float)(in.far_count / V);
    f[20] = lg(in.far_count) / lg(V);
    f[21] = lg(V) / 32.f;
    f[22] = lg(E) / 32.f;
    f[23] = (float)(in.settled / V);
}

struct Policy;

// The policy loaded on the current device, or nullptr (heuristic fallback).
Policy* policy_get();

// The policy for a learned run on g: none below kPolicyMinEdges edges.  Each
// decision costs about 10 us of inference and a read-back; on such graphs a
// whole BFS takes about half a millisecond, and the measured choices were
// worth less (RMAT-20 BFS ran 0.86-0.91x under the network).
constexpr uint64_t kPolicyMinEdges = 1ull << 26;

// Which of the network's decisions a learned run applies.  The delta is
// trained on the cost of the whole rest of the run.  A BFS level's or an
// SSSP round's variant is trained on that step alone, and a step's choice
// also shapes the next one (a dense round hands the next round a queue in
// vertex order, a pushed one in discovery order): the step costs predicted
// the trials faithfully, yet following them made RMAT-23/24 SSSP 0.82-0.89x
// and BFS 0.91-0.97x of the heuristic.  Those heads are trained and
// evaluated (cgb_policy_collect, cgb_policy_forward) but not applied.
constexpr bool kPolicyLevels = false;  // BFS push / pull and expansion variant
constexpr bool kPolicyRounds = false;  // SSSP round variant
Policy* policy_for(const cgb_graph* g);
const float* policy_params_device(Policy* p);

// Queues the network on the graph's stream: features from `in` (with the
// counters of the level or round just run patched in when `patch` is 1 for
// BFS -- next frontier size, its out-edges and max degree, vertices found --
// or 2 for an SSSP near round -- next near queue, its out-edges and max
// degree, far count), outputs into the DevCounters' policy_out, read back by
// the next sync_counters.
void policy_enqueue(Policy* p, cgb_graph* g, const FeatIn& in, int patch, bool was_pull, int out_q);

// Appends one counterfactual sample (features of `in`, measured ms of the
// choices flagged in `have`) to g->collect.
void policy_log_sample(cgb_graph* g, const FeatIn& in, const float* ms, const bool* have);

// Decisions from the outputs read back with the counters; -1 = no
// confident choice (use the heuristic).  `heur` is the heuristic's own
// choice, which another choice must beat by the margin.
int policy_pick_bfs_level(const float* out, int heur);  // 0 push, 1 pull, 2 push chunked
int policy_pick_delta(const float* out);
int policy_pick_round(const float* out, int heur);  // a RoundVariant

}  // namespace cgb
