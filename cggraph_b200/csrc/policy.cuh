// Per-iteration schedule policy (learned MLP with heuristic fallback).
#pragma once

#include "engine.cuh"

namespace cgb {

constexpr int kPolicyFeatures = 24;

struct Policy;

// The loaded policy, or nullptr when none is loaded (callers then fall back
// to the heuristic).
Policy* policy_get();

// Fills the 24 features of one iteration.
void policy_features(float* feat, int algorithm, const cgb_graph* g, uint64_t frontier_vertices,
                     uint64_t frontier_edges, uint64_t unvisited_vertices, uint64_t unvisited_edges,
                     uint32_t max_frontier_degree, uint32_t iteration, int prev_direction, uint32_t delta);

// 0 = push, 1 = pull; -1 = no confident choice (use the heuristic).
int policy_choose_direction(Policy* p, const float* feat);

// Multiplier index for the SSSP delta (see kDeltaScale); -1 = heuristic.
int policy_choose_delta(Policy* p, const float* feat);

}  // namespace cgb
