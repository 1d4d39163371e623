// Per-iteration schedule policy.  Until a trained network is loaded the
// policy declines every choice and the heuristic decides.
#include "policy.cuh"

namespace cgb {

struct Policy {
    int loaded = 0;
};

Policy* policy_get() { return nullptr; }

void policy_features(float* feat, int, const cgb_graph*, uint64_t, uint64_t, uint64_t, uint64_t, uint32_t, uint32_t,
                     int, uint32_t)
{
    for (int i = 0; i < kPolicyFeatures; i++) feat[i] = 0.f;
}

int policy_choose_direction(Policy*, const float*) { return -1; }
int policy_choose_delta(Policy*, const float*) { return -1; }

}  // namespace cgb
