/* Test-infrastructure shim: only the reference's edge-list loader names this
 * type and the oracle harness never calls that loader. */
#pragma once
#include <vector>
namespace tbb { template <typename T> using concurrent_vector = std::vector<T>; }
