/* Test-infrastructure shim: only the reference's edge-list loader names this
 * type, and the oracle harness runs that loader with one OpenMP thread, so
 * its appends from the parallel loop never race. */
#pragma once
#include <vector>
namespace tbb { template <typename T> using concurrent_vector = std::vector<T>; }
