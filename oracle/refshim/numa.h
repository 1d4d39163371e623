/* Test-infrastructure shim: lets the reference's CPU engine build on a host
 * without libnuma. One NUMA node; node-local allocation is plain malloc. */
#pragma once
#include <stdlib.h>
#include <string.h>
static inline int numa_available(void) { return 0; }
static inline int numa_num_configured_nodes(void) { return 1; }
static inline int numa_max_node(void) { return 0; }
static inline int numa_run_on_node(int node) { (void)node; return 0; }
static inline void* numa_alloc_onnode(size_t size, int node) { (void)node; return malloc(size); }
static inline void* numa_alloc_local(size_t size) { return malloc(size); }
static inline void numa_free(void* p, size_t size) { (void)size; free(p); }
static inline void numa_tonode_memory(void* p, size_t size, int node) { (void)p; (void)size; (void)node; }
static inline int numa_node_of_cpu(int cpu) { (void)cpu; return 0; }
static inline int numa_num_configured_cpus(void) { return 1; }
