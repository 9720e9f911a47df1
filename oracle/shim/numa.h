/* Test-infrastructure shim (oracle build only): libnuma is not installed.
 * The pS5 entry points used by the oracle run on one NUMA node, so placement
 * calls are no-ops and node-local allocation is plain malloc. */
#pragma once
#include <stdlib.h>
static inline int numa_run_on_node(int node) { (void)node; return 0; }
static inline void numa_set_preferred(int node) { (void)node; }
static inline int numa_num_configured_nodes(void) { return 1; }
static inline void numa_tonode_memory(void* p, size_t s, int node) { (void)p; (void)s; (void)node; }
static inline void* numa_alloc_onnode(size_t s, int node) { (void)node; return malloc(s); }
static inline void numa_free(void* p, size_t s) { (void)s; free(p); }
struct bitmask { unsigned long size; unsigned long* maskp; };
static struct bitmask* const numa_all_nodes_ptr = 0;
static struct bitmask* const numa_all_cpus_ptr = 0;
static inline void numa_set_interleave_mask(struct bitmask* m) { (void)m; }
static inline void numa_interleave_memory(void* p, size_t s, struct bitmask* m) { (void)p; (void)s; (void)m; }
static inline void numa_set_strict(int flag) { (void)flag; }
