/* Minimal libnuma stand-in so the reference compiles where libnuma is absent
 * (test infrastructure for oracle/_ref only).  Single-node semantics:
 * page-aligned allocation and a no-op node binding. */
#ifndef THV_REF_NUMA_SHIM_H
#define THV_REF_NUMA_SHIM_H
#include <stdlib.h>
#include <string.h>
static inline void *numa_alloc_onnode(size_t size, int node) {
  (void)node;
  void *p = NULL;
  if (posix_memalign(&p, 4096, size ? size : 4096) != 0) return NULL;
  memset(p, 0, size);
  return p;
}
static inline int numa_run_on_node(int node) { (void)node; return 0; }
#endif
