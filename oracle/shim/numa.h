/*
 * Single-node stand-in for the libnuma API, used only to compile the
 * reference Polymer sources as a CPU checker (libnuma is not installed in
 * this image).  Every call behaves as on a machine with ONE NUMA node:
 * allocations are anonymous zero-filled mappings (what numa_alloc_local
 * returns), placement and binding calls do nothing, and the CPU count is
 * taken from PM_REF_THREADS (default: all online CPUs), which the reference
 * uses as CORES_PER_NODE worker threads.  Test infrastructure, not product.
 */
#ifndef PM_ORACLE_NUMA_SHIM_H
#define PM_ORACLE_NUMA_SHIM_H
#include <stdlib.h>
#include <sys/mman.h>
#include <unistd.h>

struct bitmask { unsigned long size; unsigned long *maskp; };
static struct bitmask pm_shim_all_nodes_ = {1, 0};
static struct bitmask *numa_all_nodes_ptr = &pm_shim_all_nodes_;

static inline void *numa_alloc_local(size_t size) {
  void *p = mmap(0, size ? size : 1, PROT_READ | PROT_WRITE,
                 MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
  return p == MAP_FAILED ? 0 : p;
}
static inline void numa_free(void *p, size_t size) { if (p) munmap(p, size ? size : 1); }
static inline void numa_tonode_memory(void *p, size_t size, int node) { (void)p; (void)size; (void)node; }
static inline int numa_num_configured_nodes(void) { return 1; }
static inline int numa_num_configured_cpus(void) {
  const char *e = getenv("PM_REF_THREADS");
  if (e && atoi(e) > 0) return atoi(e);
  long c = sysconf(_SC_NPROCESSORS_ONLN);
  return c > 0 ? (int)c : 1;
}
static inline struct bitmask *numa_parse_nodestring(const char *s) { (void)s; return &pm_shim_all_nodes_; }
static inline void numa_bind(struct bitmask *m) { (void)m; }
static inline void numa_set_interleave_mask(struct bitmask *m) { (void)m; }
#endif
