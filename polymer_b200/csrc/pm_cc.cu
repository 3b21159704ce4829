// pm_cc.cu -- Connected Components of a symmetric graph by union-find.
//
// numa-Components.C computes labels by min-label propagation (CC_F
// 55-106, loop 233-281): labels start at the vertex id (387-391) and each
// round lowers a label to the least label among its neighbours.  On a
// symmetric graph the fixpoint is the minimum vertex id of each connected
// component, a value independent of the schedule, so any exact algorithm
// that yields that minimum gives the reference's labels bit for bit.
//
// This file computes it with a concurrent union-find in the scheme of
// Afforest (Sutton, Ben-Nun and Barak, IPDPS 2018):
//   1. every vertex links to its first kSampleRounds neighbours (one round
//      per neighbour index, a compression after each);
//   2. the root shared by most of kModeSamples fixed vertices is taken as
//      the largest intermediate component L;
//   3. every vertex whose root is not L links to its remaining neighbours.
//      A vertex of L skips them: an edge between L and another component
//      is also stored the other way round (the graph is symmetric), and the
//      other endpoint, not in L, links it; an edge inside L needs nothing;
//   4. a last compression points every vertex at its root.
// Links always hang the larger root under the smaller one with a CAS, so
// parent[v] <= v holds throughout, a root is the least id of its tree, and
// the final root of each component is its minimum vertex id: exactly the
// labels of the propagation.  The parent array is the caller's label array.
// Label propagation stays available (tunable PM_TUNE_CC_MODE = 1) and is
// what directed and partitioned handles use.
#include <algorithm>

#include "pm_graph.cuh"

namespace pm {

constexpr int kSampleRounds = 2;
constexpr int kModeSamples = 1024;
constexpr int kSlotCcMode = 31;  // scratch slot of the largest component's root

#define GRID_STRIDE(i, count)                                                       \
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (count);     \
       i += (int64_t)gridDim.x * blockDim.x)

__device__ __forceinline__ int32_t ld_parent(const int32_t *p, int32_t v) {
  return *((volatile const int32_t *)p + v);
}

// Hangs the root of u's tree and the root of v's tree together, the larger
// under the smaller (Afforest's link).
__device__ __forceinline__ void uf_link(int32_t *parent, int32_t u, int32_t v) {
  int32_t p1 = ld_parent(parent, u), p2 = ld_parent(parent, v);
  while (p1 != p2) {
    const int32_t high = max(p1, p2), low = min(p1, p2);
    const int32_t p_high = ld_parent(parent, high);
    if (p_high == low) break;  // already hung there
    if (p_high == high && atomicCAS(parent + high, high, low) == high) break;  // high was a root
    p1 = ld_parent(parent, ld_parent(parent, high));
    p2 = ld_parent(parent, low);
  }
}

__device__ __forceinline__ int32_t uf_root(const int32_t *parent, int32_t v) {
  int32_t p = ld_parent(parent, v);
  while (true) {
    const int32_t q = ld_parent(parent, p);
    if (q == p) return p;
    p = q;
  }
}

__global__ void k_uf_init(int32_t *parent, int64_t n) {
  GRID_STRIDE(v, n) parent[v] = (int32_t)v;
}

// Round r of the sampling: v links to its r-th neighbour (when it has one).
__global__ void k_uf_sample(GraphView g, int32_t *parent, int r, unsigned long long *edges) {
  unsigned long long mine = 0;
  GRID_STRIDE(v, g.n) {
    const int32_t o0 = __ldg(g.out.off + v), o1 = __ldg(g.out.off + v + 1);
    if (o1 - o0 > r) {
      uf_link(parent, (int32_t)v, checked_id(g, __ldg(g.out.idx + o0 + r)));
      ++mine;
    }
  }
  mine = warp_sum(mine);
  if (lane_id() == 0 && mine) atomicAdd(edges, mine);
}

// parent[v] := root of v.  Writes only v's own entry; a concurrent reader of
// parent[v] sees either the old value or the root, both ancestors of v.
__global__ void k_uf_compress(int32_t *parent, int64_t n) {
  GRID_STRIDE(v, n) {
    const int32_t r = uf_root(parent, (int32_t)v);
    if (ld_parent(parent, (int32_t)v) != r) parent[v] = r;
  }
}

// The root most of kModeSamples spread vertices share (ties: the smaller
// root), one CTA of kModeSamples threads; the vertices are v = i * n / S.
__global__ void __launch_bounds__(kModeSamples) k_uf_mode(const int32_t *parent, int64_t n, int32_t *mode) {
  __shared__ int32_t s_root[kModeSamples];
  __shared__ unsigned long long s_best;
  const int i = threadIdx.x;
  const int64_t v = (int64_t)i * n / kModeSamples;
  s_root[i] = uf_root(parent, (int32_t)v);
  if (i == 0) s_best = ~0ull;
  __syncthreads();
  int cnt = 0;
  for (int j = 0; j < kModeSamples; ++j) cnt += s_root[j] == s_root[i];
  // key: larger count first, then smaller root
  const unsigned long long key = ((unsigned long long)(kModeSamples - cnt) << 32) | (uint32_t)s_root[i];
  atomicMin(&s_best, key);
  __syncthreads();
  if (i == 0) *mode = (int32_t)(uint32_t)(s_best & 0xffffffffull);
}

// Step 3: a warp takes 32 vertices; each vertex outside the largest
// component with neighbours past the sampled ones has them linked by the
// whole warp, one vertex after another.
__global__ void k_uf_rest(GraphView g, int32_t *parent, const int32_t *mode, unsigned long long *edges) {
  const int lane = lane_id();
  const int32_t L = *mode;
  unsigned long long mine = 0;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t base = ((int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32; base < g.n;
       base += warps * 32) {
    const int64_t v = base + lane;
    int32_t o0 = 0, o1 = 0;
    bool todo = false;
    if (v < g.n) {
      o0 = __ldg(g.out.off + v) + kSampleRounds;
      o1 = __ldg(g.out.off + v + 1);
      todo = o1 > o0 && uf_root(parent, (int32_t)v) != L;
    }
    unsigned bal = __ballot_sync(0xffffffffu, todo);
    while (bal) {
      const int l = __ffs(bal) - 1;
      bal &= bal - 1;
      const int32_t u = (int32_t)(base + l);
      const int32_t e0 = __shfl_sync(0xffffffffu, o0, l), e1 = __shfl_sync(0xffffffffu, o1, l);
      for (int32_t e = e0 + lane; e < e1; e += 32) {
        uf_link(parent, u, checked_id(g, __ldg(g.out.idx + e)));
        ++mine;
      }
    }
  }
  mine = warp_sum(mine);
  if (lane == 0 && mine) atomicAdd(edges, mine);
}

void run_cc_union_find(pm_graph *g, int32_t *d_labels, pm_traversal_stats *st) {
  Engine &E = g->E;
  const int64_t n = g->n;
  E.reset_counters();
  unsigned long long *edges = &E.d_cnt->edges;
  int32_t *mode = (int32_t *)g->scratch_buf(kSlotCcMode, 16);
  E.tag = "cc";
  E.prof.begin(E.tag, E.stream);
  const int grid = E.grid_for(n, 256, 16);
  PM_LAUNCH(k_uf_init, grid, 256, 0, E.stream, d_labels, n);
  for (int r = 0; r < kSampleRounds; ++r) {
    PM_LAUNCH(k_uf_sample, grid, 256, 0, E.stream, E.g, d_labels, r, edges);
    PM_LAUNCH(k_uf_compress, grid, 256, 0, E.stream, d_labels, n);
  }
  PM_LAUNCH(k_uf_mode, 1, kModeSamples, 0, E.stream, d_labels, n, mode);
  PM_LAUNCH(k_uf_rest, E.grid_for((n + 31) / 32 * 32, 256, 16), 256, 0, E.stream, E.g, d_labels, mode, edges);
  PM_LAUNCH(k_uf_compress, grid, 256, 0, E.stream, d_labels, n);
  E.prof.end(E.stream);
  const Counters *h = E.read_counters();
  if (st) {
    pm_traversal_stats s{};
    s.rounds = kSampleRounds + 1;  // union-find passes over the vertices
    s.dense_rounds = 0;
    s.edges_visited = (int64_t)h[0].edges;  // edges linked
    s.reached = n;
    *st = s;
  }
}

}  // namespace pm
