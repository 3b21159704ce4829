// pm_batch.cu -- batched workloads on the engine: multi-source BFS with one
// bit per source in a uint64 word per vertex.
#include "pm_graph.cuh"

namespace pm {

// ===========================================================================
// Multi-source BFS, up to 64 sources (BFS_F of numa-BFS.C:59-79 with the
// parent test replaced by per-source visited bits).  front[v] / next[v] hold
// the sources whose frontier contains v; visited[v] the sources that reached
// v; depth[l * n + v] is v's level from source l.
// Dense rounds: next[v] = OR of front over in-neighbours, minus visited[v]
// (a pull-reduce with OR; commit records the new bits and their depth).
// Sparse rounds: every frontier vertex ORs its word into its out-neighbours'
// next words; a vertexMap over the output queue then records them.
// ===========================================================================
using u64 = unsigned long long;

__device__ __forceinline__ void msbfs_record(u64 nb, int32_t *depth, int64_t n, int v, int32_t level) {
  while (nb) {
    const int l = __ffsll((long long)nb) - 1;
    nb &= nb - 1;
    depth[(int64_t)l * n + v] = level;
  }
}

struct MSBFS_F {
  const u64 *front;
  u64 *next;
  u64 *visited;
  int32_t *depth;
  int64_t n;
  int32_t level;
  u64 full;
  using Acc = u64;
  __device__ __forceinline__ bool cond(int d) const { return *((volatile u64 *)visited + d) != full; }
  __device__ __forceinline__ bool updateAtomic(int s, int d, int) const {
    const u64 x = __ldg(front + s) & ~*((volatile u64 *)visited + d);
    if (!x) return false;
    atomicOr(next + d, x);
    return true;
  }
  __device__ __forceinline__ Acc identity() const { return 0ull; }
  __device__ __forceinline__ Acc edge(int s, int, int) const { return __ldg(front + s); }
  __device__ __forceinline__ Acc combine(Acc a, Acc b) const { return a | b; }
  __device__ __forceinline__ bool commit(int d, Acc acc, double &) const {
    const u64 nb = acc & ~visited[d];
    next[d] = nb;
    if (nb) {
      visited[d] |= nb;
      msbfs_record(nb, depth, n, d, level);
    }
    return nb != 0;
  }
};

// Records the bits that a sparse round ORed into next[v].
struct MSBFS_Commit {
  u64 *next;
  u64 *visited;
  int32_t *depth;
  int64_t n;
  int32_t level;
  __device__ __forceinline__ void operator()(int v) const {
    const u64 nb = next[v] & ~visited[v];
    next[v] = nb;
    if (nb) {
      visited[v] |= nb;
      msbfs_record(nb, depth, n, v, level);
    }
  }
};

__global__ void k_msbfs_seed(const int32_t *sources, int k, u64 *front, u64 *visited, uint32_t *bits,
                             int32_t *depth, int64_t n) {
  const int l = threadIdx.x;
  if (l < k) {
    const int v = sources[l];
    atomicOr(front + v, 1ull << l);
    atomicOr(visited + v, 1ull << l);
    atomicOr(bits + (v >> 5), 1u << (v & 31));
    depth[(int64_t)l * n + v] = 0;
  }
}

// reached = sum popc(visited), edges = sum outdeg(v) * popc(visited[v])
__global__ void k_msbfs_totals(const u64 *visited, const int32_t *out_off, int64_t n, Counters *cnt) {
  unsigned long long r = 0, e = 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
    const int c = __popcll(visited[v]);
    r += c;
    e += (unsigned long long)c * (unsigned long long)(out_off[v + 1] - out_off[v]);
  }
  r = warp_sum(r);
  e = warp_sum(e);
  if (lane_id() == 0 && r) {
    atomicAdd(&cnt->size, r);
    atomicAdd(&cnt->edges, e);
  }
}

void run_msbfs(pm_graph *g, const int32_t *d_sources, int k, int32_t *d_depth, int64_t threshold,
               pm_traversal_stats *st) {
  Engine &E = g->E;
  const int64_t n = g->n;
  u64 *front = (u64 *)g->scratch_buf(0, (size_t)n * 8);
  u64 *next = (u64 *)g->scratch_buf(1, (size_t)n * 8);
  u64 *visited = (u64 *)g->scratch_buf(2, (size_t)n * 8);
  PM_CUDA(cudaMemsetAsync(front, 0, (size_t)n * 8, E.stream));
  PM_CUDA(cudaMemsetAsync(visited, 0, (size_t)n * 8, E.stream));
  PM_CUDA(cudaMemsetAsync(d_depth, 0xff, (size_t)n * k * 4, E.stream));
  VertexSubset cur = g->subset(0), nxt = g->subset(1);
  PM_CUDA(cudaMemsetAsync(cur.bits, 0, cur.words() * 4, E.stream));
  PM_LAUNCH(k_msbfs_seed, 1, 64, 0, E.stream, d_sources, k, front, visited, cur.bits, d_depth, n);
  cur.has_queue = false;
  subset_recount(E, cur);
  const u64 full = k == 64 ? ~0ull : ((1ull << k) - 1ull);
  pm_traversal_stats s{};
  E.tag = "bfs_multi";
  for (int32_t level = 1; cur.size > 0; ++level) {
    PM_CUDA(cudaMemsetAsync(next, 0, (size_t)n * 8, E.stream));
    bool dense = false;
    edgeMapReduce<int>(E, cur, MSBFS_F{front, next, visited, d_depth, n, level, full}, nxt, threshold,
                       nullptr, nullptr, &dense);
    if (!dense) vertexMap(E, nxt, MSBFS_Commit{next, visited, d_depth, n, level});
    s.rounds++;
    s.dense_rounds += dense;
    std::swap(front, next);
    std::swap(cur, nxt);
  }
  PM_CUDA(cudaMemsetAsync(E.d_cnt + 2, 0, sizeof(Counters), E.stream));
  PM_LAUNCH(k_msbfs_totals, E.grid_for(n, 256, 8), 256, 0, E.stream, visited, E.g.out.off, n, E.d_cnt + 2);
  const Counters *h = E.read_counters();
  s.reached = (int64_t)h[2].size;
  s.edges_visited = (int64_t)h[2].edges;
  if (st) *st = s;
}

}  // namespace pm
