// pm_batch.cu -- batched workloads: multi-source BFS (one bit per source in a
// uint64 word per vertex), multi-source BellmanFord (64 int32 distance lanes
// per vertex), personalised PageRank for 32 seeds, and PageRank on every part
// of a disjoint union in one persistent launch.
#include <cooperative_groups.h>

#include <cub/cub.cuh>

#include "pm_graph.cuh"

namespace cg = cooperative_groups;

namespace pm {

// ===========================================================================
// Multi-source BFS, up to 64 sources (BFS_F of numa-BFS.C:59-79 with the
// parent test replaced by per-source visited bits).  front[v] / next[v] hold
// the sources whose frontier contains v; visited[v] the sources that reached
// v; depth[l * n + v] is v's level from source l.
// Dense rounds: next[v] = OR of front over in-neighbours, minus visited[v]
// (a pull-reduce with OR; commit keeps the new bits).
// Sparse rounds: every frontier vertex ORs its word into its out-neighbours'
// next words; a vertexMap over the output queue then masks them.
// So next[v] ends every level as exactly the sources that reached v at that
// level.  The levels' words stay in a ring of kMsbfsSlots-or-fewer slots and
// the depths are written from them in tiles (k_msbfs_depths): one coalesced
// pass over the k x n output instead of a fill plus one scattered 4-byte
// store per (source, vertex).
// ===========================================================================
using u64 = unsigned long long;

constexpr int kMsbfsSlots = 16;     // level words kept before a flush
constexpr int kMsbfsTile = 128;     // vertices per depth tile (one per thread)

// Depths of the levels L0 .. L0+cnt-1, whose new-bits words sit in ring
// slots (L0 + j) % slots.  first: no depth has been written yet, so the
// block writes all k rows of its tile (-1 where no flushed level has the
// lane) through shared memory, one 128-byte row segment per warp store;
// otherwise only the lanes found are stored, straight to the output.
__global__ void __launch_bounds__(kMsbfsTile) k_msbfs_depths(const u64 *__restrict__ ring, int slots,
                                                             int32_t L0, int cnt, int k, int64_t n,
                                                             bool first, int32_t *__restrict__ depth) {
  __shared__ int32_t tile[64][kMsbfsTile];
  const int t = threadIdx.x;
  const int64_t v0 = (int64_t)blockIdx.x * kMsbfsTile;
  const int64_t v = v0 + t;
  if (first)
    for (int l = 0; l < k; ++l) tile[l][t] = -1;
  if (v < n)
    for (int j = 0; j < cnt; ++j) {
      u64 w = ring[(int64_t)((L0 + j) % slots) * n + v];
      while (w) {
        const int l = __ffsll((long long)w) - 1;
        w &= w - 1;
        if (first)
          tile[l][t] = L0 + j;  // bank t % 32 whatever l is
        else
          depth[(int64_t)l * n + v] = L0 + j;
      }
    }
  if (!first) return;
  __syncthreads();
  if (v < n)
    for (int l = 0; l < k; ++l) depth[(int64_t)l * n + v] = tile[l][t];
}

struct MSBFS_F {
  const u64 *front;
  u64 *next;
  u64 *visited;
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
  __device__ __forceinline__ bool commit(int d, Acc acc, double2 &) const {
    const u64 nb = acc & ~visited[d];
    next[d] = nb;
    if (nb) visited[d] |= nb;
    return nb != 0;
  }
};

// Keeps only the new bits that a sparse round ORed into next[v].
struct MSBFS_Commit {
  u64 *next;
  u64 *visited;
  __device__ __forceinline__ void operator()(int v) const {
    const u64 nb = next[v] & ~visited[v];
    next[v] = nb;
    if (nb) visited[v] |= nb;
  }
};

__global__ void k_msbfs_seed(const int32_t *sources, int k, u64 *front, u64 *visited, uint32_t *bits) {
  const int l = threadIdx.x;
  if (l < k) {
    const int v = sources[l];
    atomicOr(front + v, 1ull << l);
    atomicOr(visited + v, 1ull << l);
    atomicOr(bits + (v >> 5), 1u << (v & 31));
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
  // Level t's new-bits words live in ring slot t % slots (about 1 GiB of
  // ring at most, 3 slots at least: the front, the level being built, and
  // one more so a flush never waits for every level).
  const int slots = (int)std::max<int64_t>(3, std::min<int64_t>(kMsbfsSlots, (int64_t(1) << 30) / (8 * n)));
  u64 *ring = (u64 *)g->scratch_buf(0, (size_t)n * 8 * slots);
  u64 *visited = (u64 *)g->scratch_buf(2, (size_t)n * 8);
  auto slot = [&](int32_t t) { return ring + (int64_t)(t % slots) * n; };
  PM_CUDA(cudaMemsetAsync(slot(0), 0, (size_t)n * 8, E.stream));
  PM_CUDA(cudaMemsetAsync(visited, 0, (size_t)n * 8, E.stream));
  VertexSubset cur = g->subset(0), nxt = g->subset(1);
  PM_CUDA(cudaMemsetAsync(cur.bits, 0, cur.words() * 4, E.stream));
  PM_LAUNCH(k_msbfs_seed, 1, 64, 0, E.stream, d_sources, k, slot(0), visited, cur.bits);
  cur.has_queue = false;
  subset_recount(E, cur);
  const u64 full = k == 64 ? ~0ull : ((1ull << k) - 1ull);
  const unsigned tiles = (unsigned)((n + kMsbfsTile - 1) / kMsbfsTile);
  int32_t flushed = 0;  // levels below this have their depths written
  auto flush = [&](int32_t upto) {  // levels [flushed, upto]
    PM_LAUNCH(k_msbfs_depths, tiles, kMsbfsTile, 0, E.stream, ring, slots, flushed, upto - flushed + 1, k, n,
              flushed == 0, d_depth);
    flushed = upto + 1;
  };
  pm_traversal_stats s{};
  E.tag = "bfs_multi";
  int32_t level = 1;
  for (; cur.size > 0; ++level) {
    if (level - flushed == slots) flush(level - 1);  // slot(level) still holds an unwritten level
    u64 *next = slot(level);
    PM_CUDA(cudaMemsetAsync(next, 0, (size_t)n * 8, E.stream));
    bool dense = false;
    edgeMapReduce<int>(E, cur, MSBFS_F{slot(level - 1), next, visited, full}, nxt, threshold, nullptr, nullptr,
                       &dense);
    if (!dense) vertexMap(E, nxt, MSBFS_Commit{next, visited});
    s.rounds++;
    s.dense_rounds += dense;
    std::swap(cur, nxt);
  }
  flush(level - 1);
  PM_CUDA(cudaMemsetAsync(E.d_cnt + 2, 0, sizeof(Counters), E.stream));
  PM_LAUNCH(k_msbfs_totals, E.grid_for(n, 256, 8), 256, 0, E.stream, visited, E.g.out.off, n, E.d_cnt + 2);
  const Counters *h = E.read_counters();
  s.reached = (int64_t)h[2].size;
  s.edges_visited = (int64_t)h[2].edges;
  if (st) *st = s;
}

// ===========================================================================
// Multi-source BellmanFord, up to 64 sources (BF_F of numa-BellmanFord.C:
// 61-85 with one int32 distance lane per source).  dist is vertex-major,
// 64 lanes per vertex (256 bytes, one warp-wide pair of 128-byte rows);
// active[v] has bit l set when lane l of v fell in the last round.  A round
// follows BF's direction rule on the union frontier (|F| + outdeg(F) >=
// threshold is dense):
//  * dense: a warp owns a CSC row, thread t owns lanes t and t+32; for each
//    in-edge whose source has active lanes it gathers the source's row and
//    relaxes those lanes; the row's new active word is written in full;
//  * sparse: the frontier's out-edges are cut into 32-edge chunks (a scan of
//    the queued out-degrees); for each edge the warp relaxes the active lanes
//    of the target with atomicMin and ORs the lanes that fell into the
//    target's next active word.
// Distances only fall, so reading a row another warp is lowering in the same
// round is harmless: the lower value is a real path length and the lane that
// fell is in the next frontier either way.
// ===========================================================================
constexpr int kLanes = 64;
constexpr int kBfUnroll = 4;      // pull: in-edges whose row gathers are in flight together per warp
constexpr int kBfPushUnroll = 2;  // push: out-edges whose target rows are read together per warp

// active -> queue of frontier vertices with out-edges (and their degrees);
// c->size = |F|, c->edges = outdeg(F), c->aux = queue length.
__global__ void k_bf_multi_frontier(const u64 *__restrict__ active, const int32_t *__restrict__ out_off,
                                    int64_t n, int32_t *__restrict__ queue, int32_t *__restrict__ qdeg,
                                    Counters *c) {
  const int lane = lane_id();
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  unsigned long long size = 0, edges = 0;
  for (int64_t base = ((int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32; base < n;
       base += warps * 32) {
    const int64_t v = base + lane;
    int deg = 0;
    bool act = false;
    if (v < n) {
      act = active[v] != 0ull;
      if (act) deg = __ldg(out_off + v + 1) - __ldg(out_off + v);
    }
    size += act;
    edges += (unsigned)deg;
    const unsigned push = __ballot_sync(0xffffffffu, deg > 0);
    if (push) {
      unsigned long long pos = 0;
      if (lane == 0) pos = atomicAdd(&c->aux, (unsigned long long)__popc(push));
      pos = shfl_idx(pos, 0) + __popc(push & ((1u << lane) - 1u));
      if (deg > 0) {
        queue[pos] = (int32_t)v;
        qdeg[pos] = deg;
      }
    }
  }
  size = warp_sum(size);
  edges = warp_sum(edges);
  if (lane == 0 && size) {
    atomicAdd(&c->size, size);
    atomicAdd(&c->edges, edges);
  }
}

__global__ void __launch_bounds__(256) k_bf_multi_push(const int32_t *__restrict__ out_off,
                                                       const int32_t *__restrict__ out_idx,
                                                       const int32_t *__restrict__ w_out,
                                                       const int32_t *__restrict__ queue,
                                                       const int32_t *__restrict__ qoff, int q, int64_t total,
                                                       int32_t *dist, const u64 *__restrict__ active,
                                                       u64 *next_active) {
  const int lane = lane_id();
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t chunk = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); chunk * 32 < total;
       chunk += warps) {
    const int64_t t0 = chunk * 32;
    // last queue entry whose first edge is <= t0 (qoff is increasing: every
    // queued vertex has at least one out-edge)
    int lo = 0, hi = q - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(qoff + mid) <= t0) lo = mid;
      else hi = mid - 1;
    }
    // queue entries starting inside the chunk mark their first position
    const int bi = lo + 1 + lane;
    unsigned start = 0;
    if (bi < q) {
      const int64_t p = (int64_t)__ldg(qoff + bi) - t0;
      if (p < 32) start = 1u << p;
    }
    start = __reduce_or_sync(0xffffffffu, start);
    const int64_t t = t0 + lane;
    const bool valid = t < total;
    int s = -1, d = 0;
    int32_t w = 0;
    if (valid) {
      const int qi = lo + __popc(start << (31 - lane));
      s = __ldg(queue + qi);
      const int64_t e = (int64_t)__ldg(out_off + s) + (t - __ldg(qoff + qi));
      d = __ldg(out_idx + e);
      w = __ldg(w_out + e);
    }
    const int cnt = (int)min((int64_t)32, total - t0);
    int cur = -1;
    u64 a = 0;
    int32_t slo = 0, shi = 0;
    for (int j0 = 0; j0 < cnt; j0 += kBfPushUnroll) {
      // kBfPushUnroll edges at a time: the targets' rows are read, and their
      // atomics issued, before any result is waited for.
      int dj[kBfPushUnroll];
      int32_t nlo[kBfPushUnroll], nhi[kBfPushUnroll], olo[kBfPushUnroll], ohi[kBfPushUnroll];
#pragma unroll
      for (int u = 0; u < kBfPushUnroll; ++u) {
        const int j = min(j0 + u, cnt - 1);
        const bool take = j0 + u < cnt;
        const int sj = __shfl_sync(0xffffffffu, s, j);
        dj[u] = __shfl_sync(0xffffffffu, d, j);
        const int32_t wj = __shfl_sync(0xffffffffu, w, j);
        if (sj != cur) {
          cur = sj;
          a = __ldg(active + sj);
          slo = dist[(int64_t)sj * kLanes + lane];
          shi = dist[(int64_t)sj * kLanes + 32 + lane];
        }
        nlo[u] = take && ((a >> lane) & 1ull) ? slo + wj : kDevBFInf;
        nhi[u] = take && ((a >> (32 + lane)) & 1ull) ? shi + wj : kDevBFInf;
        olo[u] = nlo[u] < kDevBFInf ? *(volatile int32_t *)(dist + (int64_t)dj[u] * kLanes + lane) : 0;
        ohi[u] = nhi[u] < kDevBFInf ? *(volatile int32_t *)(dist + (int64_t)dj[u] * kLanes + 32 + lane) : 0;
      }
      // A lane below the distance read above lowers it with an atomic
      // whose result is unused and is marked active: it fell, or another
      // push lowered it further meanwhile (an extra relaxation next round,
      // the same distances).
#pragma unroll
      for (int u = 0; u < kBfPushUnroll; ++u) {
        if (nlo[u] < olo[u]) atomicMin(dist + (int64_t)dj[u] * kLanes + lane, nlo[u]);
        if (nhi[u] < ohi[u]) atomicMin(dist + (int64_t)dj[u] * kLanes + 32 + lane, nhi[u]);
      }
#pragma unroll
      for (int u = 0; u < kBfPushUnroll; ++u) {
        const u64 mask = (u64)__ballot_sync(0xffffffffu, nlo[u] < olo[u]) |
                         ((u64)__ballot_sync(0xffffffffu, nhi[u] < ohi[u]) << 32);
        if (lane == 0 && mask) atomicOr(next_active + dj[u], mask);
      }
    }
  }
}

// Relaxes lanes lo / hi of row v over in-edges [e0, e1) whose sources have
// active lanes (one warp; thread t owns lanes t and t + 32).
__device__ __forceinline__ void bf_multi_relax(const int32_t *__restrict__ in_idx,
                                               const int32_t *__restrict__ w_in, const int32_t *dist,
                                               const u64 *__restrict__ active, int64_t e0, int64_t e1,
                                               int32_t &lo, int32_t &hi) {
  const int lane = lane_id();
  for (int64_t base = e0; base < e1; base += 32) {
    const int64_t e = base + lane;
    int s = 0;
    u64 act = 0;
    int32_t w = 0;
    if (e < e1) {
      s = __ldg(in_idx + e);
      act = __ldg(active + s);
      w = __ldg(w_in + e);
    }
    unsigned todo = __ballot_sync(0xffffffffu, act != 0);
    // Up to kBfUnroll active in-edges per step: their row gathers are all
    // issued before the first min consumes one.
    while (todo) {
      int32_t vlo[kBfUnroll], vhi[kBfUnroll];
#pragma unroll
      for (int u = 0; u < kBfUnroll; ++u) {
        const int j = todo ? __ffs(todo) - 1 : 0;
        const bool take = todo != 0;
        todo &= todo - 1;
        const int sj = __shfl_sync(0xffffffffu, s, j);
        const u64 aj = shfl_idx(act, j) & (take ? ~0ull : 0ull);
        const int32_t wj = __shfl_sync(0xffffffffu, w, j);
        vlo[u] = ((aj >> lane) & 1ull) ? dist[(int64_t)sj * kLanes + lane] + wj : kDevBFInf;
        vhi[u] = ((aj >> (32 + lane)) & 1ull) ? dist[(int64_t)sj * kLanes + 32 + lane] + wj : kDevBFInf;
      }
#pragma unroll
      for (int u = 0; u < kBfUnroll; ++u) {
        lo = min(lo, vlo[u]);
        hi = min(hi, vhi[u]);
      }
    }
  }
}

constexpr int kBfPiece = 512;  // in-edges of one warp's piece of a heavy row

// Dense round.  Persistent warps take tickets: the first ones are 512-edge
// pieces of the heavy rows (in-degree > g.heavy_deg; they lower the row with
// atomicMin and OR the fallen lanes into next_active, which starts at zero),
// the rest are merge-path row groups whose light rows each warp relaxes in
// full and whose next_active words it writes.
__global__ void __launch_bounds__(256) k_bf_multi_pull(GraphView g, const int32_t *__restrict__ w_in,
                                                       int32_t *dist, const u64 *__restrict__ active,
                                                       u64 *next_active, int64_t heavy_pieces,
                                                       Counters *cnt) {
  const int lane = lane_id();
  for (;;) {
    long long t = 0;
    if (lane == 0) t = (long long)atomicAdd(&cnt->aux, 1ull);
    t = shfl_idx(t, 0);
    if (t < heavy_pieces) {
      const int c = (int)(t / (kChunkEdges / kBfPiece));
      const int piece = (int)(t % (kChunkEdges / kBfPiece));
      const int r = __ldg(g.in.hrow + c);
      const int64_t row_end = __ldg(g.in.off + r + 1);
      const int64_t e0 = (int64_t)__ldg(g.in.off + r) +
                         (int64_t)(c - __ldg(g.in.hfirst + r)) * kChunkEdges + (int64_t)piece * kBfPiece;
      if (e0 >= row_end) continue;
      const int64_t e1 = min(e0 + kBfPiece, row_end);
      int32_t lo = kDevBFInf, hi = kDevBFInf;
      bf_multi_relax(g.in.idx, w_in, dist, active, e0, e1, lo, hi);
      bool fell_lo = false, fell_hi = false;
      int32_t *p = dist + (int64_t)r * kLanes + lane;
      if (lo < *(volatile int32_t *)p) fell_lo = lo < atomicMin(p, lo);
      if (hi < *(volatile int32_t *)(p + 32)) fell_hi = hi < atomicMin(p + 32, hi);
      const u64 mask = (u64)__ballot_sync(0xffffffffu, fell_lo) | ((u64)__ballot_sync(0xffffffffu, fell_hi) << 32);
      if (lane == 0 && mask) atomicOr(next_active + r, mask);
      continue;
    }
    const long long grp = t - heavy_pieces;
    if (grp >= g.in.ngroups) break;
    const int r0 = __ldg(g.in.gstart + grp), r1 = __ldg(g.in.gstart + grp + 1);
    for (int v = r0; v < r1; ++v) {
      const int e0 = __ldg(g.in.off + v), e1 = __ldg(g.in.off + v + 1);
      if (e1 - e0 > g.heavy_deg) continue;
      const int32_t old_lo = dist[(int64_t)v * kLanes + lane];
      const int32_t old_hi = dist[(int64_t)v * kLanes + 32 + lane];
      int32_t lo = old_lo, hi = old_hi;
      bf_multi_relax(g.in.idx, w_in, dist, active, e0, e1, lo, hi);
      const unsigned ch_lo = __ballot_sync(0xffffffffu, lo < old_lo);
      const unsigned ch_hi = __ballot_sync(0xffffffffu, hi < old_hi);
      if (lo < old_lo) dist[(int64_t)v * kLanes + lane] = lo;
      if (hi < old_hi) dist[(int64_t)v * kLanes + 32 + lane] = hi;
      if (lane == 0) next_active[v] = (u64)ch_lo | ((u64)ch_hi << 32);
    }
  }
}

__global__ void k_bf_multi_init(int32_t *dist, u64 *active, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n * kLanes; i += stride)
    dist[i] = kDevBFInf;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) active[i] = 0ull;
}

__global__ void k_bf_multi_seed(const int32_t *sources, int k, int32_t *dist, u64 *active) {
  const int l = threadIdx.x;
  if (l < k) {
    const int v = sources[l];
    dist[(int64_t)v * kLanes + l] = 0;
    atomicOr(active + v, 1ull << l);
  }
}

// One count per block: the warps' sums meet in shared memory and thread 0
// adds the block's total (blockDim = 32 x 8), so a transpose of millions of
// tiles issues one atomic per block instead of one per warp.
__device__ __forceinline__ void block_count_add(unsigned long long v, unsigned long long *dst) {
  __shared__ unsigned long long s_part[8];
  v = warp_sum(v);
  const int w = threadIdx.y;  // one warp per threadIdx.y (blockDim.x == 32)
  if (threadIdx.x == 0) s_part[w] = v;
  __syncthreads();
  if (threadIdx.x == 0 && w == 0) {
    unsigned long long t = 0;
    for (int i = 0; i < (int)blockDim.y; ++i) t += s_part[i];
    if (t) atomicAdd(dst, t);
  }
}

// dist vertex-major (n x 64) -> out source-major (k x n), through 32x32
// tiles (grid-stride over the vertex tiles); c->size counts the finite
// distances (reached (source, vertex) pairs).
__global__ void __launch_bounds__(256) k_bf_multi_transpose(const int32_t *__restrict__ dist, int64_t n, int k,
                                                            int32_t *__restrict__ out, Counters *c) {
  __shared__ int32_t tile[32][33];
  const int l0 = blockIdx.y * 32;
  unsigned long long reached = 0;
  for (int64_t v0 = (int64_t)blockIdx.x * 32; v0 < n; v0 += (int64_t)gridDim.x * 32) {
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
      const int64_t v = v0 + r;
      tile[r][threadIdx.x] = v < n ? dist[v * kLanes + l0 + threadIdx.x] : kDevBFInf;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
      const int l = l0 + r;
      const int64_t v = v0 + threadIdx.x;
      if (l < k && v < n) {
        const int32_t x = tile[threadIdx.x][r];
        out[(int64_t)l * n + v] = x;
        reached += x < kDevBFInf;
      }
    }
    __syncthreads();
  }
  block_count_add(reached, &c->size);
}

void run_bf_multi(pm_graph *g, const int32_t *d_sources, int k, int32_t *d_dist_out, int64_t threshold,
                  pm_traversal_stats *st) {
  Engine &E = g->E;
  const int64_t n = g->n;
  int32_t *dist = (int32_t *)g->scratch_buf(0, (size_t)n * kLanes * 4);
  u64 *act = (u64 *)g->scratch_buf(1, (size_t)n * 8);
  u64 *nxt = (u64 *)g->scratch_buf(2, (size_t)n * 8);
  int32_t *qdeg = (int32_t *)g->scratch_buf(3, (size_t)n * 4);
  int32_t *qoff = (int32_t *)g->scratch_buf(4, (size_t)n * 4);
  int32_t *queue = g->subset(0).queue;
  size_t tmp_bytes = 0;
  PM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, qdeg, qoff, (int)n, E.stream));
  void *tmp = g->scratch_buf(5, std::max<size_t>(tmp_bytes, 16));
  PM_LAUNCH(k_bf_multi_init, E.grid_for(n * kLanes, 256, 16), 256, 0, E.stream, dist, act, n);
  PM_LAUNCH(k_bf_multi_seed, 1, 64, 0, E.stream, d_sources, k, dist, act);
  static const int pull_per_sm = [] {
    int r = 0;
    PM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, k_bf_multi_pull, 256, 0));
    return std::max(r, 1);
  }();
  static const int push_per_sm = [] {
    int r = 0;
    PM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, k_bf_multi_push, 256, 0));
    return std::max(r, 1);
  }();
  const int64_t heavy_pieces = (int64_t)E.g.in.nchunks * (kChunkEdges / kBfPiece);
  const int pull_grid = E.persistent_grid((heavy_pieces + E.g.in.ngroups + 7) / 8, pull_per_sm);
  const int32_t *w_in = g->w_i32_in.as<int32_t>(), *w_out = g->w_i32_out.as<int32_t>();
  pm_traversal_stats s{};
  E.tag = "bellman_ford_multi";
  for (;;) {
    PM_CUDA(cudaMemsetAsync(E.d_cnt, 0, 3 * sizeof(Counters), E.stream));
    PM_LAUNCH(k_bf_multi_frontier, E.grid_for(n, 256, 8), 256, 0, E.stream, act, E.g.out.off, n, queue, qdeg,
              E.d_cnt + 1);
    const Counters *h = E.read_counters();
    const int64_t size = (int64_t)h[1].size, edges = (int64_t)h[1].edges, q = (int64_t)h[1].aux;
    if (size == 0) break;
    if (s.rounds > n + 1) fail(PM_ERR_INVALID_ARG, "BellmanFord did not converge");
    s.edges_visited += edges;
    const bool dense = size + edges >= threshold;
    E.prof.begin(E.tag, E.stream);
    PM_CUDA(cudaMemsetAsync(nxt, 0, (size_t)n * 8, E.stream));
    if (dense) {
      PM_LAUNCH(k_bf_multi_pull, pull_grid, 256, 0, E.stream, E.g, w_in, dist, act, nxt, heavy_pieces,
                E.d_cnt);
    } else {
      if (q > 0) {
        PM_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, qdeg, qoff, (int)q, E.stream));
        const int64_t chunks = (edges + 31) / 32;
        const int grid = (int)std::max<int64_t>(
            1, std::min<int64_t>((chunks + 7) / 8, (int64_t)E.num_sms * push_per_sm));
        PM_LAUNCH(k_bf_multi_push, grid, 256, 0, E.stream, E.g.out.off, E.g.out.idx, w_out, queue, qoff, (int)q,
                  edges, dist, act, nxt);
      }
    }
    E.prof.end(E.stream);
    s.rounds++;
    s.dense_rounds += dense;
    std::swap(act, nxt);
  }
  PM_CUDA(cudaMemsetAsync(E.d_cnt + 2, 0, sizeof(Counters), E.stream));
  dim3 tb(32, 8), tg((unsigned)std::min<int64_t>((n + 31) / 32, (int64_t)E.num_sms * 16), 2);
  PM_LAUNCH(k_bf_multi_transpose, tg, tb, 0, E.stream, dist, n, k, d_dist_out, E.d_cnt + 2);
  s.reached = (int64_t)E.read_counters()[2].size;
  if (st) *st = s;
}

// ===========================================================================
// Personalised PageRank for up to 32 seeds in one SpMM-shaped pull per
// iteration (PR_F's push p[s]/outdeg(s) and PR_Vertex_F's damping,
// numa-PageRank.C:87-90, 125-137, applied to 32 vectors at once, teleport to
// each vector's seed).  The contribution matrix C (n x 32 floats, row-major,
// C[u][j] = x_j[u] / outdeg(u)) is gathered one 128-byte row per in-edge, a
// full cache line; a warp owns a row and its lanes the 32 columns.  Rows
// with more than g.heavy_deg in-edges are summed by chunk CTAs first.
// ===========================================================================
constexpr int kPprCols = 32;

__device__ __forceinline__ float ppr_row_sum(const int32_t *__restrict__ idx, int64_t e0, int64_t e1,
                                             const float *__restrict__ c, int lane, int stride_slices,
                                             int first_slice) {
  float acc = 0.f;
  for (int64_t base = e0 + (int64_t)first_slice * 32; base < e1; base += (int64_t)stride_slices * 32) {
    const int cnt = (int)min((int64_t)32, e1 - base);
    const int my_s = lane < cnt ? __ldg(idx + base + lane) : 0;
    for (int j0 = 0; j0 < cnt; j0 += 8) {
      float v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int s = __shfl_sync(0xffffffffu, my_s, (j0 + u) & 31);
        v[u] = (j0 + u < cnt) ? __ldg(c + (int64_t)s * kPprCols + lane) : 0.f;
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) acc += v[u];
    }
  }
  return acc;
}

__global__ void __launch_bounds__(256) k_ppr_heavy(GraphView g, const float *__restrict__ c,
                                                   float *__restrict__ partials) {
  __shared__ float s_part[8][kPprCols];
  const int ch = blockIdx.x;
  if (ch >= g.in.nchunks) return;
  const int lane = lane_id(), wid = threadIdx.x >> 5;
  const int r = __ldg(g.in.hrow + ch);
  const int k = ch - __ldg(g.in.hfirst + r);
  const int64_t e0 = (int64_t)__ldg(g.in.off + r) + (int64_t)k * kChunkEdges;
  const int64_t e1 = min(e0 + kChunkEdges, (int64_t)__ldg(g.in.off + r + 1));
  s_part[wid][lane] = ppr_row_sum(g.in.idx, e0, e1, c, lane, 8, wid);
  __syncthreads();
  if (wid == 0) {
    float t = 0.f;
    for (int w = 0; w < 8; ++w) t += s_part[w][lane];
    partials[(int64_t)ch * kPprCols + lane] = t;
  }
}

__global__ void __launch_bounds__(256) k_ppr_pull(GraphView g, const float *__restrict__ c_cur,
                                                  float *__restrict__ c_next, float *__restrict__ y_out,
                                                  int k_out, const float *__restrict__ partials,
                                                  const int32_t *__restrict__ seeds, float damping,
                                                  Counters *ticket) {
  const int lane = lane_id();
  const int my_seed = lane < k_out ? __ldg(seeds + lane) : -1;
  for (;;) {
    int grp = 0;
    if (lane == 0) grp = (int)atomicAdd(&ticket->aux, 1ull);
    grp = __shfl_sync(0xffffffffu, grp, 0);
    if (grp >= g.in.ngroups) break;
    const int r0 = __ldg(g.in.gstart + grp), r1 = __ldg(g.in.gstart + grp + 1);
    for (int r = r0; r < r1; ++r) {
      const int64_t o0 = __ldg(g.in.off + r), o1 = __ldg(g.in.off + r + 1);
      float acc;
      if (o1 - o0 > g.heavy_deg) {
        const int first = __ldg(g.in.hfirst + r);
        const int nch = (int)((o1 - o0 + kChunkEdges - 1) / kChunkEdges);
        acc = 0.f;
        for (int q = 0; q < nch; ++q) acc += partials[(int64_t)(first + q) * kPprCols + lane];
      } else {
        acc = ppr_row_sum(g.in.idx, o0, o1, c_cur, lane, 1, 0);
      }
      const float y = damping * acc + (r == my_seed ? 1.0f - damping : 0.0f);
      if (y_out && lane < k_out) y_out[(int64_t)r * k_out + lane] = y;
      const int od = __ldg(g.out.off + r + 1) - __ldg(g.out.off + r);
      c_next[(int64_t)r * kPprCols + lane] = od > 0 ? y / (float)od : 0.f;
    }
  }
}

__global__ void k_ppr_seed(const int32_t *seeds, int k, const int32_t *out_off, float *c, float *y0,
                           int k_out) {
  const int j = threadIdx.x;
  if (j < k) {
    const int v = seeds[j];
    const int od = out_off[v + 1] - out_off[v];
    c[(int64_t)v * kPprCols + j] = od > 0 ? 1.0f / (float)od : 0.f;
    if (y0) y0[(int64_t)v * k_out + j] = 1.0f;
  }
}

void run_ppr(pm_graph *g, const int32_t *d_seeds, int k, int iters, double damping, float *d_out) {
  Engine &E = g->E;
  const int64_t n = g->n;
  float *c0 = (float *)g->scratch_buf(0, (size_t)n * kPprCols * 4);
  float *c1 = (float *)g->scratch_buf(1, (size_t)n * kPprCols * 4);
  float *part = (float *)g->scratch_buf(2, (size_t)std::max(E.g.in.nchunks, 1) * kPprCols * 4);
  PM_CUDA(cudaMemsetAsync(c0, 0, (size_t)n * kPprCols * 4, E.stream));
  if (iters == 0) PM_CUDA(cudaMemsetAsync(d_out, 0, (size_t)n * k * 4, E.stream));
  PM_LAUNCH(k_ppr_seed, 1, 32, 0, E.stream, d_seeds, k, E.g.out.off, c0, iters == 0 ? d_out : nullptr, k);
  static const int per_sm = [] {
    int r = 0;
    PM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, k_ppr_pull, 256, 0));
    return std::max(r, 1);
  }();
  const int grid = E.persistent_grid(((int64_t)E.g.in.ngroups + 7) / 8, per_sm);
  E.run_loop(loop_key("ppr", iters, k, damping, c0, c1, part, d_seeds, d_out), [&] {
    float *a = c0, *b = c1;
    for (int it = 0; it < iters; ++it) {
      PM_CUDA(cudaMemsetAsync(E.d_cnt, 0, sizeof(Counters), E.stream));
      E.prof.begin("ppr", E.stream);
      if (E.g.in.nchunks > 0)
        PM_LAUNCH(k_ppr_heavy, E.g.in.nchunks, 256, 0, E.stream, E.g, a, part);
      PM_LAUNCH(k_ppr_pull, grid, 256, 0, E.stream, E.g, a, b, it == iters - 1 ? d_out : nullptr, k, part,
                d_seeds, (float)damping, E.d_cnt);
      E.prof.end(E.stream);
      std::swap(a, b);
    }
  });
}

// ===========================================================================
// Many independent graphs (the parts of a disjoint union) each running
// PageRank with Polymer's semantics (PR_F / PR_Vertex_F / PR_Vertex_Reset,
// numa-PageRank.C:64-148, n = the part's own vertex count), all in ONE
// persistent launch.  Thread-block clusters of kPartCluster CTAs take parts
// from a work queue, largest first; the CTAs of a cluster split the part's
// vertices and separate the phases of an iteration with the cluster barrier
// (barrier.cluster, a hardware barrier: no flag is polled).  One thread per
// vertex sums its in-edges; the frontier rides in the contribution sign as in
// run_pagerank.
// ===========================================================================
constexpr int kPartCluster = 8;
constexpr int kPartThreads = 512;

__global__ void __cluster_dims__(kPartCluster, 1, 1) __launch_bounds__(kPartThreads)
    k_pagerank_parts(GraphView g, const int64_t *__restrict__ vbase, const int32_t *__restrict__ order,
                     int count, int iters, float damping, float *pc, float *pn, float *c0, float *c1,
                     float *out, Counters *queue) {
  cg::cluster_group cluster = cg::this_cluster();
  __shared__ int s_part;
  const int rank = (int)cluster.block_rank();
  const int64_t stride = (int64_t)kPartCluster * kPartThreads;
  for (;;) {
    if (rank == 0 && threadIdx.x == 0) s_part = (int)atomicAdd(&queue->aux, 1ull);
    cluster.sync();
    const int part = *cluster.map_shared_rank(&s_part, 0);
    cluster.sync();  // every CTA has read the ticket before the next one is drawn
    if (part >= count) break;
    const int p = __ldg(order + part);
    const int64_t v0 = __ldg(vbase + p), v1 = __ldg(vbase + p + 1);
    const float p0 = 1.0f / (float)(v1 - v0);
    const float added = (1.0f - damping) * p0;
    const int64_t first = v0 + (int64_t)rank * kPartThreads + threadIdx.x;
    for (int64_t v = first; v < v1; v += stride) {
      const int deg = __ldg(g.out.off + v + 1) - __ldg(g.out.off + v);
      pc[v] = p0;
      pn[v] = 0.0f;
      c0[v] = deg > 0 ? p0 / (float)deg : 0.0f;
    }
    cluster.sync();
    float *A = pc, *B = pn, *cc = c0, *cn = c1;
    for (int it = 0; it < iters; ++it) {
      for (int64_t v = first; v < v1; v += stride) {
        const int e0 = __ldg(g.in.off + v), e1 = __ldg(g.in.off + v + 1);
        float acc = -0.0f;
        int e = e0;
        for (; e + 3 < e1; e += 4) {
          const int s0 = __ldg(g.in.idx + e), s1 = __ldg(g.in.idx + e + 1);
          const int s2 = __ldg(g.in.idx + e + 2), s3 = __ldg(g.in.idx + e + 3);
          acc += (cc[s0] + cc[s1]) + (cc[s2] + cc[s3]);
        }
        for (; e < e1; ++e) acc += cc[__ldg(g.in.idx + e)];
        const bool in_f = !signbit(cc[v]);
        const bool hit = !signbit(acc);
        float nb = B[v] + acc;
        if (in_f) {
          nb = damping * nb + added;
          A[v] = 0.0f;
        }
        B[v] = nb;
        const int deg = __ldg(g.out.off + v + 1) - __ldg(g.out.off + v);
        cn[v] = hit ? (deg > 0 ? nb / (float)deg : 0.0f) : -0.0f;
      }
      cluster.sync();
      float *t = A; A = B; B = t;
      t = cc; cc = cn; cn = t;
    }
    for (int64_t v = first; v < v1; v += stride) out[v] = A[v];
    cluster.sync();
  }
}

void run_pagerank_parts(pm_graph *g, int iters, double damping, float *d_out) {
  Engine &E = g->E;
  const int64_t n = g->n;
  const int count = (int)g->parts.size() - 1;
  float *pc = (float *)g->scratch_buf(0, (size_t)n * 4);
  float *pn = (float *)g->scratch_buf(1, (size_t)n * 4);
  float *c0 = (float *)g->scratch_buf(2, (size_t)n * 4);
  float *c1 = (float *)g->scratch_buf(3, (size_t)n * 4);
  static const int clusters = [] {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kPartCluster * 64);
    cfg.blockDim = dim3(kPartThreads);
    int r = 0;
    PM_CUDA(cudaOccupancyMaxActiveClusters(&r, (void *)k_pagerank_parts, &cfg));
    return std::max(r, 1);
  }();
  const int grid = kPartCluster * std::max(1, std::min(clusters, count));
  PM_CUDA(cudaMemsetAsync(E.d_cnt, 0, sizeof(Counters), E.stream));
  E.prof.begin("pagerank_parts", E.stream);
  PM_LAUNCH(k_pagerank_parts, grid, kPartThreads, 0, E.stream, E.g, g->parts_vbase.as<int64_t>(),
            g->parts_order.as<int32_t>(), count, iters, (float)damping, pc, pn, c0, c1, d_out, E.d_cnt);
  E.prof.end(E.stream);
}

}  // namespace pm
