// pm_apps.cu -- the six Polymer applications as host loops over the engine.
//
// Each app keeps the reference's functor (cond / updateAtomic for pushes,
// identity / edge / combine / commit for the reducing pull, with the
// application's vertexMap fused into commit) and its iteration loop, with
// the NUMA worker/sub-worker scaffolding replaced by kernel launches on the
// graph's stream.
#include <cmath>
#include <cstring>

#include "pm_graph.cuh"

namespace pm {

// ===========================================================================
// BFS  (numa-BFS.C:59-79 BFS_F, loop 258-296)
// ===========================================================================
struct BFS_F {
  int32_t *parents;
  int32_t *depth;
  int32_t level;
  // cond: not visited yet
  __device__ __forceinline__ bool cond(int d) const {
    return *((volatile int32_t *)parents + d) == -1;
  }
  // updateAtomic: CAS(Parents[d], -1, s)
  __device__ __forceinline__ bool updateAtomic(int s, int d, int) const {
    if (atomicCAS(parents + d, -1, s) == -1) {
      depth[d] = level;
      return true;
    }
    return false;
  }
};

__global__ void k_bfs_init(int32_t *parents, int32_t *depth, int64_t n, int32_t src) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
    parents[v] = v == src ? src : -1;
    depth[v] = v == src ? 0 : -1;
  }
}

// ---------------------------------------------------------------------------
// BFS with its rounds driven on the GPU.  The host loop above reads the
// frontier's size and out-degree sum back after every round to pick the next
// round's direction (about 20 us of idle GPU per level).  Here one CUDA graph
// holds a WHILE node whose body runs two rounds (frontier A -> B, B -> A): a
// one-thread kernel decides each round's direction from the counters on the
// device (the same rule, |F| + outdeg(F) >= threshold), the sparse and dense
// kernels return at once when it is not their round, and the round's last
// kernel updates the frontier state and ends the loop when the frontier is
// empty.  The host synchronises once per BFS.
struct BFS_GF {  // BFS_F with the level read from the round state
  int32_t *parents;
  int32_t *depth;
  const RoundGate *gate;
  __device__ __forceinline__ bool cond(int d) const {
    return *((volatile int32_t *)parents + d) == -1;
  }
  __device__ __forceinline__ bool updateAtomic(int s, int d, int) const {
    if (atomicCAS(parents + d, -1, s) == -1) {
      depth[d] = gate->level;
      return true;
    }
    return false;
  }
};

struct DevRound {
  RoundGate gate;
  unsigned long long rounds, dense_rounds, reached, edges_visited, slots;
  unsigned int err, pad;
};

static_assert(sizeof(DevRound) <= 3 * sizeof(Counters), "DevRound is read back through the pinned counter words");

// The frontier {src} (its bitmap word; the bitmap was cleared) and the round
// state of a BFS from src.
__global__ void k_round_init(DevRound *dr, uint32_t *bits, const int32_t *out_off, int32_t src) {
  bits[src >> 5] = 1u << (src & 31);
  dr->gate.size = 1;
  dr->gate.edges = (unsigned long long)(out_off[src + 1] - out_off[src]);
  dr->gate.active = 1;
  dr->gate.dense = 0;
  dr->gate.qsize = 1;
  dr->gate.level = 0;
  dr->rounds = dr->dense_rounds = dr->edges_visited = dr->slots = 0;
  dr->reached = 1;
  dr->err = 0;
}

// The round's direction and fresh counters (their error words are kept).
__global__ void k_round_begin(DevRound *dr, Counters *cnt, int64_t threshold) {
  RoundGate &g = dr->gate;
  g.active = g.size > 0;
  g.dense = (long long)(g.size + g.edges) >= threshold;
  g.qsize = (int32_t)g.size;
  if (g.active) g.level += 1;
  for (int i = 0; i < 3; ++i) {
    cnt[i].size = cnt[i].edges = cnt[i].aux = 0;
    cnt[i].daux = cnt[i].daux2 = 0.0;
  }
}

__global__ void k_round_end(DevRound *dr, const Counters *cnt, cudaGraphConditionalHandle loop,
                            int32_t max_level) {
  RoundGate &g = dr->gate;
  dr->slots += 1;
  if (g.active) {
    dr->rounds += 1;
    dr->dense_rounds += g.dense;
    dr->edges_visited += g.edges;
    dr->reached += cnt[0].size;
    g.size = cnt[0].size;
    g.edges = cnt[0].edges;
  }
  dr->err |= cnt[0].err | cnt[1].err | cnt[2].err;
  const bool more = g.size > 0 && g.level < max_level && dr->err == 0;
  cudaGraphSetConditional(loop, more ? 1u : 0u);
}

// Runs a traversal's rounds inside one CUDA graph (built once per key): a
// WHILE node whose body is round(A, B) then round(B, A), each between
// k_round_begin and k_round_end.  The round state in dr is set up on the
// stream before the call; on return it is read back into h.
template <class Round>
static void run_rounds(pm_graph *g, DevRound *dr, const std::string &key, int64_t threshold, const char *tag,
                       Round &&round, DevRound &h) {
  Engine &E = g->E;
  VertexSubset A = g->subset(0), B = g->subset(1);
  LoopGraph *lg = nullptr;
  for (auto &x : E.graphs)
    if (x.key == key) lg = &x;
  if (!lg) {
    if (E.graphs.size() >= 16) {
      E.drop_graph(E.graphs.front());
      E.graphs.erase(E.graphs.begin());
    }
    LoopGraph fresh;
    fresh.key = key;
    cudaGraph_t graph = nullptr;
    PM_CUDA(cudaGraphCreate(&graph, 0));
    bool capturing = false;
    const long long before = launches(false);
    try {
      cudaGraphConditionalHandle loop;
      PM_CUDA(cudaGraphConditionalHandleCreate(&loop, graph, 1, cudaGraphCondAssignDefault));
      cudaGraphNodeParams cp = {};
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = loop;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      cudaGraphNode_t node;
      PM_CUDA(cudaGraphAddNode(&node, graph, nullptr, 0, &cp));
      cudaGraph_t body = cp.conditional.phGraph_out[0];
      PM_CUDA(cudaStreamBeginCaptureToGraph(E.stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
      capturing = true;
      const int32_t max_level = (int32_t)std::min<int64_t>(g->n + 1, 0x7ffffff0);
      auto one = [&](VertexSubset &cur, VertexSubset &next) {
        PM_LAUNCH(k_round_begin, 1, 1, 0, E.stream, dr, E.d_cnt, threshold);
        round(cur, next, (const RoundGate *)&dr->gate);
        PM_LAUNCH(k_round_end, 1, 1, 0, E.stream, dr, E.d_cnt, loop, max_level);
      };
      one(A, B);
      one(B, A);
      cudaGraph_t captured = nullptr;
      capturing = false;
      PM_CUDA(cudaStreamEndCapture(E.stream, &captured));
      const long long captured_launches = launches(false) - before;
      fresh.launches = captured_launches / 2;  // kernels of one round
      count_launch((int)-captured_launches);   // captured, not run
      PM_CUDA(cudaGraphInstantiate(&fresh.exec, graph, 0));
    } catch (...) {
      if (capturing) {  // leave the stream usable; the body graph belongs to `graph`
        cudaGraph_t captured = nullptr;
        cudaStreamEndCapture(E.stream, &captured);
        (void)cudaGetLastError();
        count_launch((int)-(launches(false) - before));
      }
      cudaGraphDestroy(graph);
      throw;
    }
    cudaGraphDestroy(graph);
    E.graphs.push_back(std::move(fresh));
    lg = &E.graphs.back();
  }
  E.prof.begin(tag, E.stream);
  PM_CUDA(cudaGraphLaunch(lg->exec, E.stream));
  E.prof.end(E.stream);
  PM_CUDA(cudaMemcpyAsync(E.h_cnt, dr, sizeof(DevRound), cudaMemcpyDeviceToHost, E.stream));
  PM_CUDA(cudaStreamSynchronize(E.stream));
  std::memcpy(&h, E.h_cnt, sizeof h);
  count_launch((int)(lg->launches * (long long)h.slots));
  if (h.err)
    fail(h.err & kErrTimeout ? PM_ERR_TIMEOUT : PM_ERR_CUDA,
         std::string("device error word ") + std::to_string(h.err) +
             (h.err & kErrQueueOverflow ? " (queue overflow)" : "") + (h.err & kErrRange ? " (id out of range)" : ""));
}

// The sparse half of a round driven on the GPU (returns at once in dense
// rounds): the frontier bitmap to a queue, then the push.
template <class F, class W>
static void gated_sparse(Engine &E, VertexSubset &cur, VertexSubset &next, F f, const W *w_out,
                         const RoundGate *gate) {
  PM_CUDA(cudaMemsetAsync(next.bits, 0, next.words() * 4, E.stream));
  PM_LAUNCH(k_bits_to_queue, E.grid_for(((cur.words() + 31) / 32) * 32, 256, 8), 256, 0, E.stream, cur.n,
            E.g.out.off, cur.bits, cur.queue, E.d_cnt + 2, gate);
  PM_LAUNCH((k_sparse_push<F, W>), E.num_sms * 8, 256, 0, E.stream, E.g, cur.queue, 0, f, w_out, next.queue,
            next.bits, next.n, E.d_cnt, E.hubs, E.d_cnt + 1, gate);
  PM_LAUNCH((k_sparse_push_hubs<F, W>), E.num_sms * 4, 256, 0, E.stream, E.g, f, w_out, E.hubs, E.d_cnt + 1,
            next.queue, next.bits, next.n, E.d_cnt, gate);
}

static void fill_stats(const DevRound &h, pm_traversal_stats *st) {
  if (!st) return;
  *st = pm_traversal_stats{};
  st->rounds = (int64_t)h.rounds;
  st->dense_rounds = (int64_t)h.dense_rounds;
  st->reached = (int64_t)h.reached;
  st->edges_visited = (int64_t)h.edges_visited;
}

static void run_bfs_graph(pm_graph *g, int32_t src, int32_t *d_parents, int32_t *d_depth, int64_t threshold,
                          pm_traversal_stats *st) {
  Engine &E = g->E;
  VertexSubset A = g->subset(0);
  auto *dr = (DevRound *)g->scratch_buf(30, sizeof(DevRound));
  PM_LAUNCH(k_bfs_init, E.grid_for(g->n, 256, 16), 256, 0, E.stream, d_parents, d_depth, g->n, src);
  PM_CUDA(cudaMemsetAsync(A.bits, 0, A.words() * 4, E.stream));
  PM_LAUNCH(k_round_init, 1, 1, 0, E.stream, dr, A.bits, E.g.out.off, src);
  char key[160];
  std::snprintf(key, sizeof key, "bfs_rounds|%lld|%p|%p|%p", (long long)threshold, (void *)d_parents,
                (void *)d_depth, (void *)dr);
  const int64_t nthreads = ((int64_t)E.g.n + 31) & ~31ll;
  DevRound h{};
  run_rounds(g, dr, key, threshold, "bfs", [&](VertexSubset &cur, VertexSubset &next, const RoundGate *gate) {
    const BFS_GF f{d_parents, d_depth, gate};
    gated_sparse<BFS_GF, int>(E, cur, next, f, (const int *)nullptr, gate);
    PM_LAUNCH((k_dense_pull<BFS_GF, int>), E.grid_for(nthreads, 256, 16), 256, 0, E.stream, E.g, cur.bits, f,
              (const int *)nullptr, next.bits, E.defer, E.d_cnt, E.d_cnt + 1, gate);
    PM_LAUNCH((k_dense_pull_defer<BFS_GF, int>), E.num_sms * 8, 256, 0, E.stream, E.g, cur.bits, f,
              (const int *)nullptr, next.bits, E.defer, E.d_cnt, E.d_cnt + 1, gate);
  }, h);
  fill_stats(h, st);
}

void run_bfs(pm_graph *g, int32_t src, int32_t *d_parents, int32_t *d_depth, int64_t threshold,
             pm_traversal_stats *st) {
  if (g->E.tune.cuda_graphs && !g->is_part) {
    run_bfs_graph(g, src, d_parents, d_depth, threshold, st);
    return;
  }
  Engine &E = g->E;
  VertexSubset cur = g->subset(0), next = g->subset(1);
  PM_LAUNCH(k_bfs_init, E.grid_for(g->n, 256, 16), 256, 0, E.stream, d_parents, d_depth, g->n, src);
  subset_single(E, cur, src);
  pm_traversal_stats s{};
  s.reached = 1;
  E.tag = "bfs";
  for (int32_t level = 1; cur.size > 0; ++level) {
    bool dense = false;
    s.edges_visited += cur.edges;
    edgeMap<int>(E, cur, BFS_F{d_parents, d_depth, level}, next, threshold, DENSE_PARALLEL, nullptr,
                 nullptr, &dense);
    part_round(g, next);  // a partition: the next frontier of every rank
    s.rounds++;
    s.dense_rounds += dense;
    s.reached += next.size;
    std::swap(cur, next);
  }
  part_exchange(g, d_parents, 4);  // a partition: every rank's parents and depths
  part_exchange(g, d_depth, 4);
  if (st) *st = s;
}

// ===========================================================================
// Connected components  (numa-Components.C:55-119 CC_F / CC_Vertex_F,
// loop 233-281, edgeMapCustom 121-175)
// The reference activates d when writeMin(IDs[d], IDs[s]) succeeds while
// IDs[d] still equals prevIDs[d]; prevIDs equals IDs for every vertex at the
// start of a round, so that is "the first lowering of d in this round" --
// here the dedup bit of the next frontier.  The result is the same.
// ===========================================================================
struct CC_F {
  int32_t *ids;
  const uint32_t *cur;
  using Acc = int32_t;
  __device__ __forceinline__ bool cond(int) const { return true; }
  // writeMin (utils.h): nothing to do when the label is already no larger
  __device__ __forceinline__ bool updateAtomic(int s, int d, int) const {
    int32_t v = *((volatile int32_t *)ids + s);
    return v < *((volatile int32_t *)ids + d) && v < atomicMin(ids + d, v);
  }
  // updateAtomic as an atomicMin of push_value (warp-aggregated pushes)
  __device__ __forceinline__ int32_t *min_target() const { return ids; }
  __device__ __forceinline__ int32_t push_value(int s, int) const { return *((volatile int32_t *)ids + s); }
  __device__ __forceinline__ Acc identity() const { return 0x7fffffff; }
  __device__ __forceinline__ Acc edge(int s, int, int) const {
    return test_bit(cur, s) ? *((volatile int32_t *)ids + s) : 0x7fffffff;
  }
  __device__ __forceinline__ Acc combine(Acc a, Acc b) const { return min(a, b); }
  __device__ __forceinline__ bool commit(int d, Acc acc, double2 &) const {
    if (acc < ids[d]) {
      ids[d] = acc;
      return true;
    }
    return false;
  }
};

__global__ void k_iota32(int32_t *a, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) a[v] = (int32_t)v;
}

void run_cc_union_find(pm_graph *g, int32_t *d_labels, pm_traversal_stats *st);

// Symmetric whole-graph handles take the union-find of pm_cc.cu (the same
// labels, PM_TUNE_CC_MODE 0, the default); directed graphs, partitions and
// mode 1 run the reference's label propagation below.
void run_cc(pm_graph *g, int32_t *d_labels, int64_t threshold, pm_traversal_stats *st) {
  if (g->symmetric && !g->is_part && g->E.tune.cc_mode == 0) {
    run_cc_union_find(g, d_labels, st);
    return;
  }
  Engine &E = g->E;
  VertexSubset cur = g->subset(0), next = g->subset(1);
  PM_LAUNCH(k_iota32, E.grid_for(g->n, 256, 16), 256, 0, E.stream, d_labels, g->n);
  subset_all(E, cur);
  pm_traversal_stats s{};
  E.tag = "cc";
  while (cur.size > 0) {
    bool dense = false;
    s.edges_visited += cur.edges;
    edgeMapReduce<int>(E, cur, CC_F{d_labels, cur.bits}, next, threshold, nullptr, nullptr, &dense);
    part_exchange(g, d_labels, 4);  // a partition: labels and frontier of every rank
    part_round(g, next);
    s.rounds++;
    s.dense_rounds += dense;
    std::swap(cur, next);
  }
  s.reached = g->n;
  if (st) *st = s;
}

// ===========================================================================
// BellmanFord  (numa-BellmanFord.C:61-95 BF_F / BF_Vertex_F, loop 166-211)
// Next frontier = vertices whose distance fell this round (Ligra's reset of
// Visited on the output; the reference resets on the current frontier,
// which can lose re-improved vertices).  Dense rounds pull min(dist[s] + w)
// over the CSC instead of pushing writeMin over the CSR; both compute the
// same round result.
// ===========================================================================
struct BF_F {
  int32_t *dist;
  const uint32_t *cur;
  using Acc = int32_t;
  __device__ __forceinline__ bool cond(int) const { return true; }
  // writeMin (utils.h): nothing to do when the distance is already no larger
  __device__ __forceinline__ bool updateAtomic(int s, int d, int32_t w) const {
    int32_t nd = *((volatile int32_t *)dist + s) + w;
    return nd < *((volatile int32_t *)dist + d) && nd < atomicMin(dist + d, nd);
  }
  // updateAtomic as an atomicMin of push_value (warp-aggregated pushes)
  __device__ __forceinline__ int32_t *min_target() const { return dist; }
  __device__ __forceinline__ int32_t push_value(int s, int32_t w) const {
    return *((volatile int32_t *)dist + s) + w;
  }
  __device__ __forceinline__ Acc identity() const { return 0x7fffffff; }
  __device__ __forceinline__ Acc edge(int s, int, int32_t w) const {
    return test_bit(cur, s) ? *((volatile int32_t *)dist + s) + w : 0x7fffffff;
  }
  __device__ __forceinline__ Acc combine(Acc a, Acc b) const { return min(a, b); }
  __device__ __forceinline__ bool commit(int d, Acc acc, double2 &) const {
    if (acc < dist[d]) {
      dist[d] = acc;
      return true;
    }
    return false;
  }
};

// Dense pulls read a snapshot taken at the start of the round: fd[s] =
// dist[s] for frontier sources, INT_MAX for the others, so that an edge costs
// one gather (BF_F's bit test and then the distance are two dependent loads;
// the pull was latency-bound on them).  Relaxing from the round's snapshot
// is the synchronous form of the same rounds and reaches the same fixpoint.
struct BF_FD {
  int32_t *dist;
  const int32_t *fd;
  using Acc = int32_t;
  __device__ __forceinline__ bool cond(int) const { return true; }
  // writeMin (utils.h): nothing to do when the distance is already no larger
  __device__ __forceinline__ bool updateAtomic(int s, int d, int32_t w) const {
    int32_t nd = *((volatile int32_t *)dist + s) + w;
    return nd < *((volatile int32_t *)dist + d) && nd < atomicMin(dist + d, nd);
  }
  // updateAtomic as an atomicMin of push_value (warp-aggregated pushes)
  __device__ __forceinline__ int32_t *min_target() const { return dist; }
  __device__ __forceinline__ int32_t push_value(int s, int32_t w) const {
    return *((volatile int32_t *)dist + s) + w;
  }
  __device__ __forceinline__ Acc identity() const { return 0x7fffffff; }
  __device__ __forceinline__ Acc edge(int s, int, int32_t w) const {
    const int32_t v = __ldg(fd + s);
    return v == 0x7fffffff ? v : v + w;
  }
  __device__ __forceinline__ Acc combine(Acc a, Acc b) const { return min(a, b); }
  __device__ __forceinline__ bool commit(int d, Acc acc, double2 &) const {
    if (acc < dist[d]) {
      dist[d] = acc;
      return true;
    }
    return false;
  }
};

__global__ void k_bf_snapshot(int32_t n, const uint32_t *__restrict__ bits, const int32_t *__restrict__ dist,
                              int32_t *__restrict__ fd) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
    fd[v] = test_bit(bits, (int)v) ? dist[v] : 0x7fffffff;
}

// Dense BellmanFord round as a push whose atomics return nothing
// (PM_TUNE_BF_DENSE 2).  The frontier's rows (light ones here, heavy ones by
// 4096-edge chunks below) relax their out-edges with atomicMin whose result
// is unused, so the warp never waits for an atomic; each lane takes
// kBfRedEdges consecutive edges of a window and issues their id and weight
// loads before their atomics, and skips the atomic when the target's
// distance, as this SM last saw it, is already no larger (distances only
// fall, so a value seen earlier is never below the current one; the hub
// targets would otherwise take an atomic from most of their in-edges every
// round, one after another at one L2 slice).  A source's distance is read once, at its
// batch's start: a source lowered later in the round is in the next frontier
// and pushes again, so the rounds end at the same distances.  The next
// frontier is what fell during the round: k_bf_fell compares the distances
// with a copy taken before it.
constexpr int kBfRedEdges = 4;

__global__ void __launch_bounds__(256) k_bf_push_red(GraphView g, const uint32_t *__restrict__ cur,
                                                     const int32_t *__restrict__ w, int32_t *dist) {
  __shared__ int s_pos[8][33];
  __shared__ int s_off[8][32];
  __shared__ int32_t s_ds[8][32];
  const int lane = lane_id(), wid = threadIdx.x >> 5;
  const int grp = blockIdx.x * 8 + wid;
  if (grp >= g.out.ngroups) return;
  int *pos_s = s_pos[wid], *off_s = s_off[wid];
  int32_t *ds_s = s_ds[wid];
  const int r_begin = __ldg(g.out.gstart + grp), r_end = __ldg(g.out.gstart + grp + 1);
  for (int rb = r_begin; rb < r_end; rb += 32) {  // group starts are multiples of 32
    const uint32_t word = __ldg(cur + (rb >> 5));
    if (word == 0) continue;
    const int r = rb + lane;
    int o0 = 0, deg = 0;
    int32_t ds = 0;
    if (r < r_end && ((word >> lane) & 1u)) {
      o0 = __ldg(g.out.off + r);
      deg = __ldg(g.out.off + r + 1) - o0;
      ds = *((volatile const int32_t *)dist + r);
      if (deg > g.heavy_deg || ds >= kDevBFInf) deg = 0;
    }
    int total;
    const int pos = warp_excl_scan(deg, &total);
    __syncwarp();  // the previous batch's windows are done with the arrays
    pos_s[lane] = pos;
    if (lane == 31) pos_s[32] = total;
    off_s[lane] = o0;
    ds_s[lane] = ds;
    __syncwarp();
    for (int c = 0; c < total; c += 32 * kBfRedEdges) {
      const int q0 = c + lane * kBfRedEdges;
      if (q0 >= total) continue;
      int j = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1)
        if (pos_s[j + step] <= q0) j += step;
      int nxt = pos_s[j + 1];
      int32_t dst[kBfRedEdges], nd[kBfRedEdges];
#pragma unroll
      for (int k = 0; k < kBfRedEdges; ++k) {
        const int q = q0 + k;
        dst[k] = -1;
        if (q < total) {
          while (q >= nxt) nxt = pos_s[++j + 1];
          const int64_t e = (int64_t)off_s[j] + (q - pos_s[j]);
          dst[k] = checked_id(g, __ldg(g.out.idx + e));
          nd[k] = ds_s[j] + __ldg(w + e);
        }
      }
      int32_t seen[kBfRedEdges];
#pragma unroll
      for (int k = 0; k < kBfRedEdges; ++k) seen[k] = dst[k] >= 0 ? __ldca(dist + dst[k]) : 0;
#pragma unroll
      for (int k = 0; k < kBfRedEdges; ++k)
        if (dst[k] >= 0 && nd[k] < seen[k]) atomicMin(dist + dst[k], nd[k]);
    }
  }
}

__global__ void __launch_bounds__(kChunkThreads) k_bf_heavy_red(GraphView g, const uint32_t *__restrict__ cur,
                                                                const int32_t *__restrict__ w, int32_t *dist) {
  const int c = blockIdx.x;
  if (c >= g.out.nchunks) return;
  const int r = __ldg(g.out.hrow + c);
  if (!test_bit(cur, r)) return;
  const int32_t ds = *((volatile const int32_t *)dist + r);
  if (ds >= kDevBFInf) return;
  const int k = c - __ldg(g.out.hfirst + r);
  const int64_t e0 = (int64_t)__ldg(g.out.off + r) + (int64_t)k * kChunkEdges;
  const int64_t e1 = min(e0 + kChunkEdges, (int64_t)__ldg(g.out.off + r + 1));
  for (int64_t e = e0 + threadIdx.x; e < e1; e += kChunkThreads) {
    const int d = checked_id(g, __ldg(g.out.idx + e));
    const int32_t nd = ds + __ldg(w + e);
    if (nd < __ldca(dist + d)) atomicMin(dist + d, nd);
  }
}

// next = {v : dist[v] < before[v]}, with its size and out-degree sum.
__global__ void k_bf_fell(int32_t n, const int32_t *__restrict__ out_off, const int32_t *__restrict__ dist,
                          const int32_t *__restrict__ before, uint32_t *__restrict__ next, Counters *c) {
  const int64_t ntot = ((int64_t)n + 31) & ~31ll;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  unsigned long long s = 0, e = 0;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntot; t += stride) {
    const int v = (int)t;
    const bool fell = v < n && __ldcs(dist + v) < __ldcs(before + v);
    const unsigned word = __ballot_sync(0xffffffffu, fell);
    if (lane_id() == 0) next[v >> 5] = word;
    if (fell) {
      s++;
      e += __ldg(out_off + v + 1) - __ldg(out_off + v);
    }
  }
  s = warp_sum(s);
  e = warp_sum(e);
  if (lane_id() == 0 && s) {
    atomicAdd(&c->size, s);
    atomicAdd(&c->edges, e);
  }
}

static void bf_round_red(pm_graph *g, VertexSubset &from, VertexSubset &next, int32_t *d_dist,
                         const int32_t *w_out) {
  Engine &E = g->E;
  const int64_t n = g->n;
  int32_t *before = (int32_t *)g->scratch_buf(37, (size_t)n * 4);
  Counters *dc = (Counters *)g->scratch_buf(32, 2 * sizeof(Counters));
  PM_CUDA(cudaMemcpyAsync(before, d_dist, (size_t)n * 4, cudaMemcpyDeviceToDevice, E.stream));
  if (E.g.out.nchunks > 0)
    PM_LAUNCH(k_bf_heavy_red, E.g.out.nchunks, kChunkThreads, 0, E.stream, E.g, from.bits, w_out, d_dist);
  PM_LAUNCH(k_bf_push_red, (E.g.out.ngroups + 7) / 8, 256, 0, E.stream, E.g, from.bits, w_out, d_dist);
  PM_CUDA(cudaMemsetAsync(dc, 0, sizeof(Counters), E.stream));
  PM_LAUNCH(k_bf_fell, E.grid_for(n, 256, 16), 256, 0, E.stream, (int32_t)n, E.g.out.off, d_dist, before,
            next.bits, dc);
  Counters hc;
  PM_CUDA(cudaMemcpyAsync(&hc, dc, sizeof(Counters), cudaMemcpyDeviceToHost, E.stream));
  PM_CUDA(cudaStreamSynchronize(E.stream));
  next.size = (int64_t)hc.size;
  next.edges = (int64_t)hc.edges;
  next.has_queue = false;
}

// One BellmanFord round from `from` into `next`: the reference's dense push
// (DENSE_FORWARD) when push, else the pull-reduce, which for a dense round
// reads the frontier's distances from a snapshot.
static void bf_round(pm_graph *g, VertexSubset &from, VertexSubset &next, int64_t threshold, bool push,
                     int32_t *d_dist, const int32_t *w_out, const int32_t *w_in, bool *dense) {
  Engine &E = g->E;
  if (push) {
    edgeMap<int32_t>(E, from, BF_F{d_dist, from.bits}, next, threshold, DENSE_FORWARD, w_out, w_in, dense);
  } else if (E.tune.bf_dense == 2 && go_dense(from, threshold) && !g->is_part) {
    bf_round_red(g, from, next, d_dist, w_out);
    *dense = true;
  } else if (go_dense(from, threshold) && !g->is_part) {
    int32_t *fd = (int32_t *)g->scratch_buf(36, (size_t)g->n * 4);
    PM_LAUNCH(k_bf_snapshot, E.grid_for(g->n, 256, 16), 256, 0, E.stream, (int32_t)g->n, from.bits, d_dist, fd);
    edgeMapReduce<int32_t>(E, from, BF_FD{d_dist, fd}, next, threshold, w_out, w_in, dense);
  } else {
    edgeMapReduce<int32_t>(E, from, BF_F{d_dist, from.bits}, next, threshold, w_out, w_in, dense);
  }
}

__global__ void k_bf_init(int32_t *dist, int64_t n, int32_t src) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
    dist[v] = v == src ? 0 : kDevBFInf;
}

// Delta-stepping schedule (tunable bf_delta = Delta > 0).  The frontier F
// holds the vertices whose distance fell and whose out-edges are not yet
// relaxed.  Each round relaxes only F_near = {v in F : dist[v] < T}; the
// others stay in F for a later round.  When F_near is empty, T moves to the
// least distance left in F plus Delta.  Any order of relaxing the vertices
// whose distance fell ends at the exact shortest distances, so the result
// is the plain rounds' result; relaxing near vertices first lets fewer
// distances fall twice.
__global__ void k_bf_split(int32_t n, const int32_t *__restrict__ out_off, const uint32_t *__restrict__ cur,
                           const int32_t *dist, int32_t T, uint32_t *__restrict__ near, uint32_t *__restrict__ far,
                           Counters *c) {
  const int64_t words = ((int64_t)n + 31) / 32;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  unsigned long long ns = 0, ne = 0, fs = 0, far_top = 0;  // far_top: max of (kDevBFInf - dist)
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < words; i += stride) {
    uint32_t w = cur[i], wn = 0, wf = 0;
    while (w) {
      const int b = __ffs(w) - 1;
      w &= w - 1;
      const int v = (int)(i * 32 + b);
      const int32_t d = *((volatile const int32_t *)dist + v);
      if (d < T) {
        wn |= 1u << b;
        ns++;
        ne += __ldg(out_off + v + 1) - __ldg(out_off + v);
      } else {
        wf |= 1u << b;
        fs++;
        far_top = max(far_top, (unsigned long long)(kDevBFInf - min(d, kDevBFInf)));
      }
    }
    near[i] = wn;
    far[i] = wf;
  }
  ns = warp_sum(ns);
  ne = warp_sum(ne);
  fs = warp_sum(fs);
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) far_top = max(far_top, __shfl_down_sync(0xffffffffu, far_top, d));
  if (lane_id() == 0) {
    if (ns) {
      atomicAdd(&c[0].size, ns);
      atomicAdd(&c[0].edges, ne);
    }
    if (fs) {
      atomicAdd(&c[1].size, fs);
      atomicMax(&c[1].aux, far_top);
    }
  }
}

// dst |= src, counting the union's size and out-degree sum.
__global__ void k_bits_or_count(int32_t n, const int32_t *__restrict__ out_off, uint32_t *dst,
                                const uint32_t *__restrict__ src, Counters *c) {
  const int64_t words = ((int64_t)n + 31) / 32;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  unsigned long long s = 0, e = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < words; i += stride) {
    uint32_t w = dst[i] | src[i];
    dst[i] = w;
    s += __popc(w);
    while (w) {
      const int b = __ffs(w) - 1;
      w &= w - 1;
      const int v = (int)(i * 32 + b);
      e += __ldg(out_off + v + 1) - __ldg(out_off + v);
    }
  }
  s = warp_sum(s);
  e = warp_sum(e);
  if (lane_id() == 0 && s) {
    atomicAdd(&c->size, s);
    atomicAdd(&c->edges, e);
  }
}

static void run_bellman_ford_delta(pm_graph *g, int32_t *d_dist, int64_t threshold, bool push, VertexSubset &cur,
                                   VertexSubset &next, pm_traversal_stats &s) {
  Engine &E = g->E;
  const int64_t n = g->n;
  const int32_t delta = E.tune.bf_delta;
  const int32_t *w_out = g->w_i32_out.as<int32_t>(), *w_in = g->w_i32_in.as<int32_t>();
  VertexSubset near;
  near.n = (int32_t)n;
  near.bits = (uint32_t *)g->scratch_buf(33, (size_t)cur.words() * 4);
  near.queue = (int32_t *)g->scratch_buf(34, (size_t)n * 4);
  uint32_t *far = (uint32_t *)g->scratch_buf(35, (size_t)cur.words() * 4);
  Counters *dc = (Counters *)g->scratch_buf(32, 2 * sizeof(Counters));
  Counters hc[2];
  const int grid = E.grid_for(cur.words(), 256, 16);
  int64_t T = delta;
  while (cur.size > 0) {
    PM_CUDA(cudaMemsetAsync(dc, 0, 2 * sizeof(Counters), E.stream));
    PM_LAUNCH(k_bf_split, grid, 256, 0, E.stream, (int32_t)n, E.g.out.off, cur.bits, d_dist,
              (int32_t)std::min<int64_t>(T, kDevBFInf), near.bits, far, dc);
    PM_CUDA(cudaMemcpyAsync(hc, dc, 2 * sizeof(Counters), cudaMemcpyDeviceToHost, E.stream));
    PM_CUDA(cudaStreamSynchronize(E.stream));
    near.size = (int64_t)hc[0].size;
    near.edges = (int64_t)hc[0].edges;
    near.has_queue = false;
    if (near.size == 0) {  // the rest lies at T or beyond: next bound from the least of it
      const int64_t least = (int64_t)kDevBFInf - (int64_t)hc[1].aux;
      T = std::max<int64_t>(T, least) + delta;
      continue;
    }
    bool dense = false;
    s.edges_visited += near.edges;
    bf_round(g, near, next, threshold, push, d_dist, w_out, w_in, &dense);
    // the new frontier: what fell this round and what waited
    PM_CUDA(cudaMemsetAsync(dc, 0, sizeof(Counters), E.stream));
    PM_LAUNCH(k_bits_or_count, grid, 256, 0, E.stream, (int32_t)n, E.g.out.off, next.bits, far, dc);
    PM_CUDA(cudaMemcpyAsync(hc, dc, sizeof(Counters), cudaMemcpyDeviceToHost, E.stream));
    PM_CUDA(cudaStreamSynchronize(E.stream));
    next.size = (int64_t)hc[0].size;
    next.edges = (int64_t)hc[0].edges;
    next.has_queue = false;
    s.rounds++;
    s.dense_rounds += dense;
    std::swap(cur, next);
    if (s.rounds > 4 * (g->n + 1)) fail(PM_ERR_INVALID_ARG, "BellmanFord did not converge");
  }
}

void run_bellman_ford(pm_graph *g, int32_t src, int32_t *d_dist, int64_t threshold,
                      pm_traversal_stats *st) {
  Engine &E = g->E;
  VertexSubset cur = g->subset(0), next = g->subset(1);
  PM_LAUNCH(k_bf_init, E.grid_for(g->n, 256, 16), 256, 0, E.stream, d_dist, g->n, src);
  subset_single(E, cur, src);
  pm_traversal_stats s{};
  s.reached = 1;
  const int32_t *w_out = g->w_i32_out.as<int32_t>(), *w_in = g->w_i32_in.as<int32_t>();
  E.tag = "bellman_ford";
  // dense rounds: the pull-reduce, or the reference's dense push (DENSE_FORWARD,
  // numa-BellmanFord.C:182), which reads only the frontier's out-edges
  const bool push = E.tune.bf_dense == 1 && !g->is_part;
  if (E.tune.bf_delta > 0 && !g->is_part) {
    run_bellman_ford_delta(g, d_dist, threshold, push, cur, next, s);
    if (st) *st = s;
    return;
  }
  while (cur.size > 0) {
    bool dense = false;
    s.edges_visited += cur.edges;
    bf_round(g, cur, next, threshold, push, d_dist, w_out, w_in, &dense);
    part_exchange(g, d_dist, 4);  // a partition: distances and frontier of every rank
    part_round(g, next);
    s.rounds++;
    s.dense_rounds += dense;
    std::swap(cur, next);
    if (s.rounds > g->n + 1) fail(PM_ERR_INVALID_ARG, "BellmanFord did not converge");
  }
  if (st) *st = s;
}

// ===========================================================================
// PageRank  (numa-PageRank.C:64-148 PR_F / PR_Vertex_F / PR_Vertex_Reset,
// loop 273-335)
// One pull-reduce per iteration.  The frontier rides in the contribution
// array: c[s] = p[s] / outdeg(s) when s is in the frontier (>= +0), and
// -0.0 when it is not.  -0.0 is the exact additive identity, so the sum of
// a row's contributions is -0.0 exactly when no in-neighbour is in the
// frontier: its sign bit is the next-frontier bit.  commit() applies the
// push sum to the stale p_next, damps frontier vertices (PR_Vertex_F),
// zeroes their p_curr (PR_Vertex_Reset) and writes next round's
// contribution; the FP64 L1 residual is reduced on the side.
// ===========================================================================
template <class T>
struct PR_F {
  const T *c_cur;
  T *c_next;
  T *pc;
  T *pn;
  const int32_t *out_off;
  T damping, added;
  using Acc = T;
  static constexpr bool kHubs = true;  // edge() is a plain load of c_cur[s]
  __device__ __forceinline__ bool cond(int) const { return true; }
  __device__ __forceinline__ Acc identity() const { return T(-0.0); }
  __device__ __forceinline__ Acc edge(int s, int, int) const { return __ldg(c_cur + s); }
  __device__ __forceinline__ Acc edge_value(Acc v, int, int) const { return v; }
  __device__ __forceinline__ Acc combine(Acc a, Acc b) const { return a + b; }
  __device__ __forceinline__ bool commit(int d, Acc acc, double2 &resid) const {
    const bool in_f = !signbit(__ldg(c_cur + d));
    const bool hit = !signbit(acc);
    const T old = pc[d];
    T nb = pn[d] + acc;
    if (in_f) {
      nb = damping * nb + added;
      pc[d] = T(0);
    }
    pn[d] = nb;
    const int deg = __ldg(out_off + d + 1) - __ldg(out_off + d);
    c_next[d] = hit ? (deg > 0 ? nb / T(deg) : T(0)) : T(-0.0);
    resid.x += fabs((double)nb - (double)old);
    resid.y += fabs((double)nb);
    return hit;
  }
};

template <class T>
__global__ void k_pr_init(T *pc, T *pn, T *c, const int32_t *out_off, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const T p0 = T(1) / T(n);
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
    pc[v] = p0;
    pn[v] = T(0);
    int deg = out_off[v + 1] - out_off[v];
    c[v] = deg > 0 ? p0 / T(deg) : T(0);
  }
}

__global__ void k_copy_daux(const Counters *cnt, double *dst) { *dst = cnt->daux; }

template <class T>
void run_pagerank(pm_graph *g, int iters, double damping, T *d_out, double *d_resid) {
  Engine &E = g->E;
  const int64_t n = g->n;
  T *pc = (T *)g->scratch_buf(0, (size_t)n * sizeof(T));
  T *pn = (T *)g->scratch_buf(1, (size_t)n * sizeof(T));
  T *c0 = (T *)g->scratch_buf(2, (size_t)n * sizeof(T));
  T *c1 = (T *)g->scratch_buf(3, (size_t)n * sizeof(T));
  // out-degrees of the whole graph (a partition's CSR holds only its own
  // destinations' edges)
  const int32_t *deg_off = g->is_part ? g->glob_off.as<int32_t>() : E.g.out.off;
  PM_LAUNCH((k_pr_init<T>), E.grid_for(n, 256, 16), 256, 0, E.stream, pc, pn, c0, deg_off, n);
  const T dmp = (T)damping, added = (T)((1.0 - damping) * (1.0 / (double)n));
  // FP32: the contributions of the highest out-degree sources come from each
  // SM's shared memory (hub_cache tunable; same values, same sums)
  HubCache<T> hubs;
  if constexpr (std::is_same<T, float>::value) {
    ensure_hubs(g);
    if (g->hub_count > 0) hubs = HubCache<T>{g->hub_idx.as<int32_t>(), g->hub_vals.as<T>(), g->hub_count};
  }
  E.run_loop(loop_key("pagerank", (int)sizeof(T), iters, damping, pc, pn, c0, c1, d_resid), [&] {
    T *a = pc, *b = pn, *x = c0, *y = c1;
    for (int it = 0; it < iters; ++it) {
      PM_CUDA(cudaMemsetAsync(E.d_cnt, 0, sizeof(Counters), E.stream));
      E.prof.begin("pagerank", E.stream);
      if constexpr (std::is_same<T, float>::value)
        if (hubs.count > 0) hub_values(g, x);
      launch_pull_reduce<int>(E, PR_F<T>{x, y, a, b, deg_off, dmp, added}, nullptr, nullptr, E.d_cnt, hubs);
      E.prof.end(E.stream);
      part_exchange(g, y, sizeof(T));  // a partition: next contributions of every rank
      if (d_resid) PM_LAUNCH(k_copy_daux, 1, 1, 0, E.stream, E.d_cnt, d_resid + it);
      std::swap(a, b);
      std::swap(x, y);
    }
  });
  part_exchange(g, iters % 2 ? pn : pc, sizeof(T));  // a partition: every rank's ranks
  PM_CUDA(cudaMemcpyAsync(d_out, iters % 2 ? pn : pc, (size_t)n * sizeof(T), cudaMemcpyDeviceToDevice,
                          E.stream));
}

// ===========================================================================
// SpMV  (numa-SPMV.C:56-110 SPMV_F / SPMV_Vertex_Reset, loop 168-193)
// All vertices are active every iteration: y[d] = sum w(s,d) x[s] as a
// pull over the CSC with the weights permuted to CSC order; x <- y.
// ===========================================================================
template <class T>
struct SPMV_F {
  const T *x;
  T *y;
  using Acc = T;
  static constexpr int kLaneEdges = 5;  // 5 % faster per pass than 6 at scale 24
  __device__ __forceinline__ bool cond(int) const { return true; }
  __device__ __forceinline__ Acc identity() const { return T(-0.0); }
  __device__ __forceinline__ Acc edge(int s, int, float w) const { return T(w) * __ldg(x + s); }
  __device__ __forceinline__ Acc combine(Acc a, Acc b) const { return a + b; }
  __device__ __forceinline__ bool commit(int d, Acc acc, double2 &norm) const {
    const T v = acc + T(0);
    y[d] = v;
    norm.x += fabs((double)v);
    return false;
  }
};

// T = float: the FP32 storage and sums of the benchmark; T = double: the same
// iteration in FP64, the yardstick for the FP32 result's error.
template <class T>
void run_spmv(pm_graph *g, const T *d_x0, int iters, T *d_y, double *d_norm) {
  Engine &E = g->E;
  const int64_t n = g->n;
  T *x = (T *)g->scratch_buf(0, (size_t)n * sizeof(T));
  T *y = (T *)g->scratch_buf(1, (size_t)n * sizeof(T));
  PM_CUDA(cudaMemcpyAsync(x, d_x0, (size_t)n * sizeof(T), cudaMemcpyDeviceToDevice, E.stream));
  const WPair *w_in = ensure_f32_pairs(g);
  E.run_loop(loop_key("spmv", (int)sizeof(T), iters, x, y, w_in, d_norm), [&] {
    T *a = x, *b = y;
    for (int it = 0; it < iters; ++it) {
      PM_CUDA(cudaMemsetAsync(E.d_cnt, 0, sizeof(Counters), E.stream));
      E.prof.begin("spmv", E.stream);
      launch_pull_reduce<WPair>(E, SPMV_F<T>{a, b}, w_in, nullptr, E.d_cnt);
      E.prof.end(E.stream);
      part_exchange(g, b, sizeof(T));  // a partition: every rank's y
      if (d_norm) PM_LAUNCH(k_copy_daux, 1, 1, 0, E.stream, E.d_cnt, d_norm + it);
      std::swap(a, b);
    }
  });
  PM_CUDA(cudaMemcpyAsync(d_y, iters % 2 ? y : x, (size_t)n * sizeof(T), cudaMemcpyDeviceToDevice, E.stream));
}

// ===========================================================================
// Belief propagation, 2 states  (numa-BP.C:89-140 BP_F / BP_Vertex_Reset,
// edgeMapDenseBPNoRep 179-230, loop 280-316)
// With one psi for every edge the message of an edge s->d depends on d
// alone, so prod'_d *= belief_d ^ k_d where k_d counts d's in-neighbours in
// the frontier: the pull reduces k_d and commit() applies it, in logs.
// Messages are normalised to sum 1 (see pm_bp in the header).
// ===========================================================================
template <class T> struct Vec2;
template <> struct Vec2<float> { using type = float2; };
template <> struct Vec2<double> { using type = double2; };
__device__ __forceinline__ float bp_exp(float x) { return expf(x); }
__device__ __forceinline__ double bp_exp(double x) { return exp(x); }
__device__ __forceinline__ float bp_log(float x) { return logf(x); }
__device__ __forceinline__ double bp_log(double x) { return log(x); }

template <class T>
struct BP_F {
  using V = typename Vec2<T>::type;
  const uint32_t *cur;
  const V *lc;
  V *ln;
  const V *prior;
  T p00, p01, p10, p11;
  using Acc = int32_t;
  static constexpr int kLaneEdges = 5;  // 2 % faster per pass than 6 at scale 24
  __device__ __forceinline__ bool cond(int) const { return true; }
  __device__ __forceinline__ Acc identity() const { return 0; }
  __device__ __forceinline__ Acc edge(int s, int, int) const { return test_bit(cur, s) ? 1 : 0; }
  __device__ __forceinline__ Acc combine(Acc a, Acc b) const { return a + b; }
  __device__ __forceinline__ bool commit(int d, Acc k, double2 &) const {
    const bool in_f = test_bit(cur, d);
    V out;
    if (in_f)
      out.x = out.y = T(0);
    else
      out = ln[d];
    if (k > 0) {
      const V l = lc[d], pr = prior[d];
      const T lm = l.x > l.y ? l.x : l.y;
      const T a0 = pr.x * bp_exp(l.x - lm), a1 = pr.y * bp_exp(l.y - lm);
      const T b0 = p00 * a0 + p01 * a1, b1 = p10 * a0 + p11 * a1;
      const T lz = bp_log(b0 + b1);
      out.x += (T)k * (bp_log(b0) - lz);
      out.y += (T)k * (bp_log(b1) - lz);
    }
    if (in_f || k > 0) ln[d] = out;
    return k > 0;
  }
};

template <class T>
void run_bp(pm_graph *g, const T *d_prior, const T *psi, int iters, T *d_out) {
  using V = typename Vec2<T>::type;
  Engine &E = g->E;
  const int64_t n = g->n;
  V *lc = (V *)g->scratch_buf(0, (size_t)n * sizeof(V));
  V *ln = (V *)g->scratch_buf(1, (size_t)n * sizeof(V));
  PM_CUDA(cudaMemsetAsync(lc, 0, (size_t)n * sizeof(V), E.stream));
  PM_CUDA(cudaMemsetAsync(ln, 0, (size_t)n * sizeof(V), E.stream));
  VertexSubset cur = g->subset(0), next = g->subset(1);
  subset_all(E, cur);
  E.run_loop(loop_key("bp", (int)sizeof(T), iters, lc, ln, cur.bits, next.bits, d_prior, (double)psi[0],
                      (double)psi[1], (double)psi[2], (double)psi[3]),
             [&] {
               V *a = lc, *b = ln;
               uint32_t *fa = cur.bits, *fb = next.bits;
               for (int it = 0; it < iters; ++it) {
                 PM_CUDA(cudaMemsetAsync(E.d_cnt, 0, sizeof(Counters), E.stream));
                 E.prof.begin("bp", E.stream);
                 launch_pull_reduce<int>(
                     E, BP_F<T>{fa, a, b, (const V *)d_prior, psi[0], psi[1], psi[2], psi[3]}, nullptr,
                     fb, E.d_cnt);
                 E.prof.end(E.stream);
                 part_exchange_bits(g, fb);  // a partition: the next frontier of every rank
                 std::swap(a, b);
                 std::swap(fa, fb);
               }
             });
  part_exchange(g, iters % 2 ? ln : lc, sizeof(V));  // a partition: every rank's log-products
  PM_CUDA(cudaMemcpyAsync(d_out, iters % 2 ? ln : lc, (size_t)n * sizeof(V), cudaMemcpyDeviceToDevice,
                          E.stream));
}

// ===========================================================================
// PageRankDelta  (numa-PageRankDelta.C:64-132 PR_F / PR_Vertex_F_FirstRound /
// PR_Vertex_F / PR_Vertex_Reset, loop 198-230)
// Only vertices whose rank moved by more than eps2 of itself push their
// change.  c[s] holds Delta[s]/outdeg(s) for s in the frontier and 0 elsewhere.
// Dense rounds pull sum c[s] over the CSC and commit the vertexFilter of
// every row (the reference's filter over All) into a second array; sparse
// rounds push c[s] to the out-neighbours with atomicAdd into ngh, then clear
// c on the old frontier and commit the touched vertices only (an untouched
// vertex gets Delta = 0: its rank stays and it leaves the frontier).  The
// first round (p = 0, Delta = 1/n, frontier = all) always runs dense.
// ===========================================================================
template <class T>
__device__ __forceinline__ bool prd_commit(T acc, bool first, T damping, T added, T one_over_n, T eps2,
                                           T &p, T &c, int deg) {
  T dl;
  if (first) {
    const T p0 = p;
    dl = damping * (p0 + acc) + added - p0;
    p = p0 + dl;
    dl -= one_over_n;
  } else {
    dl = acc * damping;
    p += dl;
  }
  const bool in = fabs(dl) > eps2 * p;
  c = in && deg > 0 ? dl / T(deg) : T(0);
  return in;
}

template <class T>
struct PRD_F {
  const T *c_cur;
  T *c_next;
  T *p;
  T *ngh;  // sparse rounds: atomically summed pushes
  const int32_t *out_off;
  T damping, added, one_over_n, eps2;
  bool first;
  using Acc = T;
  __device__ __forceinline__ bool cond(int) const { return true; }
  __device__ __forceinline__ bool updateAtomic(int s, int d, int) const {
    atomicAdd(ngh + d, __ldg(c_cur + s));
    return true;
  }
  __device__ __forceinline__ Acc identity() const { return T(0); }
  __device__ __forceinline__ Acc edge(int s, int, int) const { return __ldg(c_cur + s); }
  __device__ __forceinline__ Acc combine(Acc a, Acc b) const { return a + b; }
  __device__ __forceinline__ bool commit(int d, Acc acc, double2 &) const {
    T pd = p[d], cd;
    const bool in = prd_commit(acc, first, damping, added, one_over_n, eps2, pd, cd,
                               __ldg(out_off + d + 1) - __ldg(out_off + d));
    p[d] = pd;
    c_next[d] = cd;
    return in;
  }
};

template <class T>
struct PRD_Clear {
  T *c;
  __device__ __forceinline__ void operator()(int v) const { c[v] = T(0); }
};

template <class T>
struct PRD_SparseCommit {
  T *c, *p, *ngh;
  const int32_t *out_off;
  T damping, eps2;
  __device__ __forceinline__ bool operator()(int v) const {
    const T acc = ngh[v];
    ngh[v] = T(0);
    T pv = p[v], cv;
    const bool in = prd_commit(acc, false, damping, T(0), T(0), eps2, pv, cv,
                               __ldg(out_off + v + 1) - __ldg(out_off + v));
    p[v] = pv;
    c[v] = cv;
    return in;
  }
};

template <class T>
__global__ void k_prd_init(T *c, T *p, T *ngh, const int32_t *out_off, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const T d0 = T(1) / T(n);
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
    const int deg = out_off[v + 1] - out_off[v];
    c[v] = deg > 0 ? d0 / T(deg) : T(0);
    p[v] = T(0);
    ngh[v] = T(0);
  }
}

template <class T>
void run_pagerank_delta(pm_graph *g, int iters, double damping, double eps2, T *d_out, int64_t threshold,
                        pm_traversal_stats *st) {
  Engine &E = g->E;
  const int64_t n = g->n;
  T *c0 = (T *)g->scratch_buf(0, (size_t)n * sizeof(T));
  T *c1 = (T *)g->scratch_buf(1, (size_t)n * sizeof(T));
  T *p = (T *)g->scratch_buf(2, (size_t)n * sizeof(T));
  T *ngh = (T *)g->scratch_buf(3, (size_t)n * sizeof(T));
  PM_LAUNCH((k_prd_init<T>), E.grid_for(n, 256, 16), 256, 0, E.stream, c0, p, ngh, E.g.out.off, n);
  VertexSubset cur = g->subset(0), next = g->subset(1);
  subset_all(E, cur);
  const T one_over_n = T(1.0 / (double)n), added = T((1.0 - damping) / (double)n);
  pm_traversal_stats s{};
  E.tag = "pagerank_delta";
  for (int it = 0; it < iters; ++it) {
    const bool first = it == 0;
    PRD_F<T> f{c0, c1, p, ngh, E.g.out.off, (T)damping, added, one_over_n, (T)eps2, first};
    bool dense = false;
    s.edges_visited += cur.edges;
    // the first round commits every vertex, so it always pulls
    edgeMapReduce<int>(E, cur, f, next, first ? 0 : threshold, nullptr, nullptr, &dense);
    if (dense) {
      std::swap(c0, c1);
      std::swap(cur, next);
    } else {
      vertexMap(E, cur, PRD_Clear<T>{c0});
      vertexFilter(E, next, PRD_SparseCommit<T>{c0, p, ngh, E.g.out.off, (T)damping, (T)eps2}, cur);
    }
    s.rounds++;
    s.dense_rounds += dense;
  }
  s.reached = cur.size;
  PM_CUDA(cudaMemcpyAsync(d_out, p, (size_t)n * sizeof(T), cudaMemcpyDeviceToDevice, E.stream));
  if (st) *st = s;
}

// explicit instantiations used by the C ABI
template void run_pagerank<float>(pm_graph *, int, double, float *, double *);
template void run_pagerank<double>(pm_graph *, int, double, double *, double *);
template void run_spmv<float>(pm_graph *, const float *, int, float *, double *);
template void run_spmv<double>(pm_graph *, const double *, int, double *, double *);
template void run_bp<float>(pm_graph *, const float *, const float *, int, float *);
template void run_bp<double>(pm_graph *, const double *, const double *, int, double *);
template void run_pagerank_delta<float>(pm_graph *, int, double, double, float *, int64_t, pm_traversal_stats *);
template void run_pagerank_delta<double>(pm_graph *, int, double, double, double *, int64_t,
                                         pm_traversal_stats *);

}  // namespace pm
