// polymer.cuh -- the B200 edgeMap / vertexMap engine.
//
// This header keeps the programming model of Polymer's polymer.h: a graph,
// a vertexSubset (frontier), edgeMap(G, frontier, F, threshold, option),
// vertexMap and vertexFilter, with user functors that expose
//   cond(d)                 -> should d still be updated       (polymer.h:2240-2309)
//   updateAtomic(s, d, w)   -> apply s->d, true if d activated (sparse / dense push)
// and, for the reducing dense pull (edgeMapDenseReduce, polymer.h:1097-1168),
//   identity()/edge(s,d,w)/combine(a,b)/commit(d,acc)  (initFunc/reduceFunc/
//   combineFunc of the reference; commit also runs the fused vertexMap).
// Functors are __device__ objects passed by value to the kernels and inlined
// at compile time, as the reference's templates are inlined on the CPU.
//
// Device layout (one GPU, everything resident in HBM):
//   CSR out-edges and CSC in-edges, int32 offsets (n+1) and ids (m);
//   a frontier is a bitmap of ceil(n/32) words plus, when it came from a
//   sparse round, a queue of int32 ids (the reference's LocalFrontier b / s,
//   polymer.h:527-639).
// Kernels:
//   k_sparse_push   queue -> queue+bitmap, CTA / warp / scan-gather expansion,
//                   warp-aggregated queue appends          (edgeMapSparseV3)
//   k_dense_pull    bitmap -> bitmap, one thread per vertex over the CSC with
//                   early exit on cond, long rows deferred to one warp each
//                                                          (edgeMapDense*)
//   k_pull_reduce   bitmap -> bitmap, edge-balanced warp groups with a
//                   segmented warp reduction; rows above kHeavyDeg are summed
//                   by k_heavy_reduce chunks first          (edgeMapDenseReduce)
//   k_dense_push    bitmap -> bitmap over the CSR with atomics
//                                                          (edgeMapDenseForward)
#pragma once
#include <algorithm>
#include <array>
#include <cstdio>
#include <cstring>
#include <type_traits>
#include <utility>
#include <vector>

#include "pm_common.cuh"

namespace pm {

constexpr int kGroupWork = 1024;   // work units (edges + kRowWork per row) of one warp group
constexpr int kRowWork = 4;       // a row costs about as much as this many edges
constexpr int kHeavyDeg = 1024;    // default: rows above this degree are split in chunks
constexpr int kChunkEdges = 4096;  // edges of one heavy chunk (one CTA)
constexpr int kChunkThreads = 256;
constexpr int kPullScan = 32;      // edges a thread scans before deferring a row
// Sparse-push degree bins.  A frontier just under the dense threshold can
// hold tens of thousands of rows of a few hundred edges: expanded one row at
// a time per CTA, a few CTAs serialise most of the round, so rows from 256
// edges up are spread over the whole grid (scale-22 BFS x16: 4096 -> 256
// took 11.6 ms to 6.8 ms).
constexpr int kCtaExpand = 128;    // default: sparse push CTA-wide expansion from this degree
constexpr int kGridExpand = 256;   // default: sparse push rows from this degree use the whole grid
constexpr int kMaxHubs = 4096;     // hub rows one sparse round can hand to the grid kernel

// One adjacency direction.
struct Adj {
  const int32_t *off = nullptr;     // n+1
  const int32_t *idx = nullptr;     // m
  const int32_t *gstart = nullptr;  // ngroups+1 warp-group row starts (32-aligned; last = n)
  const int32_t *hrow = nullptr;    // heavy chunk -> row
  const int32_t *hfirst = nullptr;  // row -> its first heavy chunk (rows with deg > heavy_deg)
  int32_t ngroups = 0;
  int32_t nchunks = 0;
};

// Checked builds (-DPM_CHECK=1, libpolymer_b200_check.so; the stand-in for a
// memory checker): a vertex id read from the graph or a queue is tested
// against [0, n) before it indexes anything.  A bad one sets the graph's
// check word and is replaced by vertex 0, so the kernel stays in bounds and
// the call ends with PM_ERR_BAD_GRAPH.  Default builds compile the tests (and
// the word) out: their kernels are the same code as without the option.
#ifndef PM_CHECK
#define PM_CHECK 0
#endif

struct GraphView {
  int32_t n = 0;
  int64_t m = 0;
  int32_t heavy_deg = kHeavyDeg;      // rows with more edges than this are chunked
  int32_t cta_expand = kCtaExpand;    // sparse push degree bins
  int32_t grid_expand = kGridExpand;
  int32_t push_agg = 0;               // warp-aggregated min pushes (MinPush functors)
  Adj out;  // CSR
  Adj in;   // CSC (aliases out for symmetric graphs)
#if PM_CHECK
  unsigned *check = nullptr;  // the graph's bounds-check word
#endif
};
__device__ __forceinline__ int checked_id(const GraphView &g, int v) {
#if PM_CHECK
  if ((unsigned)v >= (unsigned)g.n) {
    atomicOr(g.check, 1u);
    return 0;
  }
#endif
  return v;
}
// A pull source: with the hub cache, ~s < hub_count names a cached hub.
template <bool HUBS>
__device__ __forceinline__ int checked_src(const GraphView &g, int hub_count, int s) {
#if PM_CHECK
  if (HUBS && s < 0) {
    if (~s < hub_count) return s;
    atomicOr(g.check, 1u);
    return 0;
  }
  return checked_id(g, s);
#else
  (void)hub_count;
  return s;
#endif
}

__device__ __forceinline__ bool test_bit(const uint32_t *__restrict__ b, int v) {
  return (__ldg(b + (v >> 5)) >> (v & 31)) & 1u;
}
// Sets bit v; true if this call set it (the bit was clear).
__device__ __forceinline__ bool set_bit_new(uint32_t *b, int v) {
  uint32_t mask = 1u << (v & 31);
  return !(atomicOr(b + (v >> 5), mask) & mask);
}

template <class W>
__device__ __forceinline__ W load_w(const W *w, int64_t e) {
  return w ? __ldg(w + e) : W(0);
}

// Float weights stored beside their source ids, one 8-byte record per CSC
// slot, so that a pull reads both with one load.
struct __align__(8) WPair {
  int32_t src;
  float w;
};
template <class W> struct EdgeT { using type = W; };  // weight type F::edge receives
template <> struct EdgeT<WPair> { using type = float; };

// Source id of CSC slot e; with paired weights also its weight (into wv).
// The ids (and pairs) are read once per pass: streaming loads (evict-first
// in L1 and L2) leave the caches to the gathered values -- SpMV passes 3 %
// faster at scale 24, PageRank 0.7 %.
template <class W>
__device__ __forceinline__ int load_src(const int32_t *__restrict__ idx, const W *__restrict__ w, int64_t e,
                                        typename EdgeT<W>::type &wv) {
  if constexpr (std::is_same<W, WPair>::value) {
    const int2 p = __ldcs(reinterpret_cast<const int2 *>(w) + e);
    wv = __int_as_float(p.y);
    return p.x;
  } else {
    return __ldcs(idx + e);
  }
}
// Weight of CSC slot e (already loaded by load_src when paired).
template <class W>
__device__ __forceinline__ typename EdgeT<W>::type edge_w(const W *w, int64_t e, typename EdgeT<W>::type wv) {
  if constexpr (std::is_same<W, WPair>::value)
    return wv;
  else
    return load_w(w, e);
}

// ---------------------------------------------------------------------------
// Warp-collective append of activated vertices to the next queue.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void emit_queue(bool act, int d, int32_t *queue, int32_t qcap,
                                           Counters *cnt) {
  unsigned bal = __ballot_sync(0xffffffffu, act);
  if (!bal) return;
  int lane = lane_id();
  int leader = __ffs(bal) - 1;
  unsigned long long base = 0;
  if (lane == leader) base = atomicAdd(&cnt->size, (unsigned long long)__popc(bal));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (act) {
    unsigned long long p = base + __popc(bal & ((1u << lane) - 1u));
    if (p < (unsigned long long)qcap)
      queue[p] = d;
    else
      atomicOr(&cnt->err, (unsigned)kErrQueueOverflow);
  }
}

// ---------------------------------------------------------------------------
// Sparse push (edgeMapSparseV3, polymer.h:1928-2003): expand the out-edges of
// every queued vertex; d joins the next frontier when cond(d) &&
// updateAtomic(s, d, w) holds and its bit was not yet set this round.
// Load balance: rows >= g.cta_expand are expanded by the whole CTA, rows >= 32
// by one warp, the rest through a CTA-wide scan of their degrees.
// ---------------------------------------------------------------------------
// updateAtomic with the edge weight when the functor takes one
// (polymer-wgh.h), without it otherwise (polymer.h's unweighted functors,
// e.g. numa-Components.C:71-75).
template <class F, class Wv, class = void>
struct TakesWeight : std::false_type {};
template <class F, class Wv>
struct TakesWeight<F, Wv, std::void_t<decltype(std::declval<F &>().updateAtomic(0, 0, std::declval<Wv>()))>>
    : std::true_type {};
template <class F, class Wv>
__device__ __forceinline__ bool update_atomic(F &f, int s, int d, Wv w) {
  if constexpr (TakesWeight<F, Wv>::value)
    return f.updateAtomic(s, d, w);
  else
    return f.updateAtomic(s, d);
}

template <class F, class W>
__device__ __forceinline__ bool push_edge(const GraphView &g, F &f, const W *w, int s, int64_t e,
                                          uint32_t *next_bits, int &d_out) {
  int d = checked_id(g, __ldg(g.out.idx + e));
  d_out = d;
  if (f.cond(d) && update_atomic(f, s, d, load_w(w, e))) return set_bit_new(next_bits, d);
  return false;
}

// A functor whose updateAtomic(s, d, w) is "atomicMin(min_target() + d,
// push_value(s, w)) lowered the value" (Components' labels, BellmanFord's
// distances) declares those two members; its pushes from many sources are
// then warp-aggregated on the sparse push's short rows when the tunable
// push_agg is set: lanes with the same target combine their values with one
// warp reduction and the group's first lane issues a single atomicMin.  The
// target ends at the same minimum and is activated when the minimum lowered
// it, as with one atomic per edge.
template <class F, class = void>
struct MinPush : std::false_type {};
template <class F>
struct MinPush<F, std::void_t<decltype(std::declval<const F &>().min_target())>> : std::true_type {};

// Warp-collective (every lane of the warp calls it; valid marks the lanes
// with an edge): the aggregated form of push_edge for MinPush functors.
template <class F, class W>
__device__ __forceinline__ bool push_edge_min(const GraphView &g, F &f, const W *w, bool valid, int s,
                                              int64_t e, uint32_t *next_bits, int &d_out) {
  int d = -1;
  int32_t v = 0x7fffffff;
  if (valid) {
    d = checked_id(g, __ldg(g.out.idx + e));
    valid = f.cond(d);
    if (valid) v = f.push_value(s, load_w(w, e));
  }
  d_out = d;
  // lanes without an edge get keys no target has (ids are >= 0)
  const unsigned peers = __match_any_sync(0xffffffffu, valid ? d : -1 - (int)(threadIdx.x & 31));
  const int32_t gmin = __reduce_min_sync(peers, v);
  if (!valid || (int)(threadIdx.x & 31) != __ffs(peers) - 1) return false;
  return gmin < *((volatile int32_t *)f.min_target() + d) && gmin < atomicMin(f.min_target() + d, gmin) &&
         set_bit_new(next_bits, d);
}

template <class F, class W>
__global__ void __launch_bounds__(256) k_sparse_push(GraphView g, const int32_t *__restrict__ queue,
                                                     int32_t qsize, F f, const W *__restrict__ w,
                                                     int32_t *__restrict__ next_queue,
                                                     uint32_t *__restrict__ next_bits, int32_t qcap,
                                                     Counters *cnt, int32_t *__restrict__ hubs,
                                                     Counters *hub_cnt, const RoundGate *gate = nullptr) {
  __shared__ int s_pos[256];
  __shared__ int s_v[256];
  __shared__ int s_o[256];
  __shared__ int s_warp_tot[8];
  __shared__ int s_owner, s_cv, s_co, s_cd;
  if (gate) {  // a round driven on the GPU: the queue is what k_bits_to_queue
    // wrote just before, counted in cnt[2] (cnt is the engine's counter array)
    if (!gate->active || gate->dense) return;
    qsize = (int32_t)min(cnt[2].size, (unsigned long long)qcap);
  }
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  unsigned long long my_edges = 0;
  for (int64_t base = (int64_t)blockIdx.x * 256; base < qsize; base += (int64_t)gridDim.x * 256) {
    int64_t i = base + tid;
    int v = -1, o = 0, deg = 0;
    if (i < qsize) {
      v = queue[i];
      if (v >= 0 && v < g.n) {
        o = __ldg(g.out.off + v);
        deg = __ldg(g.out.off + v + 1) - o;
      } else {
        atomicOr(&cnt->err, (unsigned)kErrRange);
      }
      // hub rows go to k_sparse_push_hubs, which spreads them over the grid
      if (deg >= g.grid_expand) {
        unsigned long long slot = atomicAdd(&hub_cnt->size, 1ull);
        if (slot < (unsigned long long)kMaxHubs) {
          hubs[slot] = v;
          deg = 0;
        }
      }
    }
    // CTA-wide expansion of long rows.
    for (;;) {
      if (tid == 0) s_owner = -1;
      __syncthreads();
      if (deg >= g.cta_expand) s_owner = tid;
      __syncthreads();
      int owner = s_owner;
      if (owner < 0) break;
      if (tid == owner) { s_cv = v; s_co = o; s_cd = deg; deg = 0; }
      __syncthreads();
      int cv = s_cv, co = s_co, cd = s_cd;
      for (int r = 0; r < cd; r += 256) {
        int k = r + tid, d = -1;
        bool act = k < cd && push_edge(g, f, w, cv, (int64_t)co + k, next_bits, d);
        if (act) my_edges += __ldg(g.out.off + d + 1) - __ldg(g.out.off + d);
        emit_queue(act, d, next_queue, qcap, cnt);
      }
      __syncthreads();
    }
    // Warp-wide expansion of medium rows.
    for (;;) {
      unsigned bal = __ballot_sync(0xffffffffu, deg >= 32);
      if (!bal) break;
      int leader = __ffs(bal) - 1;
      int wv = __shfl_sync(0xffffffffu, v, leader);
      int wo = __shfl_sync(0xffffffffu, o, leader);
      int wd = __shfl_sync(0xffffffffu, deg, leader);
      if (lane == leader) deg = 0;
      for (int r = 0; r < wd; r += 32) {
        int k = r + lane, d = -1;
        bool act = k < wd && push_edge(g, f, w, wv, (int64_t)wo + k, next_bits, d);
        if (act) my_edges += __ldg(g.out.off + d + 1) - __ldg(g.out.off + d);
        emit_queue(act, d, next_queue, qcap, cnt);
      }
    }
    // Scan-based gather of the short rows.
    int wtot;
    int pos = warp_excl_scan(deg, &wtot);
    if (lane == 0) s_warp_tot[wid] = wtot;
    __syncthreads();
    int woff = 0, total = 0;
    for (int k = 0; k < 8; ++k) {
      if (k < wid) woff += s_warp_tot[k];
      total += s_warp_tot[k];
    }
    s_pos[tid] = pos + woff;
    s_v[tid] = v;
    s_o[tid] = o;
    __syncthreads();
    for (int r = 0; r < total; r += 256) {
      int k = r + tid, d = -1;
      bool act = false;
      int lo = 0;
      if (k < total) {
        int hi = 255;  // last j with s_pos[j] <= k
        while (lo < hi) {
          int mid = (lo + hi + 1) >> 1;
          if (s_pos[mid] <= k) lo = mid; else hi = mid - 1;
        }
        if (!MinPush<F>::value || !g.push_agg)
          act = push_edge(g, f, w, s_v[lo], (int64_t)s_o[lo] + (k - s_pos[lo]), next_bits, d);
      }
      // the short rows of different sources share targets (hubs): aggregate
      if constexpr (MinPush<F>::value) {
        if (g.push_agg)  // a kernel argument: the same branch for the whole warp
          act = push_edge_min(g, f, w, k < total, k < total ? s_v[lo] : 0,
                              k < total ? (int64_t)s_o[lo] + (k - s_pos[lo]) : 0, next_bits, d);
      }
      if (act) my_edges += __ldg(g.out.off + d + 1) - __ldg(g.out.off + d);
      emit_queue(act, d, next_queue, qcap, cnt);
    }
    __syncthreads();
  }
  my_edges = warp_sum(my_edges);
  if (lane == 0 && my_edges) atomicAdd(&cnt->edges, my_edges);
}

// Hub rows of a sparse round: every CTA builds the prefix sum of the hubs'
// degrees in shared memory, then the grid shares their flattened edges, each
// thread kLaneEdges consecutive ones at a time.
template <class F, class W>
__global__ void __launch_bounds__(256) k_sparse_push_hubs(GraphView g, F f, const W *__restrict__ w,
                                                          const int32_t *__restrict__ hubs,
                                                          const Counters *hub_cnt,
                                                          int32_t *__restrict__ next_queue,
                                                          uint32_t *__restrict__ next_bits,
                                                          int32_t qcap, Counters *cnt,
                                                          const RoundGate *gate = nullptr) {
  constexpr int K = 8;
  __shared__ int s_pos[kMaxHubs + 1];
  __shared__ int s_warp[8];
  if (gate && (!gate->active || gate->dense)) return;  // not a sparse round
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int nh = (int)min(hub_cnt->size, (unsigned long long)kMaxHubs);
  if (nh == 0) return;
  // exclusive scan of the hub degrees: thread t owns a contiguous slice
  const int per = (nh + 255) / 256;
  const int h0 = min(tid * per, nh), h1 = min(h0 + per, nh);
  int local = 0;
  for (int h = h0; h < h1; ++h) {
    const int v = hubs[h];
    local += __ldg(g.out.off + v + 1) - __ldg(g.out.off + v);
  }
  int wtot;
  int pre = warp_excl_scan(local, &wtot);
  if (lane == 0) s_warp[wid] = wtot;
  __syncthreads();
  int base = 0, total = 0;
  for (int k = 0; k < 8; ++k) {
    if (k < wid) base += s_warp[k];
    total += s_warp[k];
  }
  int run = base + pre;
  for (int h = h0; h < h1; ++h) {
    s_pos[h] = run;
    const int v = hubs[h];
    run += __ldg(g.out.off + v + 1) - __ldg(g.out.off + v);
  }
  if (tid == 0) s_pos[nh] = total;
  __syncthreads();
  unsigned long long my_edges = 0;
  const int64_t stride = (int64_t)gridDim.x * 256 * K;
  for (int64_t q0 = ((int64_t)blockIdx.x * 256 + tid) * K; q0 - tid * K < total; q0 += stride) {
    int h = 0;
    if (q0 < total) {  // last hub whose flat start is <= q0
      int lo = 0, hi = nh - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (s_pos[mid] <= q0) lo = mid; else hi = mid - 1;
      }
      h = lo;
    }
    int v = q0 < total ? hubs[h] : 0;
    int64_t o = q0 < total ? (int64_t)__ldg(g.out.off + v) : 0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int64_t q = q0 + k;
      int d = -1;
      bool act = false;
      if (q < total) {
        while (q >= s_pos[h + 1]) {
          ++h;
          v = hubs[h];
          o = __ldg(g.out.off + v);
        }
        act = push_edge(g, f, w, v, o + (q - s_pos[h]), next_bits, d);
      }
      if (act) my_edges += __ldg(g.out.off + d + 1) - __ldg(g.out.off + d);
      emit_queue(act, d, next_queue, qcap, cnt);
    }
  }
  my_edges = warp_sum(my_edges);
  if (lane == 0 && my_edges) atomicAdd(&cnt->edges, my_edges);
}

// ---------------------------------------------------------------------------
// Dense pull with early exit (edgeMapDenseDynamic polymer.h:1170-1261,
// edgeMapDenseNoRep numa-BFS.C:113-159): for every vertex v with cond(v),
// scan in-neighbours s in the frontier, call updateAtomic(s, v, w) and stop
// once cond(v) is false.  One thread per vertex scans up to kPullScan edges;
// rows still open after that are deferred to k_dense_pull_defer (one warp
// per row).  A warp owns 32 consecutive vertices = one bitmap word.
// ---------------------------------------------------------------------------
template <class F, class W>
__global__ void __launch_bounds__(256) k_dense_pull(GraphView g, const uint32_t *__restrict__ cur,
                                                    F f, const W *__restrict__ w,
                                                    uint32_t *__restrict__ next,
                                                    int32_t *__restrict__ defer, Counters *cnt,
                                                    Counters *dcnt, const RoundGate *gate = nullptr) {
  if (gate && (!gate->active || !gate->dense)) return;  // not a dense round
  const int lane = lane_id();
  unsigned long long my_edges = 0, my_size = 0;
  const int64_t nthreads = (int64_t)gridDim.x * blockDim.x;
  const int64_t ntot = ((int64_t)g.n + 31) & ~31ll;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntot; t += nthreads) {
    int v = (int)t;
    bool act = false, deferred = false;
    if (v < g.n && f.cond(v)) {
      int o0 = __ldg(g.in.off + v), o1 = __ldg(g.in.off + v + 1);
      int lim = min(o1, o0 + kPullScan);
      int e = o0;
      for (; e < lim; ++e) {
        int s = checked_id(g, __ldg(g.in.idx + e));
        if (test_bit(cur, s) && update_atomic(f, s, v, load_w(w, e))) act = true;
        if (!f.cond(v)) break;
      }
      deferred = (e == lim) && lim < o1 && f.cond(v);
    }
    unsigned word = __ballot_sync(0xffffffffu, act);
    if (lane == 0) next[v >> 5] = word;
    if (act) {
      my_size++;
      my_edges += __ldg(g.out.off + v + 1) - __ldg(g.out.off + v);
    }
    unsigned db = __ballot_sync(0xffffffffu, deferred);
    if (db) {
      int leader = __ffs(db) - 1;
      unsigned long long base = 0;
      if (lane == leader) base = atomicAdd(&dcnt->size, (unsigned long long)__popc(db));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (deferred) defer[base + __popc(db & ((1u << lane) - 1u))] = v;
    }
  }
  my_size = warp_sum(my_size);
  my_edges = warp_sum(my_edges);
  if (lane == 0 && my_size) {
    atomicAdd(&cnt->size, my_size);
    atomicAdd(&cnt->edges, my_edges);
  }
}

template <class F, class W>
__global__ void __launch_bounds__(256) k_dense_pull_defer(GraphView g,
                                                          const uint32_t *__restrict__ cur, F f,
                                                          const W *__restrict__ w,
                                                          uint32_t *__restrict__ next,
                                                          const int32_t *__restrict__ defer,
                                                          Counters *cnt, const Counters *dcnt,
                                                          const RoundGate *gate = nullptr) {
  if (gate && (!gate->active || !gate->dense)) return;  // not a dense round
  const int lane = lane_id();
  const int64_t nd = (int64_t)dcnt->size;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t k = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); k < nd; k += nwarps) {
    int v = defer[k];
    int o0 = __ldg(g.in.off + v) + kPullScan, o1 = __ldg(g.in.off + v + 1);
    bool act = false, open = true;
    for (int base = o0; base < o1 && open; base += 32) {
      int e = base + lane;
      int s = e < o1 ? checked_id(g, __ldg(g.in.idx + e)) : 0;
      unsigned bal = __ballot_sync(0xffffffffu, e < o1 && test_bit(cur, s));
      while (bal && open) {
        int l = __ffs(bal) - 1;
        bal &= bal - 1;
        int ss = __shfl_sync(0xffffffffu, s, l);
        int ok = 0, c = 1;
        if (lane == 0) {
          ok = update_atomic(f, ss, v, load_w(w, (int64_t)base + l));
          c = f.cond(v);
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        c = __shfl_sync(0xffffffffu, c, 0);
        act |= ok != 0;
        open = c != 0;
      }
    }
    // The first kernel may already have set v's bit (and counted it).
    if (act && lane == 0 && set_bit_new(next, v)) {
      atomicAdd(&cnt->size, 1ull);
      atomicAdd(&cnt->edges, (unsigned long long)(__ldg(g.out.off + v + 1) - __ldg(g.out.off + v)));
    }
  }
}

// ---------------------------------------------------------------------------
// Dense pull-reduce (edgeMapDenseReduce, polymer.h:1097-1168).  A warp takes
// one group: about kGroupWork units of rows and edges on the merge path
// (32-aligned row ranges).  It walks them 32 rows at a time and lays their edges
// out flat (consecutive rows are consecutive in the CSC).  Each lane takes
// kLaneEdges consecutive flat edges per window: it issues all their id loads
// and f.edge() gathers before folding any, which keeps kLaneEdges loads in
// flight per lane, folds them locally per row, stores rows that start and
// end inside it, and hands its first / last partial row to a segmented warp
// reduction keyed by row.  Row sums collect in shared memory; the row's lane
// then runs f.commit() (the fused vertexMap).  Rows with more than g.heavy_deg
// edges are reduced first by k_heavy_reduce (one CTA per kChunkEdges chunk)
// into partials[], which the owning lane folds in chunk order.  The order of
// every reduction is fixed, so results are deterministic.
// ---------------------------------------------------------------------------
// Edges per lane per window and the minimum resident CTAs per SM of the
// pull-reduce (a register cap of 40 at 256 threads): measured on R-MAT scale
// 24, these beat 8 edges and the uncapped 48-64 registers by 12 % (PageRank),
// 27 % (SpMV) and 18 % (BP) per pass -- more resident warps hide the gathers.
#ifndef PM_LANE_EDGES
#define PM_LANE_EDGES 6
#endif
#ifndef PM_PULL_BLOCK
#define PM_PULL_BLOCK 256
#endif
#ifndef PM_PULL_MINB
#define PM_PULL_MINB 6
#endif
constexpr int kLaneEdges = PM_LANE_EDGES;
constexpr int kPullBlock = PM_PULL_BLOCK;
// The pull with a hub cache runs two CTAs of kHubBlock threads per SM (the
// 48 warps of the plain pull at its occupancy limit, 40 registers each), so
// each SM holds two copies of the cached values, kHubMax of them at most
// (64 KB each in FP32).
constexpr int kHubBlock = 768;
constexpr int kHubMax = 16384;

#ifndef PM_STAGE_IDS
#define PM_STAGE_IDS 512
#endif
// Staged pull (k_pull_reduce with STAGE): the CSC ids of a warp's batch of 32
// rows, when they are at most kStageIds, are copied into the warp's slice of
// shared memory by one bulk copy (cp.async.bulk global -> shared, completed
// on an mbarrier) and read from there.  The id loads then cost no L1 tag
// look-ups, which the gathers of the same SM are bound by, and a window
// waits for one copy per batch instead of its own id loads.  The copy's
// source starts at the 16-byte boundary below the batch's first id and its
// size is rounded up to 16 bytes (never past the last aligned id of the
// array: a batch ending beyond it reads from global memory).
constexpr int kStageIds = PM_STAGE_IDS;
constexpr int kStageWaitTries = 1 << 20;  // polls of a copy's mbarrier before giving up
// dynamic shared memory of a staged kPullBlock CTA: the warps' mbarriers in
// the first 128 bytes, then each warp's kStageIds ids
constexpr size_t kStageSmem = 128 + (size_t)(kPullBlock / 32) * kStageIds * 4;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bytes: a multiple of 16; src and dst 16-byte aligned; src in this GPU's memory
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// orders this thread's earlier generic accesses to shared memory before
// later asynchronous (bulk copy) writes to it
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Sources whose values a pull keeps in shared memory: idx is the CSC source
// array with the cached sources' slots stored as ~slot, vals their values
// for this pass.
template <class V>
struct HubCache {
  const int32_t *idx = nullptr;
  const V *vals = nullptr;
  int count = 0;
};

// Functors that can take a cached value declare kHubs and edge_value(v, row,
// w) = edge(s, row, w) for v the value edge() would load for s.
template <class F, class = void>
struct HubTrait {
  static constexpr bool value = false;
};
template <class F>
struct HubTrait<F, std::void_t<decltype(F::kHubs)>> {
  static constexpr bool value = F::kHubs;
};

// Edges per lane of a functor's light pull: F::kLaneEdges when it declares
// one, else kLaneEdges (the best values differ by functor: measured per pass).
template <class F, class = void>
struct LaneEdgesTrait {
  static constexpr int value = kLaneEdges;
};
template <class F>
struct LaneEdgesTrait<F, std::void_t<decltype(F::kLaneEdges)>> {
  static constexpr int value = F::kLaneEdges;
};

template <bool HUBS, class F, class WV>
__device__ __forceinline__ typename F::Acc pull_edge(const F &f, int s, int row, WV wv,
                                                     const typename F::Acc *s_hub) {
  if constexpr (HUBS) {
    if (s < 0) return f.edge_value(s_hub[~s], row, wv);
  }
  return f.edge(s, row, wv);
}
template <class F, class W>
__global__ void __launch_bounds__(kChunkThreads) k_heavy_reduce(GraphView g, F f,
                                                                const W *__restrict__ w,
                                                                typename F::Acc *partials) {
  using Acc = typename F::Acc;
  __shared__ Acc s_red[kChunkThreads / 32];
  const int c = blockIdx.x;
  if (c >= g.in.nchunks) return;
  const int r = __ldg(g.in.hrow + c);
  const int k = c - __ldg(g.in.hfirst + r);
  const int64_t e0 = (int64_t)__ldg(g.in.off + r) + (int64_t)k * kChunkEdges;
  const int64_t e1 = min(e0 + kChunkEdges, (int64_t)__ldg(g.in.off + r + 1));
  Acc acc = f.identity();
  if (f.cond(r)) {
    static_assert(kChunkEdges % kChunkThreads == 0, "chunk must be a multiple of the CTA");
    constexpr int U = kChunkEdges / kChunkThreads;
    int src[U];
    typename EdgeT<W>::type wv[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t e = e0 + threadIdx.x + (int64_t)u * kChunkThreads;
      src[u] = e < e1 ? checked_id(g, load_src(g.in.idx, w, e, wv[u])) : 0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t e = e0 + threadIdx.x + (int64_t)u * kChunkThreads;
      if (e < e1) acc = f.combine(acc, f.edge(src[u], r, edge_w(w, e, wv[u])));
    }
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) acc = f.combine(acc, shfl_down(acc, d));
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    Acc t = s_red[0];
    for (int i = 1; i < kChunkThreads / 32; ++i) t = f.combine(t, s_red[i]);
    partials[c] = t;
  }
}

// One heavy chunk summed by one warp (the fused pull below): lane-strided
// loads, 4 per lane in flight, a warp reduction, the partial published with
// a fence and counted in done[hfirst[r]] for the row's committing lane.
template <class F, class W>
__device__ __forceinline__ void warp_heavy_chunk(const GraphView &g, const F &f, const W *w, int c,
                                                 typename F::Acc *partials, int32_t *done) {
  using Acc = typename F::Acc;
  const int lane = lane_id();
  const int r = __ldg(g.in.hrow + c);
  const int first = __ldg(g.in.hfirst + r);
  const int64_t e0 = (int64_t)__ldg(g.in.off + r) + (int64_t)(c - first) * kChunkEdges;
  const int64_t e1 = min(e0 + kChunkEdges, (int64_t)__ldg(g.in.off + r + 1));
  Acc acc = f.identity();
  if (f.cond(r)) {
    constexpr int U = 4;  // loads in flight per lane (the kernel's register cap)
    for (int64_t base = e0; base < e1; base += 32 * U) {
      int src[U];
      typename EdgeT<W>::type wv[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int64_t e = base + 32 * u + lane;
        src[u] = e < e1 ? checked_id(g, load_src(g.in.idx, w, e, wv[u])) : 0;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int64_t e = base + 32 * u + lane;
        if (e < e1) acc = f.combine(acc, f.edge(src[u], r, edge_w(w, e, wv[u])));
      }
    }
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) acc = f.combine(acc, shfl_down(acc, d));
  if (lane == 0) {
    partials[c] = acc;
    __threadfence();
    atomicAdd(done + first, 1);
  }
}

__device__ __forceinline__ int ld_acquire_gpu(const int32_t *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
constexpr int kHeavyWaitSpins = 1 << 22;  // x ~256 ns: gives up after about a second

// Waits until *p >= target (acquire), at most max_spins polls 256 ns apart.
// On giving up it sets kErrTimeout in *err and returns false: the kernel
// goes on and the host turns the error word into PM_ERR_TIMEOUT.
__device__ __forceinline__ bool wait_at_least(const int32_t *p, int32_t target, int max_spins, unsigned *err) {
  int spins = 0;
  while (ld_acquire_gpu(p) < target) {
    if (++spins > max_spins) {
      atomicOr(err, (unsigned)kErrTimeout);
      return false;
    }
    __nanosleep(256);
  }
  return true;
}

// MODE 0: the partials of the heavy rows were summed by k_heavy_reduce
// before this launch.  MODE 1 (fused): the first g.in.nchunks tickets are
// heavy chunks, summed here by warp_heavy_chunk, and a heavy row's lane waits
// (bounded) for its chunks before it commits: every chunk ticket precedes
// every group ticket, so its warp is already running.  MODE 2 (overlapped):
// k_heavy_reduce runs at the same time on a second stream and this kernel
// leaves the heavy rows alone; k_heavy_commit commits them afterwards.
//
// HUBS (MODE 0 only): the light rows' sources come from hubs.idx, where the
// cached sources appear as ~slot and their values are read from shared
// memory (loaded from hubs.vals once per CTA); two kHubBlock-thread CTAs per
// SM.  The values are the ones edge() would load, so results are unchanged.
template <class F, class W, int MODE = 0, bool HUBS = false, bool STAGE = false>
__global__ void __launch_bounds__(HUBS ? kHubBlock : kPullBlock, HUBS ? 2 : PM_PULL_MINB)
    k_pull_reduce(GraphView g, F f, const W *__restrict__ w, typename F::Acc *partials, int32_t *hdone,
                  uint32_t *__restrict__ next, Counters *cnt, HubCache<typename F::Acc> hubs = {}) {
  static_assert(!STAGE || (MODE == 0 && !HUBS && std::is_same<W, int>::value),
                "staged ids: heavy mode 0, ids without paired weights, no hub cache");
  using Acc = typename F::Acc;
  constexpr int K = LaneEdgesTrait<F>::value, WIN = 32 * K, NW = (HUBS ? kHubBlock : kPullBlock) / 32;
  __shared__ Acc s_acc[NW][32];
  __shared__ int s_pos[NW][33];
  __shared__ int s_off[NW][32];
  extern __shared__ __align__(16) unsigned char s_dyn[];
  Acc *s_hub = reinterpret_cast<Acc *>(s_dyn);
  const int32_t *lidx = g.in.idx;  // light rows' sources
  if constexpr (HUBS) {
    for (int i = threadIdx.x; i < hubs.count; i += kHubBlock) s_hub[i] = hubs.vals[i];
    __syncthreads();
    lidx = hubs.idx;
  }
  const int lane = lane_id(), wid = threadIdx.x >> 5;
  Acc *acc_s = s_acc[wid];
  int *pos_s = s_pos[wid];
  int *off_s = s_off[wid];
  // STAGE: [NW mbarriers][pad to 128 B][NW x kStageIds ids]
  uint64_t *st_bar = reinterpret_cast<uint64_t *>(s_dyn) + wid;
  int32_t *st_ids = reinterpret_cast<int32_t *>(s_dyn + 128) + (size_t)wid * kStageIds;
  // bit 0: the mbarrier's phase; bit 1: a copy did not complete in time, the
  // warp reads its ids from global memory from then on
  uint32_t st_state = 0;
  if constexpr (STAGE) {
    if (lane == 0) {
      mbar_init(st_bar, 1);
      mbar_init_fence();
    }
    __syncwarp();
  }
  unsigned long long my_size = 0, my_edges = 0;
  double2 my_aux = make_double2(0.0, 0.0);
  // persistent warps: each takes the next group from a ticket counter
  for (;;) {
  int grp = 0;
  if (lane == 0) grp = (int)atomicAdd(&cnt->aux, 1ull);
  grp = __shfl_sync(0xffffffffu, grp, 0);
  if constexpr (MODE == 1) {
    if (grp < g.in.nchunks) {
      warp_heavy_chunk(g, f, w, grp, partials, hdone);
      continue;
    }
    grp -= g.in.nchunks;
  }
  if (grp >= g.in.ngroups) break;
  const int r_begin = __ldg(g.in.gstart + grp), r_end = __ldg(g.in.gstart + grp + 1);
  for (int rb = r_begin; rb < r_end; rb += 32) {
    const int r = rb + lane;
    const bool valid = r < r_end;
    int o0 = 0, deg = 0;
    bool live = false;
    if (valid) {
      o0 = __ldg(g.in.off + r);
      deg = __ldg(g.in.off + r + 1) - o0;
      live = f.cond(r);
    }
    const bool heavy = deg > g.heavy_deg;
    const int ldeg = (live && !heavy) ? deg : 0;
    // STAGE: the batch's CSC ids into this warp's shared slice
    int st_base = 0;
    bool staged = false;
    if constexpr (STAGE) {
      // ids are int here (m < 2^31); the copy is [a, b), 16-byte aligned,
      // and ends at or before the last aligned id of the array
      const int last = min(31, r_end - rb - 1);
      const int first_e = __shfl_sync(0xffffffffu, o0, 0);
      const int end_e = __shfl_sync(0xffffffffu, o0 + deg, last);
      const int a = first_e & ~3, b = (int)(((int64_t)end_e + 3) & ~3ll);
      staged = !(st_state & 2u) && end_e > first_e && b - a <= kStageIds && (int64_t)b <= (g.m & ~3ll);
      if (staged) {
        // every lane is done with the previous batch's ids (the __syncwarp
        // that ends a batch); the copy runs while the batch is laid out
        if (lane == 0) {
          fence_proxy_async_smem();
          mbar_expect_tx(st_bar, (uint32_t)((b - a) * 4));
          bulk_copy_g2s(st_ids, g.in.idx + a, (uint32_t)((b - a) * 4), st_bar);
        }
        st_base = a;
      }
    }
    int total;
    const int pos = warp_excl_scan(ldeg, &total);
    pos_s[lane] = pos;
    if (lane == 31) pos_s[32] = total;
    off_s[lane] = o0;
    acc_s[lane] = f.identity();
    if constexpr (STAGE) {
      if (staged) {
        // lane 0 waits for the copy (bounded), the warp learns the outcome
        int done = 0;
        if (lane == 0) {
          for (int i = 0; i < kStageWaitTries && !done; ++i) done = mbar_try_wait(st_bar, st_state & 1u);
          if (!done) {
            // not complete in time: report it, wait once more (bounded) for
            // the copy in flight, and read this and later batches from
            // global memory
            atomicOr(&cnt->err, (unsigned)kErrTimeout);
            for (int i = 0; i < kStageWaitTries && !done; ++i) done = mbar_try_wait(st_bar, st_state & 1u);
            done = 0;
          }
        }
        if (!__shfl_sync(0xffffffffu, done, 0)) {
          staged = false;
          st_state |= 2u;
        }
        st_state ^= 1u;
      }
    }
    __syncwarp();
    for (int c = 0; c < total; c += WIN) {
      const int q0 = c + lane * K;
      const bool active = q0 < total;
      // row (lane index j) and CSC slot of each of this lane's K flat edges
      int j = 0;
      if (active) {
#pragma unroll
        for (int step = 16; step > 0; step >>= 1)
          if (pos_s[j + step] <= q0) j += step;
      }
      int rows[K], es[K], src[K];
      int nxt = pos_s[j + 1];
      // all K edges of this lane lie in row j (nxt <= total)
      const bool single = active && q0 + K <= nxt;
      // ... and every active lane lies in lane 0's row: one row spans the window
      const int j0 = __shfl_sync(0xffffffffu, j, 0);
      const bool uniform = __all_sync(0xffffffffu, !active || (single && j == j0));
      if (uniform) {
        // The window's edges are one contiguous run of row j0: read them
        // lane-strided (one 128-byte line per load) and reduce the warp.
        const int e0 = off_s[j0] + (c - pos_s[j0]);
        const int cnt = min(WIN, total - c);
        Acc s = f.identity();
        typename EdgeT<W>::type wv[K];
#pragma unroll
        for (int k = 0; k < K; ++k)
          src[k] = (32 * k + lane < cnt)
                       ? checked_src<HUBS>(g, hubs.count,
                                           (STAGE && staged) ? st_ids[e0 + 32 * k + lane - st_base]
                                                             : load_src(lidx, w, (int64_t)e0 + 32 * k + lane, wv[k]))
                       : 0;
#pragma unroll
        for (int k = 0; k < K; ++k)
          if (32 * k + lane < cnt)
            s = f.combine(s, pull_edge<HUBS>(f, src[k], rb + j0, edge_w(w, (int64_t)e0 + 32 * k + lane, wv[k]),
                                             s_hub));
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) s = f.combine(s, shfl_down(s, d));
        if (lane == 0) acc_s[j0] = f.combine(acc_s[j0], s);
        __syncwarp();
        continue;
      }
      if (single) {
        const int e0 = off_s[j] + (q0 - pos_s[j]);
#pragma unroll
        for (int k = 0; k < K; ++k) {
          rows[k] = j;
          es[k] = e0 + k;
        }
      } else {
#pragma unroll
        for (int k = 0; k < K; ++k) {
          const int q = q0 + k;
          if (q < total)
            while (q >= nxt) nxt = pos_s[++j + 1];
          rows[k] = j;
          es[k] = off_s[j] + (q - pos_s[j]);
        }
      }
      typename EdgeT<W>::type wv[K];
#pragma unroll
      for (int k = 0; k < K; ++k)
        src[k] = (q0 + k < total)
                     ? checked_src<HUBS>(g, hubs.count,
                                         (STAGE && staged) ? st_ids[es[k] - st_base] : load_src(lidx, w, es[k], wv[k]))
                     : 0;
      Acc vals[K];
#pragma unroll
      for (int k = 0; k < K; ++k)
        vals[k] = (q0 + k < total) ? pull_edge<HUBS>(f, src[k], rb + rows[k], edge_w(w, es[k], wv[k]), s_hub)
                                   : f.identity();
      // Local fold: the first segment is the head, rows that start and end
      // inside the lane are stored directly, the last segment is the tail.
      Acc head = f.identity(), run = f.identity();
      int jr = rows[0];
      bool split = false;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if (q0 + k < total) {
          if (rows[k] != jr) {
            if (!split) {
              head = run;
              split = true;
            } else {
              acc_s[jr] = f.combine(acc_s[jr], run);
            }
            run = f.identity();
            jr = rows[k];
          }
          run = f.combine(run, vals[k]);
        }
      }
      Acc tail = f.identity();
      if (split) tail = run; else head = run;
      const int jf = rows[0], jl = jr;
      // the previous lane's tail continues into this lane's head
      const int p_jl = __shfl_up_sync(0xffffffffu, jl, 1);
      const int p_split = __shfl_up_sync(0xffffffffu, (int)(split && active), 1);
      const Acc p_tail = shfl_up(tail, 1);
      if (active && lane > 0 && p_split && p_jl == jf) head = f.combine(p_tail, head);
      // segmented suffix reduction of the heads, keyed by row
      const int key = active ? jf : 64 + lane;
      Acc v = head;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        Acc t = shfl_down(v, d);
        int tk = __shfl_down_sync(0xffffffffu, key, d);
        if (lane + d < 32 && tk == key) v = f.combine(v, t);
      }
      const int prev_key = __shfl_up_sync(0xffffffffu, key, 1);
      const int next_key = __shfl_down_sync(0xffffffffu, key, 1);
      if (active && (lane == 0 || prev_key != key)) acc_s[jf] = f.combine(acc_s[jf], v);
      // a tail that the next lane does not continue is complete here
      if (active && split && (lane == 31 || next_key != jl)) acc_s[jl] = f.combine(acc_s[jl], tail);
      __syncwarp();
    }
    Acc acc = acc_s[lane];
    bool deferred = false;  // MODE 2: k_heavy_commit finishes this row
    if constexpr (MODE == 2) deferred = live && heavy;
    if (live && heavy && !deferred) {
      const int first = __ldg(g.in.hfirst + r);
      const int nch = (deg + kChunkEdges - 1) / kChunkEdges;
      if constexpr (MODE == 1) {
        wait_at_least(hdone + first, nch, kHeavyWaitSpins, &cnt->err);
        for (int k = 0; k < nch; ++k) acc = f.combine(acc, __ldcg(partials + first + k));
      } else {
        for (int k = 0; k < nch; ++k) acc = f.combine(acc, partials[first + k]);
      }
    }
    const bool act = live && !deferred && f.commit(r, acc, my_aux);
    const unsigned word = __ballot_sync(0xffffffffu, act);
    if (next && lane == 0) next[rb >> 5] = word;
    if (act) {
      my_size++;
      my_edges += __ldg(g.out.off + r + 1) - __ldg(g.out.off + r);
    }
    __syncwarp();
  }
  }  // group loop
  my_size = warp_sum(my_size);
  my_edges = warp_sum(my_edges);
  my_aux.x = warp_sum(my_aux.x);
  my_aux.y = warp_sum(my_aux.y);
  if (lane == 0) {
    if (my_size) {
      atomicAdd(&cnt->size, my_size);
      atomicAdd(&cnt->edges, my_edges);
    }
    if (my_aux.x != 0.0) atomicAdd(&cnt->daux, my_aux.x);
    if (my_aux.y != 0.0) atomicAdd(&cnt->daux2, my_aux.y);
  }
}

// The heavy rows of an overlapped pull (MODE 2): one thread per heavy row
// (the first chunk of each row) folds the row's partials in chunk order,
// commits, and ORs its bit into the next frontier.
template <class F>
__global__ void __launch_bounds__(256) k_heavy_commit(GraphView g, F f, const typename F::Acc *partials,
                                                     uint32_t *next, Counters *cnt) {
  using Acc = typename F::Acc;
  unsigned long long my_size = 0, my_edges = 0;
  double2 my_aux = make_double2(0.0, 0.0);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < g.in.nchunks; c += stride) {
    const int r = __ldg(g.in.hrow + c);
    const int first = __ldg(g.in.hfirst + r);
    if (c != first || !f.cond(r)) continue;
    const int deg = __ldg(g.in.off + r + 1) - __ldg(g.in.off + r);
    const int nch = (deg + kChunkEdges - 1) / kChunkEdges;
    Acc acc = f.identity();
    for (int k = 0; k < nch; ++k) acc = f.combine(acc, partials[first + k]);
    if (f.commit(r, acc, my_aux)) {
      if (next) atomicOr(next + (r >> 5), 1u << (r & 31));
      my_size++;
      my_edges += __ldg(g.out.off + r + 1) - __ldg(g.out.off + r);
    }
  }
  my_size = warp_sum(my_size);
  my_edges = warp_sum(my_edges);
  my_aux.x = warp_sum(my_aux.x);
  my_aux.y = warp_sum(my_aux.y);
  if (lane_id() == 0) {
    if (my_size) {
      atomicAdd(&cnt->size, my_size);
      atomicAdd(&cnt->edges, my_edges);
    }
    if (my_aux.x != 0.0) atomicAdd(&cnt->daux, my_aux.x);
    if (my_aux.y != 0.0) atomicAdd(&cnt->daux2, my_aux.y);
  }
}

// ---------------------------------------------------------------------------
// Functors in the reference's own reducing-pull shape.  Polymer's
// applications give edgeMapDenseReduce (polymer.h:1097-1168; weighted
// polymer-wgh.h:951-1010) three members over a 16-byte scratch per vertex:
//   initFunc(void *data, int d)
//   reduceFunc(void *data, int s[, W w]) -> true when d is activated
//   combineFunc(void *data, int d)
// (numa-Components.C:77-99, numa-PageRank.C:98-119).  edgeMapReduce takes
// such a functor as it is (the members __device__): its dense rounds run
// k_pull_seq, which folds each vertex's frontier in-neighbours in CSC order
// on one thread, exactly the reference's loop, because reduceFunc is a
// sequential fold with no combine of two partial states.  Its sparse rounds
// are the usual push with updateAtomic(s, d[, w]).  The reference's atomics
// (utils.h:244-310) are below with the same names and results, so such a
// functor's bodies compile unchanged apart from the __device__ qualifiers.
// ---------------------------------------------------------------------------
template <class F, class = void>
struct RefReduceShape : std::false_type {};
template <class F>
struct RefReduceShape<F, std::void_t<decltype(std::declval<F &>().initFunc((void *)nullptr, 0)),
                                     decltype(std::declval<F &>().combineFunc((void *)nullptr, 0))>>
    : std::true_type {};

template <class F, class Wv, class = void>
struct ReduceTakesWeight : std::false_type {};
template <class F, class Wv>
struct ReduceTakesWeight<F, Wv,
                         std::void_t<decltype(std::declval<F &>().reduceFunc((void *)nullptr, 0, std::declval<Wv>()))>>
    : std::true_type {};
template <class F, class Wv>
__device__ __forceinline__ bool reduce_func(F &f, void *data, int s, Wv w) {
  if constexpr (ReduceTakesWeight<F, Wv>::value)
    return f.reduceFunc(data, s, w);
  else
    return f.reduceFunc(data, s);
}

// CAS / writeMin / writeAdd / fetchAndAdd of utils.h:244-310 on the GPU.
template <class ET>
__device__ __forceinline__ bool CAS(ET *ptr, ET oldv, ET newv) {
  static_assert(sizeof(ET) == 4 || sizeof(ET) == 8, "CAS on 4- or 8-byte values");
  if constexpr (sizeof(ET) == 8) {
    unsigned long long o, nv;
    memcpy(&o, &oldv, 8);
    memcpy(&nv, &newv, 8);
    return atomicCAS(reinterpret_cast<unsigned long long *>(ptr), o, nv) == o;
  } else {
    unsigned o, nv;
    memcpy(&o, &oldv, 4);
    memcpy(&nv, &newv, 4);
    return atomicCAS(reinterpret_cast<unsigned *>(ptr), o, nv) == o;
  }
}
// true when this call lowered *a to b
template <class ET>
__device__ __forceinline__ bool writeMin(ET *a, ET b) {
  if constexpr (std::is_same<ET, int>::value || std::is_same<ET, unsigned>::value ||
                std::is_same<ET, long long>::value || std::is_same<ET, unsigned long long>::value) {
    return b < atomicMin(a, b);
  } else {
    ET c = *((volatile ET *)a);
    while (c > b) {
      if (CAS(a, c, b)) return true;
      c = *((volatile ET *)a);
    }
    return false;
  }
}
template <class ET>
__device__ __forceinline__ void writeAdd(ET *a, ET b) {
  atomicAdd(a, b);
}
template <class ET>
__device__ __forceinline__ ET fetchAndAdd(ET *a, ET b) {
  return atomicAdd(a, b);
}

template <class F, class W>
__global__ void __launch_bounds__(256) k_pull_seq(GraphView g, const uint32_t *__restrict__ cur, F f,
                                                  const W *__restrict__ w, uint32_t *__restrict__ next,
                                                  Counters *cnt) {
  const int lane = lane_id();
  unsigned long long my_size = 0, my_edges = 0;
  const int64_t nthreads = (int64_t)gridDim.x * blockDim.x;
  const int64_t ntot = ((int64_t)g.n + 31) & ~31ll;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntot; t += nthreads) {
    const int v = (int)t;
    bool act = false;
    if (v < g.n && f.cond(v)) {
      double data[2];  // the reference's per-vertex scratch (polymer.h:1140)
      f.initFunc((void *)data, v);
      const int o0 = __ldg(g.in.off + v), o1 = __ldg(g.in.off + v + 1);
      for (int e = o0; e < o1; ++e) {
        const int s = checked_id(g, __ldg(g.in.idx + e));
        if (test_bit(cur, s) && reduce_func(f, (void *)data, s, load_w(w, e))) act = true;
        if (!f.cond(v)) break;
      }
      if (o1 > o0) f.combineFunc((void *)data, v);
    }
    const unsigned word = __ballot_sync(0xffffffffu, act);
    if (lane == 0) next[v >> 5] = word;
    if (act) {
      my_size++;
      my_edges += __ldg(g.out.off + v + 1) - __ldg(g.out.off + v);
    }
  }
  my_size = warp_sum(my_size);
  my_edges = warp_sum(my_edges);
  if (lane == 0 && my_size) {
    atomicAdd(&cnt->size, my_size);
    atomicAdd(&cnt->edges, my_edges);
  }
}

// ---------------------------------------------------------------------------
// Dense push (edgeMapDenseForward, polymer.h:970-1032): every vertex in the
// frontier bitmap pushes over its out-edges with atomics; d's bit is set
// when cond(d) && updateAtomic(s, d, w).  Same warp groups as the pull, over
// the CSR, with inactive rows contributing no edges; heavy rows are pushed
// by the chunk kernel.
// ---------------------------------------------------------------------------
template <class F, class W>
__global__ void __launch_bounds__(256) k_dense_push(GraphView g, const uint32_t *__restrict__ cur,
                                                    F f, const W *__restrict__ w,
                                                    uint32_t *__restrict__ next, Counters *cnt) {
  const int lane = lane_id(), wid = threadIdx.x >> 5;
  const int grp = blockIdx.x * 8 + wid;
  if (grp >= g.out.ngroups) return;
  const int r_begin = __ldg(g.out.gstart + grp), r_end = __ldg(g.out.gstart + grp + 1);
  unsigned long long my_size = 0, my_edges = 0;
  for (int rb = r_begin; rb < r_end; rb += 32) {
    const int r = rb + lane;
    int o0 = 0, deg = 0;
    if (r < r_end && test_bit(cur, r)) {
      o0 = __ldg(g.out.off + r);
      deg = __ldg(g.out.off + r + 1) - o0;
    }
    const int ldeg = deg > g.heavy_deg ? 0 : deg;
    int total;
    const int pos = warp_excl_scan(ldeg, &total);
    for (int c = 0; c < total; c += 32) {
      const int q = c + lane;
      int j = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        int cand = j + step;
        if (__shfl_sync(0xffffffffu, pos, cand) <= q) j = cand;
      }
      const int oj = __shfl_sync(0xffffffffu, o0, j);
      const int pj = __shfl_sync(0xffffffffu, pos, j);
      if (q < total) {
        const int64_t e = (int64_t)oj + (q - pj);
        const int d = checked_id(g, __ldg(g.out.idx + e));
        if (f.cond(d) && update_atomic(f, rb + j, d, load_w(w, e)) && set_bit_new(next, d)) {
          my_size++;
          my_edges += __ldg(g.out.off + d + 1) - __ldg(g.out.off + d);
        }
      }
    }
  }
  my_size = warp_sum(my_size);
  my_edges = warp_sum(my_edges);
  if (lane == 0 && my_size) {
    atomicAdd(&cnt->size, my_size);
    atomicAdd(&cnt->edges, my_edges);
  }
}

template <class F, class W>
__global__ void __launch_bounds__(kChunkThreads) k_heavy_push(GraphView g,
                                                              const uint32_t *__restrict__ cur, F f,
                                                              const W *__restrict__ w,
                                                              uint32_t *__restrict__ next,
                                                              Counters *cnt) {
  const int c = blockIdx.x;
  if (c >= g.out.nchunks) return;
  const int r = __ldg(g.out.hrow + c);
  if (!test_bit(cur, r)) return;
  const int k = c - __ldg(g.out.hfirst + r);
  const int64_t e0 = (int64_t)__ldg(g.out.off + r) + (int64_t)k * kChunkEdges;
  const int64_t e1 = min(e0 + kChunkEdges, (int64_t)__ldg(g.out.off + r + 1));
  unsigned long long my_size = 0, my_edges = 0;
  for (int64_t e = e0 + threadIdx.x; e < e1; e += kChunkThreads) {
    const int d = checked_id(g, __ldg(g.out.idx + e));
    if (f.cond(d) && update_atomic(f, r, d, load_w(w, e)) && set_bit_new(next, d)) {
      my_size++;
      my_edges += __ldg(g.out.off + d + 1) - __ldg(g.out.off + d);
    }
  }
  my_size = warp_sum(my_size);
  my_edges = warp_sum(my_edges);
  if (lane_id() == 0 && my_size) {
    atomicAdd(&cnt->size, my_size);
    atomicAdd(&cnt->edges, my_edges);
  }
}

// ---------------------------------------------------------------------------
// Frontier plumbing.
// ---------------------------------------------------------------------------
// Bitmap -> queue (LocalFrontier::toSparse, polymer.h:552-567): ballot/popc
// compaction, one queue atomic per warp; also counts |F| and sum outdeg(F).
__global__ void k_bits_to_queue(int32_t n, const int32_t *__restrict__ out_off,
                                const uint32_t *__restrict__ bits, int32_t *__restrict__ queue,
                                Counters *cnt, const RoundGate *gate = nullptr);
// Queue -> bitmap (LocalFrontier::toDense, polymer.h:594-601).
__global__ void k_queue_to_bits(const int32_t *__restrict__ queue, int32_t size,
                                uint32_t *__restrict__ bits);
// |F| and sum outdeg(F) of a bitmap (vertexCounter, polymer.h:2311-2338).
__global__ void k_bits_stats(int32_t n, const int32_t *__restrict__ out_off,
                             const uint32_t *__restrict__ bits, Counters *cnt);

// vertexMap over a bitmap (polymer.h:2340-2381).
template <class F>
__global__ void k_vertex_map_bits(int32_t n, const uint32_t *__restrict__ bits, F f) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
    if (test_bit(bits, (int)v)) f((int)v);
}
// vertexMap over a sparse frontier (the queue of a sparse round).
template <class F>
__global__ void k_vertex_map_queue(const int32_t *__restrict__ queue, int32_t size, F f) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < size; i += stride) f(queue[i]);
}
// vertexMap over all vertices.
template <class F>
__global__ void k_vertex_map_all(int32_t n, F f) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) f((int)v);
}
// vertexFilter (polymer.h:2399-2441): out bit = in bit && f(v); counts |out|.
template <class F>
__global__ void k_vertex_filter(int32_t n, const int32_t *__restrict__ out_off,
                                const uint32_t *__restrict__ bits, F f,
                                uint32_t *__restrict__ out, Counters *cnt) {
  const int lane = lane_id();
  const int64_t ntot = ((int64_t)n + 31) & ~31ll;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  unsigned long long my_size = 0, my_edges = 0;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntot; t += stride) {
    int v = (int)t;
    bool keep = v < n && test_bit(bits, v) && f(v);
    unsigned word = __ballot_sync(0xffffffffu, keep);
    if (lane == 0) out[v >> 5] = word;
    if (keep) {
      my_size++;
      my_edges += __ldg(out_off + v + 1) - __ldg(out_off + v);
    }
  }
  my_size = warp_sum(my_size);
  my_edges = warp_sum(my_edges);
  if (lane == 0 && my_size) {
    atomicAdd(&cnt->size, my_size);
    atomicAdd(&cnt->edges, my_edges);
  }
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
enum Option { DENSE = 0, DENSE_PARALLEL = 1, DENSE_FORWARD = 2 };  // polymer.h:913-915

// A frontier on the device (the reference's vertices / LocalFrontier).
struct VertexSubset {
  int32_t n = 0;
  uint32_t *bits = nullptr;   // ceil(n/32) words, always valid
  int32_t *queue = nullptr;   // capacity n; valid when has_queue
  bool has_queue = false;
  int64_t size = 0;           // |F|
  int64_t edges = 0;          // sum of out-degrees of F
  int64_t words() const { return ((int64_t)n + 31) / 32; }
};

// CUDA-event brackets around application passes (pm_profile_*).  Pending
// brackets are folded into per-tag totals (milliseconds, passes) once the
// stream has drained.  While a loop is being captured into a CUDA graph the
// brackets become external event-record nodes owned by that graph; each
// replay re-records them and fold_graph() adds their times.
struct Profiler {
  struct Rec {
    std::string tag;
    cudaEvent_t a, b;
  };
  struct Total {
    std::string tag;
    double ms = 0.0;
    int64_t passes = 0;
  };
  bool enabled = false;
  bool capturing = false;
  std::vector<Rec> recs;          // pending, launched directly
  std::vector<Rec> captured;      // recorded by the capture in progress
  std::vector<Total> totals;
  std::vector<cudaEvent_t> pool;
  cudaEvent_t take() {
    if (!pool.empty()) {
      cudaEvent_t e = pool.back();
      pool.pop_back();
      return e;
    }
    cudaEvent_t e;
    PM_CUDA(cudaEventCreate(&e));
    return e;
  }
  void record(cudaEvent_t e, cudaStream_t s) {
    if (capturing)
      PM_CUDA(cudaEventRecordWithFlags(e, s, cudaEventRecordExternal));
    else
      PM_CUDA(cudaEventRecord(e, s));
  }
  void begin(const char *tag, cudaStream_t s) {
    if (!enabled) return;
    Rec r{tag, take(), take()};
    record(r.a, s);
    (capturing ? captured : recs).push_back(r);
  }
  void end(cudaStream_t s) {
    if (!enabled) return;
    std::vector<Rec> &v = capturing ? captured : recs;
    if (!v.empty()) record(v.back().b, s);
  }
  void add(const Rec &r) {
    float ms = 0.f;
    PM_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
    for (auto &t : totals)
      if (t.tag == r.tag) {
        t.ms += ms;
        t.passes++;
        return;
      }
    totals.push_back(Total{r.tag, (double)ms, 1});
  }
  // The stream has drained: fold the pending brackets.
  void fold() {
    for (auto &r : recs) {
      add(r);
      pool.push_back(r.a);
      pool.push_back(r.b);
    }
    recs.clear();
  }
  void fold_graph(const std::vector<Rec> &g) {
    for (auto &r : g) add(r);
  }
  void release(std::vector<Rec> &v) {
    for (auto &r : v) {
      pool.push_back(r.a);
      pool.push_back(r.b);
    }
    v.clear();
  }
  ~Profiler() {
    release(recs);
    release(captured);
    for (auto e : pool) cudaEventDestroy(e);
  }
};

// Run-time tunables of one graph (pm_graph_set_tunable, pm_tune).
struct Tunables {
  int32_t heavy_deg = kHeavyDeg;     // rows with more edges are split in chunks
  int32_t cta_expand = kCtaExpand;   // sparse push: CTA-wide expansion from this degree
  int32_t grid_expand = kGridExpand; // sparse push: grid-wide hub expansion from this degree
  int32_t pull_ctas_per_sm = 0;      // persistent pull-reduce CTAs per SM (0 = occupancy limit)
  int32_t bfs_div = 20, cc_div = 8, bf_div = 20;  // default threshold = m / div
  int32_t cuda_graphs = 1;           // capture the fixed-iteration loops
  int32_t heavy_mode = 0;            // heavy chunks: 0 a launch before the pull, 1 inside it,
                                     // 2 a launch beside it on a second stream
  int32_t hub_cache = 0;             // FP32 PageRank: sources cached in shared memory (0 = off)
  int32_t multi_div = 8;             // multi-source BFS / BellmanFord: default threshold = m / div
  int32_t bf_dense = 2;              // BellmanFord dense rounds: 0 pull-reduce over the CSC,
                                     // 1 push over the frontier's out-edges (DENSE_FORWARD),
                                     // 2 that push with atomics whose result is unused
  int32_t cc_mode = 0;               // Components on a symmetric graph: 0 union-find,
                                     // 1 label propagation (the reference's rounds)
  int32_t bf_delta = 0;              // BellmanFord: > 0 relaxes only frontier vertices below a
                                     // bound that moves by this much (delta-stepping); 0 all
  int32_t pull_stage = 0;            // pull-reduce: 1 copies each batch's CSC ids to shared
                                     // memory with one bulk copy (unweighted / int weights)
  int32_t push_agg = 0;              // sparse push: 1 warp-aggregates the atomicMin updates of
                                     // Components and BellmanFord
};

// Key of a captured loop: its name and every value its launches bake in.
inline void key_part(std::string &k, const void *p) {
  char b[24];
  snprintf(b, sizeof b, "|%p", p);
  k += b;
}
inline void key_part(std::string &k, double x) {
  uint64_t u;
  memcpy(&u, &x, 8);
  k += "|" + std::to_string(u);
}
inline void key_part(std::string &k, int64_t x) { k += "|" + std::to_string(x); }
inline void key_part(std::string &k, int x) { k += "|" + std::to_string(x); }
template <class... A>
std::string loop_key(const char *name, A... a) {
  std::string k(name);
  (key_part(k, a), ...);
  return k;
}

// A captured iteration loop, keyed by everything its launches bake in.
struct LoopGraph {
  std::string key;
  int uses = 0;                    // runs of this loop so far
  cudaGraphExec_t exec = nullptr;  // captured at the second run
  long long launches = 0;
  std::vector<Profiler::Rec> recs;
};

// Per-graph execution context: stream, counters, scratch.
struct Engine {
  GraphView g;
  cudaStream_t stream = nullptr;
  bool host_steps = false;     // loops call back to the host between passes: never captured
  Counters *d_cnt = nullptr;   // [0] next frontier, [1] deferred rows, [2] aux
  Counters *h_cnt = nullptr;   // pinned mirror
  int32_t *defer = nullptr;    // n
  int32_t *hubs = nullptr;     // kMaxHubs
  void *partials = nullptr;    // max(in.nchunks, 1) * 16 bytes
  int32_t *hdone = nullptr;    // max(in.nchunks, 1) chunk counters of the fused pull
  cudaStream_t side = nullptr;   // second stream of the overlapped pull (created on first use)
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  int num_sms = 148;
  Profiler prof;
  Tunables tune;
  std::vector<LoopGraph> graphs;  // most recent last
  const char *tag = "edgemap";  // profile tag of the running application

  int grid_for(int64_t threads, int block = 256, int per_sm = 8) const {
    int64_t b = (threads + block - 1) / block;
    int64_t cap = (int64_t)num_sms * per_sm;
    return (int)std::max<int64_t>(1, std::min(b, cap));
  }
  // CTAs of a persistent kernel: the occupancy limit, or the tuned count.
  int persistent_grid(int64_t want, int occupancy_per_sm) const {
    int per_sm = occupancy_per_sm;
    if (tune.pull_ctas_per_sm > 0) per_sm = std::min(per_sm, tune.pull_ctas_per_sm);
    return (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)num_sms * std::max(per_sm, 1)));
  }
  void reset_counters() {
    PM_CUDA(cudaMemsetAsync(d_cnt, 0, 3 * sizeof(Counters), stream));
  }
  // Blocks until the counters are on the host.
  const Counters *read_counters() {
    PM_CUDA(cudaMemcpyAsync(h_cnt, d_cnt, 3 * sizeof(Counters), cudaMemcpyDeviceToHost, stream));
    PM_CUDA(cudaStreamSynchronize(stream));
    for (int i = 0; i < 3; ++i)
      if (h_cnt[i].err) {
        unsigned e = h_cnt[i].err;
        fail(e & kErrTimeout ? PM_ERR_TIMEOUT : PM_ERR_CUDA,
             std::string("device error word ") + std::to_string(e) +
                 (e & kErrQueueOverflow ? " (queue overflow)" : "") +
                 (e & kErrRange ? " (id out of range)" : ""));
      }
    return h_cnt;
  }
  void ensure_side_stream() {
    if (side) return;
    PM_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
    PM_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    PM_CUDA(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
  }
  void release_side_stream() {
    if (side) {
      cudaStreamSynchronize(side);
      cudaStreamDestroy(side);
    }
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    side = nullptr;
    ev_fork = ev_join = nullptr;
  }
  void drop_graph(LoopGraph &lg) {
    if (lg.exec) cudaGraphExecDestroy(lg.exec);
    lg.exec = nullptr;
    prof.release(lg.recs);
  }
  void release_graphs() {
    for (auto &lg : graphs) drop_graph(lg);
    graphs.clear();
  }
  // Runs body() -- launches on `stream` only, no host synchronisation --
  // directly the first time `key` is seen, captured into a CUDA graph the
  // second time, and by replaying that graph from then on (when CUDA graphs
  // are on; a loop run once costs no capture).  The key must name every value
  // the launches bake in: pointers, sizes, scalars and whether profiling is on.
  template <class Body>
  void run_loop(const std::string &key_in, Body &&body) {
    if (!tune.cuda_graphs || host_steps) {
      body();
      return;
    }
    const std::string key = key_in + (prof.enabled ? "|prof" : "|-");
    LoopGraph *lg = nullptr;
    for (auto &x : graphs)
      if (x.key == key) lg = &x;
    if (!lg) {
      if (graphs.size() >= 16) {
        drop_graph(graphs.front());
        graphs.erase(graphs.begin());
      }
      graphs.push_back(LoopGraph{});
      graphs.back().key = key;
      lg = &graphs.back();
    }
    if (++lg->uses == 1) {
      body();
      return;
    }
    if (!lg->exec) {
      LoopGraph &fresh = *lg;
      const long long before = launches(false);
      PM_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeRelaxed));
      prof.capturing = true;
      cudaGraph_t cg = nullptr;
      try {
        body();
      } catch (...) {
        prof.capturing = false;
        prof.release(prof.captured);
        cudaStreamEndCapture(stream, &cg);
        if (cg) cudaGraphDestroy(cg);
        throw;
      }
      prof.capturing = false;
      fresh.recs.swap(prof.captured);
      PM_CUDA(cudaStreamEndCapture(stream, &cg));
      const cudaError_t ie = cudaGraphInstantiate(&fresh.exec, cg, 0);
      cudaGraphDestroy(cg);
      if (ie != cudaSuccess) {
        prof.release(fresh.recs);
        fail_cuda(ie, "cudaGraphInstantiate", __FILE__, __LINE__);
      }
      fresh.launches = launches(false) - before;
      count_launch((int)-fresh.launches);  // captured, not run
    }
    PM_CUDA(cudaGraphLaunch(lg->exec, stream));
    count_launch((int)lg->launches);
    if (prof.enabled && !lg->recs.empty()) {
      PM_CUDA(cudaStreamSynchronize(stream));
      prof.fold_graph(lg->recs);
    }
  }
};

// Recount s.size / s.edges from s.bits (vertexCounter, polymer.h:2311-2338).
PM_CXX_API void subset_recount(Engine &E, VertexSubset &s);
// Make sure s.queue holds s (compaction of the bitmap).
PM_CXX_API void subset_to_queue(Engine &E, VertexSubset &s);
// Single vertex frontier.
PM_CXX_API void subset_single(Engine &E, VertexSubset &s, int32_t v);
// All vertices.
PM_CXX_API void subset_all(Engine &E, VertexSubset &s);
PM_CXX_API void subset_clear(Engine &E, VertexSubset &s);

// Direction switch of edgeMap (polymer.h:2247, 2260): dense when
// |F| + outdeg(F) >= threshold.
inline bool go_dense(const VertexSubset &cur, int64_t threshold) {
  return cur.size + cur.edges >= threshold;
}

template <class W, class F>
void launch_sparse_push(Engine &E, VertexSubset &cur, F f, const W *w_out, VertexSubset &next) {
  subset_to_queue(E, cur);
  PM_CUDA(cudaMemsetAsync(next.bits, 0, next.words() * 4, E.stream));
  if (cur.size > 0) {
    int grid = E.grid_for(cur.size, 256, 8);
    PM_LAUNCH((k_sparse_push<F, W>), grid, 256, 0, E.stream, E.g, cur.queue, (int32_t)cur.size, f,
              w_out, next.queue, next.bits, next.n, E.d_cnt, E.hubs, E.d_cnt + 1);
    PM_LAUNCH((k_sparse_push_hubs<F, W>), E.num_sms * 4, 256, 0, E.stream, E.g, f, w_out, E.hubs,
              E.d_cnt + 1, next.queue, next.bits, next.n, E.d_cnt);
  }
  next.has_queue = true;
}

template <class W, class F>
void launch_dense_pull(Engine &E, VertexSubset &cur, F f, const W *w_in, VertexSubset &next) {
  int64_t nthreads = ((int64_t)E.g.n + 31) & ~31ll;
  PM_LAUNCH((k_dense_pull<F, W>), E.grid_for(nthreads, 256, 16), 256, 0, E.stream, E.g, cur.bits, f,
            w_in, next.bits, E.defer, E.d_cnt, E.d_cnt + 1);
  PM_LAUNCH((k_dense_pull_defer<F, W>), E.num_sms * 8, 256, 0, E.stream, E.g, cur.bits, f, w_in,
            next.bits, E.defer, E.d_cnt, E.d_cnt + 1);
  next.has_queue = false;
}

template <class W, class F>
void launch_dense_push(Engine &E, VertexSubset &cur, F f, const W *w_out, VertexSubset &next) {
  PM_CUDA(cudaMemsetAsync(next.bits, 0, next.words() * 4, E.stream));
  if (E.g.out.nchunks > 0)
    PM_LAUNCH((k_heavy_push<F, W>), E.g.out.nchunks, kChunkThreads, 0, E.stream, E.g, cur.bits, f,
              w_out, next.bits, E.d_cnt);
  PM_LAUNCH((k_dense_push<F, W>), (E.g.out.ngroups + 7) / 8, 256, 0, E.stream, E.g, cur.bits, f,
            w_out, next.bits, E.d_cnt);
  next.has_queue = false;
}

template <class W, class F>
void launch_pull_seq(Engine &E, VertexSubset &cur, F f, const W *w_in, VertexSubset &next) {
  const int64_t nthreads = ((int64_t)E.g.n + 31) & ~31ll;
  PM_LAUNCH((k_pull_seq<F, W>), E.grid_for(nthreads, 256, 16), 256, 0, E.stream, E.g, cur.bits, f, w_in,
            next.bits, E.d_cnt);
  next.has_queue = false;
}

// Pull-reduce over the CSC into counters cnt (size / edges of the output,
// daux = sum of the FP64 values commit() adds); next_bits may be null.
template <class W, class F>
void launch_pull_reduce(Engine &E, F f, const W *w_in, uint32_t *next_bits, Counters *cnt,
                        HubCache<typename F::Acc> hubs = {}) {
  static_assert(sizeof(typename F::Acc) <= 16, "accumulator larger than the partials slot");
  using Acc = typename F::Acc;
  Acc *partials = reinterpret_cast<Acc *>(E.partials);
  const int mode = E.g.in.nchunks > 0 ? E.tune.heavy_mode : 0;
  if constexpr (HubTrait<F>::value) {
    if (hubs.count > 0 && mode == 0) {
      // kHubBlock-thread CTAs, each holding the cached values
      static const int hub_per_sm = [] {
        PM_CUDA(cudaFuncSetAttribute((const void *)k_pull_reduce<F, W, 0, true>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, kHubMax * (int)sizeof(Acc)));
        int r = 0;
        PM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, k_pull_reduce<F, W, 0, true>, kHubBlock,
                                                              kHubMax * sizeof(Acc)));
        return std::max(r, 1);
      }();
      if (E.g.in.nchunks > 0)
        PM_LAUNCH((k_heavy_reduce<F, W>), E.g.in.nchunks, kChunkThreads, 0, E.stream, E.g, f, w_in, partials);
      const int64_t want = ((int64_t)E.g.in.ngroups + kHubBlock / 32 - 1) / (kHubBlock / 32);
      PM_LAUNCH((k_pull_reduce<F, W, 0, true>), E.persistent_grid(want, hub_per_sm), kHubBlock,
                (size_t)hubs.count * sizeof(Acc), E.stream, E.g, f, w_in, partials, (int32_t *)nullptr, next_bits,
                cnt, hubs);
      return;
    }
  }
  if (mode == 1) {
    PM_CUDA(cudaMemsetAsync(E.hdone, 0, (size_t)E.g.in.nchunks * 4, E.stream));
  } else if (mode == 2) {
    E.ensure_side_stream();
    PM_CUDA(cudaEventRecord(E.ev_fork, E.stream));
    PM_CUDA(cudaStreamWaitEvent(E.side, E.ev_fork, 0));
    PM_LAUNCH((k_heavy_reduce<F, W>), E.g.in.nchunks, kChunkThreads, 0, E.side, E.g, f, w_in, partials);
    PM_CUDA(cudaEventRecord(E.ev_join, E.side));
  } else if (E.g.in.nchunks > 0) {
    PM_LAUNCH((k_heavy_reduce<F, W>), E.g.in.nchunks, kChunkThreads, 0, E.stream, E.g, f, w_in, partials);
  }
  // persistent grid: as many CTAs as fit on the device at once
  // resident CTAs per SM of each mode's kernel (thread-safe one-time init)
  static const std::array<int, 3> per_sm = [] {
    std::array<int, 3> r{};
    PM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r[0], k_pull_reduce<F, W, 0>, kPullBlock, 0));
    PM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r[1], k_pull_reduce<F, W, 1>, kPullBlock, 0));
    PM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r[2], k_pull_reduce<F, W, 2>, kPullBlock, 0));
    for (int &x : r) x = std::max(x, 1);
    return r;
  }();
  const int64_t tickets = (int64_t)E.g.in.ngroups + (mode == 1 ? E.g.in.nchunks : 0);
  const int64_t want = (tickets + kPullBlock / 32 - 1) / (kPullBlock / 32);
  if (mode == 1) {
    PM_LAUNCH((k_pull_reduce<F, W, 1>), E.persistent_grid(want, per_sm[1]), kPullBlock, 0, E.stream, E.g, f,
              w_in, partials, E.hdone, next_bits, cnt);
  } else if (mode == 2) {
    PM_LAUNCH((k_pull_reduce<F, W, 2>), E.persistent_grid(want, per_sm[2]), kPullBlock, 0, E.stream, E.g, f,
              w_in, partials, (int32_t *)nullptr, next_bits, cnt);
    PM_CUDA(cudaStreamWaitEvent(E.stream, E.ev_join, 0));
    PM_LAUNCH((k_heavy_commit<F>), E.grid_for(E.g.in.nchunks, 256, 4), 256, 0, E.stream, E.g, f,
              (const Acc *)partials, next_bits, cnt);
  } else {
    if constexpr (std::is_same<W, int>::value) {
      // staged ids: the bulk copies need a 16-byte aligned id array
      if (E.tune.pull_stage && ((uintptr_t)E.g.in.idx & 15) == 0) {
        constexpr size_t smem = kStageSmem;
        static const int stage_per_sm = [] {
          int r = 0;
          PM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, k_pull_reduce<F, W, 0, false, true>,
                                                                kPullBlock, smem));
          return std::max(r, 1);
        }();
        PM_LAUNCH((k_pull_reduce<F, W, 0, false, true>), E.persistent_grid(want, stage_per_sm), kPullBlock, smem,
                  E.stream, E.g, f, w_in, partials, (int32_t *)nullptr, next_bits, cnt, HubCache<Acc>{});
        return;
      }
    }
    PM_LAUNCH((k_pull_reduce<F, W, 0>), E.persistent_grid(want, per_sm[0]), kPullBlock, 0, E.stream, E.g, f,
              w_in, partials, (int32_t *)nullptr, next_bits, cnt);
  }
}

// edgeMap (polymer.h:2240-2309): sparse push below the threshold, otherwise
// dense pull (option DENSE / DENSE_PARALLEL) or dense push (DENSE_FORWARD).
// On return next holds the output frontier with its size and out-degree sum.
template <class W = int, class F>
void edgeMap(Engine &E, VertexSubset &cur, F f, VertexSubset &next, int64_t threshold,
             Option option = DENSE, const W *w_out = nullptr, const W *w_in = nullptr,
             bool *took_dense = nullptr) {
  E.reset_counters();
  const bool dense = go_dense(cur, threshold);
  if (took_dense) *took_dense = dense;
  E.prof.begin(E.tag, E.stream);
  if (dense) {
    if (option == DENSE_FORWARD)
      launch_dense_push<W>(E, cur, f, w_out, next);
    else
      launch_dense_pull<W>(E, cur, f, w_in, next);
  } else {
    launch_sparse_push<W>(E, cur, f, w_out, next);
  }
  E.prof.end(E.stream);
  const Counters *h = E.read_counters();
  next.size = (int64_t)h[0].size;
  next.edges = (int64_t)h[0].edges;
}

// edgeMap with a reducing dense path (edgeMapCustom numa-Components.C:121-175
// / edgeMapDenseReduce): dense rounds run the pull-reduce with fused commit
// (functors with identity / edge / combine / commit) or the reference's
// sequential fold (functors with initFunc / reduceFunc / combineFunc),
// sparse rounds the push with updateAtomic.
template <class W = int, class F>
void edgeMapReduce(Engine &E, VertexSubset &cur, F f, VertexSubset &next, int64_t threshold,
                   const W *w_out = nullptr, const W *w_in = nullptr, bool *took_dense = nullptr) {
  E.reset_counters();
  const bool dense = go_dense(cur, threshold);
  if (took_dense) *took_dense = dense;
  E.prof.begin(E.tag, E.stream);
  if (dense) {
    if constexpr (RefReduceShape<F>::value) {
      launch_pull_seq<W>(E, cur, f, w_in, next);
    } else {
      launch_pull_reduce<W>(E, f, w_in, next.bits, E.d_cnt);
      next.has_queue = false;
    }
  } else {
    launch_sparse_push<W>(E, cur, f, w_out, next);
  }
  E.prof.end(E.stream);
  const Counters *h = E.read_counters();
  next.size = (int64_t)h[0].size;
  next.edges = (int64_t)h[0].edges;
}

// vertexMap (polymer.h:2340-2381): over the queue when the subset has one,
// else over the bitmap.
template <class F>
void vertexMap(Engine &E, VertexSubset &s, F f) {
  if (s.has_queue) {
    if (s.size > 0)
      PM_LAUNCH((k_vertex_map_queue<F>), E.grid_for(s.size, 256, 16), 256, 0, E.stream, s.queue,
                (int32_t)s.size, f);
  } else {
    PM_LAUNCH((k_vertex_map_bits<F>), E.grid_for(s.n, 256, 16), 256, 0, E.stream, s.n, s.bits, f);
  }
}

template <class F>
void vertexMapAll(Engine &E, int32_t n, F f) {
  PM_LAUNCH((k_vertex_map_all<F>), E.grid_for(n, 256, 16), 256, 0, E.stream, n, f);
}

template <class F>
void vertexFilter(Engine &E, VertexSubset &s, F f, VertexSubset &out) {
  E.reset_counters();
  int64_t nthreads = ((int64_t)s.n + 31) & ~31ll;
  PM_LAUNCH((k_vertex_filter<F>), E.grid_for(nthreads, 256, 16), 256, 0, E.stream, s.n,
            E.g.out.off, s.bits, f, out.bits, E.d_cnt);
  const Counters *h = E.read_counters();
  out.size = (int64_t)h[0].size;
  out.edges = (int64_t)h[0].edges;
  out.has_queue = false;
}

}  // namespace pm
