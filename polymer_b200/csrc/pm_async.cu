// pm_async.cu -- asynchronous BFS: one persistent launch, no level barriers
// (the GPU form of numa-BFS-async-pipe.C with edgeMapSparseAsyncPipe,
// polymer.h:1513-1751, where NUMA nodes pass chunks of discovered vertices
// around a ring until an end-game message has gone round twice).
//
// Semantics (BFS_F of numa-BFS-async-pipe.C:52-72): a vertex is claimed by
// the first in-neighbour whose CAS on Parents[d] succeeds, whatever its
// level, so the result is the set reached from src and a parent tree over it
// (every parent edge exists; following parents ends at src, since a parent
// was claimed before it could claim its child) -- not a BFS tree.
//
// Work queue: items are (vertex, chunk) in 64 bits; a vertex with more than
// kAsyncChunk out-edges is split in chunks.  A warp takes a ticket (the next
// slot, one atomicAdd), waits for that slot to be written, relaxes the item's
// edges lane-strided and appends the vertices it claimed with one
// reservation per warp.  `outstanding` counts items enqueued and not yet
// finished: children are counted before their parent is retired, so it
// reaches 0 only when the traversal is complete, and every warp then exits.
// Every wait (for an item, for a slot) is bounded; a wait that runs out sets
// kErrTimeout and all warps leave.
#include <algorithm>

#include "pm_graph.cuh"

namespace pm {

namespace {

constexpr int kAsyncChunk = 2048;                 // edges of one queue item
constexpr unsigned long long kEmptySlot = ~0ull;  // queue slot not yet written
constexpr long long kAsyncSpins = 1ll << 22;      // x <= ~1 us: a few seconds at most

struct AsyncCtl {
  unsigned long long head, tail, outstanding, reached, edges;
  unsigned err, pad;
};

__device__ __forceinline__ unsigned long long item_of(int v, int c) {
  return ((unsigned long long)(unsigned)v << 32) | (unsigned)c;
}

__device__ __forceinline__ unsigned long long ld_volatile(const unsigned long long *p) {
  return *(const volatile unsigned long long *)p;
}

__global__ void k_async_init(unsigned long long *queue, int64_t cap, int32_t *parents, int64_t n, int src) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += stride) queue[i] = kEmptySlot;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
    parents[v] = v == src ? src : -1;
}

// The source's items (one per chunk of its out-edges), before the traversal.
__global__ void k_async_seed(GraphView g, unsigned long long *queue, int src, AsyncCtl *ctl) {
  const int deg = g.out.off[src + 1] - g.out.off[src];
  const int nch = (deg + kAsyncChunk - 1) / kAsyncChunk;
  for (int c = 0; c < nch; ++c) queue[c] = item_of(src, c);
  ctl->head = 0;
  ctl->tail = (unsigned long long)nch;
  ctl->outstanding = (unsigned long long)nch;
  ctl->reached = 1;
  ctl->edges = 0;
  ctl->err = 0;
}

// Appends the items of one warp (lanes with want set) and counts them as
// outstanding first.  Returns nothing; slots are written after reservation.
__device__ __forceinline__ void warp_enqueue(bool want, unsigned long long item, unsigned long long *queue,
                                             int64_t cap, AsyncCtl *ctl) {
  const int lane = lane_id();
  const unsigned mask = __ballot_sync(0xffffffffu, want);
  if (!mask) return;
  unsigned long long base = 0;
  if (lane == 0) {
    atomicAdd(&ctl->outstanding, (unsigned long long)__popc(mask));
    base = atomicAdd(&ctl->tail, (unsigned long long)__popc(mask));
  }
  base = shfl_idx(base, 0);
  if (want) {
    const unsigned long long pos = base + __popc(mask & ((1u << lane) - 1u));
    if (pos < (unsigned long long)cap)
      queue[pos] = item;
    else
      atomicOr(&ctl->err, (unsigned)kErrQueueOverflow);
  }
}

__global__ void __launch_bounds__(256) k_bfs_async(GraphView g, int32_t *parents, unsigned long long *queue,
                                                  int64_t cap, AsyncCtl *ctl) {
  const int lane = lane_id();
  unsigned long long my_edges = 0, my_reached = 0;
  for (;;) {
    // lane 0 takes a ticket (one atomicAdd, no retry loop: thousands of warps
    // contend for the head) and waits for the item of that slot, or for the
    // end: outstanding == 0 means nothing is queued or in flight, so the
    // slot will never be written.  Bounded, with backoff.
    unsigned long long item = kEmptySlot;
    if (lane == 0) {
      const unsigned long long pos = atomicAdd(&ctl->head, 1ull);
      long long spins = 0;
      unsigned sleep = 32;
      for (;;) {
        if (pos < (unsigned long long)cap && (item = ld_volatile(queue + pos)) != kEmptySlot) break;
        if (ld_volatile(&ctl->outstanding) == 0 || *(volatile unsigned *)&ctl->err) break;
        if (++spins > kAsyncSpins) {
          atomicOr(&ctl->err, (unsigned)kErrTimeout);
          break;
        }
        __nanosleep(sleep);
        if (sleep < 1024) sleep <<= 1;
      }
    }
    item = shfl_idx(item, 0);
    if (item == kEmptySlot) break;
    const int v = (int)(item >> 32), c = (int)(item & 0xffffffffu);
    const int64_t r0 = __ldg(g.out.off + v), r1 = __ldg(g.out.off + v + 1);
    const int64_t e0 = r0 + (int64_t)c * kAsyncChunk, e1 = std::min(e0 + kAsyncChunk, r1);
    for (int64_t base = e0; base < e1; base += 32) {
      const int64_t e = base + lane;
      bool claimed = false;
      int d = 0;
      if (e < e1) {
        d = __ldg(g.out.idx + e);
        claimed = *((volatile int32_t *)parents + d) == -1 && atomicCAS(parents + d, -1, v) == -1;
      }
      // a claimed vertex goes back to the queue, one item per chunk of its edges
      int dnch = 0;
      if (claimed) {
        const int ddeg = __ldg(g.out.off + d + 1) - __ldg(g.out.off + d);
        dnch = ddeg > 0 ? (ddeg + kAsyncChunk - 1) / kAsyncChunk : 0;
        my_reached++;
      }
      warp_enqueue(dnch > 0, item_of(d, 0), queue, cap, ctl);
      // hub chunks beyond the first, rare: one lane at a time
      unsigned hubs = __ballot_sync(0xffffffffu, dnch > 1);
      while (hubs) {
        const int j = __ffs(hubs) - 1;
        hubs &= hubs - 1;
        const int hd = __shfl_sync(0xffffffffu, d, j);
        const int hn = __shfl_sync(0xffffffffu, dnch, j);
        for (int c0 = 1; c0 < hn; c0 += 32) warp_enqueue(c0 + lane < hn, item_of(hd, c0 + lane), queue, cap, ctl);
      }
    }
    if (lane == 0) {
      my_edges += (unsigned long long)(e1 - e0);
      __threadfence();
      atomicAdd(&ctl->outstanding, ~0ull);  // retire the item (minus one)
    }
  }
  my_reached = warp_sum(my_reached);
  if (lane == 0) {
    if (my_reached) atomicAdd(&ctl->reached, my_reached);
    if (my_edges) atomicAdd(&ctl->edges, my_edges);
  }
}

}  // namespace

void run_bfs_async(pm_graph *g, int32_t src, int32_t *d_parents, pm_traversal_stats *st) {
  Engine &E = g->E;
  const int64_t n = g->n, m = g->m;
  // every vertex is claimed once; a claimed vertex of degree d takes
  // ceil(d / kAsyncChunk) items
  const int64_t cap = n + m / kAsyncChunk + 2;
  auto *queue = (unsigned long long *)g->scratch_buf(0, (size_t)cap * 8);
  auto *ctl = (AsyncCtl *)g->scratch_buf(1, sizeof(AsyncCtl));
  PM_LAUNCH(k_async_init, E.grid_for(std::max(cap, n), 256, 16), 256, 0, E.stream, queue, cap, d_parents, n, src);
  PM_LAUNCH(k_async_seed, 1, 1, 0, E.stream, E.g, queue, src, ctl);
  static const int per_sm = [] {
    int r = 0;
    PM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, k_bfs_async, 256, 0));
    return std::max(r, 1);
  }();
  E.prof.begin("bfs_async", E.stream);
  PM_LAUNCH(k_bfs_async, E.num_sms * per_sm, 256, 0, E.stream, E.g, d_parents, queue, cap, ctl);
  E.prof.end(E.stream);
  AsyncCtl h{};
  PM_CUDA(cudaMemcpyAsync(&h, ctl, sizeof h, cudaMemcpyDeviceToHost, E.stream));
  PM_CUDA(cudaStreamSynchronize(E.stream));
  if (h.err & kErrTimeout) fail(PM_ERR_TIMEOUT, "asynchronous BFS: a bounded wait ran out");
  if (h.err) fail(PM_ERR_CUDA, "asynchronous BFS: queue overflow");
  if (st) {
    *st = pm_traversal_stats{};
    st->rounds = 1;
    st->reached = (int64_t)h.reached;
    st->edges_visited = (int64_t)h.edges;
  }
}

}  // namespace pm
