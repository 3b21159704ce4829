// pm_alloc.cu -- the library's device allocator: cudaMalloc behind a cache of
// freed blocks.  A graph build allocates and frees a few dozen buffers of up
// to gigabytes (CSR/CSC copies, sort keys and values, tables, workspaces);
// cudaMalloc / cudaFree of such blocks cost a fraction of a millisecond each
// and cudaFree synchronises the device, so a workload that builds and
// destroys graphs (the end-to-end path) spends tens of milliseconds in them.
// Freed blocks are kept per device and handed out again for requests of
// close size.  Reuse is stream-ordered: a block freed inside a library call
// carries an event recorded on that call's stream, and the call that takes
// it makes its own stream wait on the event (a GPU-side dependency, no host
// wait), so host threads that drive distinct handles do not serialise.
#include <algorithm>
#include <atomic>
#include <mutex>
#include <vector>

#include "pm_graph.cuh"

namespace pm {

namespace {

// How a cached block may be reused: `ev` recorded after its last use (the
// taker waits on it), or nothing known about its last use (the taker
// synchronises the device), or idle.
struct Block {
  void *p;
  size_t cap;
  int device;
  cudaEvent_t ev;  // null unless recorded
  bool idle;
};

struct Cache {
  std::mutex mu;
  std::vector<Block> free;
  std::vector<std::pair<int, cudaEvent_t>> events;  // unused events, by device
  size_t cached = 0;
  int64_t limit = -1;  // bytes; -1: a quarter of the device memory, 0: off
  std::vector<int64_t> auto_limit;  // per device
};

thread_local AllocCtx t_ctx;

Cache &cache() {
  static Cache *c = new Cache();  // never destroyed: blocks outlive static teardown order
  return *c;
}

size_t round_cap(size_t b) {
  const size_t g = b < (1u << 20) ? 512 : (2u << 20);
  return (b + g - 1) / g * g;
}

int64_t limit_for(Cache &c, int dev) {
  if (c.limit >= 0) return c.limit;
  if ((int)c.auto_limit.size() <= dev) c.auto_limit.resize(dev + 1, -1);
  if (c.auto_limit[dev] < 0) {
    size_t fr = 0, tot = 0;
    c.auto_limit[dev] = cudaMemGetInfo(&fr, &tot) == cudaSuccess ? (int64_t)(tot / 4) : 0;
    (void)cudaGetLastError();
  }
  return c.auto_limit[dev];
}

// An event of device `dev` (current) from the pool, or a new one.
cudaEvent_t take_event(Cache &c, int dev) {
  for (size_t i = c.events.size(); i-- > 0;)
    if (c.events[i].first == dev) {
      cudaEvent_t e = c.events[i].second;
      c.events.erase(c.events.begin() + i);
      return e;
    }
  cudaEvent_t e = nullptr;
  if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
    (void)cudaGetLastError();
    return nullptr;
  }
  return e;
}

void release_all(Cache &c) {
  int cur = 0;
  cudaGetDevice(&cur);
  for (const Block &b : c.free) {
    cudaSetDevice(b.device);
    cudaFree(b.p);  // synchronises the device: the block's last use is over
    if (b.ev) c.events.push_back({b.device, b.ev});
  }
  cudaSetDevice(cur);
  (void)cudaGetLastError();
  c.free.clear();
  c.cached = 0;
}

}  // namespace

// Allocation-failure injection for tests: the k-th dev_alloc from now on
// (k >= 1) fails as an out-of-memory would; -1: off.
std::atomic<long long> g_fail_after{-1};

void set_alloc_fail_after(long long k) { g_fail_after.store(k < 1 ? -1 : k); }

AllocCtx alloc_ctx() { return t_ctx; }
void set_alloc_ctx(AllocCtx c) { t_ctx = c; }

void *dev_alloc(size_t bytes, size_t *cap, int *device) {
  Cache &c = cache();
  const size_t want = round_cap(bytes);
  if (g_fail_after.load() > 0 && g_fail_after.fetch_sub(1) == 1) {
    g_fail_after.store(-1);
    fail(PM_ERR_OOM, "injected allocation failure (pm_test_fail_alloc_after) of " + std::to_string(want) + " bytes");
  }
  int dev = 0;
  PM_CUDA(cudaGetDevice(&dev));
  Block b{nullptr, 0, dev, nullptr, false};
  {
    std::lock_guard<std::mutex> lk(c.mu);
    // the smallest cached block of this device that fits within 25 % (+2 MB)
    int best = -1;
    for (int i = 0; i < (int)c.free.size(); ++i) {
      const Block &f = c.free[i];
      if (f.device != dev || f.cap < want || f.cap > want + want / 4 + (2u << 20)) continue;
      if (best < 0 || f.cap < c.free[best].cap) best = i;
    }
    if (best >= 0) {
      b = c.free[best];
      c.free.erase(c.free.begin() + best);
      c.cached -= b.cap;
    }
  }
  if (b.p) {
    // after the previous owner's last use: in stream order, or on the host
    // when this thread names no stream, or by a device synchronisation when
    // nothing is known about that use
    cudaError_t e = cudaSuccess;
    if (b.ev)
      e = t_ctx.stream ? cudaStreamWaitEvent(t_ctx.stream, b.ev, 0) : cudaEventSynchronize(b.ev);
    else if (!b.idle)
      e = cudaDeviceSynchronize();
    if (b.ev) {
      std::lock_guard<std::mutex> lk(c.mu);
      c.events.push_back({b.device, b.ev});  // a later record does not move this wait
    }
    if (e != cudaSuccess) {
      cudaFree(b.p);
      fail_cuda(e, "reuse of a cached device block", __FILE__, __LINE__);
    }
    *cap = b.cap;
    *device = dev;
    return b.p;
  }
  void *p = nullptr;
  cudaError_t e = cudaMalloc(&p, want);
  if (e == cudaErrorMemoryAllocation) {  // give the cache back and try once more
    (void)cudaGetLastError();
    {
      std::lock_guard<std::mutex> lk(c.mu);
      release_all(c);
    }
    e = cudaMalloc(&p, want);
  }
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    fail(PM_ERR_OOM, "cudaMalloc of " + std::to_string(want) + " bytes failed: " + cudaGetErrorString(e));
  }
  *cap = want;
  *device = dev;
  return p;
}

void dev_free(void *p, size_t cap, int dev) {
  if (!p) return;
  Cache &c = cache();
  {
    std::lock_guard<std::mutex> lk(c.mu);
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess) (void)cudaGetLastError();
    // the cap of the block's device (measured with that device current)
    if (cur != dev) cudaSetDevice(dev);
    const int64_t lim = limit_for(c, dev);
    if (cur != dev && cur >= 0) cudaSetDevice(cur);
    if (lim > 0 && (int64_t)(c.cached + cap) <= lim) {
      Block b{p, cap, dev, nullptr, t_ctx.idle};
      if (!b.idle && t_ctx.stream && cur == dev) {
        b.ev = take_event(c, dev);
        if (b.ev && cudaEventRecord(b.ev, t_ctx.stream) != cudaSuccess) {
          (void)cudaGetLastError();
          c.events.push_back({dev, b.ev});
          b.ev = nullptr;  // the taker synchronises the device instead
        }
      }
      c.free.push_back(b);
      c.cached += cap;
      return;
    }
  }
  int cur = -1;
  if (cudaGetDevice(&cur) != cudaSuccess) (void)cudaGetLastError();
  if (cur != dev) cudaSetDevice(dev);
  cudaFree(p);
  if (cur != dev && cur >= 0) cudaSetDevice(cur);
  (void)cudaGetLastError();
}

void set_memory_cache(int64_t limit) {
  Cache &c = cache();
  std::lock_guard<std::mutex> lk(c.mu);
  c.limit = limit < 0 ? -1 : limit;
  if (limit >= 0 && (int64_t)c.cached > limit) release_all(c);
}

void release_memory_cache() {
  Cache &c = cache();
  std::lock_guard<std::mutex> lk(c.mu);
  release_all(c);
}

// Pinned host words of the graph handles (a few dozen bytes each), kept for
// reuse: cudaFreeHost synchronises the device, which would make a thread
// that destroys a handle wait for every other thread's kernels and copies.
namespace {
std::mutex g_pin_mu;
std::vector<std::pair<size_t, void *>> g_pin_free;
}  // namespace

void *pinned_small_alloc(size_t bytes) {
  {
    std::lock_guard<std::mutex> lk(g_pin_mu);
    for (size_t i = 0; i < g_pin_free.size(); ++i)
      if (g_pin_free[i].first == bytes) {
        void *p = g_pin_free[i].second;
        g_pin_free.erase(g_pin_free.begin() + i);
        return p;
      }
  }
  void *p = nullptr;
  PM_CUDA(cudaMallocHost(&p, bytes));
  return p;
}

void pinned_small_free(void *p, size_t bytes) {
  if (!p) return;
  std::lock_guard<std::mutex> lk(g_pin_mu);
  g_pin_free.push_back({bytes, p});
}

int64_t memory_cached() {
  Cache &c = cache();
  std::lock_guard<std::mutex> lk(c.mu);
  return (int64_t)c.cached;
}

}  // namespace pm
