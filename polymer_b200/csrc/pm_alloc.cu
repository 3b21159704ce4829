// pm_alloc.cu -- the library's device allocator: cudaMalloc behind a cache of
// freed blocks.  A graph build allocates and frees a few dozen buffers of up
// to gigabytes (CSR/CSC copies, sort keys and values, tables, workspaces);
// cudaMalloc / cudaFree of such blocks cost a fraction of a millisecond each
// and cudaFree synchronises the device, so a workload that builds and
// destroys graphs (the end-to-end path) spends tens of milliseconds in them.
// Freed blocks are kept per device and handed out again for requests of
// close size; a block taken from the cache is preceded by a device
// synchronisation, since kernels of its previous owner may still run.
#include <algorithm>
#include <mutex>
#include <vector>

#include "pm_graph.cuh"

namespace pm {

namespace {

struct Block {
  void *p;
  size_t cap;
  int device;
};

struct Cache {
  std::mutex mu;
  std::vector<Block> free;
  size_t cached = 0;
  int64_t limit = -1;  // bytes; -1: a quarter of the device memory, 0: off
  std::vector<int64_t> auto_limit;  // per device
};

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

void release_all(Cache &c) {
  int cur = 0;
  cudaGetDevice(&cur);
  for (const Block &b : c.free) {
    cudaSetDevice(b.device);
    cudaFree(b.p);
  }
  cudaSetDevice(cur);
  (void)cudaGetLastError();
  c.free.clear();
  c.cached = 0;
}

}  // namespace

void *dev_alloc(size_t bytes, size_t *cap, int *device) {
  Cache &c = cache();
  const size_t want = round_cap(bytes);
  int dev = 0;
  PM_CUDA(cudaGetDevice(&dev));
  {
    std::lock_guard<std::mutex> lk(c.mu);
    // the smallest cached block of this device that fits within 25 % (+2 MB)
    int best = -1;
    for (int i = 0; i < (int)c.free.size(); ++i) {
      const Block &b = c.free[i];
      if (b.device != dev || b.cap < want || b.cap > want + want / 4 + (2u << 20)) continue;
      if (best < 0 || b.cap < c.free[best].cap) best = i;
    }
    if (best >= 0) {
      const Block b = c.free[best];
      c.free.erase(c.free.begin() + best);
      c.cached -= b.cap;
      PM_CUDA(cudaDeviceSynchronize());
      *cap = b.cap;
      *device = dev;
      return b.p;
    }
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
      c.free.push_back(Block{p, cap, dev});
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

int64_t memory_cached() {
  Cache &c = cache();
  std::lock_guard<std::mutex> lk(c.mu);
  return (int64_t)c.cached;
}

}  // namespace pm
