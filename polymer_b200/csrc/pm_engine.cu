// pm_engine.cu -- frontier plumbing kernels and error handling of the engine.
#include <atomic>
#include <cstdarg>
#include <cstdio>

#include "polymer.cuh"

namespace pm {

static std::atomic<long long> g_launches{0};

void count_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long launches(bool reset) {
  return reset ? g_launches.exchange(0) : g_launches.load();
}

[[noreturn]] void fail(pm_status s, const std::string &msg) { throw Failure(s, msg); }

[[noreturn]] void fail_cuda(cudaError_t e, const char *what, const char *file, int line) {
  char buf[512];
  snprintf(buf, sizeof buf, "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
  fail(e == cudaErrorMemoryAllocation ? PM_ERR_OOM
       : e == cudaErrorNoDevice       ? PM_ERR_NO_DEVICE
                                      : PM_ERR_CUDA,
       buf);
}

__global__ void k_bits_to_queue(int32_t n, const int32_t *__restrict__ out_off,
                                const uint32_t *__restrict__ bits, int32_t *__restrict__ queue,
                                Counters *cnt, const RoundGate *gate) {
  if (gate && (!gate->active || gate->dense)) return;  // not a sparse round
  const int lane = lane_id();
  const int64_t nw = ((int64_t)n + 31) / 32;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  unsigned long long my_edges = 0;
  // A warp takes 32 consecutive words; each lane one word.
  for (int64_t wb = ((int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32; wb < nw;
       wb += warps * 32) {
    int64_t wi = wb + lane;
    uint32_t word = wi < nw ? bits[wi] : 0u;
    if (wi == nw - 1 && (n & 31)) word &= (1u << (n & 31)) - 1u;
    int c = __popc(word);
    int tot;
    int pre = warp_excl_scan(c, &tot);
    unsigned long long base = 0;
    if (lane == 0 && tot) base = atomicAdd(&cnt->size, (unsigned long long)tot);
    base = __shfl_sync(0xffffffffu, base, 0);
    int k = 0;
    while (word) {
      int b = __ffs(word) - 1;
      word &= word - 1;
      int v = (int)(wi * 32 + b);
      queue[base + pre + k++] = v;
      my_edges += __ldg(out_off + v + 1) - __ldg(out_off + v);
    }
  }
  my_edges = warp_sum(my_edges);
  if (lane == 0 && my_edges) atomicAdd(&cnt->edges, my_edges);
}

__global__ void k_queue_to_bits(const int32_t *__restrict__ queue, int32_t size,
                                uint32_t *__restrict__ bits) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < size; i += stride) {
    int v = queue[i];
    atomicOr(bits + (v >> 5), 1u << (v & 31));
  }
}

__global__ void k_bits_stats(int32_t n, const int32_t *__restrict__ out_off,
                             const uint32_t *__restrict__ bits, Counters *cnt) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  unsigned long long my_size = 0, my_edges = 0;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
    if (test_bit(bits, (int)v)) {
      my_size++;
      my_edges += __ldg(out_off + v + 1) - __ldg(out_off + v);
    }
  }
  my_size = warp_sum(my_size);
  my_edges = warp_sum(my_edges);
  if (lane_id() == 0 && my_size) {
    atomicAdd(&cnt->size, my_size);
    atomicAdd(&cnt->edges, my_edges);
  }
}

__global__ void k_set_single(uint32_t *bits, int32_t *queue, int32_t v) {
  bits[v >> 5] = 1u << (v & 31);
  queue[0] = v;
}

__global__ void k_set_all(uint32_t *bits, int32_t n) {
  const int64_t nw = ((int64_t)n + 31) / 32;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nw; i += stride) {
    uint32_t w = 0xffffffffu;
    if (i == nw - 1 && (n & 31)) w = (1u << (n & 31)) - 1u;
    bits[i] = w;
  }
}

void subset_recount(Engine &E, VertexSubset &s) {
  PM_CUDA(cudaMemsetAsync(E.d_cnt + 2, 0, sizeof(Counters), E.stream));
  PM_LAUNCH(k_bits_stats, E.grid_for(s.n, 256, 8), 256, 0, E.stream, s.n, E.g.out.off, s.bits,
            E.d_cnt + 2);
  const Counters *h = E.read_counters();
  s.size = (int64_t)h[2].size;
  s.edges = (int64_t)h[2].edges;
}

void subset_to_queue(Engine &E, VertexSubset &s) {
  if (s.has_queue) return;
  PM_CUDA(cudaMemsetAsync(E.d_cnt + 2, 0, sizeof(Counters), E.stream));
  int64_t warps = (s.words() + 31) / 32;
  PM_LAUNCH(k_bits_to_queue, E.grid_for(warps * 32, 256, 8), 256, 0, E.stream, s.n, E.g.out.off,
            s.bits, s.queue, E.d_cnt + 2);
  s.has_queue = true;
}

void subset_single(Engine &E, VertexSubset &s, int32_t v) {
  PM_CUDA(cudaMemsetAsync(s.bits, 0, s.words() * 4, E.stream));
  PM_LAUNCH(k_set_single, 1, 1, 0, E.stream, s.bits, s.queue, v);
  int32_t o[2];
  PM_CUDA(cudaMemcpyAsync(o, E.g.out.off + v, sizeof o, cudaMemcpyDeviceToHost, E.stream));
  PM_CUDA(cudaStreamSynchronize(E.stream));
  s.has_queue = true;
  s.size = 1;
  s.edges = o[1] - o[0];
}

void subset_all(Engine &E, VertexSubset &s) {
  PM_LAUNCH(k_set_all, E.grid_for(s.words(), 256, 4), 256, 0, E.stream, s.bits, s.n);
  s.has_queue = false;
  s.size = s.n;
  s.edges = E.g.m;
}

void subset_clear(Engine &E, VertexSubset &s) {
  PM_CUDA(cudaMemsetAsync(s.bits, 0, s.words() * 4, E.stream));
  s.has_queue = true;
  s.size = 0;
  s.edges = 0;
}

}  // namespace pm
