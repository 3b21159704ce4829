// pm_static.cu -- PageRank for callers that must not allocate GPU memory.
//
// Some hosts cannot call cudaMalloc while they run: a plugin inside a
// process whose memory pool another runtime owns, code running between
// kernels of a captured or latency-critical pipeline, or a caller that has
// handed all device memory to its own allocator.  pm_pagerank_static gives
// them PageRank with Polymer's frontier semantics (the same results as
// pm_pagerank with PM_F32, up to FP32 summation order) while allocating
// nothing: the caller passes the graph and the output in device memory, and
// the working vectors live in one fixed array compiled into this library.
//
// The array is a file-scope __device__ variable, so every GPU that loads the
// library holds its kStaticBytes from load until process exit, and every call
// on that GPU reuses it.  It keeps whatever the last call left in it; each
// call rewrites all of it before use.  Two calls that overlap on the same GPU
// (different streams or host threads without ordering) race on it.
//
// Host code cannot pass the array's name to a kernel: on the host that name
// is a stand-in, not a device address.  The first call on each device looks
// the address up with cudaGetSymbolAddress while that device is current and
// caches it; make that first call before any stream capture.
#include <algorithm>
#include <mutex>

#include "pm_common.cuh"

namespace pm {

// Largest graph the fixed array serves, and its layout: two float vectors of
// kStaticMaxVertices entries (current / next ranks) and two frontier bitmaps.
constexpr int64_t kStaticMaxVertices = 1 << 20;
constexpr int64_t kStaticWords = kStaticMaxVertices / 32;
constexpr size_t kStaticBytes = (size_t)kStaticMaxVertices * 4 * 2 + (size_t)kStaticWords * 4 * 2;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticBytes];

struct StaticView {
  float *p_curr, *p_next;
  uint32_t *f_cur, *f_next;
};

static StaticView static_view(unsigned char *base) {
  StaticView v;
  v.p_curr = reinterpret_cast<float *>(base);
  v.p_next = v.p_curr + kStaticMaxVertices;
  v.f_cur = reinterpret_cast<uint32_t *>(v.p_next + kStaticMaxVertices);
  v.f_next = v.f_cur + kStaticWords;
  return v;
}

// Device address of g_static_scratch, looked up once per device.
static unsigned char *static_scratch_address(int device) {
  static std::mutex mu;
  static unsigned char *addr[64] = {};
  if (device < 0 || device >= 64) fail(PM_ERR_INVALID_ARG, "device index out of range");
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess) fail_cuda(e, "cudaGetSymbolAddress(g_static_scratch)", __FILE__, __LINE__);
    addr[device] = static_cast<unsigned char *>(p);
  }
  return addr[device];
}

// p = 1/n, p_next = 0, every vertex in the frontier.
__global__ void k_static_init(StaticView v, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const float p0 = 1.0f / (float)n;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    v.p_curr[i] = p0;
    v.p_next[i] = 0.0f;
  }
  const int64_t words = (n + 31) / 32;
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < words; w += stride) {
    uint32_t bits = 0xffffffffu;
    if (w == words - 1 && (n & 31)) bits = (1u << (n & 31)) - 1u;
    v.f_cur[w] = bits;
    v.f_next[w] = 0u;
  }
}

// PR_F push (numa-PageRank.C:87-90 / edgeMapDenseForwardOTHER 177-230): a
// warp per frontier source adds p[s]/outdeg(s) into p_next of every
// out-neighbour and marks it in the next frontier.
__global__ void k_static_push(const int32_t *__restrict__ off, const int32_t *__restrict__ idx,
                              int64_t n, float *p_curr, float *p_next, const uint32_t *f_cur,
                              uint32_t *f_next) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t s = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); s < n; s += warps) {
    if (!((f_cur[s >> 5] >> (s & 31)) & 1u)) continue;
    const int32_t e0 = off[s], e1 = off[s + 1];
    if (e1 == e0) continue;
    const float c = p_curr[s] / (float)(e1 - e0);
    for (int32_t e = e0 + lane; e < e1; e += 32) {
      const int32_t d = idx[e];
      atomicAdd(p_next + d, c);
      atomicOr(f_next + (d >> 5), 1u << (d & 31));
    }
  }
}

// PR_Vertex_F then PR_Vertex_Reset (numa-PageRank.C:125-148) on the current
// frontier; clears the current bitmap for its next use as "next".
__global__ void k_static_vertex(int64_t n, float *p_curr, float *p_next, uint32_t *f_cur,
                                float damping, float added) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    if ((f_cur[i >> 5] >> (i & 31)) & 1u) {
      p_next[i] = damping * p_next[i] + added;
      p_curr[i] = 0.0f;
    }
  }
}

__global__ void k_static_clear(uint32_t *bits, int64_t words) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < words; w += stride) bits[w] = 0u;
}

__global__ void k_static_copy(const float *src, float *dst, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) dst[i] = src[i];
}

static void run_pagerank_static(const int32_t *off, const int32_t *idx, int64_t n, int iters,
                                 double damping, float *ranks, cudaStream_t st, int num_sms) {
  int device = 0;
  PM_CUDA(cudaGetDevice(&device));
  StaticView v = static_view(static_scratch_address(device));
  const int64_t words = (n + 31) / 32;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)num_sms * 8));
  PM_LAUNCH(k_static_init, grid, 256, 0, st, v, n);
  const float added = (float)((1.0 - damping) * (1.0 / (double)n));
  for (int it = 0; it < iters; ++it) {
    PM_LAUNCH(k_static_push, (int)std::max<int64_t>(1, std::min<int64_t>((n + 7) / 8, (int64_t)num_sms * 16)),
              256, 0, st, off, idx, n, v.p_curr, v.p_next, v.f_cur, v.f_next);
    PM_LAUNCH(k_static_vertex, grid, 256, 0, st, n, v.p_curr, v.p_next, v.f_cur, (float)damping, added);
    std::swap(v.p_curr, v.p_next);
    std::swap(v.f_cur, v.f_next);
    // the old frontier becomes the next one: clear it
    PM_LAUNCH(k_static_clear, grid, 256, 0, st, v.f_next, words);
  }
  PM_LAUNCH(k_static_copy, grid, 256, 0, st, v.p_curr, ranks, n);
}

}  // namespace pm

// C linkage and export come from the declaration in polymer_b200.h.
pm_status pm_pagerank_static(const int32_t *offsets, const int32_t *edges, int64_t n, int64_t m,
                             int iters, double damping, float *ranks, void *stream) {
  try {
    if (!offsets || !ranks || (m > 0 && !edges))
      pm::fail(PM_ERR_INVALID_ARG, "null offsets/edges/ranks");
    if (n < 1 || n > pm::kStaticMaxVertices)
      pm::fail(PM_ERR_INVALID_ARG, "pm_pagerank_static serves 1 <= n <= " +
                                       std::to_string(pm::kStaticMaxVertices) + " vertices, got " +
                                       std::to_string(n));
    if (m < 0 || m >= (1ll << 31) - 1) pm::fail(PM_ERR_INVALID_ARG, "m must be in [0, 2^31-2]");
    if (iters < 0) pm::fail(PM_ERR_INVALID_ARG, "iters must be >= 0");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int device = 0, sms = 148;
    PM_CUDA(cudaGetDevice(&device));
    PM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    pm::run_pagerank_static(offsets, edges, n, iters, damping, ranks, st, sms);
    PM_CUDA(cudaStreamSynchronize(st));
    pm::set_last_error("");
    return PM_OK;
  } catch (const pm::Failure &f) {
    pm::set_last_error(f.what());
    return f.status;
  }
}
