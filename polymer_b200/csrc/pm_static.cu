// pm_static.cu -- PageRank for callers that must not allocate GPU memory.
//
// Some hosts cannot call cudaMalloc while they run: a plugin inside a
// process whose memory pool another runtime owns, code running between
// kernels of a latency-critical pipeline, or a caller that has handed all
// device memory to its own allocator.  pm_pagerank_static gives them
// PageRank with Polymer's frontier semantics (the same results as
// pm_pagerank with PM_F32, up to FP32 summation order) while allocating
// nothing: the caller passes the graph and the output in device memory, and
// the working vectors live in one fixed array compiled into this library.
//
// The array is a file-scope __device__ variable of kStaticBytes.  With
// CUDA's lazy module loading (the default) the device memory behind it is
// reserved when this file's module is first used on a device, which is the
// first call of pm_pagerank_static there: make that call before handing the
// rest of the device's memory to another allocator.  From then on it stays
// reserved until the process exits, and every call on that GPU reuses it.
// It keeps whatever the last call left in it; each call clears the status
// word and rewrites the vectors before use.  Two calls that overlap on the
// same GPU (different streams or host threads without ordering) race on it.
//
// Host code cannot pass the array's name to a kernel: on the host that name
// is a stand-in, not a device address.  The first call on each device looks
// the address up with cudaGetSymbolAddress while that device is current and
// caches it; make that first call before any stream capture.
//
// The CSR comes straight from the caller, without the validation a graph
// handle gets at creation, so each call first checks it on the device
// (offsets monotone within [0, m], offsets[0] == 0, offsets[n] == m, every
// id in [0, n), no self loop) and returns PM_ERR_BAD_GRAPH, without running
// PageRank, when a check fails.  The push kernel also skips any id outside
// [0, n), so no access leaves the caller's arrays or the fixed array.
#include <algorithm>
#include <mutex>

#include "pm_common.cuh"

namespace pm {

// Largest graph the fixed array serves, and its layout: two float vectors of
// kStaticMaxVertices entries (current / next ranks), two frontier bitmaps and
// a 256-byte tail whose first word is the call's status (kBad* bits).
constexpr int64_t kStaticMaxVertices = 1 << 20;
constexpr int64_t kStaticWords = kStaticMaxVertices / 32;
constexpr size_t kStaticStatusOffset = (size_t)kStaticMaxVertices * 4 * 2 + (size_t)kStaticWords * 4 * 2;
constexpr size_t kStaticBytes = kStaticStatusOffset + 256;
constexpr unsigned kBadOffsets = 1u;    // offsets not monotone or outside [0, m]
constexpr unsigned kBadEnds = 2u;       // offsets[0] != 0 or offsets[n] != m
constexpr unsigned kBadId = 4u;         // an edge id outside [0, n)
constexpr unsigned kSelfLoop = 8u;      // an edge s -> s

static __device__ __align__(256) unsigned char g_static_scratch[kStaticBytes];

struct StaticView {
  float *p_curr, *p_next;
  uint32_t *f_cur, *f_next;
  unsigned *status;
};

static StaticView static_view(unsigned char *base) {
  StaticView v;
  v.p_curr = reinterpret_cast<float *>(base);
  v.p_next = v.p_curr + kStaticMaxVertices;
  v.f_cur = reinterpret_cast<uint32_t *>(v.p_next + kStaticMaxVertices);
  v.f_next = v.f_cur + kStaticWords;
  v.status = reinterpret_cast<unsigned *>(base + kStaticStatusOffset);
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

// The caller's CSR, checked before use: a warp per vertex reads its two
// offsets and, when they are sane, its edges (every read stays inside
// offsets[0..n] and edges[0..m)).
__global__ void k_static_validate(const int32_t *__restrict__ off, const int32_t *__restrict__ idx, int64_t n,
                                  int64_t m, unsigned *status) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  unsigned bad = 0;
  if (blockIdx.x == 0 && threadIdx.x == 0 && (off[0] != 0 || (int64_t)off[n] != m)) bad |= kBadEnds;
  for (int64_t s = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); s < n; s += warps) {
    const int32_t e0 = off[s], e1 = off[s + 1];
    if (e0 < 0 || e1 < e0 || (int64_t)e1 > m) {
      bad |= kBadOffsets;
      continue;
    }
    for (int32_t e = e0 + lane; e < e1; e += 32) {
      const int32_t d = idx[e];
      if (d < 0 || (int64_t)d >= n) bad |= kBadId;
      else if (d == (int32_t)s) bad |= kSelfLoop;
    }
  }
  if (bad) atomicOr(status, bad);
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
// Ids outside [0, n) are skipped and flagged (the validation above has
// already refused such a CSR; this keeps every access in bounds regardless).
__global__ void k_static_push(const int32_t *__restrict__ off, const int32_t *__restrict__ idx,
                              int64_t n, float *p_curr, float *p_next, const uint32_t *f_cur,
                              uint32_t *f_next, unsigned *status) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t s = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); s < n; s += warps) {
    if (!((f_cur[s >> 5] >> (s & 31)) & 1u)) continue;
    const int32_t e0 = off[s], e1 = off[s + 1];
    if (e1 == e0) continue;
    const float c = p_curr[s] / (float)(e1 - e0);
    for (int32_t e = e0 + lane; e < e1; e += 32) {
      const int32_t d = idx[e];
      if (d < 0 || (int64_t)d >= n) {
        atomicOr(status, kBadId);
        continue;
      }
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

static std::string static_bad_graph_text(unsigned bad) {
  return std::string("pm_pagerank_static: invalid CSR:") + (bad & kBadOffsets ? " offsets not monotone in [0, m]" : "") +
         (bad & kBadEnds ? " offsets[0] != 0 or offsets[n] != m" : "") +
         (bad & kBadId ? " edge id out of range" : "") + (bad & kSelfLoop ? " self loop" : "");
}

static void run_pagerank_static(const int32_t *off, const int32_t *idx, int64_t n, int64_t m, int iters,
                                 double damping, float *ranks, cudaStream_t st, int num_sms) {
  int device = 0;
  PM_CUDA(cudaGetDevice(&device));
  StaticView v = static_view(static_scratch_address(device));
  const int64_t words = (n + 31) / 32;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)num_sms * 8));
  const int warp_grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 7) / 8, (int64_t)num_sms * 16));
  // the status word keeps the previous call's value: clear it, check the
  // CSR, and read the verdict into a host variable before any PageRank work
  PM_CUDA(cudaMemsetAsync(v.status, 0, sizeof(unsigned), st));
  PM_LAUNCH(k_static_validate, warp_grid, 256, 0, st, off, idx, n, m, v.status);
  unsigned bad = 0;
  PM_CUDA(cudaMemcpyAsync(&bad, v.status, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  PM_CUDA(cudaStreamSynchronize(st));
  if (bad) fail(PM_ERR_BAD_GRAPH, static_bad_graph_text(bad));
  PM_LAUNCH(k_static_init, grid, 256, 0, st, v, n);
  const float added = (float)((1.0 - damping) * (1.0 / (double)n));
  for (int it = 0; it < iters; ++it) {
    PM_LAUNCH(k_static_push, warp_grid, 256, 0, st, off, idx, n, v.p_curr, v.p_next, v.f_cur, v.f_next,
              v.status);
    PM_LAUNCH(k_static_vertex, grid, 256, 0, st, n, v.p_curr, v.p_next, v.f_cur, (float)damping, added);
    std::swap(v.p_curr, v.p_next);
    std::swap(v.f_cur, v.f_next);
    // the old frontier becomes the next one: clear it
    PM_LAUNCH(k_static_clear, grid, 256, 0, st, v.f_next, words);
  }
  PM_LAUNCH(k_static_copy, grid, 256, 0, st, v.p_curr, ranks, n);
  PM_CUDA(cudaMemcpyAsync(&bad, v.status, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  PM_CUDA(cudaStreamSynchronize(st));
  if (bad) fail(PM_ERR_BAD_GRAPH, static_bad_graph_text(bad));
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
    pm::run_pagerank_static(offsets, edges, n, m, iters, damping, ranks, st, sms);
    pm::set_last_error("");
    return PM_OK;
  } catch (const pm::Failure &f) {
    pm::set_last_error(f.what());
    return f.status;
  }
}
