// pm_hubs.cu -- the hub cache of the FP32 PageRank pull.
//
// Every edge of a pull gathers its source's contribution, a 4-byte load at a
// scattered address; the SM's load pipe serves about one scattered address
// per cycle, which bounds the pass.  A source is gathered once per out-edge,
// so the sources of highest out-degree take a large share of the gathers
// (the top 16384 sources: 29 % of the edges of a scale-24 R-MAT).
// Their contributions are copied once per pass into a compact array, each
// SM loads it into shared memory, and the pull reads those sources from
// there: the CSC source array is kept a second time with the cached sources
// written as ~slot.  The values are copies, so the sums and results are the
// same bit for bit.
#include <algorithm>
#include <vector>

#include <cub/cub.cuh>

#include "pm_graph.cuh"

namespace pm {

namespace {

constexpr int kDegBins = 1 << 16;  // out-degrees from kDegBins - 1 up share the last bin

__global__ void k_deg_hist(const int32_t *off, int64_t n, unsigned int *hist) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
    atomicAdd(hist + min(off[v + 1] - off[v], kDegBins - 1), 1u);
}

__global__ void k_hub_flags(const int32_t *off, int64_t n, int32_t t, int32_t *flag) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
    flag[v] = off[v + 1] - off[v] >= t;
}

__global__ void k_hub_slots(const int32_t *flag, const int32_t *pre, int64_t n, int32_t *slot_of, int32_t *ids) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
    slot_of[v] = flag[v] ? pre[v] : -1;
    if (flag[v]) ids[pre[v]] = (int32_t)v;
  }
}

__global__ void k_hub_tag(const int32_t *idx, int64_t m, const int32_t *slot_of, int32_t *tagged) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += stride) {
    const int32_t s = idx[e], k = slot_of[s];
    tagged[e] = k >= 0 ? ~k : s;
  }
}

__global__ void k_hub_vals(const int32_t *ids, int count, const float *x, float *vals) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) vals[i] = x[ids[i]];
}

int grid_for(int64_t threads) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((threads + 255) / 256, 148 * 32));
}

}  // namespace

void ensure_hubs(pm_graph *g) {
  const int want = std::min(g->E.tune.hub_cache, kHubMax);
  if (g->hub_for == want) return;
  g->hub_count = 0;
  g->hub_for = want;
  const int64_t n = g->n, m = g->m;
  if (want <= 0 || m == 0) return;
  cudaStream_t st = g->E.stream;
  // the smallest degree t >= 2 with at most `want` sources of degree >= t
  DevBuf hist((size_t)kDegBins * 4);
  PM_CUDA(cudaMemsetAsync(hist.p, 0, (size_t)kDegBins * 4, st));
  PM_LAUNCH(k_deg_hist, grid_for(n), 256, 0, st, g->out.off.as<int32_t>(), n, hist.as<unsigned int>());
  std::vector<unsigned int> h(kDegBins);
  PM_CUDA(cudaMemcpyAsync(h.data(), hist.p, (size_t)kDegBins * 4, cudaMemcpyDeviceToHost, st));
  PM_CUDA(cudaStreamSynchronize(st));
  int64_t count = 0;
  int t = kDegBins;  // no hubs unless a threshold fits
  for (int d = kDegBins - 1; d >= 2; --d) {
    if (count + h[d] > (uint64_t)want) break;
    count += h[d];
    t = d;
  }
  if (count == 0) return;
  DevBuf flag((size_t)(n + 1) * 4), pre((size_t)(n + 1) * 4), slot_of((size_t)n * 4);
  PM_CUDA(cudaMemsetAsync(flag.as<int32_t>() + n, 0, 4, st));
  PM_LAUNCH(k_hub_flags, grid_for(n), 256, 0, st, g->out.off.as<int32_t>(), n, t, flag.as<int32_t>());
  size_t tmp = 0;
  PM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, flag.as<int32_t>(), pre.as<int32_t>(), (int)(n + 1), st));
  DevBuf tb(std::max<size_t>(tmp, 16));
  PM_CUDA(cub::DeviceScan::ExclusiveSum(tb.p, tmp, flag.as<int32_t>(), pre.as<int32_t>(), (int)(n + 1), st));
  g->hub_ids.alloc((size_t)count * 4);
  g->hub_vals.alloc((size_t)count * 4);
  g->hub_idx.alloc((size_t)m * 4);
  PM_LAUNCH(k_hub_slots, grid_for(n), 256, 0, st, flag.as<int32_t>(), pre.as<int32_t>(), n, slot_of.as<int32_t>(),
            g->hub_ids.as<int32_t>());
  PM_LAUNCH(k_hub_tag, grid_for(m), 256, 0, st, g->E.g.in.idx, m, slot_of.as<int32_t>(), g->hub_idx.as<int32_t>());
  PM_CUDA(cudaStreamSynchronize(st));
  g->hub_count = (int)count;
}

void hub_values(pm_graph *g, const float *x) {
  PM_LAUNCH(k_hub_vals, (g->hub_count + 255) / 256, 256, 0, g->E.stream, g->hub_ids.as<int32_t>(), g->hub_count, x,
            g->hub_vals.as<float>());
}

}  // namespace pm
