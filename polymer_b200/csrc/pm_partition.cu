// pm_partition.cu -- 1D vertex partition of one graph over several
// processes, one per GPU: the reference's NUMA split (partitionByDegree,
// polymer.h:131-192; graphFilter / graphFilter2Direction, 346-497), where
// each node keeps the edges whose destination it owns and every node sees
// the whole frontier.
//
// The vertex ranges are cut where the in-edges plus a per-row term (the pull
// work) reach equal shares, on 32-vertex boundaries, as the reference
// balances its shards by in-degree.  Rank r owns the range [lo, hi) and
// holds the edges whose destination lies in it, with global vertex ids: a
// CSR over all n sources (sparse pushes from the global frontier reach only
// its own destinations) and a CSC whose rows outside the range are empty
// (pulls visit only its own rows).  Vertex state is replicated; after every
// pass each rank's range of the state the next pass reads (contributions,
// x, labels, distances, the frontier bitmap) is gathered into every rank's
// copy by the handle's exchange function -- an allgather the caller
// supplies (NCCL through torch.distributed in the Python binding), so the
// library links no communication library.
#include <algorithm>

#include <cub/cub.cuh>

#include "pm_graph.cuh"

namespace pm {

namespace {

__global__ void k_in_degrees(const int32_t *idx, int64_t m, int32_t *deg) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += stride) atomicAdd(deg + idx[e], 1);
}

// Interior bounds: bound r (1 <= r < nranks) is the first vertex v whose work
// prefix in_pre[v] + kRowWork * v reaches r / nranks of the total, rounded
// down to a multiple of 32.  in_pre has n + 1 entries (exclusive sums).
__global__ void k_bounds(const int64_t *in_pre, int64_t n, int nranks, int64_t *bounds) {
  const int r = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (r > nranks) return;
  if (r == 0 || r == nranks) {
    bounds[r] = r == 0 ? 0 : n;
    return;
  }
  const double total = (double)in_pre[n] + (double)kRowWork * (double)n;
  const double target = total * r / nranks;
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if ((double)in_pre[mid] + (double)kRowWork * (double)mid < target) lo = mid + 1; else hi = mid;
  }
  bounds[r] = lo & ~31ll;
}

__global__ void k_range_flags(const int32_t *idx, int64_t m, int32_t lo, int32_t hi, int32_t *keep) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += stride)
    keep[e] = idx[e] >= lo && idx[e] < hi;
}

// new_off[r] = kept edges before old off[r]; pre has m + 1 entries.
__global__ void k_remap(const int32_t *off, const int32_t *pre, int64_t n, int32_t *noff) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v <= n; v += stride) noff[v] = pre[off[v]];
}

__global__ void k_compact(const int32_t *val, const int32_t *keep, const int32_t *pre, int64_t m, int32_t *out) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += stride)
    if (keep[e]) out[pre[e]] = val[e];
}

int grid_for(int64_t threads) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((threads + 255) / 256, 148 * 32));
}

// Degree-balanced bounds of the CSR in g (partitionByDegree by in-degree).
std::vector<int64_t> balanced_bounds(pm_graph *g, int nranks) {
  cudaStream_t st = g->E.stream;
  const int64_t n = g->n, m = g->m;
  DevBuf deg((size_t)(n + 1) * 4), pre((size_t)(n + 1) * 8), db((size_t)(nranks + 1) * 8);
  PM_CUDA(cudaMemsetAsync(deg.p, 0, (size_t)(n + 1) * 4, st));
  if (m) PM_LAUNCH(k_in_degrees, grid_for(m), 256, 0, st, g->out.idx.as<int32_t>(), m, deg.as<int32_t>());
  size_t tmp = 0;
  PM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, deg.as<int32_t>(), pre.as<int64_t>(), (int)(n + 1), st));
  DevBuf tb(std::max<size_t>(tmp, 16));
  PM_CUDA(cub::DeviceScan::ExclusiveSum(tb.p, tmp, deg.as<int32_t>(), pre.as<int64_t>(), (int)(n + 1), st));
  PM_LAUNCH(k_bounds, 1, ((nranks + 1 + 31) / 32) * 32, 0, st, pre.as<int64_t>(), n, nranks, db.as<int64_t>());
  std::vector<int64_t> b(nranks + 1);
  PM_CUDA(cudaMemcpyAsync(b.data(), db.p, (size_t)(nranks + 1) * 8, cudaMemcpyDeviceToHost, st));
  PM_CUDA(cudaStreamSynchronize(st));
  for (int r = 1; r <= nranks; ++r) b[r] = std::max(b[r], b[r - 1]);  // monotone after the rounding
  return b;
}

}  // namespace

void restrict_to_partition(pm_graph *g, int rank, int nranks, DevBuf *w) {
  cudaStream_t st = g->E.stream;
  const int64_t n = g->n, m = g->m;
  std::vector<int64_t> b = balanced_bounds(g, nranks);
  g->is_part = true;
  g->part_rank = rank;
  g->part_count = nranks;
  g->part_bounds = b;
  g->part_wbounds.resize(nranks + 1);
  for (int r = 0; r <= nranks; ++r) g->part_wbounds[r] = (b[r] + 31) / 32;  // interior bounds are whole words
  const int64_t lo = b[rank], hi = b[rank + 1];
  g->part_lo = lo;
  g->part_hi = hi;
  g->E.host_steps = true;
  // the whole graph's offsets: global out-degrees (PageRank's contributions)
  g->glob_off.alloc((size_t)(n + 1) * 4);
  PM_CUDA(cudaMemcpyAsync(g->glob_off.p, g->out.off.p, (size_t)(n + 1) * 4, cudaMemcpyDeviceToDevice, st));
  if (m == 0) {
    PM_CUDA(cudaStreamSynchronize(st));
    return;
  }
  // keep[m] = 0 closes the scan: pre[m] is the kept count
  DevBuf keep((size_t)(m + 1) * 4), pre((size_t)(m + 1) * 4);
  PM_CUDA(cudaMemsetAsync(keep.as<int32_t>() + m, 0, 4, st));
  PM_LAUNCH(k_range_flags, grid_for(m), 256, 0, st, g->out.idx.as<int32_t>(), m, (int32_t)lo, (int32_t)hi,
            keep.as<int32_t>());
  size_t tmp = 0;
  PM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, keep.as<int32_t>(), pre.as<int32_t>(), (int)(m + 1), st));
  DevBuf tb(std::max<size_t>(tmp, 16));
  PM_CUDA(cub::DeviceScan::ExclusiveSum(tb.p, tmp, keep.as<int32_t>(), pre.as<int32_t>(), (int)(m + 1), st));
  int32_t m_new = 0;
  PM_CUDA(cudaMemcpyAsync(&m_new, pre.as<int32_t>() + m, 4, cudaMemcpyDeviceToHost, st));
  PM_CUDA(cudaStreamSynchronize(st));
  DevBuf noff((size_t)(n + 1) * 4), nidx((size_t)std::max<int32_t>(m_new, 1) * 4);
  PM_LAUNCH(k_remap, grid_for(n + 1), 256, 0, st, g->out.off.as<int32_t>(), pre.as<int32_t>(), n,
            noff.as<int32_t>());
  PM_LAUNCH(k_compact, grid_for(m), 256, 0, st, g->out.idx.as<int32_t>(), keep.as<int32_t>(), pre.as<int32_t>(),
            m, nidx.as<int32_t>());
  if (w && w->p) {
    DevBuf nw((size_t)std::max<int32_t>(m_new, 1) * 4);
    PM_LAUNCH(k_compact, grid_for(m), 256, 0, st, w->as<int32_t>(), keep.as<int32_t>(), pre.as<int32_t>(), m,
              nw.as<int32_t>());
    *w = std::move(nw);
  }
  g->out.off = std::move(noff);
  g->out.idx = std::move(nidx);
  g->m = m_new;
  PM_CUDA(cudaStreamSynchronize(st));
}

void part_exchange(pm_graph *g, void *buf, size_t elem_bytes) {
  if (!g->is_part || g->part_count == 1) return;
  if (!g->part_fn) fail(PM_ERR_INVALID_ARG, "partition graph without an exchange function (pm_graph_set_exchange)");
  const int rc = g->part_fn(g->part_user, buf, (int64_t)elem_bytes, g->part_bounds.data(), g->part_count,
                            (void *)g->E.stream);
  if (rc != 0) fail(PM_ERR_CUDA, "partition exchange function returned " + std::to_string(rc));
}

void part_exchange_bits(pm_graph *g, uint32_t *bits) {
  if (!g->is_part || g->part_count == 1) return;
  if (!g->part_fn) fail(PM_ERR_INVALID_ARG, "partition graph without an exchange function (pm_graph_set_exchange)");
  const int rc = g->part_fn(g->part_user, bits, 4, g->part_wbounds.data(), g->part_count, (void *)g->E.stream);
  if (rc != 0) fail(PM_ERR_CUDA, "partition exchange function returned " + std::to_string(rc));
}

void part_round(pm_graph *g, VertexSubset &next) {
  if (!g->is_part) return;
  if (g->part_count > 1) {
    if (!g->part_fn) fail(PM_ERR_INVALID_ARG, "partition graph without an exchange function (pm_graph_set_exchange)");
    const int rc = g->part_fn(g->part_user, next.bits, 4, g->part_wbounds.data(), g->part_count, (void *)g->E.stream);
    if (rc != 0) fail(PM_ERR_CUDA, "partition exchange function returned " + std::to_string(rc));
  }
  next.has_queue = false;
  subset_recount(g->E, next);
}

}  // namespace pm
