// pm_graph.cu -- device graph construction: validation, self-loop removal,
// CSC transpose, warp-group and heavy-chunk tables, the seeded R-MAT
// generator and synthetic weights.  Off the hot path; sorts and scans use
// CUB (library code) as plain primitives.
#include <cub/cub.cuh>

#include <cmath>

#include "pm_graph.cuh"

namespace pm {

static int grid1d(int64_t threads, int block = 256) {
  int64_t b = (threads + block - 1) / block;
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 32));
}

#define GRID_STRIDE(i, count)                                                       \
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (count);     \
       i += (int64_t)gridDim.x * blockDim.x)

// ---- validation -----------------------------------------------------------
__global__ void k_validate(const int32_t *off, const int32_t *idx, int64_t n, int64_t m,
                           unsigned int *err, unsigned int *self_loops) {
  GRID_STRIDE(v, n) {
    int32_t a = off[v], b = off[v + 1];
    if (a > b || a < 0 || b > m) atomicOr(err, 1u);
  }
  GRID_STRIDE(e, m) {
    int32_t d = idx[e];
    if (d < 0 || d >= n) atomicOr(err, 2u);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && (off[0] != 0 || off[n] != m)) atomicOr(err, 4u);
  (void)self_loops;
}


// Source row of every CSR edge: each non-empty row marks its first edge with
// its id, and an inclusive max-scan carries the id over the row's edges
// (rows ascend with the edge index).  Six times faster than a binary search
// of the offsets per edge at scale 24.
__global__ void k_row_heads(const int32_t *off, int64_t n, int32_t *heads) {
  GRID_STRIDE(r, n) if (off[r + 1] > off[r]) heads[off[r]] = (int32_t)r;
}
struct MaxI32 {
  __device__ __forceinline__ int32_t operator()(int32_t a, int32_t b) const { return a > b ? a : b; }
};
static void fill_edge_src(const int32_t *off, int64_t n, int64_t m, int32_t *src, cudaStream_t st) {
  if (m == 0) return;
  DevBuf heads((size_t)m * 4);
  PM_CUDA(cudaMemsetAsync(heads.p, 0, (size_t)m * 4, st));
  PM_LAUNCH(k_row_heads, grid1d(n), 256, 0, st, off, n, heads.as<int32_t>());
  size_t tmp = 0;
  PM_CUDA(cub::DeviceScan::InclusiveScan(nullptr, tmp, heads.as<int32_t>(), src, MaxI32(), (int)m, st));
  DevBuf tb(std::max<size_t>(tmp, 16));
  PM_CUDA(cub::DeviceScan::InclusiveScan(tb.p, tmp, heads.as<int32_t>(), src, MaxI32(), (int)m, st));
  PM_CUDA(cudaStreamSynchronize(st));  // the temporaries are freed on return
}

__global__ void k_self_flags(const int32_t *src, const int32_t *idx, int64_t m, int32_t *keep,
                             unsigned int *count) {
  unsigned int c = 0;
  GRID_STRIDE(e, m) {
    int32_t k = src[e] != idx[e];
    keep[e] = k;
    c += !k;
  }
  if (c) atomicAdd(count, c);
}

// new_off[r] = number of kept edges before old off[r]; pre has m+1 entries.
__global__ void k_remap_offsets(const int32_t *off, const int32_t *pre, int64_t n, int32_t *noff) {
  GRID_STRIDE(v, n + 1) noff[v] = pre[off[v]];
}

__global__ void k_compact_edges(const int32_t *idx, const int32_t *keep, const int32_t *pre,
                                int64_t m, int32_t *nidx) {
  GRID_STRIDE(e, m) if (keep[e]) nidx[pre[e]] = idx[e];
}

// ---- CSC ----------------------------------------------------------------
__global__ void k_iota(int32_t *a, int64_t count) { GRID_STRIDE(i, count) a[i] = (int32_t)i; }

__global__ void k_gather_src(const int32_t *src, const int32_t *eid, int64_t m, int32_t *tidx) {
  GRID_STRIDE(p, m) tidx[p] = src[eid[p]];
}

// toff[v] = first position of key v in the sorted destination array.
__global__ void k_lower_bound_offsets(const int32_t *keys, int64_t m, int64_t n, int32_t *toff) {
  GRID_STRIDE(v, n + 1) {
    int64_t lo = 0, hi = m;
    while (lo < hi) {
      int64_t mid = (lo + hi) >> 1;
      if (keys[mid] < v) lo = mid + 1; else hi = mid;
    }
    toff[v] = (int32_t)lo;
  }
}

// Symmetric graph: CSC slot p (row d, neighbour s) -> CSR edge s->d.

// ---- load-balance tables ---------------------------------------------------
// Warp groups split the merge path of rows and edges over the rows [r0, r1)
// (all rows, or a partition's own range; r0 a multiple of 32): with the work
// key key(r) = off[r] - off[r0] + kRowWork * (r - r0) (strictly increasing),
// gstart[g] is the first row whose key is >= g * kGroupWork, rounded down to
// a multiple of 32; gstart[G] = r1.  A group therefore holds about
// kGroupWork units of edges plus rows, however the degrees are distributed.
__global__ void k_group_starts(const int32_t *off, int64_t r0, int64_t r1, int32_t G, int32_t *gstart) {
  GRID_STRIDE(g, (int64_t)G + 1) {
    if (g == G) { gstart[g] = (int32_t)r1; continue; }
    const int64_t target = g * (int64_t)kGroupWork, base = off[r0];
    int64_t lo = r0, hi = r1;
    while (lo < hi) {
      int64_t mid = (lo + hi) >> 1;
      if ((int64_t)off[mid] - base + (int64_t)kRowWork * (mid - r0) < target) lo = mid + 1; else hi = mid;
    }
    gstart[g] = (int32_t)(std::min<int64_t>(lo, r1) & ~31ll);
  }
}

__global__ void k_heavy_counts(const int32_t *off, int64_t n, int32_t heavy_deg, int32_t *nch,
                               int32_t *maxdeg) {
  int32_t md = 0;
  GRID_STRIDE(v, n) {
    int32_t d = off[v + 1] - off[v];
    nch[v] = d > heavy_deg ? (d + kChunkEdges - 1) / kChunkEdges : 0;
    md = max(md, d);
  }
  atomicMax(maxdeg, md);
}

__global__ void k_heavy_rows(const int32_t *nch, const int32_t *first, int64_t n, int32_t *hrow) {
  GRID_STRIDE(v, n) {
    int32_t c = nch[v];
    for (int32_t k = 0; k < c; ++k) hrow[first[v] + k] = (int32_t)v;
  }
}

template <class T>
__global__ void k_gather(const T *src, const int32_t *perm, int64_t count, T *dst) {
  GRID_STRIDE(i, count) dst[i] = src[perm[i]];
}

// ---- R-MAT -----------------------------------------------------------------
// Quadrant thresholds on a 24-bit draw: a = .57, a+b = .76, a+b+c = .95.
constexpr uint32_t kRmatA = 9563013u, kRmatAB = 12750684u, kRmatABC = 15938355u;

__global__ void k_rmat_keys(int scale, uint64_t seed, int64_t draws, int symmetric,
                            uint64_t *keys) {
  const uint64_t sentinel = (uint64_t)1 << (32 + scale);  // sorts after every edge
  GRID_STRIDE(k, draws) {
    uint32_t s = 0, d = 0;
    for (int l = 0; l < scale; ++l) {
      uint32_t u = (uint32_t)(hash64(seed, (uint64_t)k * (uint64_t)scale + (uint64_t)l) >> 40);
      uint32_t row = u >= kRmatAB;
      uint32_t col = (u >= kRmatA && u < kRmatAB) || u >= kRmatABC;
      s = (s << 1) | row;
      d = (d << 1) | col;
    }
    bool loop = s == d;
    keys[k] = loop ? sentinel : (((uint64_t)s << 32) | d);
    if (symmetric) keys[draws + k] = loop ? sentinel : (((uint64_t)d << 32) | s);
  }
}

__global__ void k_keys_to_csr_idx(const uint64_t *keys, int64_t m, int32_t *idx) {
  GRID_STRIDE(e, m) idx[e] = (int32_t)(keys[e] & 0xffffffffull);
}

__global__ void k_keys_offsets(const uint64_t *keys, int64_t m, int64_t n, int32_t *off) {
  GRID_STRIDE(v, n + 1) {
    uint64_t target = (uint64_t)v << 32;
    int64_t lo = 0, hi = m;
    while (lo < hi) {
      int64_t mid = (lo + hi) >> 1;
      if (keys[mid] < target) lo = mid + 1; else hi = mid;
    }
    off[v] = (int32_t)lo;
  }
}

// Synthetic weights: the rules of the oracle (pmo_weight_int / _unit).
__global__ void k_weights_i32(const int32_t *src, const int32_t *idx, int64_t m, uint64_t seed,
                              int32_t wmax, int32_t *w) {
  GRID_STRIDE(e, m) {
    uint32_t u = (uint32_t)src[e], v = (uint32_t)idx[e];
    uint32_t a = u < v ? u : v, b = u < v ? v : u;
    w[e] = 1 + (int32_t)((hash64(seed, ((uint64_t)a << 32) | b) >> 32) % (uint64_t)wmax);
  }
}
__global__ void k_weights_f32(const int32_t *src, const int32_t *idx, int64_t m, uint64_t seed,
                              float *w) {
  GRID_STRIDE(e, m) {
    uint64_t key = ((uint64_t)(uint32_t)src[e] << 32) | (uint32_t)idx[e];
    w[e] = (float)((hash64(seed, key) >> 40) + 1) * (1.0f / 16777216.0f);
  }
}
__global__ void k_uniform_f32(uint64_t seed, int open, int64_t count, float *x) {
  GRID_STRIDE(i, count) {
    uint64_t h = hash64(seed, (uint64_t)i);
    x[i] = open ? (float)(((h >> 41) << 1) | 1) * (1.0f / 16777216.0f)
                : (float)(h >> 40) * (1.0f / 16777216.0f);
  }
}

// ---------------------------------------------------------------------------
// Rows with more than heavy_deg edges: chunk counts, their prefix sum
// (hfirst) and the chunk -> row table (hrow).
static void build_heavy(pm_graph *g, AdjBuf &a, cudaStream_t st, int32_t heavy_deg) {
  const int64_t n = g->n;
  DevBuf nch((size_t)(n + 1) * 4), md(4);
  PM_CUDA(cudaMemsetAsync(md.p, 0, 4, st));
  PM_CUDA(cudaMemsetAsync(nch.p, 0, (size_t)(n + 1) * 4, st));
  PM_LAUNCH(k_heavy_counts, grid1d(n), 256, 0, st, a.off.as<int32_t>(), n, heavy_deg, nch.as<int32_t>(),
            md.as<int32_t>());
  a.hfirst.alloc((size_t)(n + 1) * 4);
  size_t tmp = 0;
  PM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, nch.as<int32_t>(), a.hfirst.as<int32_t>(),
                                        (int)(n + 1), st));
  DevBuf tb(tmp);
  PM_CUDA(cub::DeviceScan::ExclusiveSum(tb.p, tmp, nch.as<int32_t>(), a.hfirst.as<int32_t>(),
                                        (int)(n + 1), st));
  int32_t total = 0, maxdeg = 0;
  PM_CUDA(cudaMemcpyAsync(&total, a.hfirst.as<int32_t>() + n, 4, cudaMemcpyDeviceToHost, st));
  PM_CUDA(cudaMemcpyAsync(&maxdeg, md.p, 4, cudaMemcpyDeviceToHost, st));
  PM_CUDA(cudaStreamSynchronize(st));
  a.nchunks = total;
  a.hrow.alloc((size_t)std::max(total, 1) * 4);
  if (total > 0)
    PM_LAUNCH(k_heavy_rows, grid1d(n), 256, 0, st, nch.as<int32_t>(), a.hfirst.as<int32_t>(), n,
              a.hrow.as<int32_t>());
  if (&a == &g->out) g->max_out_deg = maxdeg;
}

// Group and heavy tables of one adjacency; the rows [r0, r1) are the rows
// the pulls over it visit (all rows, or a partition's own range, which holds
// every edge of a partition's CSC).
static void build_tables(pm_graph *g, AdjBuf &a, cudaStream_t st, int64_t r0, int64_t r1) {
  const int64_t m = g->m;
  a.ngroups = (int32_t)((m + kRowWork * (r1 - r0) + kGroupWork - 1) / kGroupWork);
  if (a.ngroups < 1) a.ngroups = 1;
  a.gstart.alloc((size_t)(a.ngroups + 1) * 4);
  PM_LAUNCH(k_group_starts, grid1d(a.ngroups + 1), 256, 0, st, a.off.as<int32_t>(), r0, r1, a.ngroups,
            a.gstart.as<int32_t>());
  build_heavy(g, a, st, g->E.tune.heavy_deg);
}

// Views of the adjacency and the tunables the kernels read.
static void set_views(pm_graph *g) {
  GraphView &v = g->E.g;
  v.n = (int32_t)g->n;
  v.m = g->m;
  v.out = g->out.view();
  v.in = g->symmetric ? v.out : g->in.view();
  v.heavy_deg = g->E.tune.heavy_deg;
  v.cta_expand = g->E.tune.cta_expand;
  v.grid_expand = g->E.tune.grid_expand;
  v.push_agg = g->E.tune.push_agg;
#if PM_CHECK
  if (!g->check_word.p) {
    g->check_word.alloc(16);
    PM_CUDA(cudaMemsetAsync(g->check_word.p, 0, 16, g->E.stream));
  }
  v.check = g->check_word.as<unsigned>();
#endif
}

void apply_tunables(pm_graph *g, int32_t old_heavy_deg) {
  cudaStream_t st = g->E.stream;
  g->E.release_graphs();  // captured launches hold the old views
  if (g->E.tune.heavy_deg != old_heavy_deg) {
    build_heavy(g, g->out, st, g->E.tune.heavy_deg);
    if (!g->symmetric) build_heavy(g, g->in, st, g->E.tune.heavy_deg);
  }
  set_views(g);
  const GraphView &v = g->E.g;
  const size_t pbytes = (size_t)std::max(std::max(v.in.nchunks, v.out.nchunks), 1) * 16;
  if (g->partials.bytes < pbytes) g->partials.alloc(pbytes);
  if (g->hdone.bytes < pbytes / 4) g->hdone.alloc(pbytes / 4);
  g->E.partials = g->partials.p;
  g->E.hdone = g->hdone.as<int32_t>();
  PM_CUDA(cudaStreamSynchronize(st));
}

void finish_graph(pm_graph *g) {
  cudaStream_t st = g->E.stream;
  const int64_t n = g->n, m = g->m;
  // Source of every CSR edge (needed for the transpose and weight rules).
  DevBuf src((size_t)std::max<int64_t>(m, 1) * 4);
  fill_edge_src(g->out.off.as<int32_t>(), n, m, src.as<int32_t>(), st);
  build_tables(g, g->out, st, 0, n);
  // Stable radix sort of (dst, edge id): sources stay ascending per row, so
  // slot p of the sorted order is the CSC slot of the edge it holds.  For a
  // symmetric graph the CSC is the CSR itself and this is the reverse-edge
  // map (five times faster than a binary search per edge at scale 22).
  int bits = 1;
  while ((1ll << bits) < n) ++bits;
  DevBuf kout((size_t)std::max<int64_t>(m, 1) * 4);
  g->in_eid.alloc((size_t)std::max<int64_t>(m, 1) * 4);
  if (m) {
    DevBuf vin((size_t)m * 4);
    PM_LAUNCH(k_iota, grid1d(m), 256, 0, st, vin.as<int32_t>(), m);
    size_t tmp = 0;
    PM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, g->out.idx.as<int32_t>(), kout.as<int32_t>(),
                                            vin.as<int32_t>(), g->in_eid.as<int32_t>(), (int)m, 0, bits, st));
    DevBuf tb(std::max<size_t>(tmp, 16));
    PM_CUDA(cub::DeviceRadixSort::SortPairs(tb.p, tmp, g->out.idx.as<int32_t>(), kout.as<int32_t>(),
                                            vin.as<int32_t>(), g->in_eid.as<int32_t>(), (int)m, 0, bits, st));
    PM_CUDA(cudaStreamSynchronize(st));
  }
  if (!g->symmetric) {
    g->in.off.alloc((size_t)(n + 1) * 4);
    g->in.idx.alloc((size_t)std::max<int64_t>(m, 1) * 4);
    PM_LAUNCH(k_lower_bound_offsets, grid1d(n + 1), 256, 0, st, kout.as<int32_t>(), m, n,
              g->in.off.as<int32_t>());
    if (m)
      PM_LAUNCH(k_gather_src, grid1d(m), 256, 0, st, src.as<int32_t>(), g->in_eid.as<int32_t>(), m,
                g->in.idx.as<int32_t>());
    // a partition's CSC holds only its own rows: its pulls visit only them
    build_tables(g, g->in, st, g->is_part ? g->part_lo : 0, g->is_part ? g->part_hi : n);
  }
  // Views and workspaces.
  set_views(g);
  const GraphView &v = g->E.g;
  const int64_t words = (n + 31) / 32 + 1;
  g->bits0.alloc((size_t)words * 4);
  g->bits1.alloc((size_t)words * 4);
  g->queue0.alloc((size_t)(n + 1) * 4);
  g->queue1.alloc((size_t)(n + 1) * 4);
  g->defer.alloc((size_t)(n + 1) * 4);
  g->hubs.alloc((size_t)kMaxHubs * 4);
  // partial sums of heavy chunks, for pulls over the CSC or over the CSR
  g->partials.alloc((size_t)std::max(std::max(v.in.nchunks, v.out.nchunks), 1) * 16);
  g->hdone.alloc((size_t)std::max(std::max(v.in.nchunks, v.out.nchunks), 1) * 4);
  g->cnt.alloc(3 * sizeof(Counters));
  PM_CUDA(cudaMemsetAsync(g->cnt.p, 0, 3 * sizeof(Counters), st));  // error words start clear
  g->E.d_cnt = g->cnt.as<Counters>();
  g->E.defer = g->defer.as<int32_t>();
  g->E.hubs = g->hubs.as<int32_t>();
  g->E.partials = g->partials.p;
  g->E.hdone = g->hdone.as<int32_t>();
  PM_CUDA(cudaStreamSynchronize(st));
}

void permute_weights_i32(pm_graph *g) {
  const int64_t m = g->m;
  g->w_i32_in.alloc((size_t)std::max<int64_t>(m, 1) * 4);
  if (m)
    PM_LAUNCH(k_gather<int32_t>, grid1d(m), 256, 0, g->E.stream, g->w_i32_out.as<int32_t>(),
              g->in_eid.as<int32_t>(), m, g->w_i32_in.as<int32_t>());
  PM_CUDA(cudaStreamSynchronize(g->E.stream));
}
void permute_weights_f32(pm_graph *g) {
  const int64_t m = g->m;
  g->w_f32_pair_in.reset();  // rebuilt from the new weights on first use
  g->w_f32_pair_out.reset();
  g->w_f32_in.alloc((size_t)std::max<int64_t>(m, 1) * 4);
  if (m)
    PM_LAUNCH(k_gather<float>, grid1d(m), 256, 0, g->E.stream, g->w_f32_out.as<float>(),
              g->in_eid.as<int32_t>(), m, g->w_f32_in.as<float>());
  PM_CUDA(cudaStreamSynchronize(g->E.stream));
}

// Validate a CSR already on the device; optionally drop self loops (and
// the matching entries of w, int32 weights in CSR order, when given).
void ingest_csr(pm_graph *g, bool skip_self_loops, DevBuf *w) {
  cudaStream_t st = g->E.stream;
  const int64_t n = g->n, m = g->m;
  DevBuf err(8);
  PM_CUDA(cudaMemsetAsync(err.p, 0, 8, st));
  PM_LAUNCH(k_validate, grid1d(std::max(n, m)), 256, 0, st, g->out.off.as<int32_t>(),
            g->out.idx.as<int32_t>(), n, m, err.as<unsigned int>(), err.as<unsigned int>() + 1);
  unsigned int h_err[2] = {0, 0};
  PM_CUDA(cudaMemcpyAsync(h_err, err.p, 8, cudaMemcpyDeviceToHost, st));
  PM_CUDA(cudaStreamSynchronize(st));
  if (h_err[0])
    fail(PM_ERR_BAD_GRAPH, std::string("invalid CSR:") + (h_err[0] & 1 ? " offsets not monotone" : "") +
                               (h_err[0] & 2 ? " edge id out of range" : "") +
                               (h_err[0] & 4 ? " offsets[0] != 0 or offsets[n] != m" : ""));
  if (m == 0) return;
  DevBuf src((size_t)m * 4), keep((size_t)m * 4), cntb(4);
  PM_CUDA(cudaMemsetAsync(cntb.p, 0, 4, st));
  fill_edge_src(g->out.off.as<int32_t>(), n, m, src.as<int32_t>(), st);
  PM_LAUNCH(k_self_flags, grid1d(m), 256, 0, st, src.as<int32_t>(), g->out.idx.as<int32_t>(), m,
            keep.as<int32_t>(), cntb.as<unsigned int>());
  unsigned int loops = 0;
  PM_CUDA(cudaMemcpyAsync(&loops, cntb.p, 4, cudaMemcpyDeviceToHost, st));
  PM_CUDA(cudaStreamSynchronize(st));
  if (loops == 0) return;
  if (!skip_self_loops) {
    g->has_self_loops = true;
    return;
  }
  DevBuf pre((size_t)(m + 1) * 4);
  size_t tmp = 0;
  PM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, keep.as<int32_t>(), pre.as<int32_t>(), (int)m, st));
  DevBuf tb(tmp);
  PM_CUDA(cub::DeviceScan::ExclusiveSum(tb.p, tmp, keep.as<int32_t>(), pre.as<int32_t>(), (int)m, st));
  int32_t m_new = (int32_t)(m - loops);
  PM_CUDA(cudaMemcpyAsync(pre.as<int32_t>() + m, &m_new, 4, cudaMemcpyHostToDevice, st));
  DevBuf noff((size_t)(n + 1) * 4), nidx((size_t)std::max<int32_t>(m_new, 1) * 4);
  PM_LAUNCH(k_remap_offsets, grid1d(n + 1), 256, 0, st, g->out.off.as<int32_t>(), pre.as<int32_t>(), n,
            noff.as<int32_t>());
  PM_LAUNCH(k_compact_edges, grid1d(m), 256, 0, st, g->out.idx.as<int32_t>(), keep.as<int32_t>(),
            pre.as<int32_t>(), m, nidx.as<int32_t>());
  if (w && w->p) {
    DevBuf nw((size_t)std::max<int32_t>(m_new, 1) * 4);
    PM_LAUNCH(k_compact_edges, grid1d(m), 256, 0, st, w->as<int32_t>(), keep.as<int32_t>(), pre.as<int32_t>(),
              m, nw.as<int32_t>());
    PM_CUDA(cudaStreamSynchronize(st));
    *w = std::move(nw);
  }
  PM_CUDA(cudaStreamSynchronize(st));
  g->out.off = std::move(noff);
  g->out.idx = std::move(nidx);
  g->m = m_new;
}

// Seeded R-MAT straight into the device CSR.
// Sorts the (src << 32 | dst) keys in a (self loops replaced by a sentinel
// >= n << 32 below 2^(end_bit)), drops duplicates and the sentinel, and
// builds g's CSR.
static void keys_to_csr(pm_graph *g, DevBuf &a, DevBuf &b, int64_t nkeys, int64_t n, int end_bit) {
  cudaStream_t st = g->E.stream;
  cub::DoubleBuffer<uint64_t> db(a.as<uint64_t>(), b.as<uint64_t>());
  size_t tmp = 0;
  PM_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tmp, db, (int)nkeys, 0, end_bit, st));
  DevBuf tb(tmp);
  PM_CUDA(cub::DeviceRadixSort::SortKeys(tb.p, tmp, db, (int)nkeys, 0, end_bit, st));
  uint64_t *sorted = db.Current();
  uint64_t *uniq = db.Alternate();
  DevBuf nsel(8);
  size_t tmp2 = 0;
  PM_CUDA(cub::DeviceSelect::Unique(nullptr, tmp2, sorted, uniq, nsel.as<int64_t>(), (int64_t)nkeys, st));
  DevBuf tb2(tmp2);
  PM_CUDA(cub::DeviceSelect::Unique(tb2.p, tmp2, sorted, uniq, nsel.as<int64_t>(), (int64_t)nkeys, st));
  int64_t nu = 0;
  PM_CUDA(cudaMemcpyAsync(&nu, nsel.p, 8, cudaMemcpyDeviceToHost, st));
  PM_CUDA(cudaStreamSynchronize(st));
  // The sentinel (self loops) sorts last; drop it if present.
  uint64_t last = 0;
  if (nu > 0) {
    PM_CUDA(cudaMemcpyAsync(&last, uniq + (nu - 1), 8, cudaMemcpyDeviceToHost, st));
    PM_CUDA(cudaStreamSynchronize(st));
  }
  const int64_t m = nu > 0 && (last >> 32) >= (uint64_t)n ? nu - 1 : nu;
  if (m >= (1ll << 31) - 1) fail(PM_ERR_INVALID_ARG, "graph exceeds int32 edge offsets");
  g->n = n;
  g->m = m;
  g->out.off.alloc((size_t)(n + 1) * 4);
  g->out.idx.alloc((size_t)std::max<int64_t>(m, 1) * 4);
  if (m) PM_LAUNCH(k_keys_to_csr_idx, grid1d(m), 256, 0, st, uniq, m, g->out.idx.as<int32_t>());
  PM_LAUNCH(k_keys_offsets, grid1d(n + 1), 256, 0, st, uniq, m, n, g->out.off.as<int32_t>());
  PM_CUDA(cudaStreamSynchronize(st));
}

void generate_rmat(pm_graph *g, int scale, int ef, uint64_t seed) {
  const int64_t n = (int64_t)1 << scale;
  const int64_t draws = n * ef;
  const int64_t nkeys = draws * (g->symmetric ? 2 : 1);
  DevBuf a((size_t)nkeys * 8), b((size_t)nkeys * 8);
  PM_LAUNCH(k_rmat_keys, grid1d(draws), 256, 0, g->E.stream, scale, seed, draws, (int)g->symmetric,
            a.as<uint64_t>());
  keys_to_csr(g, a, b, nkeys, n, 33 + scale);
}

// Erdos-Renyi batch: the rule of the oracle's pmo_er_batch.
__global__ void k_er_keys(const int64_t *vbase, const int64_t *dbase, int count, int64_t draws,
                          uint64_t seed2, uint64_t sentinel, uint64_t *keys) {
  GRID_STRIDE(k, draws) {
    int lo = 0, hi = count - 1;  // graph of draw k: last i with dbase[i] <= k
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (dbase[mid] <= k) lo = mid; else hi = mid - 1;
    }
    const uint64_t ni = (uint64_t)(vbase[lo + 1] - vbase[lo]);
    const uint64_t h = hash64(seed2, (uint64_t)k);
    const uint64_t s = (uint64_t)vbase[lo] + (h >> 32) % ni;
    const uint64_t d = (uint64_t)vbase[lo] + (h & 0xffffffffull) % ni;
    keys[k] = s == d ? sentinel : ((s << 32) | d);
  }
}

// Part sizes of the ER batch (host; the oracle's pmo_er_part_sizes).
std::vector<int64_t> er_part_sizes(int count, int64_t n_min, int64_t n_max, uint64_t seed) {
  std::vector<int64_t> vbase(count + 1, 0);
  for (int i = 0; i < count; ++i) {
    const double u = (double)(hash64(seed, (uint64_t)i) >> 11) * (1.0 / 9007199254740992.0);
    int64_t ni = (int64_t)std::floor(std::exp(std::log((double)n_min) +
                                              u * (std::log((double)n_max) - std::log((double)n_min))));
    ni = std::min(std::max(ni, n_min), n_max);
    vbase[i + 1] = vbase[i] + ni;
  }
  return vbase;
}

void set_parts(pm_graph *g, const std::vector<int64_t> &vbase);

void generate_er_batch(pm_graph *g, int count, int64_t n_min, int64_t n_max, int avg_degree,
                       uint64_t seed) {
  std::vector<int64_t> vbase = er_part_sizes(count, n_min, n_max, seed);
  const int64_t n = vbase[count];
  std::vector<int64_t> dbase(count + 1);
  for (int i = 0; i <= count; ++i) dbase[i] = vbase[i] * avg_degree;
  const int64_t draws = dbase[count];
  if (n >= (1ll << 31) - 1 || draws >= (1ll << 31) - 1)
    fail(PM_ERR_INVALID_ARG, "batch exceeds int32 ids or edge offsets");
  int bits = 1;
  while ((1ll << bits) <= n) ++bits;
  DevBuf dv((size_t)(count + 1) * 8), dd((size_t)(count + 1) * 8);
  PM_CUDA(cudaMemcpyAsync(dv.p, vbase.data(), (count + 1) * 8, cudaMemcpyHostToDevice, g->E.stream));
  PM_CUDA(cudaMemcpyAsync(dd.p, dbase.data(), (count + 1) * 8, cudaMemcpyHostToDevice, g->E.stream));
  DevBuf a((size_t)std::max<int64_t>(draws, 1) * 8), b((size_t)std::max<int64_t>(draws, 1) * 8);
  PM_LAUNCH(k_er_keys, grid1d(draws), 256, 0, g->E.stream, dv.as<int64_t>(), dd.as<int64_t>(), count,
            draws, seed ^ 0xE5E5E5E5ull, (uint64_t)1 << (32 + bits), a.as<uint64_t>());
  keys_to_csr(g, a, b, draws, n, 33 + bits);
  set_parts(g, vbase);
}

// err |= 1 when an edge leaves its source's part.
__global__ void k_check_parts(const int32_t *off, const int32_t *idx, int64_t n, const int64_t *vbase,
                              int count, unsigned int *err) {
  GRID_STRIDE(v, n) {
    int lo = 0, hi = count - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (vbase[mid] <= v) lo = mid; else hi = mid - 1;
    }
    const int64_t a = vbase[lo], b = vbase[lo + 1];
    for (int32_t e = off[v]; e < off[v + 1]; ++e)
      if (idx[e] < a || idx[e] >= b) atomicOr(err, 1u);
  }
}

void check_parts(pm_graph *g, const std::vector<int64_t> &vbase) {
  const int count = (int)vbase.size() - 1;
  if (count < 1 || vbase[0] != 0 || vbase[count] != g->n)
    fail(PM_ERR_INVALID_ARG, "parts must start at 0 and end at n");
  for (int i = 0; i < count; ++i)
    if (vbase[i + 1] <= vbase[i]) fail(PM_ERR_INVALID_ARG, "parts must be non-empty and increasing");
  DevBuf dv((size_t)(count + 1) * 8), err(4);
  PM_CUDA(cudaMemcpyAsync(dv.p, vbase.data(), (count + 1) * 8, cudaMemcpyHostToDevice, g->E.stream));
  PM_CUDA(cudaMemsetAsync(err.p, 0, 4, g->E.stream));
  PM_LAUNCH(k_check_parts, grid1d(g->n), 256, 0, g->E.stream, g->out.off.as<int32_t>(),
            g->out.idx.as<int32_t>(), g->n, dv.as<int64_t>(), count, err.as<unsigned int>());
  unsigned int h = 0;
  PM_CUDA(cudaMemcpyAsync(&h, err.p, 4, cudaMemcpyDeviceToHost, g->E.stream));
  PM_CUDA(cudaStreamSynchronize(g->E.stream));
  if (h) fail(PM_ERR_BAD_GRAPH, "an edge crosses two parts");
}

// Part boundaries and the largest-first processing order.
void set_parts(pm_graph *g, const std::vector<int64_t> &vbase) {
  const int count = (int)vbase.size() - 1;
  std::vector<int32_t> order(count);
  for (int i = 0; i < count; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    return vbase[a + 1] - vbase[a] > vbase[b + 1] - vbase[b];
  });
  g->parts_vbase.alloc((size_t)(count + 1) * 8);
  g->parts_order.alloc((size_t)std::max(count, 1) * 4);
  PM_CUDA(cudaMemcpyAsync(g->parts_vbase.p, vbase.data(), (count + 1) * 8, cudaMemcpyHostToDevice,
                          g->E.stream));
  PM_CUDA(cudaMemcpyAsync(g->parts_order.p, order.data(), count * 4, cudaMemcpyHostToDevice, g->E.stream));
  PM_CUDA(cudaStreamSynchronize(g->E.stream));
  g->parts = vbase;
}

void gen_weights(pm_graph *g, uint64_t seed, int32_t wmax, bool is_float) {
  cudaStream_t st = g->E.stream;
  const int64_t n = g->n, m = g->m;
  DevBuf src((size_t)std::max<int64_t>(m, 1) * 4);
  fill_edge_src(g->out.off.as<int32_t>(), n, m, src.as<int32_t>(), st);
  if (is_float) {
    g->w_f32_out.alloc((size_t)std::max<int64_t>(m, 1) * 4);
    if (m) PM_LAUNCH(k_weights_f32, grid1d(m), 256, 0, st, src.as<int32_t>(), g->out.idx.as<int32_t>(), m,
                     seed, g->w_f32_out.as<float>());
    permute_weights_f32(g);
  } else {
    g->w_i32_out.alloc((size_t)std::max<int64_t>(m, 1) * 4);
    if (m) PM_LAUNCH(k_weights_i32, grid1d(m), 256, 0, st, src.as<int32_t>(), g->out.idx.as<int32_t>(), m,
                     seed, wmax, g->w_i32_out.as<int32_t>());
    permute_weights_i32(g);
  }
}

__global__ void k_make_pairs(const int32_t *__restrict__ idx, const float *__restrict__ w, int64_t m,
                             WPair *__restrict__ out) {
  GRID_STRIDE(e, m) out[e] = WPair{idx[e], w[e]};
}

const WPair *ensure_f32_pairs(pm_graph *g, bool csr) {
  DevBuf &pairs = csr ? g->w_f32_pair_out : g->w_f32_pair_in;
  const DevBuf &w = csr ? g->w_f32_out : g->w_f32_in;
  if (!pairs.p) {
    if (!w.p) fail(PM_ERR_INVALID_ARG, "graph has no float weights");
    pairs.alloc((size_t)std::max<int64_t>(g->m, 1) * sizeof(WPair));
    if (g->m)
      PM_LAUNCH(k_make_pairs, grid1d(g->m), 256, 0, g->E.stream, csr ? g->E.g.out.idx : g->E.g.in.idx,
                w.as<float>(), g->m, pairs.as<WPair>());
  }
  return pairs.as<WPair>();
}

void ensure_out_src(pm_graph *g) {
  if (g->out_src.p) return;
  g->out_src.alloc((size_t)std::max<int64_t>(g->m, 1) * 4);
  fill_edge_src(g->out.off.as<int32_t>(), g->n, g->m, g->out_src.as<int32_t>(), g->E.stream);
}

// Lognormal(0,1) weights normalised per source row (the oracle's
// pmo_lognormal_weights rule, evaluated in FP32 with CUDA's libm).
__global__ void k_lognormal_rows(const int32_t *off, int64_t n, uint64_t seed, float *w) {
  const float two_pi = 6.28318530717958647692f;
  GRID_STRIDE(s, n) {
    float sum = 0.0f;
    for (int64_t e = off[s]; e < off[s + 1]; ++e) {
      const double u1 = (double)((hash64(seed, 2 * (uint64_t)e) >> 11) + 1) * (1.0 / 9007199254740992.0);
      const double u2 = (double)(hash64(seed, 2 * (uint64_t)e + 1) >> 11) * (1.0 / 9007199254740992.0);
      const float x = expf(sqrtf(-2.0f * logf((float)u1)) * cosf(two_pi * (float)u2));
      w[e] = x;
      sum += x;
    }
    for (int64_t e = off[s]; e < off[s + 1]; ++e) w[e] /= sum;
  }
}

void gen_weights_lognormal(pm_graph *g, uint64_t seed) {
  g->w_f32_out.alloc((size_t)std::max<int64_t>(g->m, 1) * 4);
  PM_LAUNCH(k_lognormal_rows, grid1d(g->n), 256, 0, g->E.stream, g->out.off.as<int32_t>(), g->n, seed,
            g->w_f32_out.as<float>());
  permute_weights_f32(g);
}

void fill_uniform(pm_graph *g, uint64_t seed, int open, float *out, int64_t count) {
  PM_LAUNCH(k_uniform_f32, grid1d(count), 256, 0, g->E.stream, seed, open, count, out);
  PM_CUDA(cudaStreamSynchronize(g->E.stream));
}

}  // namespace pm

pm_graph::~pm_graph() {
  if (E.stream) cudaStreamSynchronize(E.stream);
  E.release_graphs();
  E.release_side_stream();
  pm::pinned_small_free(h_cnt, 3 * sizeof(pm::Counters));
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  if (own_stream) cudaStreamSynchronize(own_stream);
  if (own_stream) cudaStreamDestroy(own_stream);
  // nothing of this handle is in flight: its buffers go back idle
  saved = pm::alloc_ctx();
  pm::set_alloc_ctx(pm::AllocCtx{nullptr, true});
}
