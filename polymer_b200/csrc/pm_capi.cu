// pm_capi.cu -- the extern "C" boundary (include/polymer_b200.h).
// Every entry point validates its arguments, stages host arrays through the
// handle's device scratch, runs on the graph's stream and converts internal
// failures into a pm_status plus a thread-local message.
#include <cstdio>
#include <cstring>

#include <nvtx3/nvToolsExt.h>

#include "pm_graph.cuh"

namespace pm {
long long launches(bool reset);
void ingest_csr(pm_graph *g, bool skip_self_loops, DevBuf *w = nullptr);
void parse_pbbs_text(pm_graph *g, const char *path, DevBuf &off, DevBuf &idx, DevBuf &w, int64_t &n,
                     int64_t &m);
void read_graph_dump(pm_graph *g, const char *path, DevBuf &off, DevBuf &idx, int64_t &n, int64_t &m);
void write_graph_dump(pm_graph *g, const char *path);
void read_pbbs_binary(const char *base, std::vector<int32_t> &off, std::vector<int32_t> &idx, int64_t &n,
                      int64_t &m);
void generate_rmat(pm_graph *g, int scale, int ef, uint64_t seed);
void gen_weights(pm_graph *g, uint64_t seed, int32_t wmax, bool is_float);
void fill_uniform(pm_graph *g, uint64_t seed, int open, float *out, int64_t count);
void run_bfs(pm_graph *g, int32_t src, int32_t *d_parents, int32_t *d_depth, int64_t threshold,
             pm_traversal_stats *st);
void run_cc(pm_graph *g, int32_t *d_labels, int64_t threshold, pm_traversal_stats *st);
void run_bellman_ford(pm_graph *g, int32_t src, int32_t *d_dist, int64_t threshold,
                      pm_traversal_stats *st);
template <class T>
void run_pagerank(pm_graph *g, int iters, double damping, T *d_out, double *d_resid);
template <class T>
void run_pagerank_delta(pm_graph *g, int iters, double damping, double eps2, T *d_out, int64_t threshold,
                        pm_traversal_stats *st);
template <class T>
void run_spmv(pm_graph *g, const T *d_x0, int iters, T *d_y, double *d_norm);
template <class T>
void run_bp(pm_graph *g, const T *d_prior, const T *psi, int iters, T *d_out);
void run_msbfs(pm_graph *g, const int32_t *d_sources, int k, int32_t *d_depth, int64_t threshold,
               pm_traversal_stats *st);
void run_bf_multi(pm_graph *g, const int32_t *d_sources, int k, int32_t *d_dist, int64_t threshold,
                  pm_traversal_stats *st);
void run_bfs_async(pm_graph *g, int32_t src, int32_t *d_parents, pm_traversal_stats *st);
void run_ppr(pm_graph *g, const int32_t *d_seeds, int k, int iters, double damping, float *d_out);
void run_pagerank_parts(pm_graph *g, int iters, double damping, float *d_out);
void generate_er_batch(pm_graph *g, int count, int64_t n_min, int64_t n_max, int avg_degree,
                       uint64_t seed);
void check_parts(pm_graph *g, const std::vector<int64_t> &vbase);
int run_weighted_pagerank(pm_graph *g, double damping, double tol, int max_iters, float *d_p,
                          double *resid);
int run_pagerank_adjoint(pm_graph *g, double damping, double tol, int max_iters, const float *d_p,
                         const float *d_g, float *d_dw, float *d_lambda, double *resid);
void run_spmv_backward(pm_graph *g, const float *d_x, const float *d_gy, float *d_dx, float *d_dw);
void gen_weights_lognormal(pm_graph *g, uint64_t seed);
void set_parts(pm_graph *g, const std::vector<int64_t> &vbase);
void set_tunable(pm_graph *g, int key, int64_t value);
void set_memory_cache(int64_t limit);
void release_memory_cache();
int64_t memory_cached();
Tunables default_tunables();
int64_t get_tunable(pm_graph *g, int key);
void tune(pm_graph *g, const int *apps, int count, pm_tune_report *rep);
}  // namespace pm

using namespace pm;

static thread_local std::string t_last_error;

namespace pm {
void set_last_error(const std::string &msg) { t_last_error = msg; }
}  // namespace pm

// The bounded wait of the fused heavy-row pull (wait_at_least) on a flag that
// nothing sets: it must give up, report kErrTimeout and return.
__global__ void k_test_wait(const int32_t *flag, unsigned *err, int max_polls) {
  if (threadIdx.x == 0) wait_at_least(flag, 1, max_polls, err);
}

// Scratch slots used for staging at the boundary (the algorithms use 0..3).
enum { kSlotIn0 = 8, kSlotIn1 = 9, kSlotOut0 = 10, kSlotOut1 = 11, kSlotAux = 12 };

// One NVTX range per C-ABI call, named after the entry point, so a profiler
// can select one application's kernels (ncu --nvtx --nvtx-include
// "pm_pagerank/"); with no tool attached a push or pop is a pointer test.
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};

template <class Fn>
static pm_status guard(const char *name, Fn &&fn) {
  NvtxRange range(name);
  AllocScope scope(AllocCtx{});  // enter() names the call's stream
  try {
    fn();
    t_last_error.clear();
    return PM_OK;
  } catch (const Failure &f) {
    t_last_error = f.what();
    return f.status;
  } catch (const std::bad_alloc &) {
    t_last_error = "host allocation failed";
    return PM_ERR_OOM;
  } catch (const std::exception &e) {
    t_last_error = e.what();
    return PM_ERR_CUDA;
  }
}

static void need(bool ok, const char *msg) {
  if (!ok) fail(PM_ERR_INVALID_ARG, msg);
}

static void use_device(int dev) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    (void)cudaGetLastError();
    fail(PM_ERR_NO_DEVICE, "no CUDA device visible");
  }
  need(dev >= 0 && dev < count, "device index out of range");
  PM_CUDA(cudaSetDevice(dev));
}

static pm_graph *new_graph(int device, bool symmetric) {
  use_device(device);
  auto *g = new pm_graph();
  g->device = device;
  g->symmetric = symmetric;
  g->E.tune = default_tunables();
  try {
    PM_CUDA(cudaStreamCreateWithFlags(&g->E.stream, cudaStreamNonBlocking));
    g->own_stream = g->E.stream;
    set_alloc_ctx(AllocCtx{g->E.stream, false});
    g->h_cnt = (Counters *)pinned_small_alloc(3 * sizeof(Counters));
    g->E.h_cnt = g->h_cnt;
    PM_CUDA(cudaEventCreate(&g->ev0));
    PM_CUDA(cudaEventCreate(&g->ev1));
    PM_CUDA(cudaDeviceGetAttribute(&g->E.num_sms, cudaDevAttrMultiProcessorCount, device));
  } catch (...) {
    delete g;
    throw;
  }
  return g;
}

// Copy count elements between host/device and a device buffer on the stream.
static void to_device(pm_graph *g, void *dst, const void *src, size_t bytes, uint32_t mem) {
  if (bytes == 0) return;
  PM_CUDA(cudaMemcpyAsync(dst, src, bytes,
                          mem == PM_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                          g->E.stream));
}
static void from_device(pm_graph *g, void *dst, const void *src, size_t bytes, uint32_t mem) {
  if (bytes == 0) return;
  PM_CUDA(cudaMemcpyAsync(dst, src, bytes,
                          mem == PM_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                          g->E.stream));
}
static void finish(pm_graph *g) {
  PM_CUDA(cudaStreamSynchronize(g->E.stream));
#if PM_CHECK
  unsigned bad = 0;
  if (g->check_word.p) {
    PM_CUDA(cudaMemcpy(&bad, g->check_word.p, 4, cudaMemcpyDeviceToHost));
    if (bad) PM_CUDA(cudaMemset(g->check_word.p, 0, 4));
  }
  if (bad) fail(PM_ERR_BAD_GRAPH, "checked build: a kernel read a vertex id outside [0, n)");
#endif
}
static void check_mem(uint32_t mem) { need(mem == PM_MEM_HOST || mem == PM_MEM_DEVICE, "mem must be PM_MEM_HOST or PM_MEM_DEVICE"); }
// The calls a partition graph serves: pm_pagerank, pm_spmv, pm_bp, pm_bfs,
// pm_components, pm_bellman_ford (and the handle queries); the others need
// the whole graph on one device.
static void whole_graph(const pm_graph *g, const char *what) {
  if (g->is_part) fail(PM_ERR_NOT_SUPPORTED, std::string(what) + " needs the whole graph, not a partition");
}

static void enter(pm_graph *g) {
  need(g != nullptr, "null graph handle");
  PM_CUDA(cudaSetDevice(g->device));
  set_alloc_ctx(AllocCtx{g->E.stream, false});  // this call's buffers live in this stream's order
}

extern "C" {

pm_status pm_graph_create(const int32_t *offsets, const int32_t *edges, int64_t n, int64_t m,
                          uint32_t flags, uint32_t mem, int device, pm_graph **out) {
  return guard(__func__, [&] {
    need(out != nullptr, "out is null");
    *out = nullptr;
    need(n > 0 && n < (1ll << 31) - 1, "n must be in [1, 2^31-2]");
    need(m >= 0 && m < (1ll << 31) - 1, "m must be in [0, 2^31-2]");
    need(offsets != nullptr && (m == 0 || edges != nullptr), "null offsets/edges");
    check_mem(mem);
    pm_graph *g = new_graph(device, (flags & PM_GRAPH_SYMMETRIC) != 0);
    try {
      g->n = n;
      g->m = m;
      g->out.off.alloc((size_t)(n + 1) * 4);
      g->out.idx.alloc((size_t)std::max<int64_t>(m, 1) * 4);
      to_device(g, g->out.off.p, offsets, (size_t)(n + 1) * 4, mem);
      to_device(g, g->out.idx.p, edges, (size_t)m * 4, mem);
      ingest_csr(g, (flags & PM_GRAPH_SKIP_SELF_LOOPS) != 0);
      finish_graph(g);
    } catch (...) {
      delete g;
      throw;
    }
    *out = g;
  });
}

pm_status pm_graph_create_weighted(const int32_t *offsets, const int32_t *edges, const void *weights, int wtype,
                                   int64_t n, int64_t m, uint32_t flags, uint32_t mem, int device,
                                   pm_graph **out) {
  return guard(__func__, [&] {
    need(out != nullptr, "out is null");
    *out = nullptr;
    need(n > 0 && n < (1ll << 31) - 1, "n must be in [1, 2^31-2]");
    need(m >= 0 && m < (1ll << 31) - 1, "m must be in [0, 2^31-2]");
    need(offsets != nullptr && (m == 0 || (edges != nullptr && weights != nullptr)), "null offsets/edges/weights");
    need(wtype == PM_F32 || wtype == PM_I32, "wtype must be PM_F32 or PM_I32");
    check_mem(mem);
    pm_graph *g = new_graph(device, (flags & PM_GRAPH_SYMMETRIC) != 0);
    cudaStream_t ws = nullptr;
    cudaEvent_t wdone = nullptr;
    try {
      g->n = n;
      g->m = m;
      g->out.off.alloc((size_t)(n + 1) * 4);
      g->out.idx.alloc((size_t)std::max<int64_t>(m, 1) * 4);
      DevBuf w((size_t)std::max<int64_t>(m, 1) * 4);
      // the CSR first; the weights follow on a second stream while the
      // graph is validated and transposed
      to_device(g, g->out.off.p, offsets, (size_t)(n + 1) * 4, mem);
      to_device(g, g->out.idx.p, edges, (size_t)m * 4, mem);
      PM_CUDA(cudaStreamCreateWithFlags(&ws, cudaStreamNonBlocking));
      PM_CUDA(cudaEventCreateWithFlags(&wdone, cudaEventDisableTiming));
      PM_CUDA(cudaEventRecord(wdone, g->E.stream));
      PM_CUDA(cudaStreamWaitEvent(ws, wdone, 0));
      if (m)
        PM_CUDA(cudaMemcpyAsync(w.p, weights, (size_t)m * 4,
                                mem == PM_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ws));
      PM_CUDA(cudaEventRecord(wdone, ws));
      const bool skip = (flags & PM_GRAPH_SKIP_SELF_LOOPS) != 0;
      if (skip) PM_CUDA(cudaStreamWaitEvent(g->E.stream, wdone, 0));  // loops drop their weights
      ingest_csr(g, skip, &w);
      finish_graph(g);
      PM_CUDA(cudaStreamWaitEvent(g->E.stream, wdone, 0));
      if (wtype == PM_F32) {
        g->w_f32_out = std::move(w);
        permute_weights_f32(g);
      } else {
        g->w_i32_out = std::move(w);
        permute_weights_i32(g);
      }
      PM_CUDA(cudaStreamSynchronize(ws));
    } catch (...) {
      if (ws) cudaStreamSynchronize(ws);
      if (ws) cudaStreamDestroy(ws);
      if (wdone) cudaEventDestroy(wdone);
      delete g;
      throw;
    }
    cudaStreamDestroy(ws);
    cudaEventDestroy(wdone);
    *out = g;
  });
}

pm_status pm_graph_create_partition(const int32_t *offsets, const int32_t *edges, const void *weights, int wtype,
                                    int64_t n, int64_t m, uint32_t flags, uint32_t mem, int rank, int nranks,
                                    int device, pm_graph **out) {
  return guard(__func__, [&] {
    need(out != nullptr, "out is null");
    *out = nullptr;
    need(n > 0 && n < (1ll << 31) - 1, "n must be in [1, 2^31-2]");
    need(m >= 0 && m < (1ll << 31) - 1, "m must be in [0, 2^31-2]");
    need(offsets != nullptr && (m == 0 || edges != nullptr), "null offsets/edges");
    need(weights == nullptr || wtype == PM_F32 || wtype == PM_I32, "wtype must be PM_F32 or PM_I32");
    need(nranks >= 1 && nranks <= 1024, "nranks must be in [1, 1024]");
    need(rank >= 0 && rank < nranks, "rank out of range");
    check_mem(mem);
    // the edge subset of one rank is not symmetric: kept as a directed graph
    pm_graph *g = new_graph(device, false);
    try {
      g->n = n;
      g->m = m;
      g->out.off.alloc((size_t)(n + 1) * 4);
      g->out.idx.alloc((size_t)std::max<int64_t>(m, 1) * 4);
      to_device(g, g->out.off.p, offsets, (size_t)(n + 1) * 4, mem);
      to_device(g, g->out.idx.p, edges, (size_t)m * 4, mem);
      DevBuf w;
      if (weights) {
        w.alloc((size_t)std::max<int64_t>(m, 1) * 4);
        to_device(g, w.p, weights, (size_t)m * 4, mem);
      }
      ingest_csr(g, (flags & PM_GRAPH_SKIP_SELF_LOOPS) != 0, weights ? &w : nullptr);
      restrict_to_partition(g, rank, nranks, weights ? &w : nullptr);
      finish_graph(g);
      if (weights && wtype == PM_F32) {
        g->w_f32_out = std::move(w);
        permute_weights_f32(g);
      } else if (weights) {
        g->w_i32_out = std::move(w);
        permute_weights_i32(g);
      }
      finish(g);
    } catch (...) {
      delete g;
      throw;
    }
    *out = g;
  });
}

pm_status pm_graph_set_exchange(pm_graph *g, pm_allgather_fn fn, void *user) {
  return guard(__func__, [&] {
    enter(g);
    need(g->is_part, "not a partition graph");
    g->part_fn = fn;
    g->part_user = user;
  });
}

pm_status pm_graph_partition_info(const pm_graph *g, int *rank, int *nranks, int64_t *bounds) {
  return guard(__func__, [&] {
    need(g != nullptr, "null graph handle");
    if (rank) *rank = g->part_rank;
    if (nranks) *nranks = g->part_count;
    if (bounds) {
      if (g->is_part)
        std::copy(g->part_bounds.begin(), g->part_bounds.end(), bounds);
      else {
        bounds[0] = 0;
        bounds[1] = g->n;
      }
    }
  });
}

pm_status pm_graph_load_pbbs(const char *path, uint32_t flags, int device, pm_graph **out) {
  return guard(__func__, [&] {
    need(out != nullptr, "out is null");
    *out = nullptr;
    need(path != nullptr, "null path");
    pm_graph *g = new_graph(device, (flags & PM_GRAPH_SYMMETRIC) != 0);
    try {
      DevBuf w;
      int64_t n = 0, m = 0;
      if (flags & PM_LOAD_DUMP) {
        read_graph_dump(g, path, g->out.off, g->out.idx, n, m);
      } else if (flags & PM_LOAD_BINARY) {
        std::vector<int32_t> off, idx;
        read_pbbs_binary(path, off, idx, n, m);
        g->out.off.alloc((size_t)(n + 1) * 4);
        g->out.idx.alloc((size_t)std::max<int64_t>(m, 1) * 4);
        to_device(g, g->out.off.p, off.data(), (size_t)(n + 1) * 4, PM_MEM_HOST);
        to_device(g, g->out.idx.p, idx.data(), (size_t)m * 4, PM_MEM_HOST);
        finish(g);
      } else {
        parse_pbbs_text(g, path, g->out.off, g->out.idx, w, n, m);
      }
      g->n = n;
      g->m = m;
      ingest_csr(g, (flags & PM_GRAPH_SKIP_SELF_LOOPS) != 0, &w);
      finish_graph(g);
      if (w.p) {
        g->w_i32_out = std::move(w);
        permute_weights_i32(g);
      }
    } catch (...) {
      delete g;
      throw;
    }
    *out = g;
  });
}

pm_status pm_graph_save_dump(pm_graph *g, const char *path) {
  return guard(__func__, [&] {
    enter(g);
    whole_graph(g, "pm_graph_save_dump");
    need(path != nullptr, "null path");
    write_graph_dump(g, path);
  });
}

pm_status pm_graph_create_rmat(int scale, int edge_factor, uint64_t seed, uint32_t flags, int device,
                               pm_graph **out) {
  return guard(__func__, [&] {
    need(out != nullptr, "out is null");
    *out = nullptr;
    need(scale >= 1 && scale <= 28, "scale must be in [1, 28]");
    need(edge_factor >= 1 && edge_factor <= 64, "edge_factor must be in [1, 64]");
    need(((int64_t)edge_factor << scale) * ((flags & PM_GRAPH_SYMMETRIC) ? 2 : 1) < (1ll << 31) - 1,
         "graph exceeds int32 edge offsets");
    pm_graph *g = new_graph(device, (flags & PM_GRAPH_SYMMETRIC) != 0);
    try {
      generate_rmat(g, scale, edge_factor, seed);
      finish_graph(g);
    } catch (...) {
      delete g;
      throw;
    }
    *out = g;
  });
}

pm_status pm_graph_create_er_batch(int count, int64_t n_min, int64_t n_max, int avg_degree,
                                   uint64_t seed, int device, pm_graph **out) {
  return guard(__func__, [&] {
    need(out != nullptr, "out is null");
    *out = nullptr;
    need(count >= 1 && count <= 1 << 20, "count must be in [1, 2^20]");
    need(n_min >= 2 && n_max >= n_min && n_max < (1ll << 30), "need 2 <= n_min <= n_max < 2^30");
    need(avg_degree >= 1 && avg_degree <= 64, "avg_degree must be in [1, 64]");
    pm_graph *g = new_graph(device, false);
    try {
      generate_er_batch(g, count, n_min, n_max, avg_degree, seed);
      finish_graph(g);
    } catch (...) {
      delete g;
      throw;
    }
    *out = g;
  });
}

pm_status pm_graph_set_parts(pm_graph *g, const int64_t *vbase, int count) {
  return guard(__func__, [&] {
    enter(g);
    whole_graph(g, "pm_graph_set_parts");
    need(vbase != nullptr && count >= 1, "need count >= 1 part offsets");
    std::vector<int64_t> v(vbase, vbase + count + 1);
    check_parts(g, v);
    set_parts(g, v);
  });
}

pm_status pm_graph_get_parts(pm_graph *g, int64_t *vbase, int *count) {
  return guard(__func__, [&] {
    need(g != nullptr, "null graph handle");
    const int c = g->parts.empty() ? 0 : (int)g->parts.size() - 1;
    if (count) *count = c;
    if (vbase && c) memcpy(vbase, g->parts.data(), (size_t)(c + 1) * 8);
  });
}

pm_status pm_pagerank_parts(pm_graph *g, int iters, double damping, float *ranks, uint32_t mem) {
  return guard(__func__, [&] {
    enter(g);
    whole_graph(g, "pm_pagerank_parts");
    check_mem(mem);
    need(ranks != nullptr, "null ranks");
    need(iters >= 0, "iters must be >= 0");
    need(!g->parts.empty(), "graph has no parts (pm_graph_set_parts)");
    need(!g->has_self_loops,
         "PageRank needs a graph without self loops (create it with PM_GRAPH_SKIP_SELF_LOOPS)");
    const size_t bytes = (size_t)g->n * 4;
    float *dr = mem == PM_MEM_DEVICE ? ranks : (float *)g->scratch_buf(kSlotOut0, bytes);
    run_pagerank_parts(g, iters, damping, dr);
    if (mem == PM_MEM_HOST) from_device(g, ranks, dr, bytes, mem);
    finish(g);
  });
}

pm_status pm_graph_destroy(pm_graph *g) {
  return guard(__func__, [&] {
    if (!g) return;
    cudaSetDevice(g->device);
    delete g;
  });
}

pm_status pm_graph_info(const pm_graph *g, int64_t *n, int64_t *m, int64_t *max_out_degree) {
  return guard(__func__, [&] {
    need(g != nullptr, "null graph handle");
    if (n) *n = g->n;
    if (m) *m = g->m;
    if (max_out_degree) *max_out_degree = g->max_out_deg;
  });
}

pm_status pm_graph_get_csr(pm_graph *g, int32_t *offsets, int32_t *edges, uint32_t mem) {
  return guard(__func__, [&] {
    enter(g);
    check_mem(mem);
    if (offsets) from_device(g, offsets, g->out.off.p, (size_t)(g->n + 1) * 4, mem);
    if (edges) from_device(g, edges, g->out.idx.p, (size_t)g->m * 4, mem);
    finish(g);
  });
}

pm_status pm_graph_set_weights_i32(pm_graph *g, const int32_t *w, uint32_t mem) {
  return guard(__func__, [&] {
    enter(g);
    whole_graph(g, "pm_graph_set_weights_i32");
    check_mem(mem);
    need(w != nullptr || g->m == 0, "null weights");
    g->w_i32_out.alloc((size_t)std::max<int64_t>(g->m, 1) * 4);
    to_device(g, g->w_i32_out.p, w, (size_t)g->m * 4, mem);
    permute_weights_i32(g);
  });
}

pm_status pm_graph_set_weights_f32(pm_graph *g, const float *w, uint32_t mem) {
  return guard(__func__, [&] {
    enter(g);
    whole_graph(g, "pm_graph_set_weights_f32");
    check_mem(mem);
    need(w != nullptr || g->m == 0, "null weights");
    g->w_f32_out.alloc((size_t)std::max<int64_t>(g->m, 1) * 4);
    to_device(g, g->w_f32_out.p, w, (size_t)g->m * 4, mem);
    permute_weights_f32(g);
  });
}

pm_status pm_graph_gen_weights_i32(pm_graph *g, uint64_t seed, int32_t wmax) {
  return guard(__func__, [&] {
    enter(g);
    whole_graph(g, "pm_graph_gen_weights_i32");
    need(wmax >= 1, "wmax must be >= 1");
    gen_weights(g, seed, wmax, false);
  });
}

pm_status pm_graph_gen_weights_f32(pm_graph *g, uint64_t seed) {
  return guard(__func__, [&] {
    enter(g);
    whole_graph(g, "pm_graph_gen_weights_f32");
    gen_weights(g, seed, 0, true);
  });
}

pm_status pm_graph_get_weights_f32(pm_graph *g, float *w, uint32_t mem) {
  return guard(__func__, [&] {
    enter(g);
    check_mem(mem);
    need(g->w_f32_out.p != nullptr, "graph has no float weights");
    from_device(g, w, g->w_f32_out.p, (size_t)g->m * 4, mem);
    finish(g);
  });
}

pm_status pm_graph_get_weights_i32(pm_graph *g, int32_t *w, uint32_t mem) {
  return guard(__func__, [&] {
    enter(g);
    check_mem(mem);
    need(g->w_i32_out.p != nullptr, "graph has no int weights");
    from_device(g, w, g->w_i32_out.p, (size_t)g->m * 4, mem);
    finish(g);
  });
}

pm_status pm_fill_uniform_f32(pm_graph *g, uint64_t seed, int open_interval, float *out,
                              int64_t count) {
  return guard(__func__, [&] {
    enter(g);
    need(out != nullptr && count >= 0, "bad output");
    fill_uniform(g, seed, open_interval, out, count);
  });
}

pm_status pm_bfs(pm_graph *g, int32_t src, int32_t *parents, int32_t *depth, uint32_t mem,
                 int64_t threshold, pm_traversal_stats *stats) {
  return guard(__func__, [&] {
    enter(g);
    check_mem(mem);
    need(src >= 0 && src < g->n, "source out of range");
    const size_t bytes = (size_t)g->n * 4;
    int32_t *dp = (int32_t *)g->scratch_buf(kSlotOut0, bytes);
    int32_t *dd = (int32_t *)g->scratch_buf(kSlotOut1, bytes);
    run_bfs(g, src, dp, dd, threshold < 0 ? g->m / g->E.tune.bfs_div : threshold, stats);
    if (parents) from_device(g, parents, dp, bytes, mem);
    if (depth) from_device(g, depth, dd, bytes, mem);
    finish(g);
  });
}

pm_status pm_bfs_async(pm_graph *g, int32_t src, int32_t *parents, uint32_t mem, pm_traversal_stats *stats) {
  return guard(__func__, [&] {
    enter(g);
    whole_graph(g, "pm_bfs_async");
    check_mem(mem);
    need(parents != nullptr, "null parents");
    need(src >= 0 && src < g->n, "source out of range");
    const size_t bytes = (size_t)g->n * 4;
    int32_t *dp = mem == PM_MEM_DEVICE ? parents : (int32_t *)g->scratch_buf(kSlotOut0, bytes);
    run_bfs_async(g, src, dp, stats);
    if (mem == PM_MEM_HOST) from_device(g, parents, dp, bytes, mem);
    finish(g);
  });
}

// Checks k and the sources (read back when they live on the device) and
// stages them in the handle's scratch; returns their device copy.
static const int32_t *stage_sources(pm_graph *g, const int32_t *sources, int k, uint32_t mem) {
  need(k >= 1 && k <= 64, "k must be in [1, 64]");
  int32_t hs[64];
  if (mem == PM_MEM_DEVICE)
    PM_CUDA(cudaMemcpy(hs, sources, (size_t)k * 4, cudaMemcpyDeviceToHost));
  else
    memcpy(hs, sources, (size_t)k * 4);
  for (int l = 0; l < k; ++l) need(hs[l] >= 0 && hs[l] < g->n, "source out of range");
  int32_t *ds = (int32_t *)g->scratch_buf(kSlotIn0, 64 * 4);
  PM_CUDA(cudaMemcpyAsync(ds, hs, (size_t)k * 4, cudaMemcpyHostToDevice, g->E.stream));
  return ds;
}

pm_status pm_bfs_multi(pm_graph *g, const int32_t *sources, int k, int32_t *depth, uint32_t mem,
                       int64_t threshold, pm_traversal_stats *stats) {
  return guard(__func__, [&] {
    enter(g);
    whole_graph(g, "pm_bfs_multi");
    check_mem(mem);
    need(sources != nullptr && depth != nullptr, "null sources/depth");
    const int32_t *ds = stage_sources(g, sources, k, mem);
    const size_t bytes = (size_t)g->n * k * 4;
    int32_t *dd = mem == PM_MEM_DEVICE ? depth : (int32_t *)g->scratch_buf(kSlotOut0, bytes);
    run_msbfs(g, ds, k, dd, threshold < 0 ? g->m / g->E.tune.multi_div : threshold, stats);
    if (mem == PM_MEM_HOST) from_device(g, depth, dd, bytes, mem);
    finish(g);
  });
}

pm_status pm_bellman_ford_multi(pm_graph *g, const int32_t *sources, int k, int32_t *dist, uint32_t mem,
                                int64_t threshold, pm_traversal_stats *stats) {
  return guard(__func__, [&] {
    enter(g);
    whole_graph(g, "pm_bellman_ford_multi");
    check_mem(mem);
    need(sources != nullptr && dist != nullptr, "null sources/dist");
    need(g->w_i32_out.p != nullptr, "graph has no int32 weights (pm_graph_set_weights_i32)");
    const int32_t *ds = stage_sources(g, sources, k, mem);
    const size_t bytes = (size_t)g->n * k * 4;
    int32_t *dd = mem == PM_MEM_DEVICE ? dist : (int32_t *)g->scratch_buf(kSlotOut0, bytes);
    run_bf_multi(g, ds, k, dd, threshold < 0 ? g->m / g->E.tune.multi_div : threshold, stats);
    if (mem == PM_MEM_HOST) from_device(g, dist, dd, bytes, mem);
    finish(g);
  });
}

pm_status pm_components(pm_graph *g, int32_t *labels, uint32_t mem, int64_t threshold,
                        pm_traversal_stats *stats) {
  return guard(__func__, [&] {
    enter(g);
    check_mem(mem);
    need(labels != nullptr, "null labels");
    const size_t bytes = (size_t)g->n * 4;
    int32_t *dl = mem == PM_MEM_DEVICE ? labels : (int32_t *)g->scratch_buf(kSlotOut0, bytes);
    run_cc(g, dl, threshold < 0 ? g->m / g->E.tune.cc_div : threshold, stats);
    if (mem == PM_MEM_HOST) from_device(g, labels, dl, bytes, mem);
    finish(g);
  });
}

pm_status pm_bellman_ford(pm_graph *g, int32_t src, int32_t *dist, uint32_t mem, int64_t threshold,
                          pm_traversal_stats *stats) {
  return guard(__func__, [&] {
    enter(g);
    check_mem(mem);
    need(dist != nullptr, "null dist");
    need(src >= 0 && src < g->n, "source out of range");
    need(g->w_i32_out.p != nullptr, "graph has no int32 weights (pm_graph_set_weights_i32)");
    const size_t bytes = (size_t)g->n * 4;
    int32_t *dd = mem == PM_MEM_DEVICE ? dist : (int32_t *)g->scratch_buf(kSlotOut0, bytes);
    run_bellman_ford(g, src, dd, threshold < 0 ? g->m / g->E.tune.bf_div : threshold, stats);
    if (mem == PM_MEM_HOST) from_device(g, dist, dd, bytes, mem);
    finish(g);
  });
}

pm_status pm_pagerank(pm_graph *g, int iters, double damping, int dtype, void *ranks, uint32_t mem,
                      double *resid) {
  return guard(__func__, [&] {
    enter(g);
    check_mem(mem);
    need(ranks != nullptr, "null ranks");
    need(iters >= 0, "iters must be >= 0");
    need(dtype == PM_F32 || dtype == PM_F64, "dtype must be PM_F32 or PM_F64");
    need(!g->has_self_loops,
         "PageRank needs a graph without self loops (create it with PM_GRAPH_SKIP_SELF_LOOPS)");
    const size_t es = dtype == PM_F64 ? 8 : 4;
    const size_t bytes = (size_t)g->n * es;
    void *dr = mem == PM_MEM_DEVICE ? ranks : g->scratch_buf(kSlotOut0, bytes);
    double *dres = resid ? (double *)g->scratch_buf(kSlotAux, (size_t)std::max(iters, 1) * 8) : nullptr;
    if (dtype == PM_F64)
      run_pagerank<double>(g, iters, damping, (double *)dr, dres);
    else
      run_pagerank<float>(g, iters, damping, (float *)dr, dres);
    if (mem == PM_MEM_HOST) from_device(g, ranks, dr, bytes, mem);
    if (resid && iters > 0) from_device(g, resid, dres, (size_t)iters * 8, PM_MEM_HOST);
    finish(g);
  });
}

pm_status pm_pagerank_delta(pm_graph *g, int iters, double damping, double epsilon, int dtype, void *ranks,
                            uint32_t mem, int64_t threshold, pm_traversal_stats *stats) {
  return guard(__func__, [&] {
    enter(g);
    whole_graph(g, "pm_pagerank_delta");
    check_mem(mem);
    need(ranks != nullptr, "null ranks");
    need(iters >= 1, "iters must be >= 1 (the reference loops until maxIter)");
    need(damping > 0.0 && damping < 1.0, "damping must be in (0, 1)");
    need(epsilon >= 0.0 && std::isfinite(epsilon), "epsilon must be finite and >= 0");
    need(dtype == PM_F32 || dtype == PM_F64, "dtype must be PM_F32 or PM_F64");
    need(!g->has_self_loops,
         "PageRankDelta needs a graph without self loops (create it with PM_GRAPH_SKIP_SELF_LOOPS)");
    const size_t bytes = (size_t)g->n * (dtype == PM_F64 ? 8 : 4);
    void *dr = mem == PM_MEM_DEVICE ? ranks : g->scratch_buf(kSlotOut0, bytes);
    const int64_t thr = threshold < 0 ? g->m / 20 : threshold;
    if (dtype == PM_F64)
      run_pagerank_delta<double>(g, iters, damping, epsilon, (double *)dr, thr, stats);
    else
      run_pagerank_delta<float>(g, iters, damping, epsilon, (float *)dr, thr, stats);
    if (mem == PM_MEM_HOST) from_device(g, ranks, dr, bytes, mem);
    finish(g);
  });
}

pm_status pm_ppr(pm_graph *g, const int32_t *seeds, int k, int iters, double damping, float *out,
                 uint32_t mem) {
  return guard(__func__, [&] {
    enter(g);
    whole_graph(g, "pm_ppr");
    check_mem(mem);
    need(seeds != nullptr && out != nullptr, "null seeds/out");
    need(k >= 1 && k <= 32, "k must be in [1, 32]");
    need(iters >= 0, "iters must be >= 0");
    need(!g->has_self_loops,
         "PageRank needs a graph without self loops (create it with PM_GRAPH_SKIP_SELF_LOOPS)");
    int32_t hs[32];
    if (mem == PM_MEM_DEVICE)
      PM_CUDA(cudaMemcpy(hs, seeds, (size_t)k * 4, cudaMemcpyDeviceToHost));
    else
      memcpy(hs, seeds, (size_t)k * 4);
    for (int j = 0; j < k; ++j) need(hs[j] >= 0 && hs[j] < g->n, "seed out of range");
    int32_t *ds = (int32_t *)g->scratch_buf(kSlotIn0, 32 * 4);
    PM_CUDA(cudaMemcpyAsync(ds, hs, (size_t)k * 4, cudaMemcpyHostToDevice, g->E.stream));
    const size_t bytes = (size_t)g->n * k * 4;
    float *dout = mem == PM_MEM_DEVICE ? out : (float *)g->scratch_buf(kSlotOut0, bytes);
    run_ppr(g, ds, k, iters, damping, dout);
    if (mem == PM_MEM_HOST) from_device(g, out, dout, bytes, mem);
    finish(g);
  });
}

extern "C++" {
template <class T>
static void spmv_call(pm_graph *g, const T *x0, int iters, T *y, uint32_t mem, double *norm1) {
  enter(g);
  check_mem(mem);
  need(x0 != nullptr && y != nullptr, "null x0/y");
  need(iters >= 0, "iters must be >= 0");
  need(g->w_f32_out.p != nullptr, "graph has no float weights (pm_graph_set_weights_f32)");
  const size_t bytes = (size_t)g->n * sizeof(T);
  const T *dx = x0;
  if (mem == PM_MEM_HOST) {
    T *t = (T *)g->scratch_buf(kSlotIn0, bytes);
    to_device(g, t, x0, bytes, mem);
    dx = t;
  }
  T *dy = mem == PM_MEM_DEVICE ? y : (T *)g->scratch_buf(kSlotOut0, bytes);
  double *dn = norm1 ? (double *)g->scratch_buf(kSlotAux, (size_t)std::max(iters, 1) * 8) : nullptr;
  run_spmv<T>(g, dx, iters, dy, dn);
  if (mem == PM_MEM_HOST) from_device(g, y, dy, bytes, mem);
  if (norm1 && iters > 0) from_device(g, norm1, dn, (size_t)iters * 8, PM_MEM_HOST);
  finish(g);
}
}  // extern "C++"

pm_status pm_spmv(pm_graph *g, const float *x0, int iters, float *y, uint32_t mem, double *norm1) {
  return guard(__func__, [&] { spmv_call<float>(g, x0, iters, y, mem, norm1); });
}

pm_status pm_spmv_f64(pm_graph *g, const double *x0, int iters, double *y, uint32_t mem, double *norm1) {
  return guard(__func__, [&] { spmv_call<double>(g, x0, iters, y, mem, norm1); });
}

static void need_weights_f32(pm_graph *g) {
  need(g->w_f32_out.p != nullptr, "graph has no float weights (pm_graph_set_weights_f32)");
}

// Device copy of a float input (or the pointer itself for device memory).
static const float *stage_in(pm_graph *g, const float *x, size_t count, int slot, uint32_t mem) {
  if (mem == PM_MEM_DEVICE) return x;
  float *t = (float *)g->scratch_buf(slot, count * 4);
  to_device(g, t, x, count * 4, mem);
  return t;
}

pm_status pm_weighted_pagerank(pm_graph *g, double damping, double tol, int max_iters, float *p,
                               uint32_t mem, int *iters, double *resid) {
  return guard(__func__, [&] {
    enter(g);
    whole_graph(g, "pm_weighted_pagerank");
    check_mem(mem);
    need(p != nullptr, "null p");
    need(max_iters >= 1 && tol >= 0, "need max_iters >= 1 and tol >= 0");
    need_weights_f32(g);
    const size_t bytes = (size_t)g->n * 4;
    float *dp = mem == PM_MEM_DEVICE ? p : (float *)g->scratch_buf(kSlotOut0, bytes);
    const int it = run_weighted_pagerank(g, damping, tol, max_iters, dp, resid);
    if (iters) *iters = it;
    if (mem == PM_MEM_HOST) from_device(g, p, dp, bytes, mem);
    finish(g);
  });
}

pm_status pm_pagerank_adjoint(pm_graph *g, double damping, double tol, int max_iters, const float *p,
                              const float *grad_p, float *dw, float *lambda, uint32_t mem, int *iters,
                              double *resid) {
  return guard(__func__, [&] {
    enter(g);
    whole_graph(g, "pm_pagerank_adjoint");
    check_mem(mem);
    need(p != nullptr && grad_p != nullptr && dw != nullptr, "null p/grad_p/dw");
    need(max_iters >= 1 && tol >= 0, "need max_iters >= 1 and tol >= 0");
    need_weights_f32(g);
    const size_t n = (size_t)g->n, m = (size_t)g->m;
    const float *dp = stage_in(g, p, n, kSlotIn0, mem);
    const float *dg = stage_in(g, grad_p, n, kSlotIn1, mem);
    float *ddw = mem == PM_MEM_DEVICE ? dw : (float *)g->scratch_buf(kSlotOut0, std::max<size_t>(m, 1) * 4);
    float *dl = lambda == nullptr ? nullptr
                : mem == PM_MEM_DEVICE ? lambda : (float *)g->scratch_buf(kSlotOut1, n * 4);
    const int it = run_pagerank_adjoint(g, damping, tol, max_iters, dp, dg, ddw, dl, resid);
    if (iters) *iters = it;
    if (mem == PM_MEM_HOST) {
      from_device(g, dw, ddw, m * 4, mem);
      if (lambda) from_device(g, lambda, dl, n * 4, mem);
    }
    finish(g);
  });
}

pm_status pm_spmv_backward(pm_graph *g, const float *x, const float *grad_y, float *dx, float *dw,
                           uint32_t mem) {
  return guard(__func__, [&] {
    enter(g);
    whole_graph(g, "pm_spmv_backward");
    check_mem(mem);
    need(x != nullptr && grad_y != nullptr, "null x/grad_y");
    need_weights_f32(g);
    const size_t n = (size_t)g->n, m = (size_t)g->m;
    const float *dx_in = stage_in(g, x, n, kSlotIn0, mem);
    const float *dgy = stage_in(g, grad_y, n, kSlotIn1, mem);
    float *ddx = dx == nullptr ? nullptr : mem == PM_MEM_DEVICE ? dx : (float *)g->scratch_buf(kSlotOut0, n * 4);
    float *ddw = dw == nullptr ? nullptr
                 : mem == PM_MEM_DEVICE ? dw : (float *)g->scratch_buf(kSlotOut1, std::max<size_t>(m, 1) * 4);
    run_spmv_backward(g, dx_in, dgy, ddx, ddw);
    if (mem == PM_MEM_HOST) {
      if (dx) from_device(g, dx, ddx, n * 4, mem);
      if (dw) from_device(g, dw, ddw, m * 4, mem);
    }
    finish(g);
  });
}

pm_status pm_graph_gen_weights_lognormal(pm_graph *g, uint64_t seed) {
  return guard(__func__, [&] {
    enter(g);
    whole_graph(g, "pm_graph_gen_weights_lognormal");
    gen_weights_lognormal(g, seed);
  });
}

extern "C++" {
template <class T>
static void bp_call(pm_graph *g, const T *prior, const T *psi, int iters, T *log_prod, uint32_t mem) {
  enter(g);
  check_mem(mem);
  need(prior != nullptr && psi != nullptr && log_prod != nullptr, "null prior/psi/log_prod");
  need(iters >= 0, "iters must be >= 0");
  const uintptr_t align = 2 * sizeof(T) - 1;
  need(mem == PM_MEM_HOST || (((uintptr_t)prior | (uintptr_t)log_prod) & align) == 0,
       sizeof(T) == 4 ? "device prior/log_prod must be 8-byte aligned"
                      : "device prior/log_prod must be 16-byte aligned");
  const size_t bytes = (size_t)g->n * 2 * sizeof(T);
  T hpsi[4];
  if (mem == PM_MEM_DEVICE) {
    PM_CUDA(cudaMemcpy(hpsi, psi, sizeof hpsi, cudaMemcpyDeviceToHost));
  } else {
    memcpy(hpsi, psi, sizeof hpsi);
  }
  for (T p : hpsi) need(p > T(0) && std::isfinite(p), "psi entries must be positive and finite");
  const T *dp = prior;
  if (mem == PM_MEM_HOST) {
    T *t = (T *)g->scratch_buf(kSlotIn0, bytes);
    to_device(g, t, prior, bytes, mem);
    dp = t;
  }
  T *dout = mem == PM_MEM_DEVICE ? log_prod : (T *)g->scratch_buf(kSlotOut0, bytes);
  run_bp<T>(g, dp, hpsi, iters, dout);
  if (mem == PM_MEM_HOST) from_device(g, log_prod, dout, bytes, mem);
  finish(g);
}
}  // extern "C++"

pm_status pm_bp(pm_graph *g, const float *prior, const float *psi, int iters, float *log_prod,
                uint32_t mem) {
  return guard(__func__, [&] { bp_call<float>(g, prior, psi, iters, log_prod, mem); });
}

pm_status pm_bp_f64(pm_graph *g, const double *prior, const double *psi, int iters, double *log_prod,
                    uint32_t mem) {
  return guard(__func__, [&] { bp_call<double>(g, prior, psi, iters, log_prod, mem); });
}

pm_status pm_timer_begin(pm_graph *g) {
  return guard(__func__, [&] {
    enter(g);
    PM_CUDA(cudaEventRecord(g->ev0, g->E.stream));
  });
}

pm_status pm_timer_end(pm_graph *g, float *ms) {
  return guard(__func__, [&] {
    enter(g);
    PM_CUDA(cudaEventRecord(g->ev1, g->E.stream));
    PM_CUDA(cudaEventSynchronize(g->ev1));
    float t = 0.f;
    PM_CUDA(cudaEventElapsedTime(&t, g->ev0, g->ev1));
    if (ms) *ms = t;
  });
}

pm_status pm_profile_enable(pm_graph *g, int enable) {
  return guard(__func__, [&] {
    enter(g);
    g->E.prof.enabled = enable != 0;
  });
}

pm_status pm_profile_read(pm_graph *g, const char *tag, double *total_ms, int64_t *passes,
                          int reset) {
  return guard(__func__, [&] {
    enter(g);
    need(tag != nullptr, "null tag");
    finish(g);
    Profiler &P = g->E.prof;
    P.fold();
    double tot = 0.0;
    int64_t cnt = 0;
    for (auto &t : P.totals)
      if (t.tag == tag) {
        tot = t.ms;
        cnt = t.passes;
      }
    if (total_ms) *total_ms = tot;
    if (passes) *passes = cnt;
    if (reset) P.totals.clear();
  });
}

pm_status pm_graph_set_stream(pm_graph *g, void *stream) {
  return guard(__func__, [&] {
    enter(g);
    finish(g);  // nothing of this handle stays in flight on the old stream
    g->E.release_graphs();  // captured loops were recorded for the old stream's work
    g->E.stream = stream ? (cudaStream_t)stream : g->own_stream;
    set_alloc_ctx(AllocCtx{g->E.stream, false});
  });
}

pm_status pm_graph_set_tunable(pm_graph *g, int key, int64_t value) {
  return guard(__func__, [&] {
    if (g) enter(g);
    set_tunable(g, key, value);
  });
}

pm_status pm_graph_get_tunable(pm_graph *g, int key, int64_t *value) {
  return guard(__func__, [&] {
    if (g) enter(g);
    need(value != nullptr, "null value");
    *value = get_tunable(g, key);
  });
}

pm_status pm_tune(pm_graph *g, int app, pm_tune_report *report) {
  return guard(__func__, [&] {
    enter(g);
    whole_graph(g, "pm_tune");
    tune(g, &app, 1, report);
    finish(g);
  });
}

pm_status pm_tune_mix(pm_graph *g, const int *apps, int count, pm_tune_report *report) {
  return guard(__func__, [&] {
    enter(g);
    whole_graph(g, "pm_tune_mix");
    need(apps != nullptr, "null apps");
    tune(g, apps, count, report);
    finish(g);
  });
}

pm_status pm_set_memory_cache(int64_t max_bytes) {
  return guard(__func__, [&] { set_memory_cache(max_bytes); });
}

pm_status pm_release_memory_cache(void) {
  return guard(__func__, [&] { release_memory_cache(); });
}

pm_status pm_memory_cache_info(int64_t *cached_bytes) {
  return guard(__func__, [&] {
    need(cached_bytes != nullptr, "null cached_bytes");
    *cached_bytes = memory_cached();
  });
}

pm_status pm_host_alloc(uint64_t bytes, void **out) {
  return guard(__func__, [&] {
    need(out != nullptr, "out is null");
    *out = nullptr;
    PM_CUDA(cudaMallocHost(out, bytes ? bytes : 1));
  });
}

pm_status pm_host_free(void *p) {
  return guard(__func__, [&] {
    if (p) PM_CUDA(cudaFreeHost(p));
  });
}

pm_status pm_test_fail_alloc_after(int64_t k) {
  return guard(__func__, [&] { set_alloc_fail_after((long long)k); });
}

pm_status pm_test_wait_timeout(int device, int32_t max_polls) {
  return guard(__func__, [&] {
    use_device(device);
    need(max_polls >= 1 && max_polls <= kHeavyWaitSpins, "max_polls must be in [1, 2^22]");
    DevBuf b(8);  // [0] the flag nothing sets, [1] the error word
    PM_CUDA(cudaMemset(b.p, 0, 8));
    PM_LAUNCH(k_test_wait, 1, 32, 0, (cudaStream_t)0, b.as<int32_t>(), reinterpret_cast<unsigned *>(b.as<int32_t>() + 1),
              max_polls);
    unsigned err = 0;
    PM_CUDA(cudaMemcpy(&err, b.as<int32_t>() + 1, 4, cudaMemcpyDeviceToHost));
    if (err & kErrTimeout)
      fail(PM_ERR_TIMEOUT, "a bounded device wait ran out after " + std::to_string(max_polls) + " polls");
  });
}

int64_t pm_kernel_launches(int reset) { return (int64_t)launches(reset != 0); }

const char *pm_last_error(void) { return t_last_error.c_str(); }

const char *pm_version(void) { return "polymer_b200 0.1 (sm_100a)"; }

}  // extern "C"
