// pm_adjoint.cu -- weighted PageRank fixed point, its adjoint, and the
// backward pass of weighted SpMV, all on the pull-reduce engine.
//
// Weights W are per CSR edge (pm_graph_set_weights_f32).  With
// (A_W^T x)[v] = sum_{e = s->v} W_e x[s]:
//   forward   p = damping * A_W^T p + (1 - damping)/n      (pull over the CSC)
//   adjoint   lambda = damping * A_W lambda + g            (pull over the CSR)
//             dL/dW_e = damping * lambda[v] * p[s]         (edge pass)
//   SpMV      y = A_W^T x;  dx = A_W gy (pull over the CSR), dW_e = gy[v] x[s]
// Fixed points iterate until sum|x_{t+1} - x_t| <= tol * sum|x_{t+1}|; the
// two sums are reduced in FP64 on the device and read back once per pass.
#include "pm_graph.cuh"

namespace pm {

// Weighted PageRank pass: p_next[v] = damping * sum W_e p[s] + (1-damping)/n.
struct WPR_F {
  const float *p;
  float *p_next;
  float damping, base;
  using Acc = float;
  __device__ __forceinline__ bool cond(int) const { return true; }
  __device__ __forceinline__ Acc identity() const { return 0.0f; }
  __device__ __forceinline__ Acc edge(int s, int, float w) const { return w * __ldg(p + s); }
  __device__ __forceinline__ Acc combine(Acc a, Acc b) const { return a + b; }
  __device__ __forceinline__ bool commit(int v, Acc acc, double2 &r) const {
    const float x = damping * acc + base;
    r.x += fabs((double)x - (double)p[v]);
    r.y += fabs((double)x);
    p_next[v] = x;
    return false;
  }
};

// Adjoint pass over the CSR (rows are sources): l_next[s] = damping * sum
// W_e l[v] + g[s].  In the transposed view "s" of edge() is the CSR
// destination v.
struct ADJ_F {
  const float *l;
  float *l_next;
  const float *g;
  float damping;
  using Acc = float;
  __device__ __forceinline__ bool cond(int) const { return true; }
  __device__ __forceinline__ Acc identity() const { return 0.0f; }
  __device__ __forceinline__ Acc edge(int v, int, float w) const { return w * __ldg(l + v); }
  __device__ __forceinline__ Acc combine(Acc a, Acc b) const { return a + b; }
  __device__ __forceinline__ bool commit(int s, Acc acc, double2 &r) const {
    const float x = damping * acc + __ldg(g + s);
    r.x += fabs((double)x - (double)l[s]);
    r.y += fabs((double)x);
    l_next[s] = x;
    return false;
  }
};

// SpMV backward, dx part: dx[s] = sum W_e gy[v] over the CSR.
struct SPMVB_F {
  const float *gy;
  float *dx;
  using Acc = float;
  __device__ __forceinline__ bool cond(int) const { return true; }
  __device__ __forceinline__ Acc identity() const { return 0.0f; }
  __device__ __forceinline__ Acc edge(int v, int, float w) const { return w * __ldg(gy + v); }
  __device__ __forceinline__ Acc combine(Acc a, Acc b) const { return a + b; }
  __device__ __forceinline__ bool commit(int s, Acc acc, double2 &) const {
    dx[s] = acc;
    return false;
  }
};

// dw[e] = scale * a[idx[e]] * b[src[e]] for every CSR edge.
__global__ void k_edge_product(const int32_t *__restrict__ idx, const int32_t *__restrict__ src,
                               const float *__restrict__ a, const float *__restrict__ b, float scale,
                               int64_t m, float *__restrict__ dw) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += stride)
    dw[e] = scale * __ldg(a + __ldg(idx + e)) * __ldg(b + __ldg(src + e));
}

__global__ void k_fill_f32(float *x, int64_t n, float v) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) x[i] = v;
}

void ensure_out_src(pm_graph *g);

// The engine pulls over g.in; while a CsrPull is alive it pulls over the
// CSR instead (rows are sources, edge() sees the CSR destination).
struct CsrPull {
  Engine &E;
  GraphView saved;
  explicit CsrPull(Engine &e) : E(e), saved(e.g) { E.g.in = saved.out; }
  ~CsrPull() { E.g = saved; }
};

// Iterates launch(cur, next) until the relative L1 change is <= tol; returns
// the number of passes, the final relative change in *resid, and leaves the
// result in cur.
template <class Launch>
static int iterate_to_tol(Engine &E, float *&cur, float *&next, double tol, int max_iters,
                          double *resid, const char *tag, Launch launch) {
  int it = 0;
  double rel = 0.0;
  while (it < max_iters) {
    PM_CUDA(cudaMemsetAsync(E.d_cnt, 0, sizeof(Counters), E.stream));
    E.prof.begin(tag, E.stream);
    launch(cur, next);
    E.prof.end(E.stream);
    const Counters *h = E.read_counters();
    rel = h[0].daux2 > 0 ? h[0].daux / h[0].daux2 : 0.0;
    std::swap(cur, next);
    ++it;
    if (rel <= tol) break;
  }
  if (resid) *resid = rel;
  return it;
}

int run_weighted_pagerank(pm_graph *g, double damping, double tol, int max_iters, float *d_p,
                          double *resid) {
  Engine &E = g->E;
  const int64_t n = g->n;
  float *a = (float *)g->scratch_buf(0, (size_t)n * 4);
  float *b = (float *)g->scratch_buf(1, (size_t)n * 4);
  PM_LAUNCH(k_fill_f32, E.grid_for(n, 256, 8), 256, 0, E.stream, a, n, (float)(1.0 / (double)n));
  const WPair *w_in = ensure_f32_pairs(g);
  const float base = (float)((1.0 - damping) / (double)n);
  const int it = iterate_to_tol(E, a, b, tol, max_iters, resid, "weighted_pagerank",
                                [&](float *cur, float *nxt) {
                                  launch_pull_reduce<WPair>(E, WPR_F{cur, nxt, (float)damping, base},
                                                            w_in, nullptr, E.d_cnt);
                                });
  PM_CUDA(cudaMemcpyAsync(d_p, a, (size_t)n * 4, cudaMemcpyDeviceToDevice, E.stream));
  return it;
}

int run_pagerank_adjoint(pm_graph *g, double damping, double tol, int max_iters, const float *d_p,
                         const float *d_g, float *d_dw, float *d_lambda, double *resid) {
  Engine &E = g->E;
  const int64_t n = g->n, m = g->m;
  ensure_out_src(g);
  float *a = (float *)g->scratch_buf(0, (size_t)n * 4);
  float *b = (float *)g->scratch_buf(1, (size_t)n * 4);
  PM_CUDA(cudaMemcpyAsync(a, d_g, (size_t)n * 4, cudaMemcpyDeviceToDevice, E.stream));
  const WPair *w_out = ensure_f32_pairs(g, true);
  int it = 0;
  {
    CsrPull view(E);
    it = iterate_to_tol(E, a, b, tol, max_iters, resid, "pagerank_adjoint", [&](float *cur, float *nxt) {
      launch_pull_reduce<WPair>(E, ADJ_F{cur, nxt, d_g, (float)damping}, w_out, nullptr, E.d_cnt);
    });
  }
  E.prof.begin("pagerank_adjoint_dw", E.stream);
  if (m)
    PM_LAUNCH(k_edge_product, E.grid_for(m, 256, 8), 256, 0, E.stream, E.g.out.idx,
              g->out_src.as<int32_t>(), a, d_p, (float)damping, m, d_dw);
  E.prof.end(E.stream);
  if (d_lambda) PM_CUDA(cudaMemcpyAsync(d_lambda, a, (size_t)n * 4, cudaMemcpyDeviceToDevice, E.stream));
  return it;
}

void run_spmv_backward(pm_graph *g, const float *d_x, const float *d_gy, float *d_dx, float *d_dw) {
  Engine &E = g->E;
  const int64_t m = g->m;
  ensure_out_src(g);
  const WPair *w_out = d_dx ? ensure_f32_pairs(g, true) : nullptr;
  PM_CUDA(cudaMemsetAsync(E.d_cnt, 0, sizeof(Counters), E.stream));
  E.prof.begin("spmv_backward", E.stream);
  if (d_dx) {
    CsrPull view(E);
    launch_pull_reduce<WPair>(E, SPMVB_F{d_gy, d_dx}, w_out, nullptr, E.d_cnt);
  }
  if (d_dw && m)
    PM_LAUNCH(k_edge_product, E.grid_for(m, 256, 8), 256, 0, E.stream, E.g.out.idx,
              g->out_src.as<int32_t>(), d_gy, d_x, 1.0f, m, d_dw);
  E.prof.end(E.stream);
}

}  // namespace pm
