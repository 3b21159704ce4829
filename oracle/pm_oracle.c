/*
 * pm_oracle.c -- CPU restatement of Polymer's hot path (TEST INFRASTRUCTURE).
 *
 * This file is the checker for the CUDA engine, never part of it: only the
 * tests, the smoke check and the CPU-baseline leg of the benchmark load it.
 * Every algorithm follows the reference application it cites, step by step,
 * in FP64 (or exact integers), with every sum in a fixed order, so that its
 * results are deterministic.  The value loops at scale (PageRank, SpMV, BP,
 * PPR) run their push passes as pulls over the transpose, destinations in
 * parallel (OpenMP): each destination still adds its in-neighbours'
 * contributions in ascending source order, the order of the sequential push,
 * so the results are bit-identical to it whatever the thread count.  Parity of this restatement with the compiled reference is
 * pinned by tests that run the reference binaries built from the original
 * sources (recipe in oracle/Makefile) on the same PBBS files.
 *
 * Graphs are CSR: off[n+1] (int32), idx[m] (int32), edges sorted by source
 * and, within a source, by destination.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define PMO_API __attribute__((visibility("default")))

/* ------------------------------------------------------------------------ */
/* Counter-based random numbers: the SplitMix64 output function applied to  */
/* seed + (c + 1) * golden-ratio increment (Steele, Lea & Flood, 2014).      */
/* The GPU generator evaluates the same function, so both sides build the    */
/* identical synthetic graph from (scale, edge factor, seed).                */
/* ------------------------------------------------------------------------ */
PMO_API uint64_t pmo_hash(uint64_t seed, uint64_t c) {
  uint64_t z = seed + (c + 1ull) * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

/* R-MAT quadrant thresholds on a 24-bit uniform draw:
 * a = 0.57, a+b = 0.76, a+b+c = 0.95 (times 2^24, truncated). */
#define PMO_RMAT_A 9563013u
#define PMO_RMAT_AB 12750684u
#define PMO_RMAT_ABC 15938355u

/* Raw R-MAT edge k as a 64-bit key (src << 32 | dst).  One draw per level,
 * most significant bit first: quadrant a=(0,0), b=(0,1), c=(1,0), d=(1,1). */
PMO_API uint64_t pmo_rmat_edge(int scale, uint64_t seed, uint64_t k) {
  uint32_t s = 0, d = 0;
  for (int l = 0; l < scale; ++l) {
    uint32_t u = (uint32_t)(pmo_hash(seed, k * (uint64_t)scale + (uint64_t)l) >> 40);
    uint32_t row = u >= PMO_RMAT_AB;
    uint32_t col = (u >= PMO_RMAT_A && u < PMO_RMAT_AB) || u >= PMO_RMAT_ABC;
    s = (s << 1) | row;
    d = (d << 1) | col;
  }
  return ((uint64_t)s << 32) | d;
}

static void radix_sort_u64(uint64_t *a, int64_t n) {
  uint64_t *tmp = (uint64_t *)malloc((size_t)(n > 0 ? n : 1) * sizeof(uint64_t));
  int64_t *cnt = (int64_t *)malloc(65536 * sizeof(int64_t));
  for (int pass = 0; pass < 4; ++pass) {
    int sh = pass * 16;
    memset(cnt, 0, 65536 * sizeof(int64_t));
    for (int64_t i = 0; i < n; ++i) cnt[(a[i] >> sh) & 0xFFFF]++;
    int64_t acc = 0;
    for (int b = 0; b < 65536; ++b) { int64_t c = cnt[b]; cnt[b] = acc; acc += c; }
    for (int64_t i = 0; i < n; ++i) tmp[cnt[(a[i] >> sh) & 0xFFFF]++] = a[i];
    uint64_t *t = a; a = tmp; tmp = t;
  }
  /* four passes: the sorted data is back in the caller's buffer */
  free(tmp);
  free(cnt);
}

/* Sort + dedup edge keys in place, drop self loops, optionally add reverse
 * edges first (keys must then have room for 2*cnt entries).  Writes the CSR
 * offsets (n+1) and returns m; the destinations are written to idx. */
PMO_API int64_t pmo_keys_to_csr(uint64_t *keys, int64_t cnt, int64_t n, int symmetric,
                                int32_t *off, int32_t *idx) {
  int64_t k = 0;
  for (int64_t i = 0; i < cnt; ++i) {
    uint32_t s = (uint32_t)(keys[i] >> 32), d = (uint32_t)keys[i];
    if (s == d) continue;
    keys[k++] = keys[i];
  }
  if (symmetric) {
    int64_t base = k;
    for (int64_t i = 0; i < base; ++i) {
      uint64_t s = keys[i] >> 32, d = keys[i] & 0xFFFFFFFFull;
      keys[k++] = (d << 32) | s;
    }
  }
  radix_sort_u64(keys, k);
  int64_t m = 0;
  for (int64_t i = 0; i < k; ++i)
    if (i == 0 || keys[i] != keys[i - 1]) keys[m++] = keys[i];
  for (int64_t v = 0; v <= n; ++v) off[v] = 0;
  for (int64_t e = 0; e < m; ++e) {
    off[(keys[e] >> 32) + 1]++;
    idx[e] = (int32_t)(keys[e] & 0xFFFFFFFFull);
  }
  for (int64_t v = 0; v < n; ++v) off[v + 1] += off[v];
  return m;
}

/* Convenience: generate the whole R-MAT graph (n = 2^scale, n*ef draws).
 * idx must hold (symmetric ? 2 : 1) * n * ef entries. */
PMO_API int64_t pmo_rmat_graph(int scale, int ef, uint64_t seed, int symmetric,
                               int32_t *off, int32_t *idx) {
  int64_t n = (int64_t)1 << scale;
  int64_t draws = n * ef;
  uint64_t *keys = (uint64_t *)malloc((size_t)draws * (symmetric ? 2 : 1) * sizeof(uint64_t));
  for (int64_t k = 0; k < draws; ++k) keys[k] = pmo_rmat_edge(scale, seed, (uint64_t)k);
  int64_t m = pmo_keys_to_csr(keys, draws, n, symmetric, off, idx);
  free(keys);
  return m;
}

/* Batch of `count` directed Erdos-Renyi graphs as one disjoint union:      */
/* graph i has n_i = floor(exp(ln n_min + u_i (ln n_max - ln n_min))) with   */
/* u_i = (hash(seed, i) >> 11) * 2^-53 (log-uniform), and n_i * avg_degree   */
/* draws (src, dst) = (h >> 32, h & 0xffffffff) mod n_i with h = hash(seed2, */
/* running draw index), seed2 = seed ^ 0xE5E5E5E5; ids offset by vbase[i];   */
/* self loops and duplicates removed, sorted.  vbase gets count+1 entries.   */
PMO_API int64_t pmo_er_part_sizes(int count, int64_t n_min, int64_t n_max, uint64_t seed,
                                  int64_t *vbase) {
  vbase[0] = 0;
  for (int i = 0; i < count; ++i) {
    double u = (double)(pmo_hash(seed, (uint64_t)i) >> 11) * (1.0 / 9007199254740992.0);
    int64_t ni = (int64_t)floor(exp(log((double)n_min) + u * (log((double)n_max) - log((double)n_min))));
    if (ni < n_min) ni = n_min;
    if (ni > n_max) ni = n_max;
    vbase[i + 1] = vbase[i] + ni;
  }
  return vbase[count];
}

PMO_API int64_t pmo_er_batch(int count, int64_t n_min, int64_t n_max, int avg_degree, uint64_t seed,
                             int64_t *vbase, int32_t *off, int32_t *idx) {
  int64_t n = pmo_er_part_sizes(count, n_min, n_max, seed, vbase);
  int64_t draws = n * avg_degree;
  uint64_t *keys = (uint64_t *)malloc((size_t)(draws > 0 ? draws : 1) * sizeof(uint64_t));
  uint64_t seed2 = seed ^ 0xE5E5E5E5ull;
  int64_t k = 0;
  for (int i = 0; i < count; ++i) {
    int64_t ni = vbase[i + 1] - vbase[i];
    for (int64_t j = 0; j < ni * avg_degree; ++j, ++k) {
      uint64_t h = pmo_hash(seed2, (uint64_t)k);
      uint64_t s = (uint64_t)vbase[i] + (h >> 32) % (uint64_t)ni;
      uint64_t d = (uint64_t)vbase[i] + (h & 0xffffffffull) % (uint64_t)ni;
      keys[k] = (s << 32) | d;
    }
  }
  int64_t m = pmo_keys_to_csr(keys, draws, n, 0, off, idx);
  free(keys);
  return m;
}

/* Edge weight rules shared with the GPU generator (k_weights_i32 / k_weights_f32):
 * a hash of the edge's endpoints, so both sides draw the same weight per edge. */
PMO_API int32_t pmo_weight_int(uint64_t seed, uint32_t u, uint32_t v, int32_t wmax) {
  uint32_t a = u < v ? u : v, b = u < v ? v : u; /* symmetric: w(u,v) == w(v,u) */
  uint64_t key = ((uint64_t)a << 32) | b;
  return 1 + (int32_t)((pmo_hash(seed, key) >> 32) % (uint64_t)wmax);
}
PMO_API float pmo_weight_unit(uint64_t seed, uint32_t u, uint32_t v) {
  uint64_t key = ((uint64_t)u << 32) | v; /* (0, 1], exact in FP32 */
  return (float)((pmo_hash(seed, key) >> 40) + 1) * (1.0f / 16777216.0f);
}
PMO_API float pmo_uniform01(uint64_t seed, uint64_t i) { /* [0, 1), exact in FP32 */
  return (float)(pmo_hash(seed, i) >> 40) * (1.0f / 16777216.0f);
}
PMO_API float pmo_uniform_open(uint64_t seed, uint64_t i) { /* (0, 1), exact in FP32 */
  return (float)(((pmo_hash(seed, i) >> 41) << 1) | 1) * (1.0f / 16777216.0f);
}

PMO_API void pmo_fill_weights_int(int64_t n, const int32_t *off, const int32_t *idx,
                                  uint64_t seed, int32_t wmax, int32_t *w) {
  for (int64_t s = 0; s < n; ++s)
    for (int64_t e = off[s]; e < off[s + 1]; ++e)
      w[e] = pmo_weight_int(seed, (uint32_t)s, (uint32_t)idx[e], wmax);
}
PMO_API void pmo_fill_weights_unit(int64_t n, const int32_t *off, const int32_t *idx,
                                   uint64_t seed, float *w) {
  for (int64_t s = 0; s < n; ++s)
    for (int64_t e = off[s]; e < off[s + 1]; ++e)
      w[e] = pmo_weight_unit(seed, (uint32_t)s, (uint32_t)idx[e]);
}
PMO_API void pmo_fill_uniform01(uint64_t seed, int64_t count, float *x) {
  for (int64_t i = 0; i < count; ++i) x[i] = pmo_uniform01(seed, (uint64_t)i);
}
PMO_API void pmo_fill_uniform_open(uint64_t seed, int64_t count, float *x) {
  for (int64_t i = 0; i < count; ++i) x[i] = pmo_uniform_open(seed, (uint64_t)i);
}

/* Seeded distinct sources with out-degree > 0: candidate j is
 * hash(seed, j) mod n, accepted when not isolated and not already taken. */
PMO_API int pmo_pick_sources(int64_t n, const int32_t *off, uint64_t seed, int k, int32_t *out) {
  int got = 0;
  for (uint64_t j = 0; got < k && j < (uint64_t)n * 64; ++j) {
    int32_t v = (int32_t)(pmo_hash(seed, j) % (uint64_t)n);
    if (off[v + 1] == off[v]) continue;
    int dup = 0;
    for (int t = 0; t < got; ++t) dup |= out[t] == v;
    if (!dup) out[got++] = v;
  }
  return got;
}

/* CSR -> CSC (in-edges), sources ascending within a destination; eid maps
 * each CSC slot back to its CSR edge id (for per-edge data). */
PMO_API void pmo_transpose(int64_t n, const int32_t *off, const int32_t *idx,
                           int32_t *toff, int32_t *tidx, int32_t *eid) {
  int64_t m = off[n];
  for (int64_t v = 0; v <= n; ++v) toff[v] = 0;
  for (int64_t e = 0; e < m; ++e) toff[idx[e] + 1]++;
  for (int64_t v = 0; v < n; ++v) toff[v + 1] += toff[v];
  int32_t *fill = (int32_t *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int32_t));
  for (int64_t v = 0; v < n; ++v) fill[v] = toff[v];
  for (int64_t s = 0; s < n; ++s)
    for (int64_t e = off[s]; e < off[s + 1]; ++e) {
      int32_t p = fill[idx[e]]++;
      tidx[p] = (int32_t)s;
      if (eid) eid[p] = (int32_t)e;
    }
  free(fill);
}

/* ------------------------------------------------------------------------ */
/* PageRank, Polymer semantics (numa-PageRank.C).                            */
/*  PR_F::updateValVer        numa-PageRank.C:87-90  p_next[d] += p[s]/deg(s) */
/*  edgeMapDenseForwardOTHER  numa-PageRank.C:177-230 push over frontier,     */
/*                            next bit for every out-neighbour               */
/*  PR_Vertex_F               numa-PageRank.C:125-137 on the CURRENT frontier */
/*  PR_Vertex_Reset           numa-PageRank.C:140-148 p_curr = 0 on frontier  */
/*  loop / swap / switch      numa-PageRank.C:273-335                         */
/*  init p=1/n, p_next=0, F=V numa-PageRank.C:398-430                         */
/* The graph must be free of self loops (readGraphSkipRing, IO-numa.h:192).  */
/* resid (optional) receives sum |p_{t+1} - p_t| for each iteration.          */
/* ------------------------------------------------------------------------ */
/* Transpose (CSC) with sources ascending per destination; *eid optional. */
static void csc_alloc(int64_t n, const int32_t *off, const int32_t *idx, int32_t **toff, int32_t **tidx,
                      int32_t **eid) {
  int64_t m = off[n];
  *toff = (int32_t *)malloc((size_t)(n + 1) * sizeof(int32_t));
  *tidx = (int32_t *)malloc((size_t)(m > 0 ? m : 1) * sizeof(int32_t));
  if (eid) *eid = (int32_t *)malloc((size_t)(m > 0 ? m : 1) * sizeof(int32_t));
  pmo_transpose(n, off, idx, *toff, *tidx, eid ? *eid : NULL);
}

PMO_API void pmo_pagerank(int64_t n, const int32_t *off, const int32_t *idx, int iters,
                          double damping, double *out, double *resid) {
  double *pc = (double *)malloc((size_t)n * sizeof(double));
  double *pn = (double *)malloc((size_t)n * sizeof(double));
  unsigned char *F = (unsigned char *)malloc((size_t)n);
  unsigned char *Nx = (unsigned char *)malloc((size_t)n);
  int32_t *toff, *tidx;
  csc_alloc(n, off, idx, &toff, &tidx, NULL);
  double added = (1.0 - damping) * (1.0 / (double)n);
  for (int64_t i = 0; i < n; ++i) { pc[i] = 1.0 / (double)n; pn[i] = 0.0; F[i] = 1; }
  for (int it = 0; it < iters; ++it) {
    /* PR_F push, p_next[d] += p[s]/deg(s) for s in F, as a pull: d adds its */
    /* frontier in-neighbours in ascending s; d joins the next frontier when */
    /* it has one (edgeMapDenseForwardOTHER's next bit).                     */
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t d = 0; d < n; ++d) {
      double acc = pn[d];
      unsigned char hit = 0;
      for (int64_t e = toff[d]; e < toff[d + 1]; ++e) {
        int32_t s = tidx[e];
        if (!F[s]) continue;
        acc += pc[s] / (double)(off[s + 1] - off[s]);
        hit = 1;
      }
      pn[d] = acc;
      Nx[d] = hit;
    }
    for (int64_t i = 0; i < n; ++i)
      if (F[i]) pn[i] = damping * pn[i] + added;
    double r = 0.0;
    for (int64_t i = 0; i < n; ++i) r += fabs(pn[i] - pc[i]);
    if (resid) resid[it] = r;
    for (int64_t i = 0; i < n; ++i)
      if (F[i]) pc[i] = 0.0;
    double *t = pc; pc = pn; pn = t;
    unsigned char *tb = F; F = Nx; Nx = tb;
  }
  memcpy(out, pc, (size_t)n * sizeof(double));
  free(pc); free(pn); free(F); free(Nx); free(toff); free(tidx);
}

/* ------------------------------------------------------------------------ */
/* PageRankDelta (numa-PageRankDelta.C): PR_F pushes Delta[s]/outdeg(s) from */
/* the frontier into nghSum (64-90, DENSE_FORWARD with threshold 0, 211);    */
/* then a vertexFilter over ALL vertices (215-219): the first round          */
/* PR_Vertex_F_FirstRound (93-107) sets Delta = d*(p + nghSum) + (1-d)/n - p, */
/* p += Delta, Delta -= 1/n; later rounds PR_Vertex_F (109-121) set          */
/* Delta = d*nghSum, p += Delta; a vertex stays in the frontier when          */
/* |Delta| > eps2 * p; PR_Vertex_Reset zeroes nghSum (124-132).  Starts at    */
/* p = 0, Delta = 1/n, frontier = all (281-286).  fsize (optional, iters     */
/* entries): frontier size after each round.                                 */
/* ------------------------------------------------------------------------ */
PMO_API void pmo_pagerank_delta(int64_t n, const int32_t *off, const int32_t *idx, int iters,
                                double damping, double eps2, double *p_out, int64_t *fsize) {
  double *p = (double *)calloc((size_t)n, sizeof(double));
  double *delta = (double *)malloc((size_t)n * sizeof(double));
  double *ngh = (double *)calloc((size_t)n, sizeof(double));
  unsigned char *F = (unsigned char *)malloc((size_t)n);
  const double one_over_n = 1.0 / (double)n, added = (1.0 - damping) * one_over_n;
  for (int64_t i = 0; i < n; ++i) { delta[i] = one_over_n; F[i] = 1; }
  for (int it = 0; it < iters; ++it) {
    for (int64_t s = 0; s < n; ++s) {
      if (!F[s]) continue;
      const int64_t deg = off[s + 1] - off[s];
      for (int64_t e = off[s]; e < off[s + 1]; ++e) ngh[idx[e]] += delta[s] / (double)deg;
    }
    int64_t cnt = 0;
    for (int64_t i = 0; i < n; ++i) {
      if (it == 0) {
        delta[i] = damping * (p[i] + ngh[i]) + added - p[i];
        p[i] += delta[i];
        delta[i] -= one_over_n;
      } else {
        delta[i] = ngh[i] * damping;
        p[i] += delta[i];
      }
      F[i] = fabs(delta[i]) > eps2 * p[i];
      cnt += F[i];
      ngh[i] = 0.0;
    }
    if (fsize) fsize[it] = cnt;
  }
  memcpy(p_out, p, (size_t)n * sizeof(double));
  free(p); free(delta); free(ngh); free(F);
}

/* ------------------------------------------------------------------------ */
/* Personalised PageRank for k seeds (no reference; built from PR_F's push  */
/* p[s]/outdeg(s), numa-PageRank.C:87-90, and PR_Vertex_F's damping,        */
/* 125-137, with the teleport going to the seed):                           */
/*   x_0 = e_seed,  x_{t+1}[d] = damping * sum_{s->d} x_t[s]/outdeg(s)      */
/*                              + (1 - damping) * [d == seed]               */
/* on every vertex, no dangling redistribution (as PR_F).  out: n x k,      */
/* row-major (out[v*k + j] for seed j).                                      */
/* ------------------------------------------------------------------------ */
PMO_API void pmo_ppr(int64_t n, const int32_t *off, const int32_t *idx, const int32_t *seeds, int k,
                     int iters, double damping, double *out) {
  double *x = (double *)calloc((size_t)n * k, sizeof(double));
  double *y = (double *)malloc((size_t)n * k * sizeof(double));
  int32_t *toff, *tidx;
  csc_alloc(n, off, idx, &toff, &tidx, NULL);
  for (int j = 0; j < k; ++j) x[(int64_t)seeds[j] * k + j] = 1.0;
  for (int it = 0; it < iters; ++it) {
    /* y[d] = sum over in-neighbours s (ascending) of x[s]/deg(s), per seed */
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t d = 0; d < n; ++d) {
      double *yd = y + d * k;
      for (int j = 0; j < k; ++j) yd[j] = 0.0;
      for (int64_t e = toff[d]; e < toff[d + 1]; ++e) {
        int32_t s = tidx[e];
        double deg = (double)(off[s + 1] - off[s]);
        for (int j = 0; j < k; ++j) yd[j] += x[(int64_t)s * k + j] / deg;
      }
    }
    for (int64_t i = 0; i < n * k; ++i) y[i] *= damping;
    for (int j = 0; j < k; ++j) y[(int64_t)seeds[j] * k + j] += 1.0 - damping;
    double *t = x; x = y; y = t;
  }
  memcpy(out, x, (size_t)n * k * sizeof(double));
  free(x); free(y); free(toff); free(tidx);
}

/* ------------------------------------------------------------------------ */
/* Weighted PageRank and its adjoint (no reference counterpart; the          */
/* weighted push of SPMV_F, numa-SPMV.C:72-81, with PR_Vertex_F's damping,   */
/* numa-PageRank.C:125-137, on every vertex):                                */
/*   p = damping * A_W^T p + (1 - damping)/n,  (A_W^T p)[v] = sum_{e=s->v}   */
/*   W_e p[s],  p_0 = 1/n, iterated until sum|p_{t+1} - p_t| <= tol*sum|p|.   */
/* For a cotangent g (dL/dp) the adjoint solves lambda = damping * A_W       */
/* lambda + g, (A_W lambda)[s] = sum_{e=s->v} W_e lambda[v], by the same     */
/* iteration from lambda_0 = g, and dL/dW_e = damping * lambda[v] * p[s].    */
/* Weights are per CSR edge; returns the number of iterations.               */
/* ------------------------------------------------------------------------ */
PMO_API int pmo_weighted_pagerank(int64_t n, const int32_t *off, const int32_t *idx, const double *w,
                                  double damping, double tol, int max_iters, double *p) {
  double *q = (double *)malloc((size_t)n * sizeof(double));
  for (int64_t i = 0; i < n; ++i) p[i] = 1.0 / (double)n;
  int it = 0;
  while (it < max_iters) {
    for (int64_t i = 0; i < n; ++i) q[i] = 0.0;
    for (int64_t s = 0; s < n; ++s)
      for (int64_t e = off[s]; e < off[s + 1]; ++e) q[idx[e]] += w[e] * p[s];
    double r = 0.0, tot = 0.0;
    for (int64_t i = 0; i < n; ++i) {
      q[i] = damping * q[i] + (1.0 - damping) / (double)n;
      r += fabs(q[i] - p[i]);
      tot += fabs(q[i]);
    }
    memcpy(p, q, (size_t)n * sizeof(double));
    ++it;
    if (r <= tol * tot) break;
  }
  free(q);
  return it;
}

PMO_API int pmo_pagerank_adjoint(int64_t n, const int32_t *off, const int32_t *idx, const double *w,
                                 double damping, double tol, int max_iters, const double *p,
                                 const double *g, double *lambda, double *dw) {
  double *q = (double *)malloc((size_t)n * sizeof(double));
  memcpy(lambda, g, (size_t)n * sizeof(double));
  int it = 0;
  while (it < max_iters) {
    double r = 0.0, tot = 0.0;
    for (int64_t s = 0; s < n; ++s) {
      double acc = 0.0;
      for (int64_t e = off[s]; e < off[s + 1]; ++e) acc += w[e] * lambda[idx[e]];
      q[s] = damping * acc + g[s];
    }
    for (int64_t i = 0; i < n; ++i) {
      r += fabs(q[i] - lambda[i]);
      tot += fabs(q[i]);
    }
    memcpy(lambda, q, (size_t)n * sizeof(double));
    ++it;
    if (r <= tol * tot) break;
  }
  for (int64_t s = 0; s < n; ++s)
    for (int64_t e = off[s]; e < off[s + 1]; ++e) dw[e] = damping * lambda[idx[e]] * p[s];
  free(q);
  return it;
}

/* One weighted SpMV y = A_W^T x and its backward for cotangent gy:          */
/* dx[s] = sum_{e=s->v} W_e gy[v],  dW_e = gy[v] * x[s].                     */
PMO_API void pmo_spmv_backward(int64_t n, const int32_t *off, const int32_t *idx, const double *w,
                               const double *x, const double *gy, double *dx, double *dw) {
  for (int64_t s = 0; s < n; ++s) {
    double acc = 0.0;
    for (int64_t e = off[s]; e < off[s + 1]; ++e) {
      acc += w[e] * gy[idx[e]];
      dw[e] = gy[idx[e]] * x[s];
    }
    dx[s] = acc;
  }
}

/* Lognormal(0, 1) edge weights normalised per source row (sum 1 over the   */
/* out-edges of every vertex): z = sqrt(-2 ln u1) cos(2 pi u2) (Box-Muller)  */
/* from u1 = ((h1 >> 11) + 1) 2^-53, u2 = (h2 >> 11) 2^-53, h1/h2 = hash(seed,*/
/* 2e), hash(seed, 2e+1).                                                    */
PMO_API void pmo_lognormal_weights(int64_t n, const int32_t *off, uint64_t seed, double *w) {
  const double two_pi = 6.283185307179586476925286766559;
  for (int64_t s = 0; s < n; ++s) {
    double sum = 0.0;
    for (int64_t e = off[s]; e < off[s + 1]; ++e) {
      double u1 = (double)((pmo_hash(seed, 2 * (uint64_t)e) >> 11) + 1) * (1.0 / 9007199254740992.0);
      double u2 = (double)(pmo_hash(seed, 2 * (uint64_t)e + 1) >> 11) * (1.0 / 9007199254740992.0);
      w[e] = exp(sqrt(-2.0 * log(u1)) * cos(two_pi * u2));
      sum += w[e];
    }
    for (int64_t e = off[s]; e < off[s + 1]; ++e) w[e] /= sum;
  }
}

/* ------------------------------------------------------------------------ */
/* SpMV (numa-SPMV.C): every iteration pushes over ALL vertices             */
/* (SPMV_F::updateAtomic numa-SPMV.C:72-81, loop 168-193), then resets      */
/* p_curr = 0 and swaps, so x_{t+1}[d] = sum_{s->d} w(s,d) * x_t[s].         */
/* w is given per CSR edge (FP64 here; the reference stores int weights).    */
/* ------------------------------------------------------------------------ */
PMO_API void pmo_spmv(int64_t n, const int32_t *off, const int32_t *idx, const double *w,
                      const double *x0, int iters, double *out) {
  double *x = (double *)malloc((size_t)n * sizeof(double));
  double *y = (double *)malloc((size_t)n * sizeof(double));
  int32_t *toff, *tidx, *eid;
  csc_alloc(n, off, idx, &toff, &tidx, &eid);
  memcpy(x, x0, (size_t)n * sizeof(double));
  for (int it = 0; it < iters; ++it) {
    /* SPMV_F push y[d] += x[s] * w_e as a pull, sources ascending */
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t d = 0; d < n; ++d) {
      double acc = 0.0;
      for (int64_t e = toff[d]; e < toff[d + 1]; ++e) acc += x[tidx[e]] * w[eid[e]];
      y[d] = acc;
    }
    double *t = x; x = y; y = t;
  }
  memcpy(out, x, (size_t)n * sizeof(double));
  free(x); free(y); free(toff); free(tidx); free(eid);
}

/* ------------------------------------------------------------------------ */
/* BFS (numa-BFS.C): BFS_F numa-BFS.C:59-79 -- cond(d) = Parents[d] == -1,   */
/* updateAtomic = CAS(Parents[d], -1, s); Parents[src] = src (350).  The     */
/* depth of a vertex is the level at which it entered the frontier; depths   */
/* are unique, parents are any in-neighbour one level up.  Returns the       */
/* number of reached vertices (what the reference prints with -result).      */
/* parents may be NULL.  Level-synchronous, frontier order ascending.        */
/* ------------------------------------------------------------------------ */
PMO_API int64_t pmo_bfs(int64_t n, const int32_t *off, const int32_t *idx, int32_t src,
                        int32_t *depth, int32_t *parents) {
  int32_t *q = (int32_t *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int32_t));
  for (int64_t i = 0; i < n; ++i) { depth[i] = -1; if (parents) parents[i] = -1; }
  int64_t head = 0, tail = 0;
  depth[src] = 0;
  if (parents) parents[src] = src;
  q[tail++] = src;
  while (head < tail) {
    int32_t s = q[head++];
    for (int64_t e = off[s]; e < off[s + 1]; ++e) {
      int32_t d = idx[e];
      if (depth[d] == -1) {
        depth[d] = depth[s] + 1;
        if (parents) parents[d] = s;
        q[tail++] = d;
      }
    }
  }
  free(q);
  return tail;
}

/* ------------------------------------------------------------------------ */
/* Connected components by min-label propagation (numa-Components.C):        */
/* labels start at the vertex id (387-391); CC_F::updateAtomic (77-81)       */
/* writeMin(IDs[d], IDs[s]) along every out-edge of the frontier, the       */
/* frontier is the set of vertices whose label dropped (origID == prevIDs,   */
/* CC_Vertex_F 109-119).  Fixpoint: label[v] = min id of any vertex that     */
/* reaches v (for a symmetric graph: the minimum id of v's component).       */
/* Computed here by a Jacobi sweep to the fixpoint.  Returns #rounds.       */
/* ------------------------------------------------------------------------ */
PMO_API int pmo_cc(int64_t n, const int32_t *off, const int32_t *idx, int32_t *labels) {
  unsigned char *F = (unsigned char *)malloc((size_t)n);
  unsigned char *Nx = (unsigned char *)malloc((size_t)n);
  for (int64_t i = 0; i < n; ++i) { labels[i] = (int32_t)i; F[i] = 1; }
  int rounds = 0;
  for (;;) {
    int any = 0;
    memset(Nx, 0, (size_t)n);
    for (int64_t s = 0; s < n; ++s) {
      if (!F[s]) continue;
      for (int64_t e = off[s]; e < off[s + 1]; ++e) {
        int32_t d = idx[e];
        if (labels[s] < labels[d]) { labels[d] = labels[s]; Nx[d] = 1; any = 1; }
      }
    }
    ++rounds;
    unsigned char *t = F; F = Nx; Nx = t;
    if (!any) break;
  }
  free(F); free(Nx);
  return rounds;
}

/* ------------------------------------------------------------------------ */
/* BellmanFord (numa-BellmanFord.C): BF_F::updateAtomic (78-82)              */
/* writeMin(dist[d], dist[s] + w) && CAS(Visited[d], 0, 1); dist starts at   */
/* INT_MAX/2 (283) with dist[src] = 0.  The reference resets Visited on the  */
/* current frontier (BF_Vertex_F at 185), which can drop a vertex whose      */
/* distance falls again while still marked; this restatement resets it on   */
/* the output frontier as Ligra's BellmanFord does, which converges to the   */
/* exact shortest-path distances.  Returns #rounds, or -1 on a negative      */
/* cycle (not reachable with the positive weights used here).               */
/* ------------------------------------------------------------------------ */
#define PMO_BF_INF 1073741823
PMO_API int pmo_bellman_ford(int64_t n, const int32_t *off, const int32_t *idx, const int32_t *w,
                             int32_t src, int32_t *dist) {
  unsigned char *F = (unsigned char *)calloc((size_t)n, 1);
  unsigned char *Nx = (unsigned char *)calloc((size_t)n, 1);
  for (int64_t i = 0; i < n; ++i) dist[i] = PMO_BF_INF;
  dist[src] = 0;
  F[src] = 1;
  int rounds = 0, any = 1;
  while (any) {
    any = 0;
    memset(Nx, 0, (size_t)n);
    for (int64_t s = 0; s < n; ++s) {
      if (!F[s]) continue;
      for (int64_t e = off[s]; e < off[s + 1]; ++e) {
        int32_t d = idx[e];
        int32_t nd = dist[s] + w[e];
        if (nd < dist[d]) { dist[d] = nd; Nx[d] = 1; any = 1; }
      }
    }
    unsigned char *t = F; F = Nx; Nx = t;
    if (++rounds > n + 1) { rounds = -1; break; }
  }
  free(F); free(Nx);
  return rounds;
}

/* Dijkstra with a binary heap: an independent check of pmo_bellman_ford. */
PMO_API void pmo_dijkstra(int64_t n, const int32_t *off, const int32_t *idx, const int32_t *w,
                          int32_t src, int32_t *dist) {
  int64_t cap = off[n] + 1;
  int64_t *hk = (int64_t *)malloc((size_t)cap * sizeof(int64_t));
  int64_t hn = 0;
  for (int64_t i = 0; i < n; ++i) dist[i] = PMO_BF_INF;
  dist[src] = 0;
  hk[hn++] = ((int64_t)0 << 32) | src;
  while (hn > 0) {
    int64_t top = hk[0];
    hk[0] = hk[--hn];
    for (int64_t i = 0;;) { /* sift down */
      int64_t l = 2 * i + 1, r = l + 1, b = i;
      if (l < hn && hk[l] < hk[b]) b = l;
      if (r < hn && hk[r] < hk[b]) b = r;
      if (b == i) break;
      int64_t t = hk[i]; hk[i] = hk[b]; hk[b] = t; i = b;
    }
    int32_t du = (int32_t)(top >> 32), u = (int32_t)(top & 0xFFFFFFFF);
    if (du != dist[u]) continue;
    for (int64_t e = off[u]; e < off[u + 1]; ++e) {
      int32_t v = idx[e], nd = du + w[e];
      if (nd < dist[v]) {
        dist[v] = nd;
        int64_t i = hn++;
        hk[i] = ((int64_t)nd << 32) | v;
        while (i > 0 && hk[(i - 1) / 2] > hk[i]) { /* sift up */
          int64_t p = (i - 1) / 2, t = hk[i]; hk[i] = hk[p]; hk[p] = t; i = p;
        }
      }
    }
  }
  free(hk);
}

/* ------------------------------------------------------------------------ */
/* Belief propagation, 2 states (numa-BP.C).  BP_F::updateAtomic (112-125):  */
/* for an out-edge e = (s -> d):                                             */
/*   belief_e[i] = sum_j prior_d[j] * psi_e[i][j] * prod_curr_d[j]           */
/*   prod_next_d[i] *= belief_e[i]                                           */
/* BP_Vertex_Reset (130-140) sets prod_next = 1 on the current frontier      */
/* before the edge pass; edgeMapDenseBPNoRep (179-230) sets the next bit of  */
/* every out-neighbour; prod arrays swap every round (loop 280-316).         */
/* The reference leaves prod_curr zero and priors uninitialised; here both   */
/* products start at 1 and priors are inputs.  Products are carried as       */
/* natural logs (L = log prod) and every message is normalised to sum 1     */
/* (standard loopy BP): without that, log prod grows like indegree^t and     */
/* leaves even the FP64 range on hubs.  With a_j = prior_d[j] *              */
/* exp(L_d[j] - max_j L_d[j]):  b_e[i] = sum_j psi_e[i][j] a_j,              */
/* L_next_d[i] += log(b_e[i] / (b_e[0] + b_e[1])).                           */
/* psi: 4 doubles per CSR edge ([i][j] row major) or NULL for psi_uniform.   */
/* ------------------------------------------------------------------------ */
PMO_API void pmo_bp(int64_t n, const int32_t *off, const int32_t *idx, const double *prior,
                    const double *psi_edge, const double *psi_uniform, int iters,
                    double *out_logprod) {
  double *Lc = (double *)malloc((size_t)n * 2 * sizeof(double));
  double *Ln = (double *)malloc((size_t)n * 2 * sizeof(double));
  unsigned char *F = (unsigned char *)malloc((size_t)n);
  unsigned char *Nx = (unsigned char *)malloc((size_t)n);
  int32_t *toff, *tidx, *eid;
  csc_alloc(n, off, idx, &toff, &tidx, &eid);
  for (int64_t i = 0; i < 2 * n; ++i) { Lc[i] = 0.0; Ln[i] = 0.0; }
  for (int64_t i = 0; i < n; ++i) F[i] = 1;
  for (int it = 0; it < iters; ++it) {
    for (int64_t i = 0; i < n; ++i)
      if (F[i]) { Ln[2 * i] = 0.0; Ln[2 * i + 1] = 0.0; }
    /* the edge pass as a pull: d adds the message of every frontier        */
    /* in-neighbour's edge in ascending source order.  The message of edge  */
    /* s -> d depends on d's state and the edge's psi only; with a uniform  */
    /* psi it is the same value for every in-edge of d and is computed once. */
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t d = 0; d < n; ++d) {
      double l0 = Lc[2 * d], l1 = Lc[2 * d + 1];
      double lm = l0 > l1 ? l0 : l1;
      double a0 = prior[2 * d] * exp(l0 - lm), a1 = prior[2 * d + 1] * exp(l1 - lm);
      double acc0 = Ln[2 * d], acc1 = Ln[2 * d + 1];
      double u0 = 0.0, u1 = 0.0;
      int have_u = 0;
      unsigned char hit = 0;
      for (int64_t e = toff[d]; e < toff[d + 1]; ++e) {
        if (!F[tidx[e]]) continue;
        double m0, m1;
        if (psi_edge || !have_u) {
          const double *psi = psi_edge ? psi_edge + 4 * (int64_t)eid[e] : psi_uniform;
          double b0 = psi[0] * a0 + psi[1] * a1, b1 = psi[2] * a0 + psi[3] * a1;
          double lz = log(b0 + b1);
          m0 = log(b0) - lz;
          m1 = log(b1) - lz;
          if (!psi_edge) { u0 = m0; u1 = m1; have_u = 1; }
        } else {
          m0 = u0;
          m1 = u1;
        }
        acc0 += m0;
        acc1 += m1;
        hit = 1;
      }
      Ln[2 * d] = acc0;
      Ln[2 * d + 1] = acc1;
      Nx[d] = hit;
    }
    double *t = Lc; Lc = Ln; Ln = t;
    unsigned char *tb = F; F = Nx; Nx = tb;
  }
  memcpy(out_logprod, Lc, (size_t)n * 2 * sizeof(double));
  free(Lc); free(Ln); free(F); free(Nx); free(toff); free(tidx); free(eid);
}

/* ------------------------------------------------------------------------ */
/* BP as the reference writes it, in linear products (FP64):                 */
/* BP_F::updateAtomic (numa-BP.C:112-125) for each out-edge e = (s -> d) of   */
/* a frontier source s, sources ascending: belief_e[i] = sum_j prior_d[j] *  */
/* psi[i][j] * prod_curr_d[j]; prod_next_d[i] *= belief_e[i]; d joins the    */
/* next frontier.  BP_Vertex_Reset (130-140) sets prod_next = 1 on the       */
/* current frontier first; the arrays swap every round (loop 280-316).       */
/* Products start at 1 in prod_curr and 0 in prod_next (the zero-filled      */
/* mapping), every vertex in the first frontier.  normalize != 0 divides     */
/* each belief by its sum before the product (the messages pmo_bp uses, in   */
/* the linear domain).  psi: 4 doubles [i][j] for every edge.  out: n x 2.   */
/* ------------------------------------------------------------------------ */
PMO_API void pmo_bp_raw(int64_t n, const int32_t *off, const int32_t *idx, const double *prior,
                        const double *psi, int iters, int normalize, double *out_prod) {
  double *Pc = (double *)malloc((size_t)n * 2 * sizeof(double));
  double *Pn = (double *)malloc((size_t)n * 2 * sizeof(double));
  unsigned char *F = (unsigned char *)malloc((size_t)n);
  unsigned char *Nx = (unsigned char *)malloc((size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    Pc[2 * i] = Pc[2 * i + 1] = 1.0;
    Pn[2 * i] = Pn[2 * i + 1] = 0.0;
    F[i] = 1;
  }
  for (int it = 0; it < iters; ++it) {
    memset(Nx, 0, (size_t)n);
    for (int64_t i = 0; i < n; ++i)
      if (F[i]) { Pn[2 * i] = 1.0; Pn[2 * i + 1] = 1.0; }
    for (int64_t s = 0; s < n; ++s) {
      if (!F[s]) continue;
      for (int64_t e = off[s]; e < off[s + 1]; ++e) {
        int32_t d = idx[e];
        double b[2];
        for (int i = 0; i < 2; ++i) {
          b[i] = 0.0;
          for (int j = 0; j < 2; ++j) b[i] += prior[2 * d + j] * psi[2 * i + j] * Pc[2 * d + j];
        }
        if (normalize) {
          double z = b[0] + b[1];
          b[0] /= z;
          b[1] /= z;
        }
        Pn[2 * d] *= b[0];
        Pn[2 * d + 1] *= b[1];
        Nx[d] = 1;
      }
    }
    double *t = Pc; Pc = Pn; Pn = t;
    unsigned char *tb = F; F = Nx; Nx = tb;
  }
  memcpy(out_prod, Pc, (size_t)n * 2 * sizeof(double));
  free(Pc); free(Pn); free(F); free(Nx);
}

/* ------------------------------------------------------------------------ */
/* PBBS writers read by the reference loaders (IO-numa.h / IO.h):            */
/*  AdjacencyGraph text (IO-numa.h:112-188), WeightedAdjacencyGraph text     */
/*  (IO-numa.h:318-402: offsets, then destinations, then weights) and the    */
/*  binary triple <name>.config (n), <name>.adj (uint32 edges), <name>.idx   */
/*  (int32 offsets) (IO-numa.h:404-450).                                     */
/* ------------------------------------------------------------------------ */
PMO_API int pmo_write_adj_text(const char *path, int64_t n, const int32_t *off, const int32_t *idx,
                               const int32_t *w) {
  FILE *f = fopen(path, "w");
  if (!f) return -1;
  int64_t m = off[n];
  fprintf(f, "%s\n%lld\n%lld\n", w ? "WeightedAdjacencyGraph" : "AdjacencyGraph", (long long)n,
          (long long)m);
  for (int64_t v = 0; v < n; ++v) fprintf(f, "%d\n", off[v]);
  for (int64_t e = 0; e < m; ++e) fprintf(f, "%d\n", idx[e]);
  if (w)
    for (int64_t e = 0; e < m; ++e) fprintf(f, "%d\n", w[e]);
  return fclose(f);
}

PMO_API int pmo_write_adj_binary(const char *base, int64_t n, const int32_t *off, const int32_t *idx) {
  char path[4096];
  int64_t m = off[n];
  snprintf(path, sizeof path, "%s.config", base);
  FILE *f = fopen(path, "w");
  if (!f) return -1;
  fprintf(f, "%lld\n", (long long)n);
  fclose(f);
  snprintf(path, sizeof path, "%s.adj", base);
  f = fopen(path, "wb");
  if (!f) return -1;
  if (m && fwrite(idx, sizeof(int32_t), (size_t)m, f) != (size_t)m) { fclose(f); return -1; }
  fclose(f);
  snprintf(path, sizeof path, "%s.idx", base);
  f = fopen(path, "wb");
  if (!f) return -1;
  if (n && fwrite(off, sizeof(int32_t), (size_t)n, f) != (size_t)n) { fclose(f); return -1; }
  return fclose(f);
}
