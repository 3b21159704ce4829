/*
 * polymer_b200.h -- C ABI of the B200 edgeMap/vertexMap engine.
 *
 * Polymer has no FFI of its own: its applications are C++ programs whose
 * entry functions (PageRank(), BFS(), Components(), BF_main(), SPMV_main(),
 * BeliefPropagation()) take a graph built by readGraph() and run the hot
 * loops on CPU threads.  Each entry point below replaces one of those
 * functions (cited as file:line of the reference), with plain pointers and
 * sizes, so that a C, C++, Go (cgo), Java (JNI) or Python (ctypes) host can
 * call it.  Every function returns a pm_status and never aborts; the text
 * of the last error on the calling thread is pm_last_error().
 *
 * Memory: arrays passed with PM_MEM_HOST are ordinary host memory (pinned
 * or pageable); PM_MEM_DEVICE arrays are device pointers on the graph's
 * device.  Calls are synchronous: on return every output has been written.
 * A graph handle owns its device copy of the graph (CSR + CSC, int32 ids and
 * offsets), its frontier workspaces and a CUDA stream; distinct handles may
 * be used from distinct host threads.
 */
#ifndef POLYMER_B200_H
#define POLYMER_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define PM_API __attribute__((visibility("default")))
#else
#define PM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum pm_status {
  PM_OK = 0,
  PM_ERR_INVALID_ARG = 1, /* bad size, id out of range, null pointer      */
  PM_ERR_OOM = 2,         /* device or pinned allocation failed            */
  PM_ERR_CUDA = 3,        /* a CUDA runtime call failed                   */
  PM_ERR_TIMEOUT = 4,     /* a bounded device-side wait gave up            */
  PM_ERR_BAD_GRAPH = 5,   /* offsets not monotone, edge id out of range   */
  PM_ERR_NOT_SUPPORTED = 6,
  PM_ERR_NO_DEVICE = 7
} pm_status;

typedef struct pm_graph pm_graph;

/* memory-space flags for array arguments */
#define PM_MEM_HOST 0u
#define PM_MEM_DEVICE 1u

/* pm_graph_create flags */
#define PM_GRAPH_SYMMETRIC 2u       /* CSR already holds both directions (the
                                       reference's "-s" flag): CSC aliases CSR */
#define PM_GRAPH_SKIP_SELF_LOOPS 4u /* drop u->u edges while loading, as
                                       readGraphSkipRing does (IO-numa.h:192) */
#define PM_GRAPH_KEEP_EDGE_IDS 8u   /* keep the CSC->CSR edge-id map resident */

/* value types */
#define PM_F32 0
#define PM_F64 1
#define PM_I32 2

/* Build a device graph from a CSR (PBBS AdjacencyGraph layout: offsets of
 * n+1 entries -- append m to the n offsets a PBBS file holds -- and m
 * destination ids).  Replaces readGraph()/readGraphSkipRing()
 * (IO-numa.h:739-750), which build graph<vertex> with in-edges by sorting
 * (dst, src) pairs (IO-numa.h:145-180); here the CSC is built on the device.
 * mem: PM_MEM_HOST or PM_MEM_DEVICE for offsets/edges. */
PM_API pm_status pm_graph_create(const int32_t *offsets, const int32_t *edges, int64_t n, int64_t m,
                          uint32_t flags, uint32_t mem, int device, pm_graph **out);

/* Read a PBBS graph file into a device graph.  Replaces readGraph() /
 * readGraphSkipRing() / readWghGraph() (IO-numa.h:112-160, 318-470, 739-755).
 * Text (default): "AdjacencyGraph" or "WeightedAdjacencyGraph", then n, m,
 * the n offsets, the m edge ids and, when weighted, m int32 weights, all
 * separated by whitespace; the header is read on the host, the body is
 * tokenised and parsed on the GPU.  With PM_LOAD_BINARY, path is the base of
 * <path>.config (n as text), <path>.adj (m uint32 ids) and <path>.idx (n int32
 * offsets).  Other flags as pm_graph_create (PM_GRAPH_SYMMETRIC,
 * PM_GRAPH_SKIP_SELF_LOOPS: weights of dropped self loops go with them).
 * Weighted files set the int32 weights (as pm_graph_set_weights_i32).
 * PM_ERR_BAD_GRAPH for a bad header, a count that does not match, a word
 * that is not an integer or a value outside int32; PM_ERR_INVALID_ARG when a
 * file cannot be opened. */
#define PM_LOAD_BINARY 16u
/* With PM_LOAD_DUMP, path is a graph dump as dumpGraphToBin writes it and
 * loadGraphFromBin reads it (IO-numa.h:758-900): int64 total bytes, int32 n,
 * int64 m, then per vertex int32 words -1, id, out-degree, in-degree, the
 * out-neighbours, the in-neighbours (at most 2^31 words).  Parsed on the GPU;
 * PM_ERR_BAD_GRAPH for a wrong size, record count, id, degree or length. */
#define PM_LOAD_DUMP 32u
PM_API pm_status pm_graph_load_pbbs(const char *path, uint32_t flags, int device, pm_graph **out);

/* Write g as a graph dump (the layout of PM_LOAD_DUMP; dumpGraphToBin,
 * IO-numa.h:837-900): the records are assembled on the device and written
 * with one copy out.  Not for partition handles. */
PM_API pm_status pm_graph_save_dump(pm_graph *g, const char *path);

/* pm_graph_create with edge weights in CSR order (the weighted readers'
 * layout, readWghGraph IO-numa.h:318-402): wtype PM_I32 (BellmanFord) or
 * PM_F32 (SpMV).  The weights are copied on a second stream while the graph
 * is validated and transposed, so with pinned host arrays their transfer
 * overlaps the build; the result equals pm_graph_create followed by
 * pm_graph_set_weights_*. */
PM_API pm_status pm_graph_create_weighted(const int32_t *offsets, const int32_t *edges, const void *weights,
                                          int wtype, int64_t n, int64_t m, uint32_t flags, uint32_t mem,
                                          int device, pm_graph **out);

/* Build the seeded synthetic R-MAT graph (a,b,c,d = .57,.19,.19,.05;
 * n = 2^scale, n*edge_factor draws, self loops and duplicates removed,
 * sorted by source) directly on the device.  The same generator, evaluated
 * on the CPU, produces the same edge set.  PM_GRAPH_SYMMETRIC symmetrises
 * (union of both directions).  The reference ships no generator. */
PM_API pm_status pm_graph_create_rmat(int scale, int edge_factor, uint64_t seed, uint32_t flags,
                               int device, pm_graph **out);

/* A batch of `count` independent directed Erdos-Renyi graphs stored as one
 * disjoint union: part i has n_i vertices, log-uniform in [n_min, n_max], and
 * n_i * avg_degree seeded draws (self loops, duplicates removed); vertex ids
 * of part i start at parts[i] (pm_graph_get_parts).  The oracle's generator
 * builds the same graph.  No reference counterpart (the reference runs one
 * graph per process). */
PM_API pm_status pm_graph_create_er_batch(int count, int64_t n_min, int64_t n_max, int avg_degree,
                                          uint64_t seed, int device, pm_graph **out);

/* Declare g a disjoint union of count parts: part i owns vertices
 * [vbase[i], vbase[i+1]) (host array of count+1 offsets, vbase[0] = 0,
 * vbase[count] = n).  Rejected with PM_ERR_BAD_GRAPH if an edge crosses
 * parts. */
PM_API pm_status pm_graph_set_parts(pm_graph *g, const int64_t *vbase, int count);

/* ---- one graph over several processes (1D vertex partition) -------------
 * Replaces the reference's NUMA split: partitionByDegree (polymer.h:131-192)
 * cuts the vertices into ranges of about equal in-degree, and graphFilter /
 * graphFilter2Direction (polymer.h:346-497) give each node the edges whose
 * destination it owns.  Here each process (one per GPU) calls
 * pm_graph_create_partition with the WHOLE CSR (as pm_graph_create /
 * pm_graph_create_weighted; weights may be NULL) and its rank: the ranges cut
 * the in-edges plus a per-vertex term into equal shares on 32-vertex
 * boundaries, the same on every rank, and the handle keeps the edges whose
 * destination lies in its own range.  Vertex state is replicated: after
 * every pass the library calls the exchange function set with
 * pm_graph_set_exchange, which must gather every rank's range of buf into
 * every rank's buf:
 *   buf holds bounds[nranks] entries of elem_bytes; rank r's range is
 *   [bounds[r], bounds[r+1]); the call is ordered after the work queued on
 *   `stream` (a cudaStream_t) and the work queued on it afterwards must see
 *   the gathered buf (an NCCL allgather-v on that stream, for instance);
 *   return 0, or nonzero to fail the running call with PM_ERR_CUDA.
 * Every rank must run the same calls in the same order.  pm_pagerank,
 * pm_spmv, pm_bp, pm_bfs, pm_components and pm_bellman_ford run on a partition and
 * return the whole result on every rank (the optional residual / norm
 * arrays and the statistics count this rank's rows and edges); the other
 * application calls return PM_ERR_NOT_SUPPORTED.  On a partition handle,
 * pm_graph_info gives the whole graph's n and this rank's edge count, and
 * pm_graph_get_csr this rank's edges (all n sources, global ids).
 * nranks 1..1024. */
typedef int (*pm_allgather_fn)(void *user, void *buf, int64_t elem_bytes, const int64_t *bounds, int nranks,
                               void *stream);
PM_API pm_status pm_graph_create_partition(const int32_t *offsets, const int32_t *edges, const void *weights,
                                           int wtype, int64_t n, int64_t m, uint32_t flags, uint32_t mem,
                                           int rank, int nranks, int device, pm_graph **out);
PM_API pm_status pm_graph_set_exchange(pm_graph *g, pm_allgather_fn fn, void *user);
/* rank, nranks and the nranks+1 range bounds (0, n and 1 for a whole graph);
 * any pointer may be NULL. */
PM_API pm_status pm_graph_partition_info(const pm_graph *g, int *rank, int *nranks, int64_t *bounds);
/* Part offsets (count+1 entries into vbase when vbase is not NULL). */
PM_API pm_status pm_graph_get_parts(pm_graph *g, int64_t *vbase, int *count);

PM_API pm_status pm_graph_destroy(pm_graph *g);

/* n, m (directed stored edges) and max out-degree. */
PM_API pm_status pm_graph_info(const pm_graph *g, int64_t *n, int64_t *m, int64_t *max_out_degree);

/* Copy the CSR back (offsets n+1, edges m). */
PM_API pm_status pm_graph_get_csr(pm_graph *g, int32_t *offsets, int32_t *edges, uint32_t mem);

/* Edge weights in CSR order, as the weighted readers attach them
 * (readWghGraph, IO-numa.h:318-402 / IO.h; weights at neighbors[2j+1],
 * graph.h:89-113).  int32 for BellmanFord, float for SpMV. */
PM_API pm_status pm_graph_set_weights_i32(pm_graph *g, const int32_t *w, uint32_t mem);
PM_API pm_status pm_graph_set_weights_f32(pm_graph *g, const float *w, uint32_t mem);
/* Synthetic weights on the device: int32 uniform in [1, wmax] with
 * w(u,v) == w(v,u); float uniform in (0, 1]. Same rules as the oracle. */
PM_API pm_status pm_graph_gen_weights_i32(pm_graph *g, uint64_t seed, int32_t wmax);
PM_API pm_status pm_graph_gen_weights_f32(pm_graph *g, uint64_t seed);
/* Read the weights back in CSR order. */
PM_API pm_status pm_graph_get_weights_f32(pm_graph *g, float *w, uint32_t mem);
PM_API pm_status pm_graph_get_weights_i32(pm_graph *g, int32_t *w, uint32_t mem);

/* Seeded uniform vectors on the device ([0,1) or (0,1)), for synthetic
 * SpMV / BP inputs. out is a device array of count floats. */
PM_API pm_status pm_fill_uniform_f32(pm_graph *g, uint64_t seed, int open_interval, float *out,
                              int64_t count);

typedef struct pm_traversal_stats {
  int32_t rounds;         /* edgeMap calls until the frontier emptied       */
  int32_t dense_rounds;   /* of which took the dense (pull) direction       */
  int64_t edges_visited;  /* sum over rounds of the out-degree of the frontier
                             (the edges a push traversal scans)             */
  int64_t reached;        /* vertices with a finite result                  */
} pm_traversal_stats;

/* Breadth-first search from src.  Replaces BFS(start, GA) (numa-BFS.C:476)
 * with BFS_F (numa-BFS.C:59-79): parents[v] = some in-neighbour one level
 * up (parents[src] = src, -1 when unreached); depth[v] = level (or -1).
 * Either output may be NULL.  threshold: direction switch, dense (pull)
 * when |F| + outdeg(F) >= threshold; < 0 selects m / PM_TUNE_BFS_DIV (default
 * 20); 0 forces dense
 * every level as the reference's BFS does (numa-BFS.C:268). */
PM_API pm_status pm_bfs(pm_graph *g, int32_t src, int32_t *parents, int32_t *depth, uint32_t mem,
                 int64_t threshold, pm_traversal_stats *stats);

/* Asynchronous BFS: reachability from src with a parent tree, in one
 * persistent launch without level barriers.  Replaces BFS(start, GA) of
 * numa-BFS-async-pipe.C (BFS_F 52-72 driven by edgeMapSparseAsyncPipe,
 * polymer.h:1513-1751): each vertex is claimed by the first in-neighbour whose
 * CAS on parents[d] succeeds, whatever its level, so parents is a valid tree
 * over exactly the vertices pm_bfs reaches (parents[src] = src, -1 when
 * unreached; every parent edge exists; no cycles) but not a BFS tree.
 * stats->reached = reached vertices ("Vert visited" of the reference),
 * stats->edges_visited = out-edges scanned.  Waits inside the kernel are
 * bounded: PM_ERR_TIMEOUT if one runs out. */
PM_API pm_status pm_bfs_async(pm_graph *g, int32_t src, int32_t *parents, uint32_t mem,
                              pm_traversal_stats *stats);

/* Multi-source BFS: k <= 64 sources in one traversal, one bit per source in
 * a uint64 word per vertex (BFS_F of numa-BFS.C:59-79 with the parent CAS
 * replaced by per-source visited bits; the reference runs one BFS per
 * process).  depth: k*n int32, source-major (depth[l*n + v] = level of v from
 * sources[l], -1 when unreached) -- each row equals pm_bfs's depth for that
 * source.  sources: k int32 in mem's space.  stats->reached = sum over
 * sources of reached vertices; stats->edges_visited = sum over sources of the
 * out-degrees of the reached vertices.  threshold < 0: m / PM_TUNE_MULTI_DIV
 * (the union frontier of many sources turns dense sooner than one BFS's). */
PM_API pm_status pm_bfs_multi(pm_graph *g, const int32_t *sources, int k, int32_t *depth,
                              uint32_t mem, int64_t threshold, pm_traversal_stats *stats);

/* Connected components by min-label propagation.  Replaces Components(GA)
 * (numa-Components.C:402) with CC_F / CC_Vertex_F (55-119): labels start at
 * the vertex id, every round lowers labels along the out-edges of the
 * frontier (vertices whose label fell).  threshold < 0 selects m /
 * PM_TUNE_CC_DIV (default 8, numa-Components.C:226).  labels: n int32. */
PM_API pm_status pm_components(pm_graph *g, int32_t *labels, uint32_t mem, int64_t threshold,
                        pm_traversal_stats *stats);

/* Single-source shortest paths by Bellman-Ford over int32 weights
 * (pm_graph_set_weights_i32).  Replaces BF_main(WG, start)
 * (numa-BellmanFord.C:400) with BF_F (61-85): dist starts at 1073741823
 * (INT_MAX/2, 283), dist[src] = 0, a vertex joins the next frontier when
 * its distance falls in the round.  threshold < 0 selects m /
 * PM_TUNE_BF_DIV (default 20, numa-BellmanFord.C:182). */
PM_API pm_status pm_bellman_ford(pm_graph *g, int32_t src, int32_t *dist, uint32_t mem,
                          int64_t threshold, pm_traversal_stats *stats);

/* Multi-source BellmanFord: k <= 64 sources in one traversal, 64 int32
 * distance lanes per vertex (BF_F of numa-BellmanFord.C:61-85 per lane; the
 * reference runs one source per process).  The frontier is the set of
 * vertices with a lane that fell in the last round; the direction rule of
 * pm_bellman_ford applies to it (threshold < 0: m / PM_TUNE_MULTI_DIV).  dist: k*n
 * int32, source-major (dist[l*n + v] = distance of v from sources[l],
 * 1073741823 when unreached) -- each row equals pm_bellman_ford's dist for
 * that source.  sources: k int32 in mem's space.  stats->reached = number of
 * (source, vertex) pairs reached; stats->edges_visited = sum over rounds of
 * the frontier's out-degrees. */
PM_API pm_status pm_bellman_ford_multi(pm_graph *g, const int32_t *sources, int k, int32_t *dist,
                                       uint32_t mem, int64_t threshold, pm_traversal_stats *stats);

/* PageRank with Polymer's frontier semantics.  Replaces PageRank(GA,
 * maxIter) (numa-PageRank.C:548) with PR_F / PR_Vertex_F / PR_Vertex_Reset
 * (64-148) and the loop at 273-335: p = 1/n on all vertices, each iteration
 * pushes p[s]/outdeg(s) from the frontier, damps the frontier's entries,
 * zeroes them in the old vector, swaps, and the next frontier is the set of
 * vertices that received a push.  The graph must have no self loops.
 * dtype PM_F32 (FP32 storage and sums) or PM_F64; ranks: n values of dtype.
 * resid (optional, iters doubles): sum |p_{t+1} - p_t| per iteration, FP64. */
PM_API pm_status pm_pagerank(pm_graph *g, int iters, double damping, int dtype, void *ranks,
                      uint32_t mem, double *resid);

/* PageRankDelta.  Replaces PageRankDelta(GA, maxIter)
 * (numa-PageRankDelta.C:402) with PR_F / PR_Vertex_F_FirstRound /
 * PR_Vertex_F / PR_Vertex_Reset (64-132) and the loop at 198-230: p = 0,
 * Delta = 1/n, frontier = all; each round the frontier pushes
 * Delta[s]/outdeg(s) into nghSum, then every vertex updates (first round:
 * Delta = damping*(p + nghSum) + (1-damping)/n - p, p += Delta,
 * Delta -= 1/n; later: Delta = damping*nghSum, p += Delta) and stays in the
 * frontier when |Delta| > epsilon * p.  The reference uses damping 0.85,
 * epsilon 0.01 (epsilon2, 407) and runs exactly maxIter rounds (iters >= 1
 * here: its default of -1 never stops).  threshold: the direction switch of
 * the rounds after the first (which always pulls); 0 pulls every round as the
 * reference's threshold 0 does (211); < 0 selects m/20, letting rounds with a
 * small frontier push with atomics (FP sums then vary in the last bits run
 * to run).  dtype PM_F32 or PM_F64; ranks: n values.  stats->reached = size
 * of the final frontier.  The graph must have no self loops. */
PM_API pm_status pm_pagerank_delta(pm_graph *g, int iters, double damping, double epsilon, int dtype,
                                   void *ranks, uint32_t mem, int64_t threshold,
                                   pm_traversal_stats *stats);

/* PageRank (the semantics of pm_pagerank, FP32) on every part of a disjoint
 * union independently, each with its own vertex count, all parts in ONE
 * persistent kernel launch (thread-block clusters take parts from a work
 * queue, largest first).  ranks: n floats in union vertex order. */
PM_API pm_status pm_pagerank_parts(pm_graph *g, int iters, double damping, float *ranks,
                                   uint32_t mem);

/* Personalised PageRank for k <= 32 seeds in one SpMM-shaped pass per
 * iteration.  No reference counterpart; built from PR_F's push p[s]/outdeg(s)
 * (numa-PageRank.C:87-90) and PR_Vertex_F's damping (125-137) with the
 * teleport going to the seed: x_0 = e_seed, x_{t+1}[d] = damping *
 * sum_{s->d} x_t[s]/outdeg(s) + (1 - damping) * [d == seed] on every vertex.
 * FP32 storage and sums.  out: n x k floats, row-major (out[v*k + j]). */
PM_API pm_status pm_ppr(pm_graph *g, const int32_t *seeds, int k, int iters, double damping,
                        float *out, uint32_t mem);

/* Weighted SpMV power iteration over the float weights.  Replaces
 * SPMV_main(WG, maxIter) (numa-SPMV.C:335) with SPMV_F (56-97): every
 * iteration y[d] = sum_{s->d} w(s,d) x[s] over all vertices, then x = y.
 * x0: n floats (the reference starts from 1/n, numa-SPMV.C:271). y: n
 * floats. norm1 (optional, iters doubles): FP64 L1 norm of each y. */
PM_API pm_status pm_spmv(pm_graph *g, const float *x0, int iters, float *y, uint32_t mem,
                  double *norm1);
/* pm_spmv with FP64 vectors and FP64 sums (the float weights are widened):
 * the same iteration in the reference's own precision (numa-SPMV.C keeps
 * double values), the yardstick against which the FP32 result's max-abs and
 * relative-L1 errors are measured at full size.  x0, y: n doubles. */
PM_API pm_status pm_spmv_f64(pm_graph *g, const double *x0, int iters, double *y, uint32_t mem,
                             double *norm1);

/* ---- Differentiation (no reference counterpart; weighted forms of SPMV_F,
 * numa-SPMV.C:72-81, with PR_Vertex_F's damping, numa-PageRank.C:125-137).
 * W = the float weights of pm_graph_set_weights_f32, per CSR edge, and
 * (A_W^T x)[v] = sum_{e = s->v} W_e x[s].  Fixed points iterate until
 * sum|x_{t+1} - x_t| <= tol * sum|x_{t+1}| (FP64 sums on the device) or
 * max_iters; *iters / *resid report the passes and the last relative change.
 * All float arrays live in mem's space. */

/* Weighted PageRank p = damping * A_W^T p + (1 - damping)/n from p = 1/n. */
PM_API pm_status pm_weighted_pagerank(pm_graph *g, double damping, double tol, int max_iters,
                                      float *p, uint32_t mem, int *iters, double *resid);

/* Adjoint of the weighted PageRank fixed point for a cotangent grad_p
 * (dL/dp, n floats) at the solution p: lambda = damping * A_W lambda +
 * grad_p by the transposed iteration (a pull over the CSR), then
 * dw[e] = dL/dW_e = damping * lambda[v] * p[s] for every CSR edge e = s->v
 * (m floats).  lambda (n floats) may be NULL. */
PM_API pm_status pm_pagerank_adjoint(pm_graph *g, double damping, double tol, int max_iters,
                                     const float *p, const float *grad_p, float *dw, float *lambda,
                                     uint32_t mem, int *iters, double *resid);

/* Backward of one weighted SpMV y = A_W^T x for a cotangent grad_y:
 * dx = A_W grad_y (a pull over the CSR, n floats), dw[e] = grad_y[v] * x[s]
 * (m floats).  Either output may be NULL. */
PM_API pm_status pm_spmv_backward(pm_graph *g, const float *x, const float *grad_y, float *dx,
                                  float *dw, uint32_t mem);

/* Lognormal(0, 1) weights normalised per source row, generated on the
 * device and set as the graph's float weights. */
PM_API pm_status pm_graph_gen_weights_lognormal(pm_graph *g, uint64_t seed);

/* Two-state belief propagation.  Replaces BeliefPropagation(G, maxIter)
 * (numa-BP.C:528) with BP_F / BP_Vertex_Reset (89-140) and
 * edgeMapDenseBPNoRep (179-230): for every out-edge s->d of the frontier,
 * belief[i] = sum_j prior_d[j] psi[i][j] prod_d[j], prod'_d[i] *= belief[i];
 * prod' resets to 1 on the frontier; the next frontier is every vertex that
 * received a message.  Products start at 1 and are carried as natural logs
 * (log_prod, n x 2 floats) so that vertices with thousands of in-edges do
 * not underflow.  prior: n x 2 floats; psi: 4 floats [i][j], shared by all
 * edges. */
PM_API pm_status pm_bp(pm_graph *g, const float *prior, const float *psi, int iters, float *log_prod,
                uint32_t mem);
/* pm_bp in FP64 (prior n x 2, psi 4, log_prod n x 2 doubles; device arrays
 * 16-byte aligned): the yardstick for the FP32 result's error. */
PM_API pm_status pm_bp_f64(pm_graph *g, const double *prior, const double *psi, int iters,
                           double *log_prod, uint32_t mem);

/* PageRank for callers that cannot allocate GPU memory.  No counterpart in
 * the reference.  Some hosts may not call cudaMalloc while they run (a
 * plugin in a process whose device memory another runtime pools, a caller
 * that gave all device memory to its own allocator); every other entry point
 * here allocates (a graph handle owns its CSC, tables and workspaces).  This
 * one allocates nothing: offsets (n+1) and edges (m) are a CSR already in
 * device memory, ranks (n floats) is a device output, and the working
 * vectors live in a fixed array inside the library, sized for at most
 * 1048576 vertices (about 8.3 MB, held on every GPU that loads the library
 * until the process exits); larger n is rejected with PM_ERR_INVALID_ARG.
 * Semantics are pm_pagerank's with PM_F32; pushes use atomics, so sums may
 * differ from pm_pagerank in the last bits.  Each call first checks the CSR
 * on the device and returns PM_ERR_BAD_GRAPH, computing nothing, when
 * offsets are not monotone within [0, m], offsets[0] != 0, offsets[n] != m,
 * an id lies outside [0, n) or an edge is a self loop.  Runs on `stream`
 * (NULL = default stream) of the current device, reads a status word back
 * after the check and after the last iteration, and returns when done.
 * The first call on a device looks up the array's address for that device
 * (and, with CUDA's lazy module loading, is when the array's memory is
 * reserved): make it before any stream capture and before handing the
 * device's free memory to another allocator.  All calls on a device share
 * the array: calls that overlap on the GPU race. */
PM_API pm_status pm_pagerank_static(const int32_t *offsets, const int32_t *edges, int64_t n,
                                    int64_t m, int iters, double damping, float *ranks,
                                    void *stream);

/* Device timing on the graph's stream (CUDA events): begin, then end
 * returns the elapsed milliseconds. */
PM_API pm_status pm_timer_begin(pm_graph *g);
PM_API pm_status pm_timer_end(pm_graph *g, float *ms);

/* Per-pass device profile.  When enabled, every edgeMap pass of an
 * application (one PageRank / SpMV / BP iteration, one BFS / CC /
 * BellmanFord round) is bracketed by CUDA events on the graph's stream.
 * pm_profile_read sums the passes recorded under tag ("pagerank",
 * "spmv", "bp", "bfs", "cc", "bellman_ford"): total milliseconds and count;
 * reset clears the records.  No counterpart in the reference, whose only
 * timers are gettimeofday() around whole runs (gettime.h:30-113). */
PM_API pm_status pm_profile_enable(pm_graph *g, int enable);
PM_API pm_status pm_profile_read(pm_graph *g, const char *tag, double *total_ms, int64_t *passes,
                                 int reset);

/* Run-time tunables of a graph handle.  No counterpart in the reference,
 * which fixes its load-balance cut-offs at compile time and passes each
 * application's direction-switch threshold in code (BFS 0, numa-BFS.C:268;
 * CC m/8, numa-Components.C:226; BellmanFord m/20, numa-BellmanFord.C:182).
 * Results never depend on them; only speed does. */
#define PM_TUNE_HEAVY_DEG 0        /* rows with more edges are split in 4096-edge chunks
                                      (default 1024, range [64, 2^30]) */
#define PM_TUNE_CTA_EXPAND 1       /* sparse push: CTA-wide expansion from this
                                      out-degree (default 128) */
#define PM_TUNE_GRID_EXPAND 2      /* sparse push: grid-wide expansion from this
                                      out-degree (default 256; at most 4096 such rows per
                                      round, the rest expand CTA-wide) */
#define PM_TUNE_PULL_CTAS_PER_SM 3 /* resident CTAs per SM of the persistent pulls,
                                      0 = the occupancy limit (default) */
#define PM_TUNE_BFS_DIV 4          /* threshold < 0 means m / div: BFS (default 20) */
#define PM_TUNE_CC_DIV 5           /* ... Components (default 8) */
#define PM_TUNE_BF_DIV 6           /* ... BellmanFord (default 20) */
#define PM_TUNE_CUDA_GRAPHS 7      /* 1 (default): the fixed-iteration loops of PageRank,
                                      SpMV, BP and PPR run as CUDA graphs, captured the
                                      second time a handle runs the same loop (same
                                      sizes, buffers and scalars) and replayed from
                                      then on, and BFS runs its rounds inside one CUDA
                                      graph whose WHILE node chooses each round's
                                      direction on the GPU; 0: plain launches */
#define PM_TUNE_HEAVY_MODE 8       /* how the chunks of heavy rows are summed: 0 (default)
                                      a launch before the pull; 1 inside the pull launch
                                      (warps take them first, a row's lane waits for its
                                      chunks, bounded); 2 a launch beside the pull on a
                                      second stream, the heavy rows committed after both */
#define PM_TUNE_HUB_CACHE 9        /* FP32 PageRank: the contributions of up to this many
                                      highest out-degree sources are kept in every SM's
                                      shared memory during a pass (0 = off, the default; at
                                      most 16384; results are unchanged; slower than the
                                      plain pull on the R-MAT workloads measured) */
#define PM_TUNE_MULTI_DIV 10       /* threshold < 0 means m / div: multi-source BFS and
                                      BellmanFord (default 8; their union frontiers turn
                                      dense sooner than one source's) */
#define PM_TUNE_BF_DENSE 11        /* BellmanFord's dense rounds: 0 a pull-reduce
                                      over every in-edge (min of dist[s] + w over frontier
                                      sources); 1 a push over the frontier's out-edges with
                                      atomicMin, edgeMap's DENSE_FORWARD option, which the
                                      reference's BellmanFord passes (numa-BellmanFord.C:182);
                                      2 (default) the same push with atomics whose result is
                                      unused, skipped when the target's distance is already
                                      no larger, the next frontier taken from the distances
                                      that fell.
                                      Same distances; ignored on a partition handle (pull
                                      only) */
#define PM_TUNE_CC_MODE 12         /* Components on a symmetric whole-graph handle: 0
                                      (default) a concurrent union-find (sampled links,
                                      the largest component skipped, roots are minimum
                                      ids); 1 the reference's min-label propagation rounds
                                      (threshold chooses their direction).  Same labels
                                      either way; directed and partition handles always
                                      propagate */
#define PM_TUNE_BF_DELTA 13        /* BellmanFord schedule: 0 (default) every round
                                      relaxes the whole frontier; Delta > 0 relaxes only
                                      the frontier vertices with dist < T, the others wait,
                                      and T moves to (least waiting distance) + Delta when
                                      none is below it (delta-stepping).  Same distances;
                                      range [0, 2^30]; ignored on a partition handle */
#define PM_TUNE_PULL_STAGE 14      /* pull-reduce passes (heavy mode 0, no hub cache, ids
                                      without paired weights): 1 copies each 32-row
                                      batch's CSC ids (up to 1024) into shared memory with
                                      one bulk copy and reads them there; 0 (default)
                                      reads them from global memory.  Same results */
#define PM_TUNE_PUSH_AGG 15        /* sparse push rounds of Components and BellmanFord: 1
                                      combines the atomicMin updates of a warp's lanes that
                                      share a target (one atomic per target per warp); 0
                                      (default) one atomic per edge.  Same results */
/* g == NULL sets / reads the process-wide values that handles created
 * afterwards start with (so tables that depend on them are built once);
 * changing PM_TUNE_HEAVY_DEG on a handle rebuilds its heavy-row tables. */
PM_API pm_status pm_graph_set_tunable(pm_graph *g, int key, int64_t value);
PM_API pm_status pm_graph_get_tunable(pm_graph *g, int key, int64_t *value);

/* Autotuner: coordinate descent over the tunables application `app` uses
 * (candidates per tunable, each timed three times after a warm-up on the
 * graph's stream with CUDA events, the fastest run counting, a change kept
 * when it saves more than 2 %); the winners stay set on the handle.
 * PageRank / SpMV / BP time 3 iterations (SpMV needs float weights), BFS
 * eight fixed sources, CC one run,
 * BellmanFord one source (needs int32 weights). */
#define PM_APP_PAGERANK 0
#define PM_APP_SPMV 1
#define PM_APP_BP 2
#define PM_APP_BFS 3
#define PM_APP_CC 4
#define PM_APP_BF 5
typedef struct pm_tune_report {
  int64_t trials;     /* candidate settings timed                 */
  double default_ms;  /* time of the settings the handle started with */
  double best_ms;     /* time of the settings kept                  */
} pm_tune_report;
PM_API pm_status pm_tune(pm_graph *g, int app, pm_tune_report *report);
/* The same over a mix of applications that share the handle (count <= 6):
 * the objective is their summed time, the tunables are the union of theirs,
 * and the descent sweeps them twice when the first sweep moved one -- the
 * shared cut-offs are then chosen for the mix, not for whichever application
 * was tuned last. */
PM_API pm_status pm_tune_mix(pm_graph *g, const int *apps, int count, pm_tune_report *report);

/* Run the handle's work on a caller's CUDA stream (a cudaStream_t of the
 * handle's device), so that it is ordered after the caller's earlier work on
 * that stream; NULL returns to the handle's own stream.  Calls stay
 * synchronous: each returns once its work on the stream is done.  The
 * reference runs on its own threads; no counterpart. */
PM_API pm_status pm_graph_set_stream(pm_graph *g, void *stream);

/* Device-memory cache.  The library allocates its device buffers through a
 * per-process cache: a freed buffer (a graph's arrays after
 * pm_graph_destroy, build temporaries, grown workspaces) stays reserved and
 * is handed to a later request of close size, after a device
 * synchronisation, instead of going through cudaFree / cudaMalloc.
 * max_bytes: -1 (default) caps the cache at a quarter of the device's
 * memory, 0 turns it off, > 0 caps it there; lowering the cap below what is
 * cached releases everything.  Memory held by the cache is not available to
 * other allocators in the process (a framework's own caching allocator, for
 * example) until released.  No reference counterpart. */
PM_API pm_status pm_set_memory_cache(int64_t max_bytes);
PM_API pm_status pm_release_memory_cache(void);
PM_API pm_status pm_memory_cache_info(int64_t *cached_bytes);

/* Pinned (page-locked) host memory for fast host<->device staging. */
PM_API pm_status pm_host_alloc(uint64_t bytes, void **out);
PM_API pm_status pm_host_free(void *p);

/* Number of kernels this library launched since the last reset. */
PM_API int64_t pm_kernel_launches(int reset);

/* ---- failure tests (no reference counterpart: the reference aborts or
 * prints and goes on).  Both fail on purpose, on the host's terms: nothing
 * faults, traps or hangs a GPU.
 * pm_test_fail_alloc_after(k): the k-th device allocation of the library
 * from now on fails as an out-of-memory would (PM_ERR_OOM from the call that
 * made it; the handle stays usable); k < 1 turns it off.
 * pm_test_wait_timeout(device, max_polls): runs the bounded device wait the
 * persistent kernels use (a poll every 256 ns, max_polls at most) on a flag
 * that nothing sets; it gives up, the kernel returns, and the call returns
 * PM_ERR_TIMEOUT with the device still usable.  max_polls in [1, 2^22]. */
PM_API pm_status pm_test_fail_alloc_after(int64_t k);
PM_API pm_status pm_test_wait_timeout(int device, int32_t max_polls);

PM_API const char *pm_last_error(void);
PM_API const char *pm_version(void);

#ifdef __cplusplus
}
#endif
#endif /* POLYMER_B200_H */
