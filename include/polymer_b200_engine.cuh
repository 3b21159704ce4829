/*
 * polymer_b200_engine.cuh -- the C++/CUDA engine API, for applications that
 * bring their own functors, as Polymer's applications do against polymer.h.
 *
 * Polymer's API surface is a header of templates: a graph, a vertex subset,
 * edgeMap(G, frontier, F, threshold, option), vertexMap and vertexFilter
 * (polymer.h:2224-2441), with functors providing cond / update /
 * updateAtomic (and initFunc / reduceFunc / combineFunc for the reducing
 * pull).  The same surface here, over a device graph handle:
 *
 *   pm_graph *g;                      // pm_graph_create / _rmat / _load_pbbs
 *   pm::Engine &E = g->E;             // stream, counters, views of CSR + CSC
 *   pm::VertexSubset cur = g->subset(0), next = g->subset(1);
 *   pm::subset_single(E, cur, src);   // or subset_all
 *   pm::edgeMap<int>(E, cur, F{...}, next, threshold);        // sparse push / dense pull
 *   pm::edgeMapReduce<int>(E, cur, F{...}, next, threshold);  // sparse push / pull-reduce
 *   pm::vertexMap(E, cur, V{...});
 *   pm::vertexFilter(E, cur, P{...}, out);
 *
 * Functor contract (all __device__, const members):
 *   bool cond(int d)                          -- d may still be updated
 *   bool updateAtomic(int s, int d, W w)      -- safe under concurrency; true
 *                                                when d joins the next frontier
 *   Acc identity(); Acc edge(int s, int d, W w); Acc combine(Acc, Acc);
 *   bool commit(int d, Acc acc, double2 &aux) -- reducing pull: fold the row
 *                                                (the vertexMap fused into it);
 *                                                true when d joins the frontier
 * W is the weight type of the weight arrays passed to edgeMap (int when none).
 * Frontier sizes and out-degree sums come back in VertexSubset::size / edges.
 *
 * Build an application .cu with
 *   nvcc -gencode arch=compute_100a,code=sm_100a -std=c++17 --expt-relaxed-constexpr \
 *        -I<repo>/include app.cu -L<repo>/polymer_b200 -lpolymer_b200
 * Engine calls report failures as pm::Failure exceptions (a pm_status plus a
 * message); catch them at your own C boundary.
 */
#ifndef POLYMER_B200_ENGINE_CUH
#define POLYMER_B200_ENGINE_CUH

#include "polymer_b200.h"
#include "pm/pm_graph.cuh"

#endif
