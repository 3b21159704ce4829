// An application written against the engine API (include/polymer_b200_engine.cuh)
// with its own functors, compiled outside the library, as a Polymer application
// is written against polymer.h: connected components by MAX-label propagation
// (the mirror image of numa-Components.C's min labels), through edgeMapReduce
// (sparse push or pull-reduce) or, with push != 0, edgeMap with the
// DENSE_FORWARD option (sparse push or dense push over the frontier's
// out-edges, updateAtomic only), vertexMapAll and a vertexFilter that counts
// the component roots.  Test infrastructure: built and loaded by
// tests/test_gpu_engine_api.py.
#include <utility>

#include "polymer_b200_engine.cuh"

namespace {

struct MaxLabel_F {
  int32_t *ids;
  const uint32_t *cur;  // the frontier: only its sources carry a label this round
  using Acc = int32_t;
  __device__ __forceinline__ bool cond(int) const { return true; }
  __device__ __forceinline__ bool updateAtomic(int s, int d, int) const {
    const int32_t v = *((volatile int32_t *)ids + s);
    return v > atomicMax(ids + d, v);
  }
  __device__ __forceinline__ Acc identity() const { return -1; }
  __device__ __forceinline__ Acc edge(int s, int, int) const {
    return pm::test_bit(cur, s) ? *((volatile int32_t *)ids + s) : -1;
  }
  __device__ __forceinline__ Acc combine(Acc a, Acc b) const { return a > b ? a : b; }
  __device__ __forceinline__ bool commit(int d, Acc acc, double2 &) const {
    if (acc > ids[d]) {
      ids[d] = acc;
      return true;
    }
    return false;
  }
};

struct Init_F {
  int32_t *ids;
  __device__ __forceinline__ void operator()(int v) const { ids[v] = v; }
};

struct Root_F {
  const int32_t *ids;
  __device__ __forceinline__ bool operator()(int v) const { return ids[v] == v; }
};

}  // namespace

// labels: n int32 on the graph's device.  Returns a pm_status.
extern "C" __attribute__((visibility("default"))) int user_max_label(pm_graph *g, int32_t *labels,
                                                                    int64_t threshold, int push, int64_t *roots,
                                                                    int *rounds, int *dense_rounds) {
  try {
    PM_CUDA(cudaSetDevice(g->device));
    pm::Engine &E = g->E;
    pm::VertexSubset cur = g->subset(0), next = g->subset(1);
    pm::vertexMapAll(E, (int32_t)g->n, Init_F{labels});
    pm::subset_all(E, cur);
    int r = 0, dr = 0;
    while (cur.size > 0) {
      bool dense = false;
      if (push)
        pm::edgeMap<int>(E, cur, MaxLabel_F{labels, cur.bits}, next, threshold, pm::DENSE_FORWARD, nullptr,
                         nullptr, &dense);
      else
        pm::edgeMapReduce<int>(E, cur, MaxLabel_F{labels, cur.bits}, next, threshold, nullptr, nullptr, &dense);
      std::swap(cur, next);
      ++r;
      dr += dense;
    }
    pm::subset_all(E, cur);
    pm::VertexSubset out = g->subset(1);
    pm::vertexFilter(E, cur, Root_F{labels}, out);
    *roots = out.size;
    *rounds = r;
    *dense_rounds = dr;
    PM_CUDA(cudaStreamSynchronize(E.stream));
    return 0;
  } catch (const pm::Failure &f) {
    pm::set_last_error(f.what());
    return (int)f.status;
  }
}
