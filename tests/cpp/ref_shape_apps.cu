// Applications whose functors keep the shape of the reference's own
// (Polymer's reducing-pull contract: initFunc / reduceFunc / combineFunc over
// a 16-byte scratch, a two-argument updateAtomic, the writeMin / writeAdd
// atomics of utils.h), compiled outside the library against
// include/polymer_b200_engine.cuh and run through pm::edgeMapReduce and
// pm::vertexMap.  Test infrastructure: built and loaded by
// tests/test_gpu_engine_api.py.
//   ref_components: the min-label loop of numa-Components.C:233-281 with
//     CC_F / CC_Vertex_F as numa-Components.C:55-119 define them.
//   ref_pagerank:   the loop of numa-PageRank.C:273-335 (edgeMap, then
//     PR_Vertex_F and PR_Vertex_Reset on the frontier, swap) with PR_F's
//     reducing members (numa-PageRank.C:98-119) and FP64 ranks.
#include <utility>

#include "polymer_b200_engine.cuh"

namespace {

using pm::writeAdd;
using pm::writeMin;

struct CC_F {
  int32_t *IDs;
  int32_t *prevIDs;
  __device__ bool updateAtomic(int s, int d) {
    int32_t origID = IDs[d];
    return writeMin(&IDs[d], *((volatile int32_t *)IDs + s)) && origID == prevIDs[d];
  }
  __device__ void initFunc(void *dataPtr, int d) {
    int32_t *tmp = (int32_t *)dataPtr;
    tmp[0] = IDs[d];
    tmp[1] = prevIDs[d];
  }
  __device__ bool reduceFunc(void *dataPtr, int s) {
    int32_t *tmp = (int32_t *)dataPtr;
    int32_t origID = tmp[0];
    int32_t v = *((volatile int32_t *)IDs + s);
    if (v < origID) {
      tmp[0] = min(origID, v);
      if (origID == tmp[1]) return true;
    }
    return false;
  }
  __device__ bool combineFunc(void *dataPtr, int d) {
    int32_t newVal = *(int32_t *)dataPtr;
    int32_t origID = IDs[d];
    return writeMin(&IDs[d], newVal) && origID == prevIDs[d];
  }
  __device__ bool cond(int) { return true; }
};

struct CC_Vertex_F {
  int32_t *IDs;
  int32_t *prevIDs;
  __device__ bool operator()(int i) {
    prevIDs[i] = IDs[i];
    return true;
  }
};

struct Init_Ids {
  int32_t *IDs, *prevIDs;
  __device__ void operator()(int i) const { IDs[i] = prevIDs[i] = i; }
};

struct PR_F {
  double *p_curr, *p_next;
  const int32_t *out_off;  // the graph's CSR offsets: out-degree of s
  __device__ double outdeg(int s) const { return (double)(out_off[s + 1] - out_off[s]); }
  __device__ bool updateAtomic(int s, int d) {
    writeAdd(&p_next[d], p_curr[s] / outdeg(s));
    return true;
  }
  __device__ void initFunc(void *dataPtr, int) { *(double *)dataPtr = 0.0; }
  __device__ bool reduceFunc(void *dataPtr, int s) {
    *(double *)dataPtr += p_curr[s] / outdeg(s);
    return true;
  }
  __device__ bool combineFunc(void *dataPtr, int d) {
    writeAdd(&p_next[d], *(double *)dataPtr);
    return true;
  }
  __device__ bool cond(int) { return true; }
};

struct PR_Vertex_F {
  double *p_curr, *p_next;
  double damping, addedConstant;
  __device__ bool operator()(int i) {
    p_next[i] = damping * p_next[i] + addedConstant;
    return true;
  }
};

struct PR_Vertex_Reset {
  double *p_curr;
  __device__ bool operator()(int i) {
    p_curr[i] = 0.0;
    return true;
  }
};

struct Init_P {
  double *p_curr, *p_next;
  double p0;
  __device__ void operator()(int i) const {
    p_curr[i] = p0;
    p_next[i] = 0.0;
  }
};

template <class Body>
int guarded(pm_graph *g, Body body) {
  try {
    PM_CUDA(cudaSetDevice(g->device));
    body();
    PM_CUDA(cudaStreamSynchronize(g->E.stream));
    return 0;
  } catch (const pm::Failure &f) {
    pm::set_last_error(f.what());
    return (int)f.status;
  }
}

}  // namespace

// ids, prev: n int32 each on the graph's device; ids ends as the labels.
extern "C" __attribute__((visibility("default"))) int ref_components(pm_graph *g, int32_t *ids, int32_t *prev,
                                                                    int64_t threshold, int *rounds,
                                                                    int *dense_rounds) {
  return guarded(g, [&] {
    pm::Engine &E = g->E;
    pm::VertexSubset cur = g->subset(0), next = g->subset(1);
    pm::vertexMapAll(E, (int32_t)g->n, Init_Ids{ids, prev});
    pm::subset_all(E, cur);
    int r = 0, dr = 0;
    while (cur.size > 0) {
      pm::vertexMap(E, cur, CC_Vertex_F{ids, prev});
      bool dense = false;
      pm::edgeMapReduce<int>(E, cur, CC_F{ids, prev}, next, threshold, nullptr, nullptr, &dense);
      std::swap(cur, next);
      ++r;
      dr += dense;
    }
    *rounds = r;
    *dense_rounds = dr;
  });
}

// pa, pb: n doubles each on the graph's device; after maxIter iterations the
// ranks are in pa when maxIter is even, else in pb (the reference's swap).
extern "C" __attribute__((visibility("default"))) int ref_pagerank(pm_graph *g, double *pa, double *pb, int maxIter,
                                                                  int64_t threshold) {
  return guarded(g, [&] {
    pm::Engine &E = g->E;
    const double damping = 0.85, n = (double)g->n;
    pm::VertexSubset cur = g->subset(0), next = g->subset(1);
    double *p_curr = pa, *p_next = pb;
    pm::vertexMapAll(E, (int32_t)g->n, Init_P{p_curr, p_next, 1.0 / n});
    pm::subset_all(E, cur);
    for (int it = 0; it < maxIter; ++it) {
      pm::edgeMapReduce<int>(E, cur, PR_F{p_curr, p_next, E.g.out.off}, next, threshold);
      pm::vertexMap(E, cur, PR_Vertex_F{p_curr, p_next, damping, (1.0 - damping) * (1.0 / n)});
      pm::vertexMap(E, cur, PR_Vertex_Reset{p_curr});
      std::swap(p_curr, p_next);
      std::swap(cur, next);
    }
  });
}
