// pm_graph.cuh -- the graph handle behind the C ABI.
#pragma once
#include <memory>
#include <string>
#include <vector>

#include "polymer.cuh"

namespace pm {

// Device memory of the library, through a per-process cache of freed blocks
// (pm_set_memory_cache): dev_alloc returns a block of at least `bytes`
// (*cap: its size), reusing a cached block of close size; dev_free caches
// the block, or frees it when the cache is full or off.
//
// Reuse is stream-ordered.  Every C-ABI call names the stream its work runs
// on (AllocCtx, set by the call's entry and cleared on its exit).  A block
// freed inside a call carries an event recorded on that stream; the call
// that takes it makes its own stream wait on the event, so two host threads
// that run distinct handles never wait for each other's kernels.  A block
// freed with no stream known (C++ engine users outside the C ABI) makes the
// next taker synchronise the device first; a block freed while `idle` (a
// handle's destructor, after its streams were synchronised) needs neither.
struct AllocCtx {
  cudaStream_t stream = nullptr;
  bool idle = false;
};
PM_CXX_API AllocCtx alloc_ctx();
PM_CXX_API void set_alloc_ctx(AllocCtx c);
PM_CXX_API void *dev_alloc(size_t bytes, size_t *cap, int *device);
// Tests: the k-th dev_alloc from now on fails with PM_ERR_OOM (k < 1: off).
void set_alloc_fail_after(long long k);
PM_CXX_API void dev_free(void *p, size_t cap, int device);
// Small pinned host blocks, reused without cudaFreeHost (which synchronises
// the device).
PM_CXX_API void *pinned_small_alloc(size_t bytes);
PM_CXX_API void pinned_small_free(void *p, size_t bytes);

// Sets the allocation context for the lifetime of the object, then puts the
// previous one back.
struct AllocScope {
  AllocCtx saved;
  explicit AllocScope(AllocCtx c) : saved(alloc_ctx()) { set_alloc_ctx(c); }
  ~AllocScope() { set_alloc_ctx(saved); }
  AllocScope(const AllocScope &) = delete;
  AllocScope &operator=(const AllocScope &) = delete;
};

// First base of pm_graph: its destructor runs after every member's, so the
// idle context that ~pm_graph sets (its streams are synchronised by then)
// covers the members' frees and is undone afterwards.
struct IdleFreeBase {
  AllocCtx saved{};
  ~IdleFreeBase() { set_alloc_ctx(saved); }
};

// Owning device buffer.
struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;  // capacity (at least what alloc asked for)
  int device = 0;    // where the block lives
  DevBuf() = default;
  explicit DevBuf(size_t b) { alloc(b); }
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  DevBuf(DevBuf &&o) noexcept : p(o.p), bytes(o.bytes), device(o.device) { o.p = nullptr; o.bytes = 0; }
  DevBuf &operator=(DevBuf &&o) noexcept {
    reset();
    p = o.p; bytes = o.bytes; device = o.device; o.p = nullptr; o.bytes = 0;
    return *this;
  }
  ~DevBuf() { reset(); }
  void alloc(size_t b) {
    reset();
    p = dev_alloc(b ? b : 16, &bytes, &device);
  }
  void reset() {
    if (p) dev_free(p, bytes, device);
    p = nullptr;
    bytes = 0;
  }
  template <class T> T *as() const { return static_cast<T *>(p); }
};

// One adjacency direction with its load-balance tables.
struct AdjBuf {
  DevBuf off, idx, gstart, hrow, hfirst;
  int32_t ngroups = 0, nchunks = 0;
  Adj view() const {
    Adj a;
    a.off = off.as<int32_t>();
    a.idx = idx.as<int32_t>();
    a.gstart = gstart.as<int32_t>();
    a.hrow = hrow.as<int32_t>();
    a.hfirst = hfirst.as<int32_t>();
    a.ngroups = ngroups;
    a.nchunks = nchunks;
    return a;
  }
};

}  // namespace pm

struct pm_graph : pm::IdleFreeBase {
  int device = 0;
  int64_t n = 0, m = 0;
  bool symmetric = false;
  bool has_self_loops = false;
  int32_t max_out_deg = 0;
  pm::AdjBuf out, in;     // in.* empty when symmetric (views alias out)
  pm::DevBuf in_eid;      // CSC slot -> CSR edge id (directed graphs)
  pm::DevBuf out_src;     // source of every CSR edge (built on first use)
  pm::DevBuf w_i32_out, w_i32_in, w_f32_out, w_f32_in;
  pm::DevBuf w_f32_pair_in;   // {CSC source, float weight} per CSC slot, built on first use
  pm::DevBuf w_f32_pair_out;  // {CSR destination, float weight} per CSR slot, likewise
  pm::Engine E;
  cudaStream_t own_stream = nullptr;  // created with the handle; E.stream may be a caller's
  pm::DevBuf cnt, bits0, bits1, queue0, queue1, defer, hubs, partials, hdone;
  pm::DevBuf check_word;  // checked builds: set by a kernel that met an id outside [0, n)
  pm::Counters *h_cnt = nullptr;  // pinned
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<pm::DevBuf> scratch;  // per-call workspaces kept across calls
  // disjoint parts (a batch of independent graphs): vertex ranges and the
  // largest-first order in which persistent kernels take them
  std::vector<int64_t> parts;       // count+1 vertex offsets (host copy); empty if none
  pm::DevBuf parts_vbase, parts_order;
  // 1D vertex partition across processes (pm_graph_create_partition): this
  // handle holds the edges whose destination lies in [part_lo, part_hi)
  // (rank r owns [part_bounds[r], part_bounds[r+1]); part_wbounds are the
  // same bounds in bitmap words), the in-adjacency groups cover only those
  // rows, and glob_off keeps the whole graph's CSR offsets (global
  // out-degrees).  part_fn gathers every rank's range of a vertex array into
  // every rank's copy.
  bool is_part = false;
  int part_rank = 0, part_count = 1;
  int64_t part_lo = 0, part_hi = 0;
  std::vector<int64_t> part_bounds, part_wbounds;
  pm::DevBuf glob_off;
  // hub cache of the FP32 PageRank pull (pm_hubs.cu): the hub_count sources
  // of highest out-degree (hub_ids), the CSC sources with theirs tagged as
  // ~slot (hub_idx) and a pass's copy of their values (hub_vals); built for
  // hub_for sources at most (-1: not built)
  pm::DevBuf hub_ids, hub_idx, hub_vals;
  int hub_count = 0, hub_for = -1;
  int (*part_fn)(void *user, void *buf, int64_t elem_bytes, const int64_t *bounds, int nranks,
                 void *stream) = nullptr;
  void *part_user = nullptr;

  pm::VertexSubset subset(int k) {
    pm::VertexSubset s;
    s.n = (int32_t)n;
    s.bits = (k == 0 ? bits0 : bits1).as<uint32_t>();
    s.queue = (k == 0 ? queue0 : queue1).as<int32_t>();
    return s;
  }
  // Scratch slot i with at least bytes capacity (kept for reuse).
  void *scratch_buf(size_t i, size_t bytes) {
    if (scratch.size() <= i) scratch.resize(i + 1);
    if (scratch[i].bytes < bytes) scratch[i].alloc(bytes);
    return scratch[i].p;
  }
  ~pm_graph();
};

namespace pm {
// Builds every derived structure (CSC, groups, heavy chunks, workspaces)
// once out.off / out.idx hold a validated CSR on the device.
void finish_graph(pm_graph *g);
// Rebuilds what depends on E.tune (heavy tables when heavy_deg changed from
// old_heavy_deg, the views, the partials) and drops captured loops.
void apply_tunables(pm_graph *g, int32_t old_heavy_deg);
// Writes in_w = out_w[in_eid] (or aliases for symmetric graphs).
void permute_weights_i32(pm_graph *g);
void permute_weights_f32(pm_graph *g);
// The float weights paired with their CSC source ids, or with their CSR
// destination ids when csr (built once per weights).
const WPair *ensure_f32_pairs(pm_graph *g, bool csr = false);

// Hub tables for the handle's hub_cache tunable (rebuilt when it changed).
void ensure_hubs(pm_graph *g);
// vals[i] = x[ids[i]]: the cached sources' values for one pass.
void hub_values(pm_graph *g, const float *x);

// ---- 1D vertex partition (pm_partition.cu) ----
// Splits the validated CSR's vertices into nranks ranges of about equal
// in-edges + kRowWork * rows (the pull work of a range), every interior
// bound a multiple of 32 (whole bitmap words); keeps the edges (and weights)
// whose destination lies in rank's range; records the bounds and the whole
// graph's offsets.
void restrict_to_partition(pm_graph *g, int rank, int nranks, DevBuf *w);
// Every rank's range of buf (n entries of elem_bytes) into every rank's
// buf, through the handle's exchange function, in stream order.
void part_exchange(pm_graph *g, void *buf, size_t elem_bytes);
// Every rank's words of a frontier bitmap into every rank's copy.
void part_exchange_bits(pm_graph *g, uint32_t *bits);
// After a round on a partition: the next frontier's bitmap made global, its
// size and out-degree sum recounted.
void part_round(pm_graph *g, VertexSubset &next);
}  // namespace pm
