// pm_dump.cu -- the reference's graph dump: dumpGraphToBin / loadGraphFromBin
// (IO-numa.h:758-900), a graph cache file that holds both adjacency
// directions so that a reload needs no parsing.
//
// Layout (native byte order, no padding): int64 total bytes, int32 n, int64
// m, then for every vertex i in order a record of int32 words
//   -1, i, out-degree, in-degree, the out-neighbours, the in-neighbours.
// Neighbour ids are never negative, so every -1 word of the body starts a
// record.  Loading copies the body to the device once; one compaction finds
// the n record starts, every vertex checks its record (its id, its degrees,
// that it ends where the next one starts), a scan of the out-degrees gives
// the CSR offsets and a warp per vertex copies its out-list.  The in-lists
// are checked for length only: the CSC is rebuilt from the CSR, as for every
// other input.  Saving assembles the records on the device (a scan of the
// record lengths, a warp per vertex) and writes them with one copy out.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>

#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include "pm_graph.cuh"

namespace pm {

namespace {

constexpr int64_t kDumpHeader = 8 + 4 + 8;  // total bytes, n, m

__global__ void k_dump_marks(const int32_t *words, int64_t count, int32_t *flag) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < count; w += stride) flag[w] = words[w] == -1;
}

// Record i at starts[i]: its id, its degrees, its end at the next record.
__global__ void k_dump_records(const int32_t *words, int64_t nwords, const int32_t *starts, int64_t n,
                               int32_t *outdeg, unsigned *err) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int64_t p = starts[i];
    const int64_t next = i + 1 < n ? (int64_t)starts[i + 1] : nwords;
    bool ok = (i > 0 || p == 0) && p + 4 <= next && words[p + 1] == (int32_t)i;  // the body starts with record 0
    int32_t od = 0, id = 0;
    if (ok) {
      od = words[p + 2];
      id = words[p + 3];
      ok = od >= 0 && id >= 0 && p + 4 + (int64_t)od + (int64_t)id == next;
    }
    outdeg[i] = ok ? od : 0;
    if (!ok) atomicOr(err, 1u);
  }
}

__global__ void k_dump_copy(const int32_t *words, const int32_t *starts, const int32_t *off, int64_t n,
                            int32_t *idx) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
    const int64_t src = (int64_t)starts[i] + 4;
    const int32_t o0 = off[i], od = off[i + 1] - off[i];
    for (int32_t k = lane; k < od; k += 32) idx[o0 + k] = words[src + k];
  }
}

// Record lengths (4 + out-degree + in-degree) and the records themselves.
__global__ void k_dump_lengths(const int32_t *out_off, const int32_t *in_off, int64_t n, int64_t *len) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    len[i] = 4 + (int64_t)(out_off[i + 1] - out_off[i]) + (int64_t)(in_off[i + 1] - in_off[i]);
}

__global__ void k_dump_write(const int32_t *out_off, const int32_t *out_idx, const int32_t *in_off,
                             const int32_t *in_idx, const int64_t *pos, int64_t n, int32_t *words) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
    int32_t *r = words + pos[i];
    const int32_t o0 = out_off[i], od = out_off[i + 1] - o0, i0 = in_off[i], id = in_off[i + 1] - i0;
    if (lane == 0) {
      r[0] = -1;
      r[1] = (int32_t)i;
      r[2] = od;
      r[3] = id;
    }
    for (int32_t k = lane; k < od; k += 32) r[4 + k] = out_idx[o0 + k];
    for (int32_t k = lane; k < id; k += 32) r[4 + od + k] = in_idx[i0 + k];
  }
}

int grid_for(int64_t threads) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((threads + 255) / 256, 148 * 32));
}

struct File {
  FILE *f = nullptr;
  File(const char *path, const char *mode) : f(fopen(path, mode)) {}
  ~File() {
    if (f) fclose(f);
  }
};

struct PinnedBuf {
  void *p = nullptr;
  explicit PinnedBuf(size_t bytes) { PM_CUDA(cudaMallocHost(&p, bytes ? bytes : 1)); }
  ~PinnedBuf() {
    if (p) cudaFreeHost(p);
  }
};

}  // namespace

void read_graph_dump(pm_graph *g, const char *path, DevBuf &off, DevBuf &idx, int64_t &n, int64_t &m) {
  cudaStream_t st = g->E.stream;
  File file(path, "rb");
  if (!file.f) fail(PM_ERR_INVALID_ARG, std::string("cannot open ") + path);
  if (fseek(file.f, 0, SEEK_END) != 0) fail(PM_ERR_INVALID_ARG, std::string("cannot seek in ") + path);
  const int64_t size = (int64_t)ftello(file.f);
  rewind(file.f);
  unsigned char head[kDumpHeader];
  if (size < kDumpHeader || fread(head, 1, kDumpHeader, file.f) != (size_t)kDumpHeader)
    fail(PM_ERR_BAD_GRAPH, "graph dump shorter than its header");
  int64_t total = 0, mm = 0;
  int32_t nn = 0;
  std::memcpy(&total, head, 8);
  std::memcpy(&nn, head + 8, 4);
  std::memcpy(&mm, head + 12, 8);
  if (total != size) fail(PM_ERR_BAD_GRAPH, "graph dump header gives " + std::to_string(total) + " bytes, file has " +
                                              std::to_string(size));
  if (nn < 1 || mm < 0 || mm >= (1ll << 31) - 1) fail(PM_ERR_BAD_GRAPH, "graph dump n / m out of range");
  const int64_t body = size - kDumpHeader;
  if (body % 4) fail(PM_ERR_BAD_GRAPH, "graph dump body is not whole int32 words");
  const int64_t nwords = body / 4;
  if (nwords >= (1ll << 31)) fail(PM_ERR_NOT_SUPPORTED, "graph dumps of 2^31 words (8 GiB) or more");
  n = nn;
  m = mm;
  PinnedBuf hb((size_t)body);
  if (body && fread(hb.p, 1, (size_t)body, file.f) != (size_t)body) fail(PM_ERR_BAD_GRAPH, "graph dump truncated");
  DevBuf words((size_t)std::max<int64_t>(body, 4)), flag((size_t)std::max<int64_t>(nwords, 1) * 4), nsel(8),
      outdeg((size_t)(n + 1) * 4), errb(4);
  PM_CUDA(cudaMemcpyAsync(words.p, hb.p, (size_t)body, cudaMemcpyHostToDevice, st));
  if (nwords) PM_LAUNCH(k_dump_marks, grid_for(nwords), 256, 0, st, words.as<int32_t>(), nwords, flag.as<int32_t>());
  // the record starts: the positions of the -1 words
  size_t tmp = 0;
  thrust::counting_iterator<int32_t> pos(0);
  DevBuf sel((size_t)std::max<int64_t>(nwords, 1) * 4);
  PM_CUDA(cub::DeviceSelect::Flagged(nullptr, tmp, pos, flag.as<int32_t>(), sel.as<int32_t>(), nsel.as<int64_t>(),
                                     (int64_t)nwords, st));
  DevBuf tb(std::max<size_t>(tmp, 16));
  PM_CUDA(cub::DeviceSelect::Flagged(tb.p, tmp, pos, flag.as<int32_t>(), sel.as<int32_t>(), nsel.as<int64_t>(),
                                     (int64_t)nwords, st));
  int64_t records = 0;
  PM_CUDA(cudaMemcpyAsync(&records, nsel.p, 8, cudaMemcpyDeviceToHost, st));
  PM_CUDA(cudaStreamSynchronize(st));
  if (records != n)
    fail(PM_ERR_BAD_GRAPH, "graph dump holds " + std::to_string(records) + " records, header says n = " +
                               std::to_string(n));
  PM_CUDA(cudaMemsetAsync(errb.p, 0, 4, st));
  PM_CUDA(cudaMemsetAsync(outdeg.as<int32_t>() + n, 0, 4, st));
  PM_LAUNCH(k_dump_records, grid_for(n), 256, 0, st, words.as<int32_t>(), nwords, sel.as<int32_t>(), n,
            outdeg.as<int32_t>(), errb.as<unsigned>());
  off.alloc((size_t)(n + 1) * 4);
  tmp = 0;
  PM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, outdeg.as<int32_t>(), off.as<int32_t>(), (int)(n + 1), st));
  DevBuf tb2(std::max<size_t>(tmp, 16));
  PM_CUDA(cub::DeviceScan::ExclusiveSum(tb2.p, tmp, outdeg.as<int32_t>(), off.as<int32_t>(), (int)(n + 1), st));
  unsigned herr = 0;
  int32_t mcount = 0;
  PM_CUDA(cudaMemcpyAsync(&herr, errb.p, 4, cudaMemcpyDeviceToHost, st));
  PM_CUDA(cudaMemcpyAsync(&mcount, off.as<int32_t>() + n, 4, cudaMemcpyDeviceToHost, st));
  PM_CUDA(cudaStreamSynchronize(st));
  if (herr) fail(PM_ERR_BAD_GRAPH, "graph dump holds a record with a wrong id, degree or length");
  if (mcount != m)
    fail(PM_ERR_BAD_GRAPH, "graph dump out-degrees sum to " + std::to_string(mcount) + ", header says m = " +
                               std::to_string(m));
  idx.alloc((size_t)std::max<int64_t>(m, 1) * 4);
  PM_LAUNCH(k_dump_copy, grid_for(n * 32), 256, 0, st, words.as<int32_t>(), sel.as<int32_t>(), off.as<int32_t>(), n,
            idx.as<int32_t>());
  PM_CUDA(cudaStreamSynchronize(st));
}

void write_graph_dump(pm_graph *g, const char *path) {
  cudaStream_t st = g->E.stream;
  const int64_t n = g->n, m = g->m;
  const GraphView &v = g->E.g;  // v.in aliases v.out on a symmetric graph
  DevBuf len((size_t)(n + 1) * 8), pos((size_t)(n + 1) * 8);
  PM_CUDA(cudaMemsetAsync(len.as<int64_t>() + n, 0, 8, st));
  PM_LAUNCH(k_dump_lengths, grid_for(n), 256, 0, st, v.out.off, v.in.off, n, len.as<int64_t>());
  size_t tmp = 0;
  PM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, len.as<int64_t>(), pos.as<int64_t>(), (int)(n + 1), st));
  DevBuf tb(std::max<size_t>(tmp, 16));
  PM_CUDA(cub::DeviceScan::ExclusiveSum(tb.p, tmp, len.as<int64_t>(), pos.as<int64_t>(), (int)(n + 1), st));
  int64_t nwords = 0;
  PM_CUDA(cudaMemcpyAsync(&nwords, pos.as<int64_t>() + n, 8, cudaMemcpyDeviceToHost, st));
  PM_CUDA(cudaStreamSynchronize(st));
  DevBuf words((size_t)std::max<int64_t>(nwords, 1) * 4);
  PM_LAUNCH(k_dump_write, grid_for(n * 32), 256, 0, st, v.out.off, v.out.idx, v.in.off, v.in.idx,
            pos.as<int64_t>(), n, words.as<int32_t>());
  PinnedBuf hb((size_t)(kDumpHeader + nwords * 4));
  unsigned char *h = (unsigned char *)hb.p;
  const int64_t total = kDumpHeader + nwords * 4;
  const int32_t nn = (int32_t)n;
  std::memcpy(h, &total, 8);
  std::memcpy(h + 8, &nn, 4);
  std::memcpy(h + 12, &m, 8);
  PM_CUDA(cudaMemcpyAsync(h + kDumpHeader, words.p, (size_t)nwords * 4, cudaMemcpyDeviceToHost, st));
  PM_CUDA(cudaStreamSynchronize(st));
  File file(path, "wb");
  if (!file.f) fail(PM_ERR_INVALID_ARG, std::string("cannot create ") + path);
  if (fwrite(h, 1, (size_t)total, file.f) != (size_t)total) fail(PM_ERR_INVALID_ARG, std::string("cannot write ") + path);
}

}  // namespace pm
