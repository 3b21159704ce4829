// pm_ingest.cu -- PBBS graph files into device buffers.
//
// Text: "AdjacencyGraph" or "WeightedAdjacencyGraph", then n, m, n offsets,
// m edge ids (and m int32 weights), separated by any whitespace
// (readGraphFromFile / readWghGraphFromFile, IO-numa.h:112-160 and 318-402,
// with the word splitting of stringToWords, 84-110).  The header is read on
// the host; the body is copied to the device once and tokenised there: every
// 64-byte chunk counts the token starts it holds, a scan gives each chunk its
// first token index, and a second pass parses each token where it starts.
//
// Binary: <base>.config holds n as text, <base>.adj the m edge ids (uint32),
// <base>.idx the n offsets (int32) (readGraphFromBinary, IO-numa.h:404-470),
// read on the host.
#include <cstdio>
#include <cstring>
#include <vector>

#include <cub/cub.cuh>

#include "pm_graph.cuh"

namespace pm {

namespace {

constexpr int kTokChunk = 64;  // bytes a thread scans

__device__ __forceinline__ bool is_space(unsigned char c) {
  return c == ' ' || c == '\n' || c == '\r' || c == '\t' || c == 0;
}

__global__ void k_count_tokens(const unsigned char *__restrict__ b, int64_t len, int64_t nchunks,
                               int64_t *__restrict__ cnt) {
  for (int64_t ch = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; ch < nchunks;
       ch += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i0 = ch * kTokChunk, i1 = min(i0 + kTokChunk, len);
    unsigned char prev = i0 == 0 ? ' ' : b[i0 - 1];
    int64_t c = 0;
    for (int64_t i = i0; i < i1; ++i) {
      const unsigned char x = b[i];
      c += !is_space(x) && is_space(prev);
      prev = x;
    }
    cnt[ch] = c;
  }
}

// Token t of the body goes to off[t] (t < n), idx[t - n] (t < n + m) or
// w[t - n - m].  err bit 1: a character other than a sign or a digit, bit 2:
// a value outside int32.
__global__ void k_parse_tokens(const unsigned char *__restrict__ b, int64_t len, int64_t nchunks,
                               const int64_t *__restrict__ first, int64_t n, int64_t m,
                               int32_t *__restrict__ off, int32_t *__restrict__ idx, int32_t *__restrict__ w,
                               unsigned *err) {
  for (int64_t ch = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; ch < nchunks;
       ch += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i0 = ch * kTokChunk, i1 = min(i0 + kTokChunk, len);
    unsigned char prev = i0 == 0 ? ' ' : b[i0 - 1];
    int64_t t = first[ch];
    for (int64_t i = i0; i < i1; ++i) {
      const unsigned char x = b[i];
      const bool start = !is_space(x) && is_space(prev);
      prev = x;
      if (!start) continue;
      int64_t j = i;
      bool neg = false;
      if (b[j] == '-' || b[j] == '+') {
        neg = b[j] == '-';
        ++j;
      }
      long long v = 0;
      int digits = 0;
      unsigned e = 0;
      for (; j < len && !is_space(b[j]); ++j) {
        const unsigned char c = b[j];
        if (c < '0' || c > '9') {
          e |= 1u;
          break;
        }
        v = v * 10 + (c - '0');
        if (++digits > 10 || v > 2147483648ll) {
          e |= 2u;
          break;
        }
      }
      if (digits == 0) e |= 1u;
      if (neg) v = -v;
      if (v > 2147483647ll || v < -2147483648ll) e |= 2u;
      if (e) {
        atomicOr(err, e);
      } else if (t < n) {
        off[t] = (int32_t)v;
      } else if (t < n + m) {
        idx[t - n] = (int32_t)v;
      } else if (w) {
        w[t - n - m] = (int32_t)v;
      }
      ++t;
    }
  }
}

__global__ void k_set_last(int32_t *off, int64_t n, int64_t m) { off[n] = (int32_t)m; }

struct HostFile {
  FILE *f = nullptr;
  explicit HostFile(const char *path, const char *mode) : f(fopen(path, mode)) {}
  ~HostFile() {
    if (f) fclose(f);
  }
};

struct Pinned {
  void *p = nullptr;
  explicit Pinned(size_t bytes) { PM_CUDA(cudaMallocHost(&p, bytes ? bytes : 1)); }
  ~Pinned() {
    if (p) cudaFreeHost(p);
  }
};

int64_t file_size(FILE *f) {
  if (fseek(f, 0, SEEK_END) != 0) return -1;
  const long long s = ftello(f);
  if (fseek(f, 0, SEEK_SET) != 0) return -1;
  return s;
}

bool host_space(char c) { return c == ' ' || c == '\n' || c == '\r' || c == '\t' || c == 0; }

}  // namespace

void parse_pbbs_text(pm_graph *g, const char *path, DevBuf &off, DevBuf &idx, DevBuf &w, int64_t &n,
                     int64_t &m) {
  cudaStream_t st = g->E.stream;
  HostFile hf(path, "rb");
  if (!hf.f) fail(PM_ERR_INVALID_ARG, std::string("cannot open ") + path);
  const int64_t size = file_size(hf.f);
  if (size <= 0) fail(PM_ERR_BAD_GRAPH, std::string("empty or unreadable file ") + path);
  Pinned host((size_t)size + 1);
  char *s = (char *)host.p;
  if (fread(s, 1, (size_t)size, hf.f) != (size_t)size) fail(PM_ERR_BAD_GRAPH, std::string("short read of ") + path);
  s[size] = 0;
  // header: the first three words
  int64_t pos = 0;
  std::string words[3];
  for (int k = 0; k < 3; ++k) {
    while (pos < size && host_space(s[pos])) ++pos;
    const int64_t b0 = pos;
    while (pos < size && !host_space(s[pos])) ++pos;
    words[k].assign(s + b0, (size_t)(pos - b0));
  }
  bool weighted;
  if (words[0] == "AdjacencyGraph")
    weighted = false;
  else if (words[0] == "WeightedAdjacencyGraph")
    weighted = true;
  else
    fail(PM_ERR_BAD_GRAPH, "bad PBBS header '" + words[0] + "' (AdjacencyGraph or WeightedAdjacencyGraph)");
  char *endp = nullptr;
  n = strtoll(words[1].c_str(), &endp, 10);
  if (words[1].empty() || *endp) fail(PM_ERR_BAD_GRAPH, "bad vertex count '" + words[1] + "'");
  m = strtoll(words[2].c_str(), &endp, 10);
  if (words[2].empty() || *endp) fail(PM_ERR_BAD_GRAPH, "bad edge count '" + words[2] + "'");
  if (n < 1 || n >= (1ll << 31) - 1 || m < 0 || m >= (1ll << 31) - 1)
    fail(PM_ERR_BAD_GRAPH, "vertex / edge counts outside [1, 2^31-2] / [0, 2^31-2]");
  const int64_t want = n + m * (weighted ? 2 : 1);
  // the body starts at the whitespace that ends the third word
  const int64_t len = size - pos;
  const int64_t nchunks = (len + kTokChunk - 1) / kTokChunk;
  if (nchunks >= (1ll << 31)) fail(PM_ERR_NOT_SUPPORTED, "PBBS text file too large (128 GiB or more)");
  DevBuf body((size_t)std::max<int64_t>(len, 1)), cnt((size_t)std::max<int64_t>(nchunks, 1) * 8),
      first((size_t)std::max<int64_t>(nchunks, 1) * 8), errb(4);
  int64_t total = 0;
  if (len > 0) {
    PM_CUDA(cudaMemcpyAsync(body.p, s + pos, (size_t)len, cudaMemcpyHostToDevice, st));
    const int grid = (int)std::min<int64_t>((nchunks + 255) / 256, (int64_t)g->E.num_sms * 16);
    PM_LAUNCH(k_count_tokens, grid, 256, 0, st, body.as<unsigned char>(), len, nchunks, cnt.as<int64_t>());
    size_t tmp = 0;
    PM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, cnt.as<int64_t>(), first.as<int64_t>(), (int)nchunks, st));
    DevBuf tb(std::max<size_t>(tmp, 16));
    PM_CUDA(cub::DeviceScan::ExclusiveSum(tb.p, tmp, cnt.as<int64_t>(), first.as<int64_t>(), (int)nchunks, st));
    int64_t last[2] = {0, 0};
    PM_CUDA(cudaMemcpyAsync(&last[0], first.as<int64_t>() + nchunks - 1, 8, cudaMemcpyDeviceToHost, st));
    PM_CUDA(cudaMemcpyAsync(&last[1], cnt.as<int64_t>() + nchunks - 1, 8, cudaMemcpyDeviceToHost, st));
    PM_CUDA(cudaStreamSynchronize(st));
    total = last[0] + last[1];
  }
  if (total != want)
    fail(PM_ERR_BAD_GRAPH, "PBBS file holds " + std::to_string(total) + " numbers after the header, expected " +
                               std::to_string(want) + (weighted ? " (n + 2m)" : " (n + m)"));
  off.alloc((size_t)(n + 1) * 4);
  idx.alloc((size_t)std::max<int64_t>(m, 1) * 4);
  if (weighted) w.alloc((size_t)std::max<int64_t>(m, 1) * 4);
  PM_CUDA(cudaMemsetAsync(errb.p, 0, 4, st));
  if (len > 0) {
    const int grid = (int)std::min<int64_t>((nchunks + 255) / 256, (int64_t)g->E.num_sms * 16);
    PM_LAUNCH(k_parse_tokens, grid, 256, 0, st, body.as<unsigned char>(), len, nchunks, first.as<int64_t>(), n,
              m, off.as<int32_t>(), idx.as<int32_t>(), weighted ? w.as<int32_t>() : nullptr,
              errb.as<unsigned>());
  }
  PM_LAUNCH(k_set_last, 1, 1, 0, st, off.as<int32_t>(), n, m);
  unsigned herr = 0;
  PM_CUDA(cudaMemcpyAsync(&herr, errb.p, 4, cudaMemcpyDeviceToHost, st));
  PM_CUDA(cudaStreamSynchronize(st));
  if (herr & 1u) fail(PM_ERR_BAD_GRAPH, "PBBS file holds a word that is not an integer");
  if (herr & 2u) fail(PM_ERR_BAD_GRAPH, "PBBS file holds a number outside int32");
}

void read_pbbs_binary(const char *base, std::vector<int32_t> &off, std::vector<int32_t> &idx, int64_t &n,
                      int64_t &m) {
  const std::string b(base);
  {
    HostFile cf((b + ".config").c_str(), "r");
    if (!cf.f) fail(PM_ERR_INVALID_ARG, "cannot open " + b + ".config");
    long long nn = -1;
    if (fscanf(cf.f, "%lld", &nn) != 1) fail(PM_ERR_BAD_GRAPH, "no vertex count in " + b + ".config");
    n = nn;
  }
  if (n < 1 || n >= (1ll << 31) - 1) fail(PM_ERR_BAD_GRAPH, "vertex count outside [1, 2^31-2]");
  HostFile af((b + ".adj").c_str(), "rb");
  if (!af.f) fail(PM_ERR_INVALID_ARG, "cannot open " + b + ".adj");
  const int64_t asz = file_size(af.f);
  if (asz < 0 || asz % 4) fail(PM_ERR_BAD_GRAPH, b + ".adj is not a whole number of uint32 ids");
  m = asz / 4;
  if (m >= (1ll << 31) - 1) fail(PM_ERR_BAD_GRAPH, "edge count outside [0, 2^31-2]");
  HostFile xf((b + ".idx").c_str(), "rb");
  if (!xf.f) fail(PM_ERR_INVALID_ARG, "cannot open " + b + ".idx");
  const int64_t xsz = file_size(xf.f);
  if (xsz != n * 4) fail(PM_ERR_BAD_GRAPH, b + ".idx does not hold n int32 offsets");
  idx.resize((size_t)std::max<int64_t>(m, 1));
  off.resize((size_t)n + 1);
  if (m && fread(idx.data(), 4, (size_t)m, af.f) != (size_t)m) fail(PM_ERR_BAD_GRAPH, "short read of " + b + ".adj");
  if (fread(off.data(), 4, (size_t)n, xf.f) != (size_t)n) fail(PM_ERR_BAD_GRAPH, "short read of " + b + ".idx");
  off[(size_t)n] = (int32_t)m;
}

}  // namespace pm
