// gather_probe.cu -- standalone measurement of the random 4-byte gather rate
// of the GPU (the ceiling of every pull kernel of the engine): an int32 index
// stream read once (coalesced) plus one float gather per index from a table
// of 2^24 entries, for uniform and R-MAT-skewed indices and several cache
// modifiers.  Build: python -c "from polymer_b200 import _build; _build.build_gather_probe()"
#include <cstdio>
#include <cstdint>
#include <cuda_runtime.h>
#include <vector>
#include <algorithm>

#define CK(x) do { cudaError_t e = (x); if (e != cudaSuccess) { printf("%s: %s\n", #x, cudaGetErrorString(e)); return 1; } } while (0)

__global__ void k_fill_uniform(int32_t *idx, int64_t n, int32_t range, uint64_t seed) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull; z = (z ^ (z >> 27)) * 0x94D049BB133111EBull; z ^= z >> 31;
    idx[i] = (int32_t)(z % (uint64_t)range);
  }
}
// R-MAT-like source ids: skewed (low ids hot), 24 levels, a+b=0.76 for row bit 0
__global__ void k_fill_rmat(int32_t *idx, int64_t n, int scale, uint64_t seed) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t s = 0;
    for (int l = 0; l < scale; ++l) {
      uint64_t z = seed + (i * scale + l + 1) * 0x9E3779B97F4A7C15ull;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull; z = (z ^ (z >> 27)) * 0x94D049BB133111EBull; z ^= z >> 31;
      uint32_t u = (uint32_t)(z >> 40);
      s = (s << 1) | (u >= 12750684u);
    }
    idx[i] = (int32_t)s;
  }
}

template <int MODE>
__global__ void k_gather(const int32_t *__restrict__ idx, const float *__restrict__ tab, int64_t n, float *out) {
  float acc = 0.f;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  for (; i + 3 * stride < n; i += 4 * stride) {
    int a = __ldcs(idx + i), b = __ldcs(idx + i + stride), c = __ldcs(idx + i + 2 * stride), d = __ldcs(idx + i + 3 * stride);
    if (MODE == 0) acc += __ldg(tab + a) + __ldg(tab + b) + __ldg(tab + c) + __ldg(tab + d);
    else if (MODE == 1) acc += __ldcg(tab + a) + __ldcg(tab + b) + __ldcg(tab + c) + __ldcg(tab + d);
    else if (MODE == 2) acc += (float)(a + b + c + d);
    else {
      float va, vb, vc, vd;
      asm volatile("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(va) : "l"(tab + a));
      asm volatile("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(vb) : "l"(tab + b));
      asm volatile("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(vc) : "l"(tab + c));
      asm volatile("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(vd) : "l"(tab + d));
      acc += va + vb + vc + vd;
    }
  }
  for (; i < n; i += stride) acc += MODE == 2 ? (float)idx[i] : __ldg(tab + idx[i]);
  if (acc == 1234.5f) out[0] = acc;
}

int main() {
  const int64_t ne = 263428241;
  const int scale = 24;
  const int32_t nt = 1 << scale;
  int32_t *idx; float *tab, *out;
  CK(cudaMalloc(&idx, ne * 4)); CK(cudaMalloc(&tab, (size_t)nt * 4)); CK(cudaMalloc(&out, 4));
  CK(cudaMemset(tab, 0, (size_t)nt * 4));
  int nsm; cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, 0);
  cudaEvent_t a, b; cudaEventCreate(&a); cudaEventCreate(&b);
  for (int dist = 0; dist < 3; ++dist) {
    int32_t range = dist == 2 ? (1 << 20) : nt;
    if (dist == 1) k_fill_rmat<<<nsm * 8, 256>>>(idx, ne, scale, 77);
    else k_fill_uniform<<<nsm * 8, 256>>>(idx, ne, range, 77);
    CK(cudaDeviceSynchronize());
    for (int mode = 0; mode < 4; ++mode) {
      for (int blocks_per_sm : {8, 16}) {
        int grid = nsm * blocks_per_sm;
        auto run = [&]() {
          if (mode == 0) k_gather<0><<<grid, 256>>>(idx, tab, ne, out);
          else if (mode == 1) k_gather<1><<<grid, 256>>>(idx, tab, ne, out);
          else if (mode == 2) k_gather<2><<<grid, 256>>>(idx, tab, ne, out);
          else k_gather<3><<<grid, 256>>>(idx, tab, ne, out);
        };
        run(); run();
        cudaEventRecord(a);
        for (int r = 0; r < 5; ++r) run();
        cudaEventRecord(b);
        CK(cudaEventSynchronize(b));
        float ms; cudaEventElapsedTime(&ms, a, b); ms /= 5;
        printf("dist=%s mode=%s bps=%d  %.3f ms  %.1f Ggather/s  idx-stream %.0f GB/s\n",
               dist == 0 ? "uniform16M" : dist == 1 ? "rmat24" : "uniform1M",
               mode == 0 ? "ldg" : mode == 1 ? "ldcg" : mode == 2 ? "nogather" : "no_alloc", blocks_per_sm, ms,
               ne / ms / 1e6, ne * 4.0 / ms / 1e6);
      }
    }
  }
  return 0;
}
