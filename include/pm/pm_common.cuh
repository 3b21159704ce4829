// pm_common.cuh -- error plumbing and warp/block helpers shared by every
// kernel of the engine.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

#include "polymer_b200.h"

// C++ symbols the engine templates call from code compiled outside the
// library (an application's own functors, include/polymer_b200_engine.cuh)
// are exported; everything else stays hidden.
#if defined(__GNUC__)
#define PM_CXX_API __attribute__((visibility("default")))
#else
#define PM_CXX_API
#endif

namespace pm {

// Internal failures travel as exceptions and become a pm_status at the C ABI.
struct PM_CXX_API Failure : std::runtime_error {
  pm_status status;
  Failure(pm_status s, const std::string &msg) : std::runtime_error(msg), status(s) {}
};

[[noreturn]] PM_CXX_API void fail(pm_status s, const std::string &msg);
PM_CXX_API void set_last_error(const std::string &msg);  // text returned by pm_last_error()
[[noreturn]] PM_CXX_API void fail_cuda(cudaError_t e, const char *what, const char *file, int line);
PM_CXX_API void count_launch(int n = 1);
PM_CXX_API long long launches(bool reset);

#define PM_CUDA(call)                                                        \
  do {                                                                       \
    cudaError_t pm_e_ = (call);                                              \
    if (pm_e_ != cudaSuccess) ::pm::fail_cuda(pm_e_, #call, __FILE__, __LINE__); \
  } while (0)

// Every kernel launch goes through this macro: it counts the launch and
// checks the launch status.
#define PM_LAUNCH(kernel, grid, block, smem, stream, ...)                    \
  do {                                                                       \
    kernel<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__);              \
    ::pm::count_launch();                                                    \
    PM_CUDA(cudaGetLastError());                                             \
  } while (0)

constexpr int kWarp = 32;
constexpr int kDevBFInf = 1073741823;  // INT_MAX / 2

// SplitMix64 output function on seed + (c + 1) * golden increment; the same
// counter-based generator as the CPU oracle.
__host__ __device__ __forceinline__ uint64_t hash64(uint64_t seed, uint64_t c) {
  uint64_t z = seed + (c + 1ull) * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

// Shuffles for any 4- or 8-byte trivially copyable type.
template <class T>
__device__ __forceinline__ T shfl_idx(T v, int src) {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "shuffle of 4/8-byte types only");
  if constexpr (sizeof(T) == 4) {
    int x = __shfl_sync(0xffffffffu, *reinterpret_cast<int *>(&v), src);
    return *reinterpret_cast<T *>(&x);
  } else {
    long long x = __shfl_sync(0xffffffffu, *reinterpret_cast<long long *>(&v), src);
    return *reinterpret_cast<T *>(&x);
  }
}
template <class T>
__device__ __forceinline__ T shfl_down(T v, int d) {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "shuffle of 4/8-byte types only");
  if constexpr (sizeof(T) == 4) {
    int x = __shfl_down_sync(0xffffffffu, *reinterpret_cast<int *>(&v), d);
    return *reinterpret_cast<T *>(&x);
  } else {
    long long x = __shfl_down_sync(0xffffffffu, *reinterpret_cast<long long *>(&v), d);
    return *reinterpret_cast<T *>(&x);
  }
}

template <class T>
__device__ __forceinline__ T shfl_up(T v, int d) {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "shuffle of 4/8-byte types only");
  if constexpr (sizeof(T) == 4) {
    int x = __shfl_up_sync(0xffffffffu, *reinterpret_cast<int *>(&v), d);
    return *reinterpret_cast<T *>(&x);
  } else {
    long long x = __shfl_up_sync(0xffffffffu, *reinterpret_cast<long long *>(&v), d);
    return *reinterpret_cast<T *>(&x);
  }
}

// Exclusive warp prefix sum of an int; total returned in *total.
__device__ __forceinline__ int warp_excl_scan(int v, int *total) {
  int lane = lane_id();
  int x = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= d) x += t;
  }
  *total = __shfl_sync(0xffffffffu, x, 31);
  return x - v;
}

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v += shfl_down(v, d);
  return v;
}

// Per-call device counters: size and out-degree sum of the next frontier,
// plus an error word (set by bounded waits and range checks, never trapped).
struct Counters {
  unsigned long long size;
  unsigned long long edges;
  unsigned long long aux;  // algorithm-specific (e.g. edges inspected)
  double daux;             // FP64 reductions (residuals, norms)
  double daux2;            // a second one (the norm of a relative residual)
  unsigned int err;
  unsigned int pad;
};

// Round state of a traversal whose rounds run on the GPU without the host
// (a CUDA graph with a WHILE node): the frontier's size and out-degree sum,
// whether this round runs at all (active), its direction and level.  The
// frontier kernels given a gate return at once unless it is their round.
struct RoundGate {
  unsigned long long size, edges;  // the current frontier
  int32_t active, dense, qsize, level;
};

enum DeviceError : unsigned int { kErrNone = 0, kErrQueueOverflow = 1, kErrRange = 2, kErrTimeout = 4 };

}  // namespace pm
