// Internal helpers shared by the gd_poisson translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdio>
#include <string>

#include "../../include/gd_poisson.h"

namespace gd {

void set_error(const char *fmt, ...);

#define GD_CHECK_CUDA(expr)                                                         \
  do {                                                                              \
    cudaError_t _e = (expr);                                                        \
    if (_e != cudaSuccess) {                                                        \
      ::gd::set_error("%s:%d %s: %s", __FILE__, __LINE__, #expr, cudaGetErrorString(_e)); \
      return GD_ERR_CUDA;                                                           \
    }                                                                               \
  } while (0)

#define GD_CHECK_LAUNCH() GD_CHECK_CUDA(cudaGetLastError())

#define GD_REQUIRE(cond, code, ...)   \
  do {                                \
    if (!(cond)) {                    \
      ::gd::set_error(__VA_ARGS__);   \
      return (code);                  \
    }                                 \
  } while (0)

inline int ceil_div(int a, int b) { return (a + b - 1) / b; }
inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Block-wide sum of one double per thread; result valid in thread 0.  Fixed
// shuffle tree, so the result is deterministic for a fixed block size.
template <int NT>
__device__ __forceinline__ double block_sum(double v) {
  static_assert(NT % 32 == 0 && NT <= 1024, "block size");
  __shared__ double warp_part[NT / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) warp_part[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = (lane < NT / 32) ? warp_part[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace gd
