// Device helpers shared by the libb2b kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "b2b_internal.h"

namespace b2b {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ float dexp(float x) { return expf(x); }
__device__ __forceinline__ double dexp(double x) { return exp(x); }
__device__ __forceinline__ float dfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ float dexpm1(float x) { return expm1f(x); }
__device__ __forceinline__ double dexpm1(double x) { return expm1(x); }

// z / (exp(z) - 1), i.e. 1/exprel(z) with Brian2's exprel (brian2cuda/cuda_generator.py:858-867):
// the removable singularity at z = 0 evaluates to its limit 1 instead of 0/0.  Rate
// functions of the form c*x/(exp(x/a) - 1) are evaluated as c*a*z_over_expm1(x/a).
template <typename R>
__device__ __forceinline__ R z_over_expm1(R z) {
  return fabs(z) < (R)1e-16 ? (R)1 : z / dexpm1(z);
}
__device__ __forceinline__ double dfma(double a, double b, double c) { return fma(a, b, c); }

// Brian2's clip(value, a_min, a_max) (brian2cuda/cuda_generator.py:902-914).
template <typename R>
__device__ __forceinline__ R dclip(R v, R lo, R hi) {
  if (v < lo) return lo;
  if (v > hi) return hi;
  return v;
}

__device__ __forceinline__ void set_status(int32_t* status, int32_t code) {
  if (status) atomicCAS(status, 0, code);
}

// Block-wide exclusive scan of one int per thread.  Returns the thread's exclusive prefix;
// *total receives the block total.  `s_warp` needs blockDim.x/32 + 1 ints.
__device__ __forceinline__ int block_exclusive_scan(int c, int* s_warp, int* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = (blockDim.x + 31) >> 5;
  int x = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = lane < nwarps ? s_warp[lane] : 0;
    int wx = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(kFull, wx, o);
      if (lane >= o) wx += y;
    }
    if (lane < nwarps) s_warp[lane] = wx - w;   // exclusive warp offsets
    if (lane == nwarps - 1) s_warp[32] = wx;     // block total
  }
  __syncthreads();
  *total = s_warp[32];
  return s_warp[warp] + x - c;
}

// Floor modulo of a (possibly negative) step by the ring length.
__device__ __forceinline__ int ring_slot(int64_t step, int ring_len) {
  int64_t r = step % ring_len;
  return (int)(r < 0 ? r + ring_len : r);
}

}  // namespace b2b
