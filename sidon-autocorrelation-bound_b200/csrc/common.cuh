// ---------------------------------------------------------------------------
//  common.cuh -- shared device helpers for the sidon_b200 kernels (sm_100a).
//
//  Layout conventions used by every kernel:
//    * one CTA per candidate (blockIdx.x = candidate index), the candidate's
//      heights resident in dynamic shared memory for the whole launch;
//    * convolution/correlation operands are stored with zero margins so that
//      warp-uniform loops never test bounds (a zero term adds exactly +0 to a
//      non-negative sum, so margins never change a result bit);
//    * every reduction is deterministic (fixed tree, fixed order).
// ---------------------------------------------------------------------------
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/sidon_b200.h"

namespace sidon {

constexpr int kWarp = 32;

// ------------------------------ reductions --------------------------------
template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const T o = __shfl_xor_sync(0xffffffffu, v, off);
    v = o > v ? o : v;
  }
  return v;
}
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}
// Block-wide max / sum with the result broadcast to every thread.  scratch
// holds >= 32 slots.  Deterministic: the warp partials are combined in warp
// order by every thread.  Ends synchronised (scratch reusable afterwards).
template <typename T>
__device__ __forceinline__ T block_max(T v, T* scratch) {
  v = warp_max(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) scratch[wid] = v;
  __syncthreads();
  const int nw = blockDim.x >> 5;
  T r = scratch[0];
  for (int i = 1; i < nw; ++i) r = scratch[i] > r ? scratch[i] : r;
  __syncthreads();
  return r;
}
template <typename T>
__device__ __forceinline__ T block_sum(T v, T* scratch) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) scratch[wid] = v;
  __syncthreads();
  const int nw = blockDim.x >> 5;
  T r = T(0);
  for (int i = 0; i < nw; ++i) r += scratch[i];
  __syncthreads();
  return r;
}

// -------------------------- precise transcendentals -----------------------
// (b/M)^q evaluated as exp(q * log1p(d)), d = (b - M)/M in [-1, 0]: the
// difference b - M is exact for nearby values, so the weights of
// near-maximal b_k keep their digits at large q (the reference's reasoning,
// src/kernels.cuh:36-44).  The accurate libdevice exp/log1p are used.
__device__ __forceinline__ float pow_from_d(float d, float q) { return expf(q * log1pf(d)); }
__device__ __forceinline__ double pow_from_d(double d, double q) { return exp(q * log1p(d)); }
__device__ __forceinline__ float dev_exp(float x) { return expf(x); }
__device__ __forceinline__ double dev_exp(double x) { return exp(x); }
__device__ __forceinline__ float dev_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double dev_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float dev_fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double dev_fma(double a, double b, double c) { return __fma_rn(a, b, c); }

// round-up helper
__host__ __device__ constexpr inline int round_up(int x, int m) { return (x + m - 1) / m * m; }

}  // namespace sidon

// host-side helpers shared by the entry points (capi.cu)
namespace sidon_host {
int set_cuda_error(cudaError_t e);                   // records e, returns SIDON_ERR_CUDA
int check_launch();                                  // cudaGetLastError -> status
int smem_optin();                                    // per-CTA opt-in of the current device
int sm_count();                                      // SMs of the current device
int device_ok();                                     // SIDON_OK if current device is sm_100
}  // namespace sidon_host
