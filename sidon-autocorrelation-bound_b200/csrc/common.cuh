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
#include <stddef.h>
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
// log1p(d) for d in (-1, 0] (and small positive d) with the digits of d
// kept near 0: the Taylor series to d^8 for d >= -1/16 (fp32 Horner: 6.2e-8
// relative at most, checked against fp64 log1p), __logf(1 + d) below
// (absolute error about 4e-7).  Both are evaluated and one is selected:
// without a branch the weights of a chunk interleave (measured at n = 8400:
// weights phase 12.8k -> 10.6k cycles against libdevice log1pf).
__device__ __forceinline__ float log1p_nonpos(float d) {
  float t = fmaf(d, -1.f / 8.f, 1.f / 7.f);
  t = fmaf(d, t, -1.f / 6.f);
  t = fmaf(d, t, 1.f / 5.f);
  t = fmaf(d, t, -1.f / 4.f);
  t = fmaf(d, t, 1.f / 3.f);
  t = fmaf(d, t, -1.f / 2.f);
  const float series = fmaf(d * d, t, d);
  const float lg = __logf(1.f + d);
  return d >= -0.0625f ? series : lg;
}
// 2^x by the hardware approximation (ex2.approx, the operation __expf is
// built on), results below 2^-126 flushed to 0
__device__ __forceinline__ float ex2_ftz(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
// Search-time weights of the tensor-core kernels: (1 + d)^q = 2^(q log2(e)
// log1p(d)), the reference's form __expf(q * log1pf(d)) (src/kernels.cuh:43)
// with log1p_nonpos for log1pf and the exponent scaled once.  Powers below
// 2^-126 come out as 0 (weights that small add nothing the fp32 sums keep).
// Measured at n = 8400: weights phase 10.7k -> 8.3k cycles against
// __expf with an explicit zero for q d < -110.
__device__ __forceinline__ float pow_from_d_fast(float d, float q) {
  return ex2_ftz((q * 1.44269504088896341f) * log1p_nonpos(d));
}
__device__ __forceinline__ float dev_exp(float x) { return expf(x); }
__device__ __forceinline__ double dev_exp(double x) { return exp(x); }
__device__ __forceinline__ float dev_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double dev_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float dev_fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double dev_fma(double a, double b, double c) { return __fma_rn(a, b, c); }

// Refined maximum of b = a * a for the reported objective: every k whose
// approximate b_k (from a fp32 or tensor-core convolution) lies within
// `rel` of the approximate maximum is recomputed with fp64 accumulation of
// the exact fp32 products; the largest recomputed value is returned to all
// threads.  aval(i) reads height i (0 <= i < n); bval(k) the approximate b_k.
// list: >= cap ints of shared scratch; cnt: one shared int; red: >= 32
// doubles.  If more than cap candidates qualify, the approximate maximum is
// kept for the rest (they are scanned in order, the first cap recomputed).
template <typename AFn, typename BFn>
__device__ double refine_max(int n, AFn&& aval, BFn&& bval, float approx, float rel, int* list,
                             int cap, int* cnt, double* red) {
  const int nb = 2 * n - 1;
  const float thr = approx * (1.f - rel);
  if (threadIdx.x == 0) *cnt = 0;
  __syncthreads();
  for (int k = threadIdx.x; k < nb; k += blockDim.x)
    if (bval(k) >= thr) {
      const int s = atomicAdd(cnt, 1);
      if (s < cap) list[s] = k;
    }
  __syncthreads();
  const int total = *cnt, c = total < cap ? total : cap;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, NW = blockDim.x >> 5;
  double best = total > cap ? (double)approx : 0.0;
  for (int q = wid; q < c; q += NW) {
    const int k = list[q];
    const int lo = k - (n - 1) > 0 ? k - (n - 1) : 0, hi = k < n - 1 ? k : n - 1;
    double acc = 0.0;
    for (int i = lo + lane; i <= hi; i += 32) acc = __fma_rn((double)aval(i), (double)aval(k - i), acc);
    acc = warp_sum(acc);
    best = acc > best ? acc : best;
  }
  return block_max(best, red);
}

// A candidate of a uniform batch (offsets == NULL: row pid of n_fixed
// cells) or of a ragged batch (pop[offsets[pid] .. offsets[pid + 1])).
// order (NULL = identity) maps a launch slot to the candidate it runs.
struct Cand {
  int pid;
  long long off;
  int n;
};
__device__ __forceinline__ Cand cand_of(int slot, const long long* __restrict__ offsets,
                                        const int* __restrict__ order, int n_fixed) {
  Cand c;
  c.pid = order ? order[slot] : slot;
  c.off = offsets ? offsets[c.pid] : (long long)c.pid * n_fixed;
  c.n = offsets ? (int)(offsets[c.pid + 1] - c.off) : n_fixed;
  return c;
}

// round-up helper
__host__ __device__ constexpr inline int round_up(int x, int m) { return (x + m - 1) / m * m; }

// The library's device-side state word (one per device): the first error a
// kernel recorded (SIDON_ERR_TIMEOUT, SIDON_ERR_NONFINITE) and the clock-cycle
// limit of every bounded wait.  Kernels receive the address of `status`; the
// limit sits behind it in the same struct.
constexpr long long kDefaultWaitCycles = 1ll << 31;   // ~1.1 s at 1.965 GHz
struct DeviceState {
  unsigned int status;
  unsigned int reserved;
  long long wait_cycles;
};
static_assert(offsetof(DeviceState, status) == 0, "kernels address the state by its status word");
__device__ __forceinline__ long long wait_limit(const unsigned int* status) {
  return reinterpret_cast<const DeviceState*>(status)->wait_cycles;
}

}  // namespace sidon

// host-side helpers shared by the entry points (capi.cu)
namespace sidon_host {
int set_cuda_error(cudaError_t e);                   // records e, returns SIDON_ERR_CUDA
int check_launch();                                  // cudaGetLastError -> status
int smem_optin();                                    // per-CTA opt-in of the current device
int sm_count();                                      // SMs of the current device
int device_ok();                                     // SIDON_OK if current device is sm_100
// Dynamic shared memory opt-in of kernel fn for at least smem bytes on the
// current device; SIDON_ERR_SMEM beyond the device limit.  The attribute is
// set once per (device, kernel, size class) and remembered, so launches
// inside a stream capture issue no attribute call once the same launch has
// run eagerly.
int set_dyn_smem(const void* fn, size_t smem);
}  // namespace sidon_host

// a captured CUDA graph and its executable (sidon_anneal_capture,
// sidon_generation_capture; replayed by sidon_graph_launch)
struct sidon_graph_s {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};
