// ---------------------------------------------------------------------------
//  polish.cu -- the fp64 polish of the elite (src/main.cu:798-874) as one
//  stream-ordered sequence: `passes` fp64 local-search passes over K
//  candidates with a rising exponent and a shrinking step, each followed by
//  the certifying fp64 evaluation and a device-side "keep the best so far"
//  (the reference copies the best vector to the host after every pass).
// ---------------------------------------------------------------------------
#include <cmath>

#include "common.cuh"

namespace sidon {

// One CTA: the lowest-F candidate (NaN never wins, ties to the lower index);
// if it beats *best_F its heights replace best_a.
__global__ void k_keep_best(const double* __restrict__ pop, const double* __restrict__ fit,
                            int n, int K, double* __restrict__ best_a,
                            double* __restrict__ best_F) {
  __shared__ int s_bk;
  __shared__ int s_take;
  if (threadIdx.x == 0) {
    int bk = -1;
    for (int k = 0; k < K; ++k) {
      const double f = fit[k];
      if (f == f && (bk < 0 || f < fit[bk])) bk = k;
    }
    s_bk = bk;
    s_take = (bk >= 0 && fit[bk] < *best_F) ? 1 : 0;
    if (s_take) *best_F = fit[bk];
  }
  __syncthreads();
  if (!s_take) return;
  const double* src = pop + (size_t)s_bk * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) best_a[i] = src[i];
}

}  // namespace sidon

namespace sidon_host {
int launch_local_search(void* pop, void* mom, void* vel, const long long* offsets,
                        const int* order, int P, int n_fixed, int n_max, const int* skip,
                        const int* mode_arr, int iters, double pS, double pE, double lrS,
                        double lrE, double b1, double b2, int mode_default, int dtype,
                        cudaStream_t st);
int launch_eval(const void* pop, int dtype, const long long* offsets, const int* order, int P,
                int n_fixed, int n_max, double* outF, int* outN, double tol, cudaStream_t st);
}  // namespace sidon_host

using namespace sidon_host;

extern "C" int sidon_polish(double* pop, double* mom, double* vel, int n, int K, int iters,
                            int passes, double* fit, int* nactive, double* best_a,
                            double* best_F, void* stream) {
  if (K < 0 || iters < 0 || passes < 1) return SIDON_ERR_ARG;
  if (n < 1) return SIDON_ERR_N;
  int rc = device_ok();
  if (rc) return rc;
  if (K == 0) return SIDON_OK;
  if (!pop || !mom || !vel || !fit || !best_a || !best_F) return SIDON_ERR_ARG;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  for (int q = 0; q < passes; ++q) {
    const double pA = 200.0 * std::pow(4.0, q);
    const double pB = pA * 30.0;
    const double lA = 0.010 * std::pow(0.45, q);
    const double lB = lA * 0.02;
    rc = launch_local_search(pop, mom, vel, nullptr, nullptr, K, n, n, nullptr, nullptr,
                             iters / passes, pA, pB, lA, lB, 0.9, 0.999, 0, SIDON_F64, st);
    if (rc) return rc;
    rc = launch_eval(pop, SIDON_F64, nullptr, nullptr, K, n, n, fit, nactive, 1e-6, st);
    if (rc) return rc;
    sidon::k_keep_best<<<1, 256, 0, st>>>(pop, fit, n, K, best_a, best_F);
    rc = check_launch();
    if (rc) return rc;
  }
  return SIDON_OK;
}
