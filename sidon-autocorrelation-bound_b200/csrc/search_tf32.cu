// ---------------------------------------------------------------------------
//  search_tf32.cu -- the smoothed objective G_p and its adjoint with the
//  convolution and the correlation on the tensor cores in TF32x3
//  (tc_tf32.cuh): the TF32x3 mode of the precision sweep, beside FP32 SIMT,
//  BF16x1 and BF16x3 (sidon_lp_forward / sidon_lp_backward, precision
//  SIDON_PREC_TF32X3).  The arithmetic around the products is that of the
//  BF16 kernels k_lp_forward_tc / k_lp_backward_tc: M refined in fp64 over the
//  near-maximal k, S in fp64, the weights (b/M)^(p-1) in fp32.
// ---------------------------------------------------------------------------
#include "tc_tf32.cuh"

namespace sidon {
namespace tc {
namespace tf32 {

constexpr int kRefineCap = 1024;
static_assert(kRefineCap * sizeof(int) <= (size_t)kStages * kStageBytes, "list fits the ring");

__device__ __forceinline__ bool bad_height(float x) { return !(x >= 0.f && x <= 3.402823466e38f); }

__global__ void __launch_bounds__(NTHREADS, 1)
k_lp_forward(const float* __restrict__ pop, int n, float p, float* __restrict__ value,
             float* __restrict__ saved, float* __restrict__ b_out, unsigned int* status) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ int s_cnt;
  __shared__ double s_red[32];
  const int pid = blockIdx.x;
  Shared S = setup(n, smem_raw);
  Ctx& C = S.C;
  int* s_list = reinterpret_cast<int*>(C.stages);   // idle outside tile phases
  begin(S, n, n);
  const int nb = 2 * n - 1;
  const Lane ln;
  const float* a = pop + (size_t)pid * n;
  double sl = 0.0;
  bool bad = false;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float x = a[i];
    bad |= bad_height(x);
    S.sa[pidx(i)] = x;
    sl += x;
  }
  if (bad) atomicCAS(status, 0u, (unsigned int)SIDON_ERR_NONFINITE);
  const double Ssum = block_sum(sl, s_red);
  prime(C, false);
  const bool ok = run_tiles<CONV>(C, S.sa, nullptr, status);
  if (ok) gather_conv(C, ln, S.cb);
  float mloc = 0.f;
  if (ok)
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
      const float v = S.cb[pidx(k)];
      mloc = fmaxf(mloc, v);
      if (b_out) b_out[(size_t)pid * nb + k] = v;
    }
  const float Mapprox = block_max(mloc, S.red);
  const double Md = refine_max(
      n, [&](int i) { return S.sa[pidx(i)]; }, [&](int k) { return S.cb[pidx(k)]; }, Mapprox,
      2e-4f, s_list, kRefineCap, &s_cnt, s_red);
  const float M = (float)Md;
  float rloc = 0.f;
  if (ok)
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
      const float d = (S.cb[pidx(k)] - M) / M;
      rloc += d > -1.f ? pow_from_d_fast(d, p) : 0.f;
    }
  const float R = block_sum(rloc, S.red);
  if (threadIdx.x == 0) {
    const double val = 2.0 * (double)n * Md * pow((double)R, 1.0 / (double)p) / (Ssum * Ssum);
    const float v = ok ? (float)val : __int_as_float(0x7fc00000);
    value[pid] = v;
    saved[4 * pid + 0] = M;
    saved[4 * pid + 1] = (float)Ssum;
    saved[4 * pid + 2] = R;
    saved[4 * pid + 3] = v;
  }
  teardown(S);
}

__global__ void __launch_bounds__(NTHREADS, 1)
k_lp_backward(const float* __restrict__ pop, const float* __restrict__ saved,
              const float* __restrict__ b_in, int n, float p, float* __restrict__ grad,
              unsigned int* status) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const int pid = blockIdx.x;
  Shared S = setup(n, smem_raw);
  Ctx& C = S.C;
  begin(S, n, n);
  const int nb = 2 * n - 1;
  const Lane ln;
  const float* a = pop + (size_t)pid * n;
  const float M = saved[4 * pid + 0], Ssum = saved[4 * pid + 1], R = saved[4 * pid + 2];
  for (int i = threadIdx.x; i < n; i += blockDim.x) S.sa[pidx(i)] = a[i];
  __syncthreads();
  prime(C, true);
  bool ok = true;
  if (b_in) {
    for (int k = threadIdx.x; k < nb; k += blockDim.x) S.cb[pidx(k)] = b_in[(size_t)pid * nb + k];
    __syncthreads();
  } else {
    ok = run_tiles<CONV>(C, S.sa, nullptr, status);
    if (ok) gather_conv(C, ln, S.cb);
  }
  for (int k = threadIdx.x; k < nb; k += blockDim.x) {
    const float d = (S.cb[pidx(k)] - M) / M;
    S.cb[pidx(k)] = d > -1.f ? pow_from_d_fast(d, p - 1.f) : 0.f;
  }
  fence_before();
  __syncthreads();
  // the correlation in two passes over the tiles: B = the weights' hi plane,
  // then their lo plane, into the same accumulator
  if (ok) ok = run_tiles<CORR_HI>(C, S.sa, S.cb, status);
  if (ok) ok = run_tiles<CORR_LO>(C, S.sa, S.cb, status);
  if (ok) gather_corr(C, ln, S.cb);
  const float scale = 4.f * (float)n * powf(R, 1.f / p) / (Ssum * Ssum);
  const float MS = M / Ssum;
  float* g = grad + (size_t)pid * n;
  if (ok)
    for (int i = threadIdx.x; i < n; i += blockDim.x) g[i] = scale * (S.cb[pidx(i)] / R - MS);
  teardown(S);
}

}  // namespace tf32
}  // namespace tc
}  // namespace sidon

namespace sidon_host {
using namespace sidon;
unsigned int* tc_status_word();
int tc_n_ok_public(int n);

size_t smem_lp_tf32(int n) { return tc::tf32::Plan(n).total; }

// the TF32x3 plan fits the accumulators (as the BF16 kernels) and the
// shared-memory budget (n up to about 8700 on a B200)
static int tf32_n_ok(int n) {
  int rc = tc_n_ok_public(n);
  if (rc) return rc;
  return smem_lp_tf32(n) <= tc::kSmemBudget ? SIDON_OK : SIDON_ERR_SMEM;
}

int launch_lp_forward_tf32(const float* a, int n, int P, double p, float* value, float* saved,
                           float* b_out, cudaStream_t st) {
  int rc = tf32_n_ok(n);
  if (rc) return rc;
  const size_t sm = smem_lp_tf32(n);
  rc = set_dyn_smem((const void*)tc::tf32::k_lp_forward, sm);
  if (rc) return rc;
  unsigned int* sw = tc_status_word();
  if (!sw) return SIDON_ERR_CUDA;
  tc::tf32::k_lp_forward<<<P, tc::NTHREADS, sm, st>>>(a, n, (float)p, value, saved, b_out, sw);
  return check_launch();
}

int launch_lp_backward_tf32(const float* a, const float* saved, const float* b_in, int n, int P,
                            double p, float* grad, cudaStream_t st) {
  int rc = tf32_n_ok(n);
  if (rc) return rc;
  const size_t sm = smem_lp_tf32(n);
  rc = set_dyn_smem((const void*)tc::tf32::k_lp_backward, sm);
  if (rc) return rc;
  unsigned int* sw = tc_status_word();
  if (!sw) return SIDON_ERR_CUDA;
  tc::tf32::k_lp_backward<<<P, tc::NTHREADS, sm, st>>>(a, saved, b_in, n, (float)p, grad, sw);
  return check_launch();
}

}  // namespace sidon_host
