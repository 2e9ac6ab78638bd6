// ---------------------------------------------------------------------------
//  capi.cu -- the extern "C" boundary (include/sidon_b200.h): argument
//  checks, status codes, shared-memory sizing, the host fp64 evaluator, and
//  dispatch to the kernels.  Nothing here allocates device memory.
// ---------------------------------------------------------------------------
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace sidon_host {

// kernels (defined in the other translation units)
size_t smem_local_search(int n, int dtype);
size_t smem_eval(int n);
size_t smem_fw(int n);
size_t smem_certify(int n);
size_t smem_local_search_tc(int n);
int launch_local_search(void* pop, void* mom, void* vel, const long long* offsets,
                        const int* order, int P, int n_fixed, int n_max, const int* skip,
                        const int* mode_arr, int iters, double pS, double pE, double lrS,
                        double lrE, double b1, double b2, int mode_default, int dtype,
                        cudaStream_t st);
int launch_local_search_tc(float* pop, float* mom, float* vel, const long long* offsets,
                           const int* order, int P, int n_fixed, int n_max, const int* skip,
                           const int* mode_arr, int iters, double pS, double pE, double lrS,
                           double lrE, double b1, double b2, int mode_default, int precision,
                           unsigned int* seg_flags, cudaStream_t st);
int launch_lp_forward(const float* a, int n, int P, double p, float* value, float* saved,
                      float* b_out, cudaStream_t st);
int launch_lp_forward_tc(const float* a, int n, int P, double p, float* value, float* saved,
                         float* b_out, int precision, cudaStream_t st);
int launch_lp_backward_tc(const float* a, const float* saved, const float* b_in, int n, int P,
                          double p, float* grad, int precision, cudaStream_t st);
int device_status(int reset);
int launch_lp_forward_tf32(const float* a, int n, int P, double p, float* value, float* saved,
                           float* b_out, cudaStream_t st);
int launch_lp_backward_tf32(const float* a, const float* saved, const float* b_in, int n, int P,
                            double p, float* grad, cudaStream_t st);
int set_wait_limit(long long cycles);
int launch_lp_backward(const float* a, const float* saved, const float* b_in, int n, int P,
                       double p, float* grad, cudaStream_t st);
int launch_eval(const void* pop, int dtype, const long long* offsets, const int* order, int P,
                int n_fixed, int n_max, double* outF, int* outN, double tol, cudaStream_t st);
int launch_certify(const void* pop, int dtype, int n, int P, double* outF, double* outM,
                   double* outS, int* outK, cudaStream_t st);
int launch_frank_wolfe(float* pop, const long long* offsets, const int* order, int P, int n_fixed,
                       int n_max, const int* skip, int rounds, int pdhg, int nT, float tMax,
                       float tau, float sig, cudaStream_t st);
int launch_frank_wolfe_tc(float* pop, float* gbuf, float* gbbuf, const long long* offsets,
                          const int* order, int P, int n_fixed, int n_max, const int* skip,
                          int rounds, int pdhg, int nT, float tMax, float tau, float sig,
                          int precision, cudaStream_t st);
int launch_refine(const void* src, int n, int P, void* dst, int dtype, cudaStream_t st);
int launch_eval_stream(const void* pop, int dtype, int n, int P, double* outF, int* outN,
                       double tol, cudaStream_t st);
size_t certify_workspace_bytes(int P);
int launch_certify_large(const void* pop, int dtype, int n, int P, double* outF, double* outM,
                         double* outS, int* outK, void* ws, cudaStream_t st);
size_t big_workspace_bytes(int n, int P, int Q);
int big_default_q(int n);
int tuned_q(int n, int P, int precision);
int autotune_local_search(int n, int P, int precision, int* out_q, float* out_ms);
int autotune_ls_schedule(int n, int P, int precision, sidon_ls_schedule* out);
int ls_schedule(int n, int P, int precision, sidon_ls_schedule* out);
int tc_n_ok_public(int n);
int launch_local_search_big(float* pop, float* mom, float* vel, const int* skip,
                            const int* mode_arr, int n, int P, int iters, double pS, double pE,
                            double lrS, double lrE, double b1, double b2, int mode_default,
                            int precision, int Q, void* ws, size_t ws_bytes, cudaStream_t st);
int launch_frank_wolfe_big(float* pop, const int* skip, int n, int P, int rounds, int pdhg,
                           int nT, float tMax, float tau, float sig, int precision, int Q,
                           void* ws, size_t ws_bytes, cudaStream_t st);
int launch_coarsen(const void* src, int n2, int P, void* dst, int dtype, cudaStream_t st);
int launch_resample(const float* src, int m, int P, float* dst, int n, int normalise,
                    cudaStream_t st);
int launch_island_migrate(float* pop, int n, double* fit, int P, int NI, int k, int* order,
                          cudaStream_t st);
int launch_island_migrate_ragged(float* pop, const long long* offsets, double* fit, int P, int NI,
                                 int k, int* order, cudaStream_t st);
int launch_ragged_order(const long long* offsets, int P, int* order, cudaStream_t st);
int launch_variation(const void* pop, void* out, int dtype, int n, int n_off, const int* p1,
                     const int* p2, const int* op, const float* strength,
                     unsigned long long seed, unsigned long long gen, cudaStream_t st,
                     const unsigned long long* gen_dev = nullptr);
int launch_support_sig(const void* pop, int dtype, int n, int P, float tol,
                       unsigned long long* sig, int* nnz, cudaStream_t st);

static thread_local int g_last_cuda = 0;

int set_cuda_error(cudaError_t e) {
  g_last_cuda = (int)e;
  return SIDON_ERR_CUDA;
}
int check_launch() {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_cuda_error(e);
  return SIDON_OK;
}
int smem_optin() {
  int dev = 0, v = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 0;
  return v;
}
int sm_count() {
  int dev = 0, v = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 1;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 1;
  return v > 0 ? v : 1;
}
int set_dyn_smem(const void* fn, size_t smem) {
  struct Entry {
    int dev;
    const void* fn;
    size_t smem;     // dynamic bytes granted so far
    size_t stat;     // the kernel's static shared memory
  };
  static std::mutex mu;
  static std::vector<Entry> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_cuda_error(e);
  std::lock_guard<std::mutex> lock(mu);
  Entry* x = nullptr;
  for (Entry& y : done)
    if (y.dev == dev && y.fn == fn) x = &y;
  if (!x) {
    // the static shared memory counts against the same per-block limit
    cudaFuncAttributes attr;
    e = cudaFuncGetAttributes(&attr, fn);
    if (e != cudaSuccess) return set_cuda_error(e);
    done.push_back({dev, fn, 0, attr.sharedSizeBytes});
    x = &done.back();
  }
  if ((long long)(smem + x->stat) > (long long)smem_optin()) return SIDON_ERR_SMEM;
  if (x->smem >= smem) return SIDON_OK;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return set_cuda_error(e);
  x->smem = smem;
  return SIDON_OK;
}
int device_ok() {
  int dev = 0, major = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_cuda_error(e);
  e = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  if (e != cudaSuccess) return set_cuda_error(e);
  return major == 10 ? SIDON_OK : SIDON_ERR_DEVICE;
}

}  // namespace sidon_host

using namespace sidon_host;

namespace {
inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }
// common precondition checks; returns SIDON_OK or an error
inline int pre(int n, int P) {
  if (P < 0) return SIDON_ERR_ARG;
  if (n < 1) return SIDON_ERR_N;
  return device_ok();
}
}  // namespace

extern "C" {

const char* sidon_status_string(int status) {
  switch (status) {
    case SIDON_OK: return "ok";
    case SIDON_ERR_ARG: return "invalid argument";
    case SIDON_ERR_N: return "n outside the supported range";
    case SIDON_ERR_SMEM: return "working set exceeds the shared-memory opt-in";
    case SIDON_ERR_CUDA: return "CUDA runtime error";
    case SIDON_ERR_DTYPE: return "dtype/precision not supported by this call";
    case SIDON_ERR_NONFINITE: return "non-finite or negative heights";
    case SIDON_ERR_TIMEOUT: return "device-side wait timed out";
    case SIDON_ERR_DEVICE: return "current device is not sm_100";
    case SIDON_ERR_CAPACITY: return "P * n exceeds the fixed scratch of the allocation-free call";
    default: return "unknown status";
  }
}

int sidon_last_cuda_error(void) { return g_last_cuda; }

int sidon_device_status(int reset) {
  int rc = device_ok();
  if (rc) return rc;
  return device_status(reset);
}
int sidon_set_wait_limit(long long cycles) {
  int rc = device_ok();
  if (rc) return rc;
  return set_wait_limit(cycles);
}
int sidon_abi_version(void) { return 1; }

size_t sidon_smem_bytes(int op, int n, int dtype) {
  if (n < 1) return 0;
  switch (op) {
    case SIDON_OP_LOCAL_SEARCH: return smem_local_search(n, dtype);
    case SIDON_OP_EVAL: return (dtype == SIDON_F32 || dtype == SIDON_F64) ? smem_eval(n) : 0;
    case SIDON_OP_FRANK_WOLFE: return dtype == SIDON_F32 ? smem_fw(n) : 0;
    case SIDON_OP_LOCAL_SEARCH_TC:
      return (dtype == SIDON_F32 && tc_n_ok_public(n) == SIDON_OK) ? smem_local_search_tc(n) : 0;
    default: return 0;
  }
}

int sidon_max_n(int op, int dtype) {
  const long long cap = smem_optin();
  if (cap <= 0) return 0;
  int lo = 0, hi = 1 << 22;
  while (lo < hi) {                       // largest n with smem(n) <= cap (monotone in n)
    const int mid = lo + (hi - lo + 1) / 2;
    const size_t need = sidon_smem_bytes(op, mid, dtype);
    if (need != 0 && (long long)need <= cap) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

double sidon_hostF(const double* a, int n) {
  if (!a || n < 1) return NAN;
  std::vector<double> b(2 * (size_t)n - 1, 0.0);
  for (int i = 0; i < n; ++i) {
    if (a[i] == 0.0) continue;
    const double ai = a[i];
    for (int j = 0; j < n; ++j) {
      volatile double prod = ai * a[j];   // rounded product, then rounded sum
      b[i + j] += prod;
    }
  }
  double M = 0.0;
  for (double x : b) M = x > M ? x : M;
  double Ssum = 0.0;
  for (int i = 0; i < n; ++i) Ssum += a[i];
  return 2.0 * n * M / (Ssum * Ssum);
}

int sidon_eval(const void* pop, int dtype, int n, int P, double* out_F, int* out_nactive,
               double active_tol, void* stream) {
  int rc = pre(n, P);
  if (rc) return rc;
  if (P == 0) return SIDON_OK;
  if (!pop || !out_F) return SIDON_ERR_ARG;
  if (dtype != SIDON_F32 && dtype != SIDON_F64) return SIDON_ERR_DTYPE;
  if ((long long)smem_eval(n) > (long long)smem_optin())
    return launch_eval_stream(pop, dtype, n, P, out_F, out_nactive, active_tol, S(stream));
  return launch_eval(pop, dtype, nullptr, nullptr, P, n, n, out_F, out_nactive, active_tol,
                     S(stream));
}

int sidon_certify(const void* pop, int dtype, int n, int P, double* out_F, double* out_M,
                  double* out_S, int* out_kmax, void* stream) {
  int rc = pre(n, P);
  if (rc) return rc;
  if (P == 0) return SIDON_OK;
  if (!pop || !out_F) return SIDON_ERR_ARG;
  if (dtype != SIDON_F32 && dtype != SIDON_F64) return SIDON_ERR_DTYPE;
  return launch_certify(pop, dtype, n, P, out_F, out_M, out_S, out_kmax, S(stream));
}

int sidon_local_search(void* pop, void* mom, void* vel, const int* skip, const int* mode_arr,
                       int n, int P, int iters, double p_start, double p_end, double lr_start,
                       double lr_end, double beta1, double beta2, int mode_default, int dtype,
                       int precision, void* stream) {
  int rc = pre(n, P);
  if (rc) return rc;
  if (P == 0 || iters <= 0) return SIDON_OK;
  if (!pop || !mom || !vel) return SIDON_ERR_ARG;
  if (!(p_start > 0.0) || !(p_end > 0.0) || !(lr_start > 0.0) || !(lr_end > 0.0))
    return SIDON_ERR_ARG;
  if (dtype == SIDON_F32) {
    if (precision == SIDON_PREC_FP32_SIMT)
      return launch_local_search(pop, mom, vel, nullptr, nullptr, P, n, n, skip, mode_arr, iters,
                                 p_start, p_end, lr_start, lr_end, beta1, beta2, mode_default,
                                 dtype, S(stream));
    if (precision == SIDON_PREC_BF16X1 || precision == SIDON_PREC_BF16X3)
      return launch_local_search_tc((float*)pop, (float*)mom, (float*)vel, nullptr, nullptr, P,
                                    n, n, skip, mode_arr, iters, p_start, p_end, lr_start, lr_end,
                                    beta1, beta2, mode_default, precision, nullptr, S(stream));
    return SIDON_ERR_DTYPE;
  }
  if (dtype == SIDON_F64 && precision == SIDON_PREC_FP64_SIMT)
    return launch_local_search(pop, mom, vel, nullptr, nullptr, P, n, n, skip, mode_arr, iters,
                               p_start, p_end, lr_start, lr_end, beta1, beta2, mode_default,
                               dtype, S(stream));
  return SIDON_ERR_DTYPE;
}

size_t sidon_local_search_workspace_bytes(int n, int P, int dtype, int precision) {
  if (n < 1 || P < 1 || dtype != SIDON_F32) return 0;
  if (precision != SIDON_PREC_BF16X1 && precision != SIDON_PREC_BF16X3) return 0;
  return ((size_t)P * sizeof(unsigned int) + 255) / 256 * 256;
}

int sidon_local_search_ws(void* pop, void* mom, void* vel, const int* skip, const int* mode_arr,
                          int n, int P, int iters, double p_start, double p_end, double lr_start,
                          double lr_end, double beta1, double beta2, int mode_default, int dtype,
                          int precision, void* workspace, size_t workspace_bytes, void* stream) {
  const size_t need = sidon_local_search_workspace_bytes(n, P, dtype, precision);
  if (need == 0)
    return sidon_local_search(pop, mom, vel, skip, mode_arr, n, P, iters, p_start, p_end,
                              lr_start, lr_end, beta1, beta2, mode_default, dtype, precision,
                              stream);
  int rc = pre(n, P);
  if (rc) return rc;
  if (iters <= 0) return SIDON_OK;
  if (!pop || !mom || !vel) return SIDON_ERR_ARG;
  if (!workspace || workspace_bytes < need || (reinterpret_cast<uintptr_t>(workspace) & 3))
    return SIDON_ERR_ARG;
  if (!(p_start > 0.0) || !(p_end > 0.0) || !(lr_start > 0.0) || !(lr_end > 0.0))
    return SIDON_ERR_ARG;
  return launch_local_search_tc((float*)pop, (float*)mom, (float*)vel, nullptr, nullptr, P, n, n,
                                skip, mode_arr, iters, p_start, p_end, lr_start, lr_end, beta1,
                                beta2, mode_default, precision, (unsigned int*)workspace,
                                S(stream));
}

int sidon_lp_forward(const float* a, int n, int P, double p, float* value, float* saved,
                     float* b_out, int precision, void* stream) {
  int rc = pre(n, P);
  if (rc) return rc;
  if (P == 0) return SIDON_OK;
  if (!a || !value || !saved || !(p >= 1.0)) return SIDON_ERR_ARG;
  if (precision == SIDON_PREC_FP32_SIMT)
    return launch_lp_forward(a, n, P, p, value, saved, b_out, S(stream));
  if (precision == SIDON_PREC_BF16X1 || precision == SIDON_PREC_BF16X3)
    return launch_lp_forward_tc(a, n, P, p, value, saved, b_out, precision, S(stream));
  if (precision == SIDON_PREC_TF32X3)
    return launch_lp_forward_tf32(a, n, P, p, value, saved, b_out, S(stream));
  return SIDON_ERR_DTYPE;
}

int sidon_lp_backward(const float* a, const float* saved, const float* b_in, int n, int P,
                      double p, float* grad, int precision, void* stream) {
  int rc = pre(n, P);
  if (rc) return rc;
  if (P == 0) return SIDON_OK;
  if (!a || !saved || !grad || !(p >= 1.0)) return SIDON_ERR_ARG;
  if (precision == SIDON_PREC_FP32_SIMT)
    return launch_lp_backward(a, saved, b_in, n, P, p, grad, S(stream));
  if (precision == SIDON_PREC_BF16X1 || precision == SIDON_PREC_BF16X3)
    return launch_lp_backward_tc(a, saved, b_in, n, P, p, grad, precision, S(stream));
  if (precision == SIDON_PREC_TF32X3)
    return launch_lp_backward_tf32(a, saved, b_in, n, P, p, grad, S(stream));
  return SIDON_ERR_DTYPE;
}

int sidon_frank_wolfe(float* pop, const int* skip, int n, int P, int rounds, int pdhg_iters,
                      int nT, float t_max, float tau, float sigma, void* stream) {
  int rc = pre(n, P);
  if (rc) return rc;
  if (P == 0 || rounds <= 0) return SIDON_OK;
  if (!pop || pdhg_iters < 0 || nT < 1 || !(t_max > 0.f) || !(t_max <= 1.f)) return SIDON_ERR_ARG;
  return launch_frank_wolfe(pop, nullptr, nullptr, P, n, n, skip, rounds, pdhg_iters, nT, t_max,
                            tau, sigma, S(stream));
}

int sidon_frank_wolfe_tc(float* pop, float* g_scratch, float* gbar_scratch, const int* skip, int n,
                         int P, int rounds, int pdhg_iters, int nT, float t_max, float tau,
                         float sigma, int precision, void* stream) {
  int rc = pre(n, P);
  if (rc) return rc;
  if (P == 0 || rounds <= 0) return SIDON_OK;
  if (!pop || !g_scratch || !gbar_scratch || pdhg_iters < 0 || nT < 1 || !(t_max > 0.f) ||
      !(t_max <= 1.f))
    return SIDON_ERR_ARG;
  if (precision != SIDON_PREC_BF16X1 && precision != SIDON_PREC_BF16X3) return SIDON_ERR_DTYPE;
  return launch_frank_wolfe_tc(pop, g_scratch, gbar_scratch, nullptr, nullptr, P, n, n, skip,
                               rounds, pdhg_iters, nT, t_max, tau, sigma, precision, S(stream));
}

int sidon_refine(const void* src, int n, int P, void* dst, int dtype, void* stream) {
  int rc = pre(n, P);
  if (rc) return rc;
  if (P == 0) return SIDON_OK;
  if (!src || !dst || src == dst) return SIDON_ERR_ARG;
  if (dtype != SIDON_F32 && dtype != SIDON_F64) return SIDON_ERR_DTYPE;
  return launch_refine(src, n, P, dst, dtype, S(stream));
}

int sidon_coarsen(const void* src, int n2, int P, void* dst, int dtype, void* stream) {
  int rc = pre(n2, P);
  if (rc) return rc;
  if (n2 % 2) return SIDON_ERR_N;
  if (P == 0) return SIDON_OK;
  if (!src || !dst || src == dst) return SIDON_ERR_ARG;
  if (dtype != SIDON_F32 && dtype != SIDON_F64) return SIDON_ERR_DTYPE;
  return launch_coarsen(src, n2, P, dst, dtype, S(stream));
}

int sidon_resample(const float* src, int m, int P, float* dst, int n, int normalise,
                   void* stream) {
  int rc = pre(m, P);
  if (rc) return rc;
  if (n < 1) return SIDON_ERR_N;
  if (P == 0) return SIDON_OK;
  if (!src || !dst) return SIDON_ERR_ARG;
  const char* s0 = (const char*)src;
  const char* d0 = (const char*)dst;
  if (d0 < s0 + (size_t)P * m * sizeof(float) && s0 < d0 + (size_t)P * n * sizeof(float))
    return SIDON_ERR_ARG;                               // the rows must not overlap
  return launch_resample(src, m, P, dst, n, normalise ? 1 : 0, S(stream));
}

int sidon_island_migrate(float* pop, int n, double* fit, int P, int n_islands, int k_migrate,
                         int* order_out, void* stream) {
  int rc = pre(n, P);
  if (rc) return rc;
  if (P == 0) return SIDON_OK;
  if (!pop || !fit || !order_out || n_islands < 1 || k_migrate < 0) return SIDON_ERR_ARG;
  if (P % n_islands) return SIDON_ERR_ARG;
  const int PI = P / n_islands;
  if (PI > 1024 || 2 * k_migrate > PI) return SIDON_ERR_ARG;
  return launch_island_migrate(pop, n, fit, P, n_islands, k_migrate, order_out, S(stream));
}

size_t sidon_large_workspace_bytes(int n, int P, int q, int precision) {
  if (q <= 0) q = tuned_q(n, P, precision);
  if (q <= 0) q = big_default_q(n);
  return big_workspace_bytes(n, P, q);
}

int sidon_autotune_large(int n, int P, int precision, int* out_q, float* out_ms_per_step) {
  int rc = pre(n, P);
  if (rc) return rc;
  if (P < 1) return SIDON_ERR_ARG;
  if (precision != SIDON_PREC_BF16X1 && precision != SIDON_PREC_BF16X3) return SIDON_ERR_DTYPE;
  return autotune_local_search(n, P, precision, out_q, out_ms_per_step);
}

int sidon_autotune_local_search(int n, int P, int precision, sidon_ls_schedule* out) {
  int rc = pre(n, P);
  if (rc) return rc;
  if (P < 1 || !out) return SIDON_ERR_ARG;
  if (precision == SIDON_PREC_FP32_SIMT) {
    if ((long long)smem_local_search(n, SIDON_F32) > smem_optin()) return SIDON_ERR_SMEM;
  } else if (precision == SIDON_PREC_BF16X1 || precision == SIDON_PREC_BF16X3) {
    if (tc_n_ok_public(n)) return SIDON_ERR_N;
  } else {
    return SIDON_ERR_DTYPE;
  }
  return autotune_ls_schedule(n, P, precision, out);
}

int sidon_local_search_schedule(int n, int P, int precision, sidon_ls_schedule* out) {
  int rc = pre(n, P);
  if (rc) return rc;
  if (P < 1 || !out) return SIDON_ERR_ARG;
  if (precision != SIDON_PREC_FP32_SIMT && precision != SIDON_PREC_BF16X1 &&
      precision != SIDON_PREC_BF16X3)
    return SIDON_ERR_DTYPE;
  return ls_schedule(n, P, precision, out);
}

int sidon_local_search_large(float* pop, float* mom, float* vel, const int* skip,
                             const int* mode_arr, int n, int P, int iters, double p_start,
                             double p_end, double lr_start, double lr_end, double beta1,
                             double beta2, int mode_default, int precision, int q,
                             void* workspace, size_t workspace_bytes, void* stream) {
  int rc = pre(n, P);
  if (rc) return rc;
  if (P == 0 || iters <= 0) return SIDON_OK;
  if (!pop || !mom || !vel) return SIDON_ERR_ARG;
  if (!(p_start > 0.0) || !(p_end > 0.0) || !(lr_start > 0.0) || !(lr_end > 0.0))
    return SIDON_ERR_ARG;
  if (precision != SIDON_PREC_BF16X1 && precision != SIDON_PREC_BF16X3) return SIDON_ERR_DTYPE;
  return launch_local_search_big(pop, mom, vel, skip, mode_arr, n, P, iters, p_start, p_end,
                                 lr_start, lr_end, beta1, beta2, mode_default, precision, q,
                                 workspace, workspace_bytes, S(stream));
}

int sidon_frank_wolfe_large(float* pop, const int* skip, int n, int P, int rounds, int pdhg_iters,
                            int nT, float t_max, float tau, float sigma, int precision, int q,
                            void* workspace, size_t workspace_bytes, void* stream) {
  int rc = pre(n, P);
  if (rc) return rc;
  if (P == 0 || rounds <= 0) return SIDON_OK;
  if (!pop || pdhg_iters < 0 || nT < 1 || !(t_max > 0.f) || !(t_max <= 1.f)) return SIDON_ERR_ARG;
  if (precision != SIDON_PREC_BF16X1 && precision != SIDON_PREC_BF16X3) return SIDON_ERR_DTYPE;
  return launch_frank_wolfe_big(pop, skip, n, P, rounds, pdhg_iters, nT, t_max, tau, sigma,
                                precision, q, workspace, workspace_bytes, S(stream));
}

size_t sidon_certify_workspace_bytes(int P) { return P < 0 ? 0 : certify_workspace_bytes(P); }

int sidon_certify_large(const void* pop, int dtype, int n, int P, double* out_F, double* out_M,
                        double* out_S, int* out_kmax, void* workspace, void* stream) {
  int rc = pre(n, P);
  if (rc) return rc;
  if (P == 0) return SIDON_OK;
  if (!pop || !out_F || !workspace) return SIDON_ERR_ARG;
  if (dtype != SIDON_F32 && dtype != SIDON_F64) return SIDON_ERR_DTYPE;
  return launch_certify_large(pop, dtype, n, P, out_F, out_M, out_S, out_kmax, workspace,
                              S(stream));
}

int sidon_variation(const void* pop, void* out, int dtype, int n, int n_off, const int* p1,
                    const int* p2, const int* op, const float* strength, unsigned long long seed,
                    unsigned long long gen, void* stream) {
  int rc = pre(n, n_off);
  if (rc) return rc;
  if (n_off == 0) return SIDON_OK;
  if (!pop || !out || !p1 || !p2 || !op || !strength || pop == out) return SIDON_ERR_ARG;
  if (dtype != SIDON_F32 && dtype != SIDON_F64) return SIDON_ERR_DTYPE;
  return launch_variation(pop, out, dtype, n, n_off, p1, p2, op, strength, seed, gen, S(stream));
}

int sidon_support_sig(const void* pop, int dtype, int n, int P, float tol,
                      unsigned long long* sig, int* nnz, void* stream) {
  int rc = pre(n, P);
  if (rc) return rc;
  if (P == 0) return SIDON_OK;
  if (!pop || !sig || !nnz) return SIDON_ERR_ARG;
  if (dtype != SIDON_F32 && dtype != SIDON_F64) return SIDON_ERR_DTYPE;
  return launch_support_sig(pop, dtype, n, P, tol, sig, nnz, S(stream));
}

int sidon_ragged_order(const long long* offsets, int P, int* order_out, void* stream) {
  int rc = pre(1, P);
  if (rc) return rc;
  if (P == 0) return SIDON_OK;
  if (!offsets || !order_out) return SIDON_ERR_ARG;
  return launch_ragged_order(offsets, P, order_out, S(stream));
}

int sidon_local_search_ragged(float* pop, float* mom, float* vel, const long long* offsets,
                              const int* order, int n_max, const int* skip, const int* mode_arr,
                              int P, int iters, double p_start, double p_end, double lr_start,
                              double lr_end, double beta1, double beta2, int mode_default,
                              int precision, void* stream) {
  int rc = pre(n_max, P);
  if (rc) return rc;
  if (P == 0 || iters <= 0) return SIDON_OK;
  if (!pop || !mom || !vel || !offsets) return SIDON_ERR_ARG;
  if (!(p_start > 0.0) || !(p_end > 0.0) || !(lr_start > 0.0) || !(lr_end > 0.0))
    return SIDON_ERR_ARG;
  if (precision == SIDON_PREC_FP32_SIMT)
    return launch_local_search(pop, mom, vel, offsets, order, P, 0, n_max, skip, mode_arr, iters,
                               p_start, p_end, lr_start, lr_end, beta1, beta2, mode_default,
                               SIDON_F32, S(stream));
  if (precision == SIDON_PREC_BF16X1 || precision == SIDON_PREC_BF16X3)
    return launch_local_search_tc(pop, mom, vel, offsets, order, P, 0, n_max, skip, mode_arr,
                                  iters, p_start, p_end, lr_start, lr_end, beta1, beta2,
                                  mode_default, precision, nullptr, S(stream));
  return SIDON_ERR_DTYPE;
}

int sidon_eval_ragged(const void* pop, int dtype, const long long* offsets, const int* order,
                      int n_max, int P, double* out_F, int* out_nactive, double active_tol,
                      void* stream) {
  int rc = pre(n_max, P);
  if (rc) return rc;
  if (P == 0) return SIDON_OK;
  if (!pop || !offsets || !out_F) return SIDON_ERR_ARG;
  if (dtype != SIDON_F32 && dtype != SIDON_F64) return SIDON_ERR_DTYPE;
  return launch_eval(pop, dtype, offsets, order, P, 0, n_max, out_F, out_nactive, active_tol,
                     S(stream));
}

int sidon_frank_wolfe_ragged(float* pop, const long long* offsets, const int* order, int n_max,
                             const int* skip, int P, int rounds, int pdhg_iters, int nT,
                             float t_max, float tau, float sigma, void* stream) {
  int rc = pre(n_max, P);
  if (rc) return rc;
  if (P == 0 || rounds <= 0) return SIDON_OK;
  if (!pop || !offsets || pdhg_iters < 0 || nT < 1 || !(t_max > 0.f) || !(t_max <= 1.f))
    return SIDON_ERR_ARG;
  return launch_frank_wolfe(pop, offsets, order, P, 0, n_max, skip, rounds, pdhg_iters, nT, t_max,
                            tau, sigma, S(stream));
}

int sidon_frank_wolfe_tc_ragged(float* pop, float* g_scratch, float* gbar_scratch,
                                const long long* offsets, const int* order, int n_max,
                                const int* skip, int P, int rounds, int pdhg_iters, int nT,
                                float t_max, float tau, float sigma, int precision, void* stream) {
  int rc = pre(n_max, P);
  if (rc) return rc;
  if (P == 0 || rounds <= 0) return SIDON_OK;
  if (!pop || !g_scratch || !gbar_scratch || !offsets || pdhg_iters < 0 || nT < 1 ||
      !(t_max > 0.f) || !(t_max <= 1.f))
    return SIDON_ERR_ARG;
  if (precision != SIDON_PREC_BF16X1 && precision != SIDON_PREC_BF16X3) return SIDON_ERR_DTYPE;
  return launch_frank_wolfe_tc(pop, g_scratch, gbar_scratch, offsets, order, P, 0, n_max, skip,
                               rounds, pdhg_iters, nT, t_max, tau, sigma, precision, S(stream));
}

int sidon_island_migrate_ragged(float* pop, const long long* offsets, double* fit, int P,
                                int n_islands, int k_migrate, int* order_out, void* stream) {
  int rc = pre(1, P);
  if (rc) return rc;
  if (P == 0) return SIDON_OK;
  if (!pop || !offsets || !fit || !order_out || n_islands < 1 || k_migrate < 0)
    return SIDON_ERR_ARG;
  if (P % n_islands) return SIDON_ERR_ARG;
  const int PI = P / n_islands;
  if (PI > 1024 || 2 * k_migrate > PI) return SIDON_ERR_ARG;
  return launch_island_migrate_ragged(pop, offsets, fit, P, n_islands, k_migrate, order_out,
                                      S(stream));
}

}  // extern "C"
