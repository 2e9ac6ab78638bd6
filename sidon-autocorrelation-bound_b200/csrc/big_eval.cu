// ---------------------------------------------------------------------------
//  big_eval.cu -- the certifying fp64 evaluation for candidates whose heights
//  do not fit one CTA's shared memory (src/kernels.cuh:301-377 and hostF,
//  src/main.cu:95-105, at any n).
//
//  Each CTA owns W = 8 warps x 32 lanes x 7 consecutive k of one candidate
//  and streams the heights through shared memory in chunks of CI cells of i:
//  per chunk the x cells a[i0, i0 + CI) and the reversed operand window
//  a[k0 - i0 - CI + 1, k0 + W - i0) (zero outside [0, n)).  Every lane keeps
//  its 7 sums in registers across the chunks and adds the rounded products
//  fl(a_i a_(k-i)) in increasing i -- hostF's order -- so b_k, and F, match
//  hostF bit for bit.
//
//  Passes (all deterministic):
//    kMax     M = max(0, max_k b_k): atomicMax on the bits of a non-negative
//             double (order-free)
//    kCount   #{k : b_k >= M (1 - tol)} (integer atomics)
//    kList    the k with b_k >= M (1 - 1e-9), for the exact certification
//  then k_eval_finish: S summed in i order by one thread, F = 2 n M / (S S)
//  (1e30 when S <= 0).
// ---------------------------------------------------------------------------
#include "common.cuh"

namespace sidon {
namespace bigeval {

constexpr int TK = 7;
constexpr int NW = 8;
constexpr int W = NW * 32 * TK;     // outputs per CTA
constexpr int CI = 1024;            // i cells per chunk
constexpr int YW = CI + W;          // reversed operand window (one spare cell)

enum Pass { kMax = 0, kCount = 1, kList = 2 };

template <typename Tin>
__global__ void __launch_bounds__(NW * 32)
k_eval_stream(const Tin* __restrict__ pop, int n, int pass,
              unsigned long long* __restrict__ mbits, double tol, int* __restrict__ count,
              int* __restrict__ list, int cap) {
  __shared__ double xs[CI];
  __shared__ double ys[YW];
  __shared__ double red[32];
  const int p = blockIdx.y;
  const Tin* a = pop + (size_t)p * n;
  const int nb = 2 * n - 1;
  const int k0 = blockIdx.x * W;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int q = (wid * 32 + lane) * TK;           // first output of the lane, relative to k0
  double acc[TK];
#pragma unroll
  for (int t = 0; t < TK; ++t) acc[t] = 0.0;
  const int ilo = max(0, k0 - (n - 1));
  const int ihi = min(n - 1, k0 + W - 1);
  for (int i0 = ilo; i0 <= ihi; i0 += CI) {
    __syncthreads();
    for (int t = threadIdx.x; t < CI; t += blockDim.x) {
      const int i = i0 + t;
      xs[t] = (i <= ihi) ? (double)a[i] : 0.0;
    }
    // ys[r] = a[js + r], js = k0 - i0 - CI + 1
    const int js = k0 - i0 - CI + 1;
    for (int r = threadIdx.x; r < YW; r += blockDim.x) {
      const int j = js + r;
      ys[r] = (j >= 0 && j < n) ? (double)a[j] : 0.0;
    }
    __syncthreads();
    const int cnt = min(CI, ihi - i0 + 1);
    // k = k0 + q + t, i = i0 + u: operand index (k - i) - js = q + t - u + CI - 1
    const double* yb = ys + q + CI - 1;
    for (int u = 0; u < cnt; ++u) {
      const double xv = xs[u];
#pragma unroll
      for (int t = 0; t < TK; ++t) acc[t] = __dadd_rn(acc[t], __dmul_rn(xv, yb[t - u]));
    }
  }
  if (pass == kMax) {
    double m = 0.0;
#pragma unroll
    for (int t = 0; t < TK; ++t)
      if (k0 + q + t < nb) m = acc[t] > m ? acc[t] : m;
    m = block_max(m, red);
    if (threadIdx.x == 0) atomicMax(&mbits[p], (unsigned long long)__double_as_longlong(m));
  } else {
    const double M = __longlong_as_double((long long)mbits[p]);
    const double thr = pass == kCount ? M * (1.0 - tol) : M * (1.0 - 1e-9);
    int c = 0;
#pragma unroll
    for (int t = 0; t < TK; ++t) {
      const int k = k0 + q + t;
      if (k < nb && acc[t] >= thr) {
        if (pass == kCount) ++c;
        else {
          const int s = atomicAdd(&count[p], 1);
          if (s < cap) list[(size_t)p * cap + s] = k;
        }
      }
    }
    if (pass == kCount) {
      c = __reduce_add_sync(0xffffffffu, c);
      if (lane == 0 && c) atomicAdd(&count[p], c);
    }
  }
}

// one thread per candidate: S in i order (hostF), F from the max bits
template <typename Tin>
__global__ void k_eval_finish(const Tin* __restrict__ pop, int n, int P,
                              unsigned long long* mbits_F) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  const Tin* a = pop + (size_t)p * n;
  double S = 0.0;
  for (int i = 0; i < n; ++i) S = __dadd_rn(S, (double)a[i]);
  const double M = __longlong_as_double((long long)mbits_F[p]);
  const double F = (S > 0.0) ? (2.0 * (double)n * M / (S * S)) : 1e30;
  mbits_F[p] = (unsigned long long)__double_as_longlong(F);
}

}  // namespace bigeval
}  // namespace sidon

namespace sidon_host {
using namespace sidon;

// Streams a candidate of any n; outF doubles as the max-bits scratch and
// outN as the counter.  list/cap: the near-maximal k for exact
// certification (pass kList) when list != NULL.
template <typename Tin>
static int eval_stream_t(const Tin* pop, int n, int P, double* outF, int* outN, double tol,
                         int* list, int* list_count, int cap, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(outF, 0, sizeof(double) * (size_t)P, st);
  if (e != cudaSuccess) return set_cuda_error(e);
  const dim3 grid((unsigned)((2 * (long long)n - 1 + bigeval::W - 1) / bigeval::W), (unsigned)P);
  auto* mb = reinterpret_cast<unsigned long long*>(outF);
  bigeval::k_eval_stream<Tin><<<grid, bigeval::NW * 32, 0, st>>>(pop, n, bigeval::kMax, mb, tol,
                                                                  nullptr, nullptr, 0);
  int rc = check_launch();
  if (rc) return rc;
  if (outN) {
    e = cudaMemsetAsync(outN, 0, sizeof(int) * (size_t)P, st);
    if (e != cudaSuccess) return set_cuda_error(e);
    bigeval::k_eval_stream<Tin><<<grid, bigeval::NW * 32, 0, st>>>(pop, n, bigeval::kCount, mb,
                                                                    tol, outN, nullptr, 0);
    rc = check_launch();
    if (rc) return rc;
  }
  if (list) {
    e = cudaMemsetAsync(list_count, 0, sizeof(int) * (size_t)P, st);
    if (e != cudaSuccess) return set_cuda_error(e);
    bigeval::k_eval_stream<Tin><<<grid, bigeval::NW * 32, 0, st>>>(pop, n, bigeval::kList, mb,
                                                                    tol, list_count, list, cap);
    rc = check_launch();
    if (rc) return rc;
    return SIDON_OK;          // the certification finishes from the list
  }
  bigeval::k_eval_finish<Tin><<<(P + 127) / 128, 128, 0, st>>>(pop, n, P, mb);
  return check_launch();
}

int launch_eval_stream(const void* pop, int dtype, int n, int P, double* outF, int* outN,
                       double tol, cudaStream_t st) {
  if (dtype == SIDON_F32)
    return eval_stream_t((const float*)pop, n, P, outF, outN, tol, nullptr, nullptr, 0, st);
  return eval_stream_t((const double*)pop, n, P, outF, outN, tol, nullptr, nullptr, 0, st);
}

// max bits into outM-as-scratch and the near-maximal k list (certification)
int launch_eval_stream_list(const void* pop, int dtype, int n, int P, double* mbits, int* list,
                            int* list_count, int cap, cudaStream_t st) {
  if (dtype == SIDON_F32)
    return eval_stream_t((const float*)pop, n, P, mbits, nullptr, 0.0, list, list_count, cap, st);
  return eval_stream_t((const double*)pop, n, P, mbits, nullptr, 0.0, list, list_count, cap, st);
}

}  // namespace sidon_host
