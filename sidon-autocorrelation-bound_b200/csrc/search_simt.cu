// ---------------------------------------------------------------------------
//  search_simt.cu -- CUDA-core kernels of the hot path:
//    k_local_search   L^p-annealed projected Adam / mirror descent
//                     (src/kernels.cuh:177-289), fp32 and fp64
//    k_lp_forward     G_p(a) = 2n ||a*a||_p / S^2 and the saved {M, S, R}
//    k_lp_backward    dG_p/da with b recomputed (or read back)
//    k_eval           certifying fp64 F + active-peak count
//                     (src/kernels.cuh:301-377, hostF arithmetic)
//    k_frank_wolfe    Chambolle-Pock Frank-Wolfe step (src/kernels.cuh:408-532)
//
//  One CTA per candidate; a candidate is a row of a uniform [P][n] batch or
//  a slice of a ragged batch (offsets[P+1]).  A ragged launch sizes CTAs for
//  n_max and lets each candidate use the threads a uniform launch at its own
//  n would have (Team), so results match the uniform kernels bit for bit.
//  Shared memory (T = element type, MG = margin):
//    sA [MG | n | MG]        heights (window + broadcast operand)
//    sC [MG | 2n-1 | MG]     b, then the weights c (correlation window)
//    sRed[32]                reduction scratch
// ---------------------------------------------------------------------------
#include "conv_simt.cuh"

namespace sidon {

template <typename T, int TK>
__host__ __device__ constexpr size_t ls_smem_elems(int n) {
  return (size_t)(n + 2 * margin<TK>()) + (size_t)(2 * n - 1 + 2 * margin<TK>()) + 32;
}

template <typename T>
__device__ __forceinline__ void zero_fill(T* p, int count) {
  for (int i = threadIdx.x; i < count; i += blockDim.x) p[i] = T(0);
}

// ------------------------------ local search ------------------------------
// The step's elementwise pieces, shared by the CTA and the warp kernels so
// that both compile them to the same arithmetic.
// weight c_k = (1+d)^(p-1) with d = (b_k - M)/M (0 for d = -1); adds
// c_k (1+d) to *r
template <typename T>
__device__ __forceinline__ T ls_weight(T b, T M, T pexp, T* r) {
  const T d = (b - M) / M;
  const T cw = d > T(-1) ? pow_from_d(d, pexp - T(1)) : T(0);
  *r += cw * (T(1) + d);
  return cw;
}
// Adam (mode 0, moments m / v updated in place) or mirror (mode 1) step of
// height x0 with gradient term g_i = G/R - M, then the projection
template <typename T>
__device__ __forceinline__ T ls_update(T x0, T G, T R, T M, int mode, T lr, T lrn, T beta1, T beta2,
                                       T bc1, T bc2, T* m, T* v) {
  const T gi = G / R - M;
  T x;
  if (mode == 0) {
    const T mm = dev_fma(beta1, *m, (T(1) - beta1) * gi);
    const T vv = dev_fma(beta2, *v, (T(1) - beta2) * gi * gi);
    *m = mm;
    *v = vv;
    const T step = lrn * (mm * bc1) / (dev_sqrt(vv * bc2) + T(1e-30));
    x = x0 - step;
    if (x < T(0)) x = T(0);
  } else {
    T e = -lr * (gi / M);
    if (e > T(4)) e = T(4);
    if (e < T(-4)) e = T(-4);
    x = x0 * dev_exp(e);
  }
  return x;
}

template <typename T, int TK>
__global__ void __launch_bounds__(1024, 1)
k_local_search(T* pop, T* mom, T* vel, const long long* __restrict__ offsets,
               const int* __restrict__ order, int n_fixed, int n_max,
               const int* __restrict__ skip, const int* __restrict__ mode_arr, int iters,
               T pStart, T pEnd, T lrStart, T lrEnd, T beta1, T beta2, int mode_default) {
  constexpr int MG = margin<TK>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Cand cd = cand_of(blockIdx.x, offsets, order, n_fixed);
  const int pid = cd.pid, n = cd.n;
  if (skip && skip[pid]) return;
  if (n < 1 || n > n_max) return;
  const Team tm(32 * warps_for<TK>(n));
  const int mode = mode_arr ? mode_arr[pid] : mode_default;
  T* a = pop + cd.off;
  T* m = mom + cd.off;
  T* v = vel + cd.off;
  const int nb = 2 * n - 1;
  T* base = reinterpret_cast<T*>(smem_raw);
  T* sA = base + MG;                        // [-MG, n + MG)
  T* sC = base + (n + 2 * MG) + MG;         // [-MG, 2n - 1 + MG)
  T* sRed = base + (n + 2 * MG) + (2 * n - 1 + 2 * MG);

  zero_fill(base, (int)ls_smem_elems<T, TK>(n));
  __syncthreads();
  for (int i = tm.t0; i < n; i += tm.nt) { sA[i] = a[i]; m[i] = T(0); v[i] = T(0); }
  __syncthreads();

  const T lnPr = T(log(double(pEnd) / double(pStart)));
  const T lnLr = T(log(double(lrEnd) / double(lrStart)));
  T b1t = T(1), b2t = T(1);

  for (int it = 0; it < iters; ++it) {
    const T frac = iters > 1 ? T(it) / T(iters - 1) : T(0);
    const T pexp = pStart * dev_exp(lnPr * frac);
    const T lr = lrStart * dev_exp(lnLr * frac);

    // b = a * a, and the running max in the same pass
    T mloc = T(0);
    conv_warp_tiles<TK, true>(sA, sA, n, tm, [&](int k, T val) {
      sC[k] = val;
      mloc = val > mloc ? val : mloc;
    });
    const T M = block_max(mloc, sRed);      // (barrier inside: sC complete)
    if (!(M > T(0))) break;

    // c_k = (1+d)^(p-1), R = sum c_k (1+d), d = (b_k - M)/M
    T rloc = T(0);
    for (int k = tm.t0; k < nb; k += tm.nt) sC[k] = ls_weight(sC[k], M, pexp, &rloc);
    const T R = block_sum(rloc, sRed);      // (barrier inside: c complete)

    b1t *= beta1;
    b2t *= beta2;
    const T bc1 = T(1) / (T(1) - b1t), bc2 = T(1) / (T(1) - b2t);
    const T lrn = lr / T(n);

    // G = corr(c, a); update fused into the epilogue; the new heights are
    // staged in the candidate's own row of pop (sA is still being read).
    corr_warp_tiles<TK>(sA, sC, n, tm, [&](int i, T G) {
      a[i] = ls_update(sA[i], G, R, M, mode, lr, lrn, beta1, beta2, bc1, bc2, m + i, v + i);
    });
    __syncthreads();

    T sloc = T(0);
    for (int i = tm.t0; i < n; i += tm.nt) {
      const T x = a[i];
      sA[i] = x;
      sloc += x;
    }
    T S = block_sum(sloc, sRed);
    if (!(S > T(0))) {
      for (int i = tm.t0; i < n; i += tm.nt) sA[i] = T(1) / T(n);
      S = T(1);
    }
    const T inv = T(1) / S;
    for (int i = tm.t0; i < n; i += tm.nt) sA[i] *= inv;
    __syncthreads();
  }
  for (int i = tm.t0; i < n; i += tm.nt) a[i] = sA[i];
}

// Small and middle candidates: the local search (and Frank-Wolfe) kernels
// with narrower lane tiles.  With 15-output tiles a team of 4 warps leaves
// most of its warps without a tile at small n (one correlation tile of 480
// outputs for n <= 480); the narrowest odd TK whose 4-warp tiles still span
// n (128 TK >= n) spreads the convolution and the correlation over all four.
// Results are bit for bit those of the 15-output kernels: every output is the
// same fma chain whatever the tiling, and the team (4 warps for n <= 1920),
// its per-thread sums and their order are the same.
__host__ __device__ constexpr int tile_for(int n) {
  return n <= 128 * 7 ? 7 : n <= 128 * 9 ? 9 : n <= 128 * 11 ? 11 : n <= 128 * 13 ? 13 : 15;
}

// ----------------------------- G_p forward --------------------------------
// value = 2n M R^(1/p) / S^2 with M = max b, R = sum (b/M)^p, S = sum a.  M is
// refined in fp64 over the near-maximal k and S summed in fp64, so the
// reported objective carries fp64-level error; R uses the fp32 b.
constexpr int kRefineCap = 1024;

template <int TK>
__global__ void __launch_bounds__(1024, 1)
k_lp_forward(const float* __restrict__ pop, int n, float p, float* __restrict__ value,
             float* __restrict__ saved, float* __restrict__ b_out) {
  constexpr int MG = margin<TK>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_list[kRefineCap];
  __shared__ int s_cnt;
  __shared__ double s_red[32];
  float* base = reinterpret_cast<float*>(smem_raw);
  float* sA = base + MG;
  float* sC = base + (n + 2 * MG) + MG;
  float* sRed = base + (n + 2 * MG) + (2 * n - 1 + 2 * MG);
  const int pid = blockIdx.x;
  const float* a = pop + (size_t)pid * n;
  const int nb = 2 * n - 1;
  const Team tm;
  zero_fill(base, (int)ls_smem_elems<float, TK>(n));
  __syncthreads();
  double sl = 0.0;
  for (int i = tm.t0; i < n; i += tm.nt) { const float x = a[i]; sA[i] = x; sl += x; }
  const double S = block_sum(sl, s_red);
  float mloc = 0.f;
  conv_warp_tiles<TK, true>(sA, sA, n, tm, [&](int k, float val) {
    sC[k] = val;
    mloc = val > mloc ? val : mloc;
  });
  const float Mapprox = block_max(mloc, sRed);
  const double Md = refine_max(
      n, [&](int i) { return sA[i]; }, [&](int k) { return sC[k]; }, Mapprox, 5e-4f, s_list,
      kRefineCap, &s_cnt, s_red);
  const float M = (float)Md;
  float rloc = 0.f;
  for (int k = tm.t0; k < nb; k += tm.nt) {
    const float d = (sC[k] - M) / M;
    rloc += d > -1.f ? pow_from_d(d, p) : 0.f;
    if (b_out) b_out[(size_t)pid * nb + k] = sC[k];
  }
  const float R = block_sum(rloc, sRed);
  if (threadIdx.x == 0) {
    const double val = 2.0 * (double)n * Md * pow((double)R, 1.0 / (double)p) / (S * S);
    value[pid] = (float)val;
    saved[4 * pid + 0] = M;
    saved[4 * pid + 1] = (float)S;
    saved[4 * pid + 2] = R;
    saved[4 * pid + 3] = (float)val;
  }
}

// ----------------------------- G_p backward -------------------------------
// grad_i = (4n R^(1/p)/S^2) (G_i/R - M/S),  G_i = sum_j (b_{i+j}/M)^(p-1) a_j
template <int TK>
__global__ void __launch_bounds__(1024, 1)
k_lp_backward(const float* __restrict__ pop, const float* __restrict__ saved,
              const float* __restrict__ b_in, int n, float p, float* __restrict__ grad) {
  constexpr int MG = margin<TK>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float* base = reinterpret_cast<float*>(smem_raw);
  float* sA = base + MG;
  float* sC = base + (n + 2 * MG) + MG;
  const int pid = blockIdx.x;
  const float* a = pop + (size_t)pid * n;
  const int nb = 2 * n - 1;
  const float M = saved[4 * pid + 0], S = saved[4 * pid + 1], R = saved[4 * pid + 2];
  const Team tm;
  zero_fill(base, (int)ls_smem_elems<float, TK>(n));
  __syncthreads();
  for (int i = tm.t0; i < n; i += tm.nt) sA[i] = a[i];
  __syncthreads();
  if (b_in) {
    for (int k = tm.t0; k < nb; k += tm.nt) sC[k] = b_in[(size_t)pid * nb + k];
  } else {
    conv_warp_tiles<TK, true>(sA, sA, n, tm, [&](int k, float val) { sC[k] = val; });
  }
  __syncthreads();
  for (int k = tm.t0; k < nb; k += tm.nt) {
    const float d = (sC[k] - M) / M;
    sC[k] = d > -1.f ? pow_from_d(d, p - 1.f) : 0.f;
  }
  __syncthreads();
  const float scale = 4.f * (float)n * powf(R, 1.f / p) / (S * S);
  const float MS = M / S;
  float* g = grad + (size_t)pid * n;
  corr_warp_tiles<TK>(sA, sC, n, tm, [&](int i, float G) { g[i] = scale * (G / R - MS); });
}

// ---------------------------- certifying eval -----------------------------
// fp64, hostF arithmetic: b_k = sum_i fl(a_i a_{k-i}) added in i order;
// S = sequential sum in i order; F = 2 n M / (S S) (src/main.cu:95-105).
// nActive = #{k : b_k >= M (1 - tol)} by a second pass (src/kernels.cuh:347-375).
template <typename Tin, int TK>
__global__ void __launch_bounds__(1024, 1)
k_eval(const Tin* __restrict__ pop, const long long* __restrict__ offsets,
       const int* __restrict__ order, int n_fixed, int n_max, double* __restrict__ outF,
       int* __restrict__ outN, double tol) {
  constexpr int MG = margin<TK>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double sS;
  const Cand cd = cand_of(blockIdx.x, offsets, order, n_fixed);
  const int pid = cd.pid, n = cd.n;
  if (n < 1 || n > n_max) return;
  const Team tm(32 * warps_for<TK>(n));
  double* base = reinterpret_cast<double*>(smem_raw);
  double* sA = base + MG;
  double* sRed = base + (n + 2 * MG);
  const Tin* a = pop + cd.off;
  zero_fill(base, n + 2 * MG);
  __syncthreads();
  for (int i = tm.t0; i < n; i += tm.nt) sA[i] = (double)a[i];
  __syncthreads();
  double mloc = 0.0;
  conv_warp_tiles<TK, false>(sA, sA, n, tm, [&](int, double val) { mloc = val > mloc ? val : mloc; });
  if (threadIdx.x == 0) {
    double S = 0.0;
    for (int i = 0; i < n; ++i) S = __dadd_rn(S, sA[i]);
    sS = S;
  }
  const double M = block_max(mloc, sRed);
  const double S = sS;
  if (outN) {
    const double thr = M * (1.0 - tol);
    double cl = 0.0;
    conv_warp_tiles<TK, false>(sA, sA, n, tm, [&](int, double val) { cl += (val >= thr) ? 1.0 : 0.0; });
    const double cnt = block_sum(cl, sRed);
    if (threadIdx.x == 0) outN[pid] = (int)(cnt + 0.5);
  }
  if (threadIdx.x == 0) outF[pid] = (S > 0.0) ? (2.0 * (double)n * M / (S * S)) : 1e30;
}

// --------------------------- Frank-Wolfe / PDHG ---------------------------
// sA [MG|n|MG] heights, sG [n] g, sGb [MG|n|MG] gbar / line-search point,
// sL [MG|2n-1|MG] lambda, sRed[32].
template <int TK>
__host__ __device__ constexpr size_t fw_smem_elems(int n) {
  return (size_t)(n + 2 * margin<TK>()) * 2 + (size_t)n + (size_t)(2 * n - 1 + 2 * margin<TK>()) +
         32;
}

template <int TK>
__global__ void __launch_bounds__(1024, 1)
k_frank_wolfe(float* pop, const long long* __restrict__ offsets, const int* __restrict__ order,
              int n_fixed, int n_max, const int* __restrict__ skip, int rounds, int pdhgIters,
              int nT, float tMax, float tau, float sig) {
  constexpr int MG = margin<TK>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Cand cd = cand_of(blockIdx.x, offsets, order, n_fixed);
  const int pid = cd.pid, n = cd.n;
  if (skip && skip[pid]) return;
  if (n < 1 || n > n_max) return;
  const Team tm(32 * warps_for<TK>(n));
  float* base = reinterpret_cast<float*>(smem_raw);
  float* sA = base + MG;
  float* sGb = base + (n + 2 * MG) + MG;
  float* sG = base + 2 * (n + 2 * MG);
  float* sL = sG + n + MG;
  float* sRed = sG + n + (2 * n - 1 + 2 * MG);
  float* a = pop + cd.off;
  const int nb = 2 * n - 1;
  zero_fill(base, (int)fw_smem_elems<TK>(n));
  __syncthreads();
  float sl = 0.f;
  for (int i = tm.t0; i < n; i += tm.nt) { const float x = a[i]; sA[i] = x; sl += x; }
  const float s0 = block_sum(sl, sRed);
  if (!(s0 > 0.f)) return;
  {
    const float inv = 1.f / s0;
    for (int i = tm.t0; i < n; i += tm.nt) sA[i] *= inv;
    __syncthreads();
  }
  if (!(tau > 0.f)) tau = 0.9f / (float)n;
  if (!(sig > 0.f)) sig = 0.9f * (float)n;

  for (int r = 0; r < rounds; ++r) {
    float ml = 0.f;
    conv_warp_tiles<TK, true>(sA, sA, n, tm, [&](int, float val) { ml = val > ml ? val : ml; });
    const float M = block_max(ml, sRed);
    if (!(M > 0.f)) break;

    for (int i = tm.t0; i < n; i += tm.nt) { sG[i] = sA[i]; sGb[i] = sA[i]; }
    for (int k = tm.t0; k < nb; k += tm.nt) sL[k] = 0.f;
    __syncthreads();

    for (int it = 0; it < pdhgIters; ++it) {
      // lambda <- [lambda + sigma (a * gbar - M)]_+   (conv fused)
      conv_warp_tiles<TK, true>(sA, sGb, n, tm, [&](int k, float val) {
        const float l = sL[k] + sig * (val - M);
        sL[k] = l > 0.f ? l : 0.f;
      });
      __syncthreads();
      // g_new <- [g + tau (1 - A^T lambda)]_+  parked in gbar
      corr_warp_tiles<TK>(sA, sL, n, tm, [&](int i, float cv) {
        const float gn = sG[i] + tau * (1.f - cv);
        sGb[i] = gn > 0.f ? gn : 0.f;
      });
      __syncthreads();
      for (int i = tm.t0; i < n; i += tm.nt) {
        const float gn = sGb[i], go = sG[i];
        sG[i] = gn;
        sGb[i] = 2.f * gn - go;
      }
      __syncthreads();
    }

    float sg = 0.f;
    for (int i = tm.t0; i < n; i += tm.nt) sg += sG[i];
    sg = block_sum(sg, sRed);
    if (!(sg > 0.f)) break;
    {
      const float inv = 1.f / sg;
      for (int i = tm.t0; i < n; i += tm.nt) sG[i] *= inv;
      __syncthreads();
    }
    // sum a = sum g = 1  =>  F(h) = 2n max(h*h) for every t
    float bestT = 0.f, bestM = M;
    for (int s = 1; s <= nT; ++s) {
      const float t = tMax * (float)s / (float)nT;
      for (int i = tm.t0; i < n; i += tm.nt) sGb[i] = (1.f - t) * sA[i] + t * sG[i];
      __syncthreads();
      float lc = 0.f;
      conv_warp_tiles<TK, true>(sGb, sGb, n, tm, [&](int, float val) { lc = val > lc ? val : lc; });
      const float mm = block_max(lc, sRed);
      if (mm < bestM) { bestM = mm; bestT = t; }
    }
    if (!(bestT > 0.f)) break;
    for (int i = tm.t0; i < n; i += tm.nt) sA[i] = (1.f - bestT) * sA[i] + bestT * sG[i];
    __syncthreads();
  }
  for (int i = tm.t0; i < n; i += tm.nt) a[i] = sA[i];
}

}  // namespace sidon

// =========================== host launch wrappers ==========================
namespace sidon_host {
using namespace sidon;

constexpr int kTK32 = 15;   // outputs per lane, fp32 kernels (odd: conflict-free windows)
constexpr int kTK64 = 7;    // outputs per lane, fp64 kernels

size_t smem_local_search(int n, int dtype) {
  if (dtype == SIDON_F32) return sizeof(float) * ls_smem_elems<float, kTK32>(n);
  if (dtype == SIDON_F64) return sizeof(double) * ls_smem_elems<double, kTK64>(n);
  return 0;
}
size_t smem_eval(int n) { return sizeof(double) * ((size_t)n + 2 * margin<kTK64>() + 32); }
size_t smem_fw(int n) { return sizeof(float) * fw_smem_elems<kTK32>(n); }

static int prep(const void* fn, size_t smem) { return set_dyn_smem(fn, smem); }

// uniform fp32 launches with TK-output lane tiles (TK < kTK32, 4-warp team)
template <int TK>
static int launch_ls_tiles(void* pop, void* mom, void* vel, int P, int n, const int* skip,
                           const int* mode_arr, int iters, double pS, double pE, double lrS,
                           double lrE, double b1, double b2, int mode_default, cudaStream_t st) {
  const size_t sm = sizeof(float) * ls_smem_elems<float, TK>(n);
  const int rc = prep((const void*)k_local_search<float, TK>, sm);
  if (rc) return rc;
  k_local_search<float, TK><<<P, 32 * warps_for<kTK32>(n), sm, st>>>(
      (float*)pop, (float*)mom, (float*)vel, nullptr, nullptr, n, n, skip, mode_arr, iters,
      (float)pS, (float)pE, (float)lrS, (float)lrE, (float)b1, (float)b2, mode_default);
  return check_launch();
}
template <int TK>
static int launch_fw_tiles(float* pop, int P, int n, const int* skip, int rounds, int pdhg, int nT,
                           float tMax, float tau, float sig, cudaStream_t st) {
  const size_t sm = sizeof(float) * fw_smem_elems<TK>(n);
  const int rc = prep((const void*)k_frank_wolfe<TK>, sm);
  if (rc) return rc;
  k_frank_wolfe<TK><<<P, 32 * warps_for<kTK32>(n), sm, st>>>(
      pop, nullptr, nullptr, n, n, skip, rounds, pdhg, nT, tMax, tau, sig);
  return check_launch();
}
// shared-memory attributes of the narrow-tile kernel at n (ahead of a capture)
static int prep_tiles(int n, bool local_search) {
  const int tk = tile_for(n);
  if (tk >= kTK32) return SIDON_OK;
#define SIDON_PREP_TILES(TK)                                                                 \
  return local_search                                                                        \
             ? prep((const void*)k_local_search<float, TK>,                                  \
                    sizeof(float) * ls_smem_elems<float, TK>(n))                             \
             : prep((const void*)k_frank_wolfe<TK>, sizeof(float) * fw_smem_elems<TK>(n))
  switch (tk) {
    case 7: SIDON_PREP_TILES(7);
    case 9: SIDON_PREP_TILES(9);
    case 11: SIDON_PREP_TILES(11);
    default: SIDON_PREP_TILES(13);
  }
#undef SIDON_PREP_TILES
}

// The shared-memory attributes of the fp32 local search, the fp32-input
// evaluation and the Frank-Wolfe kernels at n_max, set ahead of a stream
// capture.
int prepare_simt(int n_max, bool local_search) {
  int rc = SIDON_OK;
  if (local_search) {
    rc = prep((const void*)k_local_search<float, kTK32>, smem_local_search(n_max, SIDON_F32));
    if (!rc) rc = prep_tiles(n_max, true);
  }
  if (!rc) rc = prep((const void*)k_eval<float, kTK64>, smem_eval(n_max));
  if (!rc) rc = prep((const void*)k_frank_wolfe<kTK32>, smem_fw(n_max));
  if (!rc) rc = prep_tiles(n_max, false);
  return rc;
}

bool tuned_simt_tile(int n, int P, int* tk);
int launch_local_search_simt_tile(void* pop, void* mom, void* vel, int P, int n, const int* skip,
                                  const int* mode_arr, int iters, double pS, double pE,
                                  double lrS, double lrE, double b1, double b2, int mode_default,
                                  int tk, cudaStream_t st);

int simt_tile_default(int n) { return tile_for(n); }

// the odd lane tiles the fp32 local search can run at n (all give the same
// results bit for bit), narrowest first; returns their count
int simt_tile_choices(int n, int* out, int cap) {
  int cnt = 0;
  for (int tk = tile_for(n); tk <= kTK32 && cnt < cap; tk += 2) out[cnt++] = tk;
  return cnt;
}

int launch_local_search(void* pop, void* mom, void* vel, const long long* offsets,
                        const int* order, int P, int n_fixed, int n_max, const int* skip,
                        const int* mode_arr, int iters, double pS, double pE, double lrS,
                        double lrE, double b1, double b2, int mode_default, int dtype,
                        cudaStream_t st) {
  int tk = tile_for(n_max);
  if (dtype == SIDON_F32 && !offsets && tuned_simt_tile(n_max, P, &tk))
    return launch_local_search_simt_tile(pop, mom, vel, P, n_max, skip, mode_arr, iters, pS, pE,
                                         lrS, lrE, b1, b2, mode_default, tk, st);
  if (dtype == SIDON_F32 && !offsets && tile_for(n_max) < kTK32) {
    // uniform candidates of n <= 1664: narrower lane tiles over the same
    // 4-warp team (bitwise the kTK32 kernel's results)
    switch (tile_for(n_max)) {
      case 7: return launch_ls_tiles<7>(pop, mom, vel, P, n_max, skip, mode_arr, iters, pS, pE,
                                        lrS, lrE, b1, b2, mode_default, st);
      case 9: return launch_ls_tiles<9>(pop, mom, vel, P, n_max, skip, mode_arr, iters, pS, pE,
                                        lrS, lrE, b1, b2, mode_default, st);
      case 11: return launch_ls_tiles<11>(pop, mom, vel, P, n_max, skip, mode_arr, iters, pS, pE,
                                          lrS, lrE, b1, b2, mode_default, st);
      default: return launch_ls_tiles<13>(pop, mom, vel, P, n_max, skip, mode_arr, iters, pS, pE,
                                          lrS, lrE, b1, b2, mode_default, st);
    }
  }
  if (dtype == SIDON_F32) {
    const size_t sm = smem_local_search(n_max, dtype);
    const void* fn = (const void*)k_local_search<float, kTK32>;
    int rc = prep(fn, sm);
    if (rc) return rc;
    k_local_search<float, kTK32><<<P, 32 * warps_for<kTK32>(n_max), sm, st>>>(
        (float*)pop, (float*)mom, (float*)vel, offsets, order, n_fixed, n_max, skip, mode_arr,
        iters, (float)pS, (float)pE, (float)lrS, (float)lrE, (float)b1, (float)b2, mode_default);
  } else {
    const size_t sm = smem_local_search(n_max, dtype);
    const void* fn = (const void*)k_local_search<double, kTK64>;
    int rc = prep(fn, sm);
    if (rc) return rc;
    k_local_search<double, kTK64><<<P, 32 * warps_for<kTK64>(n_max), sm, st>>>(
        (double*)pop, (double*)mom, (double*)vel, offsets, order, n_fixed, n_max, skip,
        mode_arr, iters, pS, pE, lrS, lrE, b1, b2, mode_default);
  }
  return check_launch();
}

// The uniform fp32 local search with lane tile tk (one of simt_tile_choices).
int launch_local_search_simt_tile(void* pop, void* mom, void* vel, int P, int n, const int* skip,
                                  const int* mode_arr, int iters, double pS, double pE,
                                  double lrS, double lrE, double b1, double b2, int mode_default,
                                  int tk, cudaStream_t st) {
  switch (tk) {
    case 7: return launch_ls_tiles<7>(pop, mom, vel, P, n, skip, mode_arr, iters, pS, pE, lrS,
                                      lrE, b1, b2, mode_default, st);
    case 9: return launch_ls_tiles<9>(pop, mom, vel, P, n, skip, mode_arr, iters, pS, pE, lrS,
                                      lrE, b1, b2, mode_default, st);
    case 11: return launch_ls_tiles<11>(pop, mom, vel, P, n, skip, mode_arr, iters, pS, pE, lrS,
                                        lrE, b1, b2, mode_default, st);
    case 13: return launch_ls_tiles<13>(pop, mom, vel, P, n, skip, mode_arr, iters, pS, pE, lrS,
                                        lrE, b1, b2, mode_default, st);
    case kTK32: {
      const size_t sm = smem_local_search(n, SIDON_F32);
      const void* fn = (const void*)k_local_search<float, kTK32>;
      int rc = prep(fn, sm);
      if (rc) return rc;
      k_local_search<float, kTK32><<<P, 32 * warps_for<kTK32>(n), sm, st>>>(
          (float*)pop, (float*)mom, (float*)vel, nullptr, nullptr, n, n, skip, mode_arr, iters,
          (float)pS, (float)pE, (float)lrS, (float)lrE, (float)b1, (float)b2, mode_default);
      return check_launch();
    }
    default: return SIDON_ERR_ARG;
  }
}

int launch_lp_forward(const float* a, int n, int P, double p, float* value, float* saved,
                      float* b_out, cudaStream_t st) {
  const size_t sm = smem_local_search(n, SIDON_F32);
  int rc = prep((const void*)k_lp_forward<kTK32>, sm);
  if (rc) return rc;
  k_lp_forward<kTK32><<<P, 32 * warps_for<kTK32>(n), sm, st>>>(a, n, (float)p, value, saved, b_out);
  return check_launch();
}

int launch_lp_backward(const float* a, const float* saved, const float* b_in, int n, int P,
                       double p, float* grad, cudaStream_t st) {
  const size_t sm = smem_local_search(n, SIDON_F32);
  int rc = prep((const void*)k_lp_backward<kTK32>, sm);
  if (rc) return rc;
  k_lp_backward<kTK32><<<P, 32 * warps_for<kTK32>(n), sm, st>>>(a, saved, b_in, n, (float)p, grad);
  return check_launch();
}

int launch_eval(const void* pop, int dtype, const long long* offsets, const int* order, int P,
                int n_fixed, int n_max, double* outF, int* outN, double tol, cudaStream_t st) {
  const size_t sm = smem_eval(n_max);
  const int threads = 32 * warps_for<kTK64>(n_max);
  if (dtype == SIDON_F32) {
    int rc = prep((const void*)k_eval<float, kTK64>, sm);
    if (rc) return rc;
    k_eval<float, kTK64><<<P, threads, sm, st>>>((const float*)pop, offsets, order, n_fixed,
                                                 n_max, outF, outN, tol);
  } else {
    int rc = prep((const void*)k_eval<double, kTK64>, sm);
    if (rc) return rc;
    k_eval<double, kTK64><<<P, threads, sm, st>>>((const double*)pop, offsets, order, n_fixed,
                                                  n_max, outF, outN, tol);
  }
  return check_launch();
}

int launch_frank_wolfe(float* pop, const long long* offsets, const int* order, int P, int n_fixed,
                       int n_max, const int* skip, int rounds, int pdhg, int nT, float tMax,
                       float tau, float sig, cudaStream_t st) {
  if (!offsets && tile_for(n_max) < kTK32) {
    // uniform candidates of n <= 1664: narrower lane tiles over the same
    // 4-warp team (bitwise the kTK32 kernel's results)
    switch (tile_for(n_max)) {
      case 7: return launch_fw_tiles<7>(pop, P, n_max, skip, rounds, pdhg, nT, tMax, tau, sig, st);
      case 9: return launch_fw_tiles<9>(pop, P, n_max, skip, rounds, pdhg, nT, tMax, tau, sig, st);
      case 11: return launch_fw_tiles<11>(pop, P, n_max, skip, rounds, pdhg, nT, tMax, tau, sig, st);
      default: return launch_fw_tiles<13>(pop, P, n_max, skip, rounds, pdhg, nT, tMax, tau, sig, st);
    }
  }
  const size_t sm = smem_fw(n_max);
  int rc = prep((const void*)k_frank_wolfe<kTK32>, sm);
  if (rc) return rc;
  k_frank_wolfe<kTK32><<<P, 32 * warps_for<kTK32>(n_max), sm, st>>>(
      pop, offsets, order, n_fixed, n_max, skip, rounds, pdhg, nT, tMax, tau, sig);
  return check_launch();
}

}  // namespace sidon_host
