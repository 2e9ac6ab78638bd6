/* ---------------------------------------------------------------------------
 * sidon_oracle.c -- CPU restatement of the reference hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: tests/, the smoke
 * check of __graft_entry__ and the cpu_baseline leg of bench.py may load it;
 * nothing on the product path does.  Every function cites the reference
 * file:line it restates (paths are relative to the reference project root).
 *
 * Objective:  F(a) = 2 n max_k b_k / (sum_i a_i)^2 ,  b = a*a ,  a >= 0.
 *
 * Arithmetic conventions (chosen so that the CUDA kernels can be compared
 * bit for bit where that is meaningful):
 *   - fp32 convolutions / correlations are fmaf chains over the summation
 *     index in increasing order, starting from +0 (one rounding per term),
 *     exactly as a per-output FFMA chain on the GPU;
 *   - the fp64 certifying evaluation follows hostF (src/main.cu:95-105):
 *     product rounded, then added, i ascending; S summed sequentially.
 * ------------------------------------------------------------------------- */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define SO_EXPORT __attribute__((visibility("default")))

/* ======================= F in fp64, hostF semantics ======================= */
/* src/main.cu:95-105: b[i+j] += a_i a_j for a_i != 0 (i-major), M = max b,
 * S = sum a (sequential), F = 2 n M / S^2.  b is returned when b_out != NULL. */
SO_EXPORT double so_hostF_b(const double* a, int n, double* b_out) {
  const int nb = 2 * n - 1;
  double* b = (double*)calloc((size_t)nb, sizeof(double));
  for (int i = 0; i < n; ++i) {
    if (a[i] == 0.0) continue;
    const double ai = a[i];
    for (int j = 0; j < n; ++j) {
      volatile double prod = ai * a[j];   /* keep mul and add separately rounded */
      b[i + j] += prod;
    }
  }
  double M = 0.0;
  for (int k = 0; k < nb; ++k) M = b[k] > M ? b[k] : M;
  double S = 0.0;
  for (int i = 0; i < n; ++i) S += a[i];
  if (b_out) memcpy(b_out, b, sizeof(double) * (size_t)nb);
  free(b);
  return 2.0 * (double)n * M / (S * S);
}

SO_EXPORT double so_hostF(const double* a, int n) { return so_hostF_b(a, n, NULL); }

/* ================= certifying evaluation over a population =============== */
/* src/kernels.cuh:301-377 (kEval): F per candidate plus the number of k with
 * b_k >= M (1 - tol).  b is formed in hostF order (see header); F = 1e30 when
 * S <= 0 (kernels.cuh:376). */
SO_EXPORT void so_eval(const double* pop, int n, int P, double tol, double* F, int* nact) {
  const int nb = 2 * n - 1;
  double* b = (double*)malloc(sizeof(double) * (size_t)nb);
  for (int p = 0; p < P; ++p) {
    const double* a = pop + (size_t)p * n;
    for (int k = 0; k < nb; ++k) b[k] = 0.0;
    for (int i = 0; i < n; ++i) {
      if (a[i] == 0.0) continue;
      for (int j = 0; j < n; ++j) { volatile double prod = a[i] * a[j]; b[i + j] += prod; }
    }
    double M = 0.0, S = 0.0;
    for (int k = 0; k < nb; ++k) M = b[k] > M ? b[k] : M;
    for (int i = 0; i < n; ++i) S += a[i];
    if (nact) {
      const double thr = M * (1.0 - tol);
      int c = 0;
      for (int k = 0; k < nb; ++k) c += (b[k] >= thr);
      nact[p] = c;
    }
    F[p] = (S > 0.0) ? (2.0 * (double)n * M / (S * S)) : 1e30;
  }
  free(b);
}

/* =================== long-double verifier (probe --verify) ================ */
/* tools/probe.cpp:146-195: b_k as a direct sum over i ascending in long
 * double, M, S, F, the round-off bound 3 n eps / (1 - n eps) with eps = 2^-63,
 * and the count of b_k within 1e-9 of M.  Returns 1 if any a_i < 0. */
SO_EXPORT int so_verify_ld(const double* a_in, int n, long double* F, long double* M_out,
                           long double* S_out, int* kmax_out, int* nactive_out,
                           long double* relbound) {
  long double* a = (long double*)malloc(sizeof(long double) * (size_t)n);
  int neg = 0;
  for (int i = 0; i < n; ++i) { a[i] = (long double)a_in[i]; if (a[i] < 0) neg = 1; }
  const int nb = 2 * n - 1;
  long double* b = (long double*)malloc(sizeof(long double) * (size_t)nb);
#pragma omp parallel for schedule(static)
  for (int k = 0; k < nb; ++k) {
    const int ilo = k - n + 1 > 0 ? k - n + 1 : 0, ihi = k < n - 1 ? k : n - 1;
    long double s = 0.0L;
    for (int i = ilo; i <= ihi; ++i) s += a[i] * a[k - i];
    b[k] = s;
  }
  long double M = 0, S = 0; int kmax = 0;
  for (int k = 0; k < nb; ++k) if (b[k] > M) { M = b[k]; kmax = k; }
  for (int i = 0; i < n; ++i) S += a[i];
  const long double eps = 1.084202172485504434e-19L;
  const long double gam = (long double)n * eps / (1 - (long double)n * eps);
  int nAct = 0;
  for (int k = 0; k < nb; ++k) if (b[k] >= M * (1 - 1e-9L)) ++nAct;
  *F = 2.0L * (long double)n * M / (S * S);
  if (M_out) *M_out = M;
  if (S_out) *S_out = S;
  if (kmax_out) *kmax_out = kmax;
  if (nactive_out) *nactive_out = nAct;
  if (relbound) *relbound = 3 * gam;
  free(a); free(b);
  return neg;
}

/* ============================ fp32 primitives ============================= */
/* src/kernels.cuh:97-135 (crossconv/autoconv): b_k = sum_i x_i y_{k-i},
 * k = 0..2n-2, one fmaf chain per k over i ascending. */
static void conv_f32(const float* x, const float* y, float* b, int n) {
  for (int k = 0; k < 2 * n - 1; ++k) {
    const int ilo = k - (n - 1) > 0 ? k - (n - 1) : 0, ihi = k < n - 1 ? k : n - 1;
    float acc = 0.0f;
    for (int i = ilo; i <= ihi; ++i) acc = fmaf(x[i], y[k - i], acc);
    b[k] = acc;
  }
}
/* src/kernels.cuh:142-158 (corrTile): G_i = sum_j c_{i+j} a_j, j ascending. */
static void corr_f32(const float* a, const float* c, float* G, int n) {
  for (int i = 0; i < n; ++i) {
    float acc = 0.0f;
    for (int j = 0; j < n; ++j) acc = fmaf(a[j], c[i + j], acc);
    G[i] = acc;
  }
}
SO_EXPORT void so_conv_f32(const float* x, const float* y, float* b, int n) { conv_f32(x, y, b, n); }
SO_EXPORT void so_corr_f32(const float* a, const float* c, float* G, int n) { corr_f32(a, c, G, n); }

/* fp64 twins (used by the fp64 local search) */
static void conv_f64(const double* x, const double* y, double* b, int n) {
  for (int k = 0; k < 2 * n - 1; ++k) {
    const int ilo = k - (n - 1) > 0 ? k - (n - 1) : 0, ihi = k < n - 1 ? k : n - 1;
    double acc = 0.0;
    for (int i = ilo; i <= ihi; ++i) acc = fma(x[i], y[k - i], acc);
    b[k] = acc;
  }
}
static void corr_f64(const double* a, const double* c, double* G, int n) {
  for (int i = 0; i < n; ++i) {
    double acc = 0.0;
    for (int j = 0; j < n; ++j) acc = fma(a[j], c[i + j], acc);
    G[i] = acc;
  }
}

/* ===================== L^p-annealed projected Adam ======================== */
/* src/kernels.cuh:177-289 (kLocalSearch), one candidate, in the kernel's
 * update order: conv, M, weights c_k = (1+d)^(p-1) with d = (b_k-M)/M and
 * R = sum c_k (1+d), bias corrections, correlation G, g_i = G_i/R - M,
 * Adam (mode 0) or mirror step (mode 1), projection, renormalisation.
 * mom/vel are zeroed at entry (kernels.cuh:196). */
#define SO_LS_BODY(T, CONV, CORR, EXP, LOG1P, SQRT, FMA)                                   \
  const int nb = 2 * n - 1;                                                                \
  T* b = (T*)malloc(sizeof(T) * (size_t)(2 * n));                                          \
  T* G = (T*)malloc(sizeof(T) * (size_t)n);                                                \
  T* m = (T*)calloc((size_t)n, sizeof(T));                                                 \
  T* v = (T*)calloc((size_t)n, sizeof(T));                                                 \
  const T lnPr = (T)log((double)pEnd / (double)pStart);                                    \
  const T lnLr = (T)log((double)lrEnd / (double)lrStart);                                  \
  T b1t = (T)1, b2t = (T)1;                                                                \
  for (int it = 0; it < iters; ++it) {                                                     \
    const T frac = iters > 1 ? (T)it / (T)(iters - 1) : (T)0;                              \
    const T pexp = pStart * EXP(lnPr * frac);                                              \
    const T lr = lrStart * EXP(lnLr * frac);                                               \
    CONV(a, a, b, n);                                                                      \
    T M = (T)0;                                                                            \
    for (int k = 0; k < nb; ++k) M = b[k] > M ? b[k] : M;                                  \
    if (!(M > (T)0)) break;                                                                \
    T R = (T)0;                                                                            \
    for (int k = 0; k < nb; ++k) {                                                         \
      const T d = (b[k] - M) / M;                                                          \
      const T c = d > (T)-1 ? EXP((pexp - (T)1) * LOG1P(d)) : (T)0;                        \
      R += c * ((T)1 + d);                                                                 \
      b[k] = c;                                                                            \
    }                                                                                      \
    b[nb] = (T)0;                                                                          \
    b1t *= beta1; b2t *= beta2;                                                            \
    const T bc1 = (T)1 / ((T)1 - b1t), bc2 = (T)1 / ((T)1 - b2t);                          \
    CORR(a, b, G, n);                                                                      \
    T S = (T)0;                                                                            \
    for (int i = 0; i < n; ++i) {                                                          \
      const T gi = G[i] / R - M;                                                           \
      T x;                                                                                 \
      if (mode == 0) {                                                                     \
        const T mm = FMA(beta1, m[i], ((T)1 - beta1) * gi);                                \
        const T vv = FMA(beta2, v[i], ((T)1 - beta2) * gi * gi);                           \
        m[i] = mm; v[i] = vv;                                                              \
        const T step = (lr / (T)n) * (mm * bc1) / (SQRT(vv * bc2) + (T)1e-30);             \
        x = a[i] - step;                                                                   \
        if (x < (T)0) x = (T)0;                                                            \
      } else {                                                                             \
        T e = -lr * (gi / M);                                                              \
        if (e > (T)4) e = (T)4;                                                            \
        if (e < (T)-4) e = (T)-4;                                                          \
        x = a[i] * EXP(e);                                                                 \
      }                                                                                    \
      a[i] = x; S += x;                                                                    \
    }                                                                                      \
    if (!(S > (T)0)) { for (int i = 0; i < n; ++i) a[i] = (T)1 / (T)n; S = (T)1; }         \
    const T inv = (T)1 / S;                                                                \
    for (int i = 0; i < n; ++i) a[i] *= inv;                                               \
  }                                                                                        \
  free(b); free(G); free(m); free(v);

static void ls_f32(float* a, int n, int iters, float pStart, float pEnd, float lrStart,
                   float lrEnd, float beta1, float beta2, int mode) {
  SO_LS_BODY(float, conv_f32, corr_f32, expf, log1pf, sqrtf, fmaf)
}
static void ls_f64(double* a, int n, int iters, double pStart, double pEnd, double lrStart,
                   double lrEnd, double beta1, double beta2, int mode) {
  SO_LS_BODY(double, conv_f64, corr_f64, exp, log1p, sqrt, fma)
}

/* Population driver with the kernel's skip[] / modeArr[] semantics
 * (kernels.cuh:188-190): skipped candidates are left untouched. */
SO_EXPORT void so_local_search_f32(float* pop, int n, int P, int iters, float pS, float pE,
                                   float lrS, float lrE, float b1, float b2, const int* skip,
                                   const int* mode_arr, int mode_default) {
#pragma omp parallel for schedule(dynamic)
  for (int p = 0; p < P; ++p) {
    if (skip && skip[p]) continue;
    ls_f32(pop + (size_t)p * n, n, iters, pS, pE, lrS, lrE, b1, b2,
           mode_arr ? mode_arr[p] : mode_default);
  }
}
SO_EXPORT void so_local_search_f64(double* pop, int n, int P, int iters, double pS, double pE,
                                   double lrS, double lrE, double b1, double b2, const int* skip,
                                   const int* mode_arr, int mode_default) {
#pragma omp parallel for schedule(dynamic)
  for (int p = 0; p < P; ++p) {
    if (skip && skip[p]) continue;
    ls_f64(pop + (size_t)p * n, n, iters, pS, pE, lrS, lrE, b1, b2,
           mode_arr ? mode_arr[p] : mode_default);
  }
}

/* One step's intermediates at fp32 (for single-step parity): b = a*a, M,
 * c (in place of b), R, G.  Mirrors kernels.cuh:213-239. */
SO_EXPORT void so_lp_step_terms_f32(const float* a, int n, float p, float* b_out, float* c_out,
                                    float* G_out, float* MR_out) {
  const int nb = 2 * n - 1;
  float* b = (float*)malloc(sizeof(float) * (size_t)(2 * n));
  conv_f32(a, a, b, n);
  if (b_out) memcpy(b_out, b, sizeof(float) * (size_t)nb);
  float M = 0.f;
  for (int k = 0; k < nb; ++k) M = b[k] > M ? b[k] : M;
  float R = 0.f;
  for (int k = 0; k < nb; ++k) {
    const float d = (b[k] - M) / M;
    const float c = d > -1.f ? expf((p - 1.f) * log1pf(d)) : 0.f;
    R += c * (1.f + d);
    b[k] = c;
  }
  b[nb] = 0.f;
  if (c_out) memcpy(c_out, b, sizeof(float) * (size_t)nb);
  if (G_out) corr_f32(a, b, G_out, n);
  MR_out[0] = M; MR_out[1] = R;
  free(b);
}

/* ====================== smoothed objective and gradient =================== */
/* G_p(a) = 2n ||a*a||_p / (sum a)^2 (the objective the reference's anneal
 * minimises, kernels.cuh:168-172).  With M = max|b|, u = |b|/M,
 * R = sum u^p:  G_p = 2n M R^(1/p) / S^2 and
 *   dG_p/da_i = (4n R^(1/p) / S^2) (G_i / R - M / S),  G_i = sum_j u_{i+j}^(p-1) a_j,
 * the gradient whose descent direction the reference uses when S = 1
 * (kernels.cuh:169-172, tools/probe.cpp:87-92).  |b| keeps the value defined
 * for finite-difference probes that step a coordinate below zero.  Long
 * double throughout. */
SO_EXPORT double so_lp_value_ld(const double* a_in, int n, double p) {
  const int nb = 2 * n - 1;
  long double* a = (long double*)malloc(sizeof(long double) * (size_t)n);
  long double* b = (long double*)malloc(sizeof(long double) * (size_t)nb);
  for (int i = 0; i < n; ++i) a[i] = a_in[i];
  long double S = 0, M = 0;
  for (int i = 0; i < n; ++i) S += a[i];
  for (int k = 0; k < nb; ++k) {
    const int ilo = k - n + 1 > 0 ? k - n + 1 : 0, ihi = k < n - 1 ? k : n - 1;
    long double s = 0;
    for (int i = ilo; i <= ihi; ++i) s += a[i] * a[k - i];
    b[k] = fabsl(s);
    if (b[k] > M) M = b[k];
  }
  long double R = 0;
  for (int k = 0; k < nb; ++k) R += powl(b[k] / M, (long double)p);
  const long double val = 2.0L * n * M * powl(R, 1.0L / (long double)p) / (S * S);
  free(a); free(b);
  return (double)val;
}

SO_EXPORT void so_lp_grad_ld(const double* a_in, int n, double p, double* grad, double* value) {
  const int nb = 2 * n - 1;
  long double* a = (long double*)malloc(sizeof(long double) * (size_t)n);
  long double* c = (long double*)malloc(sizeof(long double) * (size_t)nb);
  for (int i = 0; i < n; ++i) a[i] = a_in[i];
  long double S = 0, M = 0;
  for (int i = 0; i < n; ++i) S += a[i];
  for (int k = 0; k < nb; ++k) {
    const int ilo = k - n + 1 > 0 ? k - n + 1 : 0, ihi = k < n - 1 ? k : n - 1;
    long double s = 0;
    for (int i = ilo; i <= ihi; ++i) s += a[i] * a[k - i];
    c[k] = s;
    if (s > M) M = s;
  }
  long double R = 0;
  for (int k = 0; k < nb; ++k) {
    const long double u = c[k] / M;
    R += powl(u, (long double)p);
    c[k] = powl(u, (long double)p - 1.0L);
  }
  const long double Rp = powl(R, 1.0L / (long double)p);
  const long double scale = 4.0L * n * Rp / (S * S);
  for (int i = 0; i < n; ++i) {
    long double g = 0;
    for (int j = 0; j < n; ++j) g += c[i + j] * a[j];
    grad[i] = (double)(scale * (g / R - M / S));
  }
  if (value) *value = (double)(2.0L * n * M * Rp / (S * S));
  free(a); free(c);
}

/* ============== Frank-Wolfe step solved by Chambolle-Pock ================= */
/* src/kernels.cuh:408-532 (kFrankWolfe), fp32, in the kernel's order.
 * tau_scale / sig_scale: tau = tau_scale / n, sigma = sig_scale * n
 * (the reference uses 0.9 and 0.9, kernels.cuh:440). */
static void fw_f32(float* a, int n, int rounds, int pdhgIters, int nT, float tMax, float tau_c,
                   float sig_c) {
  const int nb = 2 * n - 1;
  float* G = (float*)malloc(sizeof(float) * (size_t)n);
  float* Gb = (float*)malloc(sizeof(float) * (size_t)n);
  float* lam = (float*)calloc((size_t)(2 * n), sizeof(float));
  float* tmp = (float*)malloc(sizeof(float) * (size_t)(2 * n));
  float* cc = (float*)malloc(sizeof(float) * (size_t)n);
  float s = 0.f;
  for (int i = 0; i < n; ++i) s += a[i];
  if (!(s > 0.f)) goto done;
  {
    const float inv = 1.f / s;
    for (int i = 0; i < n; ++i) a[i] *= inv;
  }
  {
    const float tau = tau_c / (float)n, sig = sig_c * (float)n;
    for (int r = 0; r < rounds; ++r) {
      conv_f32(a, a, tmp, n);
      float M = 0.f;
      for (int k = 0; k < nb; ++k) M = tmp[k] > M ? tmp[k] : M;
      if (!(M > 0.f)) break;
      for (int i = 0; i < n; ++i) { G[i] = a[i]; Gb[i] = a[i]; }
      for (int k = 0; k < 2 * n; ++k) lam[k] = 0.f;
      for (int it = 0; it < pdhgIters; ++it) {
        conv_f32(a, Gb, tmp, n);
        for (int k = 0; k < nb; ++k) {
          const float l = lam[k] + sig * (tmp[k] - M);
          lam[k] = l > 0.f ? l : 0.f;
        }
        corr_f32(a, lam, cc, n);
        for (int i = 0; i < n; ++i) {
          const float gn = G[i] + tau * (1.f - cc[i]);
          Gb[i] = gn > 0.f ? gn : 0.f;
        }
        for (int i = 0; i < n; ++i) {
          const float gn = Gb[i], go = G[i];
          G[i] = gn;
          Gb[i] = 2.f * gn - go;
        }
      }
      float sg = 0.f;
      for (int i = 0; i < n; ++i) sg += G[i];
      if (!(sg > 0.f)) break;
      {
        const float inv = 1.f / sg;
        for (int i = 0; i < n; ++i) G[i] *= inv;
      }
      float bestT = 0.f, bestM = M;
      for (int st = 1; st <= nT; ++st) {
        const float t = tMax * (float)st / (float)nT;
        for (int i = 0; i < n; ++i) Gb[i] = (1.f - t) * a[i] + t * G[i];
        conv_f32(Gb, Gb, tmp, n);
        float mm = 0.f;
        for (int k = 0; k < nb; ++k) mm = tmp[k] > mm ? tmp[k] : mm;
        if (mm < bestM) { bestM = mm; bestT = t; }
      }
      if (!(bestT > 0.f)) break;
      for (int i = 0; i < n; ++i) a[i] = (1.f - bestT) * a[i] + bestT * G[i];
    }
  }
done:
  free(G); free(Gb); free(lam); free(tmp); free(cc);
}

SO_EXPORT void so_frank_wolfe_f32(float* pop, int n, int P, int rounds, int pdhgIters, int nT,
                                  float tMax, float tau_c, float sig_c, const int* skip) {
#pragma omp parallel for schedule(dynamic)
  for (int p = 0; p < P; ++p) {
    if (skip && skip[p]) continue;
    fw_f32(pop + (size_t)p * n, n, rounds, pdhgIters, nT, tMax, tau_c, sig_c);
  }
}

/* ============================ cell-split ladder =========================== */
/* src/kernels.cuh:538-547 (kRefine) and src/main.cu:494-495: a'_{2i} = a'_{2i+1} = a_i. */
SO_EXPORT void so_refine_f64(const double* src, int n, int P, double* dst) {
  for (int p = 0; p < P; ++p)
    for (int i = 0; i < n; ++i) {
      const double x = src[(size_t)p * n + i];
      dst[(size_t)p * 2 * n + 2 * i] = x;
      dst[(size_t)p * 2 * n + 2 * i + 1] = x;
    }
}
/* src/kernels.cuh:550-557 (kCoarsen): d_i = 0.5 (s_{2i} + s_{2i+1}). */
SO_EXPORT void so_coarsen_f64(const double* src, int n2, int P, double* dst) {
  for (int p = 0; p < P; ++p)
    for (int i = 0; i < n2 / 2; ++i)
      dst[(size_t)p * (n2 / 2) + i] =
          0.5 * (src[(size_t)p * n2 + 2 * i] + src[(size_t)p * n2 + 2 * i + 1]);
}

/* ========================= island ranking + migration ===================== */
/* src/main.cu:676-692: each island (PI consecutive slots) is ranked by fp64
 * fitness, ascending; ties are broken by slot index (the reference's
 * std::sort leaves tie order unspecified) and NaN ranks last (undefined for
 * std::sort).  Migration: the j-th best of
 * island i overwrites the j-th worst of island (i+1) mod NI, j < k (k = 1 is
 * the reference's "best of i -> worst of i+1").  order_out[i*PI + r] = slot of
 * rank r in island i, computed before migration.  Requires 2k <= PI. */
static const double* g_fit_cmp;
static int cmp_slot(const void* x, const void* y) {
  const int a = *(const int*)x, b = *(const int*)y;
  const double fa = g_fit_cmp[a], fb = g_fit_cmp[b];
  const int na = fa != fa, nb = fb != fb;   /* NaN ranks after every number */
  if (na != nb) return na - nb;
  if (!na) {
    if (fa < fb) return -1;
    if (fa > fb) return 1;
  }
  return (a > b) - (a < b);
}
SO_EXPORT int so_island_migrate_f32(float* pop, int n, double* fit, int P, int NI, int k,
                                    int* order_out) {
  if (NI <= 0 || P % NI) return 1;
  const int PI = P / NI;
  if (2 * k > PI) return 2;
  int* ord = order_out ? order_out : (int*)malloc(sizeof(int) * (size_t)P);
  for (int i = 0; i < NI; ++i) {
    for (int r = 0; r < PI; ++r) ord[i * PI + r] = i * PI + r;
    g_fit_cmp = fit;
    qsort(ord + i * PI, (size_t)PI, sizeof(int), cmp_slot);
  }
  if (k > 0) {
    for (int i = 0; i < NI; ++i) {
      const int nx = (i + 1) % NI;
      for (int j = 0; j < k; ++j) {
        const int src = ord[i * PI + j], dst = ord[nx * PI + PI - 1 - j];
        memcpy(pop + (size_t)dst * n, pop + (size_t)src * n, sizeof(float) * (size_t)n);
      }
    }
    /* fitness follows the copied rows */
    double* f2 = (double*)malloc(sizeof(double) * (size_t)P);
    memcpy(f2, fit, sizeof(double) * (size_t)P);
    for (int i = 0; i < NI; ++i) {
      const int nx = (i + 1) % NI;
      for (int j = 0; j < k; ++j) f2[ord[nx * PI + PI - 1 - j]] = fit[ord[i * PI + j]];
    }
    memcpy(fit, f2, sizeof(double) * (size_t)P);
    free(f2);
  }
  if (!order_out) free(ord);
  return 0;
}

/* src/main.cu:555-562 (injectDouble) for an fp32 source: nearest-neighbour
 * resample x_t = src[min(m-1, floor(t m / n))], S = sum of x_t in t order
 * (fp64), dst_t = fl32(x_t / S) when S > 0 (else the resampled values). */
SO_EXPORT void so_resample_f32(const float* src, int m, float* dst, int n) {
  double S = 0.0;
  for (int t = 0; t < n; ++t) {
    long long q = (long long)t * m / n;
    if (q > m - 1) q = m - 1;
    dst[t] = src[q];
    S += (double)src[q];
  }
  if (S > 0.0)
    for (int t = 0; t < n; ++t) dst[t] = (float)((double)dst[t] / S);
}

/* Ragged island migration: ranking as so_island_migrate_f32; a migrant of
 * the destination's size is copied with its fitness, one of another size is
 * resampled by so_resample_f32 and its fitness set to NaN.  Candidate p is
 * pop[off[p] .. off[p+1]). */
SO_EXPORT int so_island_migrate_ragged_f32(float* pop, const long long* off, double* fit, int P,
                                           int NI, int k, int* order_out) {
  if (NI <= 0 || P % NI) return 1;
  const int PI = P / NI;
  if (2 * k > PI) return 2;
  int* ord = order_out ? order_out : (int*)malloc(sizeof(int) * (size_t)P);
  for (int i = 0; i < NI; ++i) {
    for (int r = 0; r < PI; ++r) ord[i * PI + r] = i * PI + r;
    g_fit_cmp = fit;
    qsort(ord + i * PI, (size_t)PI, sizeof(int), cmp_slot);
  }
  if (k > 0) {
    double* f2 = (double*)malloc(sizeof(double) * (size_t)P);
    memcpy(f2, fit, sizeof(double) * (size_t)P);
    for (int i = 0; i < NI; ++i) {
      const int nx = (i + 1) % NI;
      for (int j = 0; j < k; ++j) {
        const int src = ord[i * PI + j], dst = ord[nx * PI + PI - 1 - j];
        const int m = (int)(off[src + 1] - off[src]), n = (int)(off[dst + 1] - off[dst]);
        if (m == n) {
          memcpy(pop + off[dst], pop + off[src], sizeof(float) * (size_t)n);
          f2[dst] = fit[src];
        } else {
          so_resample_f32(pop + off[src], m, pop + off[dst], n);
          f2[dst] = NAN;
        }
      }
    }
    memcpy(fit, f2, sizeof(double) * (size_t)P);
    free(f2);
  }
  if (!order_out) free(ord);
  return 0;
}

/* ============================ exact certification ========================= */
/* F from EXACT M = max_k b_k and EXACT S = sum a, each rounded once to fp64
 * (round to nearest even), then F = 2 n M / (S S) in fp64.  Exact b_k comes
 * from a fixed-point accumulator of 64-bit limbs covering 2^-1216..2^+1088
 * (every product of two finite doubles above the subnormal range is exact
 * in it).  Because refinement maps M -> 2M and S -> 2S exactly, this F is
 * bit-identical before and after a cell split.  No reference counterpart:
 * the reference's hostF (src/main.cu:95-105) is not split-invariant to the
 * last bit. */
#define XLIMBS 36
#define XLO (-1216)
typedef struct { uint64_t w[XLIMBS]; } xacc;

static void xacc_add_u64(xacc* A, uint64_t mant, int e) {
  /* adds mant * 2^e, mant < 2^64, e >= XLO */
  const int sh = e - XLO;
  int li = sh >> 6, bo = sh & 63;
  unsigned __int128 v = (unsigned __int128)mant << bo;
  uint64_t lo = (uint64_t)v, hi = (uint64_t)(v >> 64);
  uint64_t old = A->w[li];
  A->w[li] = old + lo;
  uint64_t carry = (A->w[li] < old);
  ++li;
  while ((hi || carry) && li < XLIMBS) {
    old = A->w[li];
    uint64_t t = old + hi;
    uint64_t c1 = (t < old);
    uint64_t t2 = t + carry;
    uint64_t c2 = (t2 < t);
    A->w[li] = t2;
    carry = c1 + c2;
    hi = 0;
    ++li;
  }
}
static void xacc_add_double(xacc* A, double x) {
  /* x >= 0 finite */
  if (x == 0.0) return;
  int e;
  const double fr = frexp(x, &e);              /* x = fr * 2^e, fr in [0.5,1) */
  const uint64_t mant = (uint64_t)ldexp(fr, 53);  /* exact 53-bit integer */
  xacc_add_u64(A, mant, e - 53);               /* e - 53 >= -1127 > XLO for every double */
}
static int xacc_cmp(const xacc* A, const xacc* B) {
  for (int i = XLIMBS - 1; i >= 0; --i) {
    if (A->w[i] != B->w[i]) return A->w[i] > B->w[i] ? 1 : -1;
  }
  return 0;
}
static double xacc_to_double(const xacc* A) {
  int top = XLIMBS - 1;
  while (top >= 0 && A->w[top] == 0) --top;
  if (top < 0) return 0.0;
  const int lz = __builtin_clzll(A->w[top]);
  const int msb = top * 64 + (63 - lz);        /* bit index of the leading one */
  /* take 53 bits [msb-52, msb], round bit msb-53, sticky below */
  uint64_t mant = 0;
  for (int bit = msb; bit >= msb - 52; --bit) {
    mant <<= 1;
    if (bit >= 0) mant |= (A->w[bit >> 6] >> (bit & 63)) & 1ull;
  }
  int rb = 0, sticky = 0;
  const int rbit = msb - 53;
  if (rbit >= 0) {
    const int li = rbit >> 6, bo = rbit & 63;
    rb = (int)((A->w[li] >> bo) & 1ull);
    if (bo > 0 && (A->w[li] & ((1ull << bo) - 1ull))) sticky = 1;
    for (int j = li - 1; j >= 0 && !sticky; --j)
      if (A->w[j]) sticky = 1;
  }
  if (rb && (sticky || (mant & 1ull))) ++mant;
  return ldexp((double)mant, msb - 52 + XLO);
}

/* Exact b_k for one k of a double vector: products split by FMA into
 * p + e with both exact doubles (p = fl(ab), e = fma(a,b,-p)); e may be
 * negative, so positive and negative parts are accumulated apart. */
static void exact_bk(const double* a, int n, int k, xacc* pos, xacc* neg) {
  memset(pos, 0, sizeof(xacc));
  memset(neg, 0, sizeof(xacc));
  const int ilo = k - n + 1 > 0 ? k - n + 1 : 0, ihi = k < n - 1 ? k : n - 1;
  for (int i = ilo; i <= ihi; ++i) {
    const double x = a[i], y = a[k - i];
    if (x == 0.0 || y == 0.0) continue;
    const double p = x * y;
    const double e = fma(x, y, -p);
    xacc_add_double(pos, p);
    if (e > 0) xacc_add_double(pos, e);
    else if (e < 0) xacc_add_double(neg, -e);
  }
}
static void xacc_sub(xacc* A, const xacc* B) {  /* A -= B, A >= B */
  uint64_t borrow = 0;
  for (int i = 0; i < XLIMBS; ++i) {
    const uint64_t a = A->w[i], b = B->w[i];
    const uint64_t d = a - b - borrow;
    borrow = (a < b) || (a - b < borrow);
    A->w[i] = d;
  }
}

SO_EXPORT double so_certify_exact(const double* a, int n, int* kmax_out, double* M_out,
                                  double* S_out) {
  xacc best, cur, neg, S;
  memset(&best, 0, sizeof best);
  int kbest = 0;
  for (int k = 0; k < 2 * n - 1; ++k) {
    exact_bk(a, n, k, &cur, &neg);
    xacc_sub(&cur, &neg);
    if (xacc_cmp(&cur, &best) > 0) { best = cur; kbest = k; }
  }
  memset(&S, 0, sizeof S);
  for (int i = 0; i < n; ++i) xacc_add_double(&S, a[i]);
  const double M = xacc_to_double(&best), Sd = xacc_to_double(&S);
  if (kmax_out) *kmax_out = kbest;
  if (M_out) *M_out = M;
  if (S_out) *S_out = Sd;
  if (!(Sd > 0.0)) return 1e30;
  return 2.0 * (double)n * M / (Sd * Sd);
}

/* exact b_k rounded once, for one k (used by tests of the GPU certifier) */
SO_EXPORT double so_exact_bk(const double* a, int n, int k) {
  xacc cur, neg;
  exact_bk(a, n, k, &cur, &neg);
  xacc_sub(&cur, &neg);
  return xacc_to_double(&cur);
}

SO_EXPORT int so_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}


/* ========================= variation + support signature ================= */
/* Test oracle for csrc/variation.cu, which follows the operator semantics of
 * src/kernels.cuh:558-849 with its own random streams.  Philox4x32-10 is the
 * published counter-based generator (Salmon, Moraes, Dror, Shaw, SC 2011);
 * the known-answer vectors of its authors pin this restatement. */
SO_EXPORT void so_philox4x32(const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3], k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0, n1 = (uint32_t)p1;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1, n3 = (uint32_t)p0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}
static float var_u01(uint32_t w) { return ((float)(w >> 8) + 0.5f) * (1.0f / 16777216.0f); }
static void var_params(unsigned long long seed, unsigned long long gen, int j, float* u) {
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  for (int q = 0; q < 16; ++q) {
    const uint32_t c[4] = {(uint32_t)q, (uint32_t)j, (uint32_t)gen, (uint32_t)(gen >> 32) << 1};
    uint32_t r[4];
    so_philox4x32(c, key, r);
    for (int t = 0; t < 4; ++t) u[4 * q + t] = var_u01(r[t]);
  }
}
static float var_normal(unsigned long long seed, unsigned long long gen, int j, int i) {
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  const uint32_t c[4] = {(uint32_t)i, (uint32_t)j, (uint32_t)gen,
                         ((uint32_t)(gen >> 32) << 1) | 1u};
  uint32_t r[4];
  so_philox4x32(c, key, r);
  const double a = (double)var_u01(r[0]), b = (double)var_u01(r[1]);
  return (float)(sqrt(-2.0 * log(a)) * cos(6.283185307179586 * b));
}
/* the kernels' fixed-order fp64 block sum: 256 strided partial sums, a
 * 32-lane xor butterfly per warp (lane 0's value), warps added in order */
static double var_sum(const double* x, int n, int stride) {
  double part[256];
  for (int t = 0; t < 256; ++t) {
    double s = 0.0;
    for (int i = t; i < n; i += 256) s += x[(size_t)i * stride];
    part[t] = s;
  }
  double r = 0.0;
  for (int w = 0; w < 8; ++w) {
    double v[32], nv[32];
    for (int l = 0; l < 32; ++l) v[l] = part[32 * w + l];
    for (int off = 16; off > 0; off >>= 1) {
      for (int l = 0; l < 32; ++l) nv[l] = v[l] + v[l ^ off];
      memcpy(v, nv, sizeof v);
    }
    r += v[0];
  }
  return r;
}
static double var_mean_f32(const float* A, int n) {
  double* x = (double*)malloc(sizeof(double) * (size_t)n);
  for (int i = 0; i < n; ++i) x[i] = (double)A[i];
  const double m = var_sum(x, n, 1) / (double)n;
  free(x);
  return m;
}
SO_EXPORT void so_variation_f32(const float* pop, float* out, int n, int n_off, const int* p1,
                                const int* p2, const int* opv, const float* strength,
                                unsigned long long seed, unsigned long long gen) {
  float u[64];
  const float fn = (float)n;
  for (int j = 0; j < n_off; ++j) {
    const float* A = pop + (size_t)p1[j] * n;
    const float* B = pop + (size_t)p2[j] * n;
    float* O = out + (size_t)j * n;
    const float sg = strength[j];
    var_params(seed, gen, j, u);
    switch (opv[j]) {
      case 0: {
        const float lam = -0.3f + 1.6f * u[0];
        for (int i = 0; i < n; ++i) { const float x = lam * A[i] + (1.f - lam) * B[i]; O[i] = x > 0.f ? x : 0.f; }
        break;
      }
      case 1: {
        int c1 = (int)(u[1] * fn), c2 = (int)(u[2] * fn);
        if (c1 > c2) { const int t = c1; c1 = c2; c2 = t; }
        for (int i = 0; i < n; ++i) O[i] = (i >= c1 && i < c2) ? B[i] : A[i];
        break;
      }
      case 2:
        for (int i = 0; i < n; ++i) O[i] = A[i] * expf(sg * var_normal(seed, gen, j, i));
        break;
      case 3: {
        const int nf = 1 + (int)(u[3] * 5.0f);
        for (int i = 0; i < n; ++i) {
          float m = 0.f;
          for (int f = 0; f < nf; ++f) {
            const float freq = 1.0f + u[4 + f] * 12.0f, ph = 6.2831853f * u[12 + f];
            m += cosf(6.2831853f * freq * (float)i / fn + ph) / (float)nf;
          }
          const float x = A[i] * (1.0f + sg * 3.0f * m);
          O[i] = x > 0.f ? x : 0.f;
        }
        break;
      }
      case 4: {
        const float mean = (float)var_mean_f32(A, n);
        for (int i = 0; i < n; ++i) {
          const float x = A[i] + sg * mean * var_normal(seed, gen, j, i);
          O[i] = x > 0.f ? x : 0.f;
        }
        break;
      }
      case 5: {
        const float mean = (float)var_mean_f32(A, n);
        const float thr = mean * (0.05f + 0.9f * u[20]);
        for (int i = 0; i < n; ++i) O[i] = A[i] < thr ? 0.f : A[i];
        break;
      }
      case 6: {
        const int hard = u[21] < 0.5f;
        for (int i = 0; i < n; ++i) O[i] = hard ? A[n - 1 - i] : 0.5f * (A[i] + A[n - 1 - i]);
        break;
      }
      case 7: {
        const int sh = (int)((u[22] - 0.5f) * fn * 0.25f);
        for (int i = 0; i < n; ++i) { const int k = i - sh; O[i] = (k >= 0 && k < n) ? A[k] : 0.f; }
        break;
      }
      case 8: {
        const int len = 1 + (int)(u[23] * 0.5f * fn);
        const int st0 = (int)(u[24] * (float)(n - len > 0 ? n - len : 1));
        for (int i = 0; i < n; ++i) O[i] = (i >= st0 && i < st0 + len) ? B[i] : A[i];
        break;
      }
      case 9: {
        const int nf = 2 + (int)(u[25] * 6.0f);
        const float base = 0.3f + 0.7f * u[26];
        for (int i = 0; i < n; ++i) {
          float m = 0.f;
          for (int f = 0; f < nf; ++f) {
            const float freq = 1.0f + u[4 + (f % 8)] * 10.0f, ph = 6.2831853f * u[12 + (f % 8)];
            m += cosf(6.2831853f * freq * (float)i / fn + ph);
          }
          const float val = base + m / (float)nf + 0.4f * var_normal(seed, gen, j, i);
          O[i] = val > 0.f ? val : 0.f;
        }
        break;
      }
      case 10: {
        const int loc = (int)(u[27] * fn), wdt = 1 + (int)(u[28] * fn * 0.03f);
        const float mean = (float)var_mean_f32(A, n);
        const float amp = mean * (1.0f + 6.0f * u[29]);
        for (int i = 0; i < n; ++i) { float x = A[i]; if (i >= loc - wdt && i <= loc + wdt) x += amp; O[i] = x; }
        break;
      }
      case 11: {
        const int flip = u[30] < 0.5f;
        const float atom = 30.f + 250.f * u[31];
        const float pl1 = 0.28f + 0.16f * u[32];
        const float pl2 = pl1 + 0.10f + 0.14f * u[33];
        const float hump = pl2 + 0.02f + 0.08f * u[34];
        const float gap0 = 0.70f + 0.16f * u[35];
        const float gap1 = gap0 + 0.05f + 0.15f * u[36];
        const float tail = 3.0f + 14.0f * u[37];
        const int nf = 3 + (int)(u[38] * 6.f);
        for (int i = 0; i < n; ++i) {
          const int d = flip ? (n - 1 - i) : i;
          const float x = ((float)d + 0.5f) / fn;
          float rough = 0.f;
          for (int f = 0; f < nf; ++f)
            rough += cosf(6.2831853f * (2.f + u[40 + f] * 40.f) * x + 6.2831853f * u[48 + f]);
          rough /= (float)nf;
          float v;
          if (x < pl1) v = 4.2f * (1.f + 0.45f * rough);
          else if (x < pl2) v = 0.7f * (1.f + 0.80f * rough);
          else if (x < hump) v = 5.2f * (1.f + 0.30f * rough);
          else if (x < gap0) v = 2.0f * (1.f + 0.70f * rough);
          else if (x < gap1) v = 0.f;
          else v = tail * (1.f + 0.20f * rough);
          if (d == 0) v += atom;
          else if (d < 4) v += atom * 0.10f / (float)d;
          O[i] = v > 0.f ? v : 0.f;
        }
        break;
      }
      case 12: {
        const float mean = (float)var_mean_f32(A, n);
        const int len = 1 + (int)((0.015f + 0.13f * u[30]) * fn);
        const int st0 = (int)(u[31] * (float)(n > len ? n - len : 1));
        const int carve = u[32] < 0.7f;
        const float fill = mean * (0.2f + 1.8f * u[33]);
        for (int i = 0; i < n; ++i) {
          float x = A[i];
          if (i >= st0 && i < st0 + len) x = carve ? 0.f : (x + fill);
          O[i] = x;
        }
        break;
      }
      case 13: {
        const float mean = (float)var_mean_f32(A, n);
        const int left = u[30] < 0.5f;
        const int w = 1 + (int)(u[31] * 0.012f * fn);
        const float add = mean * (-20.f + 260.f * u[32]);
        for (int i = 0; i < n; ++i) {
          const int d = left ? i : (n - 1 - i);
          float x = A[i];
          if (d < w) { x += add / (float)(1 + d); if (x < 0.f) x = 0.f; }
          O[i] = x;
        }
        break;
      }
      default:
        for (int i = 0; i < n; ++i) O[i] = A[i];
        break;
    }
    double* x = (double*)malloc(sizeof(double) * (size_t)n);
    for (int i = 0; i < n; ++i) x[i] = (double)O[i];
    const double S = var_sum(x, n, 1);
    free(x);
    if (S > 0.0) {
      const float inv = (float)(1.0 / S);
      for (int i = 0; i < n; ++i) O[i] *= inv;
    } else {
      for (int i = 0; i < n; ++i) O[i] = 1.f / (float)n;
    }
  }
}
SO_EXPORT void so_support_sig_f32(const float* pop, int n, int P, float tol,
                                  unsigned long long* sig, int* nnz) {
  for (int p = 0; p < P; ++p) {
    const float* a = pop + (size_t)p * n;
    const double thr = var_mean_f32(a, n) * (double)tol;
    unsigned long long h = 0ull;
    int c = 0;
    for (int i = 0; i < n; ++i)
      if ((double)a[i] > thr) {
        ++c;
        unsigned long long x = (unsigned long long)i * 0x9E3779B97F4A7C15ull;
        x ^= x >> 29; x *= 0xBF58476D1CE4E5B9ull; x ^= x >> 32;
        h ^= x;
      }
    sig[p] = h;
    nnz[p] = c;
  }
}


/* ========================= memetic generation policy ===================== */
/* Test oracle for csrc/generation.cu: the selection policy of the reference
 * driver's generation loop (src/main.cu:586-785) restated sequentially, in
 * the reference's loop order and fp64 expressions, with the generation
 * kernels' Philox draws in place of the driver's mt19937_64.  The tabu map
 * is a plain list (key, best F, revisits); state is struct
 * sidon_generation_state of include/sidon_b200.h. */
#include "../include/sidon_b200.h"

#define GEN_NOPS 14

/* main.cu:466-467 */
SO_EXPORT void so_gen_init(sidon_generation_state* s) {
  memset(s, 0, sizeof *s);
  s->best_F = 1e30;
  s->level_best_F = 1e30;
  for (int o = 0; o < GEN_NOPS; ++o) s->op_weight[o] = 1.0;
  s->op_weight[11] = 2.5; s->op_weight[12] = 1.8; s->op_weight[13] = 1.8;
}

/* main.cu:566-585: operator record of the seeds, mirror descent on every
 * fourth island, per-level counters */
SO_EXPORT void so_gen_begin(sidon_generation_state* s, int* cur_op, int* mode, int P, int PI,
                            int n, int level, const int* seed_op) {
  for (int p = 0; p < P; ++p) {
    cur_op[p] = seed_op ? seed_op[p] : 9;
    mode[p] = ((p / PI) % 4 == 3) ? 1 : 0;
  }
  s->gen = 0; s->level = level; s->n = n; s->since_improve = 0;
  s->level_best_F = 1e30; s->improved = 0;
}

/* main.cu:606-629: tiers and their effort counters; skip is [3][P] */
SO_EXPORT void so_gen_tiers(sidon_generation_state* s, const int* cur_op, int P, int n,
                            int cold_iters, int med_iters, int warm_iters, int* skip) {
  const double n2 = (double)n * (double)n;
  int cold_cap = (int)(0.18 * P); if (cold_cap < 1) cold_cap = 1;
  int nc = 0, cnt[3] = {0, 0, 0};
  for (int p = 0; p < P; ++p) {
    const int o = cur_op[p];
    int t = 2;
    if ((o == 9 || o == 11) && nc < cold_cap) { t = 0; ++nc; }
    else if (o == 9 || o == 11 || o == 10 || o == 5 || o == 7 || o == 8 || o == 12 || o == 13)
      t = 1;
    for (int k = 0; k < 3; ++k) skip[k * P + p] = t == k ? 0 : 1;
    ++cnt[t];
  }
  const int iters[3] = {cold_iters, med_iters, warm_iters};
  s->n_cold = cnt[0]; s->n_med = cnt[1];
  for (int t = 0; t < 3; ++t)
    if (cnt[t] > 0) {
      s->ls_steps += (long long)cnt[t] * iters[t];
      s->flop += 4.0 * n2 * (double)cnt[t] * (double)iters[t];
    }
}

static int gen_before(double fa, int a, double fb, int b) {
  const int na = fa != fa, nb = fb != fb;
  if (na != nb) return nb;
  if (!na && fa != fb) return fa < fb;
  return a < b;
}
static int gen_pos(double u, int m) { const int k = (int)(u * (double)m); return k < m - 1 ? k : m - 1; }
static double gen_u53(uint32_t hi, uint32_t lo) {
  return ((double)(hi >> 5) * 67108864.0 + (double)(lo >> 6)) * (1.0 / 9007199254740992.0);
}
static int gen_find(const unsigned long long* key, int cnt, unsigned long long k) {
  for (int i = 0; i < cnt; ++i) if (key[i] == k) return i;
  return -1;
}

/* main.cu:641-730: incumbent, level best, tabu list, island ranking,
 * migration every 12 generations, offspring plan.  fit / nact / nnz are the
 * evaluation's, sig is updated by the migration, parent_fit receives the
 * migrated fitness.  The tabu list has room for tcap entries (*tcount
 * used); a full list sets status SIDON_ERR_CAPACITY. */
SO_EXPORT void so_gen_select(sidon_generation_state* s, float* pop, int n, int P, int NI,
                             int elite, int tenure, unsigned long long seed, int fw_ran,
                             int fw_rounds, int fw_iters, const double* fit, const int* nact,
                             unsigned long long* sig, const int* nnz, double* parent_fit,
                             int* rank, int* p1, int* p2, int* op, float* strength,
                             float* best_row, unsigned long long* tkey, double* tbest,
                             int* thits, int* tcount, int tcap, unsigned long long* var_gen) {
  const int PI = P / NI, gen = s->gen;
  const double n2 = (double)n * (double)n;
  int bi = 0;
  for (int p = 1; p < P; ++p) if (fit[p] < fit[bi]) bi = p;
  const int impr = fit[bi] < s->best_F - 1e-13;
  if (impr) {
    s->best_F = fit[bi]; s->best_n = n;
    memcpy(best_row, pop + (size_t)bi * n, sizeof(float) * (size_t)n);
  }
  if (fit[bi] < s->level_best_F - 1e-13) { s->level_best_F = fit[bi]; s->since_improve = 0; }
  else s->since_improve += 1;
  s->best_slot = bi; s->improved = impr;
  s->best_nactive = nact[bi]; s->best_nnz = nnz[bi];
  if (fw_ran) {
    s->fw_steps += (long long)fw_rounds * P;
    s->flop += (double)P * (double)fw_rounds * (4.0 * n2 * (double)fw_iters + 2.0 * n2 * 13.0);
  }
  s->evals += P;
  s->flop += 2.0 * n2 * (double)P;
  *var_gen = (unsigned long long)(gen + 1000 * s->level);

  /* tabu (main.cu:653-661) */
  for (int p = 0; p < P; ++p) {
    int e = gen_find(tkey, *tcount, sig[p]);
    if (e < 0) {
      if (*tcount >= tcap) { if (s->status == 0) s->status = SIDON_ERR_CAPACITY; continue; }
      e = (*tcount)++;
      tkey[e] = sig[p]; tbest[e] = fit[p]; thits[e] = 0;
      s->cells += 1;
    } else if (fit[p] < tbest[e] - 1e-12) {
      tbest[e] = fit[p]; thits[e] = 0;
    } else {
      thits[e] += 1;
    }
  }

  /* rank inside each island: insertion sort, ascending F, NaN last, ties by slot */
  for (int i = 0; i < NI; ++i) {
    int* L = rank + i * PI;
    for (int r = 0; r < PI; ++r) {
      const int p = i * PI + r;
      int k = r;
      while (k > 0 && gen_before(fit[p], p, fit[L[k - 1]], L[k - 1])) { L[k] = L[k - 1]; --k; }
      L[k] = p;
    }
  }
  for (int p = 0; p < P; ++p) parent_fit[p] = fit[p];

  /* migration (main.cu:672-680) */
  if (gen > 0 && gen % 12 == 0)
    for (int i = 0; i < NI; ++i) {
      const int src = rank[i * PI], dst = rank[((i + 1) % NI) * PI + PI - 1];
      memmove(pop + (size_t)dst * n, pop + (size_t)src * n, sizeof(float) * (size_t)n);
      parent_fit[dst] = parent_fit[src];
      sig[dst] = sig[src];
    }

  /* offspring plan (main.cu:682-730) */
  double warm = (double)gen / 40.0; if (warm > 1.0) warm = 1.0;
  double stagn = (double)s->since_improve / 25.0; if (stagn > 1.0) stagn = 1.0;
  double cum[GEN_NOPS], tot = 0.0, c = 0.0;
  for (int o = 0; o < GEN_NOPS; ++o) tot += s->op_weight[o];
  for (int o = 0; o < GEN_NOPS; ++o) { c += s->op_weight[o] / tot; cum[o] = c; }
  cum[GEN_NOPS - 1] = 1.0;
  const uint32_t key[2] = {(uint32_t)seed ^ 0x243F6A88u, (uint32_t)(seed >> 32) ^ 0x85A308D3u};
  static const int divers[7] = {5, 7, 9, 10, 8, 11, 12};
  for (int slot = 0; slot < P; ++slot) {
    const int i = slot / PI, r = slot - i * PI;
    const int* isl = rank + i * PI;
    if (r < elite) {
      p1[slot] = p2[slot] = isl[r]; op[slot] = 20; strength[slot] = 0.f;
      continue;
    }
    double u[8];
    for (int q = 0; q < 4; ++q) {
      const uint32_t ctr[4] = {(uint32_t)slot, (uint32_t)gen, (uint32_t)s->level, (uint32_t)q};
      uint32_t x[4];
      so_philox4x32(ctr, key, x);
      u[2 * q] = gen_u53(x[0], x[1]);
      u[2 * q + 1] = gen_u53(x[2], x[3]);
    }
    int a = isl[gen_pos(u[0], PI)], b = isl[gen_pos(u[1], PI)];
    const int pa = parent_fit[a] < parent_fit[b] ? a : b;
    a = isl[gen_pos(u[2], PI)]; b = isl[gen_pos(u[3], PI)];
    const int pb = parent_fit[a] < parent_fit[b] ? a : b;
    int o = 0;
    while (o < GEN_NOPS - 1 && cum[o] < u[4]) ++o;
    const int e = gen_find(tkey, *tcount, sig[pa]);
    const int hits = e >= 0 ? thits[e] : 0;
    const double cb = e >= 0 ? tbest[e] : 1e30;
    if (hits > tenure && cb > s->best_F * (1.0 + 2e-4)) o = divers[gen_pos(u[5], 7)];
    if (stagn > 0.7 && u[6] < 0.10) o = 9;
    p1[slot] = pa; p2[slot] = pb; op[slot] = o;
    strength[slot] = (float)((0.03 + 0.35 * u[7]) * (0.5 + warm) * (1.0 + 1.5 * stagn));
    s->op_use[o] += 1.0;
  }
}

/* main.cu:743-754: operator record, reinjection of the incumbent every 10th
 * generation over the worst slot of island 0 */
SO_EXPORT void so_gen_post(const sidon_generation_state* s, float* pop, int n, int P, int PI,
                           const int* op, int* cur_op, const int* rank, const float* best_row) {
  for (int p = 0; p < P; ++p) cur_op[p] = op[p];
  if (s->gen % 10 == 9 && s->best_n == n) {
    const int slot = rank[PI - 1];
    memcpy(pop + (size_t)slot * n, best_row, sizeof(float) * (size_t)n);
    cur_op[slot] = 20;
  }
}

/* main.cu:756-769: bandit credit every 5th generation; the counter */
SO_EXPORT void so_gen_credit(sidon_generation_state* s, int P, const int* op, const int* p1,
                             const double* child_fit, const double* parent_fit) {
  const int gen = s->gen;
  if (gen > 0 && gen % 5 == 0) {
    for (int p = 0; p < P; ++p)
      if (op[p] >= 0 && op[p] < GEN_NOPS && child_fit[p] < parent_fit[p1[p]]) s->op_win[op[p]] += 1.0;
    for (int o = 0; o < GEN_NOPS; ++o) {
      const double rate = s->op_use[o] > 20 ? s->op_win[o] / s->op_use[o] : 0.25;
      double x = 0.85 * s->op_weight[o] + 0.15 * (0.15 + 3.0 * rate);
      x = x < 4.0 ? x : 4.0;
      x = x > 0.05 ? x : 0.05;
      s->op_weight[o] = x;
    }
    for (int o = 0; o < GEN_NOPS; ++o) { s->op_use[o] *= 0.7; s->op_win[o] *= 0.7; }
  }
  s->gen = gen + 1;
}
