// ---------------------------------------------------------------------------
//  big_tc.cu -- the tensor-core local search and Frank-Wolfe step for
//  candidates too long for one CTA (n up to 65536 and beyond).
//
//  Super-block decomposition.  The heights are cut into R super-blocks
//  s_0 .. s_(R-1) of Q cells (Q a multiple of 64 that one CTA handles,
//  e.g. 8192; the last one zero-padded).  Then
//      a * y     = sum_(I,J) shift_((I+J) Q) (s_I * y_J)
//      corr(c,a) restricted to outputs in super-block I' =
//                  sum_J corr(c[(I'+J) Q, (I'+J+2) Q - 1), s_J)
//  and each term is one job for the single-CTA tile engine (tc_engine.cuh):
//  a symmetric pair (I == J of a * a) is CONV_SYM, a pair I < J of a * a is
//  CONV_X counted twice, a pair of a * y (y != a) is CONV_X, a correlation
//  job is CORR with the weight segment as B.  Every job writes its outputs
//  to its own slot of a workspace; elementwise kernels then add the slots of
//  each output in a fixed order (deterministic) and apply the step's
//  epilogue (max, L^p weights, Adam / mirror update, renormalisation, or the
//  Chambolle-Pock dual / primal updates).
//
//  One local-search step = conv jobs -> reduce(b, max) -> weights ->
//  corr jobs -> update -> renormalise: six stream-ordered launches, no host
//  synchronisation.  The arithmetic of every step matches the fused kernel
//  of search_tc.cu (p, lr, bias corrections, update order), but b and G are
//  summed over super-blocks in another order, so results are not bitwise
//  those of the single-CTA kernel.
// ---------------------------------------------------------------------------
#include "tc_cta.cuh"

namespace sidon {
namespace big {
using namespace tc;

constexpr int NCH = 64;           // elementwise chunks per candidate
constexpr int ETHREADS = 256;

__host__ __device__ __forceinline__ int njobs_conv(int R, bool sym) {
  return sym ? R * (R + 1) / 2 : R * R;
}
__host__ __device__ __forceinline__ int pair_id(int I, int J, int R, bool sym) {
  return sym ? I * R - I * (I - 1) / 2 + (J - I) : I * R + J;
}
__device__ __forceinline__ void pair_of(int j, int R, bool sym, int& I, int& J) {
  if (!sym) {
    I = j / R;
    J = j % R;
    return;
  }
  I = 0;
  while (j >= R - I) {
    j -= R - I;
    ++I;
  }
  J = I + j;
}

// ------------------------------- tile jobs --------------------------------
// Convolution jobs of x * y (sym: y == x, pairs I <= J) for every candidate
// whose flag is 0.  out: [P][njobs][2Q], job outputs at local k < 2Q - 1.
__global__ void __launch_bounds__(NTHREADS, 1)
k_conv_jobs(const float* x, const float* y, int n, int Q, int R, int P, int sym,
            const int* __restrict__ flags, float* __restrict__ out, int three,
            unsigned int* status) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  Shared S = setup(Q, three != 0, smem_raw);
  Ctx& C = S.C;
  const Lane ln;
  float* X = reinterpret_cast<float*>(C.bc);
  const int NJ = njobs_conv(R, sym != 0);
  const long long total = (long long)P * NJ;
  for (long long slot = blockIdx.x; slot < total; slot += gridDim.x) {
    const int p = (int)(slot / NJ), j = (int)(slot % NJ);
    if (flags[p]) continue;
    int I, J;
    pair_of(j, R, sym != 0, I, J);
    const int lenI = min(Q, n - I * Q), lenJ = min(Q, n - J * Q);
    const float* xr = x + (size_t)p * n + (size_t)I * Q;
    begin(S, Q, Q);
    for (int i = threadIdx.x; i < lenI; i += blockDim.x) S.sa[pidx(i)] = xr[i];
    __syncthreads();
    prime(C, false);
    const bool ok = (sym && I == J)
                        ? conv_tc(C, S.sa, status)
                        : convx_tc(C, S.sa, y + (size_t)p * n + (size_t)J * Q, lenJ, status);
    if (!ok) break;
    gather_conv(C, ln, X);
    const float sc = (sym && I != J) ? 2.f : 1.f;
    float* o = out + (size_t)slot * (2 * Q);
    for (int k = threadIdx.x; k < 2 * Q - 1; k += blockDim.x) o[k] = sc * X[pidx(k)];
  }
  teardown(S);
}

// Correlation jobs: out[p][I'][J][i] = sum_j c[p][(I'+J) Q + i + j] s_J[j],
// i < Q.  c: [P][L] weights (L = 2 R Q, zero beyond 2n - 1).
__global__ void __launch_bounds__(NTHREADS, 1)
k_corr_jobs(const float* a, const float* c, int n, int Q, int R, int P,
            const int* __restrict__ flags, float* __restrict__ out, int three,
            unsigned int* status) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  Shared S = setup(Q, three != 0, smem_raw);
  Ctx& C = S.C;
  const Lane ln;
  float* X = reinterpret_cast<float*>(C.bc);
  const int NJ = R * R;
  const long long L = 2ll * R * Q;
  const long long total = (long long)P * NJ;
  for (long long slot = blockIdx.x; slot < total; slot += gridDim.x) {
    const int p = (int)(slot / NJ), j = (int)(slot % NJ);
    if (flags[p]) continue;
    const int Io = j / R, J = j % R;
    const int lenJ = min(Q, n - J * Q);
    const float* ar = a + (size_t)p * n + (size_t)J * Q;
    const float* cs = c + (size_t)p * L + (size_t)(Io + J) * Q;
    begin(S, Q, Q);
    for (int i = threadIdx.x; i < lenJ; i += blockDim.x) S.sa[pidx(i)] = ar[i];
    for (int t = threadIdx.x; t < 2 * Q - 1; t += blockDim.x) S.cb[pidx(t)] = cs[t];
    __syncthreads();
    prime(C, true);
    if (!corr_tc(C, S.sa, S.cb, status)) break;
    gather_corr(C, ln, X);
    float* o = out + (size_t)slot * Q;
    for (int i = threadIdx.x; i < Q; i += blockDim.x) o[i] = X[pidx(i)];
  }
  teardown(S);
}

// ---------------------------- elementwise steps ----------------------------
__device__ __forceinline__ void chunk_range(long long len, int ch, long long& k0, long long& k1) {
  const long long per = (len + NCH - 1) / NCH;
  k0 = (long long)ch * per;
  k1 = k0 + per < len ? k0 + per : len;
}

// b_k (k < L; zero for k >= 2n - 1) = sum of the pair outputs, pairs with
// I + J = K - 1 then I + J = K (K = k / Q), I ascending.  epi 0: store b and
// the chunk maximum; epi 1 (Chambolle-Pock dual step): lam_k <-
// [lam_k + sigma (b_k - M)]_+ with M = pM[p].
__global__ void __launch_bounds__(ETHREADS)
k_reduce_conv(const float* __restrict__ jobs, int n, int Q, int R, int P, int sym,
              const int* __restrict__ flags, float* __restrict__ b, float* __restrict__ pmax,
              int epi, const float* __restrict__ pM, float sigma) {
  __shared__ float red[32];
  const int p = blockIdx.y, ch = blockIdx.x;
  if (flags[p]) return;
  const int NJ = njobs_conv(R, sym != 0);
  const long long L = 2ll * R * Q;
  const int nb = 2 * n - 1;
  long long k0, k1;
  chunk_range(L, ch, k0, k1);
  const float* jp = jobs + (size_t)p * NJ * 2 * Q;
  float* bp = b + (size_t)p * L;
  const float M = epi == 1 ? pM[p] : 0.f;
  float mloc = 0.f;
  for (long long kk = k0 + threadIdx.x; kk < k1; kk += blockDim.x) {
    const int k = (int)kk;
    float v = 0.f;
    if (k < nb) {
      const int K = k / Q;
      for (int t = K - 1; t <= K; ++t) {
        if (t < 0 || t > 2 * R - 2) continue;
        const int loc = k - t * Q;
        if (loc > 2 * Q - 2) continue;
        const int Ilo = t - (R - 1) > 0 ? t - (R - 1) : 0;
        const int Ihi = sym ? t / 2 : (t < R - 1 ? t : R - 1);
        for (int I = Ilo; I <= Ihi; ++I)
          v += jp[(size_t)pair_id(I, t - I, R, sym != 0) * 2 * Q + loc];
      }
    }
    if (epi == 0) {
      bp[k] = v;
      mloc = fmaxf(mloc, v);
    } else if (k < nb) {
      const float l = bp[k] + sigma * (v - M);
      bp[k] = l > 0.f ? l : 0.f;
    }
  }
  if (epi == 0) {
    mloc = block_max(mloc, red);
    if (threadIdx.x == 0) pmax[(size_t)p * NCH + ch] = mloc;
  }
}

// the candidate's M from the chunk maxima (fixed order)
__device__ __forceinline__ float cand_max(const float* pmax, int p) {
  float M = 0.f;
  for (int c = 0; c < NCH; ++c) M = fmaxf(M, pmax[(size_t)p * NCH + c]);
  return M;
}

// c_k = (1+d)^(p-1), d = (b_k - M)/M, in place; chunk sums of c_k (1+d).
// M <= 0 stops the candidate's anneal (flag 2), as the fused kernel breaks.
__global__ void __launch_bounds__(ETHREADS)
k_weights(float* __restrict__ cb, const float* __restrict__ pmax, int n, int Q, int R, int P,
          int* __restrict__ flags, int it, int iters, float pStart, float pEnd,
          float* __restrict__ pM, float* __restrict__ pR) {
  __shared__ float red[32];
  const int p = blockIdx.y, ch = blockIdx.x;
  if (flags[p]) return;
  const float M = cand_max(pmax, p);
  if (!(M > 0.f)) {
    if (ch == 0 && threadIdx.x == 0) flags[p] = 2;
    return;
  }
  const float lnPr = (float)log((double)pEnd / (double)pStart);
  const float frac = iters > 1 ? (float)it / (float)(iters - 1) : 0.f;
  const float pexp = pStart * expf(lnPr * frac);
  const float invM = 1.f / M, q = pexp - 1.f;
  const int nb = 2 * n - 1;
  long long k0, k1;
  chunk_range(nb, ch, k0, k1);
  float* c = cb + (size_t)p * 2 * R * Q;
  float rloc = 0.f;
  for (long long k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
    const float d = (c[k] - M) * invM;
    const float cw = d > -1.f ? pow_from_d_fast(d, q) : 0.f;
    rloc += cw * (1.f + d);
    c[k] = cw;
  }
  rloc = block_sum(rloc, red);
  if (threadIdx.x == 0) {
    pR[(size_t)p * NCH + ch] = rloc;
    if (ch == 0) pM[p] = M;
  }
}

// G_i = sum_J jobs[p][I'][J][i - I' Q]; Adam / mirror step of the fused
// kernel; chunk sums of the new heights.
__global__ void __launch_bounds__(ETHREADS)
k_update(float* __restrict__ pop, float* __restrict__ mom, float* __restrict__ vel,
         const float* __restrict__ gjobs, const float* __restrict__ pM,
         const float* __restrict__ pR, int n, int Q, int R, int P, const int* __restrict__ flags,
         const int* __restrict__ mode_arr, int mode_default, int it, int iters, float lrStart,
         float lrEnd, float beta1, float beta2, const float* __restrict__ bstate,
         float* __restrict__ pS) {
  __shared__ float red[32];
  const int p = blockIdx.y, ch = blockIdx.x;
  if (flags[p]) return;
  float Rs = 0.f;
  for (int c = 0; c < NCH; ++c) Rs += pR[(size_t)p * NCH + c];
  const float M = pM[p];
  const int mode = mode_arr ? mode_arr[p] : mode_default;
  const float lnLr = (float)log((double)lrEnd / (double)lrStart);
  const float frac = iters > 1 ? (float)it / (float)(iters - 1) : 0.f;
  const float lr = lrStart * expf(lnLr * frac);
  const float b1t = bstate[0] * beta1, b2t = bstate[1] * beta2;
  const float bc1 = 1.f / (1.f - b1t), bc2 = 1.f / (1.f - b2t);
  const float lrn = lr / (float)n;
  const float invR = 1.f / Rs, invM = 1.f / M;
  long long i0, i1;
  chunk_range(n, ch, i0, i1);
  float* a = pop + (size_t)p * n;
  float* mg = mom + (size_t)p * n;
  float* vg = vel + (size_t)p * n;
  const float* gj = gjobs + (size_t)p * R * R * Q;
  float sloc = 0.f;
  for (long long ii = i0 + threadIdx.x; ii < i1; ii += blockDim.x) {
    const int i = (int)ii;
    const int Io = i / Q, il = i - Io * Q;
    float G = 0.f;
    for (int J = 0; J < R; ++J) G += gj[((size_t)Io * R + J) * Q + il];
    const float gi = G * invR - M;
    float x;
    if (mode == 0) {
      const float mm = __fmaf_rn(beta1, mg[i], (1.f - beta1) * gi);
      const float vv = __fmaf_rn(beta2, vg[i], (1.f - beta2) * gi * gi);
      mg[i] = mm;
      vg[i] = vv;
      const float step = lrn * (mm * bc1) / (sqrtf(vv * bc2) + 1e-30f);
      x = a[i] - step;
      if (x < 0.f) x = 0.f;
    } else {
      float e = -lr * (gi * invM);
      if (e > 4.f) e = 4.f;
      if (e < -4.f) e = -4.f;
      x = a[i] * __expf(e);
    }
    a[i] = x;
    sloc += x;
  }
  sloc = block_sum(sloc, red);
  if (threadIdx.x == 0) pS[(size_t)p * NCH + ch] = sloc;
}

// a <- a / S (S <= 0: the uniform 1/n), S from the chunk sums; advances the
// bias-correction powers once per step.
__global__ void __launch_bounds__(ETHREADS)
k_renorm(float* __restrict__ pop, const float* __restrict__ pS, int n, int P,
         const int* __restrict__ flags, float* __restrict__ bstate, float beta1, float beta2) {
  const int p = blockIdx.y, ch = blockIdx.x;
  if (p == 0 && ch == 0 && threadIdx.x == 0) {
    bstate[0] *= beta1;
    bstate[1] *= beta2;
  }
  if (flags[p]) return;
  float S = 0.f;
  for (int c = 0; c < NCH; ++c) S += pS[(size_t)p * NCH + c];
  const bool reset = !(S > 0.f);
  const float inv = 1.f / (reset ? 1.f : S);
  long long i0, i1;
  chunk_range(n, ch, i0, i1);
  float* a = pop + (size_t)p * n;
  for (long long i = i0 + threadIdx.x; i < i1; i += blockDim.x)
    a[i] = (reset ? 1.f / (float)n : a[i]) * inv;
}

__global__ void k_ls_init(const int* __restrict__ skip, int n, int P, int* __restrict__ flags,
                          float* __restrict__ bstate, float* __restrict__ mom,
                          float* __restrict__ vel) {
  const long long total = (long long)P * n;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int p = (int)(t / n);
    if (skip && skip[p]) continue;
    mom[t] = 0.f;
    vel[t] = 0.f;
  }
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x)
    flags[p] = (skip && skip[p]) ? 1 : 0;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    bstate[0] = 1.f;
    bstate[1] = 1.f;
  }
}

// ------------------------------ Frank-Wolfe -------------------------------
// Candidate flags: 0 running, 1 skipped, 2 stopped (a sum or M <= 0, as the
// fused kernel returns / breaks), 3 no improving line-search point.

// chunk sums of a row set (sum a, sum g)
__global__ void __launch_bounds__(ETHREADS)
k_chunk_sum(const float* __restrict__ v, int n, int P, const int* __restrict__ flags,
            float* __restrict__ part) {
  __shared__ float red[32];
  const int p = blockIdx.y, ch = blockIdx.x;
  if (flags[p]) return;
  long long i0, i1;
  chunk_range(n, ch, i0, i1);
  float s = 0.f;
  for (long long i = i0 + threadIdx.x; i < i1; i += blockDim.x) s += v[(size_t)p * n + i];
  s = block_sum(s, red);
  if (threadIdx.x == 0) part[(size_t)p * NCH + ch] = s;
}

// v <- v / sum v from the chunk sums; sum <= 0 stops the candidate
__global__ void __launch_bounds__(ETHREADS)
k_scale_by_sum(float* __restrict__ v, const float* __restrict__ part, int n, int P,
               int* __restrict__ flags) {
  const int p = blockIdx.y, ch = blockIdx.x;
  if (flags[p]) return;
  float s = 0.f;
  for (int c = 0; c < NCH; ++c) s += part[(size_t)p * NCH + c];
  if (!(s > 0.f)) {
    if (ch == 0 && threadIdx.x == 0) flags[p] = 2;
    return;
  }
  const float inv = 1.f / s;
  long long i0, i1;
  chunk_range(n, ch, i0, i1);
  for (long long i = i0 + threadIdx.x; i < i1; i += blockDim.x) v[(size_t)p * n + i] *= inv;
}

// round start: M = the refined max (M <= 0 stops), g = gbar = a0 = a,
// lam = 0
__global__ void __launch_bounds__(ETHREADS)
k_fw_round(const float* __restrict__ a, float* __restrict__ g, float* __restrict__ gb,
           float* __restrict__ a0, float* __restrict__ lam, const double* __restrict__ best,
           float* __restrict__ pM, int n, int Q, int R, int P, int* __restrict__ flags) {
  const int p = blockIdx.y, ch = blockIdx.x;
  if (flags[p]) return;
  const float M = (float)best[p];
  if (!(M > 0.f)) {
    if (ch == 0 && threadIdx.x == 0) flags[p] = 2;
    return;
  }
  if (ch == 0 && threadIdx.x == 0) pM[p] = M;
  long long i0, i1;
  chunk_range(n, ch, i0, i1);
  const size_t o = (size_t)p * n;
  for (long long i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
    const float x = a[o + i];
    g[o + i] = x;
    gb[o + i] = x;
    a0[o + i] = x;
  }
  const long long L = 2ll * R * Q;
  long long k0, k1;
  chunk_range(L, ch, k0, k1);
  for (long long k = k0 + threadIdx.x; k < k1; k += blockDim.x) lam[(size_t)p * L + k] = 0.f;
}

// primal step: G_i from the correlation jobs, g <- [g + tau (1 - G)]_+,
// gbar = 2 g_new - g_old
__global__ void __launch_bounds__(ETHREADS)
k_fw_primal(float* __restrict__ g, float* __restrict__ gb, const float* __restrict__ gjobs, int n,
            int Q, int R, int P, const int* __restrict__ flags, float tau) {
  const int p = blockIdx.y, ch = blockIdx.x;
  if (flags[p]) return;
  long long i0, i1;
  chunk_range(n, ch, i0, i1);
  const size_t o = (size_t)p * n;
  const float* gj = gjobs + (size_t)p * R * R * Q;
  for (long long ii = i0 + threadIdx.x; ii < i1; ii += blockDim.x) {
    const int i = (int)ii;
    const int Io = i / Q, il = i - Io * Q;
    float G = 0.f;
    for (int J = 0; J < R; ++J) G += gj[((size_t)Io * R + J) * Q + il];
    const float go = g[o + i];
    float gn = go + tau * (1.f - G);
    gn = gn > 0.f ? gn : 0.f;
    g[o + i] = gn;
    gb[o + i] = 2.f * gn - go;
  }
}

// h = (1 - t) a0 + t g into `a` (the line-search point, or the move)
__global__ void __launch_bounds__(ETHREADS)
k_fw_point(float* __restrict__ a, const float* __restrict__ a0, const float* __restrict__ g,
           int n, int P, const int* __restrict__ flags, const float* __restrict__ tsel,
           float t_fixed) {
  const int p = blockIdx.y, ch = blockIdx.x;
  if (flags[p]) return;
  const float t = tsel ? tsel[p] : t_fixed;
  long long i0, i1;
  chunk_range(n, ch, i0, i1);
  const size_t o = (size_t)p * n;
  for (long long i = i0 + threadIdx.x; i < i1; i += blockDim.x)
    a[o + i] = (1.f - t) * a0[o + i] + t * g[o + i];
}

// Refined max of b = h * h for one candidate per CTA: every k whose
// tensor-core b_k lies within `rel` of the approximate max is recomputed
// with fp64 accumulation (first `cap` such k in k order; beyond them the
// approximate max stands).  Then the line-search bookkeeping: s = 0 records
// the round's M (best = M, t = 0); s > 0 keeps t if the max is lower.
constexpr int kBigRefineCap = 256;
__global__ void __launch_bounds__(ETHREADS)
k_fw_refine(const float* __restrict__ h, const float* __restrict__ b,
            const float* __restrict__ pmax, int n, int Q, int R, int P,
            const int* __restrict__ flags, float rel, int s, float t,
            double* __restrict__ best, float* __restrict__ tsel) {
  __shared__ int list[kBigRefineCap];
  __shared__ int cnt;
  __shared__ double red[32];
  const int p = blockIdx.x;
  if (flags[p]) return;
  const float approx = cand_max(pmax, p);
  const long long L = 2ll * R * Q;
  const float* bp = b + (size_t)p * L;
  const float* hp = h + (size_t)p * n;
  const double m = refine_max(
      n, [&](int i) { return hp[i]; }, [&](int k) { return bp[k]; }, approx, rel, list,
      kBigRefineCap, &cnt, red);
  if (threadIdx.x == 0) {
    if (s == 0) {
      best[p] = m;
      tsel[p] = 0.f;
    } else if (m < best[p]) {
      best[p] = m;
      tsel[p] = t;
    }
  }
}

// after the line search: no improving t stops the candidate (a = a0)
__global__ void k_fw_accept(const float* __restrict__ tsel, int P, int* __restrict__ flags) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < P && !flags[p] && !(tsel[p] > 0.f)) flags[p] = 3;
}

__global__ void k_fw_init(const int* __restrict__ skip, int P, int* __restrict__ flags) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < P) flags[p] = (skip && skip[p]) ? 1 : 0;
}

}  // namespace big
}  // namespace sidon

// =========================== host drivers =================================
namespace sidon_host {
using namespace sidon;
unsigned int* tc_status_word();

namespace {

struct Work {
  float *jconv, *jcorr, *cbuf, *pmax, *pR, *pS, *pM, *bstate, *g, *gb, *a0, *tsel;
  double* best;
  int* flags;
  size_t bytes;
};

// carve the workspace of one call (256-byte aligned pieces)
Work carve(void* base, int n, int P, int Q) {
  const int R = (n + Q - 1) / Q;
  const size_t L = 2ull * R * Q;
  size_t o = 0;
  auto take = [&](size_t b) {
    const size_t at = o;
    o += (b + 255) & ~(size_t)255;
    return at;
  };
  Work w;
  unsigned char* c = reinterpret_cast<unsigned char*>(base);
  const size_t oj = take(sizeof(float) * (size_t)P * R * R * 2 * Q);
  const size_t oc = take(sizeof(float) * (size_t)P * R * R * Q);
  const size_t ob = take(sizeof(float) * (size_t)P * L);
  const size_t om = take(sizeof(float) * (size_t)P * big::NCH);
  const size_t orr = take(sizeof(float) * (size_t)P * big::NCH);
  const size_t os = take(sizeof(float) * (size_t)P * big::NCH);
  const size_t oM = take(sizeof(float) * (size_t)P);
  const size_t obs = take(sizeof(float) * 2);
  const size_t og = take(sizeof(float) * (size_t)P * n);
  const size_t ogb = take(sizeof(float) * (size_t)P * n);
  const size_t oa0 = take(sizeof(float) * (size_t)P * n);
  const size_t ot = take(sizeof(float) * (size_t)P);
  const size_t obe = take(sizeof(double) * (size_t)P);
  const size_t ofl = take(sizeof(int) * (size_t)P);
  w.bytes = o;
  if (c) {
    w.jconv = reinterpret_cast<float*>(c + oj);
    w.jcorr = reinterpret_cast<float*>(c + oc);
    w.cbuf = reinterpret_cast<float*>(c + ob);
    w.pmax = reinterpret_cast<float*>(c + om);
    w.pR = reinterpret_cast<float*>(c + orr);
    w.pS = reinterpret_cast<float*>(c + os);
    w.pM = reinterpret_cast<float*>(c + oM);
    w.bstate = reinterpret_cast<float*>(c + obs);
    w.g = reinterpret_cast<float*>(c + og);
    w.gb = reinterpret_cast<float*>(c + ogb);
    w.a0 = reinterpret_cast<float*>(c + oa0);
    w.tsel = reinterpret_cast<float*>(c + ot);
    w.best = reinterpret_cast<double*>(c + obe);
    w.flags = reinterpret_cast<int*>(c + ofl);
  }
  return w;
}

int job_grid(long long jobs) {
  const int sms = sm_count();
  return (int)(jobs < sms ? jobs : sms);
}

}  // namespace

int tc_n_ok_public(int n);
size_t smem_tc_plain(int n);

size_t big_workspace_bytes(int n, int P, int Q) {
  if (n < 1 || P < 0 || Q < 64 || Q % 64) return 0;
  return carve(nullptr, n, P, Q < n ? Q : n).bytes;
}

// the super-block size used when the caller passes 0: the largest multiple
// of 64 up to 8192 that the single-CTA engine accepts
int big_default_q(int n) {
  int q = 8192;
  while (q > 64 && tc_n_ok_public(q)) q -= 64;
  (void)n;
  return q;
}

static int big_prep(int Q) {
  int rc = tc_n_ok_public(Q);
  if (rc) return rc;
  const size_t sm = smem_tc_plain(Q);
  rc = set_dyn_smem((const void*)big::k_conv_jobs, sm);
  if (!rc) rc = set_dyn_smem((const void*)big::k_corr_jobs, sm);
  if (rc) return rc;
  return tc_status_word() ? SIDON_OK : SIDON_ERR_CUDA;
}

int launch_local_search_tc(float* pop, float* mom, float* vel, const long long* offsets,
                           const int* order, int P, int n_fixed, int n_max, const int* skip,
                           const int* mode_arr, int iters, double pS, double pE, double lrS,
                           double lrE, double b1, double b2, int mode_default, int precision,
                           unsigned int* seg_flags, cudaStream_t st);
bool fused_fits(int n);
int tuned_q(int n, int P, int precision);

// q <= 0: the tuned choice for (n, P, precision) if the tuner has run, else
// big_default_q; q >= n with n fitting one CTA: the fused kernel
int launch_local_search_big(float* pop, float* mom, float* vel, const int* skip,
                            const int* mode_arr, int n, int P, int iters, double pS, double pE,
                            double lrS, double lrE, double b1, double b2, int mode_default,
                            int precision, int Q, void* ws, size_t ws_bytes, cudaStream_t st) {
  if (Q <= 0) Q = tuned_q(n, P, precision);
  if (Q <= 0) Q = big_default_q(n);
  if (Q >= n && fused_fits(n))
    return launch_local_search_tc(pop, mom, vel, nullptr, nullptr, P, n, n, skip, mode_arr, iters,
                                  pS, pE, lrS, lrE, b1, b2, mode_default, precision, nullptr, st);
  if (Q % 64) return SIDON_ERR_ARG;
  int rc = big_prep(Q);
  if (rc) return rc;
  Work w = carve(ws, n, P, Q);
  if (!ws || ws_bytes < w.bytes) return SIDON_ERR_CAPACITY;
  const int R = (n + Q - 1) / Q;
  const int three = precision == SIDON_PREC_BF16X3 ? 1 : 0;
  unsigned int* sw = tc_status_word();
  const size_t sm = smem_tc_plain(Q);
  const dim3 eg_b(big::NCH, P), eg_n(big::NCH, P);
  big::k_ls_init<<<sm_count() * 4, 256, 0, st>>>(skip, n, P, w.flags, w.bstate, mom, vel);
  rc = check_launch();
  for (int it = 0; it < iters && !rc; ++it) {
    big::k_conv_jobs<<<job_grid((long long)P * big::njobs_conv(R, true)), tc::NTHREADS, sm, st>>>(
        pop, pop, n, Q, R, P, 1, w.flags, w.jconv, three, sw);
    big::k_reduce_conv<<<eg_b, big::ETHREADS, 0, st>>>(w.jconv, n, Q, R, P, 1, w.flags, w.cbuf,
                                                       w.pmax, 0, nullptr, 0.f);
    big::k_weights<<<eg_b, big::ETHREADS, 0, st>>>(w.cbuf, w.pmax, n, Q, R, P, w.flags, it, iters,
                                                   (float)pS, (float)pE, w.pM, w.pR);
    big::k_corr_jobs<<<job_grid((long long)P * R * R), tc::NTHREADS, sm, st>>>(
        pop, w.cbuf, n, Q, R, P, w.flags, w.jcorr, three, sw);
    big::k_update<<<eg_n, big::ETHREADS, 0, st>>>(pop, mom, vel, w.jcorr, w.pM, w.pR, n, Q, R, P,
                                                  w.flags, mode_arr, mode_default, it, iters,
                                                  (float)lrS, (float)lrE, (float)b1, (float)b2,
                                                  w.bstate, w.pS);
    big::k_renorm<<<eg_n, big::ETHREADS, 0, st>>>(pop, w.pS, n, P, w.flags, w.bstate, (float)b1,
                                                  (float)b2);
    rc = check_launch();
  }
  return rc;
}

int launch_frank_wolfe_tc(float* pop, float* gbuf, float* gbbuf, const long long* offsets,
                          const int* order, int P, int n_fixed, int n_max, const int* skip,
                          int rounds, int pdhg, int nT, float tMax, float tau, float sig,
                          int precision, cudaStream_t st);

// q as for the local search; the fused kernel takes its g / gbar rows from
// the workspace
int launch_frank_wolfe_big(float* pop, const int* skip, int n, int P, int rounds, int pdhg,
                           int nT, float tMax, float tau, float sig, int precision, int Q,
                           void* ws, size_t ws_bytes, cudaStream_t st) {
  if (Q <= 0) Q = tuned_q(n, P, precision);
  if (Q <= 0) Q = big_default_q(n);
  if (Q >= n && fused_fits(n)) {
    Work w = carve(ws, n, P, Q);
    if (!ws || ws_bytes < w.bytes) return SIDON_ERR_CAPACITY;
    return launch_frank_wolfe_tc(pop, w.g, w.gb, nullptr, nullptr, P, n, n, skip, rounds, pdhg,
                                 nT, tMax, tau, sig, precision, st);
  }
  if (Q % 64) return SIDON_ERR_ARG;
  int rc = big_prep(Q);
  if (rc) return rc;
  Work w = carve(ws, n, P, Q);
  if (!ws || ws_bytes < w.bytes) return SIDON_ERR_CAPACITY;
  const int R = (n + Q - 1) / Q;
  const int three = precision == SIDON_PREC_BF16X3 ? 1 : 0;
  unsigned int* sw = tc_status_word();
  const size_t sm = smem_tc_plain(Q);
  const dim3 eg(big::NCH, P);
  if (!(tau > 0.f)) tau = 0.9f / (float)n;
  if (!(sig > 0.f)) sig = 0.9f * (float)n;
  const int gsym = job_grid((long long)P * big::njobs_conv(R, true));
  const int gx = job_grid((long long)P * R * R);
  big::k_fw_init<<<(P + 127) / 128, 128, 0, st>>>(skip, P, w.flags);
  // normalise a
  big::k_chunk_sum<<<eg, big::ETHREADS, 0, st>>>(pop, n, P, w.flags, w.pS);
  big::k_scale_by_sum<<<eg, big::ETHREADS, 0, st>>>(pop, w.pS, n, P, w.flags);
  rc = check_launch();
  // a * a on the current point -> chunk maxima (b in cbuf)
  auto self_conv = [&](const float* h) {
    big::k_conv_jobs<<<gsym, tc::NTHREADS, sm, st>>>(h, h, n, Q, R, P, 1, w.flags, w.jconv, three,
                                                     sw);
    big::k_reduce_conv<<<eg, big::ETHREADS, 0, st>>>(w.jconv, n, Q, R, P, 1, w.flags, w.cbuf,
                                                     w.pmax, 0, nullptr, 0.f);
  };
  for (int r = 0; r < rounds && !rc; ++r) {
    self_conv(pop);
    big::k_fw_refine<<<P, big::ETHREADS, 0, st>>>(pop, w.cbuf, w.pmax, n, Q, R, P, w.flags, 2e-4f,
                                                  0, 0.f, w.best, w.tsel);
    big::k_fw_round<<<eg, big::ETHREADS, 0, st>>>(pop, w.g, w.gb, w.a0, w.cbuf, w.best, w.pM, n,
                                                  Q, R, P, w.flags);
    rc = check_launch();
    // lambda lives in cbuf from here on (zeroed by k_fw_round)
    for (int it = 0; it < pdhg && !rc; ++it) {
      big::k_conv_jobs<<<gx, tc::NTHREADS, sm, st>>>(pop, w.gb, n, Q, R, P, 0, w.flags, w.jconv,
                                                     three, sw);
      big::k_reduce_conv<<<eg, big::ETHREADS, 0, st>>>(w.jconv, n, Q, R, P, 0, w.flags, w.cbuf,
                                                       nullptr, 1, w.pM, sig);
      big::k_corr_jobs<<<gx, tc::NTHREADS, sm, st>>>(pop, w.cbuf, n, Q, R, P, w.flags, w.jcorr,
                                                     three, sw);
      big::k_fw_primal<<<eg, big::ETHREADS, 0, st>>>(w.g, w.gb, w.jcorr, n, Q, R, P, w.flags, tau);
      rc = check_launch();
    }
    if (rc) break;
    big::k_chunk_sum<<<eg, big::ETHREADS, 0, st>>>(w.g, n, P, w.flags, w.pS);
    big::k_scale_by_sum<<<eg, big::ETHREADS, 0, st>>>(w.g, w.pS, n, P, w.flags);
    for (int s = 1; s <= nT && !rc; ++s) {
      const float t = tMax * (float)s / (float)nT;
      big::k_fw_point<<<eg, big::ETHREADS, 0, st>>>(pop, w.a0, w.g, n, P, w.flags, nullptr, t);
      self_conv(pop);
      big::k_fw_refine<<<P, big::ETHREADS, 0, st>>>(pop, w.cbuf, w.pmax, n, Q, R, P, w.flags,
                                                    2e-4f, s, t, w.best, w.tsel);
      rc = check_launch();
    }
    if (rc) break;
    // the move (t = 0 restores the round's start), then stop candidates
    // without an improving t
    big::k_fw_point<<<eg, big::ETHREADS, 0, st>>>(pop, w.a0, w.g, n, P, w.flags, w.tsel, 0.f);
    big::k_fw_accept<<<(P + 127) / 128, 128, 0, st>>>(w.tsel, P, w.flags);
    rc = check_launch();
  }
  return rc;
}

}  // namespace sidon_host
