// ---------------------------------------------------------------------------
//  certify.cu -- exact certification of F on the GPU.
//
//  F = 2 n M / (S S) with M = max_k b_k and S = sum_i a_i each computed
//  EXACTLY and rounded once to fp64 (round to nearest even).  Rounding is
//  monotone, so max_k round(b_k) = round(max_k b_k): each b_k is made exact
//  and rounded on its own, and the max is taken over the rounded values.
//  A cell split maps b -> {2 b_k, b_k + b_(k-1)}, M -> 2M and S -> 2S exactly,
//  so the certified F is bit-identical before and after sidon_refine.
//
//  Per candidate (one CTA):
//   1. fp64 pass (hostF arithmetic) -> M64.  The fp64 b_k has relative error
//      below (n+1) 2^-53; every k whose exact value could be the maximum has
//      b64_k >= M64 (1 - 1e-9) for n < 10^6, so those k form the candidate set.
//   2. One warp per candidate k: lane l accumulates the terms i == l (mod 32)
//      into a carry-save fixed-point accumulator of int64 limbs holding 32
//      payload bits each (headroom for 2^31 signed additions per limb).  Each
//      product a_i a_(k-i) is split exactly into p + e (p = fl(ab),
//      e = fma(a, b, -p)); for fp32 heights e == 0.  The 32 lanes' limbs are
//      summed limb by limb, carries are propagated once, and the value is
//      rounded to nearest even.
//   3. S likewise by one warp.
//  The accumulator window [lo, lo + 32 L) is sized from the candidate's own
//  exponent range (products span 2 emin - 106 .. 2 emax + 2, plus log2 n carry
//  bits); a candidate whose range needs more than kMaxLimbs limbs gets F = NaN.
// ---------------------------------------------------------------------------
#include "conv_simt.cuh"

namespace sidon {

constexpr int kMaxLimbs = 48;         // 1536-bit window
constexpr int kMaxCand = 2048;        // candidate k per CTA before the all-k fallback
constexpr int kCertTK = 7;

struct XWin {
  int lo;      // exponent of bit 0 of limb 0
  int limbs;   // limbs in use
};

__device__ __forceinline__ void xadd(long long* acc, const XWin& w, double t, bool negate) {
  if (t == 0.0) return;
  const long long bits = __double_as_longlong(t);
  int ex = (int)((bits >> 52) & 0x7ff);
  unsigned long long mant = (unsigned long long)bits & 0xfffffffffffffull;
  if (ex == 0) ex = 1;                  // subnormal: no hidden bit
  else mant |= 1ull << 52;
  const int e = ex - 1075;              // t = mant * 2^e
  const int pos = e - w.lo;             // >= 0 by construction of the window
  const int li = pos >> 5, bo = pos & 31;
  const unsigned long long lo64 = mant << bo;
  const unsigned long long hi64 = bo ? (mant >> (64 - bo)) : 0ull;
  const long long p0 = (long long)(lo64 & 0xffffffffull);
  const long long p1 = (long long)(lo64 >> 32);
  const long long p2 = (long long)hi64;
  if (!negate) {
    acc[li] += p0; acc[li + 1] += p1; if (li + 2 < w.limbs) acc[li + 2] += p2;
  } else {
    acc[li] -= p0; acc[li + 1] -= p1; if (li + 2 < w.limbs) acc[li + 2] -= p2;
  }
}

// Sum the lanes' limbs, normalise, round to double (lane 0 returns it).
__device__ double xreduce_round(long long* acc, const XWin& w) {
  const int lane = threadIdx.x & 31;
  for (int j = 0; j < w.limbs; ++j) {
    long long v = acc[j];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    acc[j] = v;
  }
  double out = 0.0;
  if (lane == 0) {
    long long carry = 0;
    for (int j = 0; j < w.limbs; ++j) {
      const long long v = acc[j] + carry;
      carry = v >> 32;                                  // floor division
      acc[j] = v - (carry << 32);                       // in [0, 2^32)
    }
    // value = sum acc[j] 2^(32 j + lo) (+ carry beyond the window: none for b_k >= 0)
    int top = w.limbs - 1;
    while (top >= 0 && acc[top] == 0) --top;
    if (top >= 0) {
      const int lz = __clzll((unsigned long long)acc[top]) - 32;   // leading zeros in 32 bits
      const int msb = top * 32 + (31 - lz);
      // gather bits [msb-63, msb] into a 64-bit window
      unsigned long long win = 0;
      for (int b = 0; b < 64; ++b) {
        const int bit = msb - b;
        win <<= 1;
        if (bit >= 0) win |= ((unsigned long long)acc[bit >> 5] >> (bit & 31)) & 1ull;
      }
      bool sticky = false;
      const int below = msb - 64;                       // highest bit not in the window
      if (below >= 0) {
        const int li = below >> 5, bo = below & 31;
        if (((unsigned long long)acc[li] & ((2ull << bo) - 1ull)) != 0) sticky = true;
        for (int j = li - 1; j >= 0 && !sticky; --j) if (acc[j]) sticky = true;
      }
      unsigned long long mant = win >> 11;              // top 53 bits
      const unsigned long long rest = win & 0x7ffull;   // 11 bits below
      const bool rb = (rest >> 10) & 1ull;
      const bool st = ((rest & 0x3ffull) != 0) || sticky;
      if (rb && (st || (mant & 1ull))) ++mant;
      out = ldexp((double)mant, msb - 52 + w.lo);
    }
  }
  return out;
}

template <typename Tin>
__global__ void __launch_bounds__(512, 1)
k_certify(const Tin* __restrict__ pop, int n, double* __restrict__ outF, double* __restrict__ outM,
          double* __restrict__ outS, int* __restrict__ outK) {
  constexpr int MG = margin<kCertTK>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* base = reinterpret_cast<double*>(smem_raw);
  double* sA = base + MG;
  double* sRed = base + (n + 2 * MG);
  int* sCand = reinterpret_cast<int*>(sRed + 32);
  __shared__ int sNC, sEmin, sEmax;
  __shared__ unsigned long long sBest;   // max of rounded b_k (bits of a non-negative double)
  __shared__ int sBestK;
  __shared__ double sSexact;
  const int pid = blockIdx.x;
  const Tin* a = pop + (size_t)pid * n;
  for (int i = threadIdx.x; i < n + 2 * MG; i += blockDim.x) base[i] = 0.0;
  if (threadIdx.x == 0) { sNC = 0; sEmin = 1 << 20; sEmax = -(1 << 20); sBest = 0ull; sBestK = 0x7fffffff; }
  __syncthreads();
  int emin = 1 << 20, emax = -(1 << 20);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double x = (double)a[i];
    sA[i] = x;
    if (x != 0.0) {
      const int ex = (int)((__double_as_longlong(x) >> 52) & 0x7ff);
      const int e = (ex == 0 ? 1 : ex) - 1075;          // LSB exponent of x
      emin = min(emin, e);
      emax = max(emax, e + 53);                         // x < 2^(e + 53)
    }
  }
  atomicMin(&sEmin, emin);
  atomicMax(&sEmax, emax);
  __syncthreads();
  double mloc = 0.0;
  conv_warp_tiles<kCertTK, false>(sA, sA, n, Team(), [&](int, double v) { mloc = v > mloc ? v : mloc; });
  const double M64 = block_max(mloc, sRed);
  const double thr = M64 * (1.0 - 1e-9);
  conv_warp_tiles<kCertTK, false>(sA, sA, n, Team(), [&](int k, double v) {
    if (v >= thr) {
      const int slot = atomicAdd(&sNC, 1);
      if (slot < kMaxCand) sCand[slot] = k;
    }
  });
  __syncthreads();
  const int ncand = sNC;
  const bool all_k = ncand > kMaxCand;                  // too many near-ties: certify every k
  XWin w;
  // product LSB >= 2 emin (split residual included), top < 2 emax + 1 + carry bits
  w.lo = 2 * sEmin - 64;
  w.limbs = (2 * sEmax + 40 - w.lo) / 32 + 3;
  if (sEmin > sEmax) w.limbs = 3;                       // all-zero candidate
  if (w.limbs > kMaxLimbs) {   // dynamic range too wide for the window: F = NaN
    if (threadIdx.x == 0) outF[pid] = __longlong_as_double(0x7ff8000000000000ll);
    return;
  }
  long long acc[kMaxLimbs];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, NW = blockDim.x >> 5;
  const int nk = all_k ? (2 * n - 1) : ncand;
  for (int c = wid; c < nk; c += NW) {
    const int k = all_k ? c : sCand[c];
    for (int j = 0; j < w.limbs; ++j) acc[j] = 0;
    const int ilo = max(0, k - (n - 1)), ihi = min(k, n - 1);
    for (int i = ilo + lane; i <= ihi; i += 32) {
      const double x = sA[i], y = sA[k - i];
      if (x == 0.0 || y == 0.0) continue;
      const double p = x * y;
      const double e = fma(x, y, -p);
      xadd(acc, w, p, false);
      if (e > 0.0) xadd(acc, w, e, false);
      else if (e < 0.0) xadd(acc, w, -e, true);
    }
    const double bk = xreduce_round(acc, w);
    if (lane == 0) atomicMax(&sBest, (unsigned long long)__double_as_longlong(bk));
  }
  __syncthreads();
  // argmax: smallest k whose rounded exact value equals the max (second sweep)
  const double Mx = __longlong_as_double((long long)sBest);
  for (int c = wid; c < nk; c += NW) {
    const int k = all_k ? c : sCand[c];
    for (int j = 0; j < w.limbs; ++j) acc[j] = 0;
    const int ilo = max(0, k - (n - 1)), ihi = min(k, n - 1);
    for (int i = ilo + lane; i <= ihi; i += 32) {
      const double x = sA[i], y = sA[k - i];
      if (x == 0.0 || y == 0.0) continue;
      const double p = x * y;
      const double e = fma(x, y, -p);
      xadd(acc, w, p, false);
      if (e > 0.0) xadd(acc, w, e, false);
      else if (e < 0.0) xadd(acc, w, -e, true);
    }
    const double bk = xreduce_round(acc, w);
    if (lane == 0 && bk == Mx) atomicMin(&sBestK, k);
  }
  // exact S by warp 0, on a window sized for the sum of heights
  if (wid == 0) {
    XWin ws;
    ws.lo = sEmin - 8;
    ws.limbs = (sEmax + 40 - ws.lo) / 32 + 3;
    if (sEmin > sEmax) ws.limbs = 3;
    if (ws.limbs > kMaxLimbs) ws.limbs = kMaxLimbs;
    for (int j = 0; j < ws.limbs; ++j) acc[j] = 0;
    for (int i = lane; i < n; i += 32) {
      const double x = sA[i];
      if (x > 0.0) xadd(acc, ws, x, false);
    }
    const double S = xreduce_round(acc, ws);
    if (lane == 0) sSexact = S;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const double S = sSexact;
    outF[pid] = (S > 0.0) ? (2.0 * (double)n * Mx / (S * S)) : 1e30;
    if (outM) outM[pid] = Mx;
    if (outS) outS[pid] = S;
    if (outK) outK[pid] = (sBestK == 0x7fffffff) ? 0 : sBestK;
  }
}

// The same certification for a candidate of any n, from the near-maximal k
// found by the streamed fp64 pass (list[p][0 .. count[p])): the heights are
// read from global memory.  More than `cap` near-maximal k: F = NaN (the
// streamed pass would have to certify every k).
template <typename Tin>
__global__ void __launch_bounds__(512, 1)
k_certify_list(const Tin* __restrict__ pop, int n, const int* __restrict__ list,
               const int* __restrict__ count, int cap, double* __restrict__ outF,
               double* __restrict__ outM, double* __restrict__ outS, int* __restrict__ outK) {
  __shared__ int sEmin, sEmax;
  __shared__ unsigned long long sBest;
  __shared__ int sBestK;
  __shared__ double sSexact;
  const int pid = blockIdx.x;
  const Tin* a = pop + (size_t)pid * n;
  const int ncand = count[pid];
  if (ncand > cap || ncand < 1) {
    if (threadIdx.x == 0) outF[pid] = __longlong_as_double(0x7ff8000000000000ll);
    return;
  }
  const int* cand = list + (size_t)pid * cap;
  if (threadIdx.x == 0) { sEmin = 1 << 20; sEmax = -(1 << 20); sBest = 0ull; sBestK = 0x7fffffff; }
  __syncthreads();
  int emin = 1 << 20, emax = -(1 << 20);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double x = (double)a[i];
    if (x != 0.0) {
      const int ex = (int)((__double_as_longlong(x) >> 52) & 0x7ff);
      const int e = (ex == 0 ? 1 : ex) - 1075;
      emin = min(emin, e);
      emax = max(emax, e + 53);
    }
  }
  atomicMin(&sEmin, emin);
  atomicMax(&sEmax, emax);
  __syncthreads();
  XWin w;
  w.lo = 2 * sEmin - 64;
  w.limbs = (2 * sEmax + 40 - w.lo) / 32 + 3;
  if (sEmin > sEmax) w.limbs = 3;
  if (w.limbs > kMaxLimbs) {
    if (threadIdx.x == 0) outF[pid] = __longlong_as_double(0x7ff8000000000000ll);
    return;
  }
  long long acc[kMaxLimbs];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, NW = blockDim.x >> 5;
  for (int sweep = 0; sweep < 2; ++sweep) {
    const double Mx = __longlong_as_double((long long)sBest);
    for (int c = wid; c < ncand; c += NW) {
      const int k = cand[c];
      for (int j = 0; j < w.limbs; ++j) acc[j] = 0;
      const int ilo = max(0, k - (n - 1)), ihi = min(k, n - 1);
      for (int i = ilo + lane; i <= ihi; i += 32) {
        const double x = (double)a[i], y = (double)a[k - i];
        if (x == 0.0 || y == 0.0) continue;
        const double pr = x * y;
        const double e = fma(x, y, -pr);
        xadd(acc, w, pr, false);
        if (e > 0.0) xadd(acc, w, e, false);
        else if (e < 0.0) xadd(acc, w, -e, true);
      }
      const double bk = xreduce_round(acc, w);
      if (lane == 0) {
        if (sweep == 0) atomicMax(&sBest, (unsigned long long)__double_as_longlong(bk));
        else if (bk == Mx) atomicMin(&sBestK, k);
      }
    }
    __syncthreads();
  }
  if (wid == 0) {
    XWin ws;
    ws.lo = sEmin - 8;
    ws.limbs = (sEmax + 40 - ws.lo) / 32 + 3;
    if (sEmin > sEmax) ws.limbs = 3;
    if (ws.limbs > kMaxLimbs) ws.limbs = kMaxLimbs;
    for (int j = 0; j < ws.limbs; ++j) acc[j] = 0;
    for (int i = lane; i < n; i += 32) {
      const double x = (double)a[i];
      if (x > 0.0) xadd(acc, ws, x, false);
    }
    const double S = xreduce_round(acc, ws);
    if (lane == 0) sSexact = S;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const double S = sSexact;
    const double Mx = __longlong_as_double((long long)sBest);
    outF[pid] = (S > 0.0) ? (2.0 * (double)n * Mx / (S * S)) : 1e30;
    if (outM) outM[pid] = Mx;
    if (outS) outS[pid] = S;
    if (outK) outK[pid] = (sBestK == 0x7fffffff) ? 0 : sBestK;
  }
}

}  // namespace sidon

namespace sidon_host {
using namespace sidon;

size_t smem_certify(int n) {
  return sizeof(double) * ((size_t)n + 2 * margin<kCertTK>() + 32) + sizeof(int) * kMaxCand;
}

int launch_eval_stream_list(const void* pop, int dtype, int n, int P, double* mbits, int* list,
                            int* list_count, int cap, cudaStream_t st);

// near-maximal k per candidate kept by the large-n certification
constexpr int kListCap = 4096;
size_t certify_workspace_bytes(int P) {
  return (size_t)P * (kListCap + 1) * sizeof(int) + (size_t)P * sizeof(double);
}

// any n: streamed fp64 pass for the near-maximal k, then the exact sums
int launch_certify_large(const void* pop, int dtype, int n, int P, double* outF, double* outM,
                         double* outS, int* outK, void* ws, cudaStream_t st) {
  double* mbits = reinterpret_cast<double*>(ws);
  int* cnt = reinterpret_cast<int*>(mbits + P);
  int* list = cnt + P;
  int rc = launch_eval_stream_list(pop, dtype, n, P, mbits, list, cnt, kListCap, st);
  if (rc) return rc;
  if (dtype == SIDON_F32)
    k_certify_list<float><<<P, 512, 0, st>>>((const float*)pop, n, list, cnt, kListCap, outF,
                                              outM, outS, outK);
  else
    k_certify_list<double><<<P, 512, 0, st>>>((const double*)pop, n, list, cnt, kListCap, outF,
                                               outM, outS, outK);
  return check_launch();
}

int launch_certify(const void* pop, int dtype, int n, int P, double* outF, double* outM,
                   double* outS, int* outK, cudaStream_t st) {
  const size_t sm = smem_certify(n);
  if ((long long)sm > (long long)smem_optin()) return SIDON_ERR_SMEM;
  const int threads = 512;
  if (dtype == SIDON_F32) {
    cudaError_t e = cudaFuncSetAttribute((const void*)k_certify<float>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return set_cuda_error(e);
    k_certify<float><<<P, threads, sm, st>>>((const float*)pop, n, outF, outM, outS, outK);
  } else {
    cudaError_t e = cudaFuncSetAttribute((const void*)k_certify<double>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return set_cuda_error(e);
    k_certify<double><<<P, threads, sm, st>>>((const double*)pop, n, outF, outM, outS, outK);
  }
  return check_launch();
}

}  // namespace sidon_host
