// ---------------------------------------------------------------------------
//  variation.cu -- the memetic loop's variation operators and support
//  signatures on the device (semantics of src/kernels.cuh:558-849).
//
//  One CTA per offspring j: parents p1[j], p2[j], operator op[j] (0-13,
//  anything else clones p1), strength[j]; the offspring is renormalised to
//  sum 1.  Randomness comes from a counter-based generator, Philox4x32-10
//  (Salmon, Moraes, Dror, Shaw, SC 2011), evaluated as a pure function of
//  (seed, generation, offspring, element), so any element's draw is
//  reproducible alone -- on the host too (the oracle restates it).  The
//  64 per-offspring parameters u[0..63] are uniform in (0, 1) with 24-bit
//  resolution; per-element normals use Box-Muller in fp64.  The streams are
//  this library's own: the operators' meaning (which parameter drives what)
//  follows the reference, its draws do not.
//
//  Heights are read from global memory directly (every operator touches
//  each parent cell at most twice), so any n works.  Block sums (the mean
//  of ops 4, 5, 10, 12, 13 and the final renormalisation) run in fp64 in a
//  fixed order: per-thread partial sums over i = t, t + 256, ..., a warp
//  xor-butterfly, then the warps in order.
// ---------------------------------------------------------------------------
#include <cmath>

#include "common.cuh"
#include "philox.cuh"

namespace sidon {
namespace var {

constexpr int BD = 256;

using rng::U4;
using rng::philox;
using rng::u01;

// the offspring's 64 parameters: counters (q, j, gen_lo, gen_hi ^ 0), q < 16
__host__ __device__ inline void params(unsigned long long seed, unsigned long long gen, int j,
                                       float* u) {
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  for (int q = 0; q < 16; ++q) {
    const U4 r = philox({(uint32_t)q, (uint32_t)j, (uint32_t)gen, (uint32_t)(gen >> 32) << 1},
                        k0, k1);
    u[4 * q + 0] = u01(r.x);
    u[4 * q + 1] = u01(r.y);
    u[4 * q + 2] = u01(r.z);
    u[4 * q + 3] = u01(r.w);
  }
}

// standard normal for element i of offspring j (Box-Muller, fp64)
__host__ __device__ inline float normal_at(unsigned long long seed, unsigned long long gen, int j,
                                           int i) {
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  const U4 r = philox({(uint32_t)i, (uint32_t)j, (uint32_t)gen, ((uint32_t)(gen >> 32) << 1) | 1u},
                      k0, k1);
  const double a = (double)u01(r.x), b = (double)u01(r.y);
  return (float)(sqrt(-2.0 * log(a)) * cos(6.283185307179586 * b));
}

// fp64 block sum in the fixed order described above; all threads get it
__device__ inline double fixed_sum(double v, double* scratch) {
  return block_sum(v, scratch);
}

template <typename T>
__device__ inline double mean_of(const T* A, int n, double* scratch) {
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += BD) s += (double)A[i];
  return fixed_sum(s, scratch) / (double)n;
}

template <typename T>
__global__ void __launch_bounds__(BD)
k_variation(const T* __restrict__ pop, T* __restrict__ out, int n, int n_off,
            const int* __restrict__ p1, const int* __restrict__ p2, const int* __restrict__ opv,
            const float* __restrict__ strength, unsigned long long seed, unsigned long long gen,
            const unsigned long long* __restrict__ gen_dev) {
  __shared__ float u[64];
  if (gen_dev) gen = *gen_dev;   // the generation counter of a captured loop
  __shared__ double red[32];
  const int j = blockIdx.x;
  if (j >= n_off) return;
  const int o = opv[j];
  const T* A = pop + (size_t)p1[j] * n;
  const T* B = pop + (size_t)p2[j] * n;
  T* O = out + (size_t)j * n;
  const float sg = strength[j];
  if (threadIdx.x == 0) params(seed, gen, j, u);
  __syncthreads();
  const float fn = (float)n;
  switch (o) {
    case 0: {  // blend crossover, lambda in [-0.3, 1.3]
      const T lam = T(-0.3f + 1.6f * u[0]);
      for (int i = threadIdx.x; i < n; i += BD) {
        const T x = lam * A[i] + (T(1) - lam) * B[i];
        O[i] = x > T(0) ? x : T(0);
      }
      break;
    }
    case 1: {  // two-point segment crossover
      int c1 = (int)(u[1] * fn), c2 = (int)(u[2] * fn);
      if (c1 > c2) { const int t = c1; c1 = c2; c2 = t; }
      for (int i = threadIdx.x; i < n; i += BD) O[i] = (i >= c1 && i < c2) ? B[i] : A[i];
      break;
    }
    case 2: {  // log-normal multiplicative noise
      for (int i = threadIdx.x; i < n; i += BD)
        O[i] = A[i] * dev_exp(T(sg * normal_at(seed, gen, j, i)));
      break;
    }
    case 3: {  // smooth low-frequency perturbation (a few cosine modes)
      const int nf = 1 + (int)(u[3] * 5.0f);
      for (int i = threadIdx.x; i < n; i += BD) {
        float m = 0.f;
        for (int f = 0; f < nf; ++f) {
          const float freq = 1.0f + u[4 + f] * 12.0f;
          const float ph = 6.2831853f * u[12 + f];
          m += cosf(6.2831853f * freq * (float)i / fn + ph) / (float)nf;
        }
        const T x = A[i] * T(1.0f + sg * 3.0f * m);
        O[i] = x > T(0) ? x : T(0);
      }
      break;
    }
    case 4: {  // additive gaussian noise scaled by the mean height
      const T mean = T(mean_of(A, n, red));
      for (int i = threadIdx.x; i < n; i += BD) {
        const T x = A[i] + T(sg) * mean * T(normal_at(seed, gen, j, i));
        O[i] = x > T(0) ? x : T(0);
      }
      break;
    }
    case 5: {  // sparsify: zero the entries below a fraction of the mean
      const T mean = T(mean_of(A, n, red));
      const T thr = mean * T(0.05f + 0.9f * u[20]);
      for (int i = threadIdx.x; i < n; i += BD) O[i] = A[i] < thr ? T(0) : A[i];
      break;
    }
    case 6: {  // reflect (hard) or symmetrise
      const bool hard = u[21] < 0.5f;
      for (int i = threadIdx.x; i < n; i += BD)
        O[i] = hard ? A[n - 1 - i] : T(0.5) * (A[i] + A[n - 1 - i]);
      break;
    }
    case 7: {  // shift by up to n/8 either way, zero fill
      const int sh = (int)((u[22] - 0.5f) * fn * 0.25f);
      for (int i = threadIdx.x; i < n; i += BD) {
        const int k = i - sh;
        O[i] = (k >= 0 && k < n) ? A[k] : T(0);
      }
      break;
    }
    case 8: {  // splice a random block of the second parent
      const int len = 1 + (int)(u[23] * 0.5f * fn);
      const int st0 = (int)(u[24] * (float)(n - len > 0 ? n - len : 1));
      for (int i = threadIdx.x; i < n; i += BD)
        O[i] = (i >= st0 && i < st0 + len) ? B[i] : A[i];
      break;
    }
    case 9: {  // fresh random restart: smooth positive random function
      const int nf = 2 + (int)(u[25] * 6.0f);
      const float base = 0.3f + 0.7f * u[26];
      for (int i = threadIdx.x; i < n; i += BD) {
        float m = 0.f;
        for (int f = 0; f < nf; ++f) {
          const float freq = 1.0f + u[4 + (f % 8)] * 10.0f;
          const float ph = 6.2831853f * u[12 + (f % 8)];
          m += cosf(6.2831853f * freq * (float)i / fn + ph);
        }
        const float val = base + m / (float)nf + 0.4f * normal_at(seed, gen, j, i);
        O[i] = val > 0.f ? T(val) : T(0);
      }
      break;
    }
    case 10: {  // spike injection at a random location
      const int loc = (int)(u[27] * fn);
      const int wdt = 1 + (int)(u[28] * fn * 0.03f);
      const T mean = T(mean_of(A, n, red));
      const T amp = mean * T(1.0f + 6.0f * u[29]);
      for (int i = threadIdx.x; i < n; i += BD) {
        T x = A[i];
        if (i >= loc - wdt && i <= loc + wdt) x += amp;
        O[i] = x;
      }
      break;
    }
    case 11: {  // structured seed: atom, plateau, depression, hump, band, gap, spike
      const bool flip = u[30] < 0.5f;
      const float atom = 30.f + 250.f * u[31];
      const float pl1 = 0.28f + 0.16f * u[32];
      const float pl2 = pl1 + 0.10f + 0.14f * u[33];
      const float hump = pl2 + 0.02f + 0.08f * u[34];
      const float gap0 = 0.70f + 0.16f * u[35];
      const float gap1 = gap0 + 0.05f + 0.15f * u[36];
      const float tail = 3.0f + 14.0f * u[37];
      const int nf = 3 + (int)(u[38] * 6.f);
      for (int i = threadIdx.x; i < n; i += BD) {
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
        O[i] = v > 0.f ? T(v) : T(0);
      }
      break;
    }
    case 12: {  // gap surgery: carve out (or fill in) a hard support gap
      const T mean = T(mean_of(A, n, red));
      const int len = 1 + (int)((0.015f + 0.13f * u[30]) * fn);
      const int st0 = (int)(u[31] * (float)(n > len ? n - len : 1));
      const bool carve = u[32] < 0.7f;
      const T fill = mean * T(0.2f + 1.8f * u[33]);
      for (int i = threadIdx.x; i < n; i += BD) {
        T x = A[i];
        if (i >= st0 && i < st0 + len) x = carve ? T(0) : (x + fill);
        O[i] = x;
      }
      break;
    }
    case 13: {  // endpoint atom: grow or shrink the boundary spike
      const T mean = T(mean_of(A, n, red));
      const bool left = u[30] < 0.5f;
      const int w = 1 + (int)(u[31] * 0.012f * fn);
      const T add = mean * T(-20.f + 260.f * u[32]);
      for (int i = threadIdx.x; i < n; i += BD) {
        const int d = left ? i : (n - 1 - i);
        T x = A[i];
        if (d < w) {
          x += add / T(1 + d);
          if (x < T(0)) x = T(0);
        }
        O[i] = x;
      }
      break;
    }
    default: {  // clone (op 20 in the reference driver)
      for (int i = threadIdx.x; i < n; i += BD) O[i] = A[i];
      break;
    }
  }
  __syncthreads();
  // renormalise to sum 1 (F is scale invariant); a non-positive sum becomes
  // the uniform 1/n
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += BD) s += (double)O[i];
  const double S = fixed_sum(s, red);
  if (S > 0.0) {
    const T inv = T(1.0 / S);
    for (int i = threadIdx.x; i < n; i += BD) O[i] *= inv;
  } else {
    for (int i = threadIdx.x; i < n; i += BD) O[i] = T(1) / T(n);
  }
}

// Support signature (src/kernels.cuh:803-849): the xor, over every index i
// with a_i > tol * mean, of a mixed 64-bit hash of i (order free, so equal
// supports give equal signatures), and the count of such indices.  The
// mean is summed in fp64.
template <typename T>
__global__ void __launch_bounds__(BD)
k_support_sig(const T* __restrict__ pop, int n, float tol, unsigned long long* __restrict__ sig,
              int* __restrict__ nnz) {
  __shared__ double red[32];
  __shared__ unsigned long long sh[BD / 32];
  __shared__ int sc[BD / 32];
  const int p = blockIdx.x;
  const T* a = pop + (size_t)p * n;
  const double thr = mean_of(a, n, red) * (double)tol;
  unsigned long long h = 0ull;
  int c = 0;
  for (int i = threadIdx.x; i < n; i += BD) {
    if ((double)a[i] > thr) {
      ++c;
      unsigned long long x = (unsigned long long)i * 0x9E3779B97F4A7C15ull;
      x ^= x >> 29;
      x *= 0xBF58476D1CE4E5B9ull;
      x ^= x >> 32;
      h ^= x;
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    h ^= __shfl_xor_sync(0xffffffffu, h, off);
    c += __shfl_xor_sync(0xffffffffu, c, off);
  }
  if ((threadIdx.x & 31) == 0) {
    sh[threadIdx.x >> 5] = h;
    sc[threadIdx.x >> 5] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long r = 0ull;   // the empty support hashes to 0
    int cc = 0;
    for (int w = 0; w < BD / 32; ++w) {
      r ^= sh[w];
      cc += sc[w];
    }
    sig[p] = r;
    nnz[p] = cc;
  }
}

}  // namespace var
}  // namespace sidon

namespace sidon_host {
using namespace sidon;

int launch_variation(const void* pop, void* out, int dtype, int n, int n_off, const int* p1,
                     const int* p2, const int* op, const float* strength,
                     unsigned long long seed, unsigned long long gen, cudaStream_t st,
                     const unsigned long long* gen_dev) {
  if (dtype == SIDON_F32)
    var::k_variation<float><<<n_off, var::BD, 0, st>>>((const float*)pop, (float*)out, n, n_off,
                                                        p1, p2, op, strength, seed, gen, gen_dev);
  else
    var::k_variation<double><<<n_off, var::BD, 0, st>>>((const double*)pop, (double*)out, n,
                                                         n_off, p1, p2, op, strength, seed, gen,
                                                         gen_dev);
  return check_launch();
}

int launch_support_sig(const void* pop, int dtype, int n, int P, float tol,
                       unsigned long long* sig, int* nnz, cudaStream_t st) {
  if (dtype == SIDON_F32)
    var::k_support_sig<float><<<P, var::BD, 0, st>>>((const float*)pop, n, tol, sig, nnz);
  else
    var::k_support_sig<double><<<P, var::BD, 0, st>>>((const double*)pop, n, tol, sig, nnz);
  return check_launch();
}

}  // namespace sidon_host
