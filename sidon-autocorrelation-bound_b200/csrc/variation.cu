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

// ------------------------------ cell rules --------------------------------
// Every operator is one instance of a generic per-cell rule, fixed once per
// offspring from its operator id and parameters (rule_for).  A cell's value
// is built in up to four stages, each optional:
//
//   1. start  -- the parent cell A[i]; the mirrored cell A[n-1-i] or the
//                mean of the two; A[i - shift] (zero off the row); the mix
//                lam A[i] + (1 - lam) B[i]; or a value synthesised from
//                scratch (a cosine wave or the piecewise structured profile);
//   2. scale  -- times exp(sg N_i), or times (1 + 3 sg w(i)) for a cosine
//                wave w; or plus sg mean N_i (N_i a per-cell normal);
//   3. window -- inside a window of cells (an index range, or a distance
//                from one end): take B[i], zero the cell, add a constant, or
//                add a constant / (1 + distance);
//   4. floor  -- zero below a threshold, and/or clamp at zero (everywhere, or
//                in the window only).
//
// Each stage reproduces the exact float expression of the operator it
// serves (the file is compiled without fused multiply-add), so the host
// restatement in the oracle matches these cells bit for bit outside libm.

enum Start : int { S_A, S_MIRROR, S_MIRROR_MEAN, S_SHIFT, S_MIX, S_WAVE, S_PROFILE };
enum Scale : int { X_NONE, X_EXP_NOISE, X_WAVE, X_ADD_NOISE };
enum Window : int { W_NONE, W_TAKE_B, W_ZERO, W_ADD, W_ADD_DECAY };
enum Clamp : int { C_NONE, C_ALL, C_WINDOW };

template <typename T>
struct Rule {
  int start = S_A, scale = X_NONE, window = W_NONE, clamp = C_NONE;
  int lo = 0, hi = 0;          // window [lo, hi) of cell indices, or of distances
  bool from_end = false;       // window over distances from the end, not indices
  bool dist_from_right = false;
  int shift = 0;               // S_SHIFT: cell i takes A[i - shift]
  T lam = T(0);                // S_MIX weight of the first parent
  T cst = T(0);                // W_ADD / W_ADD_DECAY constant, X_ADD_NOISE sg * mean
  bool floor = false;          // zero the cells below thr
  T thr = T(0);
  float sg = 0.f;              // strength
  // cosine waves: nf terms, term f at frequency 1 + u[4 + f % 8] * fspan and
  // phase 2 pi u[12 + f % 8], each divided by nf (per_term) or the sum
  int nf = 0;
  float fspan = 0.f;
  bool per_term = false;
  float base = 0.f;            // S_WAVE offset
};

// sum of the rule's cosine terms at cell i
template <typename T>
__device__ inline float wave_at(const Rule<T>& r, const float* u, int i, float fn) {
  float m = 0.f;
  for (int f = 0; f < r.nf; ++f) {
    const float freq = 1.0f + u[4 + (f & 7)] * r.fspan;
    const float ph = 6.2831853f * u[12 + (f & 7)];
    const float c = cosf(6.2831853f * freq * (float)i / fn + ph);
    m += r.per_term ? c / (float)r.nf : c;
  }
  return m;
}

// The structured seed profile (operator 11): six segments of the unit
// interval, each a level times (1 + amp * roughness), the roughness a mix of
// nf cosines; an atom at the chosen end decaying over three more cells.
struct Profile {
  float edge[5];               // right edges of segments 0..4 (segment 5 runs to 1)
  float level[6], amp[6];
  float atom;
  int nf;
  bool flip;
};
__device__ inline Profile profile_of(const float* u) {
  Profile P;
  P.flip = u[30] < 0.5f;
  P.atom = 30.f + 250.f * u[31];
  P.edge[0] = 0.28f + 0.16f * u[32];                 // plateau
  P.edge[1] = P.edge[0] + 0.10f + 0.14f * u[33];     // depression
  P.edge[2] = P.edge[1] + 0.02f + 0.08f * u[34];     // hump
  P.edge[3] = 0.70f + 0.16f * u[35];                 // shoulder up to the gap
  P.edge[4] = P.edge[3] + 0.05f + 0.15f * u[36];     // hard gap
  const float lv[6] = {4.2f, 0.7f, 5.2f, 2.0f, 0.f, 3.0f + 14.0f * u[37]};
  const float am[6] = {0.45f, 0.80f, 0.30f, 0.70f, 0.f, 0.20f};
  for (int s = 0; s < 6; ++s) {
    P.level[s] = lv[s];
    P.amp[s] = am[s];
  }
  P.nf = 3 + (int)(u[38] * 6.f);
  return P;
}
__device__ inline float profile_at(const Profile& P, const float* u, int i, int n, float fn) {
  const int d = P.flip ? (n - 1 - i) : i;
  const float x = ((float)d + 0.5f) / fn;
  float rough = 0.f;
  for (int f = 0; f < P.nf; ++f)
    rough += cosf(6.2831853f * (2.f + u[40 + f] * 40.f) * x + 6.2831853f * u[48 + f]);
  rough /= (float)P.nf;
  int s = 0;
  while (s < 5 && !(x < P.edge[s])) ++s;
  float v = s == 4 ? 0.f : P.level[s] * (1.f + P.amp[s] * rough);
  if (d == 0) v += P.atom;
  else if (d < 4) v += P.atom * 0.10f / (float)d;
  return v;
}

// The rule of operator `op` (the reference's operator set, kernels.cuh:583-801:
// which parameter drives which breakpoint, amplitude or mode).  mean is the
// parent's mean height (fp64 block sum), needed by the ops that scale by it.
template <typename T>
__device__ inline Rule<T> rule_for(int op, const float* u, float sg, int n, T mean) {
  Rule<T> r;
  const float fn = (float)n;
  r.sg = sg;
  switch (op) {
    case 0:                                     // blend, lam in [-0.3, 1.3]
      r.start = S_MIX;
      r.lam = T(-0.3f + 1.6f * u[0]);
      r.clamp = C_ALL;
      break;
    case 1: {                                   // second parent between two cuts
      const int c1 = (int)(u[1] * fn), c2 = (int)(u[2] * fn);
      r.window = W_TAKE_B;
      r.lo = c1 < c2 ? c1 : c2;
      r.hi = c1 < c2 ? c2 : c1;
      break;
    }
    case 2:                                     // times exp(sg N_i)
      r.scale = X_EXP_NOISE;
      break;
    case 3:                                     // times 1 + 3 sg (mean of 1-5 cosines)
      r.scale = X_WAVE;
      r.nf = 1 + (int)(u[3] * 5.0f);
      r.fspan = 12.0f;
      r.per_term = true;
      r.clamp = C_ALL;
      break;
    case 4:                                     // plus sg mean N_i
      r.scale = X_ADD_NOISE;
      r.cst = T(sg) * mean;
      r.clamp = C_ALL;
      break;
    case 5:                                     // drop cells below a fraction of the mean
      r.floor = true;
      r.thr = mean * T(0.05f + 0.9f * u[20]);
      break;
    case 6:                                     // mirror, or average with the mirror
      r.start = u[21] < 0.5f ? S_MIRROR : S_MIRROR_MEAN;
      break;
    case 7:                                     // shift by up to n/8 either way
      r.start = S_SHIFT;
      r.shift = (int)((u[22] - 0.5f) * fn * 0.25f);
      break;
    case 8: {                                   // second parent on a block of up to n/2
      const int len = 1 + (int)(u[23] * 0.5f * fn);
      r.window = W_TAKE_B;
      r.lo = (int)(u[24] * (float)(n - len > 0 ? n - len : 1));
      r.hi = r.lo + len;
      break;
    }
    case 9:                                     // fresh smooth function plus noise
      r.start = S_WAVE;
      r.nf = 2 + (int)(u[25] * 6.0f);
      r.fspan = 10.0f;
      r.base = 0.3f + 0.7f * u[26];
      r.clamp = C_ALL;
      break;
    case 10: {                                  // a bump of width up to 6% of n
      const int loc = (int)(u[27] * fn);
      const int wdt = 1 + (int)(u[28] * fn * 0.03f);
      r.window = W_ADD;
      r.lo = loc - wdt;
      r.hi = loc + wdt + 1;
      r.cst = mean * T(1.0f + 6.0f * u[29]);
      break;
    }
    case 11:                                    // the structured seed profile
      r.start = S_PROFILE;
      r.clamp = C_ALL;
      break;
    case 12: {                                  // carve (or fill) a support gap
      const int len = 1 + (int)((0.015f + 0.13f * u[30]) * fn);
      r.lo = (int)(u[31] * (float)(n > len ? n - len : 1));
      r.hi = r.lo + len;
      r.window = u[32] < 0.7f ? W_ZERO : W_ADD;
      r.cst = mean * T(0.2f + 1.8f * u[33]);
      break;
    }
    case 13:                                    // grow or shrink the atom at one end
      r.window = W_ADD_DECAY;
      r.from_end = true;
      r.dist_from_right = !(u[30] < 0.5f);
      r.lo = 0;
      r.hi = 1 + (int)(u[31] * 0.012f * fn);
      r.cst = mean * T(-20.f + 260.f * u[32]);
      r.clamp = C_WINDOW;
      break;
    default:                                    // clone
      break;
  }
  return r;
}

// which operators scale by the parent's mean
__host__ __device__ inline bool needs_mean(int op) {
  return op == 4 || op == 5 || op == 10 || op == 12 || op == 13;
}

// cell i of the offspring under rule r
template <typename T>
__device__ inline T apply_rule(const Rule<T>& r, const Profile& prof, const float* u,
                               const T* A, const T* B, int i, int n, unsigned long long seed,
                               unsigned long long gen, int j) {
  const float fn = (float)n;
  T x;
  switch (r.start) {                            // 1. start
    case S_MIRROR: x = A[n - 1 - i]; break;
    case S_MIRROR_MEAN: x = T(0.5) * (A[i] + A[n - 1 - i]); break;
    case S_SHIFT: {
      const int k = i - r.shift;
      x = (k >= 0 && k < n) ? A[k] : T(0);
      break;
    }
    case S_MIX: x = r.lam * A[i] + (T(1) - r.lam) * B[i]; break;
    case S_WAVE: {
      const float v = r.base + wave_at(r, u, i, fn) / (float)r.nf +
                      0.4f * normal_at(seed, gen, j, i);
      x = T(v);
      break;
    }
    case S_PROFILE: x = T(profile_at(prof, u, i, n, fn)); break;
    default: x = A[i]; break;
  }
  switch (r.scale) {                            // 2. scale
    case X_EXP_NOISE: x = x * dev_exp(T(r.sg * normal_at(seed, gen, j, i))); break;
    case X_WAVE: x = x * T(1.0f + r.sg * 3.0f * wave_at(r, u, i, fn)); break;
    case X_ADD_NOISE: x = x + r.cst * T(normal_at(seed, gen, j, i)); break;
    default: break;
  }
  const int pos = r.from_end ? (r.dist_from_right ? n - 1 - i : i) : i;
  const bool inside = r.window != W_NONE && pos >= r.lo && pos < r.hi;
  if (inside) {                                 // 3. window
    switch (r.window) {
      case W_TAKE_B: x = B[i]; break;
      case W_ZERO: x = T(0); break;
      case W_ADD: x += r.cst; break;
      case W_ADD_DECAY: x += r.cst / T(1 + pos); break;
      default: break;
    }
  }
  // 4. floor and clamp.  The two clamps keep their operators' forms: the one
  // over every cell maps NaN and -0 to +0, the window's leaves them.
  if (r.floor && x < r.thr) x = T(0);
  if (r.clamp == C_ALL) x = x > T(0) ? x : T(0);
  if (r.clamp == C_WINDOW && inside && x < T(0)) x = T(0);
  return x;
}

template <typename T>
__global__ void __launch_bounds__(BD)
k_variation(const T* __restrict__ pop, T* __restrict__ out, int n, int n_off,
            const int* __restrict__ p1, const int* __restrict__ p2, const int* __restrict__ opv,
            const float* __restrict__ strength, unsigned long long seed, unsigned long long gen,
            const unsigned long long* __restrict__ gen_dev) {
  __shared__ float u[64];
  __shared__ double red[32];
  if (gen_dev) gen = *gen_dev;   // the generation counter of a captured loop
  const int j = blockIdx.x;
  if (j >= n_off) return;
  const int op = opv[j];
  const T* A = pop + (size_t)p1[j] * n;
  const T* B = pop + (size_t)p2[j] * n;
  T* O = out + (size_t)j * n;
  if (threadIdx.x == 0) params(seed, gen, j, u);
  __syncthreads();
  const T mean = needs_mean(op) ? T(mean_of(A, n, red)) : T(0);
  const Rule<T> r = rule_for<T>(op, u, strength[j], n, mean);
  Profile prof;
  if (r.start == S_PROFILE) prof = profile_of(u);
  for (int i = threadIdx.x; i < n; i += BD) O[i] = apply_rule(r, prof, u, A, B, i, n, seed, gen, j);
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
