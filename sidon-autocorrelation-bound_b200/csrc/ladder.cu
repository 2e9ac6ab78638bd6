// ---------------------------------------------------------------------------
//  ladder.cu -- HBM-bound population kernels:
//    k_refine   n -> 2n cell split   (src/kernels.cuh:538-547, src/main.cu:491-495)
//    k_coarsen  2n -> n pair average (src/kernels.cuh:550-557)
//    k_island_rank / k_island_migrate   per-island ranking by fp64 F and
//               best-of-i -> worst-of-(i+1) migration (src/main.cu:676-692)
//
//  The copy kernels are grid-stride over the flattened population with
//  128-bit loads where the row layout allows it; grids are sized in
//  multiples of the SM count.
// ---------------------------------------------------------------------------
#include "common.cuh"

namespace sidon {

// dst[p][2i] = dst[p][2i+1] = src[p][i]  over the flattened index j = p*n + i:
// dst[2j] = dst[2j+1] = src[j] (rows of 2n are contiguous), so the split is a
// pure element-duplication stream.  float4 in -> two float4 out.
__global__ void k_refine_f32(const float* __restrict__ src, float* __restrict__ dst, size_t total) {
  const size_t nv = total / 4;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const float4* s4 = reinterpret_cast<const float4*>(src);
  float4* d4 = reinterpret_cast<float4*>(dst);
  for (size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < nv; j += stride) {
    const float4 x = s4[j];
    d4[2 * j] = make_float4(x.x, x.x, x.y, x.y);
    d4[2 * j + 1] = make_float4(x.z, x.z, x.w, x.w);
  }
  for (size_t j = nv * 4 + (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < total; j += stride) {
    const float x = src[j];
    dst[2 * j] = x;
    dst[2 * j + 1] = x;
  }
}
__global__ void k_refine_f64(const double* __restrict__ src, double* __restrict__ dst, size_t total) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < total; j += stride) {
    const double x = src[j];
    reinterpret_cast<double2*>(dst)[j] = make_double2(x, x);
  }
}

// d[j] = 0.5 (s[2j] + s[2j+1]) over the flattened output index (rows of n2
// are contiguous and n2 is even, so pairs never straddle rows).
__global__ void k_coarsen_f32(const float* __restrict__ src, float* __restrict__ dst, size_t total) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < total; j += stride) {
    const float2 x = reinterpret_cast<const float2*>(src)[j];
    dst[j] = 0.5f * (x.x + x.y);
  }
}
__global__ void k_coarsen_f64(const double* __restrict__ src, double* __restrict__ dst, size_t total) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x; j < total; j += stride) {
    const double2 x = reinterpret_cast<const double2*>(src)[j];
    dst[j] = 0.5 * (x.x + x.y);
  }
}

// One CTA per island: bitonic sort of (fit, slot) pairs in shared memory,
// ascending by fit, ties by slot index.  PI <= 1024.
__global__ void k_island_rank(const double* __restrict__ fit, int PI, int* __restrict__ order) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  int L = 1;
  while (L < PI) L <<= 1;
  double* sk = reinterpret_cast<double*>(smem_raw);
  int* si = reinterpret_cast<int*>(sk + L);
  const int isl = blockIdx.x;
  for (int r = threadIdx.x; r < L; r += blockDim.x) {
    if (r < PI) { sk[r] = fit[(size_t)isl * PI + r]; si[r] = isl * PI + r; }
    else { sk[r] = __longlong_as_double(0x7ff0000000000000ll); si[r] = 0x7fffffff; }  // +inf pad
  }
  __syncthreads();
  for (int size = 2; size <= L; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int t = threadIdx.x; t < L / 2; t += blockDim.x) {
        const int lo = 2 * t - (t & (stride - 1));
        const int hi = lo + stride;
        const bool up = ((lo & size) == 0);
        const double ka = sk[lo], kb = sk[hi];
        const int ia = si[lo], ib = si[hi];
        // classes: 0 = number, 1 = NaN (worse than every number), 2 = padding
        const int ca = (ia == 0x7fffffff) ? 2 : (ka != ka ? 1 : 0);
        const int cb = (ib == 0x7fffffff) ? 2 : (kb != kb ? 1 : 0);
        bool a_gt_b;
        if (ca != cb) a_gt_b = ca > cb;
        else if (ca == 0 && ka != kb) a_gt_b = ka > kb;
        else a_gt_b = ia > ib;
        if (a_gt_b == up) { sk[lo] = kb; sk[hi] = ka; si[lo] = ib; si[hi] = ia; }
      }
      __syncthreads();
    }
  }
  for (int r = threadIdx.x; r < PI; r += blockDim.x) order[(size_t)isl * PI + r] = si[r];
}

// One CTA per (island i, rank j < k): row order[i][j] -> row order[i+1][PI-1-j].
// Sources are top-k rows, destinations bottom-k rows; with 2k <= PI these
// sets are disjoint, so all copies run concurrently without ordering.
__global__ void k_island_migrate(float* __restrict__ pop, int n, double* __restrict__ fit, int NI,
                                 int PI, int k, const int* __restrict__ order, int vec) {
  const int i = blockIdx.x / k, j = blockIdx.x % k;
  const int nx = (i + 1) % NI;
  const int src = order[(size_t)i * PI + j];
  const int dst = order[(size_t)nx * PI + PI - 1 - j];
  const float* s = pop + (size_t)src * n;
  float* d = pop + (size_t)dst * n;
  if (vec) {
    const float4* s4 = reinterpret_cast<const float4*>(s);
    float4* d4 = reinterpret_cast<float4*>(d);
    for (int t = threadIdx.x; t < n / 4; t += blockDim.x) d4[t] = s4[t];
  } else {
    for (int t = threadIdx.x; t < n; t += blockDim.x) d[t] = s[t];
  }
  if (threadIdx.x == 0) fit[dst] = fit[src];
}

// Ragged batch: as k_island_migrate, rows pop[offsets[p] .. offsets[p+1]).
// A source of the destination's size is copied with its fit.  Otherwise it
// is resampled to the destination's size by nearest neighbour,
// dst[t] = src[min(m-1, floor(t m / n))], and normalised to sum 1 in fp64
// (S summed in t order, dst[t] = fl(src / S)), the injection of
// src/main.cu:555-562; fit[dst] becomes NaN (unknown until re-evaluated).
__global__ void k_island_migrate_ragged(float* __restrict__ pop,
                                        const long long* __restrict__ offsets,
                                        double* __restrict__ fit, int NI, int PI, int k,
                                        const int* __restrict__ order) {
  __shared__ double sS;
  const int i = blockIdx.x / k, j = blockIdx.x % k;
  const int nx = (i + 1) % NI;
  const int src = order[(size_t)i * PI + j];
  const int dst = order[(size_t)nx * PI + PI - 1 - j];
  const long long so = offsets[src], dof = offsets[dst];
  const int m = (int)(offsets[src + 1] - so), n = (int)(offsets[dst + 1] - dof);
  const float* s = pop + so;
  float* d = pop + dof;
  if (m == n) {
    for (int t = threadIdx.x; t < n; t += blockDim.x) d[t] = s[t];
    if (threadIdx.x == 0) fit[dst] = fit[src];
    return;
  }
  if (m < 1 || n < 1) return;
  // the source and destination rows are distinct candidates (disjoint sets)
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    const long long q = (long long)t * m / n;
    d[t] = s[q < m - 1 ? q : m - 1];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double S = 0.0;
    for (int t = 0; t < n; ++t) S = __dadd_rn(S, (double)d[t]);
    sS = S;
    fit[dst] = __longlong_as_double(0x7ff8000000000000ll);
  }
  __syncthreads();
  const double S = sS;
  if (S > 0.0)
    for (int t = threadIdx.x; t < n; t += blockDim.x) d[t] = (float)__ddiv_rn((double)d[t], S);
}

// Resample every row of a [P][m] batch to n cells by nearest neighbour,
// dst[t] = src[min(m-1, floor(t m / n))] (the host resample of
// src/main.cu:496-497 and the injection of main.cu:555-562), optionally
// normalised to sum 1 as the migration above does (fp64 sum in t order,
// dst[t] = fl(dst[t] / S)).  One CTA per row.
__global__ void k_resample(const float* __restrict__ src, int m, float* __restrict__ dst, int n,
                           int normalise) {
  __shared__ double sS;
  const float* s = src + (size_t)blockIdx.x * m;
  float* d = dst + (size_t)blockIdx.x * n;
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    const long long q = (long long)t * m / n;
    d[t] = s[q < m - 1 ? q : m - 1];
  }
  if (!normalise) return;
  __syncthreads();
  if (threadIdx.x == 0) {
    double S = 0.0;
    for (int t = 0; t < n; ++t) S = __dadd_rn(S, (double)d[t]);
    sS = S;
  }
  __syncthreads();
  const double S = sS;
  if (S > 0.0)
    for (int t = threadIdx.x; t < n; t += blockDim.x) d[t] = (float)__ddiv_rn((double)d[t], S);
}

// order[r] = candidate of rank r when sorted by size descending, ties by
// index: the longest-first processing order of a ragged batch.  One thread
// per candidate counts the candidates ranked before it.
__global__ void k_ragged_order(const long long* __restrict__ offsets, int P,
                               int* __restrict__ order) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < P; c += gridDim.x * blockDim.x) {
    const long long nc = offsets[c + 1] - offsets[c];
    int r = 0;
    for (int o = 0; o < P; ++o) {
      const long long no = offsets[o + 1] - offsets[o];
      r += (no > nc) || (no == nc && o < c);
    }
    order[r] = c;
  }
}

}  // namespace sidon

namespace sidon_host {
using namespace sidon;

static int grid_for(size_t work, int threads) {
  const size_t want = (work + threads - 1) / threads;
  const size_t cap = (size_t)sm_count() * 8;
  return (int)(want < 1 ? 1 : (want > cap ? cap : want));
}

int launch_refine(const void* src, int n, int P, void* dst, int dtype, cudaStream_t st) {
  const size_t total = (size_t)n * P;
  if (dtype == SIDON_F32) {
    const bool aligned = (((uintptr_t)src | (uintptr_t)dst) & 15) == 0;
    if (!aligned) return SIDON_ERR_ARG;
    k_refine_f32<<<grid_for(total / 4 + 1, 256), 256, 0, st>>>((const float*)src, (float*)dst, total);
  } else {
    if (((uintptr_t)dst & 15) != 0) return SIDON_ERR_ARG;
    k_refine_f64<<<grid_for(total, 256), 256, 0, st>>>((const double*)src, (double*)dst, total);
  }
  return check_launch();
}

int launch_coarsen(const void* src, int n2, int P, void* dst, int dtype, cudaStream_t st) {
  const size_t total = (size_t)(n2 / 2) * P;
  if (dtype == SIDON_F32) {
    if (((uintptr_t)src & 7) != 0) return SIDON_ERR_ARG;
    k_coarsen_f32<<<grid_for(total, 256), 256, 0, st>>>((const float*)src, (float*)dst, total);
  } else {
    if (((uintptr_t)src & 15) != 0) return SIDON_ERR_ARG;
    k_coarsen_f64<<<grid_for(total, 256), 256, 0, st>>>((const double*)src, (double*)dst, total);
  }
  return check_launch();
}

int launch_resample(const float* src, int m, int P, float* dst, int n, int normalise,
                    cudaStream_t st) {
  k_resample<<<P, 256, 0, st>>>(src, m, dst, n, normalise);
  return check_launch();
}

int launch_island_migrate(float* pop, int n, double* fit, int P, int NI, int k, int* order,
                          cudaStream_t st) {
  const int PI = P / NI;
  int L = 1;
  while (L < PI) L <<= 1;
  const size_t sm = (size_t)L * (sizeof(double) + sizeof(int));
  k_island_rank<<<NI, 256, sm, st>>>(fit, PI, order);
  int rc = check_launch();
  if (rc) return rc;
  if (k > 0) {
    const int vec = ((n & 3) == 0) && (((uintptr_t)pop & 15) == 0);
    k_island_migrate<<<NI * k, 256, 0, st>>>(pop, n, fit, NI, PI, k, order, vec);
    rc = check_launch();
  }
  return rc;
}

int launch_island_migrate_ragged(float* pop, const long long* offsets, double* fit, int P, int NI,
                                 int k, int* order, cudaStream_t st) {
  const int PI = P / NI;
  int L = 1;
  while (L < PI) L <<= 1;
  const size_t sm = (size_t)L * (sizeof(double) + sizeof(int));
  k_island_rank<<<NI, 256, sm, st>>>(fit, PI, order);
  int rc = check_launch();
  if (rc) return rc;
  if (k > 0) {
    k_island_migrate_ragged<<<NI * k, 256, 0, st>>>(pop, offsets, fit, NI, PI, k, order);
    rc = check_launch();
  }
  return rc;
}

int launch_ragged_order(const long long* offsets, int P, int* order, cudaStream_t st) {
  k_ragged_order<<<grid_for((size_t)P, 128), 128, 0, st>>>(offsets, P, order);
  return check_launch();
}

}  // namespace sidon_host
