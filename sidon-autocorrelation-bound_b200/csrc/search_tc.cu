// ---------------------------------------------------------------------------
//  search_tc.cu -- tensor-core (tcgen05, BF16x3 / BF16x1) kernels:
//    k_local_search_tc  fused L^p-annealed projected Adam / mirror descent
//                       (src/kernels.cuh:177-289) with the convolution and the
//                       adjoint correlation on the tensor cores
//    k_lp_forward_tc    G_p(a) and {M, S, R}, optionally b
//    k_lp_backward_tc   dG_p/da with b recomputed on the tensor cores
//
//  One CTA (8 warps) per candidate, one CTA per SM (the shared-memory
//  working set is ~17 n bytes), 512 TMEM columns: accumulator of the
//  convolution at column 0, of the correlation at column 256.  The
//  elementwise work (max, weights, Adam) runs on the 8 warps reading TMEM.
//
//  Shared memory (offsets 1 KB aligned):
//    stages  STAGES x 8 KB   Hankel windows (hi | lo planes)
//    bc      2 x rc x 256 B  row-shifted block-matrix copies (two hi slots,
//                            or one hi + lo pair for the correlation)
//    sa      fp32 heights in the padded block layout (cell i at i + 4 floor(i/128)),
//            zero margins of >= 128 cells on both sides
//    crev    fp32 reversed weights c_rev[t] = c[2 m L - 2 - t], zero margin
//    red     64 floats of reduction scratch, mbarriers, TMEM address, abort flag
// ---------------------------------------------------------------------------
#include "conv_simt.cuh"
#include "tc_engine.cuh"

namespace sidon {
namespace tc {

__device__ unsigned int g_status_word = 0u;   // SIDON_ERR_TIMEOUT after a timed-out wait

struct Layout {
  int m, rc, sa_len, crev_len;
  size_t off_bc, off_sa, off_crev, off_red, total;
  __host__ __device__ Layout(int n, bool with_crev) {
    m = (n + L - 1) / L;
    rc = round_up(ZP + m + 24, 8);   // whole 8-row core-matrix groups
    sa_len = 132 * (m + 6);
    crev_len = with_crev ? (2 * L * m + 512) : 0;
    size_t o = (size_t)STAGES * STAGE_BYTES;
    off_bc = o;
    o += (size_t)2 * rc * 256;
    off_sa = o;
    o += (size_t)sa_len * 4;
    o = (o + 1023) & ~(size_t)1023;
    off_crev = o;
    o += (size_t)crev_len * 4;
    o = (o + 15) & ~(size_t)15;
    off_red = o;
    o += 64 * 4 + (2 * STAGES + 5) * 8 + 16;
    total = o + 1024;   // slack for aligning the dynamic base to 1 KB
  }
};

struct Shared {
  Ctx C;
  float* sa;     // cell 0
  float* crev;   // element 0
  float* red;
};

__device__ __forceinline__ Shared setup(int n, bool with_crev, bool three, unsigned char* raw) {
  const Layout Lo(n, with_crev);
  unsigned char* base = (unsigned char*)(((uintptr_t)raw + 1023) & ~(uintptr_t)1023);
  Shared S;
  S.C.stages = base;
  S.C.bc = base + Lo.off_bc;
  S.sa = reinterpret_cast<float*>(base + Lo.off_sa) + 132;
  S.crev = reinterpret_cast<float*>(base + Lo.off_crev);
  S.red = reinterpret_cast<float*>(base + Lo.off_red);
  uint64_t* bars = reinterpret_cast<uint64_t*>(S.red + 64);
  S.C.full = bars;
  S.C.empty = bars + STAGES;
  S.C.bc_full = bars + 2 * STAGES;
  S.C.bc_empty = bars + 2 * STAGES + 2;
  S.C.bar_done = bars + 2 * STAGES + 4;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 2 * STAGES + 5);
  S.C.abort = reinterpret_cast<int*>(tslot + 1);
  S.C.m = Lo.m;
  S.C.rc = Lo.rc;
  S.C.n = n;
  S.C.three = three;
  S.C.done_use = 0;
  S.C.st_next = 0;
  S.C.bc_uses[0] = S.C.bc_uses[1] = 0;
#pragma unroll
  for (int s = 0; s < STAGES; ++s) S.C.uses[s] = 0;
  // zero the fp32 buffers (margins must stay zero)
  float* z0 = reinterpret_cast<float*>(base + Lo.off_sa);
  for (int i = threadIdx.x; i < Lo.sa_len; i += blockDim.x) z0[i] = 0.f;
  for (int i = threadIdx.x; i < Lo.crev_len; i += blockDim.x) S.crev[i] = 0.f;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&S.C.full[s], NBUILD_WARPS);
      mbar_init(&S.C.empty[s], 1);
    }
    for (int s = 0; s < 2; ++s) {
      mbar_init(&S.C.bc_full[s], NBUILD_WARPS);
      mbar_init(&S.C.bc_empty[s], 1);
    }
    mbar_init(S.C.bar_done, 1);
    mbar_fence_init();
    *S.C.abort = 0;
  }
  if ((threadIdx.x >> 5) == 0) tmem_alloc(tslot, 512);
  fence_before();
  __syncthreads();
  fence_after();
  S.C.tmem = *tslot;
  return S;
}

__device__ __forceinline__ void teardown(Shared& S) {
  fence_before();
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) {
    fence_after();
    tmem_dealloc(S.C.tmem, 512);
  }
}

// lane quadrant / column-half of the calling warp
struct Lane {
  int quad, half, r;
  __device__ Lane() {
    const int w = threadIdx.x >> 5;
    quad = w & 3;
    half = w >> 2;
    r = 32 * quad + (threadIdx.x & 31);
  }
};

// ------------------------------ local search ------------------------------
__global__ void __launch_bounds__(NTHREADS, 1)
k_local_search_tc(float* pop, float* mom, float* vel, const int* __restrict__ skip,
                  const int* __restrict__ mode_arr, int n, int iters, float pStart, float pEnd,
                  float lrStart, float lrEnd, float beta1, float beta2, int mode_default, int three,
                  unsigned int* status) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const int pid = blockIdx.x;
  if (skip && skip[pid]) return;
  const int mode = mode_arr ? mode_arr[pid] : mode_default;
  float* a = pop + (size_t)pid * n;
  float* mg = mom + (size_t)pid * n;
  float* vg = vel + (size_t)pid * n;

  Shared S = setup(n, true, three != 0, smem_raw);
  Ctx& C = S.C;
  const int m = C.m, nb = 2 * n - 1;
  const int W = acc_width(m);
  const Lane ln;
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) { S.sa[pidx(i)] = a[i]; mg[i] = 0.f; vg[i] = 0.f; }
  __syncthreads();

  const float lnPr = (float)log((double)pEnd / (double)pStart);
  const float lnLr = (float)log((double)lrEnd / (double)lrStart);
  float b1t = 1.f, b2t = 1.f;
  const int nch = (2 * m + 31) / 32;

  for (int it = 0; it < iters; ++it) {
    const float frac = iters > 1 ? (float)it / (float)(iters - 1) : 0.f;
    const float pexp = pStart * expf(lnPr * frac);
    const float lr = lrStart * expf(lnLr * frac);

    zero_acc(C, COL_CONV, W);
    zero_acc(C, COL_CORR, W);
    fence_before();
    __syncthreads();
    if (!conv_tc(C, S.sa, status)) break;

    // M = max b
    float mloc = 0.f;
    for (int c = ln.half; c < nch; c += 2) {
      float v[32];
      tmem_ld32(C.tmem + ((uint32_t)(32 * ln.quad) << 16) + (uint32_t)(COL_CONV + 32 * c), v);
#pragma unroll
      for (int t = 0; t < 32; ++t) {
        const int k = (32 * c + t) * L + ln.r;
        if (k < nb) mloc = fmaxf(mloc, v[t]);
      }
    }
    const float M = block_max(mloc, S.red);
    if (!(M > 0.f)) break;
    // c_k = (1+d)^(p-1), R = sum c_k (1+d); stored reversed for the correlation
    float rloc = 0.f;
    for (int c = ln.half; c < nch; c += 2) {
      float v[32];
      tmem_ld32(C.tmem + ((uint32_t)(32 * ln.quad) << 16) + (uint32_t)(COL_CONV + 32 * c), v);
#pragma unroll
      for (int t = 0; t < 32; ++t) {
        const int k = (32 * c + t) * L + ln.r;
        if (k < nb) {
          const float d = (v[t] - M) / M;
          const float cw = d > -1.f ? pow_from_d(d, pexp - 1.f) : 0.f;
          rloc += cw * (1.f + d);
          S.crev[2 * L * m - 2 - k] = cw;
        }
      }
    }
    const float R = block_sum(rloc, S.red);   // barrier: crev complete
    b1t *= beta1;
    b2t *= beta2;
    const float bc1 = 1.f / (1.f - b1t), bc2 = 1.f / (1.f - b2t);
    const float lrn = lr / (float)n;

    fence_before();
    __syncthreads();
    if (!corr_tc(C, S.sa, S.crev, status)) break;

    float sloc = 0.f;
    for (int c = ln.half; c < nch; c += 2) {
      float v[32];
      tmem_ld32(C.tmem + ((uint32_t)(32 * ln.quad) << 16) + (uint32_t)(COL_CORR + 32 * c), v);
#pragma unroll
      for (int t = 0; t < 32; ++t) {
        const int col = 32 * c + t;
        if (col < m - 1 || col >= 2 * m - 1) continue;
        const int i = (2 * m - 2 - col) * L + L - 1 - ln.r;
        if (i >= n) continue;
        const float gi = v[t] / R - M;
        float x;
        if (mode == 0) {
          const float mm = __fmaf_rn(beta1, mg[i], (1.f - beta1) * gi);
          const float vv = __fmaf_rn(beta2, vg[i], (1.f - beta2) * gi * gi);
          mg[i] = mm;
          vg[i] = vv;
          const float step = lrn * (mm * bc1) / (sqrtf(vv * bc2) + 1e-30f);
          x = S.sa[pidx(i)] - step;
          if (x < 0.f) x = 0.f;
        } else {
          float e = -lr * (gi / M);
          if (e > 4.f) e = 4.f;
          if (e < -4.f) e = -4.f;
          x = S.sa[pidx(i)] * expf(e);
        }
        S.sa[pidx(i)] = x;
        sloc += x;
      }
    }
    float Ssum = block_sum(sloc, S.red);
    if (!(Ssum > 0.f)) {
      for (int i = threadIdx.x; i < n; i += blockDim.x) S.sa[pidx(i)] = 1.f / (float)n;
      Ssum = 1.f;
    }
    const float inv = 1.f / Ssum;
    for (int i = threadIdx.x; i < n; i += blockDim.x) S.sa[pidx(i)] *= inv;
    __syncthreads();
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) a[i] = S.sa[pidx(i)];
  teardown(S);
}

// ------------------------------ G_p forward -------------------------------
__global__ void __launch_bounds__(NTHREADS, 1)
k_lp_forward_tc(const float* __restrict__ pop, int n, float p, float* __restrict__ value,
                float* __restrict__ saved, float* __restrict__ b_out, int three,
                unsigned int* status) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const int pid = blockIdx.x;
  Shared S = setup(n, false, three != 0, smem_raw);
  Ctx& C = S.C;
  const int m = C.m, nb = 2 * n - 1, W = acc_width(m), nch = (2 * m + 31) / 32;
  const Lane ln;
  const float* a = pop + (size_t)pid * n;
  __syncthreads();
  float sl = 0.f;
  for (int i = threadIdx.x; i < n; i += blockDim.x) { const float x = a[i]; S.sa[pidx(i)] = x; sl += x; }
  const float Ssum = block_sum(sl, S.red);
  zero_acc(C, COL_CONV, W);
  fence_before();
  __syncthreads();
  const bool ok = conv_tc(C, S.sa, status);
  float mloc = 0.f;
  if (ok) {
    for (int c = ln.half; c < nch; c += 2) {
      float v[32];
      tmem_ld32(C.tmem + ((uint32_t)(32 * ln.quad) << 16) + (uint32_t)(COL_CONV + 32 * c), v);
#pragma unroll
      for (int t = 0; t < 32; ++t) {
        const int k = (32 * c + t) * L + ln.r;
        if (k < nb) {
          mloc = fmaxf(mloc, v[t]);
          if (b_out) b_out[(size_t)pid * nb + k] = v[t];
        }
      }
    }
  }
  const float M = block_max(mloc, S.red);
  float rloc = 0.f;
  if (ok) {
    for (int c = ln.half; c < nch; c += 2) {
      float v[32];
      tmem_ld32(C.tmem + ((uint32_t)(32 * ln.quad) << 16) + (uint32_t)(COL_CONV + 32 * c), v);
#pragma unroll
      for (int t = 0; t < 32; ++t) {
        const int k = (32 * c + t) * L + ln.r;
        if (k < nb) {
          const float d = (v[t] - M) / M;
          rloc += d > -1.f ? pow_from_d(d, p) : 0.f;
        }
      }
    }
  }
  const float R = block_sum(rloc, S.red);
  if (threadIdx.x == 0) {
    const float val = ok ? 2.f * (float)n * M * powf(R, 1.f / p) / (Ssum * Ssum)
                         : __int_as_float(0x7fc00000);
    value[pid] = val;
    saved[4 * pid + 0] = M;
    saved[4 * pid + 1] = Ssum;
    saved[4 * pid + 2] = R;
    saved[4 * pid + 3] = val;
  }
  teardown(S);
}

// ------------------------------ G_p backward ------------------------------
__global__ void __launch_bounds__(NTHREADS, 1)
k_lp_backward_tc(const float* __restrict__ pop, const float* __restrict__ saved,
                 const float* __restrict__ b_in, int n, float p, float* __restrict__ grad,
                 int three, unsigned int* status) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const int pid = blockIdx.x;
  Shared S = setup(n, true, three != 0, smem_raw);
  Ctx& C = S.C;
  const int m = C.m, nb = 2 * n - 1, W = acc_width(m), nch = (2 * m + 31) / 32;
  const Lane ln;
  const float* a = pop + (size_t)pid * n;
  const float M = saved[4 * pid + 0], Ssum = saved[4 * pid + 1], R = saved[4 * pid + 2];
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) S.sa[pidx(i)] = a[i];
  __syncthreads();
  zero_acc(C, COL_CONV, W);
  zero_acc(C, COL_CORR, W);
  fence_before();
  __syncthreads();
  bool ok = true;
  if (b_in) {
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
      const float d = (b_in[(size_t)pid * nb + k] - M) / M;
      S.crev[2 * L * m - 2 - k] = d > -1.f ? pow_from_d(d, p - 1.f) : 0.f;
    }
  } else {
    ok = conv_tc(C, S.sa, status);
    if (ok) {
      for (int c = ln.half; c < nch; c += 2) {
        float v[32];
        tmem_ld32(C.tmem + ((uint32_t)(32 * ln.quad) << 16) + (uint32_t)(COL_CONV + 32 * c), v);
#pragma unroll
        for (int t = 0; t < 32; ++t) {
          const int k = (32 * c + t) * L + ln.r;
          if (k < nb) {
            const float d = (v[t] - M) / M;
            S.crev[2 * L * m - 2 - k] = d > -1.f ? pow_from_d(d, p - 1.f) : 0.f;
          }
        }
      }
    }
  }
  fence_before();
  __syncthreads();
  if (ok) ok = corr_tc(C, S.sa, S.crev, status);
  const float scale = 4.f * (float)n * powf(R, 1.f / p) / (Ssum * Ssum);
  const float MS = M / Ssum;
  float* g = grad + (size_t)pid * n;
  if (ok) {
    for (int c = ln.half; c < nch; c += 2) {
      float v[32];
      tmem_ld32(C.tmem + ((uint32_t)(32 * ln.quad) << 16) + (uint32_t)(COL_CORR + 32 * c), v);
#pragma unroll
      for (int t = 0; t < 32; ++t) {
        const int col = 32 * c + t;
        if (col < m - 1 || col >= 2 * m - 1) continue;
        const int i = (2 * m - 2 - col) * L + L - 1 - ln.r;
        if (i < n) g[i] = scale * (v[t] / R - MS);
      }
    }
  }
  teardown(S);
}

}  // namespace tc
}  // namespace sidon

// =========================== host launch wrappers ==========================
namespace sidon_host {
using namespace sidon;

static unsigned int* status_word() {
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, tc::g_status_word) != cudaSuccess) return nullptr;
  return (unsigned int*)p;
}

int device_status(int reset) {
  unsigned int v = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&v, tc::g_status_word, sizeof(v));
  if (e != cudaSuccess) return set_cuda_error(e);
  if (reset) {
    const unsigned int z = 0;
    e = cudaMemcpyToSymbol(tc::g_status_word, &z, sizeof(z));
    if (e != cudaSuccess) return set_cuda_error(e);
  }
  return (int)v;
}

size_t smem_local_search_tc(int n) { return tc::Layout(n, true).total; }
static size_t smem_lp_forward_tc(int n) { return tc::Layout(n, false).total; }

static int tc_n_ok(int n) {
  const int m = (n + tc::L - 1) / tc::L;
  return (n >= 1 && 2 * round_up(2 * m + 16, 32) <= 512) ? SIDON_OK : SIDON_ERR_N;
}

static int prep_tc(const void* fn, size_t sm) {
  if ((long long)sm > (long long)smem_optin()) return SIDON_ERR_SMEM;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return set_cuda_error(e);
  return SIDON_OK;
}

int launch_local_search_tc(float* pop, float* mom, float* vel, const int* skip,
                           const int* mode_arr, int n, int P, int iters, double pS, double pE,
                           double lrS, double lrE, double b1, double b2, int mode_default,
                           int precision, cudaStream_t st) {
  int rc = tc_n_ok(n);
  if (rc) return rc;
  const size_t sm = smem_local_search_tc(n);
  rc = prep_tc((const void*)tc::k_local_search_tc, sm);
  if (rc) return rc;
  unsigned int* sw = status_word();
  if (!sw) return SIDON_ERR_CUDA;
  tc::k_local_search_tc<<<P, tc::NTHREADS, sm, st>>>(
      pop, mom, vel, skip, mode_arr, n, iters, (float)pS, (float)pE, (float)lrS, (float)lrE,
      (float)b1, (float)b2, mode_default, precision == SIDON_PREC_BF16X3 ? 1 : 0, sw);
  return check_launch();
}

int launch_lp_forward_tc(const float* a, int n, int P, double p, float* value, float* saved,
                         float* b_out, int precision, cudaStream_t st) {
  int rc = tc_n_ok(n);
  if (rc) return rc;
  const size_t sm = smem_lp_forward_tc(n);
  rc = prep_tc((const void*)tc::k_lp_forward_tc, sm);
  if (rc) return rc;
  unsigned int* sw = status_word();
  if (!sw) return SIDON_ERR_CUDA;
  tc::k_lp_forward_tc<<<P, tc::NTHREADS, sm, st>>>(a, n, (float)p, value, saved, b_out,
                                                  precision == SIDON_PREC_BF16X3 ? 1 : 0, sw);
  return check_launch();
}

int launch_lp_backward_tc(const float* a, const float* saved, const float* b_in, int n, int P,
                          double p, float* grad, int precision, cudaStream_t st) {
  int rc = tc_n_ok(n);
  if (rc) return rc;
  const size_t sm = smem_local_search_tc(n);
  rc = prep_tc((const void*)tc::k_lp_backward_tc, sm);
  if (rc) return rc;
  unsigned int* sw = status_word();
  if (!sw) return SIDON_ERR_CUDA;
  tc::k_lp_backward_tc<<<P, tc::NTHREADS, sm, st>>>(a, saved, b_in, n, (float)p, grad,
                                                   precision == SIDON_PREC_BF16X3 ? 1 : 0, sw);
  return check_launch();
}

}  // namespace sidon_host
