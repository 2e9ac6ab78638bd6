// ---------------------------------------------------------------------------
//  search_tc.cu -- tensor-core (tcgen05, BF16x3 / BF16x1) kernels:
//    k_local_search_tc  fused L^p-annealed projected Adam / mirror descent
//                       (src/kernels.cuh:177-289) with the convolution and the
//                       adjoint correlation on the tensor cores
//    k_lp_forward_tc    G_p(a) and {M, S, R}, optionally b
//    k_lp_backward_tc   dG_p/da with b recomputed on the tensor cores
//
//    k_frank_wolfe_tc   Chambolle-Pock Frank-Wolfe (src/kernels.cuh:408-532)
//
//  One CTA (8 warps) per candidate, one CTA per SM (the shared-memory
//  working set is ~24 n bytes, tc_cta.cuh), 512 TMEM columns: the
//  convolution accumulator at column 0, the correlation accumulator after
//  it.  The elementwise work (max, weights, Adam) runs on all 8 warps; the
//  weights beyond 2n-1 stay zero for the whole launch (the correlation
//  copies read whole blocks).
// ---------------------------------------------------------------------------
#include <algorithm>
#include <mutex>
#include <utility>
#include <vector>

#include "conv_simt.cuh"
#include "tc_cta.cuh"

// Phase marks inside the fused step: no code unless a profiling build
// defines SIDON_PHASE(k) (phase k of the step has just ended).
#ifndef SIDON_PHASE
#define SIDON_PHASE(k)
#endif

namespace sidon {
namespace tc {

// the device status word and the wait limit (common.cuh DeviceState)
__device__ DeviceState g_dev_state = {0u, 0u, kDefaultWaitCycles};

// cells per thread of the fused step's elementwise update: every n the
// kernels accept (conv + corr accumulators within 512 TMEM columns, n <= 9728)
// is covered by kCellsPerThread * NTHREADS
constexpr int kCellsPerThread = 26;

// ------------------------------ local search ------------------------------
// Heights must be finite and non-negative; a candidate that is not is
// computed anyway (as the reference would) and SIDON_ERR_NONFINITE is
// recorded in the status word (sidon_device_status).  bad: this thread saw one.
__device__ __forceinline__ bool bad_height(float x) { return !(x >= 0.f && x <= 3.402823466e38f); }
__device__ __forceinline__ void note_bad(bool bad, unsigned int* status) {
  if (bad) atomicCAS(status, 0u, (unsigned int)SIDON_ERR_NONFINITE);
}

// The autoconvolution's B copy of the heights in S.sa (the layout of
// build_conv_copy, hi plane), written by all threads before a candidate's
// first step; each step's renormalisation writes the next one.  Every step
// then takes the prebuilt form of the tile phase, so the kernels hold one
// copy of the convolution's tile code (measured: 3-20% faster steps than
// holding both forms, as long as the code stays small).  The caller
// synchronises before the step.
__device__ __forceinline__ void write_conv_copy(Shared& S) {
  Ctx& C = S.C;
  const int rows = C.rc;
  for (int cq = threadIdx.x; cq < rows * 8; cq += NTHREADS) {
    const int h = cq / rows, x = cq - h * rows, J = x - ZP;
    float v[8];
    if (J >= 0 && J < C.m) {
      // cells 64 J + 56 - 8 h .. + 7, reversed (zero beyond n in the padding)
      const float* q = S.sa + pidx(64 * J + 56 - 8 * h);
      const float4 u0 = *reinterpret_cast<const float4*>(q);
      const float4 u1 = *reinterpret_cast<const float4*>(q + 4);
      v[0] = u1.w; v[1] = u1.z; v[2] = u1.y; v[3] = u1.x;
      v[4] = u0.w; v[5] = u0.z; v[6] = u0.y; v[7] = u0.x;
    } else {
#pragma unroll
      for (int t = 0; t < 8; ++t) v[t] = 0.f;
    }
    conv_copy_chunk(C, x, h, v);
  }
  fence_async_smem();
}

// One L^p-Adam / mirror step of the candidate resident in S (n cells; its
// Adam moments in the global rows mg, vg; the autoconvolution copy of the
// heights in place): convolution, max, weights written into the correlation
// copy, correlation, update, renormalisation, and the next step's
// autoconvolution copy.  b1t / b2t are beta^(step+1).  Returns 0, or 1 when
// M <= 0 stops the anneal (nothing changed), or 2 when a tile phase was
// aborted.  Ends synchronised.
__device__ __forceinline__ int lp_adam_step(Shared& S, const Lane& ln, int n, int mode,
                                            float pexp, float lr, float beta1, float beta2,
                                            float b1t, float b2t, float* mg, float* vg,
                                            unsigned int* status) {
  Ctx& C = S.C;
  const int nb = 2 * n - 1;
  SIDON_PHASE(0);
  prime(C, true);
  SIDON_PHASE(1);
  if (!conv_tc_prebuilt(C, S.sa, status)) return 2;
  SIDON_PHASE(2);
  const float M = block_max(gather_conv(C, ln, S.cb), S.red);   // b in cb
  SIDON_PHASE(3);
  if (!(M > 0.f)) return 1;
  // c_k = (1+d)^(p-1), R = sum c_k (1+d), d = (b_k - M)/M, written straight
  // into the correlation's B copy: thread q takes chunks (row x, K group h)
  // = the 8 weights from 64 x + 8 h on (8 independent k per chunk), rows
  // beyond the 2m weight blocks are zero
  float rloc = 0.f;
  const float invM = 1.f / M, q = pexp - 1.f;
  {
    const int rows = C.rcc, nch8 = rows * 8;
    for (int cq = threadIdx.x; cq < nch8; cq += NTHREADS) {
      const int h = cq / rows, x = cq - h * rows;
      const int k0 = 64 * x + 8 * h;
      float v[8];
      if (k0 < nb) {
        const float4 u0 = *reinterpret_cast<const float4*>(S.cb + pidx(k0));
        const float4 u1 = *reinterpret_cast<const float4*>(S.cb + pidx(k0) + 4);
        const float bv[8] = {u0.x, u0.y, u0.z, u0.w, u1.x, u1.y, u1.z, u1.w};
#pragma unroll
        // (lanes beyond 2n-1 read the zeros begin() wrote or what the window
        // ring, which shares the scratch's region, left there: bf16 pairs of
        // finite heights, finite as fp32; their weight 0 times (1 + d) adds
        // exactly 0 to R)
        for (int j = 0; j < 8; ++j) {
          const float d = (bv[j] - M) * invM;
          const float cw = (k0 + j < nb && d > -1.f) ? pow_from_d_fast(d, q) : 0.f;
          rloc += cw * (1.f + d);
          v[j] = cw;
        }
      } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = 0.f;
      }
      corr_copy_chunk(C, x, h, v);
    }
    fence_async_smem();
  }
  const float R = block_sum(rloc, S.red);      // barrier: weights complete
  SIDON_PHASE(4);
  const float bc1 = 1.f / (1.f - b1t), bc2 = 1.f / (1.f - b2t);
  const float lrn = lr / (float)n;

  // the Adam moments of this thread's cells, loaded now so that the
  // correlation phase hides their L2 / HBM latency
  float pm[kCellsPerThread], pv[kCellsPerThread];
  static_assert(kCellsPerThread % 2 == 0, "the update takes cells in pairs");
  if (mode == 0) {
#pragma unroll
    for (int u = 0; u < kCellsPerThread; ++u) {
      const int i = threadIdx.x + u * NTHREADS;
      if (i >= n) break;        // the cells of a thread ascend: none further
      pm[u] = __ldcg(mg + i);
      pv[u] = __ldcg(vg + i);
    }
  }
  fence_before();
  __syncthreads();
  SIDON_PHASE(5);
  if (!corr_tc_prebuilt(C, S.sa, status)) return 2;
  SIDON_PHASE(6);
  gather_corr(C, ln, S.cb);                     // G in cb
  SIDON_PHASE(7);

  // Adam / mirror step (cells i = thread + u * NTHREADS), two cells at a
  // time so that their dependent chains (the division and the square root)
  // interleave; the second cell of the last pair is computed past n from the
  // zero padding and dropped.  The sum runs in cell order as before.
  float sloc = 0.f;
  const float invR = 1.f / R;
  auto new_height = [&](int u, int i, bool keep) {
    const float gi = S.cb[pidx(i)] * invR - M;
    const float x0 = S.sa[pidx(i)];
    float x;
    if (mode == 0) {
      const float mm = __fmaf_rn(beta1, pm[u], (1.f - beta1) * gi);
      const float vv = __fmaf_rn(beta2, pv[u], (1.f - beta2) * gi * gi);
      if (keep) {
        mg[i] = mm;
        vg[i] = vv;
      }
      // (hardware square root and fast division, about 2 ulp each; the
      // denominator lies in [1e-30, 2^126]; measured: update 6.9k -> 5.8k
      // cycles at n = 8400 against sqrtf)
      float sq;
      asm("sqrt.approx.f32 %0, %1;" : "=f"(sq) : "f"(vv * bc2));
      const float step = lrn * __fdividef(mm * bc1, sq + 1e-30f);
      x = x0 - step;
      if (x < 0.f) x = 0.f;
    } else {
      float e = -lr * (gi * invM);
      if (e > 4.f) e = 4.f;
      if (e < -4.f) e = -4.f;
      x = x0 * __expf(e);
    }
    return x;
  };
#pragma unroll
  for (int u = 0; u < kCellsPerThread; u += 2) {
    const int i0 = threadIdx.x + u * NTHREADS, i1 = i0 + NTHREADS;
    if (i0 >= n) break;         // (a tail predicated over all pairs would cost them all at small n)
    const bool has1 = i1 < n;
    const float x0 = new_height(u, i0, true);
    const float x1 = new_height(u + 1, i1, has1);
    S.sa[pidx(i0)] = x0;
    sloc += x0;
    if (has1) {
      S.sa[pidx(i1)] = x1;
      sloc += x1;
    }
  }
  // renormalise (sum <= 0: the uniform 1/n), chunk by chunk of 8 cells,
  // and write the next step's autoconvolution B copy from the same chunks
  const float Ssum = block_sum(sloc, S.red);
  SIDON_PHASE(8);
  const bool reset = !(Ssum > 0.f);
  const float inv = 1.f / (reset ? 1.f : Ssum);
  const float uniform = 1.f / (float)n;
  {
    const int rows = C.rc;
    for (int cq = threadIdx.x; cq < rows * 8; cq += NTHREADS) {
      const int h = cq / rows, x = cq - h * rows, J = x - ZP;
      float v[8];
      if (J >= 0 && J < C.m) {
        const int c0 = 64 * J + 56 - 8 * h;
        float* q = S.sa + pidx(c0);
        float4 u0 = *reinterpret_cast<float4*>(q);
        float4 u1 = *reinterpret_cast<float4*>(q + 4);
        float w[8] = {u0.x, u0.y, u0.z, u0.w, u1.x, u1.y, u1.z, u1.w};
#pragma unroll
        for (int j = 0; j < 8; ++j)
          if (c0 + j < n) w[j] = (reset ? uniform : w[j]) * inv;
        u0 = make_float4(w[0], w[1], w[2], w[3]);
        u1 = make_float4(w[4], w[5], w[6], w[7]);
        *reinterpret_cast<float4*>(q) = u0;
        *reinterpret_cast<float4*>(q + 4) = u1;
#pragma unroll
        for (int t = 0; t < 8; ++t) v[t] = w[7 - t];
      } else {
#pragma unroll
        for (int t = 0; t < 8; ++t) v[t] = 0.f;
      }
      conv_copy_chunk(C, x, h, v);
    }
    fence_async_smem();
  }
  __syncthreads();
  SIDON_PHASE(9);
  return 0;
}


// Candidates: uniform rows of n_fixed cells (offsets == NULL) or a ragged
// batch (row p = pop[offsets[p] .. offsets[p+1])).  CTA b runs slots
// b, b + gridDim.x, ... of `order` (NULL = 0..P-1): launched with one CTA per
// candidate it is the plain batched kernel, launched with one CTA per SM and
// a longest-first order it is the persistent ragged kernel.
__global__ void __launch_bounds__(NTHREADS, 1)
k_local_search_tc(float* pop, float* mom, float* vel, const long long* __restrict__ offsets,
                  const int* __restrict__ order, int P, int n_fixed, int n_max,
                  const int* __restrict__ skip, const int* __restrict__ mode_arr, int iters,
                  float pStart, float pEnd, float lrStart, float lrEnd, float beta1, float beta2,
                  int mode_default, int three, unsigned int* status, int ring) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  Shared S = setup(n_max, three != 0, smem_raw, ring, true);
  Ctx& C = S.C;
  const Lane ln;
  for (int slot = blockIdx.x; slot < P; slot += gridDim.x) {
  const int pid = order ? order[slot] : slot;
  if (skip && skip[pid]) continue;
  const long long off = offsets ? offsets[pid] : (long long)pid * n_fixed;
  const int n = offsets ? (int)(offsets[pid + 1] - off) : n_fixed;
  if (n < 1 || n > n_max) continue;
  if (*((volatile int*)C.abort)) break;
  const int mode = mode_arr ? mode_arr[pid] : mode_default;
  float* a = pop + off;
  float* mg = mom + off;
  float* vg = vel + off;
  begin(S, n, n_max);
  bool bad = false;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float x = a[i];
    bad |= bad_height(x);
    S.sa[pidx(i)] = x;
    mg[i] = 0.f;
    vg[i] = 0.f;
  }
  note_bad(bad, status);
  __syncthreads();
  write_conv_copy(S);
  __syncthreads();

  const float lnPr = (float)log((double)pEnd / (double)pStart);
  const float lnLr = (float)log((double)lrEnd / (double)lrStart);
  float b1t = 1.f, b2t = 1.f;

  for (int it = 0; it < iters; ++it) {
    const float frac = iters > 1 ? (float)it / (float)(iters - 1) : 0.f;
    const float pexp = pStart * expf(lnPr * frac);
    const float lr = lrStart * expf(lnLr * frac);

    b1t *= beta1;
    b2t *= beta2;
    const int rs = lp_adam_step(S, ln, n, mode, pexp, lr, beta1, beta2, b1t, b2t, mg, vg,
                                status);
    if (rs) break;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) a[i] = S.sa[pidx(i)];
  }  // candidates
  teardown(S);
}

// ------------------- local search, balanced step segments -------------------
// A uniform batch of P > G candidates (G = one resident CTA per SM) leaves SMs
// idle in the last wave of the one-CTA-per-candidate kernel (256 candidates on
// 148 SMs: 1.73 waves of work in 2 waves of time).  This kernel lays the P
// chains of `iters` steps end to end and gives CTA c the steps
// [c T / G, (c+1) T / G) of that sequence (T = P iters): at most three
// pieces -- the head of the candidate that continues into the next CTA's
// segment, whole candidates, the tail of the candidate begun by the previous
// CTA.  It runs the head first and raises that candidate's flag, and the tail
// last after waiting for its flag; as a segment holds at least `iters` steps
// (P >= G), the head is finished long before the next CTA reaches the tail,
// so the wait is a formality.  Heights and moments cross between CTAs through
// L2 (ld.global.cg); each step is lp_adam_step, the fused kernel's arithmetic,
// so every candidate's trajectory is the fused kernel's bit for bit.  The
// hand-over flags (one word per candidate) are caller memory, zeroed on the
// launch's stream before it starts, so launches on different streams with
// different flag words never see each other's; the wait gives up after the
// device state's wait limit (SIDON_ERR_TIMEOUT).

// steps [s0, s1) of candidate pid, its state read from and written to HBM
__device__ __forceinline__ void run_piece(Shared& S, const Lane& ln, float* pop, float* mom,
                                          float* vel, int pid, int n, int s0, int s1, int iters,
                                          int mode, float pStart, float lnPr, float lrStart,
                                          float lnLr, float beta1, float beta2,
                                          unsigned int* status) {
  float* a = pop + (size_t)pid * n;
  float* mg = mom + (size_t)pid * n;
  float* vg = vel + (size_t)pid * n;
  SIDON_PHASE(10);
  begin(S, n, n);
  load_heights(S, a, n);
  if (s0 == 0) {
    bool bad = false;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      bad |= bad_height(S.sa[pidx(i)]);
      mg[i] = 0.f;
      vg[i] = 0.f;
    }
    note_bad(bad, status);
  }
  write_conv_copy(S);
  __syncthreads();
  SIDON_PHASE(11);
  float b1t = 1.f, b2t = 1.f;
  for (int it = 0; it < s0; ++it) {        // beta^s0, multiplied up as the fused kernel does
    b1t *= beta1;
    b2t *= beta2;
  }
  int rs = 0;
  for (int it = s0; it < s1; ++it) {
    const float frac = iters > 1 ? (float)it / (float)(iters - 1) : 0.f;
    const float pexp = pStart * expf(lnPr * frac);
    const float lr = lrStart * expf(lnLr * frac);
    b1t *= beta1;
    b2t *= beta2;
    rs = lp_adam_step(S, ln, n, mode, pexp, lr, beta1, beta2, b1t, b2t, mg, vg, status);
    if (rs) break;          // M <= 0 stops the anneal; the heights are as they were
  }
  __syncthreads();
  if (rs != 2) {
    // back to the row, 16-byte groups where the row allows (see load_heights)
    if (((reinterpret_cast<uintptr_t>(a) & 15) == 0) && (n % 4 == 0)) {
      for (int q = threadIdx.x; q < n / 4; q += blockDim.x)
        reinterpret_cast<float4*>(a)[q] = *reinterpret_cast<const float4*>(S.sa + pidx(4 * q));
    } else {
      for (int i = threadIdx.x; i < n; i += blockDim.x) a[i] = S.sa[pidx(i)];
    }
  }
  SIDON_PHASE(12);
}

__global__ void __launch_bounds__(NTHREADS, 1)
k_local_search_tc_seg(float* pop, float* mom, float* vel, int P, int n,
                      const int* __restrict__ skip, const int* __restrict__ mode_arr, int iters,
                      float pStart, float pEnd, float lrStart, float lrEnd, float beta1,
                      float beta2, int mode_default, int three, unsigned int* status,
                      unsigned int* flags, int ring) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ int s_ok;
  Shared S = setup(n, three != 0, smem_raw, ring, true);
  SIDON_PHASE(15);
  const Lane ln;
  const float lnPr = (float)log((double)pEnd / (double)pStart);
  const float lnLr = (float)log((double)lrEnd / (double)lrStart);
  const long long T = (long long)P * iters, G = gridDim.x, c = blockIdx.x;
  const long long seg0 = c * T / G, seg1 = (c + 1) * T / G;
  if (seg1 > seg0) {
    const int first = (int)(seg0 / iters), last = (int)((seg1 - 1) / iters);
    const bool tail = (long long)first * iters < seg0;                 // begun by CTA c - 1
    const bool head = (long long)(last + 1) * iters > seg1;            // continued by CTA c + 1
    auto piece = [&](int pid) {
      const long long b0 = (long long)pid * iters;
      const int s0 = (int)((seg0 > b0 ? seg0 : b0) - b0);
      const int s1 = (int)((seg1 < b0 + iters ? seg1 : b0 + iters) - b0);
      if (!(skip && skip[pid]) && !*((volatile int*)S.C.abort))
        run_piece(S, ln, pop, mom, vel, pid, n, s0, s1, iters,
                  mode_arr ? mode_arr[pid] : mode_default, pStart, lnPr, lrStart, lnLr, beta1,
                  beta2, status);
    };
    // the pieces in order -- the head, the whole candidates, the tail --
    // through one call site, so the step loop is in the kernel once
    const int mid0 = tail ? first + 1 : first, mid1 = head ? last - 1 : last;
    const bool has_tail = tail && !(head && first == last);
    const int npieces = (head ? 1 : 0) + (mid1 >= mid0 ? mid1 - mid0 + 1 : 0) + (has_tail ? 1 : 0);
    for (int q = 0; q < npieces; ++q) {
      const bool is_head = head && q == 0, is_tail = has_tail && q == npieces - 1;
      const int pid = is_head ? last : is_tail ? first : mid0 + q - (head ? 1 : 0);
      if (is_tail) {
        if (threadIdx.x == 0) {
          s_ok = 1;
          volatile unsigned int* f = flags + first;
          const long long t0 = clock64(), lim = wait_limit(status);
          while (*f == 0u) {
            if (clock64() - t0 > lim) {
              s_ok = 0;
              atomicCAS(status, 0u, (unsigned int)SIDON_ERR_TIMEOUT);
              break;
            }
            __nanosleep(200);
          }
          __threadfence();
        }
        __syncthreads();
        if (!s_ok) break;
      }
      piece(pid);
      if (is_head) {
        __threadfence();        // every thread's heights and moments reach L2 ...
        __syncthreads();
        if (threadIdx.x == 0) atomicExch(&flags[last], 1u);   // ... before the flag
      }
    }
  }
  teardown(S);
}

// ------------------------------ G_p forward -------------------------------
// As k_lp_forward: M refined in fp64 over the near-maximal k (the split
// error of b is < 3e-5 of max b), S in fp64, R from the tensor-core b.
constexpr int kRefineCap = 1024;
static_assert(kRefineCap * sizeof(int) <= (size_t)3 * stage_bytes(1), "list fits the smallest ring");

__global__ void __launch_bounds__(NTHREADS, 1)
k_lp_forward_tc(const float* __restrict__ pop, int n, float p, float* __restrict__ value,
                float* __restrict__ saved, float* __restrict__ b_out, int three,
                unsigned int* status) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ int s_cnt;
  __shared__ double s_red[32];
  const int pid = blockIdx.x;
  Shared S = setup(n, three != 0, smem_raw);
  Ctx& C = S.C;
  // the refinement list lives in the window ring, idle outside tile phases
  int* s_list = reinterpret_cast<int*>(C.stages);
  begin(S, n, n);
  const int nb = 2 * n - 1;
  const Lane ln;
  const float* a = pop + (size_t)pid * n;
  double sl = 0.0;
  bool bad = false;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float x = a[i];
    bad |= bad_height(x);
    S.sa[pidx(i)] = x;
    sl += x;
  }
  note_bad(bad, status);
  const double Ssum = block_sum(sl, s_red);
  prime(C, false);
  const bool ok = conv_tc(C, S.sa, status);
  if (ok) gather_conv(C, ln, S.cb);
  float mloc = 0.f;
  if (ok)
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
      const float v = S.cb[pidx(k)];
      mloc = fmaxf(mloc, v);
      if (b_out) b_out[(size_t)pid * nb + k] = v;
    }
  const float Mapprox = block_max(mloc, S.red);
  const double Md = refine_max(
      n, [&](int i) { return S.sa[pidx(i)]; }, [&](int k) { return S.cb[pidx(k)]; }, Mapprox,
      2e-4f, s_list, kRefineCap, &s_cnt, s_red);
  const float M = (float)Md;
  float rloc = 0.f;
  if (ok)
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
      const float d = (S.cb[pidx(k)] - M) / M;
      rloc += d > -1.f ? pow_from_d_fast(d, p) : 0.f;
    }
  const float R = block_sum(rloc, S.red);
  if (threadIdx.x == 0) {
    const double val = 2.0 * (double)n * Md * pow((double)R, 1.0 / (double)p) / (Ssum * Ssum);
    const float v = ok ? (float)val : __int_as_float(0x7fc00000);
    value[pid] = v;
    saved[4 * pid + 0] = M;
    saved[4 * pid + 1] = (float)Ssum;
    saved[4 * pid + 2] = R;
    saved[4 * pid + 3] = v;
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
  Shared S = setup(n, three != 0, smem_raw);
  Ctx& C = S.C;
  begin(S, n, n);
  const int nb = 2 * n - 1;
  const Lane ln;
  const float* a = pop + (size_t)pid * n;
  const float M = saved[4 * pid + 0], Ssum = saved[4 * pid + 1], R = saved[4 * pid + 2];
  for (int i = threadIdx.x; i < n; i += blockDim.x) S.sa[pidx(i)] = a[i];
  __syncthreads();
  prime(C, true);
  bool ok = true;
  if (b_in) {
    for (int k = threadIdx.x; k < nb; k += blockDim.x) S.cb[pidx(k)] = b_in[(size_t)pid * nb + k];
    __syncthreads();
  } else {
    ok = conv_tc(C, S.sa, status);
    if (ok) gather_conv(C, ln, S.cb);
  }
  for (int k = threadIdx.x; k < nb; k += blockDim.x) {
    const float d = (S.cb[pidx(k)] - M) / M;
    S.cb[pidx(k)] = d > -1.f ? pow_from_d_fast(d, p - 1.f) : 0.f;
  }
  fence_before();
  __syncthreads();
  if (ok) ok = corr_tc(C, S.sa, S.cb, status);
  if (ok) gather_corr(C, ln, S.cb);
  const float scale = 4.f * (float)n * powf(R, 1.f / p) / (Ssum * Ssum);
  const float MS = M / Ssum;
  float* g = grad + (size_t)pid * n;
  if (ok)
    for (int i = threadIdx.x; i < n; i += blockDim.x) g[i] = scale * (S.cb[pidx(i)] / R - MS);
  teardown(S);
}

// --------------------------- Frank-Wolfe / PDHG ---------------------------
// The Chambolle-Pock Frank-Wolfe step of k_frank_wolfe (src/kernels.cuh:408-532)
// with its convolutions and correlations on the tensor cores:
//   lambda <- [lambda + sigma (a * gbar - M)]_+     a * gbar: CONV_X
//   g <- [g + tau (1 - corr(lambda, a))]_+           corr:     CORR
//   line search maxima of h * h, h = (1-t) a + t g:  CONV_SYM
// a stays in shared memory during the iterations, lambda in the weight
// buffer, the gather scratch in the copy region; g and gbar are plain global
// rows (caller scratch in pop's layout) that the copies read through L2.
// M and the line-search maxima are refined in fp64 over the near-maximal k
// (the tensor-core b is within 3e-5 of max b), so a move is accepted only if
// it lowers the refined maximum.
constexpr int kFwRefineCap = 1024;

__device__ __forceinline__ double refined_max_sa(const Shared& S, int n, float* X, int* list,
                                                 int* cnt, double* red) {
  const int nb = 2 * n - 1;
  float mloc = 0.f;
  for (int k = threadIdx.x; k < nb; k += blockDim.x) mloc = fmaxf(mloc, X[pidx(k)]);
  const float approx = block_max(mloc, S.red);
  if (!(approx > 0.f)) return 0.0;
  return refine_max(
      n, [&](int i) { return S.sa[pidx(i)]; }, [&](int k) { return X[pidx(k)]; }, approx, 2e-4f,
      list, kFwRefineCap, cnt, red);
}

__global__ void __launch_bounds__(NTHREADS, 1)
k_frank_wolfe_tc(float* pop, float* gbuf, float* gbbuf, const long long* __restrict__ offsets,
                 const int* __restrict__ order, int P, int n_fixed, int n_max,
                 const int* __restrict__ skip, int rounds, int pdhgIters, int nT, float tMax,
                 float tau_in, float sig_in, int three, unsigned int* status) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  __shared__ int s_cnt;
  __shared__ double s_red[32];
  Shared S = setup(n_max, three != 0, smem_raw);
  Ctx& C = S.C;
  // the refinement list lives in the window ring, idle outside tile phases
  int* s_list = reinterpret_cast<int*>(C.stages);
  const Lane ln;
  float* X = reinterpret_cast<float*>(C.bc);   // gather scratch (after a tile phase)
  bool alive = true;
  for (int slot = blockIdx.x; slot < P && alive; slot += gridDim.x) {
    const Cand cd = cand_of(slot, offsets, order, n_fixed);
    const int n = cd.n;
    if (skip && skip[cd.pid]) continue;
    if (n < 1 || n > n_max) continue;
    float* a = pop + cd.off;
    float* g = gbuf + cd.off;
    float* gb = gbbuf + cd.off;
    begin(S, n, n_max);
    const int nb = 2 * n - 1;
    float sl = 0.f;
    bool bad = false;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const float x = a[i];
      bad |= bad_height(x);
      S.sa[pidx(i)] = x;
      sl += x;
    }
    note_bad(bad, status);
    const float s0 = block_sum(sl, S.red);
    if (!(s0 > 0.f)) continue;
    {
      const float inv = 1.f / s0;
      for (int i = threadIdx.x; i < n; i += blockDim.x) S.sa[pidx(i)] *= inv;
      __syncthreads();
    }
    const float tau = tau_in > 0.f ? tau_in : 0.9f / (float)n;
    const float sig = sig_in > 0.f ? sig_in : 0.9f * (float)n;

    for (int r = 0; r < rounds; ++r) {
      prime(C, false);
      if (!conv_tc(C, S.sa, status)) { alive = false; break; }
      gather_conv(C, ln, X);
      const double Mref = refined_max_sa(S, n, X, s_list, &s_cnt, s_red);
      if (!(Mref > 0.0)) break;
      const float M = (float)Mref;
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const float x = S.sa[pidx(i)];
        g[i] = x;
        gb[i] = x;
        a[i] = x;                                  // the round's start, for the line search
      }
      for (int k = threadIdx.x; k < nb; k += blockDim.x) S.cb[pidx(k)] = 0.f;
      __syncthreads();

      for (int it = 0; it < pdhgIters; ++it) {
        prime(C, true);
        if (!convx_tc(C, S.sa, gb, n, status)) { alive = false; break; }
        gather_conv(C, ln, X);
        for (int k = threadIdx.x; k < nb; k += blockDim.x) {
          const float l = S.cb[pidx(k)] + sig * (X[pidx(k)] - M);
          S.cb[pidx(k)] = l > 0.f ? l : 0.f;
        }
        fence_before();
        __syncthreads();
        if (!corr_tc(C, S.sa, S.cb, status)) { alive = false; break; }
        gather_corr(C, ln, X);
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
          const float go = g[i];
          float gn = go + tau * (1.f - X[pidx(i)]);
          gn = gn > 0.f ? gn : 0.f;
          g[i] = gn;
          gb[i] = 2.f * gn - go;
        }
        __syncthreads();
      }
      if (!alive) break;

      float sg = 0.f;
      for (int i = threadIdx.x; i < n; i += blockDim.x) sg += g[i];
      sg = block_sum(sg, S.red);
      if (!(sg > 0.f)) break;
      const float ginv = 1.f / sg;
      for (int i = threadIdx.x; i < n; i += blockDim.x) g[i] *= ginv;
      __syncthreads();
      // sum a = sum g = 1  =>  F(h) = 2n max(h*h) for every t
      float bestT = 0.f;
      double bestM = Mref;
      for (int s = 1; s <= nT; ++s) {
        const float t = tMax * (float)s / (float)nT;
        for (int i = threadIdx.x; i < n; i += blockDim.x)
          S.sa[pidx(i)] = (1.f - t) * __ldcg(a + i) + t * __ldcg(g + i);
        __syncthreads();
        prime(C, false);
        if (!conv_tc(C, S.sa, status)) { alive = false; break; }
        gather_conv(C, ln, X);
        const double mm = refined_max_sa(S, n, X, s_list, &s_cnt, s_red);
        if (mm < bestM) { bestM = mm; bestT = t; }
      }
      if (!alive) break;
      for (int i = threadIdx.x; i < n; i += blockDim.x)
        S.sa[pidx(i)] = (1.f - bestT) * __ldcg(a + i) + bestT * __ldcg(g + i);
      __syncthreads();
      if (!(bestT > 0.f)) break;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) a[i] = S.sa[pidx(i)];
  }
  teardown(S);
}

}  // namespace tc
}  // namespace sidon

// =========================== host launch wrappers ==========================
namespace sidon_host {
using namespace sidon;

// device address of the status word, looked up once per device (so that
// launches inside a stream capture make no symbol lookup)
static unsigned int* status_word() {
  constexpr int kMaxDev = 64;
  static std::mutex mu;
  static unsigned int* addr[kMaxDev] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) return nullptr;
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, tc::g_dev_state) != cudaSuccess) return nullptr;
    addr[dev] = &static_cast<DeviceState*>(p)->status;
  }
  return addr[dev];
}

unsigned int* tc_status_word() { return status_word(); }

int device_status(int reset) {
  unsigned int v = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&v, tc::g_dev_state, sizeof(v),
                                       offsetof(DeviceState, status));
  if (e != cudaSuccess) return set_cuda_error(e);
  if (reset) {
    const unsigned int z = 0;
    e = cudaMemcpyToSymbol(tc::g_dev_state, &z, sizeof(z), offsetof(DeviceState, status));
    if (e != cudaSuccess) return set_cuda_error(e);
  }
  return (int)v;
}

// the clock-cycle limit of the bounded waits on the current device
// (cycles <= 0: the default)
int set_wait_limit(long long cycles) {
  const long long v = cycles > 0 ? cycles : kDefaultWaitCycles;
  const cudaError_t e =
      cudaMemcpyToSymbol(tc::g_dev_state, &v, sizeof(v), offsetof(DeviceState, wait_cycles));
  return e == cudaSuccess ? SIDON_OK : set_cuda_error(e);
}

// the fused local search's plan (the ring shares its region with cb)
size_t smem_local_search_tc(int n) { return tc::Layout(n, 0, true).total; }
static size_t smem_local_search_tc(int n, int ring) { return tc::Layout(n, ring, true).total; }
// the plan of the other single-CTA tensor-core kernels (G_p pair, the
// super-block jobs, Frank-Wolfe): cb holds data through their tile phases
size_t smem_tc_plain(int n) { return tc::Layout(n).total; }
static size_t smem_lp_forward_tc(int n) { return tc::Layout(n).total; }

// the two accumulators must fit the 512 TMEM columns
static int tc_n_ok(int n) {
  const int m = (n + tc::BL - 1) / tc::BL;
  return (n >= 1 && n <= tc::kCellsPerThread * tc::NTHREADS &&
          tc::conv_width(m) + tc::corr_width(m) <= 512)
             ? SIDON_OK
             : SIDON_ERR_N;
}

static int prep_tc(const void* fn, size_t sm) { return set_dyn_smem(fn, sm); }
int tc_n_ok_public(int n) { return tc_n_ok(n); }

// Everything a local-search launch at n_max sets up on the host side (the
// shared-memory attribute, the status word's address), done ahead of a
// stream capture.
int tc_ring_choices(int n, int* out, int cap);

int prepare_local_search_tc(int n_max) {
  int rc = tc_n_ok(n_max);
  if (rc) return rc;
  // the largest plan of any window ring the tuner may pick, for both kernels
  size_t sm = smem_local_search_tc(n_max);
  int rings[20];
  const int nr = tc_ring_choices(n_max, rings, 20);
  for (int r = 0; r < nr; ++r) sm = std::max(sm, smem_local_search_tc(n_max, rings[r]));
  rc = prep_tc((const void*)tc::k_local_search_tc, sm);
  if (!rc) rc = prep_tc((const void*)tc::k_local_search_tc_seg, sm);
  if (rc) return rc;
  return status_word() ? SIDON_OK : SIDON_ERR_CUDA;
}

// Whether the balanced-segment kernel can run on device dev with sm bytes
// of dynamic shared memory (cooperative launch supported, at least one
// resident CTA per SM), looked up once per (device, size): the occupancy
// query costs more host time than the rest of a launch.
static bool seg_viable(int dev, size_t sm) {
  static std::mutex mu;
  static std::vector<std::pair<std::pair<int, size_t>, bool>> known;
  std::lock_guard<std::mutex> lock(mu);
  for (const auto& k : known)
    if (k.first.first == dev && k.first.second == sm) return k.second;
  int coop = 0, per_sm = 0;
  bool ok = cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) == cudaSuccess &&
            coop &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tc::k_local_search_tc_seg,
                                                          tc::NTHREADS, sm) == cudaSuccess &&
            per_sm >= 1;
  known.push_back({{dev, sm}, ok});
  return ok;
}

// The balanced-segment kernel, or kNotHere when it does not apply (no
// cooperative launch on the device, fewer resident CTAs than SMs, or fewer
// candidates than SMs).  flags: P caller-owned words, zeroed here on the
// stream.  The launch is a cooperative one (every CTA resident at once), made
// through cudaLaunchKernelEx so that a stream capture records it as a
// cooperative kernel node.
constexpr int kNotHere = -1;
static int launch_local_search_tc_seg(float* pop, float* mom, float* vel, int P, int n,
                                      const int* skip, const int* mode_arr, int iters, double pS,
                                      double pE, double lrS, double lrE, double b1, double b2,
                                      int mode_default, int precision, int ring, size_t sm,
                                      unsigned int* sw, unsigned int* flags, cudaStream_t st) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return kNotHere;
  int rc = set_dyn_smem((const void*)tc::k_local_search_tc_seg, sm);
  if (rc) return rc;
  if (!seg_viable(dev, sm)) return kNotHere;
  const int G = sm_count();
  if (P < G) return kNotHere;
  cudaError_t e = cudaMemsetAsync(flags, 0, (size_t)P * sizeof(unsigned int), st);
  if (e != cudaSuccess) return set_cuda_error(e);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(G);
  cfg.blockDim = dim3(tc::NTHREADS);
  cfg.dynamicSmemBytes = sm;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  e = cudaLaunchKernelEx(&cfg, tc::k_local_search_tc_seg, pop, mom, vel, P, n, skip, mode_arr,
                         iters, (float)pS, (float)pE, (float)lrS, (float)lrE, (float)b1,
                         (float)b2, mode_default, precision == SIDON_PREC_BF16X3 ? 1 : 0, sw,
                         flags, ring);
  if (e != cudaSuccess) return set_cuda_error(e);
  return SIDON_OK;
}

// The fused kernel, one CTA per candidate for a uniform batch (CTAs of
// skipped candidates exit at once, so launches on disjoint candidate sets can
// share the SMs from concurrent streams); persistent (one CTA per SM) for a
// ragged batch.  ring: the window ring's tiles per stage (0: ring_for).
static int launch_plain(float* pop, float* mom, float* vel, const long long* offsets,
                        const int* order, int P, int n_fixed, int n_max, const int* skip,
                        const int* mode_arr, int iters, double pS, double pE, double lrS,
                        double lrE, double b1, double b2, int mode_default, int precision,
                        int ring, cudaStream_t st) {
  int rc = tc_n_ok(n_max);
  if (rc) return rc;
  const size_t sm = smem_local_search_tc(n_max, ring);
  rc = prep_tc((const void*)tc::k_local_search_tc, sm);
  if (rc) return rc;
  unsigned int* sw = status_word();
  if (!sw) return SIDON_ERR_CUDA;
  const int grid = offsets ? (P < sm_count() ? P : sm_count()) : P;
  tc::k_local_search_tc<<<grid, tc::NTHREADS, sm, st>>>(
      pop, mom, vel, offsets, order, P, n_fixed, n_max, skip, mode_arr, iters, (float)pS,
      (float)pE, (float)lrS, (float)lrE, (float)b1, (float)b2, mode_default,
      precision == SIDON_PREC_BF16X3 ? 1 : 0, sw, ring);
  return check_launch();
}

int launch_local_search_tc_plain(float* pop, float* mom, float* vel, const long long* offsets,
                                 const int* order, int P, int n_fixed, int n_max, const int* skip,
                                 const int* mode_arr, int iters, double pS, double pE,
                                 double lrS, double lrE, double b1, double b2, int mode_default,
                                 int precision, cudaStream_t st) {
  return launch_plain(pop, mom, vel, offsets, order, P, n_fixed, n_max, skip, mode_arr, iters, pS,
                      pE, lrS, lrE, b1, b2, mode_default, precision, 0, st);
}

bool tuned_tc_schedule(int n, int P, int precision, int* ring, int* balanced);

// The tensor-core local search.  seg_flags (P words of caller memory, or
// NULL) lets a uniform batch of more candidates than SMs run as balanced
// step segments; without it the batch runs in waves of the one-CTA-per-
// candidate kernel.  A uniform batch takes the window ring and the
// segment / wave choice the schedule tuner measured for (n, P, precision),
// if it ran; every choice gives the same results bit for bit.
int launch_local_search_tc_sched(float* pop, float* mom, float* vel, const long long* offsets,
                                 const int* order, int P, int n_fixed, int n_max, const int* skip,
                                 const int* mode_arr, int iters, double pS, double pE,
                                 double lrS, double lrE, double b1, double b2, int mode_default,
                                 int precision, int ring, int balanced, unsigned int* seg_flags,
                                 cudaStream_t st);

int launch_local_search_tc(float* pop, float* mom, float* vel, const long long* offsets,
                           const int* order, int P, int n_fixed, int n_max, const int* skip,
                           const int* mode_arr, int iters, double pS, double pE, double lrS,
                           double lrE, double b1, double b2, int mode_default, int precision,
                           unsigned int* seg_flags, cudaStream_t st) {
  int ring = 0, balanced = 1;
  if (!offsets) tuned_tc_schedule(n_fixed, P, precision, &ring, &balanced);
  return launch_local_search_tc_sched(pop, mom, vel, offsets, order, P, n_fixed, n_max, skip,
                                      mode_arr, iters, pS, pE, lrS, lrE, b1, b2, mode_default,
                                      precision, ring, balanced, seg_flags, st);
}

// the same with the schedule given: window ring (tiles per stage, 0 =
// ring_for) and balanced segments (used when seg_flags is given and P > SMs)
int launch_local_search_tc_sched(float* pop, float* mom, float* vel, const long long* offsets,
                                 const int* order, int P, int n_fixed, int n_max, const int* skip,
                                 const int* mode_arr, int iters, double pS, double pE,
                                 double lrS, double lrE, double b1, double b2, int mode_default,
                                 int precision, int ring, int balanced, unsigned int* seg_flags,
                                 cudaStream_t st) {
  int rc = tc_n_ok(n_max);
  if (rc) return rc;
  const size_t sm = smem_local_search_tc(n_max, ring);
  unsigned int* sw = status_word();
  if (!sw) return SIDON_ERR_CUDA;
  if (seg_flags && balanced && !offsets && P > sm_count()) {
    const int r = launch_local_search_tc_seg(pop, mom, vel, P, n_fixed, skip, mode_arr, iters,
                                             pS, pE, lrS, lrE, b1, b2, mode_default, precision,
                                             ring, sm, sw, seg_flags, st);
    if (r != kNotHere) return r;              // else: the one-CTA-per-candidate kernel
  }
  return launch_plain(pop, mom, vel, offsets, order, P, n_fixed, n_max, skip, mode_arr, iters,
                      pS, pE, lrS, lrE, b1, b2, mode_default, precision, ring, st);
}

// the window ring ring_for picks at n (tiles per stage; 1 = three single-tile stages)
int tc_ring_default(int n) { return tc::Layout(n, 0, true).ring.per_stage; }

// the window ring shapes (tiles per stage) the fused kernel can run at n
// within the shared-memory opt-in, in the tuner's order of trial
int tc_ring_choices(int n, int* out, int cap) {
  const tc::Layout auto_lo(n, 0, true);
  int cnt = 0;
  for (int T = 1; T <= tc::kMaxWideTiles && cnt < cap; ++T) {
    if (T > 1 && auto_lo.m < tc::kRingMinBlocks) break;   // short sequences: single tiles
    if (tc::Layout(n, T, true).total <= tc::kSmemBudget) out[cnt++] = T;
  }
  return cnt;
}

size_t smem_frank_wolfe_tc(int n) { return tc::Layout(n).total; }

int launch_frank_wolfe_tc(float* pop, float* gbuf, float* gbbuf, const long long* offsets,
                          const int* order, int P, int n_fixed, int n_max, const int* skip,
                          int rounds, int pdhg, int nT, float tMax, float tau, float sig,
                          int precision, cudaStream_t st) {
  int rc = tc_n_ok(n_max);
  if (rc) return rc;
  const size_t sm = smem_frank_wolfe_tc(n_max);
  rc = prep_tc((const void*)tc::k_frank_wolfe_tc, sm);
  if (rc) return rc;
  unsigned int* sw = status_word();
  if (!sw) return SIDON_ERR_CUDA;
  const int grid = offsets ? (P < sm_count() ? P : sm_count()) : P;
  tc::k_frank_wolfe_tc<<<grid, tc::NTHREADS, sm, st>>>(
      pop, gbuf, gbbuf, offsets, order, P, n_fixed, n_max, skip, rounds, pdhg, nT, tMax, tau,
      sig, precision == SIDON_PREC_BF16X3 ? 1 : 0, sw);
  return check_launch();
}

int prepare_frank_wolfe_tc(int n_max) {
  int rc = tc_n_ok(n_max);
  if (rc) return rc;
  rc = prep_tc((const void*)tc::k_frank_wolfe_tc, smem_frank_wolfe_tc(n_max));
  if (rc) return rc;
  return status_word() ? SIDON_OK : SIDON_ERR_CUDA;
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
  const size_t sm = smem_tc_plain(n);
  rc = prep_tc((const void*)tc::k_lp_backward_tc, sm);
  if (rc) return rc;
  unsigned int* sw = status_word();
  if (!sw) return SIDON_ERR_CUDA;
  tc::k_lp_backward_tc<<<P, tc::NTHREADS, sm, st>>>(a, saved, b_in, n, (float)p, grad,
                                                   precision == SIDON_PREC_BF16X3 ? 1 : 0, sw);
  return check_launch();
}

}  // namespace sidon_host
