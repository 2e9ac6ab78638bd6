// ---------------------------------------------------------------------------
//  tc_tf32.cuh -- the block-Toeplitz convolution / correlation of
//  tc_engine.cuh with TF32 operands split hi + lo (tcgen05.mma kind::tf32,
//  fp32 accumulation in TMEM): x = hi + lo, hi = tf32(x), lo = tf32(x - hi),
//  about 22 significant bits against BF16x3's 16.
//
//  Same geometry as the BF16 engine (64-cell blocks, 128-lane Hankel
//  windows on every second diagonal, B = the blocks of the other operand,
//  the same accumulator layout and gathers); what changes is the operand
//  width.  A K-major core matrix now holds 8 rows x 4 tf32 values, so
//    window:  core matrix (row group G, K group S) = a[start + 8 G + 4 S + i + j]
//             = CM[2 G + S][i][j] with CM[q][i][j] = a[start + 4 q + i + j]:
//             46 core matrices per tile and plane, LBO = 128 B, SBO = 256 B;
//    copies:  element (row x, K index k) at byte (k / 4) 16 rows + 16 x + 4 (k % 4),
//             LBO = 16 rows, SBO = 128 B;
//  and a 64-cell tile takes eight K8 instructions per product.
//
//  The operands are twice as wide as BF16's, so the ring holds three
//  single-tile stages and a hi|lo pair of a B copy does not fit beside the
//  heights at the precision sweep's n = 8400: the correlation runs in two
//  passes over the tiles, the first with the weights' hi plane as B
//  (A_hi B_hi + A_lo B_hi), the second with their lo plane (A_hi B_lo), both
//  accumulating into the same TMEM columns.  The symmetric autoconvolution
//  needs one B plane anyway (A_hi B_hi + A_lo2 B_hi, A_lo2 = tf32(2 lo)).
//
//  The pipeline, its barriers and bounded waits are those of
//  run_tiles_ring; only the builders and the MMA issue differ.
// ---------------------------------------------------------------------------
#pragma once
#include "tc_cta.cuh"

namespace sidon {
namespace tc {
namespace tf32 {

constexpr int kStageCms = 48;                              // 46 used, 2 of padding
constexpr int kPlaneBytes = kStageCms * 128;
constexpr int kStageBytes = 2 * kPlaneBytes;               // hi | lo planes
constexpr int kStages = 3;
constexpr int KSTEPS8 = BL / 8;                            // K8 instructions per tile and product

// tf32(x) rounded to nearest (ties away), as an fp32 bit pattern whose low 13
// mantissa bits are zero
__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
// hi and lsc * lo of x
__device__ __forceinline__ void split_tf32(float x, float lsc, uint32_t& hi, uint32_t& lo) {
  hi = to_tf32(x);
  lo = to_tf32(lsc * (x - __uint_as_float(hi)));
}

// kind::tf32 instruction descriptor: tf32 A and B, fp32 D, both K-major, M = 128
__device__ __forceinline__ uint32_t idesc_tf32(int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(L >> 4) << 24);
}
__device__ __forceinline__ void mma_tf32(uint32_t dtmem, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, 1, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(dtmem), "l"(adesc), "l"(bdesc), "r"(idesc)
      : "memory");
}

// shared-memory plan of the TF32 kernels (the BF16 plan with a three-stage
// single-tile ring of TF32 windows and a one-plane B copy of TF32 rows)
struct Plan {
  int m, rc, rcc, sa_len, cb_len;
  size_t off_bc, off_sa, off_cb, off_red, total;
  __host__ __device__ Plan(int n) {
    m = (n + BL - 1) / BL;
    rc = conv_copy_rows(m);
    rcc = corr_copy_rows(m);
    sa_len = 68 * (m + 8);
    cb_len = 68 * (2 * m + 2);
    size_t o = (size_t)kStages * kStageBytes;
    off_bc = o;
    const int rows = rcc > rc ? rcc : rc;
    const size_t region = (size_t)rows * 256;              // one plane of TF32 rows
    o += region > (size_t)cb_len * 4 ? region : (size_t)cb_len * 4;
    off_sa = o;
    o += (size_t)sa_len * 4;
    o = (o + 15) & ~(size_t)15;
    off_cb = o;
    o += (size_t)cb_len * 4;
    o = (o + 15) & ~(size_t)15;
    off_red = o;
    o += 64 * 4 + (2 * MAX_STAGES + 6) * 8 + 16;
    total = o + 1024;
  }
};

// Per-CTA set-up (the frame of setup() with the TF32 plan).
__device__ __forceinline__ Shared setup(int n, unsigned char* raw) {
  const Plan Pl(n);
  unsigned char* base = (unsigned char*)(((uintptr_t)raw + 1023) & ~(uintptr_t)1023);
  Shared S;
  S.C.stages = base;
  S.C.bc = base + Pl.off_bc;
  S.sa = reinterpret_cast<float*>(base + Pl.off_sa) + 136;
  S.cb = reinterpret_cast<float*>(base + Pl.off_cb);
  S.red = reinterpret_cast<float*>(base + Pl.off_red);
  uint64_t* bars = reinterpret_cast<uint64_t*>(S.red + 64);
  S.C.full = bars;
  S.C.empty = bars + MAX_STAGES;
  S.C.bc_full = bars + 2 * MAX_STAGES;
  S.C.bc_empty = bars + 2 * MAX_STAGES + 2;
  S.C.bar_done = bars + 2 * MAX_STAGES + 4;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 2 * MAX_STAGES + 6);
  S.C.abort = reinterpret_cast<int*>(tslot + 1);
  S.C.m = Pl.m;
  S.C.rc = Pl.rc;
  S.C.rcc = Pl.rcc;
  S.C.n = n;
  S.C.dmax = last_tile(n);
  S.C.three = true;
  S.C.ph = S.C.started = S.C.bc_ph = S.C.bc_started = S.C.done_ph = 0u;
  S.C.st_next = 0;
  S.C.nst = kStages;
  S.C.wps = 1;
  if (threadIdx.x == 0) {
    for (int s = 0; s < MAX_STAGES; ++s) {
      mbar_init(&S.C.full[s], NBUILD_WARPS);
      mbar_init(&S.C.empty[s], 1);
    }
    for (int s = 0; s < 2; ++s) {
      mbar_init(&S.C.bc_full[s], NBUILD_WARPS);
      mbar_init(&S.C.bc_empty[s], 1);
    }
    mbar_init(S.C.bar_done, 1);
    mbar_fence_init();
    S.C.abort[0] = 0;
  }
  if ((threadIdx.x >> 5) == 0) tmem_alloc(tslot, 512);
  fence_before();
  __syncthreads();
  fence_after();
  S.C.tmem = *tslot;
  return S;
}

// Window of tile w into stage st: CM[q][i][j] = a[64 w - 63 + 4 q + i + j],
// planes hi and lsc * lo; chunk t = 8 q + i (16 bytes at 16 t of a plane).
__device__ __forceinline__ void tf_stage(Ctx& C, int st, const float* sa, int w, float lsc,
                                         int bt) {
  unsigned char* hi = C.stages + st * kStageBytes;
  unsigned char* lo = hi + kPlaneBytes;
  const int base = 64 * w - 63;
  for (int t = bt; t < 8 * kStageCms; t += NBUILD) {
    const int c0 = base + 4 * (t >> 3) + (t & 7);
    uint32_t h[4], l[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) split_tf32(sa[pidx(c0 + j)], lsc, h[j], l[j]);
    *reinterpret_cast<uint4*>(hi + 16 * t) = make_uint4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<uint4*>(lo + 16 * t) = make_uint4(l[0], l[1], l[2], l[3]);
  }
}

// The tile sequences of the TF32 kernels.
enum Mode { CONV = 0, CORR_HI = 1, CORR_LO = 2 };

// Autoconvolution copy (one plane, tf32(a)): BC[x][s] = a[64 (x - ZP) + 63 - s].
__device__ __forceinline__ void tf_conv_copy(Ctx& C, const float* sa, int bt) {
  const int rows = C.rc;
  for (int c = bt; c < rows * 16; c += NBUILD) {
    const int h = c / rows, x = c - h * rows, J = x - ZP;
    uint32_t v[4] = {0u, 0u, 0u, 0u};
    if (J >= 0 && J < C.m) {
#pragma unroll
      for (int j = 0; j < 4; ++j) v[j] = to_tf32(sa[pidx(64 * J + 63 - 4 * h - j)]);
    }
    *reinterpret_cast<uint4*>(C.bc + (uint32_t)h * b_lbo(rows) + 16u * (uint32_t)x) =
        make_uint4(v[0], v[1], v[2], v[3]);
  }
}
// Correlation copy, one plane of the weights: CC[x][s] = c[64 x + s] (hi
// plane tf32(c), or lo plane tf32(c - tf32(c))), x < 2m.
__device__ __forceinline__ void tf_corr_copy(Ctx& C, const float* cb, bool lo_plane, int bt) {
  const int rows = C.rcc;
  for (int c = bt; c < rows * 16; c += NBUILD) {
    const int h = c / rows, x = c - h * rows;
    uint32_t v[4] = {0u, 0u, 0u, 0u};
    if (x < 2 * C.m) {
      const float4 u = *reinterpret_cast<const float4*>(cb + pidx(64 * x + 4 * h));
      const float w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        uint32_t hh, ll;
        split_tf32(w[j], 1.f, hh, ll);
        v[j] = lo_plane ? ll : hh;
      }
    }
    *reinterpret_cast<uint4*>(C.bc + (uint32_t)h * b_lbo(rows) + 16u * (uint32_t)x) =
        make_uint4(v[0], v[1], v[2], v[3]);
  }
}

// MMAs of tile T from stage st: K8 step kc reads K groups 2 kc, 2 kc + 1 of
// the window (core matrices 2 kc + 2 G + ...: start 256 kc) and of the copy.
template <int MODE>
__device__ __forceinline__ void tf_issue(Ctx& C, int st, uint32_t bbase, uint32_t lbo,
                                         const Tile& T) {
  const uint32_t a_hi = smem_u32(C.stages + st * kStageBytes);
  const uint32_t a_lo = a_hi + kPlaneBytes;
  const uint32_t b0 = bbase + 16u * (uint32_t)T.x0;
  const uint32_t id = idesc_tf32(T.N);
  const uint32_t d = C.tmem + (uint32_t)T.dcol;
#pragma unroll
  for (int kc = 0; kc < KSTEPS8; ++kc) {
    const uint64_t bd = sdesc(b0 + 2u * kc * lbo, lbo, 128);
    mma_tf32(d, sdesc(a_hi + kc * 256, 128, 256), bd, id);
    if (MODE != CORR_LO) mma_tf32(d, sdesc(a_lo + kc * 256, 128, 256), bd, id);
  }
}

// One pass of the tile sequence w = 0, 2, ..., dmax through the pipeline of
// run_tiles_ring (single-tile stages): the builders write the B copy of MODE
// once, then the windows; the MMA lane issues each tile and releases its
// stage.  Ends with every MMA of the pass complete and the accumulator
// readable.  wsrc: padded shared heights; cb: padded shared weights (CORR).
template <int MODE>
__device__ __forceinline__ bool run_tiles(Ctx& C, const float* wsrc, const float* cb,
                                          unsigned int* status) {
  constexpr bool corr = MODE != CONV;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const float lsc = MODE == CONV ? 2.f : 1.f;
  const int m = C.m;
  const int rows = corr ? C.rcc : C.rc;
  const uint32_t lbo = b_lbo(rows);
  int st = C.st_next;
  if (warp == MMA_WARP) {
    if (lane == 0) {
      fence_after();
      bool ok = wait_phase(C, &C.bc_full[0], C.bc_ph & 1u, status);
      C.bc_ph ^= 1u;
      const uint32_t bbase = smem_u32(C.bc);
      for (int w = 0; ok && w <= C.dmax; w += 2) {
        if (!wait_phase(C, &C.full[st], (C.ph >> st) & 1u, status)) { ok = false; break; }
        C.ph ^= 1u << st;
        fence_after();
        Tile T;
        if (corr) {
          T.dcol = col_corr(m);
          T.x0 = w;
          T.N = corr_n(m);
        } else {
          const int off = (w / DG) * DG, t = off - w;
          T.dcol = COL_CONV + off;
          T.x0 = t + ZP;
          T.N = round_up(m - t, 16);
        }
        tf_issue<MODE>(C, st, bbase, lbo, T);
        mma_commit(&C.empty[st]);
        st = (st + 1 == kStages) ? 0 : st + 1;
      }
      mma_commit(&C.bc_empty[0]);
      mma_commit(C.bar_done);
    }
    __syncwarp();
  } else if (builder_index() >= 0) {
    const int bt = builder_index();
    bool ok = true;
    if ((C.bc_started & 1u) && !wait_phase(C, &C.bc_empty[0], C.bc_ph & 1u, status)) ok = false;
    if (C.bc_started & 1u) C.bc_ph ^= 1u;
    C.bc_started |= 1u;
    if (ok) {
      if (corr) tf_corr_copy(C, cb, MODE == CORR_LO, bt);
      else tf_conv_copy(C, wsrc, bt);
      fence_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&C.bc_full[0]);
    }
    for (int w = 0; ok && w <= C.dmax; w += 2) {
      if ((C.started >> st) & 1u) {
        if (!wait_phase(C, &C.empty[st], (C.ph >> st) & 1u, status)) {
          ok = false;
          break;
        }
        C.ph ^= 1u << st;
      }
      C.started |= 1u << st;
      tf_stage(C, st, wsrc, w, lsc, bt);
      fence_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&C.full[st]);
      st = (st + 1 == kStages) ? 0 : st + 1;
    }
  }
  C.st_next = st;
  const bool ok = drain_phase(C.bar_done, C.done_ph, status);
  C.done_ph ^= 1u;
  fence_after();
  __syncthreads();
  return ok && !*((volatile int*)C.abort);
}

}  // namespace tf32
}  // namespace tc
}  // namespace sidon
