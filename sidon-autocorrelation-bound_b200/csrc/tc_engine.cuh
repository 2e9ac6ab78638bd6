// ---------------------------------------------------------------------------
//  tc_engine.cuh -- block-Toeplitz convolution / correlation on the 5th-gen
//  tensor cores (tcgen05, accumulators in TMEM), BF16 operands split hi + lo.
//
//  Blocks of L = 128 cells, m = ceil(n/L) blocks.
//
//  Block matrix (the B operand, K-major, rows J, K index s):
//      Bt[J][s] = a[J L + L - 1 - s]      (blocks of a, reversed inside a block)
//  in the canonical no-swizzle core-matrix layout: 8x8 bf16 core matrices of
//  128 B, LBO = 128 B between K-adjacent cores, SBO = 2048 B between 8-row
//  groups.
//
//  Convolution  b_{K L + r} = sum_d sum_s A_d[r][s] Bt[K - d][s]  with the
//  Hankel tile A_d[r][s] = a[(d-1) L + 1 + r + s], d = 0..m: tile d times
//  the block rows J lands in accumulator column K = J + d (TMEM lane r holds
//  b_{K L + r}).
//
//  Correlation  G_i = sum_j c_{i+j} a_j  with i = I L + L - 1 - r' and
//  c_rev[t] = c[2 m L - 2 - t]: the Hankel tile H_e[r'][s] = c_rev[e L + r' + s]
//  (e = 0..2m-2) times block row J lands in column e + J; column
//  col in [m-1, 2m-1) holds block I = 2m - 2 - col.  Only the rows that reach
//  a valid column are multiplied.
//
//  Accumulator column offsets are kept multiples of DG (TMEM alignment).
//  A tile w whose target column is w + J is issued at column off (a multiple
//  of DG), so its B rows start at block t = off - w <= 0.  The residue
//  (-t) mod 8 = w mod 8 is absorbed by a row-shifted copy of the block matrix,
//      BC_rho[x] = Bt[x - rho - Z]   (Z zero rows in front),
//  whose descriptor starts at row t + rho + Z (a multiple of 8).  Tiles run in
//  residue classes rho = 0..7, so each copy is built once per class.
//
//  A Hankel tile is never materialised as an L x L matrix.  A K-major core
//  matrix (row group R, K group S) of a Hankel tile holds
//  x[start + 8(R+S) + i + j], so the tile is the sequence of 8x8 "shifted
//  windows" CM[q][i][j] = x[base + 8q + i + j] addressed with
//  LBO = SBO = 128 B: one tile needs 31 consecutive windows (4 KB per plane)
//  built from 255 consecutive values.
//
//  Arithmetic: x = x_hi + x_lo with x_hi = bf16(x), x_lo = bf16(x - x_hi).
//  The convolution is symmetric (sum_{i+j=k} h_i l_j = sum_{i+j=k} l_i h_j),
//  so BF16x3 needs two products: b = A_hi B_hi + A_lo2 B_hi with the window
//  plane A_lo2 = bf16(2 x_lo) (exact doubling); the correlation uses
//  A_hi B_hi + A_hi B_lo + A_lo B_hi.  BF16x1 keeps A_hi B_hi.  fp32
//  accumulation in TMEM.
//
//  Synchronisation: a ring of STAGES window buffers; every tile's MMAs are
//  followed by tcgen05.commit on the stage's mbarrier, which the builders
//  wait on (bounded) before refilling that stage; the block-matrix copies
//  have their own mbarriers.  One elected thread issues all MMAs.  Every
//  wait gives up after ~2^31 clock cycles, records SIDON_ERR_TIMEOUT in the
//  library's device status word and unwinds.
// ---------------------------------------------------------------------------
#pragma once
#include <cuda_bf16.h>

#include "common.cuh"

namespace sidon {
namespace tc {

constexpr int L = 128;               // block size (= UMMA M)
constexpr int STAGES = 3;            // window ring depth
constexpr int DG = 16;               // accumulator column granule of an MMA destination
constexpr int ZP = DG;               // zero rows in front of a block-matrix copy
constexpr int WIN_CM = 32;           // core matrices per window (31 used)
constexpr int PLANE = WIN_CM * 128;  // bytes per hi or lo window plane
constexpr int STAGE_BYTES = 2 * PLANE;
constexpr int NTHREADS = 256;        // 8 warps: lanes quadrant = warp % 4
constexpr long long kWaitCycles = 1ll << 31;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// SM100 shared-memory matrix descriptor, no swizzle, K-major canonical layout.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm100
  return d;                // base offset 0, lbo mode 0, layout SWIZZLE_NONE
}

// kind::f16 instruction descriptor: bf16 A and B, fp32 D, both K-major, M = 128.
__device__ __forceinline__ uint32_t idesc_bf16(int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(L >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(dtmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :
               : "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// TMEM allocation (whole warp) / release
__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

// 32 lanes x 32 consecutive fp32 columns (one lane per thread)
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int t = 0; t < 32; ++t) v[t] = __uint_as_float(r[t]);
}
__device__ __forceinline__ void tmem_zero32(uint32_t taddr) {
  const uint32_t z = 0u;
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], "
      "{%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,"
      "%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1};" ::"r"(taddr),
      "r"(z)
      : "memory");
}
__device__ __forceinline__ void tmem_wait_st() {
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// hi/lo bf16 split: hi = bf16(x), lo = bf16(x - hi) (x - hi is exact in fp32)
__device__ __forceinline__ void split_bf16(float x, uint16_t& hi, uint16_t& lo) {
  const __nv_bfloat16 h = __float2bfloat16_rn(x);
  const __nv_bfloat16 l = __float2bfloat16_rn(x - __bfloat162float(h));
  hi = __bfloat16_as_ushort(h);
  lo = __bfloat16_as_ushort(l);
}

// Heights live in shared memory in a padded block layout: logical cell i at
// physical index i + 4 floor(i / 128) (block stride 132 floats = 33 x 16 B),
// so that loading the same 16 B of eight consecutive blocks hits eight
// distinct bank groups.
__device__ __forceinline__ int pidx(int i) { return i + 4 * (i >> 7); }

// Warp roles during the tile phases: warp MMA_WARP (lane 0) issues every
// MMA; the other warps build windows and block-matrix copies.
constexpr int MMA_WARP = NTHREADS / 32 - 1;
constexpr int NBUILD_WARPS = NTHREADS / 32 - 1;
constexpr int NBUILD = NBUILD_WARPS * 32;

// Shared state of one CTA.  Every thread holds a copy; the pipeline counters
// of a role are kept identical by every thread of that role.
struct Ctx {
  unsigned char* stages;   // STAGES x (hi plane | lo plane), 1 KB aligned
  unsigned char* bc;       // block-matrix copies: 2 planes of rc x 256 B
  uint64_t* full;          // STAGES "window ready" barriers (NBUILD_WARPS arrivals)
  uint64_t* empty;         // STAGES "window consumed" barriers (tcgen05.commit)
  uint64_t* bc_full;       // 2 "copy ready" barriers (NBUILD_WARPS arrivals)
  uint64_t* bc_empty;      // 2 "copy consumed" barriers (tcgen05.commit)
  uint64_t* bar_done;      // "all MMAs of a phase done"
  uint32_t tmem;           // TMEM base address (512 columns)
  int uses[STAGES];        // times each stage has been filled (builders) / consumed (MMA)
  int bc_uses[2];
  int done_use;
  int st_next;             // next stage in the ring
  int* abort;              // shared abort flag
  int m, rc, n;
  bool three;              // BF16x3 (else BF16x1)
};

__device__ __forceinline__ int bc_rows(int m) { return round_up(ZP + m + 24, 8); }

// bounded wait on an mbarrier phase; sets the abort flag on timeout
__device__ __forceinline__ bool wait_phase(Ctx& C, uint64_t* bar, uint32_t parity,
                                           unsigned int* status) {
  if (mbar_try(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try(bar, parity)) {
    if (*((volatile int*)C.abort)) return false;
    if (clock64() - t0 > kWaitCycles) {
      atomicExch(C.abort, 1);
      atomicCAS(status, 0u, (unsigned int)SIDON_ERR_TIMEOUT);
      return false;
    }
  }
  return true;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ uint32_t pack_bf16x2(float lo_elem, float hi_elem) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo_elem, hi_elem);   // .x = first argument
  return *reinterpret_cast<const uint32_t*>(&v);
}
__device__ __forceinline__ float bf_lo_f(uint32_t p) { return __uint_as_float(p << 16); }
__device__ __forceinline__ float bf_hi_f(uint32_t p) { return __uint_as_float(p & 0xFFFF0000u); }

// hi / lo planes of 8 values (v[0] lands at the lowest address); the lo plane
// holds lsc * (v - hi) rounded (lsc = 2 doubles it exactly).
__device__ __forceinline__ void split8(const float (&v)[8], float lsc, uint4& hi, uint4& lo) {
  uint32_t h[4], l[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    h[q] = pack_bf16x2(v[2 * q], v[2 * q + 1]);
    l[q] = pack_bf16x2(lsc * (v[2 * q] - bf_lo_f(h[q])), lsc * (v[2 * q + 1] - bf_hi_f(h[q])));
  }
  hi = make_uint4(h[0], h[1], h[2], h[3]);
  lo = make_uint4(l[0], l[1], l[2], l[3]);
}

// Row-shifted block-matrix copy into slot `slot` (hi plane, and lo plane in
// the next slot's space when want_lo): BC[x][s] = a[(x - rho - ZP) L + L-1-s]
// for block rows in [0, m).  Chunk c = ((x>>3)*16 + h)*8 + (x&7) sits at byte
// 16 c, so consecutive builder threads store consecutive 16 B; the 8
// heights of a chunk are two aligned float4 of one block (padded layout).
__device__ __forceinline__ void build_bc(Ctx& C, const float* sa, int rho, int slot, bool want_lo,
                                         int bt) {
  const int rc = C.rc;
  unsigned char* hi = C.bc + (size_t)slot * rc * 256;
  unsigned char* lo = hi + (size_t)rc * 256;
  const int chunks = rc * 16;
  for (int c = bt; c < chunks; c += NBUILD) {
    const int x = ((c >> 7) << 3) | (c & 7), h = (c >> 3) & 15;
    const int J = x - rho - ZP;
    uint4 vh = make_uint4(0, 0, 0, 0), vl = vh;
    if (J >= 0 && J < C.m) {
      // s = 8h .. 8h+7  <->  cells J L + L-1-8h down to J L + L-8-8h
      const float* src = sa + pidx(J * L) + (L - 8 - 8 * h);
      const float4 u0 = *reinterpret_cast<const float4*>(src);
      const float4 u1 = *reinterpret_cast<const float4*>(src + 4);
      const float v[8] = {u1.w, u1.z, u1.y, u1.x, u0.w, u0.z, u0.y, u0.x};
      split8(v, 1.f, vh, vl);
    }
    *reinterpret_cast<uint4*>(hi + 16 * c) = vh;
    if (want_lo) *reinterpret_cast<uint4*>(lo + 16 * c) = vl;
  }
}

// Window of tile w into stage st: CM[q'][i][j] = x[8 (16 w + q') + off + i + j]
// (x indexed through map()), planes hi and lsc*lo.
template <typename MapFn>
__device__ __forceinline__ void build_window(Ctx& C, int st, const float* x, MapFn&& map, int off,
                                             int w, float lsc, int bt) {
  unsigned char* hi = C.stages + st * STAGE_BYTES;
  unsigned char* lo = hi + PLANE;
  for (int t = bt; t < WIN_CM * 8; t += NBUILD) {
    const int base = 8 * (16 * w + (t >> 3)) + off + (t & 7);
    float v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] = x[map(base + j)];
    uint4 vh, vl;
    split8(v, lsc, vh, vl);
    *reinterpret_cast<uint4*>(hi + 16 * t) = vh;
    *reinterpret_cast<uint4*>(lo + 16 * t) = vl;
  }
}

// Zero accumulator columns [col0, col0 + ncols) (ncols multiple of 32).
__device__ __forceinline__ void zero_acc(Ctx& C, int col0, int ncols) {
  const int warp = threadIdx.x >> 5, quad = warp & 3, half = warp >> 2;
  const int halves = (blockDim.x >> 5) / 4;
  for (int c = half * 32; c < ncols; c += 32 * halves)
    tmem_zero32(C.tmem + ((uint32_t)(32 * quad) << 16) + (uint32_t)(col0 + c));
  tmem_wait_st();
}

// Tile geometry: accumulator column dcol (multiple of DG), B descriptor start
// row x0 in the class copy (multiple of 8), width N (multiple of 16).
struct Tile {
  int dcol, x0, N;
};

// Issue the MMAs of one tile (one thread).  corr selects the 3-product
// correlation arithmetic, otherwise the 2-product symmetric convolution.
__device__ __forceinline__ void issue_tile(Ctx& C, int st, int slot, const Tile& T, bool corr) {
  const uint32_t a_hi = smem_u32(C.stages + st * STAGE_BYTES);
  const uint32_t a_lo = a_hi + PLANE;
  const uint32_t b_hi = smem_u32(C.bc + (size_t)slot * C.rc * 256) + (uint32_t)(T.x0 >> 3) * 2048u;
  const uint32_t b_lo = b_hi + (uint32_t)C.rc * 256u;
  const uint32_t id = idesc_bf16(T.N);
  const uint32_t d = C.tmem + (uint32_t)T.dcol;
#pragma unroll
  for (int kc = 0; kc < L / 16; ++kc) {
    const uint64_t ah = sdesc(a_hi + kc * 256, 128, 128);
    const uint64_t bh = sdesc(b_hi + kc * 256, 128, 2048);
    mma_bf16(d, ah, bh, id, 1u);
    if (C.three) {
      const uint64_t al = sdesc(a_lo + kc * 256, 128, 128);
      mma_bf16(d, al, bh, id, 1u);
      if (corr) {
        const uint64_t bl = sdesc(b_lo + kc * 256, 128, 2048);
        mma_bf16(d, ah, bl, id, 1u);
      }
    }
  }
}

// Run tiles w = 0..ntiles-1 in residue classes w mod 8 through the
// warp-specialised pipeline.  geom(w) gives the tile; the window source is
// x[map(.)] with offset off.  Ends with every MMA of the sequence complete
// (bar_done) and the accumulator readable by all warps.
template <typename GeomFn, typename MapFn>
__device__ bool run_tiles(Ctx& C, int ntiles, const float* sa, const float* x, MapFn&& map,
                          int off, bool corr, GeomFn&& geom, unsigned int* status) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool want_lo = corr && C.three;
  const float lsc = corr ? 1.f : 2.f;
  int st = C.st_next;
  if (warp == MMA_WARP) {
    if (lane == 0) {
      fence_after();
      for (int rho = 0; rho < 8 && rho < ntiles; ++rho) {
        const int slot = corr ? 0 : (rho & 1);
        if (!wait_phase(C, &C.bc_full[slot], (uint32_t)(C.bc_uses[slot] & 1), status)) break;
        C.bc_uses[slot] += 1;
        bool ok = true;
        for (int w = rho; w < ntiles; w += 8) {
          if (!wait_phase(C, &C.full[st], (uint32_t)(C.uses[st] & 1), status)) { ok = false; break; }
          C.uses[st] += 1;
          fence_after();
          issue_tile(C, st, slot, geom(w), corr);
          mma_commit(&C.empty[st]);
          st = (st + 1 == STAGES) ? 0 : st + 1;
        }
        mma_commit(&C.bc_empty[slot]);
        if (!ok) break;
      }
      mma_commit(C.bar_done);
    }
    __syncwarp();
  } else {
    const int bt = threadIdx.x - (warp > MMA_WARP ? 32 : 0);   // 0 .. NBUILD-1
    for (int rho = 0; rho < 8 && rho < ntiles; ++rho) {
      const int slot = corr ? 0 : (rho & 1);
      const int u = C.bc_uses[slot];
      if (u > 0 && !wait_phase(C, &C.bc_empty[slot], (uint32_t)((u - 1) & 1), status)) break;
      C.bc_uses[slot] = u + 1;
      build_bc(C, sa, rho, slot, want_lo, bt);
      fence_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&C.bc_full[slot]);
      bool ok = true;
      for (int w = rho; w < ntiles; w += 8) {
        const int us = C.uses[st];
        if (us > 0 && !wait_phase(C, &C.empty[st], (uint32_t)((us - 1) & 1), status)) {
          ok = false;
          break;
        }
        C.uses[st] = us + 1;
        build_window(C, st, x, map, off, w, lsc, bt);
        fence_async_smem();
        __syncwarp();
        if (lane == 0) mbar_arrive(&C.full[st]);
        st = (st + 1 == STAGES) ? 0 : st + 1;
      }
      if (!ok) break;
    }
  }
  C.st_next = st;
  const bool ok = wait_phase(C, C.bar_done, (uint32_t)(C.done_use & 1), status);
  C.done_use += 1;
  fence_after();
  __syncthreads();
  return ok && !*((volatile int*)C.abort);
}

// accumulator column bases
constexpr int COL_CONV = 0;
constexpr int COL_CORR = 256;

__device__ __forceinline__ int acc_width(int m) { return round_up(2 * m + 16, 32); }

// b = a * a into accumulator columns of COL_CONV (column K, lane r = b_{K L + r})
__device__ __forceinline__ bool conv_tc(Ctx& C, const float* sa, unsigned int* status) {
  const int m = C.m;
  return run_tiles(C, m + 1, sa, sa, [](int i) { return pidx(i); }, -(L - 1), false,
                   [&](int d) {
                     Tile T;
                     const int off = (d / DG) * DG;
                     const int t = off - d;                       // (-DG, 0]
                     T.dcol = COL_CONV + off;
                     T.x0 = t + (d & 7) + ZP;
                     T.N = round_up(m - t, 16);
                     return T;
                   },
                   status);
}

// G = corr(c, a) into the accumulator columns of COL_CORR; crev is the
// reversed weight sequence (zero margins), sa the heights.
__device__ __forceinline__ bool corr_tc(Ctx& C, const float* sa, const float* crev,
                                        unsigned int* status) {
  const int m = C.m;
  return run_tiles(C, 2 * m - 1, sa, crev, [](int i) { return i; }, 0, true,
                   [&](int e) {
                     Tile T;
                     const int lo = max(0, m - 1 - e), hi = min(m, 2 * m - 1 - e);
                     const int off = ((e + lo) / DG) * DG;
                     const int t = off - e;                       // (lo - DG, lo]
                     T.dcol = COL_CORR + off;
                     T.x0 = t + (e & 7) + ZP;
                     T.N = round_up(hi - t, 16);
                     return T;
                   },
                   status);
}

}  // namespace tc
}  // namespace sidon
