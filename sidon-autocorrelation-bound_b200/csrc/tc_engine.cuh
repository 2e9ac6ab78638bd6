// ---------------------------------------------------------------------------
//  tc_engine.cuh -- block-Toeplitz convolution / correlation on the 5th-gen
//  tensor cores (tcgen05, accumulators in TMEM), BF16 operands split hi + lo.
//
//  Geometry.  Input blocks of BL = 64 cells, m = ceil(n/64) blocks.  A tile
//  w is the 128 x 64 Hankel window of the heights
//        A_w[R][s] = a[64 w - 63 + R + s]      (lanes R = 0..127, K index s),
//  and the tiles are w = 0, 2, 4, ... (every second diagonal: 128 lanes span
//  two 64-cell output blocks, so each product a_i a_j lands in exactly one
//  accumulator cell).  The UMMA shape is M = 128, K = 16, N = (number of
//  blocks) ~ m, which keeps every instruction above the tensor core's fixed
//  per-instruction cost (measured: ~92 cycles per M128 K16 instruction,
//  N/2 cycles of math).
//
//  Convolution  b = a * a.  B operand: the reversed blocks
//        Bt[J][s] = a[64 J + 63 - s],  J = 0..m-1.
//  Tile d accumulates A_d Bt^T into TMEM columns J + d, so cell (R, col)
//  collects products with index sum 64 col + R:
//        b_k = D[k mod 64][k / 64] + D[k mod 64 + 64][k / 64 - 1].
//
//  Correlation  G_i = sum_j c_{i+j} a_j = sum_k c_k a_{k-i}.  B operand: the
//  weight blocks  Cb[K][s] = c[64 K + s], K = 0..2m-1.  Tile t (same windows
//  of a) accumulates A_t Cb[col + t]^T into column col, and cell (R, col)
//  collects the output i = 64 col + 63 - R:
//        G_i = D2[R0][col0] + D2[R0 + 64][col0 + 1],  R0 = (63 - i) mod 64.
//
//  Shifts.  A tile's B rows are shifted by its diagonal.  The B copies are
//  stored row-contiguous within each K group (SBO = 128 B), so a shift by
//  any number of rows is a descriptor start offset of 16 B per row;
//  accumulator column offsets are kept multiples of DG (TMEM alignment) and
//  the rest of the shift (tile - offset) moves the B start:
//        conv:  BC[x] = Bt[x - ZP]  (ZP zero rows in front), rows from
//               ZP + offset - tile;
//        corr:  CC[x] = Cb[x], rows from the tile index.
//
//  A Hankel window is never materialised as a 128 x 64 matrix.  A K-major
//  core matrix (row group G, K group S) of it holds a[start + 8(G+S) + i + j],
//  so the window is the sequence of 23 8x8 "shifted windows"
//  CM[q][i][j] = a[start + 8q + i + j] addressed with LBO = SBO = 128 B.
//
//  Arithmetic: x = x_hi + x_lo with x_hi = bf16(x), x_lo = bf16(x - x_hi).
//  The autoconvolution is symmetric (sum_{i+j=k} h_i l_j = sum_{i+j=k} l_i h_j),
//  so BF16x3 needs two products: b = A_hi B_hi + A_lo2 B_hi with the window
//  plane A_lo2 = bf16(2 x_lo) (exact doubling); the cross convolution a * y
//  (B from y) and the correlation use A_hi B_hi + A_lo B_hi + A_hi B_lo.
//  BF16x1 keeps A_hi B_hi.  fp32 accumulation in TMEM.
//
//  Pipeline: one MMA warp (one elected lane issues every MMA) and builder
//  warps; a ring of stages holding the windows of one to sixteen tiles
//  each, and one copy slot per phase, each guarded by a full barrier
//  (builder arrivals) and an empty barrier (tcgen05.commit).  A stage's
//  release -- the commit, the builders' wait for it and the rebuild before
//  the MMA lane may use the stage again -- cost ~750-870 cycles per release
//  with one tile per stage (phase timers at n = 8400, against ~72 of math
//  per M128 N144 K16 instruction), so long tile sequences run two stages of
//  many tiles -- one commit per stage -- and short ones three single-tile
//  stages (see ring_for and Layout).
//  Every pipeline wait gives up after the device state's wait limit (2^31
//  clock cycles unless sidon_set_wait_limit changed it), records
//  SIDON_ERR_TIMEOUT in the library's device status word and unwinds; the
//  unwinding still waits for the MMAs already issued (drain_phase) before
//  the accumulators or the tensor memory are given up.
// ---------------------------------------------------------------------------
#pragma once
#include <cuda_bf16.h>

#include "common.cuh"

namespace sidon {
namespace tc {

constexpr int L = 128;               // UMMA M (lanes)
constexpr int BL = 64;               // input block = K of a tile
constexpr int KSTEPS = BL / 16;      // K16 instructions per tile and product
constexpr int MAX_STAGES = 3;        // window ring: at most three stages
constexpr int DG = 16;               // accumulator column granule of an MMA destination
constexpr int ZP = DG;               // zero rows in front of a block-matrix copy
// A stage of the window ring holds the windows of T consecutive tiles.  The
// window of tile w + 2 is the window of tile w moved by 128 cells = 16 core
// matrices, so the T windows are one run of 16 T + 7 core matrices (one more
// is built as padding) per plane: tile h of the stage starts at core matrix
// 16 h.
__host__ __device__ constexpr int stage_cms(int T) { return 16 * T + 8; }
__host__ __device__ constexpr int stage_plane_bytes(int T) { return stage_cms(T) * 128; }
__host__ __device__ constexpr int stage_bytes(int T) { return 2 * stage_plane_bytes(T); }
// 12 warps: lane quadrant = warp % 4 (three warps per quadrant).  Measured
// per step against 8 and 16 warps: 6% faster than 8 at n = 8400 (256
// candidates; the latency-bound gathers, weights and update get more warps,
// and the step compiles without spills), 16 slower than 8 at most n.
constexpr int NTHREADS = 384;
constexpr int WARPS_PER_QUAD = NTHREADS / 128;
constexpr long long kWaitCycles = kDefaultWaitCycles;   // limit of the drain wait

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

// Heights and weights live in shared memory in a padded block layout: logical
// index i at physical i + 4 floor(i / 64) (block stride 68 floats = 17 x 16 B),
// so that the same 16 B of eight consecutive blocks fall in eight distinct
// bank groups when a copy gathers a column of blocks.
__device__ __forceinline__ int pidx(int i) { return i + 4 * (i >> 6); }

// Warp roles during the tile phases: warp MMA_WARP (lane 0) issues every
// MMA; the warps of the other three SM sub-partitions (warp w runs on
// sub-partition w mod 4) build windows and B-matrix copies, and the other
// warps of the MMA warp's sub-partition stay idle, so that the issuing
// thread has that sub-partition's issue slots to itself (measured at
// n = 8400: tile phases 45.8k / 64.5k -> 43.2k / 62.3k cycles against
// builders in every warp).  builder_index numbers the builders 0 ..
// NBUILD - 1, or returns -1.
constexpr int MMA_WARP = NTHREADS / 32 - 1;
static_assert(MMA_WARP % 4 == 3, "the idle warps are those with w mod 4 == 3");
constexpr int NBUILD_WARPS = NTHREADS / 32 - NTHREADS / 128;
constexpr int NBUILD = NBUILD_WARPS * 32;
__device__ __forceinline__ int builder_index() {
  const int warp = threadIdx.x >> 5;
  return (warp & 3) == 3 ? -1 : (warp - (warp >> 2)) * 32 + (int)(threadIdx.x & 31);
}

// Shared state of one CTA.  Every thread holds a copy; the pipeline counters
// of a role are kept identical by every thread of that role.
struct Ctx {
  unsigned char* stages;   // nst stages of wps tiles' windows (hi plane | lo plane), 1 KB aligned
  unsigned char* bc;       // the phase's B-matrix copy (hi plane, lo plane after it)
  uint64_t* full;          // nst "windows ready" barriers (NBUILD_WARPS arrivals)
  uint64_t* empty;         // nst "windows consumed" barriers (tcgen05.commit)
  uint64_t* bc_full;       // "copy ready" barrier (NBUILD_WARPS arrivals; [0] used)
  uint64_t* bc_empty;      // "copy consumed" barrier (tcgen05.commit; [0] used)
  uint64_t* bar_done;      // "all MMAs of a phase done"
  uint32_t tmem;           // TMEM base address (512 columns)
  // pipeline phases as bit masks (registers, no dynamic indexing): bit s of
  // ph = parity of this thread's next wait on stage s (full for the MMA
  // lane, empty for the builders); bit s of started = stage s filled before
  // (builders skip the first empty wait); bc_ph / bc_started likewise for
  // the copy slots; done_ph = parity of the next bar_done wait
  uint32_t ph, started, bc_ph, bc_started, done_ph;
  int st_next;             // next stage in the ring
  int nst, wps;            // ring shape: stages, tiles per stage
  int* abort;              // shared abort flag
  int m, rc, rcc, n, dmax; // blocks, conv / corr copy rows, cells, last tile
  bool three;              // BF16x3 (else BF16x1)
};

__host__ __device__ __forceinline__ int conv_copy_rows(int m) { return round_up(ZP + m + 40, 8); }
__host__ __device__ __forceinline__ int corr_copy_rows(int m) { return round_up(2 * m + 24, 8); }
__host__ __device__ __forceinline__ int last_tile(int n) { return (((n + 62) / 64) + 1) / 2 * 2; }
__host__ __device__ __forceinline__ int conv_width(int m) { return round_up(2 * m + 17, 32); }
__host__ __device__ __forceinline__ int corr_n(int m) { return round_up(m + 1, 16); }
__host__ __device__ __forceinline__ int corr_width(int m) { return round_up(corr_n(m), 32); }

// Bounded wait on an mbarrier phase inside the tile pipeline: gives up when
// another thread has aborted, or after the device state's wait limit
// (sidon_set_wait_limit), in which case it records SIDON_ERR_TIMEOUT and sets
// the abort flag.
__device__ __forceinline__ bool wait_bar(int* abort, uint64_t* bar, uint32_t parity,
                                         unsigned int* status) {
  if (mbar_try(bar, parity)) return true;
  const long long t0 = clock64(), lim = wait_limit(status);
  while (!mbar_try(bar, parity)) {
    if (*((volatile int*)abort)) return false;
    if (clock64() - t0 > lim) {
      atomicExch(abort, 1);
      atomicCAS(status, 0u, (unsigned int)SIDON_ERR_TIMEOUT);
      return false;
    }
  }
  return true;
}
__device__ __forceinline__ bool wait_phase(Ctx& C, uint64_t* bar, uint32_t parity,
                                           unsigned int* status) {
  return wait_bar(C.abort, bar, parity, status);
}

// The end-of-phase wait for the MMA lane's final commit.  It must see every
// issued MMA complete before the CTA reads the accumulators, reuses the
// stages or releases the tensor memory, so it ignores the abort flag and the
// configurable limit: the commit arrives once the tensor pipe has drained,
// which needs no other thread.  Bounded by kWaitCycles all the same.
__device__ __forceinline__ bool drain_phase(uint64_t* bar, uint32_t parity, unsigned int* status) {
  if (mbar_try(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try(bar, parity)) {
    if (clock64() - t0 > kWaitCycles) {
      atomicCAS(status, 0u, (unsigned int)SIDON_ERR_TIMEOUT);
      return false;
    }
  }
  return true;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ uint32_t pack_bf16x2(float first, float second) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(first, second);   // .x = first (low half)
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

// B-matrix copies are row-contiguous within each K group: element (row x,
// K index k) of a plane with `rows` rows sits at byte
//      (k / 8) * 16 rows + 16 x + 2 (k % 8),
// i.e. a K-major operand with SBO = 128 B between 8-row groups and
// LBO = 16 rows bytes between K groups.  A tile whose B rows start at an
// arbitrary row x0 is then the descriptor start + 16 x0: no residue-class
// copies are needed, and each phase builds its copy once.
__host__ __device__ __forceinline__ uint32_t b_lbo(int rows) { return 16u * (uint32_t)rows; }

// Convolution copy (hi plane at `hi`, lo plane at `lo` when want_lo):
// BC[x][s] = y[64 (x - ZP) + 63 - s] for block rows x - ZP in [0, m), zero
// elsewhere, x < rc.  y is either a padded shared-memory array (ylen < 0;
// zero beyond its cells) or a plain global row of ylen cells read through
// L2 (cells >= ylen read as 0; the row may be written by this CTA between
// phases, so no read-only path).
__device__ __forceinline__ void build_conv_copy(Ctx& C, const float* y, int ylen,
                                                unsigned char* hi, unsigned char* lo,
                                                bool want_lo, int bt) {
  const int rows = C.rc;
  const int chunks = rows * 8;
  for (int c = bt; c < chunks; c += NBUILD) {
    const int h = c / rows, x = c - h * rows;
    const int J = x - ZP;
    uint4 vh = make_uint4(0, 0, 0, 0), vl = vh;
    if (J >= 0 && J < C.m) {
      // s = 8h .. 8h+7  <->  cells 64J + 63 - 8h down to 64J + 56 - 8h
      float v[8];
      if (ylen < 0) {
        const float* src = y + pidx(64 * J + 56 - 8 * h);
        const float4 u0 = *reinterpret_cast<const float4*>(src);
        const float4 u1 = *reinterpret_cast<const float4*>(src + 4);
        v[0] = u1.w; v[1] = u1.z; v[2] = u1.y; v[3] = u1.x;
        v[4] = u0.w; v[5] = u0.z; v[6] = u0.y; v[7] = u0.x;
      } else {
        // cells base .. base + 7 (base a multiple of 8): two 16-byte loads
        // when the row allows, else one load per cell
        const int base = 64 * J + 56 - 8 * h;
        if (base + 8 <= ylen && (reinterpret_cast<uintptr_t>(y + base) & 15) == 0) {
          const float4 u0 = __ldcg(reinterpret_cast<const float4*>(y + base));
          const float4 u1 = __ldcg(reinterpret_cast<const float4*>(y + base + 4));
          v[0] = u1.w; v[1] = u1.z; v[2] = u1.y; v[3] = u1.x;
          v[4] = u0.w; v[5] = u0.z; v[6] = u0.y; v[7] = u0.x;
        } else {
#pragma unroll
          for (int j = 0; j < 8; ++j) v[j] = (base + 7 - j < ylen) ? __ldcg(y + (base + 7 - j)) : 0.f;
        }
      }
      split8(v, 1.f, vh, vl);
    }
    const uint32_t off = (uint32_t)h * b_lbo(rows) + 16u * (uint32_t)x;
    *reinterpret_cast<uint4*>(hi + off) = vh;
    if (want_lo) *reinterpret_cast<uint4*>(lo + off) = vl;
  }
}

// Correlation copy (hi plane at C.bc, lo plane after it):
// CC[x][s] = c[64 x + s] for weight blocks x < 2m, zero beyond, x < rcc.
__device__ __forceinline__ void build_corr_copy(Ctx& C, const float* cb, bool want_lo, int bt) {
  const int rows = C.rcc;
  unsigned char* hi = C.bc;
  unsigned char* lo = hi + (size_t)rows * 128;
  const int chunks = rows * 8;
  for (int c = bt; c < chunks; c += NBUILD) {
    const int h = c / rows, x = c - h * rows;
    uint4 vh = make_uint4(0, 0, 0, 0), vl = vh;
    if (x < 2 * C.m) {
      const float* src = cb + pidx(64 * x + 8 * h);
      const float4 u0 = *reinterpret_cast<const float4*>(src);
      const float4 u1 = *reinterpret_cast<const float4*>(src + 4);
      const float v[8] = {u0.x, u0.y, u0.z, u0.w, u1.x, u1.y, u1.z, u1.w};
      split8(v, 1.f, vh, vl);
    }
    const uint32_t off = (uint32_t)h * b_lbo(rows) + 16u * (uint32_t)x;
    *reinterpret_cast<uint4*>(hi + off) = vh;
    if (want_lo) *reinterpret_cast<uint4*>(lo + off) = vl;
  }
}

// bf16(x) in the low half, bf16(lsc * (x - bf16(x))) in the high half
__device__ __forceinline__ uint32_t split_pack(float x, float lsc) {
  const __nv_bfloat16 h = __float2bfloat16_rn(x);
  const __nv_bfloat16 l = __float2bfloat16_rn(lsc * (x - __bfloat162float(h)));
  return (uint32_t)__bfloat16_as_ushort(h) | ((uint32_t)__bfloat16_as_ushort(l) << 16);
}

// Windows of the nt tiles w0, w0 + 2, ... into stage st of a ring of
// T-tile stages: core matrices CM[q][i][j] = a[64 w0 - 63 + 8 q + i + j],
// q < 16 nt + 8, planes hi and lsc * lo.  Chunk t = 8 q + i (16 bytes at
// offset 16 t of a plane) holds the 8 cells from 64 w0 - 63 + t on:
// consecutive chunks are windows shifted by one cell.  A warp covers 32
// chunks: every lane splits two cells (t and t + 32) once, and the 8 cells of
// its chunk arrive by warp shuffles, so each cell is loaded and split once
// per warp instead of once per chunk row.  Warp-uniform (all 32 lanes take
// part in the shuffles).  The highest cell read, 64 (w0 + 2 nt) + 32, is the
// one a single window of the stage's last tile reads.
__device__ __forceinline__ void build_stage(Ctx& C, int st, int T, const float* sa, int w0,
                                            int nt, float lsc, int bt) {
  unsigned char* hi = C.stages + st * stage_bytes(T);
  unsigned char* lo = hi + stage_plane_bytes(T);
  const int lane = bt & 31;
  const int base0 = 64 * w0 - 63;
  const int nchunk = 8 * stage_cms(nt);
  for (int t0 = bt - lane; t0 < nchunk; t0 += NBUILD) {
    const int c = base0 + t0 + lane;
    const uint32_t p0 = split_pack(sa[pidx(c)], lsc);
    const uint32_t p1 = split_pack(sa[pidx(c + 32)], lsc);
    uint32_t P[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int src = (lane + j) & 31;
      const uint32_t x0 = __shfl_sync(0xffffffffu, p0, src);
      const uint32_t x1 = __shfl_sync(0xffffffffu, p1, src);
      P[j] = (lane + j < 32) ? x0 : x1;
    }
    const uint4 vh = make_uint4(__byte_perm(P[0], P[1], 0x5410), __byte_perm(P[2], P[3], 0x5410),
                                __byte_perm(P[4], P[5], 0x5410), __byte_perm(P[6], P[7], 0x5410));
    const uint4 vl = make_uint4(__byte_perm(P[0], P[1], 0x7632), __byte_perm(P[2], P[3], 0x7632),
                                __byte_perm(P[4], P[5], 0x7632), __byte_perm(P[6], P[7], 0x7632));
    const int t = t0 + lane;
    if (t < nchunk) {
      *reinterpret_cast<uint4*>(hi + 16 * t) = vh;
      *reinterpret_cast<uint4*>(lo + 16 * t) = vl;
    }
  }
}

// Zero accumulator columns [col0, col0 + ncols) (ncols multiple of 32).
__device__ __forceinline__ void zero_acc(Ctx& C, int col0, int ncols) {
  const int warp = threadIdx.x >> 5, quad = warp & 3, sub = warp >> 2;
  for (int c = sub * 32; c < ncols; c += 32 * WARPS_PER_QUAD)
    tmem_zero32(C.tmem + ((uint32_t)(32 * quad) << 16) + (uint32_t)(col0 + c));
  tmem_wait_st();
}

// Tile geometry (the TF32 kernels): accumulator column dcol (multiple of
// DG), B descriptor start row x0 in the copy, width N (multiple of 16).
struct Tile {
  int dcol, x0, N;
};

// accumulator column bases
constexpr int COL_CONV = 0;
__device__ __forceinline__ int col_corr(int m) { return conv_width(m); }

// What a tile sequence computes.
//   CONV_SYM  b = a * a: windows and copies from the heights, 2 products
//             (A_hi B_hi + A_lo2 B_hi), two hi-only copy slots;
//   CONV_X    b = a * y: windows from a, copies from y (hi | lo, one slot),
//             3 products;
//   CORR      G = corr(c, a): windows from a, copies from the weights c
//             (hi | lo, one slot), 3 products.
enum TileMode { CONV_SYM = 0, CONV_X = 1, CORR = 2 };

// Issue the MMAs of one tile (the issuing thread, issue_phase): A
// descriptors ah / al (window hi / lo planes at K step 0), B descriptors
// bh / bl (copy hi / lo planes at the tile's first row), bstep = the B
// advance of one K16 step (16-byte units).  three_prod selects the
// 3-product arithmetic, otherwise the 2-product symmetric convolution.
__device__ __forceinline__ void issue_tile(uint32_t d, uint32_t id, uint64_t ah,
                                           uint64_t al, uint64_t bh, uint64_t bl, uint64_t bstep,
                                           bool three, bool three_prod) {
#pragma unroll
  for (int kc = 0; kc < KSTEPS; ++kc) {
    // K16 step kc = K groups 2kc, 2kc+1: A moves by 256 B, B by two K groups
    const uint64_t a = ah + (uint64_t)(16 * kc), b = bh + bstep * (uint64_t)kc;
    mma_bf16(d, a, b, id, 1u);
    if (three) {
      mma_bf16(d, al + (uint64_t)(16 * kc), b, id, 1u);
      if (three_prod) mma_bf16(d, a, bl + bstep * (uint64_t)kc, id, 1u);
    }
  }
}

// Tiles in the first stage of a tile sequence at most: the MMAs start after
// a short build, and the next, full stage is built while they run
// (measured at n = 8400 with 13-tile stages: the first full stage kept the
// tensor pipe waiting about 2k cycles per tile phase).
constexpr int kLeadTiles = 4;


// The MMA lane's part of a tile phase (run_tiles_ring): wait for the copy,
// then per stage wait for its windows, issue its tiles' MMAs and release it
// with one commit; finally commit the copy slot and bar_done.  A function of
// its own, not inlined, so that the issue loop is compiled apart from the
// kernel around it: inlined, its rate moved with unrelated changes
// elsewhere in the step (the convolution tile phase at n = 8400 measured
// 43.2k and 46.4k cycles in two builds that differed only in how begin()
// zeroes shared memory; 43.4k as a function).  Descriptors advance by
// additions (addresses below 256 KB: the 14-bit address field never
// carries).  Returns the ring position and the stage parities after the
// phase.  THREE: BF16x3 (else BF16x1), a template parameter so that the
// K-step loop has no branch (with the advanced tile geometry: n = 2048
// 45.9k -> 44.2k cycles per candidate-step, n = 8400 132.7k -> 132.3k).
struct IssueArgs {
  uint64_t *full, *empty, *bc_full, *bc_empty, *bar_done;
  int* abort;
  unsigned int* status;
  uint32_t tmem, stages, bc;
  int rows, m, dmax, wps, nst, st;
  uint32_t ph, bc_ph;
};
struct IssueRes {
  int st;
  uint32_t ph;
};
template <bool CORR, bool THREE_PROD, bool THREE>
__device__ __noinline__ IssueRes issue_phase(const IssueArgs A) {
  const uint32_t lbo = b_lbo(A.rows);
  int st = A.st;
  uint32_t ph = A.ph;
  fence_after();
  bool ok = wait_bar(A.abort, &A.bc_full[0], A.bc_ph & 1u, A.status);
  const uint64_t bh0 = sdesc(A.bc, lbo, 128);
  const uint64_t bl0 = sdesc(A.bc + (uint32_t)A.rows * 128u, lbo, 128);
  const uint64_t bstep = (uint64_t)((2u * lbo) >> 4);
  const uint64_t a0 = sdesc(A.stages, 128, 128);
  const uint64_t sstep = (uint64_t)(stage_bytes(A.wps) >> 4);
  const uint64_t aplane = (uint64_t)(stage_plane_bytes(A.wps) >> 4);
  const uint32_t id0 = idesc_bf16(0);
  constexpr bool three = THREE;
  const int m = A.m;
  int per = A.wps < kLeadTiles ? A.wps : kLeadTiles;
  for (int w = 0; ok && w <= A.dmax; w += 2 * per, per = A.wps) {
    if (!wait_bar(A.abort, &A.full[st], (ph >> st) & 1u, A.status)) { ok = false; break; }
    ph ^= 1u << st;
    fence_after();
    uint64_t ah = a0 + sstep * (uint64_t)st;
    const int hn = (A.dmax - w) / 2 + 1;
    // tile v = w + 2h: accumulator columns from dcol, B rows from x0,
    // advanced from tile to tile (x0 falls by 2 and wraps back by DG, with
    // the destination DG columns on, at every DG-th diagonal)
    int dcol, x0;
    if (CORR) {
      dcol = col_corr(m);
      x0 = w;
    } else {
      const int off = w & ~(DG - 1);
      dcol = COL_CONV + off;
      x0 = off - w + ZP;
    }
    for (int h = 0; h < per && h < hn; ++h, ah += 128) {
      const int N = CORR ? corr_n(m) : round_up(m + ZP - x0, 16);
      issue_tile(A.tmem + (uint32_t)dcol, id0 | ((uint32_t)(N >> 3) << 17), ah,
                 ah + aplane, bh0 + (uint64_t)x0, bl0 + (uint64_t)x0, bstep, three, THREE_PROD);
      if (CORR) {
        x0 += 2;
      } else {
        x0 -= 2;
        if (x0 < ZP - DG + 2) {
          x0 += DG;
          dcol += DG;
        }
      }
    }
    mma_commit(&A.empty[st]);
    st = (st + 1 == A.nst) ? 0 : st + 1;
  }
  mma_commit(&A.bc_empty[0]);
  mma_commit(A.bar_done);
  return IssueRes{st, ph};
}

// Run the tiles w = 0, 2, ..., dmax through the warp-specialised pipeline:
// the builders write the phase's B copy once (one copy slot), then the
// windows of wps consecutive tiles (the first stage: at most kLeadTiles)
// into each stage of the ring (one run of core matrices, build_stage); the
// MMA lane issues a stage's tiles in order and releases the stage with one
// commit.
// Every accumulator receives its MMAs in the same order whatever the ring
// shape, so the results do not depend on it.  Ends with every MMA of the sequence
// complete (bar_done) and the accumulator readable by all warps.
//   wsrc: padded shared heights (windows; the copy too for CONV_SYM);
//   bsrc / blen: the copy source of CONV_X (see build_conv_copy) or the
//   padded shared weights of CORR.
//   WPS: tiles per stage fixed at compile time (1: three single-tile
//   stages), or 0 to take the ring shape from C.wps / C.nst.
template <int MODE, bool PREBUILT, int WPS>
__device__ __forceinline__ bool run_tiles_ring(Ctx& C, const float* wsrc, const float* bsrc,
                                               int blen, unsigned int* status) {
  const int wps = WPS ? WPS : C.wps;
  const int nst = WPS ? 3 : C.nst;
  constexpr bool corr = MODE == CORR;
  constexpr bool three_prod = MODE != CONV_SYM;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool want_lo = three_prod && C.three;
  const float lsc = MODE == CONV_SYM ? 2.f : 1.f;
  const int m = C.m;
  const int rows = corr ? C.rcc : C.rc;
  const uint32_t lbo = b_lbo(rows);
  int st = C.st_next;
  if (warp == MMA_WARP) {
    if (lane == 0) {
      IssueArgs A;
      A.full = C.full; A.empty = C.empty; A.bc_full = C.bc_full; A.bc_empty = C.bc_empty;
      A.bar_done = C.bar_done; A.abort = C.abort; A.status = status;
      A.tmem = C.tmem; A.stages = smem_u32(C.stages); A.bc = smem_u32(C.bc);
      A.rows = rows; A.m = m; A.dmax = C.dmax; A.wps = wps; A.nst = nst; A.st = st;
      A.ph = C.ph; A.bc_ph = C.bc_ph;
      const IssueRes R = C.three ? issue_phase<corr, three_prod, true>(A)
                                 : issue_phase<corr, three_prod, false>(A);
      st = R.st;
      C.ph = R.ph;
      C.bc_ph ^= 1u;
    }
    __syncwarp();
  } else if (builder_index() >= 0) {
    const int bt = builder_index();   // 0 .. NBUILD-1
    bool ok = true;
    if ((C.bc_started & 1u) && !wait_phase(C, &C.bc_empty[0], C.bc_ph & 1u, status)) ok = false;
    if (C.bc_started & 1u) C.bc_ph ^= 1u;
    C.bc_started |= 1u;
    if (ok) {
      unsigned char* hi = C.bc;
      if (PREBUILT) {
        // the copy was written (and fenced) by the caller before this phase
      } else if (corr) build_corr_copy(C, bsrc, want_lo, bt);
      else if (MODE == CONV_X) build_conv_copy(C, bsrc, blen, hi, hi + (size_t)rows * 128, want_lo, bt);
      else build_conv_copy(C, wsrc, -1, hi, hi, false, bt);
      fence_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&C.bc_full[0]);
    }
    int per = wps < kLeadTiles ? wps : kLeadTiles;
    for (int w = 0; ok && w <= C.dmax; w += 2 * per, per = wps) {
      if ((C.started >> st) & 1u) {
        if (!wait_phase(C, &C.empty[st], (C.ph >> st) & 1u, status)) {
          ok = false;
          break;
        }
        C.ph ^= 1u << st;
      }
      C.started |= 1u << st;
      const int nt = (C.dmax - w) / 2 + 1;
      build_stage(C, st, wps, wsrc, w, nt < per ? nt : per, lsc, bt);
      fence_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&C.full[st]);
      st = (st + 1 == nst) ? 0 : st + 1;
    }
  }
  C.st_next = st;
  const bool ok = drain_phase(C.bar_done, C.done_ph, status);
  C.done_ph ^= 1u;
  fence_after();
  __syncthreads();
  return ok && !*((volatile int*)C.abort);
}

// The tile sequence on the CTA's ring (ring_for).  Three single-tile
// stages run a specialisation with the shape fixed at compile time, the
// multi-tile shapes one that reads it.  Measured per step: reading the shape
// for the single-tile ring cost 2-4% (n <= 1024 and n = 9728 keep that
// ring); specialising the multi-tile shapes as well measured 1-8% slower
// than reading them (a larger kernel).
template <int MODE, bool PREBUILT = false>
__device__ __forceinline__ bool run_tiles(Ctx& C, const float* wsrc, const float* bsrc, int blen,
                                          unsigned int* status) {
  if (C.wps == 1) return run_tiles_ring<MODE, PREBUILT, 1>(C, wsrc, bsrc, blen, status);
  return run_tiles_ring<MODE, PREBUILT, 0>(C, wsrc, bsrc, blen, status);
}

// lane quadrant of the calling warp and its index among the warps of that
// quadrant (12 warps: 4 quadrants x 3)
struct Lane {
  int quad, sub, r;     // lane quadrant, warp index within it, TMEM lane
  __device__ Lane() {
    const int w = threadIdx.x >> 5;
    quad = w & 3;
    sub = w >> 2;
    r = 32 * quad + (threadIdx.x & 31);
  }
};

// Column chunks [c0, c1) of an accumulator, the quadrant's warp h taking
// chunks c0 + h, c0 + h + WARPS_PER_QUAD, ...: visit(c, v, 0) gets chunk c's
// 32 values (one load and wait per chunk: loading two chunks per wait
// measured 1.9x slower in the convolution gather, 11.2k -> 22.0k cycles at
// n = 8400, with the step kernels spilling).
template <typename Visit>
__device__ __forceinline__ void for_chunks(uint32_t lanebase, int sub, int c0, int c1,
                                           Visit&& visit) {
  for (int c = c0 + sub; c < c1; c += WARPS_PER_QUAD) {
    float v[32];
    tmem_ld32(lanebase + (uint32_t)(32 * c), v);
    visit(c, v, 0);
  }
}

// b = a * a into X (padded layout, k < 2n-1).  Each k is the sum of two
// cells, L = (k mod 64, k / 64) in lanes 0-63 and U = (k mod 64 + 64,
// k / 64 - 1) in lanes 64-127, read by different warps: one writes its cell
// to X, then the other adds its own.  Two rounds keep every warp busy: for
// the k whose lower cell lies in the first half of the column chunks the
// upper lanes write first (round 1) and the lower lanes add (round 2), for
// the rest the lower lanes write first and the upper lanes add; the chunk
// holding the boundary column's upper cell is read in both rounds.  b_k is
// U + L either way (a sum of two floats does not depend on their order).
// (Measured: the three rounds of the earlier form took about as long each
// with four warps as with eight -- the per-chunk TMEM load is the latency.)
// Ends synchronised.  Returns the largest b_k the calling thread finalised
// (every k is finalised by exactly one thread).
__device__ __forceinline__ float gather_conv(Ctx& C, const Lane& ln, float* X) {
  const int nb = 2 * C.n - 1, nch = (2 * C.m + 1 + 31) / 32;
  const int mid = (nch + 1) / 2;                        // lower chunks [0, mid): upper first
  const int cmid = 32 * mid;                            // first lower column of the rest
  const uint32_t lanebase = C.tmem + ((uint32_t)(32 * ln.quad) << 16) + (uint32_t)COL_CONV;
  const bool upper = ln.quad >= 2;
  // cell (r, col) holds a part of k = 64 (col + sh) + rr, at X[68 (col + sh) + rr];
  // k < nb up to column kcol.  A chunk's 32 cells sit 68 floats apart, so
  // each store takes a fixed offset from the chunk's base.
  const int rr = ln.r & 63, sh = ln.r >> 6;
  const int kcol = ((nb - 1 - rr) >> 6) - sh;
  const int xr = 68 * sh + rr;
  float mloc = 0.f;
  // round 1: the first cell of every k
  if (upper) {
    if (ln.sub == 0) X[pidx(ln.r - 64)] = 0.f;          // k < 64: one cell only
    const int hi = kcol < cmid - 2 ? kcol : cmid - 2;   // the upper cell comes first below cmid - 1
    for_chunks(lanebase, ln.sub, 0, mid, [&](int c, const float (&v)[32], int o) {
      float* xc = X + (xr + 68 * 32 * c);
      const int th = hi - 32 * c;
#pragma unroll
      for (int t = 0; t < 32; ++t)
        if (t <= th) xc[68 * t] = v[o + t];
    });
  } else {
    for_chunks(lanebase, ln.sub, mid, nch, [&](int c, const float (&v)[32], int o) {
      float* xc = X + (xr + 68 * 32 * c);
      const int th = kcol - 32 * c;
#pragma unroll
      for (int t = 0; t < 32; ++t)
        if (t <= th) xc[68 * t] = v[o + t];
    });
  }
  __syncthreads();
  // round 2: the second cell, added; its thread finalises b_k (the upper
  // lanes have none to add when every k lies below 64 cmid)
  if (upper) {
    if (64 * cmid < nb)
      for_chunks(lanebase, ln.sub, mid - 1, nch, [&](int c, const float (&v)[32], int o) {
        float* xc = X + (xr + 68 * 32 * c);
        const int tl = cmid - 1 - 32 * c, th = kcol - 32 * c;
#pragma unroll
        for (int t = 0; t < 32; ++t)
          if (t >= tl && t <= th) {
            const float b = xc[68 * t] + v[o + t];
            xc[68 * t] = b;
            mloc = fmaxf(mloc, b);
          }
      });
  } else {
    for_chunks(lanebase, ln.sub, 0, mid, [&](int c, const float (&v)[32], int o) {
      float* xc = X + (xr + 68 * 32 * c);
      const int th = kcol - 32 * c;
#pragma unroll
      for (int t = 0; t < 32; ++t)
        if (t <= th) {
          const float b = xc[68 * t] + v[o + t];
          xc[68 * t] = b;
          mloc = fmaxf(mloc, b);
        }
    });
  }
  __syncthreads();
  return mloc;
}

// G_i into Y (padded layout, i < n) from the correlation accumulator: cell
// (r, col) holds a part of i = 64 col + 63 - r; the upper-lane cell of i sits
// one column right of its lower-lane cell.  Two rounds, every warp busy in
// both: for the i whose lower cell lies in the first `cmid` columns the lower
// lanes write first and the upper lanes add (their cell lies at most at
// column cmid, so the upper warps also read the chunk holding column cmid),
// for the rest the upper lanes write first and the lower lanes add.  G_i is
// L + U either way (a sum of two floats does not depend on their order).
// Ends synchronised.
__device__ __forceinline__ void gather_corr(Ctx& C, const Lane& ln, float* Y) {
  const int n = C.n, nch = (corr_n(C.m) + 31) / 32;
  const int mid = nch / 2, cmid = 32 * mid;
  const uint32_t lanebase = C.tmem + ((uint32_t)(32 * ln.quad) << 16) + (uint32_t)col_corr(C.m);
  const bool upper = ln.quad >= 2;
  // cell (r, col) holds a part of i = 64 (col - sh) + ri, at Y[68 (col - sh) + ri];
  // 0 <= i < n for columns sh .. icol
  const int ri = 63 - (ln.r & 63), sh = ln.r >> 6;
  const int icol = ((n - 1 - ri) >> 6) + sh;
  const int yr = ri - 68 * sh;
  // round 1: lower cells of columns < cmid, upper cells of columns > cmid
  if (upper) {
    const int lo = cmid + 1;
    for_chunks(lanebase, ln.sub, mid, nch, [&](int c, const float (&v)[32], int o) {
      const int yc = yr + 68 * 32 * c;
      const int tl = lo - 32 * c, th = icol - 32 * c;
#pragma unroll
      for (int t = 0; t < 32; ++t)
        if (t >= tl && t <= th) Y[yc + 68 * t] = v[o + t];
    });
  } else {
    for_chunks(lanebase, ln.sub, 0, mid, [&](int c, const float (&v)[32], int o) {
      const int yc = yr + 68 * 32 * c;
      const int th = icol - 32 * c;
#pragma unroll
      for (int t = 0; t < 32; ++t)
        if (t <= th) Y[yc + 68 * t] = v[o + t];
    });
  }
  __syncthreads();
  // round 2: the partner cells, added
  if (upper) {
    const int hi = icol < cmid ? icol : cmid;
    for_chunks(lanebase, ln.sub, 0, mid < nch ? mid + 1 : nch, [&](int c, const float (&v)[32], int o) {
      const int yc = yr + 68 * 32 * c;
      const int tl = sh - 32 * c, th = hi - 32 * c;
#pragma unroll
      for (int t = 0; t < 32; ++t)
        if (t >= tl && t <= th) Y[yc + 68 * t] += v[o + t];
    });
  } else {
    for_chunks(lanebase, ln.sub, mid, nch, [&](int c, const float (&v)[32], int o) {
      const int yc = yr + 68 * 32 * c;
      const int th = icol - 32 * c;
#pragma unroll
      for (int t = 0; t < 32; ++t)
        if (t <= th) Y[yc + 68 * t] += v[o + t];
    });
  }
  __syncthreads();
}

// b = a * a (accumulator at COL_CONV)
__device__ __forceinline__ bool conv_tc(Ctx& C, const float* sa, unsigned int* status) {
  return run_tiles<CONV_SYM>(C, sa, nullptr, 0, status);
}
// the same with the B copy already in place (conv_copy_chunk, then
// fence_async_smem and a barrier by the writers)
__device__ __forceinline__ bool conv_tc_prebuilt(Ctx& C, const float* sa, unsigned int* status) {
  return run_tiles<CONV_SYM, true>(C, sa, nullptr, 0, status);
}
// Write chunk (row x, K group h) of the autoconvolution copy (hi plane):
// v[s] = a[64 (x - ZP) + 63 - 8 h - s], s < 8 (layout of build_conv_copy).
__device__ __forceinline__ void conv_copy_chunk(Ctx& C, int x, int h, const float (&v)[8]) {
  uint4 vh, vl;
  split8(v, 1.f, vh, vl);
  *reinterpret_cast<uint4*>(C.bc + (uint32_t)h * b_lbo(C.rc) + 16u * (uint32_t)x) = vh;
}
// b = a * y (accumulator at COL_CONV); y: a plain global row of ylen cells
__device__ __forceinline__ bool convx_tc(Ctx& C, const float* sa, const float* y, int ylen,
                                         unsigned int* status) {
  return run_tiles<CONV_X>(C, sa, y, ylen, status);
}
// G = corr(c, a) (accumulator at col_corr); cb: padded weights (zero beyond 2n-1)
__device__ __forceinline__ bool corr_tc(Ctx& C, const float* sa, const float* cb,
                                        unsigned int* status) {
  return run_tiles<CORR>(C, sa, cb, 0, status);
}
// the same with the B copy already in place (corr_copy_chunk, then
// fence_async_smem and a barrier by the writers)
__device__ __forceinline__ bool corr_tc_prebuilt(Ctx& C, const float* sa, unsigned int* status) {
  return run_tiles<CORR, true>(C, sa, nullptr, 0, status);
}

// Write chunk (row x, K group h) of the correlation copy: the weights
// c[64 x + 8 h + j], j < 8, as hi and lo planes (layout of build_corr_copy).
__device__ __forceinline__ void corr_copy_chunk(Ctx& C, int x, int h, const float (&v)[8]) {
  const int rows = C.rcc;
  uint4 vh, vl;
  split8(v, 1.f, vh, vl);
  const uint32_t off = (uint32_t)h * b_lbo(rows) + 16u * (uint32_t)x;
  *reinterpret_cast<uint4*>(C.bc + off) = vh;
  if (C.three) *reinterpret_cast<uint4*>(C.bc + (size_t)rows * 128 + off) = vl;
}

}  // namespace tc
}  // namespace sidon
