// ---------------------------------------------------------------------------
//  tc_cta.cuh -- the per-CTA frame of the tensor-core kernels: the shared-
//  memory plan, barrier / TMEM set-up and release, and the per-candidate
//  reset.  One CTA = 12 warps = one tile pipeline (tc_engine.cuh).
//
//  Shared memory (see Layout):
//    stages  the window ring (ring_for): 3 stages of one tile's window
//            (6 KB: hi | lo planes of 24 core matrices) or 2 stages of the
//            windows of T = 2 .. 5 consecutive tiles (2 x (16 T + 8) core
//            matrices, 10-22 KB); in the wide plan of the fused local
//            search, 2 stages of up to 16 tiles sharing one region with cb
//    bc      the tile phase's B-matrix copy (hi, or hi | lo); after a
//            tile phase, gather scratch for up to 2n-1 outputs
//    sa      fp32 heights, padded block layout (cell i at i + 4 floor(i/64)),
//            zero margins on both sides
//    cb      fp32 padded scratch: b, then the weights c, then G
//    red     64 floats of reduction scratch, mbarriers, TMEM address, abort flag
// ---------------------------------------------------------------------------
#pragma once
#include "tc_engine.cuh"

namespace sidon {
namespace tc {

// Shared memory a multi-tile ring may grow the plan to: the sm_100
// per-block opt-in limit (227 KB) less 1 KB for the kernels' static shared
// variables (at most 264 bytes).  (The single-tile ring is taken at any size.)
constexpr size_t kSmemBudget = 232448 - 1024;
// Tile sequences of at least this many blocks take the multi-tile stages
// (per step, identical results: the same at n = 1024, 16 blocks; 3-9% faster
// from n = 2048 on; at n = 512, 8 blocks and 5 tiles, two-tile stages were 4%
// slower).
constexpr int kRingMinBlocks = 16;
constexpr int kMaxStageTiles = 5;
constexpr int kWideMinTiles = 8;     // see Layout's wide plan

struct Ring {
  int stages, per_stage;    // stages, tiles per stage
};
// The window ring for m blocks when everything else takes `other` bytes:
// two stages of as many tiles (up to five) as the budget allows when the
// sequence is long, else three single-tile stages.
__host__ __device__ __forceinline__ Ring ring_for(int m, size_t other) {
  if (m >= kRingMinBlocks)
    for (int T = kMaxStageTiles; T >= 2; --T)
      if (other + 2 * (size_t)stage_bytes(T) <= kSmemBudget) return Ring{2, T};
  return Ring{3, 1};
}
// A ring chosen by the schedule tuner: tiles per stage T (1: three
// single-tile stages, 2..5: two stages of T tiles), 0 = ring_for's choice.
// Every shape gives the same results bit for bit (each accumulator receives
// its MMAs in the same order); the tuner offers only shapes that fit.
__host__ __device__ __forceinline__ Ring ring_of(int tiles) {
  return tiles == 1 ? Ring{3, 1} : Ring{2, tiles};
}

// The widest two-stage ring a plan can hold when the ring shares its space
// with the scratch cb (the fused local search: cb is dead during both tile
// phases of a step) and everything else takes `other` bytes.
constexpr int kMaxWideTiles = 16;
__host__ __device__ __forceinline__ int wide_tiles(size_t other) {
  int T = 0;
  for (int t = 2; t <= kMaxWideTiles; ++t)
    if (other + 2 * (size_t)stage_bytes(t) <= kSmemBudget) T = t;
  return T;
}

// dynamic shared memory plan (byte offsets from a 1 KB aligned base)
//   wide = false: [ring][copy region][sa][cb][red];
//   wide = true:  [ring | cb][copy region][sa][red] -- the ring and the
//   scratch cb share one region, for kernels that use cb only outside tile
//   phases (the fused local search); the ring then grows to as many tiles
//   per stage as the budget allows (13 at n = 8400), so a tile phase commits
//   fewer stages.
struct Layout {
  int m, rc, rcc, sa_len, cb_len;
  Ring ring;
  bool wide;
  size_t off_bc, off_sa, off_cb, off_red, total;
  __host__ __device__ Layout(int n, int ring_tiles = 0, bool wide_plan = false) {
    m = (n + BL - 1) / BL;
    rc = conv_copy_rows(m);
    rcc = corr_copy_rows(m);
    sa_len = 68 * (m + 8);                 // padded heights, 136 cells of margin in front
    cb_len = 68 * (2 * m + 2);             // padded weights / gather scratch
    wide = wide_plan;
    if (wide) {
      const size_t cb_bytes = ((size_t)cb_len * 4 + 1023) & ~(size_t)1023;
      // as wide as fits, but about five stages per tile phase at least and
      // kWideMinTiles tiles per stage at least (the first stage holds at
      // most kLeadTiles, so a wide stage delays no MMA; the schedule tuner
      // chose 8-12 tiles at n = 1024-4096, 1.4-1.9% faster than 5-7)
      const int tiles = last_tile(n) / 2 + 1;
      int T = wide_tiles(place_wide(0));
      const int want = (tiles + 4) / 5 > kWideMinTiles ? (tiles + 4) / 5 : kWideMinTiles;
      if (T > want) T = want;
      if (ring_tiles > 0) ring = ring_of(ring_tiles);
      else if (m >= kRingMinBlocks && T >= 2) ring = Ring{2, T};
      else ring = ring_for(m, place_wide(cb_bytes));
      const size_t rb = (size_t)ring.stages * stage_bytes(ring.per_stage);
      place_wide(rb > cb_bytes ? rb : cb_bytes);
      return;
    }
    // the ring takes whole KB: the rest keeps its padding
    ring = ring_tiles > 0 ? ring_of(ring_tiles) : ring_for(m, place(0));
    place((size_t)ring.stages * stage_bytes(ring.per_stage));
  }
  // wide plan: cb at the start of a shared region of `o` bytes, the rest after
  // it; returns the total
  __host__ __device__ size_t place_wide(size_t o) {
    off_cb = 0;
    off_bc = o;
    const int rows = rcc > rc ? rcc : rc;
    const size_t region = (size_t)2 * rows * 128;
    o += region > (size_t)cb_len * 4 ? region : (size_t)cb_len * 4;
    off_sa = o;
    o += (size_t)sa_len * 4;
    o = (o + 15) & ~(size_t)15;
    off_red = o;
    o += 64 * 4 + (2 * MAX_STAGES + 6) * 8 + 16;
    total = o + 1024;
    return total;
  }
  // lay out everything after a ring of `o` bytes; returns the total
  __host__ __device__ size_t place(size_t o) {
    off_bc = o;
    const int rows = rcc > rc ? rcc : rc;
    // one B copy (hi, or hi|lo) of up to max(rc, rcc) rows; after a tile
    // phase, gather scratch
    // for up to 2n-1 outputs in the padded layout
    const size_t region = (size_t)2 * rows * 128;
    o += region > (size_t)cb_len * 4 ? region : (size_t)cb_len * 4;
    off_sa = o;
    o += (size_t)sa_len * 4;
    o = (o + 15) & ~(size_t)15;
    off_cb = o;
    o += (size_t)cb_len * 4;
    o = (o + 15) & ~(size_t)15;
    off_red = o;
    o += 64 * 4 + (2 * MAX_STAGES + 6) * 8 + 16;
    total = o + 1024;                      // slack for aligning the dynamic base to 1 KB
    return total;
  }
};

struct Shared {
  Ctx C;
  float* sa;     // padded heights, logical cell 0
  float* cb;     // padded weights / gather scratch, logical index 0
  float* red;
};

// Per-CTA set-up for candidates of up to n_max cells: buffer addresses,
// barriers, TMEM.  begin() then prepares one candidate.
__device__ __forceinline__ Shared setup(int n_max, bool three, unsigned char* raw,
                                        int ring_tiles = 0, bool wide = false) {
  const Layout Lo(n_max, ring_tiles, wide);
  unsigned char* base = (unsigned char*)(((uintptr_t)raw + 1023) & ~(uintptr_t)1023);
  Shared S;
  S.C.stages = base;
  S.C.bc = base + Lo.off_bc;
  S.sa = reinterpret_cast<float*>(base + Lo.off_sa) + 136;
  S.cb = reinterpret_cast<float*>(base + Lo.off_cb);
  S.red = reinterpret_cast<float*>(base + Lo.off_red);
  uint64_t* bars = reinterpret_cast<uint64_t*>(S.red + 64);
  S.C.full = bars;
  S.C.empty = bars + MAX_STAGES;
  S.C.bc_full = bars + 2 * MAX_STAGES;
  S.C.bc_empty = bars + 2 * MAX_STAGES + 2;
  S.C.bar_done = bars + 2 * MAX_STAGES + 4;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 2 * MAX_STAGES + 6);
  S.C.abort = reinterpret_cast<int*>(tslot + 1);
  S.C.m = Lo.m;
  S.C.rc = Lo.rc;
  S.C.rcc = Lo.rcc;
  S.C.n = n_max;
  S.C.dmax = last_tile(n_max);
  S.C.three = three;
  S.C.ph = S.C.started = S.C.bc_ph = S.C.bc_started = S.C.done_ph = 0u;
  S.C.st_next = 0;
  S.C.nst = Lo.ring.stages;
  S.C.wps = Lo.ring.per_stage;
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

// Prepare the CTA for a candidate of n cells (n <= n_max of setup): zero the
// height and scratch buffers (their margins must read as zero) and set the
// geometry.  Ends synchronised.
__device__ __forceinline__ void begin(Shared& S, int n, int n_max) {
  const Layout Lo(n_max), Ln(n);
  // 16-byte stores: both arrays start 16-byte aligned and hold multiples
  // of 4 floats (3.3k -> 1.1k cycles at n = 8400 against 4-byte stores)
  float4* z0 = reinterpret_cast<float4*>(S.sa - 136);
  float4* z1 = reinterpret_cast<float4*>(S.cb);
  const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
  __syncthreads();
  for (int i = threadIdx.x; i < Lo.sa_len / 4; i += blockDim.x) z0[i] = z;
  for (int i = threadIdx.x; i < Lo.cb_len / 4; i += blockDim.x) z1[i] = z;
  S.C.n = n;
  S.C.m = Ln.m;
  S.C.rc = Ln.rc;
  S.C.rcc = Ln.rcc;
  S.C.dmax = last_tile(n);
  __syncthreads();
}

// Heights of a candidate (global row a, n cells) into the padded shared
// layout S.sa, through L2.  When the row allows (16-byte aligned start, n a
// multiple of 4) every thread moves 16-byte groups of 4 cells (a group
// never straddles a 64-cell block, so it lands contiguous in the padded
// layout).  Measured at n = 8400, per candidate: 3.3k cycles, against 9.2k
// for 1-D bulk copies (cp.async.bulk, one per 64-cell block from the lanes
// of one warp, completing on an mbarrier) and about as long for 4-byte
// loads.  begin() must have run (it zeroes the margins).  Ends synchronised.
__device__ __forceinline__ void load_heights(Shared& S, const float* a, int n) {
  if (((reinterpret_cast<uintptr_t>(a) & 15) == 0) && (n % 4 == 0)) {
#pragma unroll 4
    for (int q = threadIdx.x; q < n / 4; q += blockDim.x)
      *reinterpret_cast<float4*>(S.sa + pidx(4 * q)) = __ldcg(reinterpret_cast<const float4*>(a) + q);
  } else {
    for (int i = threadIdx.x; i < n; i += blockDim.x) S.sa[pidx(i)] = __ldcg(a + i);
  }
  __syncthreads();
}

__device__ __forceinline__ void teardown(Shared& S) {
  fence_before();
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) {
    fence_after();
    tmem_dealloc(S.C.tmem, 512);
  }
}

// zero both accumulators and hand the tensor memory to the MMA warp
__device__ __forceinline__ void prime(Ctx& C, bool corr_too) {
  zero_acc(C, COL_CONV, conv_width(C.m));
  if (corr_too) zero_acc(C, col_corr(C.m), corr_width(C.m));
  fence_before();
  __syncthreads();
}

}  // namespace tc
}  // namespace sidon
