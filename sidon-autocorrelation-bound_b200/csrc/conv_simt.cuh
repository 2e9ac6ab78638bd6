// ---------------------------------------------------------------------------
//  conv_simt.cuh -- warp-tiled convolution / correlation on the CUDA cores.
//
//  Restates crossconv / corrTile (src/kernels.cuh:97-158) with a layout
//  chosen for sm_100:
//    * a warp owns a tile of W = 32*TK consecutive outputs, lane l owns TK
//      consecutive outputs k0 = kw + l*TK ... ; lanes read their window
//      operand at a stride of TK words, and TK is odd, so every window load
//      is bank-conflict free (the reference's TK = 8 stride is 8-way);
//    * all lanes of a warp run the same (warp-uniform) summation range, so
//      there is no divergence; terms outside an output's own range read the
//      zero margins and add exactly +0;
//    * the window is a rotating register file (unrolled by TK), one new
//      shared load + one broadcast load per TK FMAs;
//    * each output is ONE fma chain over the summation index in increasing
//      order, starting from +0 -- the same arithmetic as the oracle, so the
//      fp32 results are bit-identical to it;
//    * conv tiles are visited in a static longest-first order (the tile
//      holding k = n-1 carries the most terms), snaked across warps.
//
//  Operand buffers are pointers to element 0 of arrays with zero margins of
//  at least margin<TK>() elements on BOTH sides.
// ---------------------------------------------------------------------------
#pragma once
#include "common.cuh"

namespace sidon {

template <int TK>
__host__ __device__ constexpr int margin() { return 32 * TK + 32; }

// multiply-add flavours: FUSED = one fma per term (search arithmetic);
// !FUSED = product rounded, then added (hostF arithmetic, src/main.cu:100).
template <bool FUSED, typename T>
__device__ __forceinline__ T madd(T x, T y, T acc) {
  if constexpr (FUSED) return dev_fma(x, y, acc);
  else {
    if constexpr (sizeof(T) == 8) return __dadd_rn(acc, __dmul_rn(x, y));
    else return __fadd_rn(acc, __fmul_rn(x, y));
  }
}

// position p of the longest-first order -> conv tile index.  c = tile of
// k = n-1, Q tiles; distances from c alternate right/left, then the longer
// side alone.
__device__ __forceinline__ int conv_tile_at(int p, int c, int Q) {
  if (p == 0) return c;
  const int m = min(c, Q - 1 - c);
  const int j = (p + 1) >> 1;
  if (j <= m) return (p & 1) ? c + j : c - j;
  const int extra = p - 2 * m;
  return (c >= Q - 1 - c) ? (c - m - extra) : (c + m + extra);
}

// The threads of a CTA that work on the current candidate: the first nt
// (a multiple of 32).  A CTA sized for a larger candidate of a ragged batch
// leaves the others idle except at barriers, where idle warps contribute
// exact zeros to block reductions, so a candidate's result does not depend on
// the batch it runs in.
struct Team {
  int nt;  // working threads
  int t0;  // threadIdx.x for a working thread, else past every loop bound
  __device__ explicit Team(int nthreads)
      : nt(nthreads), t0((int)threadIdx.x < nthreads ? (int)threadIdx.x : 0x3fffffff) {}
  __device__ Team() : Team((int)blockDim.x) {}
  __device__ bool active() const { return t0 < nt; }
};

// b_k = sum_i x_i y_{k-i}, k in [0, 2n-1), by NW warps of which this lane's
// warp is number wid.  epi(k, value) is called once per output k < 2n-1 by
// the lane that owns it.
template <int TK, bool FUSED, typename T, typename Epi>
__device__ __forceinline__ void conv_tiles(const T* __restrict__ x, const T* __restrict__ y, int n,
                                           int wid, int NW, int lane, Epi&& epi) {
  constexpr int W = 32 * TK;
  const int nb = 2 * n - 1;
  const int Q = (nb + W - 1) / W;
  const int c = (n - 1) / W;
  for (int r = 0;; ++r) {
    const int p = r * NW + ((r & 1) ? (NW - 1 - wid) : wid);
    if (p >= Q) break;
    const int q = conv_tile_at(p, c, Q);
    const int kw = q * W;
    const int ilo = max(0, kw - (n - 1));
    const int ihi = min(kw + W - 1, n - 1);
    const int trips = (ihi - ilo + TK) / TK;
    const int k0 = kw + lane * TK;
    T acc[TK], rw[TK];
#pragma unroll
    for (int t = 0; t < TK; ++t) { acc[t] = T(0); rw[t] = y[k0 + t - ilo]; }
    const T* xp = x + ilo;
    const T* yp = y + (k0 - ilo - 1);
    for (int tr = 0; tr < trips; ++tr) {
#pragma unroll
      for (int u = 0; u < TK; ++u) {
        const T xv = xp[u];
#pragma unroll
        for (int t = 0; t < TK; ++t) acc[t] = madd<FUSED>(xv, rw[(t - u + TK) % TK], acc[t]);
        rw[(TK - 1 - u + TK) % TK] = yp[-u];
      }
      xp += TK;
      yp -= TK;
    }
#pragma unroll
    for (int t = 0; t < TK; ++t)
      if (k0 + t < nb) epi(k0 + t, acc[t]);
  }
}

// conv_tiles over the warps of a team
template <int TK, bool FUSED, typename T, typename Epi>
__device__ __forceinline__ void conv_warp_tiles(const T* __restrict__ x, const T* __restrict__ y,
                                                int n, const Team& tm, Epi&& epi) {
  if (!tm.active()) return;
  conv_tiles<TK, FUSED>(x, y, n, (int)(threadIdx.x >> 5), tm.nt >> 5, (int)(threadIdx.x & 31),
                        epi);
}

// G_i = sum_j c_{i+j} a_j, i in [0, n), by NW warps (this lane's is wid).
// epi(i, value) once per i < n.  c must be valid (zero) up to index
// 2n - 2 + margin.
template <int TI, typename T, typename Epi>
__device__ __forceinline__ void corr_tiles(const T* __restrict__ a, const T* __restrict__ cc, int n,
                                           int wid, int NW, int lane, Epi&& epi) {
  constexpr int W = 32 * TI;
  const int Q = (n + W - 1) / W;
  const int trips = (n + TI - 1) / TI;
  for (int q = wid; q < Q; q += NW) {
    const int i0 = q * W + lane * TI;
    T acc[TI], rw[TI];
#pragma unroll
    for (int s = 0; s < TI; ++s) { acc[s] = T(0); rw[s] = cc[i0 + s]; }
    const T* ap = a;
    const T* cp = cc + i0 + TI;
    for (int tr = 0; tr < trips; ++tr) {
#pragma unroll
      for (int u = 0; u < TI; ++u) {
        const T av = ap[u];
#pragma unroll
        for (int s = 0; s < TI; ++s) acc[s] = dev_fma(av, rw[(s + u) % TI], acc[s]);
        rw[u % TI] = cp[u];
      }
      ap += TI;
      cp += TI;
    }
#pragma unroll
    for (int s = 0; s < TI; ++s)
      if (i0 + s < n) epi(i0 + s, acc[s]);
  }
}

// corr_tiles over the warps of a team
template <int TI, typename T, typename Epi>
__device__ __forceinline__ void corr_warp_tiles(const T* __restrict__ a, const T* __restrict__ cc,
                                                int n, const Team& tm, Epi&& epi) {
  if (!tm.active()) return;
  corr_tiles<TI>(a, cc, n, (int)(threadIdx.x >> 5), tm.nt >> 5, (int)(threadIdx.x & 31), epi);
}

// warps a CTA should have so one round of correlation tiles covers n
template <int TI>
__host__ __device__ inline int warps_for(int n) {
  const int w = (n + 32 * TI - 1) / (32 * TI);
  return w < 4 ? 4 : (w > 32 ? 32 : w);
}

}  // namespace sidon
