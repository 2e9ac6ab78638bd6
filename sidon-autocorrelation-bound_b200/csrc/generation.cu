// ---------------------------------------------------------------------------
//  generation.cu -- one generation of the memetic island search
//  (src/main.cu:586-785) as a fixed sequence of launches on one stream:
//
//    k_tiers      anneal tier of every slot from the operator that made it
//    3 x local search (cold / medium / warm tier, skip masks, mirror islands)
//    Frank-Wolfe, fp64 evaluation, support signatures
//    k_select     incumbent, level best, tabu table, island ranking,
//                 migration, offspring plan
//    variation -> workspace, copied over the population
//    k_post       operator record, reinjection of the incumbent
//    fp64 evaluation of the offspring
//    k_credit     bandit credit, generation counter
//
//  The reference decides the policy on the host between synchronous copies;
//  here it runs in single-CTA kernels on state kept in device memory, so a
//  generation needs no host round trip and any number of them can be held
//  in one CUDA graph.  The policy kernels are tiny next to the search (one
//  CTA, O(P * island size) work); the generation's time is the local search
//  and Frank-Wolfe launches.
//
//  Arithmetic: every policy quantity is fp64 in the reference's expression
//  order, compiled without FMA contraction, so the host restatement gives
//  the same bits.  Draws: Philox4x32-10 with the key derived from the seed
//  and the counter (slot, generation, level, q), eight 53-bit uniforms per
//  slot: u0..u3 the two tournaments, u4 the operator, u5 the diversifying
//  operator, u6 the restart coin, u7 the strength.
// ---------------------------------------------------------------------------
#include <cmath>
#include <cstring>
#include <new>

#include "common.cuh"
#include "philox.cuh"

namespace sidon_host {
int launch_variation(const void* pop, void* out, int dtype, int n, int n_off, const int* p1,
                     const int* p2, const int* op, const float* strength,
                     unsigned long long seed, unsigned long long gen, cudaStream_t st,
                     const unsigned long long* gen_dev);
int prepare_local_search_tc(int n_max);
int prepare_frank_wolfe_tc(int n_max);
int prepare_simt(int n_max, bool local_search);
int tc_n_ok_public(int n);
size_t smem_local_search_tc(int n);
int launch_local_search(void* pop, void* mom, void* vel, const long long* offsets,
                        const int* order, int P, int n_fixed, int n_max, const int* skip,
                        const int* mode_arr, int iters, double pS, double pE, double lrS,
                        double lrE, double b1, double b2, int mode_default, int dtype,
                        cudaStream_t st);
int launch_local_search_tc_plain(float* pop, float* mom, float* vel, const long long* offsets,
                                 const int* order, int P, int n_fixed, int n_max, const int* skip,
                                 const int* mode_arr, int iters, double pS, double pE,
                                 double lrS, double lrE, double b1, double b2, int mode_default,
                                 int precision, cudaStream_t st);
}  // namespace sidon_host

namespace sidon {
namespace gen {

constexpr int BD = 1024;
constexpr int NOPS = 14;
constexpr int OP_CLONE = 20;
constexpr int OP_RESTART = 9;
constexpr int kMaxP = 8192;            // the signature copy of k_select: 8 P bytes of smem

// device arrays of the workspace
struct W {
  float* nxt;
  float* mom;
  float* vel;
  double* fit;
  double* parent_fit;
  double* child_fit;
  int* nact;
  int* child_nact;
  unsigned long long* sig;
  int* nnz;
  int* p1;
  int* p2;
  int* op;
  float* strength;
  int* cur_op;
  int* mode;
  int* rank;
  int* skip;                           // [3][P]
  float* best_row;
  sidon_generation_state* st;
  unsigned long long* var_gen;         // generation counter of the variation streams
  unsigned long long* tkey;
  double* tbest;
  int* thits;
  int* tused;
};

// launch-invariant parameters
struct Q {
  int n, P, NI, PI, elite, tenure, cap;
  int cold_iters, med_iters, warm_iters;
  int fw_rounds, fw_iters;
  unsigned long long seed;
};

// splitmix64 finaliser: the home slot of a signature
__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
  x ^= x >> 30;
  x *= 0xBF58476D1CE4E5B9ull;
  x ^= x >> 27;
  x *= 0x94D049BB133111EBull;
  x ^= x >> 31;
  return x;
}

// Entry of key in the open-addressing table (linear probing; key 0 lives in
// the extra entry cap).  insert: claim an empty entry when absent, *fresh
// tells whether it was claimed now.  -1: absent (lookup) or table full.
__device__ int tabu_slot(const W& w, int cap, unsigned long long key, bool insert, bool* fresh) {
  *fresh = false;
  if (key == 0ull) {
    if (insert) {
      *fresh = atomicExch(&w.tused[cap], 1) == 0;
      return cap;
    }
    return w.tused[cap] ? cap : -1;
  }
  const unsigned long long h = mix64(key);
  for (int c = 0; c < cap; ++c) {
    const int i = (int)((h + (unsigned long long)c) & (unsigned long long)(cap - 1));
    if (insert) {
      const unsigned long long prev = atomicCAS(&w.tkey[i], 0ull, key);
      if (prev == 0ull) {
        w.tused[i] = 1;
        *fresh = true;
        return i;
      }
      if (prev == key) return i;
    } else {
      const unsigned long long k = ((volatile unsigned long long*)w.tkey)[i];
      if (k == key) return i;
      if (k == 0ull) return -1;
    }
  }
  return -1;
}

// island order: ascending F, NaN last, ties by slot
__device__ __forceinline__ bool before(double fa, int a, double fb, int b) {
  const bool na = fa != fa, nb = fb != fb;
  if (na != nb) return nb;
  if (!na && fa != fb) return fa < fb;
  return a < b;
}

__device__ __forceinline__ int pos_of(double u, int m) {
  const int k = (int)(u * (double)m);
  return k < m - 1 ? k : m - 1;
}

// block-wide exclusive prefix count of a flag, with the block total
__device__ __forceinline__ int block_excl_count(bool f, int* s_warp, int* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const unsigned m = __ballot_sync(0xffffffffu, f);
  if (lane == 0) s_warp[wid] = __popc(m);
  __syncthreads();
  int before_w = 0, tot = 0;
  for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
    if (i < wid) before_w += s_warp[i];
    tot += s_warp[i];
  }
  __syncthreads();
  *total = tot;
  return before_w + __popc(m & ((1u << lane) - 1u));
}

__global__ void k_init(W w) {
  if (threadIdx.x != 0) return;
  sidon_generation_state* s = w.st;
  s->best_F = 1e30;
  s->level_best_F = 1e30;
  for (int o = 0; o < NOPS; ++o) {
    s->op_weight[o] = 1.0;
    s->op_use[o] = 0.0;
    s->op_win[o] = 0.0;
  }
  s->op_weight[11] = 2.5;
  s->op_weight[12] = 1.8;
  s->op_weight[13] = 1.8;
}

__global__ void k_begin(W w, Q q, int level, const int* __restrict__ seed_op) {
  for (int p = threadIdx.x; p < q.P; p += blockDim.x) {
    w.cur_op[p] = seed_op ? seed_op[p] : OP_RESTART;
    w.mode[p] = ((p / q.PI) % 4 == 3) ? 1 : 0;
  }
  if (threadIdx.x == 0) {
    sidon_generation_state* s = w.st;
    s->gen = 0;
    s->level = level;
    s->n = q.n;
    s->since_improve = 0;
    s->level_best_F = 1e30;
    s->improved = 0;
  }
}

__global__ void k_set_best(W w, const float* __restrict__ row, int n, double F) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) w.best_row[i] = row[i];
  if (threadIdx.x == 0) {
    w.st->best_F = F;
    w.st->best_n = n;
  }
}

// Anneal tiers (main.cu:606-616): cold = the first max(1, 0.18 P) slots
// made by op 9 or 11; medium = the other 9/11 and ops 10, 5, 7, 8, 12, 13;
// warm = the rest.  Writes the three skip masks and the effort counters.
__global__ void __launch_bounds__(BD) k_tiers(W w, Q q) {
  __shared__ int s_warp[32];
  __shared__ int s_cnt[3];
  if (threadIdx.x < 3) s_cnt[threadIdx.x] = 0;
  const int cold_cap = (int)(0.18 * (double)q.P) > 1 ? (int)(0.18 * (double)q.P) : 1;
  int carry = 0;
  for (int base = 0; base < q.P; base += blockDim.x) {
    const int p = base + threadIdx.x;
    const int o = p < q.P ? w.cur_op[p] : -1;
    const bool struc = o == 9 || o == 11;
    int tot = 0;
    const int ex = carry + block_excl_count(struc, s_warp, &tot);
    carry += tot;
    if (p < q.P) {
      int t = 2;
      if (struc && ex < cold_cap) t = 0;
      else if (struc || o == 10 || o == 5 || o == 7 || o == 8 || o == 12 || o == 13) t = 1;
      for (int k = 0; k < 3; ++k) w.skip[k * q.P + p] = t == k ? 0 : 1;
      atomicAdd(&s_cnt[t], 1);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    sidon_generation_state* s = w.st;
    const double n2 = (double)q.n * (double)q.n;
    const int iters[3] = {q.cold_iters, q.med_iters, q.warm_iters};
    s->n_cold = s_cnt[0];
    s->n_med = s_cnt[1];
    for (int t = 0; t < 3; ++t)
      if (s_cnt[t] > 0) {
        s->ls_steps += (long long)s_cnt[t] * iters[t];
        s->flop += 4.0 * n2 * (double)s_cnt[t] * (double)iters[t];
      }
  }
}

// Selection (main.cu:641-730).  One CTA; sig is staged in shared memory.
__global__ void __launch_bounds__(BD) k_select(float* __restrict__ pop, W w, Q q, int fw_ran) {
  extern __shared__ unsigned long long s_sig[];
  __shared__ double s_bf[32];
  __shared__ int s_bi[32];
  __shared__ int s_best, s_impr, s_cnt[NOPS];
  __shared__ double s_bestF;
  sidon_generation_state* st = w.st;
  const int P = q.P, n = q.n, tid = threadIdx.x;
  const int gen = st->gen;

  // incumbent: the first minimum of fit, as a strict-< scan from slot 0
  double bf = 0.0;
  int bi = -1;
  for (int p = tid; p < P; p += blockDim.x) {
    const double f = w.fit[p];
    if (f != f) continue;
    if (bi < 0 || f < bf) {
      bf = f;
      bi = p;
    }
  }
  for (int off = 16; off > 0; off >>= 1) {
    const double of = __shfl_xor_sync(0xffffffffu, bf, off);
    const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
    if (oi >= 0 && (bi < 0 || of < bf || (of == bf && oi < bi))) {
      bf = of;
      bi = oi;
    }
  }
  if ((tid & 31) == 0) {
    s_bf[tid >> 5] = bf;
    s_bi[tid >> 5] = bi;
  }
  if (tid < NOPS) s_cnt[tid] = 0;
  __syncthreads();
  if (tid == 0) {
    int b = -1;
    double v = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i)
      if (s_bi[i] >= 0 && (b < 0 || s_bf[i] < v || (s_bf[i] == v && s_bi[i] < b))) {
        v = s_bf[i];
        b = s_bi[i];
      }
    const double f0 = w.fit[0];
    if (b < 0 || f0 != f0) b = 0;          // the scan never leaves a NaN at slot 0
    const double f = w.fit[b];
    const int impr = f < st->best_F - 1e-13 ? 1 : 0;
    if (impr) {
      st->best_F = f;
      st->best_n = n;
    }
    if (f < st->level_best_F - 1e-13) {
      st->level_best_F = f;
      st->since_improve = 0;
    } else {
      st->since_improve += 1;
    }
    st->best_slot = b;
    st->improved = impr;
    st->best_nactive = w.nact[b];
    st->best_nnz = w.nnz[b];
    const double n2 = (double)n * (double)n;
    if (fw_ran) {
      st->fw_steps += (long long)q.fw_rounds * P;
      st->flop += (double)P * (double)q.fw_rounds * (4.0 * n2 * (double)q.fw_iters + 2.0 * n2 * 13.0);
    }
    st->evals += P;
    st->flop += 2.0 * n2 * (double)P;
    *w.var_gen = (unsigned long long)(gen + 1000 * st->level);
    s_best = b;
    s_impr = impr;
    s_bestF = st->best_F;
  }
  for (int p = tid; p < P; p += blockDim.x) {
    s_sig[p] = w.sig[p];
    w.parent_fit[p] = w.fit[p];
  }
  __syncthreads();
  if (s_impr) {
    const float* src = pop + (size_t)s_best * n;
    for (int i = tid; i < n; i += blockDim.x) w.best_row[i] = src[i];
  }

  // tabu table (main.cu:653-661): per signature, in slot order, a slot that
  // improves the signature's best by more than 1e-12 resets its revisits,
  // any other slot adds one.  The first slot of each signature walks its
  // group; distinct signatures own distinct entries.
  for (int p = tid; p < P; p += blockDim.x) {
    const unsigned long long key = s_sig[p];
    bool leader = true;
    for (int r = 0; r < p; ++r)
      if (s_sig[r] == key) {
        leader = false;
        break;
      }
    if (!leader) continue;
    bool fresh = false;
    const int e = tabu_slot(w, q.cap, key, true, &fresh);
    if (e < 0) {
      atomicCAS(&st->status, 0, (int)SIDON_ERR_CAPACITY);
      continue;
    }
    if (fresh) atomicAdd(&st->cells, 1);
    bool found = !fresh;
    double cb = found ? w.tbest[e] : 0.0;
    int hits = found ? w.thits[e] : 0;
    for (int r = p; r < P; ++r) {
      if (s_sig[r] != key) continue;
      const double f = w.fit[r];
      if (!found || f < cb - 1e-12) {
        cb = f;
        hits = 0;
        found = true;
      } else {
        hits += 1;
      }
    }
    w.tbest[e] = cb;
    w.thits[e] = hits;
  }

  // rank inside each island (main.cu:663-670)
  for (int p = tid; p < P; p += blockDim.x) {
    const int i = p / q.PI, b0 = i * q.PI;
    const double f = w.fit[p];
    int r = 0;
    for (int k = b0; k < b0 + q.PI; ++k)
      if (k != p && before(w.fit[k], k, f, p)) ++r;
    w.rank[b0 + r] = p;
  }
  __threadfence_block();
  __syncthreads();

  // migration every 12 generations: best of island i over the worst of
  // island i+1, in island order (main.cu:672-680)
  if (gen > 0 && gen % 12 == 0) {
    for (int i = 0; i < q.NI; ++i) {
      const int src = w.rank[i * q.PI], dst = w.rank[((i + 1) % q.NI) * q.PI + q.PI - 1];
      const float* a = pop + (size_t)src * n;
      float* b = pop + (size_t)dst * n;
      for (int k = tid; k < n; k += blockDim.x) b[k] = a[k];
      __syncthreads();
      if (tid == 0) {
        w.parent_fit[dst] = w.parent_fit[src];
        s_sig[dst] = s_sig[src];
        w.sig[dst] = s_sig[src];
      }
      __threadfence_block();
      __syncthreads();
    }
  }

  // offspring plan (main.cu:682-730)
  const double warm = fmin(1.0, (double)gen / 40.0);
  const double stagn = fmin(1.0, (double)st->since_improve / 25.0);
  double cum[NOPS];
  {
    double tot = 0.0;
    for (int o = 0; o < NOPS; ++o) tot += st->op_weight[o];
    double c = 0.0;
    for (int o = 0; o < NOPS; ++o) {
      c += st->op_weight[o] / tot;
      cum[o] = c;
    }
    cum[NOPS - 1] = 1.0;
  }
  const uint32_t k0 = (uint32_t)q.seed ^ 0x243F6A88u, k1 = (uint32_t)(q.seed >> 32) ^ 0x85A308D3u;
  const int level = st->level;
  for (int slot = tid; slot < P; slot += blockDim.x) {
    const int i = slot / q.PI, r = slot - i * q.PI;
    const int* isl = w.rank + i * q.PI;
    if (r < q.elite) {
      w.p1[slot] = isl[r];
      w.p2[slot] = isl[r];
      w.op[slot] = OP_CLONE;
      w.strength[slot] = 0.f;
      continue;
    }
    double u[8];
    for (int c = 0; c < 4; ++c) {
      const rng::U4 x =
          rng::philox({(uint32_t)slot, (uint32_t)gen, (uint32_t)level, (uint32_t)c}, k0, k1);
      u[2 * c] = rng::u53(x.x, x.y);
      u[2 * c + 1] = rng::u53(x.z, x.w);
    }
    int a = isl[pos_of(u[0], q.PI)], b = isl[pos_of(u[1], q.PI)];
    const int pa = w.parent_fit[a] < w.parent_fit[b] ? a : b;
    a = isl[pos_of(u[2], q.PI)];
    b = isl[pos_of(u[3], q.PI)];
    const int pb = w.parent_fit[a] < w.parent_fit[b] ? a : b;
    int o = 0;
    while (o < NOPS - 1 && cum[o] < u[4]) ++o;
    bool fresh = false;
    const int e = tabu_slot(w, q.cap, s_sig[pa], false, &fresh);
    const int hits = e >= 0 ? w.thits[e] : 0;
    const double cb = e >= 0 ? w.tbest[e] : 1e30;
    if (hits > q.tenure && cb > s_bestF * (1.0 + 2e-4)) {
      const int divers[7] = {5, 7, 9, 10, 8, 11, 12};
      o = divers[pos_of(u[5], 7)];
    }
    if (stagn > 0.7 && u[6] < 0.10) o = OP_RESTART;
    w.p1[slot] = pa;
    w.p2[slot] = pb;
    w.op[slot] = o;
    w.strength[slot] = (float)((0.03 + 0.35 * u[7]) * (0.5 + warm) * (1.0 + 1.5 * stagn));
    atomicAdd(&s_cnt[o], 1);
  }
  __syncthreads();
  if (tid < NOPS)
    for (int k = 0; k < s_cnt[tid]; ++k) st->op_use[tid] += 1.0;
}

// operator record and reinjection of the incumbent (main.cu:743-754)
__global__ void __launch_bounds__(BD) k_post(float* __restrict__ pop, W w, Q q) {
  for (int p = threadIdx.x; p < q.P; p += blockDim.x) w.cur_op[p] = w.op[p];
  const sidon_generation_state* st = w.st;
  if (st->gen % 10 == 9 && st->best_n == q.n) {
    const int slot = w.rank[q.PI - 1];
    float* dst = pop + (size_t)slot * q.n;
    for (int i = threadIdx.x; i < q.n; i += blockDim.x) dst[i] = w.best_row[i];
    __syncthreads();
    if (threadIdx.x == 0) w.cur_op[slot] = OP_CLONE;
  }
}

// bandit credit every 5 generations (main.cu:756-769), then the counter
__global__ void k_credit(W w, Q q) {
  if (threadIdx.x != 0) return;
  sidon_generation_state* st = w.st;
  const int gen = st->gen;
  if (gen > 0 && gen % 5 == 0) {
    for (int p = 0; p < q.P; ++p) {
      const int o = w.op[p];
      if (o >= 0 && o < NOPS && w.child_fit[p] < w.parent_fit[w.p1[p]]) st->op_win[o] += 1.0;
    }
    for (int o = 0; o < NOPS; ++o) {
      const double rate = st->op_use[o] > 20 ? st->op_win[o] / st->op_use[o] : 0.25;
      double x = 0.85 * st->op_weight[o] + 0.15 * (0.15 + 3.0 * rate);
      x = fmax(0.05, fmin(4.0, x));
      st->op_weight[o] = x;
    }
    for (int o = 0; o < NOPS; ++o) {
      st->op_use[o] *= 0.7;
      st->op_win[o] *= 0.7;
    }
  }
  st->gen = gen + 1;
}

}  // namespace gen
}  // namespace sidon

using namespace sidon_host;
namespace G = sidon::gen;

struct sidon_generation_s {
  sidon_generation_config cfg;
  int n_max = 0, P = 0, NI = 0, PI = 0, cap = 0;
  int n = 0;                   // cells of the current level (0: no level begun)
  G::W w{};
  sidon_generation_views v{};
  // the three tiers run side by side (disjoint candidates) on streams of
  // falling priority: cold, medium, warm
  cudaStream_t side[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t fork = nullptr, join[3] = {nullptr, nullptr, nullptr};
  ~sidon_generation_s() {
    for (int k = 0; k < 3; ++k) {
      if (side[k]) cudaStreamDestroy(side[k]);
      if (join[k]) cudaEventDestroy(join[k]);
    }
    if (fork) cudaEventDestroy(fork);
  }
};

namespace {

struct Layout {
  size_t off[26];
  size_t total;
};

// offsets of the workspace arrays, each 256-byte aligned
Layout layout_of(int n_max, int P, int cap) {
  const size_t Pn = (size_t)P * (size_t)n_max, Pz = (size_t)P, C1 = (size_t)cap + 1;
  const size_t sz[] = {
      Pn * 4, Pn * 4, Pn * 4,                   // nxt, mom, vel
      Pz * 8, Pz * 8, Pz * 8,                   // fit, parent_fit, child_fit
      Pz * 4, Pz * 4, Pz * 8, Pz * 4,           // nact, child_nact, sig, nnz
      Pz * 4, Pz * 4, Pz * 4, Pz * 4,           // p1, p2, op, strength
      Pz * 4, Pz * 4, Pz * 4, 3 * Pz * 4,       // cur_op, mode, rank, skip
      (size_t)n_max * 4,                        // best_row
      sizeof(sidon_generation_state), 8,        // state, var_gen
      C1 * 8, C1 * 8, C1 * 4, C1 * 4};          // tabu key, best, hits, used
  Layout L{};
  size_t o = 0;
  for (int i = 0; i < (int)(sizeof(sz) / sizeof(sz[0])); ++i) {
    L.off[i] = o;
    o += (sz[i] + 255) & ~(size_t)255;
  }
  L.total = o;
  return L;
}

int check_cfg(const sidon_generation_config& c, int n_max, int P) {
  if (n_max < 1) return SIDON_ERR_N;
  if (P < 1 || P > G::kMaxP) return SIDON_ERR_ARG;
  if (c.n_islands < 1 || P % c.n_islands || P / c.n_islands > 1024) return SIDON_ERR_ARG;
  if (c.elite < 0 || c.ls_iters < 0 || c.cold_iters < 0 || !(c.p_max > 0.f)) return SIDON_ERR_ARG;
  if (c.tabu_tenure < 0 || c.tabu_capacity < 2 || (c.tabu_capacity & (c.tabu_capacity - 1)))
    return SIDON_ERR_ARG;
  if (c.precision != SIDON_PREC_FP32_SIMT && c.precision != SIDON_PREC_BF16X1 &&
      c.precision != SIDON_PREC_BF16X3)
    return SIDON_ERR_DTYPE;
  if (c.fw_rounds < 0) return SIDON_ERR_ARG;
  if (c.fw_rounds > 0) {
    if (c.fw_iters < 0 || c.fw_nT < 1 || !(c.fw_t_max > 0.f) || !(c.fw_t_max <= 1.f))
      return SIDON_ERR_ARG;
    if (c.fw_precision != SIDON_PREC_FP32_SIMT && c.fw_precision != SIDON_PREC_BF16X1 &&
        c.fw_precision != SIDON_PREC_BF16X3)
      return SIDON_ERR_DTYPE;
  }
  return SIDON_OK;
}

G::Q params_of(const sidon_generation_s* h) {
  G::Q q{};
  q.n = h->n;
  q.P = h->P;
  q.NI = h->NI;
  q.PI = h->PI;
  q.elite = h->cfg.elite;
  q.tenure = h->cfg.tabu_tenure;
  q.cap = h->cap;
  q.cold_iters = h->cfg.cold_iters;
  q.med_iters = h->cfg.cold_iters / 3;
  q.warm_iters = h->cfg.ls_iters;
  q.fw_rounds = h->cfg.fw_rounds;
  q.fw_iters = h->cfg.fw_iters;
  q.seed = h->cfg.seed;
  return q;
}

// every kernel attribute the generation needs, set outside any capture
int prepare(const sidon_generation_s* h) {
  const int n = h->n;
  const sidon_generation_config& c = h->cfg;
  int rc = prepare_simt(n, c.precision == SIDON_PREC_FP32_SIMT);
  if (rc == SIDON_ERR_SMEM) rc = SIDON_OK;      // a step that does not fit reports it itself
  if (rc) return rc;
  if (c.precision != SIDON_PREC_FP32_SIMT) {
    rc = prepare_local_search_tc(n);
    if (rc) return rc;
  }
  if (c.fw_rounds > 0 && c.fw_precision != SIDON_PREC_FP32_SIMT) {
    rc = prepare_frank_wolfe_tc(n);
    if (rc == SIDON_ERR_N || rc == SIDON_ERR_SMEM) rc = SIDON_OK;
    if (rc) return rc;
  }
  return set_dyn_smem((const void*)G::k_select, (size_t)h->P * 8);
}

int enqueue(sidon_generation_s* h, float* pop, cudaStream_t st) {
  const G::Q q = params_of(h);
  const G::W& w = h->w;
  const sidon_generation_config& c = h->cfg;
  const int n = h->n, P = h->P;
  G::k_tiers<<<1, G::BD, 0, st>>>(w, q);
  int rc = check_launch();
  if (rc) return rc;
  // tier schedules (main.cu:627-629), in the reference's fp32 values
  const float pTop = c.p_max;
  const int iters[3] = {q.cold_iters, q.med_iters, q.warm_iters};
  const float pa[3] = {6.f, 40.f, 400.f}, pb[3] = {pTop, pTop, pTop * 3.f};
  const float la[3] = {0.085f, 0.040f, 0.012f}, lb[3] = {0.0015f, 0.0010f, 0.0003f};
  // Every step up to the evaluation acts on each candidate alone, and the
  // tiers are disjoint sets of candidates (rows of pop, mom, vel), so each
  // tier runs its local search and then its Frank-Wolfe step on its own
  // stream, forked from and joined back into the launching stream: the cold
  // tier's long chains on the highest-priority stream, so that its CTAs take
  // SMs first, the medium and warm tiers (and their Frank-Wolfe steps) on
  // streams of lower priority whose CTAs fill the SMs the cold chains leave
  // idle.  One CTA per candidate; a skipped candidate's CTA exits at once.
  // (The reference runs the tiers one after another and then the
  // Frank-Wolfe step on everybody, main.cu:627-639; the results are the
  // same.)
  cudaError_t e = cudaEventRecord(h->fork, st);
  for (int k = 0; k < 3 && e == cudaSuccess; ++k) e = cudaStreamWaitEvent(h->side[k], h->fork, 0);
  if (e != cudaSuccess) return set_cuda_error(e);
  int fw_ran = 0;
  for (int t = 0; t < 3; ++t) {
    const cudaStream_t ts = h->side[t];
    const int* skip = w.skip + (size_t)t * P;
    if (iters[t] > 0) {
      rc = c.precision == SIDON_PREC_FP32_SIMT
               ? launch_local_search(pop, w.mom, w.vel, nullptr, nullptr, P, n, n, skip, w.mode,
                                     iters[t], pa[t], pb[t], la[t], lb[t], 0.9f, 0.999f, 0,
                                     SIDON_F32, ts)
               : launch_local_search_tc_plain(pop, w.mom, w.vel, nullptr, nullptr, P, n, n, skip,
                                              w.mode, iters[t], pa[t], pb[t], la[t], lb[t], 0.9f,
                                              0.999f, 0, c.precision, ts);
      if (rc) return rc;
    }
    if (c.fw_rounds > 0 && (t == 0 || fw_ran)) {
      // the dead Adam moments of the tier's rows are the tensor-core step's
      // g / gbar rows
      rc = c.fw_precision == SIDON_PREC_FP32_SIMT
               ? sidon_frank_wolfe(pop, skip, n, P, c.fw_rounds, c.fw_iters, c.fw_nT,
                                   c.fw_t_max, 0.f, 0.f, ts)
               : sidon_frank_wolfe_tc(pop, w.mom, w.vel, skip, n, P, c.fw_rounds, c.fw_iters,
                                      c.fw_nT, c.fw_t_max, 0.f, 0.f, c.fw_precision, ts);
      if (rc == SIDON_OK) fw_ran = 1;
      else if (rc != SIDON_ERR_SMEM && rc != SIDON_ERR_N) return rc;   // main.cu:173: skipped
    }
  }
  for (int k = 0; k < 3 && e == cudaSuccess; ++k) {
    e = cudaEventRecord(h->join[k], h->side[k]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, h->join[k], 0);
  }
  if (e != cudaSuccess) return set_cuda_error(e);
  rc = sidon_eval(pop, SIDON_F32, n, P, w.fit, w.nact, 1e-4, st);
  if (rc) return rc;
  rc = sidon_support_sig(pop, SIDON_F32, n, P, 0.02f, w.sig, w.nnz, st);
  if (rc) return rc;
  G::k_select<<<1, G::BD, (size_t)P * 8, st>>>(pop, w, q, fw_ran);
  rc = check_launch();
  if (rc) return rc;
  rc = launch_variation(pop, w.nxt, SIDON_F32, n, P, w.p1, w.p2, w.op, w.strength, c.seed, 0, st,
                        w.var_gen);
  if (rc) return rc;
  e = cudaMemcpyAsync(pop, w.nxt, (size_t)P * n * sizeof(float), cudaMemcpyDeviceToDevice, st);
  if (e != cudaSuccess) return set_cuda_error(e);
  G::k_post<<<1, G::BD, 0, st>>>(pop, w, q);
  rc = check_launch();
  if (rc) return rc;
  rc = sidon_eval(pop, SIDON_F32, n, P, w.child_fit, w.child_nact, 1e-4, st);
  if (rc) return rc;
  G::k_credit<<<1, 32, 0, st>>>(w, q);
  return check_launch();
}

}  // namespace

extern "C" {

size_t sidon_generation_workspace_bytes(int n_max, int P, int tabu_capacity) {
  if (n_max < 1 || P < 1 || tabu_capacity < 2) return 0;
  return layout_of(n_max, P, tabu_capacity).total;
}

int sidon_generation_create(void* workspace, size_t bytes, int n_max, int P,
                            const sidon_generation_config* cfg, sidon_generation* out,
                            void* stream) {
  if (!out) return SIDON_ERR_ARG;
  *out = nullptr;
  if (!cfg || !workspace || ((uintptr_t)workspace & 255)) return SIDON_ERR_ARG;
  int rc = check_cfg(*cfg, n_max, P);
  if (rc) return rc;
  const Layout L = layout_of(n_max, P, cfg->tabu_capacity);
  if (bytes < L.total) return SIDON_ERR_ARG;
  rc = device_ok();
  if (rc) return rc;
  sidon_generation_s* h = new (std::nothrow) sidon_generation_s;
  if (!h) return SIDON_ERR_ARG;
  h->cfg = *cfg;
  h->n_max = n_max;
  h->P = P;
  h->NI = cfg->n_islands;
  h->PI = P / cfg->n_islands;
  h->cap = cfg->tabu_capacity;
  char* b = (char*)workspace;
  G::W& w = h->w;
  w.nxt = (float*)(b + L.off[0]);
  w.mom = (float*)(b + L.off[1]);
  w.vel = (float*)(b + L.off[2]);
  w.fit = (double*)(b + L.off[3]);
  w.parent_fit = (double*)(b + L.off[4]);
  w.child_fit = (double*)(b + L.off[5]);
  w.nact = (int*)(b + L.off[6]);
  w.child_nact = (int*)(b + L.off[7]);
  w.sig = (unsigned long long*)(b + L.off[8]);
  w.nnz = (int*)(b + L.off[9]);
  w.p1 = (int*)(b + L.off[10]);
  w.p2 = (int*)(b + L.off[11]);
  w.op = (int*)(b + L.off[12]);
  w.strength = (float*)(b + L.off[13]);
  w.cur_op = (int*)(b + L.off[14]);
  w.mode = (int*)(b + L.off[15]);
  w.rank = (int*)(b + L.off[16]);
  w.skip = (int*)(b + L.off[17]);
  w.best_row = (float*)(b + L.off[18]);
  w.st = (sidon_generation_state*)(b + L.off[19]);
  w.var_gen = (unsigned long long*)(b + L.off[20]);
  w.tkey = (unsigned long long*)(b + L.off[21]);
  w.tbest = (double*)(b + L.off[22]);
  w.thits = (int*)(b + L.off[23]);
  w.tused = (int*)(b + L.off[24]);
  sidon_generation_views& v = h->v;
  v.fit = w.fit;
  v.parent_fit = w.parent_fit;
  v.child_fit = w.child_fit;
  v.nactive = w.nact;
  v.sig = w.sig;
  v.nnz = w.nnz;
  v.p1 = w.p1;
  v.p2 = w.p2;
  v.op = w.op;
  v.strength = w.strength;
  v.cur_op = w.cur_op;
  v.mode = w.mode;
  v.rank = w.rank;
  v.tier_skip = w.skip;
  v.best_row = w.best_row;
  v.state = w.st;
  v.tabu_key = w.tkey;
  v.tabu_best = w.tbest;
  v.tabu_hits = w.thits;
  v.tabu_used = w.tused;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  int lo = 0, hi = 0;                      // least and greatest stream priority
  cudaError_t e = cudaDeviceGetStreamPriorityRange(&lo, &hi);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->fork, cudaEventDisableTiming);
  for (int k = 0; k < 3 && e == cudaSuccess; ++k) {
    const int prio = k == 0 ? hi : (k == 1 ? (hi + lo) / 2 : lo);
    e = cudaStreamCreateWithPriority(&h->side[k], cudaStreamNonBlocking, prio);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->join[k], cudaEventDisableTiming);
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(workspace, 0, L.total, st);
  if (e != cudaSuccess) {
    delete h;
    return set_cuda_error(e);
  }
  G::k_init<<<1, 32, 0, st>>>(w);
  rc = check_launch();
  if (rc) {
    delete h;
    return rc;
  }
  *out = h;
  return SIDON_OK;
}

int sidon_generation_destroy(sidon_generation h) {
  delete h;
  return SIDON_OK;
}

int sidon_generation_views_of(sidon_generation h, sidon_generation_views* out) {
  if (!h || !out) return SIDON_ERR_ARG;
  *out = h->v;
  return SIDON_OK;
}

int sidon_generation_begin_level(sidon_generation h, int n, int level, const int* seed_op,
                                 void* stream) {
  if (!h) return SIDON_ERR_ARG;
  if (n < 1 || n > h->n_max) return SIDON_ERR_N;
  if (level < 0) return SIDON_ERR_ARG;
  // the level's local search runs in one CTA per candidate
  if (h->cfg.precision == SIDON_PREC_FP32_SIMT) {
    if ((long long)sidon_smem_bytes(SIDON_OP_LOCAL_SEARCH, n, SIDON_F32) > smem_optin())
      return SIDON_ERR_SMEM;
  } else {
    const int rc = tc_n_ok_public(n);
    if (rc) return rc;
    if ((long long)smem_local_search_tc(n) > smem_optin()) return SIDON_ERR_SMEM;
  }
  h->n = n;
  G::Q q = params_of(h);
  G::k_begin<<<1, G::BD, 0, reinterpret_cast<cudaStream_t>(stream)>>>(h->w, q, level, seed_op);
  return check_launch();
}

int sidon_generation_set_best(sidon_generation h, const float* row, int n, double F,
                              void* stream) {
  if (!h || !row) return SIDON_ERR_ARG;
  if (n < 1 || n > h->n_max) return SIDON_ERR_N;
  G::k_set_best<<<1, G::BD, 0, reinterpret_cast<cudaStream_t>(stream)>>>(h->w, row, n, F);
  return check_launch();
}

int sidon_generation_step(sidon_generation h, float* pop, void* stream) {
  if (!h || !pop || h->n < 1) return SIDON_ERR_ARG;
  int rc = prepare(h);
  if (rc) return rc;
  return enqueue(h, pop, reinterpret_cast<cudaStream_t>(stream));
}

int sidon_generation_capture(sidon_generation h, float* pop, int generations,
                             sidon_graph* graph) {
  if (!graph) return SIDON_ERR_ARG;
  *graph = nullptr;
  if (!h || !pop || h->n < 1 || generations < 1) return SIDON_ERR_ARG;
  int rc = prepare(h);
  if (rc) return rc;
  sidon_graph_s* g = new (std::nothrow) sidon_graph_s;
  if (!g) return SIDON_ERR_ARG;
  cudaStream_t st = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete g;
    return set_cuda_error(e);
  }
  e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    for (int k = 0; k < generations && rc == SIDON_OK; ++k) rc = enqueue(h, pop, st);
    const cudaError_t e2 = cudaStreamEndCapture(st, &g->graph);
    if (rc == SIDON_OK && e2 != cudaSuccess) rc = set_cuda_error(e2);
  } else {
    rc = set_cuda_error(e);
  }
  if (rc == SIDON_OK) {
    // the kernel nodes keep the priorities of the streams they were
    // captured from
    e = cudaGraphInstantiate(&g->exec, g->graph, cudaGraphInstantiateFlagUseNodePriority);
    if (e != cudaSuccess) rc = set_cuda_error(e);
  }
  cudaStreamDestroy(st);
  if (rc != SIDON_OK) {
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return rc;
  }
  *graph = g;
  return SIDON_OK;
}

int sidon_generation_read_state(sidon_generation h, sidon_generation_state* out, void* stream) {
  if (!h || !out) return SIDON_ERR_ARG;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemcpyAsync(out, h->w.st, sizeof(sidon_generation_state),
                                  cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return e == cudaSuccess ? SIDON_OK : set_cuda_error(e);
}

}  // extern "C"
