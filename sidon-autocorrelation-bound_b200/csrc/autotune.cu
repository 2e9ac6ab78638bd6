// ---------------------------------------------------------------------------
//  autotune.cu -- per-(device, n, P, precision) choice of the local-search
//  schedule: the fused single-CTA kernel (one candidate per CTA; possible
//  while n fits one CTA) or the super-block jobs with super-block size q.
//  Few candidates of a mid-size n leave most SMs idle in the fused kernel;
//  smaller super-blocks make more, but narrower, tensor-core jobs -- which
//  wins depends on n and P, so it is measured: each choice runs a short
//  anneal on scratch heights (uniform 1/n) and the fastest is remembered
//  for the process.  The tuner allocates its scratch with cudaMalloc and
//  synchronises the device: call it before any stream capture, never inside
//  a hot loop.  Returns the chosen q (q >= n means the fused kernel).
// ---------------------------------------------------------------------------
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "common.cuh"

namespace sidon_host {
int tc_n_ok_public(int n);
size_t smem_local_search_tc(int n);
size_t big_workspace_bytes(int n, int P, int Q);
int launch_local_search_big(float* pop, float* mom, float* vel, const int* skip,
                            const int* mode_arr, int n, int P, int iters, double pS, double pE,
                            double lrS, double lrE, double b1, double b2, int mode_default,
                            int precision, int Q, void* ws, size_t ws_bytes, cudaStream_t st);

int launch_local_search_tc_sched(float* pop, float* mom, float* vel, const long long* offsets,
                                 const int* order, int P, int n_fixed, int n_max, const int* skip,
                                 const int* mode_arr, int iters, double pS, double pE,
                                 double lrS, double lrE, double b1, double b2, int mode_default,
                                 int precision, int ring, int balanced, unsigned int* seg_flags,
                                 cudaStream_t st);
int launch_local_search_simt_tile(void* pop, void* mom, void* vel, int P, int n, const int* skip,
                                  const int* mode_arr, int iters, double pS, double pE,
                                  double lrS, double lrE, double b1, double b2, int mode_default,
                                  int tk, cudaStream_t st);
int tc_ring_choices(int n, int* out, int cap);
int simt_tile_choices(int n, int* out, int cap);

namespace {
std::mutex g_mu;
std::map<std::tuple<int, int, int, int>, std::pair<int, float>> g_cache;
// the fused local search's schedule per (device, n, P, precision)
std::map<std::tuple<int, int, int, int>, sidon_ls_schedule> g_ls_cache;

__global__ void k_fill(float* a, long long total, float v) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x)
    a[t] = v;
}
}  // namespace

bool fused_fits(int n) {
  return tc_n_ok_public(n) == SIDON_OK && (long long)smem_local_search_tc(n) <= smem_optin();
}

// cached choice, or -1
int tuned_q(int n, int P, int precision) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -1;
  std::lock_guard<std::mutex> lock(g_mu);
  auto it = g_cache.find(std::make_tuple(dev, n, P, precision));
  return it == g_cache.end() ? -1 : it->second.first;
}

int autotune_local_search(int n, int P, int precision, int* out_q, float* out_ms) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_cuda_error(e);
  {
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_cache.find(std::make_tuple(dev, n, P, precision));
    if (it != g_cache.end()) {
      if (out_q) *out_q = it->second.first;
      if (out_ms) *out_ms = it->second.second;
      return SIDON_OK;
    }
  }
  std::vector<int> cands;
  if (fused_fits(n)) cands.push_back(n);
  for (int q : {8192, 4096, 2048, 1024})
    if (q < n && tc_n_ok_public(q) == SIDON_OK) cands.push_back(q);
  if (cands.empty()) return SIDON_ERR_N;
  size_t ws_bytes = 0;
  for (int q : cands)
    if (q < n) ws_bytes = std::max(ws_bytes, big_workspace_bytes(n, P, q));
  const size_t cells = (size_t)n * P;
  float *pop = nullptr, *mom = nullptr, *vel = nullptr;
  void* ws = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = SIDON_OK;
  if ((e = cudaMalloc(&pop, cells * 4)) != cudaSuccess || (e = cudaMalloc(&mom, cells * 4)) != cudaSuccess ||
      (e = cudaMalloc(&vel, cells * 4)) != cudaSuccess ||
      (ws_bytes && (e = cudaMalloc(&ws, ws_bytes)) != cudaSuccess) ||
      (e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreate(&e0)) != cudaSuccess || (e = cudaEventCreate(&e1)) != cudaSuccess)
    rc = set_cuda_error(e);
  int best_q = -1;
  float best_ms = 0.f;
  const int iters = 3;
  for (size_t c = 0; c < cands.size() && rc == SIDON_OK; ++c) {
    const int q = cands[c];
    float ms = 0.f;
    for (int rep = 0; rep < 2 && rc == SIDON_OK; ++rep) {       // rep 0 warms up
      k_fill<<<sm_count() * 4, 256, 0, st>>>(pop, (long long)cells, 1.f / (float)n);
      if ((e = cudaEventRecord(e0, st)) != cudaSuccess) { rc = set_cuda_error(e); break; }
      rc = launch_local_search_big(pop, mom, vel, nullptr, nullptr, n, P, iters, 2.0, 8.0, 1e-3,
                                   1e-3, 0.9, 0.999, 0, precision, q, ws, ws_bytes, st);
      if (rc) break;
      if ((e = cudaEventRecord(e1, st)) != cudaSuccess ||
          (e = cudaEventSynchronize(e1)) != cudaSuccess ||
          (e = cudaEventElapsedTime(&ms, e0, e1)) != cudaSuccess)
        rc = set_cuda_error(e);
    }
    if (rc == SIDON_OK && (best_q < 0 || ms < best_ms)) {
      best_q = q;
      best_ms = ms;
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st) cudaStreamDestroy(st);
  cudaFree(pop);
  cudaFree(mom);
  cudaFree(vel);
  if (ws) cudaFree(ws);
  if (rc) return rc;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    g_cache[std::make_tuple(dev, n, P, precision)] = {best_q, best_ms / iters};
  }
  if (out_q) *out_q = best_q;
  if (out_ms) *out_ms = best_ms / iters;
  return SIDON_OK;
}

}  // namespace sidon_host

// ------------------------- fused local-search schedule ----------------------
// For a uniform batch of P candidates of n cells the fused local search has
// three free choices that do not change a single result bit: the fp32 lane
// tile (odd TK from the narrowest that spans n with four warps up to 15), the
// tensor-core window ring (three single-tile stages, or two stages of 2-5
// tiles, as shared memory allows), and -- for more candidates than SMs --
// balanced step segments or waves of one CTA per candidate.  Which is
// fastest moves with n, P and the device (the fixed thresholds these replace:
// tile_for, ring_for, "segments whenever P > SMs"), so the tuner times each
// choice on a short anneal of scratch heights and remembers the fastest for
// the process.  It allocates and synchronises: call it before any capture.
namespace sidon_host {

static bool lookup_ls(int n, int P, int precision, sidon_ls_schedule* out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  std::lock_guard<std::mutex> lock(g_mu);
  auto it = g_ls_cache.find(std::make_tuple(dev, n, P, precision));
  if (it == g_ls_cache.end()) return false;
  *out = it->second;
  return true;
}

bool tuned_tc_schedule(int n, int P, int precision, int* ring, int* balanced) {
  sidon_ls_schedule s;
  if (!lookup_ls(n, P, precision, &s)) return false;
  *ring = s.ring_tiles;
  *balanced = s.balanced;
  return true;
}

bool tuned_simt_tile(int n, int P, int* tk) {
  sidon_ls_schedule s;
  if (!lookup_ls(n, P, SIDON_PREC_FP32_SIMT, &s)) return false;
  *tk = s.lane_tile;
  return true;
}

size_t smem_local_search_tc(int n);
int tc_ring_default(int n);
int simt_tile_default(int n);

// the schedule the next call at (n, P, precision) will use
int ls_schedule(int n, int P, int precision, sidon_ls_schedule* out) {
  if (lookup_ls(n, P, precision, out)) return SIDON_OK;
  sidon_ls_schedule s{};
  if (precision == SIDON_PREC_FP32_SIMT) {
    s.lane_tile = simt_tile_default(n);
  } else {
    s.ring_tiles = tc_ring_default(n);
    s.balanced = P > sm_count() ? 1 : 0;
  }
  s.ms_per_step = 0.f;
  s.tuned = 0;
  *out = s;
  return SIDON_OK;
}

int autotune_ls_schedule(int n, int P, int precision, sidon_ls_schedule* out) {
  if (lookup_ls(n, P, precision, out)) return SIDON_OK;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_cuda_error(e);
  const bool simt = precision == SIDON_PREC_FP32_SIMT;
  // candidate schedules
  std::vector<sidon_ls_schedule> cands;
  if (simt) {
    int tk[8];
    const int nt = simt_tile_choices(n, tk, 8);
    for (int i = 0; i < nt; ++i) cands.push_back(sidon_ls_schedule{tk[i], 0, 0, 0.f, 1});
  } else {
    int rings[20];
    const int nr = tc_ring_choices(n, rings, 20);
    for (int i = 0; i < nr; ++i) {
      cands.push_back(sidon_ls_schedule{0, rings[i], 0, 0.f, 1});
      if (P > sm_count()) cands.push_back(sidon_ls_schedule{0, rings[i], 1, 0.f, 1});
    }
  }
  if (cands.empty()) return SIDON_ERR_N;
  const size_t cells = (size_t)n * P;
  float *pop = nullptr, *mom = nullptr, *vel = nullptr;
  unsigned int* flags = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = SIDON_OK;
  if ((e = cudaMalloc(&pop, cells * 4)) != cudaSuccess ||
      (e = cudaMalloc(&mom, cells * 4)) != cudaSuccess ||
      (e = cudaMalloc(&vel, cells * 4)) != cudaSuccess ||
      (e = cudaMalloc(&flags, (size_t)P * 4)) != cudaSuccess ||
      (e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreate(&e0)) != cudaSuccess || (e = cudaEventCreate(&e1)) != cudaSuccess)
    rc = set_cuda_error(e);
  const int iters = 4;
  int best = -1;
  float best_ms = 0.f;
  for (size_t c = 0; c < cands.size() && rc == SIDON_OK; ++c) {
    const sidon_ls_schedule& s = cands[c];
    float ms = 0.f;
    for (int rep = 0; rep < 3 && rc == SIDON_OK; ++rep) {       // rep 0 warms up
      k_fill<<<sm_count() * 4, 256, 0, st>>>(pop, (long long)cells, 1.f / (float)n);
      if ((e = cudaEventRecord(e0, st)) != cudaSuccess) { rc = set_cuda_error(e); break; }
      rc = simt ? launch_local_search_simt_tile(pop, mom, vel, P, n, nullptr, nullptr, iters, 2.0,
                                                8.0, 1e-3, 1e-3, 0.9, 0.999, 0, s.lane_tile, st)
                : launch_local_search_tc_sched(pop, mom, vel, nullptr, nullptr, P, n, n, nullptr,
                                               nullptr, iters, 2.0, 8.0, 1e-3, 1e-3, 0.9, 0.999,
                                               0, precision, s.ring_tiles, s.balanced, flags, st);
      if (rc) break;
      float t = 0.f;
      if ((e = cudaEventRecord(e1, st)) != cudaSuccess ||
          (e = cudaEventSynchronize(e1)) != cudaSuccess ||
          (e = cudaEventElapsedTime(&t, e0, e1)) != cudaSuccess) {
        rc = set_cuda_error(e);
        break;
      }
      if (rep == 1 || (rep == 2 && t < ms)) ms = t;            // best of two timed runs
    }
    if (rc == SIDON_OK && (best < 0 || ms < best_ms)) {
      best = (int)c;
      best_ms = ms;
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st) cudaStreamDestroy(st);
  cudaFree(pop);
  cudaFree(mom);
  cudaFree(vel);
  cudaFree(flags);
  if (rc) return rc;
  sidon_ls_schedule s = cands[best];
  s.ms_per_step = best_ms / iters;
  s.tuned = 1;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    g_ls_cache[std::make_tuple(dev, n, P, precision)] = s;
  }
  *out = s;
  return SIDON_OK;
}

}  // namespace sidon_host
