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

namespace {
std::mutex g_mu;
std::map<std::tuple<int, int, int, int>, std::pair<int, float>> g_cache;

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
