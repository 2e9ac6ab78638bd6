// Include shim over the reference driver src/main.cu (which includes
// src/kernels.cuh), compiled from the reference tree for sm_100a; nothing
// copied.  main() is renamed; the file's static hostF / loadVec / saveVec and
// the reference kernels become callable.  TEST INFRASTRUCTURE ONLY: the
// oracle, and the reference kernels as a timed SIMT comparison point.
#define main sidon_reference_main
#include "main.cu"
#undef main

extern "C" {

// src/main.cu:95-105
double ref_hostF(const double* a, int n) { return hostF(std::vector<double>(a, a + n)); }

// src/main.cu:340-352; returns the length read (0 on failure), copies up to cap values
int ref_loadVec(const char* path, double* out, int cap) {
  std::vector<double> v;
  if (!loadVec(path, v)) return 0;
  for (int i = 0; i < (int)v.size() && i < cap; ++i) out[i] = v[i];
  return (int)v.size();
}

// src/main.cu:329-338
void ref_saveVec(const char* path, const double* a, int n, double f) {
  saveVec(path, std::vector<double>(a, a + n), f);
}

// src/kernels.cuh:177 kLocalSearch<float> on device buffers, launched as
// runLocalSearch does (src/main.cu:152-159), on `stream`.  Returns a cudaError_t.
int ref_gpu_local_search(float* pop, float* mom, float* vel, int n, int P, int iters, float pA,
                         float pB, float lrA, float lrB, void* stream) {
  const size_t sm = localSearchSmem<float>(n);
  cudaError_t e = cudaFuncSetAttribute((const void*)kLocalSearch<float>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return (int)e;
  kLocalSearch<float><<<P, BD, sm, (cudaStream_t)stream>>>(pop, mom, vel, nullptr, nullptr, n,
                                                            iters, pA, pB, lrA, lrB, 0.9f,
                                                            0.999f, 0);
  return (int)cudaGetLastError();
}

// src/kernels.cuh:301 kEval<float,double>, launched as runEval (src/main.cu:161-166).
int ref_gpu_eval(const float* pop, int n, int P, double* fit, int* nact, double tol, void* stream) {
  const size_t sm = evalSmem<double>(n);
  cudaError_t e = cudaFuncSetAttribute((const void*)kEval<float, double>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return (int)e;
  kEval<float, double><<<P, BD, sm, (cudaStream_t)stream>>>(pop, n, fit, nact, tol);
  return (int)cudaGetLastError();
}

// src/kernels.cuh:408 kFrankWolfe<float> on device rows, launched as
// runFrankWolfe does (src/main.cu:170-178).  Returns 1 when it ran, 0 when
// the candidate does not fit shared memory (the driver then skips the step),
// -cudaError on failure.
int ref_gpu_frank_wolfe(float* pop, int n, int P, int rounds, int pdhg, int nT, float tMax,
                        void* stream) {
  const size_t sm = fwSmem<float>(n);
  int optin = 0, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if ((int)sm > optin) return 0;
  cudaError_t e = cudaFuncSetAttribute((const void*)kFrankWolfe<float>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return -(int)e;
  kFrankWolfe<float><<<P, BD, sm, (cudaStream_t)stream>>>(pop, nullptr, n, rounds, pdhg, nT, tMax);
  e = cudaGetLastError();
  return e == cudaSuccess ? 1 : -(int)e;
}

// The numeric device steps of one generation of the reference driver
// (src/main.cu:606-651), launched through its own helpers on a Gpu view of
// the caller's buffers: the non-empty anneal tiers in order (skip masks
// copied host -> device as launchTier does), the Frank-Wolfe step, kEval,
// kSupportSig, and the synchronous copies of fit / nact / sig / nnz to the
// host.  tier[P] (host) holds 0 cold, 1 medium, 2 warm; mode (device) is
// modeArr.  Returns 1 when the Frank-Wolfe step ran, 0 when it did not fit,
// -cudaError on failure.
int ref_gpu_generation_search(float* pop, float* mom, float* vel, int* skip_dev, int* mode_dev,
                              const int* tier, int n, int P, int cold_iters, int lsIters,
                              float pTop, int fwRounds, int fwIters, double* fit_dev,
                              int* nact_dev, unsigned long long* sig_dev, int* nnz_dev,
                              double* fit_h, int* nact_h, unsigned long long* sig_h,
                              int* nnz_h) {
  Gpu g;
  g.n = n; g.P = P; g.pop = pop; g.mom = mom; g.vel = vel; g.fit = fit_dev; g.nact = nact_dev;
  g.modeArr = mode_dev; g.skip = skip_dev; g.sig = sig_dev; g.nnz = nnz_dev;
  int cnt[3] = {0, 0, 0};
  for (int p = 0; p < P; ++p) ++cnt[tier[p]];
  std::vector<int> sk(P);
  auto launchTier = [&](int t, int iters, float pa, float pb, float la, float lb) {
    for (int p = 0; p < P; ++p) sk[p] = tier[p] == t ? 0 : 1;
    cudaMemcpy(g.skip, sk.data(), P * sizeof(int), cudaMemcpyHostToDevice);
    runLocalSearch(g, iters, pa, pb, la, lb, g.modeArr, g.skip);
  };
  if (cnt[0]) launchTier(0, cold_iters, 6.f, pTop, 0.085f, 0.0015f);
  if (cnt[1]) launchTier(1, cold_iters / 3, 40.f, pTop, 0.040f, 0.0010f);
  if (cnt[2]) launchTier(2, lsIters, 400.f, pTop * 3.f, 0.012f, 0.0003f);
  int optin = 0, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const bool fwOk = fwRounds > 0 && runFrankWolfe(g, fwRounds, fwIters, 12, 0.30f, optin);
  runEval(g);
  runSig(g);
  cudaMemcpy(fit_h, g.fit, P * sizeof(double), cudaMemcpyDeviceToHost);
  cudaMemcpy(nact_h, g.nact, P * sizeof(int), cudaMemcpyDeviceToHost);
  cudaMemcpy(sig_h, g.sig, P * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
  cudaMemcpy(nnz_h, g.nnz, P * sizeof(int), cudaMemcpyDeviceToHost);
  const cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return -(int)e;
  return fwOk ? 1 : 0;
}

// The variation launch of the generation (src/main.cu:732-741): plan copied
// host -> device, kVariation<float> from pop into nxt.
int ref_gpu_generation_vary(const float* pop, float* nxt, int n, int P, int* p1_dev, int* p2_dev,
                            int* op_dev, float* str_dev, const int* p1, const int* p2,
                            const int* op, const float* str, unsigned long long seed,
                            unsigned long long gen) {
  cudaMemcpy(p1_dev, p1, P * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemcpy(p2_dev, p2, P * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemcpy(op_dev, op, P * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemcpy(str_dev, str, P * sizeof(float), cudaMemcpyHostToDevice);
  const size_t smv = sizeof(float) * ((size_t)2 * n + 64 + 128);
  setSmemLimit((const void*)kVariation<float>, smv);
  kVariation<float><<<P, BD, smv>>>(pop, nxt, n, P, p1_dev, p2_dev, op_dev, str_dev, seed, gen);
  return (int)cudaGetLastError();
}

}  // extern "C"
