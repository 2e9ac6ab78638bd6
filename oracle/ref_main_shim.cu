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

}  // extern "C"
