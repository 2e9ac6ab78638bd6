// Include shim over the reference CPU twin tools/probe.cpp (compiled from
// the reference tree; nothing copied).  main() is renamed so the file's
// static functions -- autoconv, objective, localSearch -- can be called.
// TEST INFRASTRUCTURE ONLY (checker and timed CPU baseline).
#define main probe_reference_main
#include "probe.cpp"
#undef main

extern "C" {

// tools/probe.cpp:62-116: fp64 L^p-annealed projected Adam on one vector
// (normalises first, returns F of the result).
double ref_probe_local_search(double* a, int n, int iters, double pA, double pB, double lrA,
                              double lrB, double b1, double b2, int mode) {
  LsCfg c;
  c.iters = iters; c.pA = pA; c.pB = pB; c.lrA = lrA; c.lrB = lrB; c.b1 = b1; c.b2 = b2;
  c.mode = mode;
  std::vector<double> v(a, a + n);
  const double f = localSearch(v, c);
  std::copy(v.begin(), v.end(), a);
  return f;
}

// The same over P candidates, OpenMP-parallel over candidates as in
// tools/probe.cpp:239 (schedule(dynamic)).
void ref_probe_local_search_batch(double* pop, int n, int P, int iters, double pA, double pB,
                                  double lrA, double lrB, double b1, double b2, int mode,
                                  double* outF) {
  LsCfg c;
  c.iters = iters; c.pA = pA; c.pB = pB; c.lrA = lrA; c.lrB = lrB; c.b1 = b1; c.b2 = b2;
  c.mode = mode;
#pragma omp parallel for schedule(dynamic)
  for (int p = 0; p < P; ++p) {
    std::vector<double> v(pop + (size_t)p * n, pop + (size_t)(p + 1) * n);
    const double f = localSearch(v, c);
    std::copy(v.begin(), v.end(), pop + (size_t)p * n);
    if (outF) outF[p] = f;
  }
}

// tools/probe.cpp:43-50 objective<long double>
long double ref_probe_objective_ld(const double* a, int n) {
  std::vector<long double> v(a, a + n), b;
  return objective(v, b);
}

int ref_probe_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
