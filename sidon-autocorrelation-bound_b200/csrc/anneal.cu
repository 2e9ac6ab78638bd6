// ---------------------------------------------------------------------------
//  anneal.cu -- the stream-ordered generation loop of the island search
//  (local search -> Frank-Wolfe -> fp64 evaluation -> migration), and its
//  capture as a CUDA graph.  Host code only: every step is one of the
//  library's own launches on one stream, with no allocation and no
//  synchronisation between them.  Replaces, for those steps, the generation
//  loop of src/main.cu:586-785 (which synchronises after every phase).
// ---------------------------------------------------------------------------
#include <algorithm>
#include <cmath>
#include <new>

#include "common.cuh"

namespace sidon_host {
int launch_local_search(void* pop, void* mom, void* vel, const long long* offsets,
                        const int* order, int P, int n_fixed, int n_max, const int* skip,
                        const int* mode_arr, int iters, double pS, double pE, double lrS,
                        double lrE, double b1, double b2, int mode_default, int dtype,
                        cudaStream_t st);
int launch_local_search_tc(float* pop, float* mom, float* vel, const long long* offsets,
                           const int* order, int P, int n_fixed, int n_max, const int* skip,
                           const int* mode_arr, int iters, double pS, double pE, double lrS,
                           double lrE, double b1, double b2, int mode_default, int precision,
                           unsigned int* seg_flags, cudaStream_t st);
int launch_eval(const void* pop, int dtype, const long long* offsets, const int* order, int P,
                int n_fixed, int n_max, double* outF, int* outN, double tol, cudaStream_t st);
int launch_frank_wolfe(float* pop, const long long* offsets, const int* order, int P, int n_fixed,
                       int n_max, const int* skip, int rounds, int pdhg, int nT, float tMax,
                       float tau, float sig, cudaStream_t st);
int launch_island_migrate(float* pop, int n, double* fit, int P, int NI, int k, int* order,
                          cudaStream_t st);
int launch_island_migrate_ragged(float* pop, const long long* offsets, double* fit, int P, int NI,
                                 int k, int* order, cudaStream_t st);
int launch_frank_wolfe_tc(float* pop, float* gbuf, float* gbbuf, const long long* offsets,
                          const int* order, int P, int n_fixed, int n_max, const int* skip,
                          int rounds, int pdhg, int nT, float tMax, float tau, float sig,
                          int precision, cudaStream_t st);
int prepare_local_search_tc(int n_max);
int prepare_frank_wolfe_tc(int n_max);
int prepare_simt(int n_max, bool local_search);
}  // namespace sidon_host

using namespace sidon_host;

namespace {

struct Args {
  float* pop;
  float* mom;
  float* vel;
  const long long* offsets;
  const int* order;
  int n_max;
  int P;
  double* fit;
  int* rank;
  sidon_anneal_config c;
};

int check_args(const Args& a) {
  const sidon_anneal_config& c = a.c;
  if (a.P < 0) return SIDON_ERR_ARG;
  if (a.n_max < 1) return SIDON_ERR_N;
  if (!a.pop || !a.mom || !a.vel || !a.fit) return SIDON_ERR_ARG;
  if (c.steps < 0 || !(c.p_start > 0.0) || !(c.p_end > 0.0) || !(c.lr_start > 0.0) ||
      !(c.lr_end > 0.0))
    return SIDON_ERR_ARG;
  if (c.precision != SIDON_PREC_FP32_SIMT && c.precision != SIDON_PREC_BF16X1 &&
      c.precision != SIDON_PREC_BF16X3)
    return SIDON_ERR_DTYPE;
  if (c.fw_every < 0 || c.migrate_every < 0) return SIDON_ERR_ARG;
  if (c.fw_every > 0 && (c.fw_rounds < 0 || c.pdhg_iters < 0 || c.fw_nT < 1 ||
                         !(c.fw_t_max > 0.f) || !(c.fw_t_max <= 1.f)))
    return SIDON_ERR_ARG;
  if (c.fw_every > 0 && c.fw_precision != SIDON_PREC_FP32_SIMT &&
      c.fw_precision != SIDON_PREC_BF16X1 && c.fw_precision != SIDON_PREC_BF16X3)
    return SIDON_ERR_DTYPE;
  if (c.migrate_every > 0) {
    if (!a.rank || c.n_islands < 1 || c.k_migrate < 0 || a.P % c.n_islands) return SIDON_ERR_ARG;
    const int PI = a.P / c.n_islands;
    if (PI > 1024 || 2 * c.k_migrate > PI) return SIDON_ERR_ARG;
  }
  return SIDON_OK;
}

// the anneal schedule value at global step s of `steps` (geometric)
double sched(double a, double b, int s, int steps) {
  if (steps <= 1) return a;
  return a * std::pow(b / a, (double)s / (double)(steps - 1));
}

int enqueue(const Args& a, cudaStream_t st) {
  const sidon_anneal_config& c = a.c;
  const bool tc = c.precision != SIDON_PREC_FP32_SIMT;
  const int n_fixed = a.offsets ? 0 : a.n_max;
  int rc = SIDON_OK;
  int s0 = 0;
  while (s0 < c.steps) {
    // next cut: the nearest multiple of fw_every / migrate_every after s0
    int s1 = c.steps;
    if (c.fw_every > 0) s1 = std::min(s1, (s0 / c.fw_every + 1) * c.fw_every);
    if (c.migrate_every > 0) s1 = std::min(s1, (s0 / c.migrate_every + 1) * c.migrate_every);
    const int L = s1 - s0;
    // p and lr of the segment's first and last step: inside the launch they
    // run geometrically between the two, i.e. along the global schedule
    const double pA = sched(c.p_start, c.p_end, s0, c.steps);
    const double pB = sched(c.p_start, c.p_end, s1 - 1, c.steps);
    const double lA = sched(c.lr_start, c.lr_end, s0, c.steps);
    const double lB = sched(c.lr_start, c.lr_end, s1 - 1, c.steps);
    if (tc)
      rc = launch_local_search_tc(a.pop, a.mom, a.vel, a.offsets, a.order, a.P, n_fixed, a.n_max,
                                  nullptr, nullptr, L, pA, pB, lA, lB, c.beta1, c.beta2, 0,
                                  c.precision, a.offsets ? nullptr : (unsigned int*)a.rank, st);
    else
      rc = launch_local_search(a.pop, a.mom, a.vel, a.offsets, a.order, a.P, n_fixed, a.n_max,
                               nullptr, nullptr, L, pA, pB, lA, lB, c.beta1, c.beta2, 0,
                               SIDON_F32, st);
    if (rc) return rc;
    if (c.fw_every > 0 && s1 % c.fw_every == 0 && c.fw_rounds > 0) {
      // the Adam moments are dead between local-search launches: they are
      // the tensor-core step's g / gbar rows
      rc = c.fw_precision == SIDON_PREC_FP32_SIMT
               ? launch_frank_wolfe(a.pop, a.offsets, a.order, a.P, n_fixed, a.n_max, nullptr,
                                   c.fw_rounds, c.pdhg_iters, c.fw_nT, c.fw_t_max, c.fw_tau,
                                   c.fw_sigma, st)
               : launch_frank_wolfe_tc(a.pop, a.mom, a.vel, a.offsets, a.order, a.P, n_fixed,
                                       a.n_max, nullptr, c.fw_rounds, c.pdhg_iters, c.fw_nT,
                                       c.fw_t_max, c.fw_tau, c.fw_sigma, c.fw_precision, st);
      if (rc) return rc;
    }
    if (c.migrate_every > 0 && s1 % c.migrate_every == 0 && s1 < c.steps) {
      rc = launch_eval(a.pop, SIDON_F32, a.offsets, a.order, a.P, n_fixed, a.n_max, a.fit, nullptr,
                       0.0, st);
      if (rc) return rc;
      rc = a.offsets ? launch_island_migrate_ragged(a.pop, a.offsets, a.fit, a.P, c.n_islands,
                                                    c.k_migrate, a.rank, st)
                     : launch_island_migrate(a.pop, a.n_max, a.fit, a.P, c.n_islands,
                                             c.k_migrate, a.rank, st);
      if (rc) return rc;
    }
    s0 = s1;
  }
  return launch_eval(a.pop, SIDON_F32, a.offsets, a.order, a.P, n_fixed, a.n_max, a.fit, nullptr,
                     0.0, st);
}

}  // namespace

extern "C" {

int sidon_anneal(float* pop, float* mom, float* vel, const long long* offsets, const int* order,
                 int n_max, int P, double* fit, int* rank, const sidon_anneal_config* cfg,
                 void* stream) {
  if (!cfg) return SIDON_ERR_ARG;
  const Args a{pop, mom, vel, offsets, order, n_max, P, fit, rank, *cfg};
  int rc = check_args(a);
  if (rc) return rc;
  rc = device_ok();
  if (rc) return rc;
  if (P == 0) return SIDON_OK;
  return enqueue(a, reinterpret_cast<cudaStream_t>(stream));
}

int sidon_anneal_capture(float* pop, float* mom, float* vel, const long long* offsets,
                         const int* order, int n_max, int P, double* fit, int* rank,
                         const sidon_anneal_config* cfg, sidon_graph* graph) {
  if (!cfg || !graph) return SIDON_ERR_ARG;
  *graph = nullptr;
  const Args a{pop, mom, vel, offsets, order, n_max, P, fit, rank, *cfg};
  int rc = check_args(a);
  if (rc) return rc;
  rc = device_ok();
  if (rc) return rc;
  // host-side set-up of every kernel the loop launches, outside the capture
  const bool tc = cfg->precision != SIDON_PREC_FP32_SIMT;
  rc = prepare_simt(n_max, !tc);
  if (!rc && tc) rc = prepare_local_search_tc(n_max);
  if (!rc && cfg->fw_every > 0 && cfg->fw_precision != SIDON_PREC_FP32_SIMT)
    rc = prepare_frank_wolfe_tc(n_max);
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
    rc = P > 0 ? enqueue(a, st) : SIDON_OK;
    const cudaError_t e2 = cudaStreamEndCapture(st, &g->graph);
    if (rc == SIDON_OK && e2 != cudaSuccess) rc = set_cuda_error(e2);
  } else {
    rc = set_cuda_error(e);
  }
  if (rc == SIDON_OK) {
    e = cudaGraphInstantiate(&g->exec, g->graph, 0);
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

int sidon_graph_launch(sidon_graph graph, void* stream) {
  if (!graph || !graph->exec) return SIDON_ERR_ARG;
  const cudaError_t e = cudaGraphLaunch(graph->exec, reinterpret_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? SIDON_OK : set_cuda_error(e);
}

int sidon_graph_destroy(sidon_graph graph) {
  if (!graph) return SIDON_OK;
  if (graph->exec) cudaGraphExecDestroy(graph->exec);
  if (graph->graph) cudaGraphDestroy(graph->graph);
  delete graph;
  return SIDON_OK;
}

}  // extern "C"
