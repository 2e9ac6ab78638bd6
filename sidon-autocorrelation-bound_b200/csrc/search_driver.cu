// ---------------------------------------------------------------------------
//  search_driver.cu -- the reference driver's search (src/main.cu:400-874)
//  behind one host call: resume adoption, the cell-split ladder with its
//  time split, the seeding of each level, the memetic generations (the
//  device-side generation loop, replayed from CUDA graphs between budget
//  checks), the carry-over to the next level, and the fp64 polish of the
//  incumbent.  Host code; it owns (allocates and frees) its device buffers,
//  as a top-level driver does.
// ---------------------------------------------------------------------------
#include <algorithm>
#include <chrono>
#include <cmath>
#include <random>
#include <vector>

#include "common.cuh"

using namespace sidon_host;

namespace {

using Clock = std::chrono::steady_clock;

double seconds_since(Clock::time_point t0) {
  return std::chrono::duration<double>(Clock::now() - t0).count();
}

// nearest-neighbour injection of a vector of m cells into n (main.cu:555-562)
void inject(const std::vector<double>& v, float* dst, int n) {
  const int m = (int)v.size();
  double S = 0.0;
  for (int i = 0; i < n; ++i) {
    const double x = v[std::min(m - 1, (int)((long long)i * m / n))];
    dst[i] = (float)x;
    S += x;
  }
  if (S > 0)
    for (int i = 0; i < n; ++i) dst[i] = (float)(dst[i] / S);
}

// ------------------------------ level seeding ------------------------------
// A fresh row is one of two random families.  Its description is drawn
// first, all at once, in the order the reference driver draws it (so level 0
// reproduces the reference's first rows); the row is then rendered from the
// description.
struct FreshRow {
  int nf = 0;                   // cosine terms (2..7)
  double freq[8] = {}, phase[8] = {};
  bool structured = false;      // the structured prior, else a smooth profile
  // structured prior: segments of the unit interval with a level and a
  // roughness amplitude each, an atom at one end
  bool flip = false;
  double atom = 0.0;
  double edge[5] = {};          // right edges of segments 0..4
  double level[6] = {4.2, 0.7, 5.2, 2.0, 0.0, 0.0};
  double rough_amp[6] = {0.45, 0.80, 0.30, 0.70, 0.0, 0.20};
  // smooth profile: base + amp * (mean of the cosines) + 0.3 N(0, 1)
  double base = 0.0, amp = 0.0;
};

// The random streams of one level: one generator, and one normal
// distribution for the whole level (it keeps the second value of each pair
// it draws for the next call, so it must not restart per row).
struct LevelDraws {
  std::mt19937_64 rng;
  std::uniform_real_distribution<double> U{0.0, 1.0};
  std::normal_distribution<double> N{0.0, 1.0};
  explicit LevelDraws(unsigned long long s) : rng(s) {}
  double uniform() { return U(rng); }
  double normal() { return N(rng); }
};

FreshRow draw_fresh(LevelDraws& g) {
  FreshRow r;
  r.nf = 2 + (int)(g.uniform() * 6);
  for (int f = 0; f < r.nf; ++f) {
    r.freq[f] = 1 + g.uniform() * 10;
    r.phase[f] = g.uniform() * 6.283185307;
  }
  r.structured = g.uniform() < 0.6;
  if (r.structured) {
    r.flip = g.uniform() < 0.5;
    r.atom = 30 + 250 * g.uniform();
    r.edge[0] = 0.28 + 0.16 * g.uniform();                  // plateau
    r.edge[1] = r.edge[0] + 0.10 + 0.14 * g.uniform();      // depression
    r.edge[2] = r.edge[1] + 0.02 + 0.08 * g.uniform();      // hump
    r.edge[3] = 0.70 + 0.16 * g.uniform();                  // ragged band
    r.edge[4] = r.edge[3] + 0.05 + 0.15 * g.uniform();      // hard gap
    r.level[5] = 3.0 + 14.0 * g.uniform();                  // terminal spike
  } else {
    r.base = 0.3 + 0.7 * g.uniform();
    r.amp = 0.2 + 1.2 * g.uniform();
  }
  return r;
}

// Render a fresh row into dst (n cells, clipped at zero).  The smooth
// family draws one normal per cell, in cell order.
void render_fresh(const FreshRow& r, float* dst, int n, LevelDraws& g) {
  for (int i = 0; i < n; ++i) {
    double v;
    if (r.structured) {
      const int d = r.flip ? (n - 1 - i) : i;         // distance from the atom's end
      const double x = (d + 0.5) / n;
      double rough = 0;
      for (int f = 0; f < r.nf; ++f)
        rough += std::cos(6.283185307 * (2 + 6 * r.freq[f]) * x + r.phase[f]);
      rough /= r.nf;
      int s = 0;                                       // first segment whose edge lies past x
      while (s < 5 && !(x < r.edge[s])) ++s;
      v = s == 4 ? 0.0 : r.level[s] * (1 + r.rough_amp[s] * rough);
      if (d == 0) v += r.atom;
      else if (d < 4) v += r.atom * 0.10 / d;
    } else {
      double m = 0;
      for (int f = 0; f < r.nf; ++f) m += std::cos(6.283185307 * r.freq[f] * i / n + r.phase[f]);
      v = r.base + r.amp * m / r.nf + 0.3 * g.normal();
    }
    dst[i] = (float)std::max(0.0, v);
  }
}

// The previous level's row carried to n cells: each cell duplicated when n
// doubles, else the nearest-neighbour resample.
void carry_over(const float* src, int n_prev, float* dst, int n) {
  if (n == 2 * n_prev) {
    for (int i = 0; i < n_prev; ++i) dst[2 * i] = dst[2 * i + 1] = src[i];
    return;
  }
  for (int i = 0; i < n; ++i) dst[i] = src[std::min(n_prev - 1, (int)((long long)i * n_prev / n))];
}

// sum 1 in fp64 (cell order); the uniform row when the sum is not positive
void normalise_row(float* dst, int n) {
  double S = 0;
  for (int i = 0; i < n; ++i) S += dst[i];
  for (int i = 0; i < n; ++i) dst[i] = S <= 0 ? 1.f / n : (float)(dst[i] / S);
}

// device buffers of a search, freed on every exit path
struct Buffers {
  void* ws = nullptr;
  float* pop = nullptr;
  int* seed_op = nullptr;
  float* row = nullptr;
  double *dp = nullptr, *dm = nullptr, *dv = nullptr, *df = nullptr, *dbest = nullptr,
         *dbestF = nullptr;
  int* dn = nullptr;
  sidon_generation gen = nullptr;
  sidon_graph graph = nullptr;
  ~Buffers() {
    if (graph) sidon_graph_destroy(graph);
    if (gen) sidon_generation_destroy(gen);
    void* ptrs[] = {ws, pop, seed_op, row, dp, dm, dv, df, dbest, dbestF, dn};
    for (void* p : ptrs)
      if (p) cudaFree(p);
  }
};

}  // namespace

extern "C" {

// Seeding of a ladder level (main.cu:483-553): row p refines the previous
// level's row p and keeps it (seed_op 20), except that the last 20 % of the
// rows start afresh; a row with no positive cell gets a fresh start (seed_op
// 9) from draw_fresh / render_fresh: with probability 0.6 the structured
// prior (endpoint atom, plateau, depression, hump, ragged band, hard gap,
// terminal spike), else a smooth random profile with gaussian noise.  Every
// row ends normalised to sum 1.  Draws: std::mt19937_64 seeded with
// seed + level, in the reference's order (level 0 draws exactly the
// reference's first numbers; later levels differ, because the reference's
// generator also serves its host-side selection draws, which run on the
// device here).
int sidon_seed_level(float* pop, int* seed_op, int n, int P, int level, const float* prev,
                     int n_prev, unsigned long long seed) {
  if (!pop || !seed_op || P < 1 || level < 0) return SIDON_ERR_ARG;
  if (n < 1) return SIDON_ERR_N;
  if (prev && n_prev < 1) return SIDON_ERR_ARG;
  LevelDraws draws(seed + (unsigned long long)level);
  const int keep = (level > 0 && prev) ? (int)(0.8 * P) : 0;   // carried-over rows
  for (int p = 0; p < P; ++p) {
    float* dst = pop + (size_t)p * n;
    std::fill(dst, dst + n, 0.f);
    if (p < keep) carry_over(prev + (size_t)p * n_prev, n_prev, dst, n);
    const bool live = std::any_of(dst, dst + n, [](float x) { return x > 0.f; });
    seed_op[p] = (p < keep && live) ? 20 : 9;
    if (!live) render_fresh(draw_fresh(draws), dst, n, draws);
    normalise_row(dst, n);
  }
  return SIDON_OK;
}

int sidon_search(const sidon_search_config* cfg, const double* resume, int n_resume,
                 double* best_out, int best_cap, int* best_n_out, double* best_F_out,
                 sidon_search_callback cb, void* user) {
  if (!cfg || !cfg->ladder || cfg->n_levels < 1 || cfg->P < 1 || !(cfg->seconds >= 0.0) ||
      cfg->gens_per_level < 0 || cfg->gens_per_graph < 1 || cfg->polish_iters < 0 ||
      cfg->polish_top < 0)
    return SIDON_ERR_ARG;
  if (resume && n_resume < 1) return SIDON_ERR_ARG;
  std::vector<int> ladder(cfg->ladder, cfg->ladder + cfg->n_levels);
  for (int n : ladder)
    if (n < 1) return SIDON_ERR_N;
  int rc = device_ok();
  if (rc) return rc;
  const auto t0 = Clock::now();
  const int P = cfg->P;
  const unsigned long long seed = cfg->gen.seed;

  // the incumbent; a resumed vector is adopted at once, and levels coarser
  // than it are dropped (main.cu:414-446)
  std::vector<double> best;
  double best_f = 1e30;
  if (resume) {
    best.assign(resume, resume + n_resume);
    best_f = sidon_hostF(best.data(), n_resume);
    size_t drop = 0;
    while (drop + 1 < ladder.size() && ladder[drop] < n_resume) ++drop;
    ladder.erase(ladder.begin(), ladder.begin() + drop);
  }
  // time split: later (finer) levels get more, 18 % kept for the polish
  // (main.cu:448-455)
  std::vector<double> budget(ladder.size());
  {
    double tot = 0;
    for (size_t l = 0; l < ladder.size(); ++l) tot += (budget[l] = std::pow(1.85, (double)l));
    for (double& x : budget) x = x / tot * cfg->seconds * 0.82;
  }
  const int n_max = *std::max_element(ladder.begin(), ladder.end());

  Buffers B;
  const size_t wsb = sidon_generation_workspace_bytes(n_max, P, cfg->gen.tabu_capacity);
  if (wsb == 0) return SIDON_ERR_ARG;
  cudaError_t e = cudaMalloc(&B.ws, wsb);
  if (e == cudaSuccess) e = cudaMalloc(&B.pop, (size_t)P * n_max * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&B.seed_op, (size_t)P * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&B.row, (size_t)std::max(n_max, n_resume) * sizeof(float));
  if (e != cudaSuccess) return set_cuda_error(e);
  rc = sidon_generation_create(B.ws, wsb, n_max, P, &cfg->gen, &B.gen, nullptr);
  if (rc) return rc;
  if (resume && n_resume <= n_max) {
    std::vector<float> r(best.begin(), best.end());
    e = cudaMemcpy(B.row, r.data(), r.size() * sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return set_cuda_error(e);
    rc = sidon_generation_set_best(B.gen, B.row, n_resume, best_f, nullptr);
    if (rc) return rc;
  }

  std::vector<float> hpop, prev;
  std::vector<int> hop(P);
  int n_prev = 0;
  for (size_t lvl = 0; lvl < ladder.size(); ++lvl) {
    const int n = ladder[lvl];
    const double t_end = seconds_since(t0) + budget[lvl];
    hpop.assign((size_t)P * n, 0.f);
    rc = sidon_seed_level(hpop.data(), hop.data(), n, P, (int)lvl, prev.empty() ? nullptr : prev.data(),
                          n_prev, seed);
    if (rc) return rc;
    // the incumbent into slot 0, the resumed vector into slot 1 (main.cu:563-564)
    if (!best.empty()) {
      inject(best, hpop.data(), n);
      hop[0] = 20;
    }
    if (resume && P > 1) {
      inject(std::vector<double>(resume, resume + n_resume), hpop.data() + n, n);
      hop[1] = 20;
    }
    e = cudaMemcpy(B.pop, hpop.data(), hpop.size() * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(B.seed_op, hop.data(), (size_t)P * sizeof(int), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return set_cuda_error(e);
    rc = sidon_generation_begin_level(B.gen, n, (int)lvl, B.seed_op, nullptr);
    if (rc) return rc;
    if (cfg->gens_per_level == 0 || cfg->gens_per_level >= cfg->gens_per_graph) {
      rc = sidon_generation_capture(B.gen, B.pop, cfg->gens_per_graph, &B.graph);
      if (rc) return rc;
    }
    int gen = 0;
    while (seconds_since(t0) < t_end && (cfg->gens_per_level == 0 || gen < cfg->gens_per_level)) {
      const int left = cfg->gens_per_level ? cfg->gens_per_level - gen : cfg->gens_per_graph;
      if (left >= cfg->gens_per_graph && B.graph) {
        rc = sidon_graph_launch(B.graph, nullptr);
      } else {
        for (int k = 0; k < left && rc == SIDON_OK; ++k) rc = sidon_generation_step(B.gen, B.pop, nullptr);
      }
      if (rc) return rc;
      sidon_generation_state s;
      rc = sidon_generation_read_state(B.gen, &s, nullptr);
      if (rc) return rc;
      if (s.status) return s.status;
      const int dev_rc = sidon_device_status(1);
      if (dev_rc) return dev_rc;
      gen = s.gen;
      int improved = 0;
      if (s.best_F < best_f && s.best_n > 0) {
        sidon_generation_views v;
        sidon_generation_views_of(B.gen, &v);
        std::vector<float> r(s.best_n);
        e = cudaMemcpy(r.data(), v.best_row, r.size() * sizeof(float), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return set_cuda_error(e);
        best.assign(r.begin(), r.end());
        best_f = s.best_F;
        improved = 1;
      }
      if (cb) {
        sidon_search_progress pr;
        pr.seconds = seconds_since(t0);
        pr.level = (int)lvl;
        pr.n = n;
        pr.gen = s.gen;
        pr.improved = improved;
        pr.best_F = best_f;
        pr.level_best_F = s.level_best_F;
        pr.evals = s.evals;
        pr.ls_steps = s.ls_steps;
        pr.fw_steps = s.fw_steps;
        pr.pflop = s.flop / 1e15;
        pr.cells = s.cells;
        pr.best_nactive = s.best_nactive;
        pr.best_nnz = s.best_nnz;
        pr.n_cold = s.n_cold;
        pr.n_med = s.n_med;
        cb(&pr, best.data(), (int)best.size(), user);
      }
    }
    if (B.graph) sidon_graph_destroy(B.graph);
    B.graph = nullptr;
    // carry the population to the next level (main.cu:786-790)
    prev.assign((size_t)P * n, 0.f);
    e = cudaMemcpy(prev.data(), B.pop, prev.size() * sizeof(float), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return set_cuda_error(e);
    n_prev = n;
  }

  // fp64 polish of the incumbent (main.cu:798-852): candidate 0 is the
  // incumbent, candidate k > 0 multiplies every height by
  // exp(0.003 (1 + k mod 8) z), z standard normal from mt19937_64(seed ^
  // 0xABCDEF); all clipped at 0 and normalised
  if (!best.empty() && cfg->polish_top > 0 && cfg->polish_iters > 0 &&
      (long long)sidon_smem_bytes(SIDON_OP_LOCAL_SEARCH, (int)best.size(), SIDON_F64) <=
          smem_optin()) {
    const int n = (int)best.size(), K = cfg->polish_top;
    std::vector<double> hp((size_t)n * K);
    std::mt19937_64 r2(seed ^ 0xABCDEF);
    std::normal_distribution<double> N01(0, 1);
    for (int k = 0; k < K; ++k) {
      double S = 0;
      for (int i = 0; i < n; ++i) {
        double x = best[i];
        if (k) x *= std::exp(0.003 * (1 + (k % 8)) * N01(r2));
        hp[(size_t)k * n + i] = std::max(0.0, x);
        S += std::max(0.0, x);
      }
      for (int i = 0; i < n; ++i) hp[(size_t)k * n + i] /= S;
    }
    const size_t Kn = (size_t)K * n * sizeof(double);
    e = cudaMalloc(&B.dp, Kn);
    if (e == cudaSuccess) e = cudaMalloc(&B.dm, Kn);
    if (e == cudaSuccess) e = cudaMalloc(&B.dv, Kn);
    if (e == cudaSuccess) e = cudaMalloc(&B.df, K * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&B.dn, K * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&B.dbest, n * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&B.dbestF, sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpy(B.dp, hp.data(), Kn, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(B.dbest, best.data(), n * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(B.dbestF, &best_f, sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return set_cuda_error(e);
    rc = sidon_polish(B.dp, B.dm, B.dv, n, K, cfg->polish_iters, 6, B.df, B.dn, B.dbest, B.dbestF,
                      nullptr);
    if (rc) return rc;
    double f = 0;
    e = cudaMemcpy(&f, B.dbestF, sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && f < best_f) {
      e = cudaMemcpy(best.data(), B.dbest, n * sizeof(double), cudaMemcpyDeviceToHost);
      best_f = f;
    }
    if (e != cudaSuccess) return set_cuda_error(e);
  }

  // report the larger of the search's F and the independent host recheck
  // (main.cu:865-873)
  if (!best.empty()) best_f = std::max(best_f, sidon_hostF(best.data(), (int)best.size()));
  if (best_n_out) *best_n_out = (int)best.size();
  if (best_F_out) *best_F_out = best_f;
  if (best_out)
    for (int i = 0; i < (int)best.size() && i < best_cap; ++i) best_out[i] = best[i];
  return SIDON_OK;
}

}  // extern "C"
