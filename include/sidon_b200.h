/* ---------------------------------------------------------------------------
 * sidon_b200.h -- C ABI of the B200 engine for the discretised
 * autoconvolution ratio
 *
 *     F(a) = 2 n max_k b_k / (sum_i a_i)^2 ,   b = a * a ,   a >= 0.
 *
 * Every entry point takes plain pointers, sizes and a CUDA stream passed as
 * void* (NULL = the legacy default stream), returns an int status (0 = ok,
 * see sidon_status) and never exits the process.  Device pointers are
 * caller-owned; nothing here allocates inside a hot call.  Populations are
 * [P][n] row-major and are updated in place, as in the reference.
 *
 * Each declaration names the reference interface it replaces (paths are
 * relative to the reference project root).
 * ------------------------------------------------------------------------- */
#ifndef SIDON_B200_H
#define SIDON_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define SIDON_API __attribute__((visibility("default")))
#else
#define SIDON_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ----------------------------- status codes ------------------------------ */
enum sidon_status {
  SIDON_OK = 0,
  SIDON_ERR_ARG = 1,          /* null pointer, P <= 0, bad parameter           */
  SIDON_ERR_N = 2,            /* n outside the supported range                 */
  SIDON_ERR_SMEM = 3,         /* working set exceeds the per-CTA smem opt-in   */
  SIDON_ERR_CUDA = 4,         /* CUDA runtime error (sidon_last_cuda_error)    */
  SIDON_ERR_DTYPE = 5,        /* dtype / precision not supported by this call  */
  SIDON_ERR_NONFINITE = 6,    /* input held NaN/Inf/negative heights           */
  SIDON_ERR_TIMEOUT = 7,      /* a bounded device-side wait ran out            */
  SIDON_ERR_DEVICE = 8,       /* current device is not an sm_100 part          */
  SIDON_ERR_CAPACITY = 9      /* P * n beyond the fixed scratch of the
                                 allocation-free local search                   */
};

enum sidon_dtype { SIDON_F32 = 0, SIDON_F64 = 1 };

/* arithmetic of the convolution/correlation inside the local search */
enum sidon_precision {
  SIDON_PREC_FP32_SIMT = 0,   /* fp32 FFMA chains on the CUDA cores            */
  SIDON_PREC_BF16X1 = 1,      /* tcgen05 block-Toeplitz, hi*hi                 */
  SIDON_PREC_BF16X3 = 2,      /* tcgen05 block-Toeplitz, hi*hi + hi*lo + lo*hi */
  SIDON_PREC_FP64_SIMT = 3,   /* fp64 DFMA chains (the polish instantiation)   */
  SIDON_PREC_TF32X3 = 4       /* tcgen05 kind::tf32, hi*hi + hi*lo + lo*hi;
                                 G_p forward / backward only                    */
};

/* operator ids for sidon_smem_bytes */
enum sidon_op {
  SIDON_OP_LOCAL_SEARCH = 0,  /* src/kernels.cuh:161-162 localSearchSmem<T>     */
  SIDON_OP_EVAL = 1,          /* src/kernels.cuh:379-380 evalSmem<Acc>          */
  SIDON_OP_FRANK_WOLFE = 2,   /* src/kernels.cuh:405-406 fwSmem<T>              */
  SIDON_OP_LOCAL_SEARCH_TC = 3
};

/* Human-readable name of a status code. */
SIDON_API const char* sidon_status_string(int status);
/* The cudaError_t value behind the last SIDON_ERR_CUDA on this thread. */
SIDON_API int sidon_last_cuda_error(void);
/* Device-side status word of the tensor-core kernels since the last reset:
 * SIDON_ERR_TIMEOUT if a bounded wait inside a kernel ran out,
 * SIDON_ERR_NONFINITE if a candidate's heights held NaN, Inf or a negative
 * value (computed anyway, as the reference would), else SIDON_OK; the first
 * event is kept.  Synchronous (copies one word from the current device);
 * reset != 0 clears it. */
SIDON_API int sidon_device_status(int reset);
/* ABI version of this library (bumped on any signature change). */
SIDON_API int sidon_abi_version(void);
/* Diagnostic: the clock-cycle limit after which every bounded device-side
 * wait of the tensor-core kernels gives up (default 2^31 cycles, about 1.1 s
 * at 1.965 GHz; cycles <= 0 restores it).  A wait that runs out records
 * SIDON_ERR_TIMEOUT in the status word (sidon_device_status), and the kernel
 * unwinds: it still waits (with the default limit) for the tensor-core
 * operations it already issued, releases its tensor memory and returns, so
 * the context stays usable.  A tiny limit makes the pipeline's own waits run
 * out; tests use it to exercise that path.  Synchronous; applies to later
 * launches on the current device.
 * No reference counterpart: the reference's kernels have no waits, and its
 * CUDA_OK macro exits the process on any error (src/kernels.cuh:20-28). */
SIDON_API int sidon_set_wait_limit(long long cycles);

/* Dynamic shared memory one CTA of `op` needs at size n and dtype, in bytes;
 * 0 if the combination is unsupported.
 * Replaces localSearchSmem / evalSmem / fwSmem (src/kernels.cuh:161-162,
 * 379-380, 405-406). */
SIDON_API size_t sidon_smem_bytes(int op, int n, int dtype);
/* Largest n the op accepts on the current device (smem opt-in bound). */
SIDON_API int sidon_max_n(int op, int dtype);

/* fp64 F on the host: direct O(n * nnz) convolution skipping a_i == 0,
 * M = max b, S = sum a (sequential), F = 2 n M / S^2.
 * Replaces hostF (src/main.cu:95-105); bit-identical to it. */
SIDON_API double sidon_hostF(const double* a, int n);

/* Certifying evaluation of a population: F per candidate in fp64 (b formed
 * as in hostF: each product rounded, then added in i order; S summed in i
 * order -- so F equals hostF bit for bit) and, if out_nactive != NULL, the
 * number of k with b_k >= M (1 - active_tol).  F = 1e30 when S <= 0.
 * Any n: beyond shared memory the heights are streamed through it.
 * pop: device [P][n] of dtype; out_F: device [P]; out_nactive: device [P].
 * Replaces kEval<T,double> + runEval (src/kernels.cuh:301-377,
 * src/main.cu:161-166). */
SIDON_API int sidon_eval(const void* pop, int dtype, int n, int P, double* out_F, int* out_nactive,
               double active_tol, void* stream);

/* Exact certification: every near-maximal b_k is recomputed EXACTLY (a
 * fixed-point accumulator; fp32 products are exact in fp64, fp64 products
 * are split with FMA) and rounded once; S is summed exactly and rounded
 * once; F = 2 n M / (S S) in fp64.  Because a cell split maps M -> 2M and
 * S -> 2S exactly, this F is bit-identical across sidon_refine.  Outputs
 * (device, [P]; any may be NULL except out_F): F, M, S, argmax k.
 * No single reference counterpart: it strengthens kEval
 * (src/kernels.cuh:301-377) for the ladder's split invariance
 * (src/kernels.cuh:535-536). */
SIDON_API int sidon_certify(const void* pop, int dtype, int n, int P, double* out_F, double* out_M,
                  double* out_S, int* out_kmax, void* stream);

/* Fused L^p-annealed projected Adam / mirror descent: `iters` steps with
 * `pop` resident in shared memory, p = p_start (p_end/p_start)^(it/(iters-1)),
 * lr likewise; mode 0 = projected Adam, 1 = exponentiated gradient;
 * skip[pid] != 0 leaves candidate pid untouched; mode_arr (may be NULL)
 * overrides mode_default per candidate.  mom/vel: device [P][n] scratch of
 * dtype, zeroed at entry as in the reference.  dtype SIDON_F32 with
 * precision FP32_SIMT / BF16X1 / BF16X3, or SIDON_F64 with FP64_SIMT.
 * One CTA per candidate, as in the reference: a batch of more candidates
 * than SMs runs in waves (sidon_local_search_ws balances them).  Uses no
 * library-global memory besides the status word, so calls on different
 * streams may overlap freely.
 * Replaces kLocalSearch<T> + runLocalSearch (src/kernels.cuh:177-289,
 * src/main.cu:152-159) and the fp64 polish launch (src/main.cu:837-839). */
SIDON_API int sidon_local_search(void* pop, void* mom, void* vel, const int* skip, const int* mode_arr,
                       int n, int P, int iters, double p_start, double p_end, double lr_start,
                       double lr_end, double beta1, double beta2, int mode_default, int dtype,
                       int precision, void* stream);

/* Workspace sidon_local_search_ws needs (bytes; 0 when the call needs none:
 * fp32 SIMT, fp64, or arguments out of range). */
SIDON_API size_t sidon_local_search_workspace_bytes(int n, int P, int dtype, int precision);
/* sidon_local_search with a caller workspace (device memory, 4-byte
 * aligned, >= sidon_local_search_workspace_bytes): a uniform BF16X1 / BF16X3
 * batch of more candidates than SMs then runs as balanced step segments
 * instead of waves -- the P chains of `iters` steps are laid end to end and
 * cut into one equal segment per SM, a candidate split between two CTAs
 * handing its heights and moments over through memory behind a flag word in
 * the workspace (zeroed on the stream before the launch).  Every candidate's
 * result equals sidon_local_search's bit for bit.  Calls that overlap on the
 * GPU need distinct workspaces.  The launch is cooperative (all CTAs
 * resident), and a stream capture records it as a cooperative kernel node.
 * Same counterpart as sidon_local_search. */
SIDON_API int sidon_local_search_ws(void* pop, void* mom, void* vel, const int* skip,
                                    const int* mode_arr, int n, int P, int iters, double p_start,
                                    double p_end, double lr_start, double lr_end, double beta1,
                                    double beta2, int mode_default, int dtype, int precision,
                                    void* workspace, size_t workspace_bytes, void* stream);

/* The fused local search of sidon_local_search for callers that cannot
 * allocate device memory -- e.g. a plugin inside an application whose
 * allocator owns every device byte, or a hot path that must never call
 * cudaMalloc/cudaFree because they can synchronise the device.  Such a caller
 * passes only its population (fp32, [P][n], in place, plus the optional skip
 * and mode_arr); the Adam moments, and the hand-over flags of a BF16 batch
 * of more candidates than SMs (run as sidon_local_search_ws runs it), live
 * in a fixed device array inside the library (8 MiB + 256 KiB), held by
 * every GPU that loads it until the process exits.
 * Limit: P * n <= 1048576 cells per call, else SIDON_ERR_CAPACITY.  precision:
 * FP32_SIMT, BF16X1 or BF16X3.  Nothing is allocated: the first call on a
 * device (with that device current) looks up the array's device address with
 * cudaGetSymbolAddress and caches it, so make that first call before any
 * stream capture, and do not use this entry point after a cudaDeviceReset
 * (the cached address belongs to the context that reset destroyed).  All
 * calls share the one array: the kernels zero a candidate's moments before
 * using them and the flags are zeroed on the stream before each launch, but
 * calls that overlap on the GPU (concurrent streams) race on both.  The
 * array is private to this entry point: no other call touches it.
 * No counterpart in the reference (its driver always allocates the moment
 * buffers, src/main.cu:118-137). */
SIDON_API int sidon_local_search_noalloc(float* pop, const int* skip, const int* mode_arr, int n,
                                         int P, int iters, double p_start, double p_end,
                                         double lr_start, double lr_end, double beta1,
                                         double beta2, int mode_default, int precision,
                                         void* stream);

/* Smoothed objective G_p(a) = 2n ||a*a||_p / (sum a)^2 for a batch (fp32
 * heights, any scale).  Writes value[P] (device) and saved[P*4] (device,
 * {M = max b, S = sum a, R = sum (b/M)^p, G_p}); b itself is not stored
 * unless b_out != NULL ([P][2n-1] device, for the stored-b comparison).
 * precision FP32_SIMT, or BF16X1 / BF16X3 / TF32X3 (b on the tensor cores;
 * TF32X3 up to the n its plan fits in shared memory, about 8700, else
 * SIDON_ERR_SMEM).
 * No reference counterpart as an entry point: it exposes the objective of
 * the anneal (src/kernels.cuh:168-172). */
SIDON_API int sidon_lp_forward(const float* a, int n, int P, double p, float* value, float* saved,
                     float* b_out, int precision, void* stream);

/* Gradient of G_p: grad_i = (4n R^(1/p)/S^2) (G_i/R - M/S) with
 * G_i = sum_j (b_{i+j}/M)^(p-1) a_j.  b is recomputed tile by tile from a
 * (b_in == NULL) or read from a stored [P][2n-1] array (b_in != NULL).
 * precision as for sidon_lp_forward (the correlation on the tensor cores
 * for BF16X1 / BF16X3 / TF32X3).
 * saved: the forward's [P*4].  grad: device [P][n] fp32.
 * Replaces the gradient that exists only inside kLocalSearch
 * (src/kernels.cuh:221-244) and its CPU twin (tools/probe.cpp:77-92). */
SIDON_API int sidon_lp_backward(const float* a, const float* saved, const float* b_in, int n, int P,
                      double p, float* grad, int precision, void* stream);

/* Frank-Wolfe / LP step solved by Chambolle-Pock: per round, M = max(a*a),
 * pdhg_iters of  lambda <- [lambda + sigma (a*gbar - M)]_+ ,
 * g <- [g + tau (1 - A^T lambda)]_+ , gbar = 2 g_new - g_old ; normalise g;
 * nT-point line search over t in (0, t_max]; move a.  tau <= 0 or
 * sigma <= 0 select the reference steps tau = 0.9/n, sigma = 0.9 n.
 * Replaces kFrankWolfe<float> + runFrankWolfe (src/kernels.cuh:408-532,
 * src/main.cu:170-178); returns SIDON_ERR_SMEM where the reference's
 * runFrankWolfe returned false. */
SIDON_API int sidon_frank_wolfe(float* pop, const int* skip, int n, int P, int rounds, int pdhg_iters,
                      int nT, float t_max, float tau, float sigma, void* stream);

/* sidon_frank_wolfe with the Chambolle-Pock convolutions and correlations
 * on the tensor cores (precision BF16X3 or BF16X1): the same rounds,
 * iterations, steps and line search; the round's M and every line-search
 * maximum are refined in fp64 over the near-maximal k, so a move is taken
 * only when it lowers the refined max_k b_k.  g_scratch / gbar_scratch:
 * device fp32 [P][n] work rows (the primal iterate and its extrapolation;
 * their contents on entry are ignored).  Not bit-identical to the fp32 step:
 * the products round differently.  Same counterpart as sidon_frank_wolfe. */
SIDON_API int sidon_frank_wolfe_tc(float* pop, float* g_scratch, float* gbar_scratch,
                                   const int* skip, int n, int P, int rounds, int pdhg_iters,
                                   int nT, float t_max, float tau, float sigma, int precision,
                                   void* stream);

/* Cell split n -> 2n: dst[p][2i] = dst[p][2i+1] = src[p][i].
 * Replaces kRefine<T> (src/kernels.cuh:538-547) and the host refine
 * (src/main.cu:491-495). */
SIDON_API int sidon_refine(const void* src, int n, int P, void* dst, int dtype, void* stream);

/* Pairwise average 2n -> n.  Replaces kCoarsen<T> (src/kernels.cuh:550-557). */
SIDON_API int sidon_coarsen(const void* src, int n2, int P, void* dst, int dtype, void* stream);

/* Nearest-neighbour resample of every row of src (fp32 [P][m]) to n cells:
 * dst[p][t] = src[p][min(m-1, floor(t m / n))]; with normalise != 0 each row
 * is then scaled to sum 1 (fp64 sum in t order, dst = fl(dst / S); rows
 * summing to 0 stay as they are).  dst (fp32 [P][n]) must not overlap src.
 * Replaces the arbitrary-ratio host resample of src/main.cu:496-497 and the
 * injection of main.cu:555-562. */
SIDON_API int sidon_resample(const float* src, int m, int P, float* dst, int n, int normalise,
                             void* stream);

/* Island selection + migration on the device: islands are n_islands
 * groups of P/n_islands consecutive slots (at most 1024 per island); each is
 * ranked by fit ascending (ties by slot index, NaN last) into order_out
 * (device [P], caller-owned, required); then the
 * j-th best of island i overwrites the j-th worst of island (i+1) mod NI for
 * j < k_migrate (rows of pop and entries of fit).  Requires
 * 2 k_migrate <= P/n_islands.  k_migrate = 0 ranks only.
 * Replaces the host ranking and D2D migration (src/main.cu:676-692). */
SIDON_API int sidon_island_migrate(float* pop, int n, double* fit, int P, int n_islands, int k_migrate,
                         int* order_out, void* stream);

/* Variation operators of the memetic loop: offspring j (one per row of
 * out, device [n_off][n] of dtype) is operator op[j] applied to parents
 * p1[j], p2[j] (rows of pop) with strength[j], then renormalised to sum 1:
 * 0 blend crossover, 1 two-point segment crossover, 2 log-normal
 * multiplicative noise, 3 smooth low-frequency perturbation, 4 additive
 * gaussian noise, 5 sparsify, 6 reflect / symmetrise, 7 shift, 8 block
 * splice from p2, 9 fresh smooth random restart, 10 spike injection,
 * 11 structured seed (endpoint atom, plateau, depression, hump, band, hard
 * gap, terminal spike), 12 gap surgery, 13 endpoint atom; any other id
 * clones p1.  Randomness: Philox4x32-10 keyed by seed, counters by
 * (gen, offspring, element) -- reproducible per element, not the
 * reference's curand streams.  out must not overlap pop.
 * Replaces kVariation<T> (src/kernels.cuh:558-801, launched at
 * src/main.cu:737-741). */
SIDON_API int sidon_variation(const void* pop, void* out, int dtype, int n, int n_off,
                              const int* p1, const int* p2, const int* op,
                              const float* strength, unsigned long long seed,
                              unsigned long long gen, void* stream);

/* Support signature per candidate: sig[p] = xor over the indices i with
 * a_i > tol * mean(a) of a mixed hash of i (equal supports, equal
 * signatures), nnz[p] = their count.  Replaces kSupportSig<T> + runSig
 * (src/kernels.cuh:803-849, src/main.cu:180-184; the reference's tol is
 * 0.02). */
SIDON_API int sidon_support_sig(const void* pop, int dtype, int n, int P, float tol,
                                unsigned long long* sig, int* nnz, void* stream);

/* fp64 polish of the elite: K candidates (device fp64 [K][n], usually small
 * perturbations of the best vector), `passes` passes of iters/passes fp64
 * Adam steps with p from 200*4^q to 30x that and lr from 0.01*0.45^q to
 * 0.02x that (pass q); after each pass the certifying evaluation (fit[K],
 * nactive[K] with active tolerance 1e-6, nactive may be NULL) and, if the
 * pass's best F is below *best_F (device double, set by the caller), that
 * candidate's heights are copied to best_a (device [n]) and *best_F updated.
 * mom/vel: fp64 [K][n] scratch.  Stream-ordered, no host round trip.
 * Replaces the polish of src/main.cu:798-874 (6 passes there). */
SIDON_API int sidon_polish(double* pop, double* mom, double* vel, int n, int K, int iters,
                           int passes, double* fit, int* nactive, double* best_a,
                           double* best_F, void* stream);

/* ---------------------------- large candidates -----------------------------
 * Candidates longer than one CTA's shared memory (the ladder's 16384,
 * 32768, 65536, ...): the heights are cut into super-blocks of q cells (a
 * multiple of 64 that the single-CTA tensor-core kernels accept; q <= 0
 * picks the autotuned size, else 8192 or the largest accepted size below
 * it; q >= n runs the fused single-CTA kernel when n fits) and every pair of
 * super-blocks is one tensor-core job; stream-ordered elementwise launches
 * combine the jobs' outputs in a fixed order.  Works for any n >= 1 (for
 * n <= q it is one job per product).  precision BF16X3 or BF16X1.  The
 * caller provides the workspace (sidon_large_workspace_bytes; no
 * allocation inside).  No reference counterpart: the reference refuses n
 * whose working set exceeds shared memory (src/main.cu:391-399). */
SIDON_API size_t sidon_large_workspace_bytes(int n, int P, int q, int precision);

/* The schedule autotuner: times a short anneal of P candidates of n cells
 * for the fused single-CTA kernel (when n fits one CTA) and for super-block
 * sizes 8192 / 4096 / 2048 / 1024, and remembers the fastest for
 * (device, n, P, precision); q <= 0 in the calls below then uses it (and
 * sidon_large_workspace_bytes sizes for it).  *out_q: the choice (q >= n =
 * the fused kernel); *out_ms_per_step: its time.  It allocates scratch with
 * cudaMalloc and synchronises: call it before any stream capture. */
SIDON_API int sidon_autotune_large(int n, int P, int precision, int* out_q,
                                   float* out_ms_per_step);

/* The fused local search's schedule for a uniform batch: choices that never
 * change a result bit, only the time.
 *   lane_tile    fp32 SIMT: outputs per lane (odd, 7..15; a narrower tile
 *                spreads small n over more warps);
 *   ring_tiles   tensor cores: tiles per stage of the window ring (1 = three
 *                single-tile stages, 2..5 = two stages of that many tiles);
 *   balanced     tensor cores, more candidates than SMs: balanced step
 *                segments (1, when the call has a workspace) or waves of one
 *                CTA per candidate (0);
 *   ms_per_step  the tuner's measurement (0 when not tuned);
 *   tuned        1 if the tuner chose it, 0 for the built-in default. */
typedef struct sidon_ls_schedule {
  int lane_tile;
  int ring_tiles;
  int balanced;
  float ms_per_step;
  int tuned;
} sidon_ls_schedule;

/* The schedule tuner of the fused local search: times a short anneal of P
 * uniform candidates of n cells under every schedule above (lane tiles for
 * FP32_SIMT; ring shapes and, for P > SMs, segments vs waves for BF16X1 /
 * BF16X3) and remembers the fastest for (device, n, P, precision); later
 * uniform calls (sidon_local_search, _ws, _noalloc, the anneal) then use it.
 * Results are unchanged bit for bit.  It allocates scratch with cudaMalloc
 * and synchronises: call it before any stream capture.
 * Replaces the reference's fixed tiling constants TK / TI
 * (src/kernels.cuh:30-33). */
SIDON_API int sidon_autotune_local_search(int n, int P, int precision, sidon_ls_schedule* out);
/* The schedule the next uniform call at (n, P, precision) will use: the
 * tuned one if the tuner ran for it in this process, else the default
 * (tuned = 0).  No reference counterpart. */
SIDON_API int sidon_local_search_schedule(int n, int P, int precision, sidon_ls_schedule* out);

/* sidon_local_search (fp32 [P][n], Adam moments in mom/vel) for any n. */
SIDON_API int sidon_local_search_large(float* pop, float* mom, float* vel, const int* skip,
                                       const int* mode_arr, int n, int P, int iters,
                                       double p_start, double p_end, double lr_start,
                                       double lr_end, double beta1, double beta2,
                                       int mode_default, int precision, int q, void* workspace,
                                       size_t workspace_bytes, void* stream);

/* sidon_frank_wolfe_tc for any n (moves accepted on fp64-refined maxima). */
SIDON_API int sidon_frank_wolfe_large(float* pop, const int* skip, int n, int P, int rounds,
                                      int pdhg_iters, int nT, float t_max, float tau,
                                      float sigma, int precision, int q, void* workspace,
                                      size_t workspace_bytes, void* stream);

/* sidon_certify for any n: a streamed fp64 pass finds the near-maximal k,
 * which are then summed exactly; more than 4096 near-maximal k gives
 * F = NaN.  workspace: sidon_certify_workspace_bytes(P) bytes.  (sidon_eval
 * itself streams automatically when n exceeds shared memory.) */
SIDON_API size_t sidon_certify_workspace_bytes(int P);
SIDON_API int sidon_certify_large(const void* pop, int dtype, int n, int P, double* out_F,
                                  double* out_M, double* out_S, int* out_kmax, void* workspace,
                                  void* stream);

/* ---------------------------- ragged batches ------------------------------
 * A ragged batch holds P candidates of different sizes back to back:
 * candidate p is pop[offsets[p] .. offsets[p+1]) (offsets: device int64
 * [P+1], non-decreasing; n_p = offsets[p+1] - offsets[p]).  n_max bounds
 * every n_p and sizes the launch; a candidate with n_p outside [1, n_max] is
 * left untouched.  order (device int [P], may be NULL = 0..P-1) is the order
 * in which the launch takes the candidates up; sidon_ragged_order writes the
 * longest-first order that balances the tail.  mom/vel (and every per-row
 * output) follow the layout of pop.  Each candidate's result is bit-identical
 * to the uniform entry point's at its own n.  No reference counterpart: the
 * reference runs one n per launch (src/main.cu:118-137). */

/* order_out[r] = candidate of rank r by size descending, ties by index. */
SIDON_API int sidon_ragged_order(const long long* offsets, int P, int* order_out, void* stream);

/* sidon_local_search over a ragged fp32 batch; precision FP32_SIMT, BF16X1
 * or BF16X3 (the tensor-core kernel runs persistently, one CTA per SM). */
SIDON_API int sidon_local_search_ragged(float* pop, float* mom, float* vel,
                                        const long long* offsets, const int* order, int n_max,
                                        const int* skip, const int* mode_arr, int P, int iters,
                                        double p_start, double p_end, double lr_start,
                                        double lr_end, double beta1, double beta2,
                                        int mode_default, int precision, void* stream);

/* sidon_eval over a ragged batch (fp32 or fp64 heights). */
SIDON_API int sidon_eval_ragged(const void* pop, int dtype, const long long* offsets,
                                const int* order, int n_max, int P, double* out_F,
                                int* out_nactive, double active_tol, void* stream);

/* sidon_frank_wolfe over a ragged fp32 batch. */
SIDON_API int sidon_frank_wolfe_ragged(float* pop, const long long* offsets, const int* order,
                                       int n_max, const int* skip, int P, int rounds,
                                       int pdhg_iters, int nT, float t_max, float tau,
                                       float sigma, void* stream);

/* sidon_frank_wolfe_tc over a ragged fp32 batch (g_scratch / gbar_scratch
 * in pop's layout); persistent, one CTA per SM. */
SIDON_API int sidon_frank_wolfe_tc_ragged(float* pop, float* g_scratch, float* gbar_scratch,
                                          const long long* offsets, const int* order, int n_max,
                                          const int* skip, int P, int rounds, int pdhg_iters,
                                          int nT, float t_max, float tau, float sigma,
                                          int precision, void* stream);

/* sidon_island_migrate over a ragged fp32 batch: a migrant of another size
 * is resampled by nearest neighbour, dst[t] = src[min(m-1, t m / n)], and
 * normalised to sum 1 in fp64 (the injection of src/main.cu:555-562); its
 * fit becomes NaN until the next evaluation.  Same-size migrants are copied
 * with their fit. */
SIDON_API int sidon_island_migrate_ragged(float* pop, const long long* offsets, double* fit,
                                          int P, int n_islands, int k_migrate, int* order_out,
                                          void* stream);

/* ------------------------------ anneal driver -----------------------------
 * The stream-ordered generation loop of the island search: `steps` Adam
 * steps with p and lr geometric over the whole anneal, cut into segments at
 * every multiple of fw_every and migrate_every; after a segment ending at a
 * multiple of fw_every a Frank-Wolfe step (fw_rounds rounds of pdhg_iters
 * Chambolle-Pock iterations), after one ending at a multiple of
 * migrate_every (before the last step) an fp64 evaluation into fit and a
 * top-k_migrate migration between the n_islands islands; at the end an fp64
 * evaluation into fit.  Adam moments restart with each segment, as they do
 * with each local-search launch of the reference driver.  Nothing is
 * allocated and nothing synchronises, so the whole loop can be captured in a
 * CUDA graph (sidon_anneal_capture).  Replaces the generation loop of
 * src/main.cu:586-785 for its local-search, Frank-Wolfe and migration
 * steps. */
typedef struct sidon_anneal_config {
  int steps;                 /* Adam steps in total */
  double p_start, p_end;     /* L^p exponent, geometric over the steps */
  double lr_start, lr_end;   /* step size, geometric over the steps */
  double beta1, beta2;
  int precision;             /* local-search precision (FP32_SIMT, BF16X1, BF16X3) */
  int fw_every;              /* Frank-Wolfe after every fw_every steps (0 = never) */
  int fw_rounds, pdhg_iters, fw_nT;
  float fw_t_max, fw_tau, fw_sigma;  /* tau, sigma <= 0: the reference steps */
  int fw_precision;          /* FP32_SIMT, or BF16X1 / BF16X3 (tensor cores, mom/vel as scratch) */
  int n_islands;             /* islands of P / n_islands consecutive candidates */
  int migrate_every;         /* migration after every migrate_every steps (0 = never) */
  int k_migrate;
} sidon_anneal_config;

/* pop: fp32, ragged (offsets != NULL) or uniform [P][n_max] (offsets ==
 * NULL); mom/vel: scratch of pop's layout; fit: device double [P] (fp64 F
 * at the end); rank: device int [P] (island ranking scratch, required when
 * migrating; may be NULL otherwise; its contents on return are unspecified:
 * between migrations it also holds the hand-over flags with which a uniform
 * tensor-core batch of more candidates than SMs runs as balanced step
 * segments, see sidon_local_search_ws); order: as for the ragged calls. */
SIDON_API int sidon_anneal(float* pop, float* mom, float* vel, const long long* offsets,
                           const int* order, int n_max, int P, double* fit, int* rank,
                           const sidon_anneal_config* cfg, void* stream);

/* Records sidon_anneal with these arguments as a CUDA graph (nothing runs)
 * and returns it in *graph; sidon_graph_launch replays it on a stream (the
 * buffers must stay valid), sidon_graph_destroy releases it. */
typedef struct sidon_graph_s* sidon_graph;
SIDON_API int sidon_anneal_capture(float* pop, float* mom, float* vel, const long long* offsets,
                                   const int* order, int n_max, int P, double* fit, int* rank,
                                   const sidon_anneal_config* cfg, sidon_graph* graph);
SIDON_API int sidon_graph_launch(sidon_graph graph, void* stream);
SIDON_API int sidon_graph_destroy(sidon_graph graph);

/* --------------------------- memetic generations ---------------------------
 * One generation of the reference driver's memetic island search
 * (src/main.cu:586-785), with its selection policy on the device so that a
 * generation -- and any number of them -- is a fixed sequence of launches on
 * one stream that a CUDA graph can hold:
 *   1. anneal tiers from the operator that produced each candidate: cold
 *      (ops 9/11, at most max(1, 0.18 P) of them, in slot order) for
 *      cold_iters steps, p 6 -> p_max, lr 0.085 -> 0.0015; medium (the
 *      other 9/11 and ops 5, 7, 8, 10, 12, 13) for cold_iters/3 steps,
 *      p 40 -> p_max, lr 0.04 -> 0.001; warm (the rest) for ls_iters steps,
 *      p 400 -> 3 p_max, lr 0.012 -> 0.0003 (main.cu:607-629); mirror
 *      descent on every fourth island (main.cu:569-572);
 *   2. a Frank-Wolfe step on every candidate (skipped where the step does
 *      not fit, main.cu:633-639); fp64 evaluation; support signatures;
 *   3. the incumbent (improvement by more than 1e-13), the level best and
 *      the generations since it improved; the tabu table over support
 *      signatures (best F per signature, revisits without an improvement
 *      of 1e-12); ranking inside each island (ties by slot); every 12th
 *      generation the best of island i over the worst of island i+1
 *      (main.cu:641-692);
 *   4. the offspring plan: `elite` clones per island, the rest from two
 *      binary tournaments inside the island and an operator drawn from the
 *      bandit weights, replaced by a diversifying operator when the
 *      parent's signature was revisited more than tabu_tenure times without
 *      being within 2e-4 of the incumbent, and by a restart (op 9) with
 *      probability 0.1 once stagnation passes 0.7; strength
 *      (0.03 + 0.35 u)(0.5 + warm)(1 + 1.5 stagnation) (main.cu:694-730);
 *   5. variation into the workspace, copied over the population; every 10th
 *      generation the incumbent over the worst slot of island 0
 *      (main.cu:737-754);
 *   6. every 5th generation the bandit credit: an operator wins when its
 *      child beats its first parent; weights 0.85 w + 0.15 (0.15 + 3 rate),
 *      clamped to [0.05, 4]; use and win counts decay by 0.7
 *      (main.cu:756-769).
 * The draws (tournaments, operator, tabu and restart choices, strength)
 * come from Philox4x32-10 streams keyed by the seed and counted by (slot,
 * generation, level), not from the reference's host mt19937_64; the
 * variation operators are those of sidon_variation.  Island ties rank by
 * slot (std::sort leaves them unspecified).
 *
 * The workspace is caller-owned device memory of
 * sidon_generation_workspace_bytes(n_max, P, tabu_capacity) bytes; the
 * handle is a small host object (created once, never inside a hot call)
 * holding its layout and the configuration. */
typedef struct sidon_generation_config {
  int n_islands;             /* islands of P / n_islands consecutive slots (<= 1024 each) */
  int elite;                 /* clones kept per island (reference: 2) */
  int ls_iters;              /* warm tier steps (reference: 4000) */
  int cold_iters;            /* cold tier steps; the medium tier runs cold_iters / 3 (20000) */
  float p_max;               /* top of the exponent anneal (20000) */
  int precision;             /* local search: FP32_SIMT, BF16X1 or BF16X3 */
  int fw_rounds;             /* Frank-Wolfe rounds per generation, 0 = off (6) */
  int fw_iters;              /* Chambolle-Pock iterations per round (500) */
  int fw_nT;                 /* line-search points (12) */
  float fw_t_max;            /* line-search range (0.30) */
  int fw_precision;          /* FP32_SIMT (the reference step), BF16X1 or BF16X3 */
  int tabu_tenure;           /* revisits before a support cell is escaped (6) */
  int tabu_capacity;         /* signature table entries, a power of two */
  unsigned long long seed;   /* Philox key of the plan draws and of the variation */
} sidon_generation_config;

/* The search state on the device, readable with sidon_generation_read_state. */
typedef struct sidon_generation_state {
  double best_F;             /* incumbent F (1e30: none) */
  double level_best_F;       /* best F seen at this level */
  double op_weight[14], op_use[14], op_win[14];   /* bandit over the 14 operators */
  double flop;               /* algorithmic flop of the search so far (main.cu:625, 637, 642) */
  long long ls_steps;        /* candidate-steps of local search */
  long long evals;           /* fp64 evaluations */
  long long fw_steps;        /* candidate Frank-Wolfe rounds */
  int gen;                   /* generations done at this level */
  int level;
  int n;                     /* cells of this level */
  int since_improve;         /* generations since level_best_F improved */
  int best_n;                /* cells of the incumbent (0: none) */
  int best_slot;             /* slot of the last generation's best candidate */
  int improved;              /* the last generation improved the incumbent */
  int best_nactive, best_nnz;/* near-maximal k and support size of that candidate */
  int n_cold, n_med;         /* tier sizes of the last generation */
  int cells;                 /* distinct support signatures seen */
  int status;                /* SIDON_OK, or SIDON_ERR_CAPACITY once the tabu table filled */
  int pad_;
} sidon_generation_state;

/* Device arrays inside the workspace, for callers that read them. */
typedef struct sidon_generation_views {
  double* fit;               /* [P] fp64 F after the Frank-Wolfe step */
  double* parent_fit;        /* [P] fit after the migration (the plan's parent fitness) */
  double* child_fit;         /* [P] fp64 F of the offspring */
  int* nactive;              /* [P] */
  unsigned long long* sig;   /* [P] support signatures */
  int* nnz;                  /* [P] */
  int* p1;                   /* [P] plan: first parent */
  int* p2;                   /* [P] plan: second parent */
  int* op;                   /* [P] plan: operator (20 = elite clone) */
  float* strength;           /* [P] plan: strength */
  int* cur_op;               /* [P] operator that produced the current slot */
  int* mode;                 /* [P] descent mode per slot */
  int* rank;                 /* [P] slots of island i in rank order at [i*PI, (i+1)*PI) */
  int* tier_skip;            /* [3][P] skip masks of the cold, medium and warm tiers */
  float* best_row;           /* [n_max] incumbent heights */
  sidon_generation_state* state;
  unsigned long long* tabu_key;   /* [tabu_capacity + 1]; the last entry holds key 0 */
  double* tabu_best;              /* [tabu_capacity + 1] */
  int* tabu_hits;                 /* [tabu_capacity + 1] */
  int* tabu_used;                 /* [tabu_capacity + 1] */
} sidon_generation_views;

typedef struct sidon_generation_s* sidon_generation;

SIDON_API size_t sidon_generation_workspace_bytes(int n_max, int P, int tabu_capacity);
/* Lays the handle over the workspace and initialises the state on the
 * stream (bandit weights 1, 2.5 / 1.8 / 1.8 for operators 11-13 as at
 * main.cu:466-467; empty tabu table; no incumbent). */
SIDON_API int sidon_generation_create(void* workspace, size_t bytes, int n_max, int P,
                                      const sidon_generation_config* cfg,
                                      sidon_generation* out, void* stream);
SIDON_API int sidon_generation_destroy(sidon_generation h);
SIDON_API int sidon_generation_views_of(sidon_generation h, sidon_generation_views* out);
/* Starts a ladder level of n cells: generation 0, no level best, seed_op
 * (device [P], or NULL for all 9) as the operator of each slot, mirror
 * descent on islands 3, 7, 11, ... (main.cu:566-585).  n must fit the
 * one-CTA local search of the configured precision (SIDON_ERR_N /
 * SIDON_ERR_SMEM otherwise: up to 9728 cells on the tensor cores; the
 * reference driver refuses n > 16384, main.cu:391-399). */
SIDON_API int sidon_generation_begin_level(sidon_generation h, int n, int level,
                                           const int* seed_op, void* stream);
/* Adopts row (device fp32 [n]) with F as the incumbent (the resumed vector
 * of main.cu:414-425). */
SIDON_API int sidon_generation_set_best(sidon_generation h, const float* row, int n, double F,
                                        void* stream);
/* Enqueues one generation on pop (device fp32 [P][n], updated in place). */
SIDON_API int sidon_generation_step(sidon_generation h, float* pop, void* stream);
/* Records `generations` generations on pop as a CUDA graph (nothing runs). */
SIDON_API int sidon_generation_capture(sidon_generation h, float* pop, int generations,
                                       sidon_graph* graph);
/* Copies the state to *out after the stream's work so far (synchronises
 * the stream; not for use inside a capture). */
SIDON_API int sidon_generation_read_state(sidon_generation h, sidon_generation_state* out,
                                          void* stream);

/* ------------------------------ search driver ------------------------------
 * Host seeding of a ladder level (src/main.cu:483-553), on host buffers:
 * pop [P][n] fp32 and seed_op [P] (the operator record that picks each
 * slot's first anneal tier: 20 carried over, 9 fresh).  Row p refines row p
 * of prev ([P][n_prev], NULL at the first level; duplicate when n = 2 n_prev,
 * else nearest-neighbour resample), the last 20 % of the rows start afresh;
 * an empty row gets the structured prior with probability 0.6, else a smooth
 * random profile; rows are normalised to sum 1.  Draws: std::mt19937_64
 * seeded with seed + level in the reference's call order. */
SIDON_API int sidon_seed_level(float* pop, int* seed_op, int n, int P, int level,
                               const float* prev, int n_prev, unsigned long long seed);

typedef struct sidon_search_progress {
  double seconds;            /* wall clock since sidon_search began */
  int level, n, gen;         /* ladder level, its cells, generations done at it */
  int improved;              /* the incumbent improved since the previous report */
  double best_F;             /* incumbent F */
  double level_best_F;
  long long evals, ls_steps, fw_steps;
  double pflop;              /* algorithmic PFLOP so far */
  int cells;                 /* distinct support signatures seen */
  int best_nactive, best_nnz;
  int n_cold, n_med;
} sidon_search_progress;

/* Called after every replay of gens_per_graph generations with the progress
 * and the incumbent's heights (host fp64, best_n cells). */
typedef void (*sidon_search_callback)(const sidon_search_progress* progress, const double* best,
                                      int best_n, void* user);

typedef struct sidon_search_config {
  const int* ladder;         /* host [n_levels]: cells per level (reference: 64 ... 2048) */
  int n_levels;
  int P;                     /* population (256) */
  double seconds;            /* wall-clock budget; 82 % split over the levels by 1.85^l */
  int gens_per_level;        /* 0: each level runs until its time share is spent */
  int gens_per_graph;        /* generations per CUDA-graph replay between budget checks */
  int polish_iters;          /* fp64 polish steps over 6 passes (40000) */
  int polish_top;            /* polish candidates (8) */
  sidon_generation_config gen;
} sidon_search_config;

/* The reference driver's whole search (src/main.cu:400-874): resume
 * adoption (the resumed vector is the incumbent at once, coarser levels are
 * dropped), the ladder levels with their time shares, per level the host
 * seeding, the incumbent injected into slot 0 and the resumed vector into
 * slot 1, sidon_generation_* generations replayed from a CUDA graph until
 * the level's share is spent, the population carried to the next level;
 * then the fp64 polish of the incumbent (sidon_polish, 6 passes, K =
 * polish_top basin-hopping starts from mt19937_64(seed ^ 0xABCDEF)).
 * Writes the incumbent (up to best_cap cells of best, host fp64), its cell
 * count and F = max(search F, hostF recheck) (main.cu:865-873).  Allocates
 * and frees its own device buffers; returns a status. */
SIDON_API int sidon_search(const sidon_search_config* cfg, const double* resume, int n_resume,
                           double* best, int best_cap, int* best_n, double* best_F,
                           sidon_search_callback cb, void* user);

#ifdef __cplusplus
}
#endif
#endif /* SIDON_B200_H */
