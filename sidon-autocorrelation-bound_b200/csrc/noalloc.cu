// ---------------------------------------------------------------------------
//  noalloc.cu -- the local search with its Adam moments in a fixed,
//  library-owned device array, for callers that cannot allocate device
//  memory themselves.
//
//  Who needs it: a host program that hands this library only its population
//  buffer -- for example a plugin running inside an application whose
//  allocator owns and accounts for every device byte, or a caller that must
//  not issue cudaMalloc/cudaFree on its hot path because those calls can
//  synchronise the whole device and fragment a tightly budgeted heap.  Such a
//  caller cannot provide the [P][n] moment buffers sidon_local_search wants.
//
//  The moments live in g_moment_scratch below: a file-scope __device__ array
//  of 2 x kMaxCells floats (8 MiB) followed by kMaxFlags words (256 KiB) for
//  the hand-over flags of the balanced-segment kernel, which every GPU that
//  loads the library holds until the process exits.  Host code cannot use
//  the array's name as a device address, so on the first call on each device
//  (with that device current) the address is looked up with
//  cudaGetSymbolAddress and cached; that cache assumes the device's context
//  lives as long as the library (do not call this after cudaDeviceReset).
//  No call here allocates: no cudaMalloc, cudaFree or allocating library
//  routine is used.
// ---------------------------------------------------------------------------
#include <mutex>

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
}  // namespace sidon_host

namespace {

// P * n of one call may not exceed this (the first moment uses the first
// kMaxCells floats of the array, the second moment the next kMaxCells).
constexpr long long kMaxCells = 1ll << 20;
// Batches of more candidates than SMs run as balanced step segments with one
// hand-over flag per candidate in the array's last kMaxFlags words; larger
// batches (P > kMaxFlags, i.e. n <= 16) run the one-CTA-per-candidate kernel.
constexpr int kMaxFlags = 1 << 16;

static __device__ __align__(256) float g_moment_scratch[2 * kMaxCells + kMaxFlags];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
float* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_moment_scratch on the current device (looked up once).
int scratch_address(float** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return sidon_host::set_cuda_error(e);
  if (dev < 0 || dev >= kMaxDevices) return SIDON_ERR_DEVICE;
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_moment_scratch);
    if (e != cudaSuccess) return sidon_host::set_cuda_error(e);
    g_scratch_ptr[dev] = static_cast<float*>(p);
  }
  *out = g_scratch_ptr[dev];
  return SIDON_OK;
}

}  // namespace

extern "C" {

int sidon_local_search_noalloc(float* pop, const int* skip, const int* mode_arr, int n, int P,
                               int iters, double p_start, double p_end, double lr_start,
                               double lr_end, double beta1, double beta2, int mode_default,
                               int precision, void* stream) {
  if (P < 0) return SIDON_ERR_ARG;
  if (n < 1) return SIDON_ERR_N;
  int rc = sidon_host::device_ok();
  if (rc) return rc;
  if (P == 0 || iters <= 0) return SIDON_OK;
  if (!pop) return SIDON_ERR_ARG;
  if ((long long)n * (long long)P > kMaxCells) return SIDON_ERR_CAPACITY;
  if (!(p_start > 0.0) || !(p_end > 0.0) || !(lr_start > 0.0) || !(lr_end > 0.0))
    return SIDON_ERR_ARG;
  float* scratch = nullptr;
  rc = scratch_address(&scratch);
  if (rc) return rc;
  // the kernels zero the moments of every candidate they run at entry, and
  // the segment flags are zeroed on the stream before the launch, so what an
  // earlier call left in the array never leaks into this one (calls that
  // overlap on the GPU race on it all the same)
  float* mom = scratch;
  float* vel = scratch + kMaxCells;
  unsigned int* flags =
      P <= kMaxFlags ? reinterpret_cast<unsigned int*>(scratch + 2 * kMaxCells) : nullptr;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (precision == SIDON_PREC_FP32_SIMT)
    return sidon_host::launch_local_search(pop, mom, vel, nullptr, nullptr, P, n, n, skip,
                                           mode_arr, iters, p_start, p_end, lr_start, lr_end,
                                           beta1, beta2, mode_default, SIDON_F32, st);
  if (precision == SIDON_PREC_BF16X1 || precision == SIDON_PREC_BF16X3)
    return sidon_host::launch_local_search_tc(pop, mom, vel, nullptr, nullptr, P, n, n, skip,
                                              mode_arr, iters, p_start, p_end, lr_start, lr_end,
                                              beta1, beta2, mode_default, precision, flags,
                                              st);
  return SIDON_ERR_DTYPE;
}

}  // extern "C"
