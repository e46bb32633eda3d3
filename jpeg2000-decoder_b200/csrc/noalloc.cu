/*
 * noalloc.cu — inverse DWT of one tile-component that allocates no device memory.
 *
 * For callers that cannot call cudaMalloc: code running while a CUDA stream is being
 * captured into a graph, real-time or callback contexts where an allocation could block or
 * fail, and hosts that hand the library pre-allocated input and output buffers from their
 * own arena and forbid it any other device allocation.  Those callers pass the Tier-1
 * coefficients of one tile-component and an output buffer; the intermediate resolution
 * levels live in a file-scope static device array instead of pooled buffers.
 *
 * The array is J2K_NOALLOC_SCRATCH_BYTES (32 MiB) and every GPU that loads the library
 * holds it until the process exits.  In host code the array's name is only a host-side
 * stand-in, so its device address is fetched once per device with cudaGetSymbolAddress
 * (with that device current) on the first call there; make that first call before any
 * stream capture.  The address is cached for the life of the process: after cudaDeviceReset
 * (or anything else that tears down and re-creates a device's primary context) the cached
 * address is stale, so such a caller must restart the process before calling again.  Calls
 * share the array: calls that overlap on the GPU (different streams, or devices reusing one
 * process-wide lock-free entry) race and must be serialised by the caller.  Nothing needs
 * clearing between calls: every scratch element a level reads was written by the previous
 * level of the same call.
 *
 * Errors: the tile-component description is checked before anything is enqueued (a table
 * whose resolutions do not nest inside the tile-component returns J2K_ERR_ARG); a CUDA error
 * already pending on the calling thread from earlier work is reported as J2K_ERR_CUDA and
 * left pending for its owner; a failed launch of this call is cleared and reported as
 * J2K_ERR_CUDA.
 */
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/j2k_gpu.h"
#include "codestream.h"
#define J2K_DWT_LEVELS_ONLY  // this unit launches the level kernels only
#include "dwt_kernel.cuh"

namespace {

constexpr size_t kScratchBytes = J2K_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_idwt_scratch[kScratchBytes];

std::mutex g_mu;
void *g_scratch_addr[kMaxDevices] = {nullptr};

int scratch_for_current_device(void **addr) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return J2K_ERR_NODEVICE;
  }
  std::lock_guard<std::mutex> g(g_mu);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_idwt_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return J2K_ERR_CUDA;
    }
    g_scratch_addr[dev] = p;
  }
  *addr = g_scratch_addr[dev];
  return J2K_OK;
}

template <bool REV>
int run_levels(const j2k_tilecomp &tc, int flags, const void *coef, void *out, int out_stride, cudaStream_t st,
               void *scratch) {
  typedef typename j2k_dev::DwtTypes<REV>::T T;
  const int L = tc.levels;
  const int sw = L >= 2 ? tc.res_w[L - 1] : 1;
  const size_t half_elems = L >= 2 ? (size_t)tc.res_w[L - 1] * tc.res_h[L - 1] : 0;
  T *half[2] = {reinterpret_cast<T *>(scratch), reinterpret_cast<T *>(scratch) + half_elems};
  const float llg = j2k::irrev_ll_gain();
  const int refc = (flags & J2K_FLAG_REF_COMPAT) ? 1 : 0;
  for (int r = 1; r <= L; ++r) {
    const int rw = tc.res_w[r], rh = tc.res_h[r], lw = tc.res_w[r - 1], lh = tc.res_h[r - 1];
    if (rw <= 0 || rh <= 0) continue;
    const T *llsrc = r == 1 ? reinterpret_cast<const T *>(coef) : half[(r - 1) & 1];
    const int stride_ll = r == 1 ? tc.w : sw;
    T *dst = r == L ? reinterpret_cast<T *>(out) : half[r & 1];
    const int stride_out = r == L ? out_stride : sw;
    const int tiles = ((rw + j2k_dev::DWT_T - 1) / j2k_dev::DWT_T) * ((rh + j2k_dev::DWT_T - 1) / j2k_dev::DWT_T);
    j2k_dev::dwt_level_explicit_kernel<REV><<<tiles, j2k_dev::DWT_THREADS, 0, st>>>(reinterpret_cast<const T *>(coef), tc.w, llsrc,
                                                                   stride_ll, dst, stride_out, rw, rh, lw, lh,
                                                                   (!REV && r > 1) ? 1 : 0, llg, refc);
    if (cudaPeekAtLastError() != cudaSuccess) {  // nothing was pending on entry: this error is ours
      cudaGetLastError();
      return J2K_ERR_CUDA;
    }
  }
  return J2K_OK;
}

// Resolutions must nest: the full resolution is the tile-component, every coarser one lies
// inside the next finer one and is half of it (rounded either way, as the band origin
// decides).  Anything else would make the level kernels address outside the caller's buffers
// or the scratch array.
bool table_consistent(const j2k_tilecomp &tc) {
  const int L = tc.levels;
  if (tc.res_w[L] != tc.w || tc.res_h[L] != tc.h) return false;
  for (int r = 0; r < L; ++r) {
    const int w = tc.res_w[r], h = tc.res_h[r], fw = tc.res_w[r + 1], fh = tc.res_h[r + 1];
    if (w < 0 || h < 0 || w > fw || h > fh) return false;
    if (w < fw / 2 || w > (fw + 1) / 2 || h < fh / 2 || h > (fh + 1) / 2) return false;
  }
  return true;
}

}  // namespace

extern "C" int j2k_gpu_tile_idwt_noalloc(const j2k_tilecomp *tc, int reversible, int flags, const void *coef, void *out,
                                         int out_stride, void *stream) {
  if (!tc || !coef || !out || out_stride < tc->w || tc->w <= 0 || tc->h <= 0) return J2K_ERR_ARG;
  if (tc->levels < 0 || tc->levels > J2K_MAX_LEVELS) return J2K_ERR_ARG;
  if (!table_consistent(*tc)) return J2K_ERR_ARG;
  const int L = tc->levels;
  const size_t need = L >= 2 ? 2 * (size_t)tc->res_w[L - 1] * tc->res_h[L - 1] * 4 : 0;
  if (need > kScratchBytes) return J2K_ERR_UNSUPPORTED;  // beyond the static scratch size
  if (cudaPeekAtLastError() != cudaSuccess) return J2K_ERR_CUDA;  // earlier work's error: left for its owner
  cudaStream_t st = (cudaStream_t)stream;
  if (L == 0) {
    // no lifting: the coefficients are the samples
    return cudaMemcpy2DAsync(out, (size_t)out_stride * 4, coef, (size_t)tc->w * 4, (size_t)tc->w * 4, tc->h,
                             cudaMemcpyDeviceToDevice, st) == cudaSuccess
               ? J2K_OK
               : J2K_ERR_CUDA;
  }
  void *scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc != J2K_OK) return rc;
  return reversible ? run_levels<true>(*tc, flags, coef, out, out_stride, st, scratch)
                    : run_levels<false>(*tc, flags, coef, out, out_stride, st, scratch);
}
