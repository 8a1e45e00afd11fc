// pac_noalloc.cu -- a convolution entry point that allocates no device memory.
//
// Some callers cannot call cudaMalloc: code that runs inside another
// framework's memory pool or under a strict device-memory budget, code that
// must not synchronise the device (cudaMalloc/cudaFree can), and launches
// that are recorded for later replay, where an allocation inside the call
// would not be repeated.  pac_convolve_1d_noalloc serves them: the caller
// passes the signal, filter and output buffers, and the only device memory
// the call uses beyond them is the fixed static array below, which every GPU
// that loads this library holds until the process exits.
//
// The array is shared by all calls on a device and keeps the last call's
// contents.  Every call rewrites all of it that it reads (twiddle tables and
// filter spectrum) before reading it, so nothing needs clearing, but two
// calls whose device work overlaps in time (different streams, or different
// host threads) race on it.
#include <cuda_runtime.h>

#include <mutex>

#include "pac.h"

namespace pac {
int set_error(int status, const char* fmt, ...);
int be_init();
int conv_in_scratch(void* scratch, size_t scratch_bytes, int logn, int batch, const double* x_re,
                    const double* x_im, const double* h_re, const double* h_im, double* y_re,
                    double* y_im, void* stream);
}  // namespace pac

// filter spectrum (2 x 2^16 doubles = 1 MiB) plus twiddle tables (< 64 KiB)
#define PAC_NOALLOC_SCRATCH_BYTES (1280 * 1024)

static __device__ __align__(256) unsigned char g_noalloc_scratch[PAC_NOALLOC_SCRATCH_BYTES];

// Device address of the scratch array on the current device.  In host code
// the symbol's name is a host-side stand-in, not a device address, so the
// address is looked up with cudaGetSymbolAddress once per device (with that
// device current) and cached.
static int scratch_on_current_device(void** out) {
  static std::mutex mu;
  static void* addr[256] = {nullptr};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return pac::set_error(PAC_ERROR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= 256) return pac::set_error(PAC_ERROR_INTERNAL, "device index %d", dev);
  std::lock_guard<std::mutex> g(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return pac::set_error(PAC_ERROR_CUDA, "cudaGetSymbolAddress(scratch): %s",
                            cudaGetErrorString(e));
    addr[dev] = p;
  }
  *out = addr[dev];
  return PAC_SUCCESS;
}

extern "C" PAC_API int pac_convolve_1d_noalloc(const double* x_re, const double* x_im,
                                               const double* h_re, const double* h_im,
                                               double* y_re, double* y_im, int n, int batch,
                                               pac_stream_t stream) {
  if (!x_re || !x_im || !h_re || !h_im || !y_re || !y_im || batch < 1)
    return pac::set_error(PAC_ERROR_INVALID_VALUE, "pac_convolve_1d_noalloc: bad argument");
  // the size limit first: it bounds every shift below
  if (n > PAC_NOALLOC_MAX_N)
    return pac::set_error(PAC_ERROR_SIZE,
                          "pac_convolve_1d_noalloc: n = %d exceeds the no-allocation limit %d "
                          "(its scratch is a fixed %d-byte static device array)",
                          n, PAC_NOALLOC_MAX_N, PAC_NOALLOC_SCRATCH_BYTES);
  if (n < 1 || (n & (n - 1)) != 0)
    return pac::set_error(PAC_ERROR_NOT_POWER,
                          "pac_convolve_1d_noalloc: n = %d is not a power of 2", n);
  int logn = 0;
  while ((1 << logn) < n) ++logn;
  int st = pac::be_init();
  if (st != PAC_SUCCESS) return st;
  void* scratch = nullptr;
  st = scratch_on_current_device(&scratch);
  if (st != PAC_SUCCESS) return st;
  return pac::conv_in_scratch(scratch, PAC_NOALLOC_SCRATCH_BYTES, logn, batch, x_re, x_im, h_re,
                              h_im, y_re, y_im, stream);
}
