// pac_cuda.cu -- sm_100a kernels and the CUDA side of the plan layer.
//
// Kernels:
//   pac_pass_kernel<T, B2>   one pass of the butterfly engine (pac_engine.cuh):
//                            DIF / DIT / fused convolution, any radix schedule
//   pac_special_kernel       a pass compiled for one geometry (pac_special.h)
//   pac_cluster_kernel       a column pass whose tile a CTA cluster shares
//   fill_*_tw                twiddle tables generated in FP64 with sincospi and
//                            rounded once to the storage type
//   pointwise, scale_copy, round_to_f32, permute   small elementwise kernels
//
// There is no host fallback: every entry point requires an sm_100 device and
// fails with PAC_ERROR_NO_DEVICE otherwise.
#include <cooperative_groups.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <set>
#include <utility>

#include "pac.h"
#include "pac_backend.h"
#include "pac_special.h"
#include "pac_tma.cuh"

namespace cg = cooperative_groups;

namespace pac {

int set_error(int status, const char* fmt, ...);

static std::atomic<long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
// the tensor-copy column passes (pac_coltma.cu)
int launch_coltma(const PassDesc& d, int elem_bytes, int b2, long long grid, int threads,
                  size_t smem, void* stream);
// the plane passes of 3D convolutions (pac_plane.cu)
int launch_plane(const PassDesc& d, int elem_bytes, int b2, long long grid, int threads,
                 size_t smem, void* stream);

static int cuda_fail(cudaError_t e, const char* what) {
  return set_error(PAC_ERROR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}
#define PAC_CU(call, what)                      \
  do {                                          \
    cudaError_t _e = (call);                    \
    if (_e != cudaSuccess) return cuda_fail(_e, what); \
  } while (0)
#define PAC_TRY_BE(expr)                 \
  do {                                   \
    int _st = (expr);                    \
    if (_st != PAC_SUCCESS) return _st;  \
  } while (0)

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
template <typename T, int B2, int TC>
__global__ void __launch_bounds__(256) pac_pass_kernel(const PassDesc d) {
  extern __shared__ __align__(16) unsigned char pac_smem[];
  __shared__ long long s_lb[128];
  T* sre = reinterpret_cast<T*>(pac_smem);
  T* sim = sre + (size_t)d.W * d.pitch;
  const long long cta = blockIdx.x;
  if ((int)threadIdx.x < d.W) {
    const int w = threadIdx.x;
    const long long g = cta * d.W + w;
    if (d.nat) {
      nat_line<B2>(d, g, &s_lb[w], &s_lb[64 + w]);
    } else {
      s_lb[w] = line_base(d, g);
      s_lb[64 + w] = s_lb[w];
    }
  }
  __syncthreads();
  pass_body<T, B2, TC>(d, cta, sre, sim, s_lb, s_lb + 64);
}

// A pass compiled for one geometry (pac_special.h): tile W = 2^LOGW lines of
// 2^LOGL elements, NT threads, register bound for MINB CTAs per SM.
template <typename T, int B2, int MODE, int SIGN, int LOGL, int COLS, int LOGW, int NT, int MINB,
          int TC, int RC>
__global__ void __launch_bounds__(NT, MINB) pac_special_kernel(const PassDesc d) {
  constexpr int W = 1 << LOGW;
  constexpr int PITCH = pitch_for((int)sizeof(T), LOGL, W, COLS, TC);
  using SP = Shape<LOGL, LOGW, PITCH, COLS, TC>;
  extern __shared__ __align__(16) unsigned char pac_smem[];
  __shared__ long long s_lb[W];
  T* sre = reinterpret_cast<T*>(pac_smem);
  T* sim = sre + (size_t)W * PITCH;
  const long long cta = blockIdx.x;
  if ((int)threadIdx.x < W) s_lb[threadIdx.x] = line_base(d, cta * W + threadIdx.x);
  __syncthreads();
  pass_body_ct<T, B2, MODE, SIGN, SP, NT, RadsCap<LOGL, B2, RC>, TC>(d, cta, sre, sim, s_lb, s_lb);
}

// Persistent CTAs over a device work queue (many passes of different
// geometry in one launch, pac_multi.cpp): thread 0 takes the next item from
// the counter and reads its pass k from the item table; the pass descriptor
// is copied into shared memory (unless the CTA's previous item had the same
// pass) and the CTA runs that pass's CTA `item - starts[k]` with the
// run-time geometry of pac_pass_kernel.
// (FP32: two CTAs per SM, the register bound the compile-time bodies are
// written for; FP64 keeps one)
template <typename T, int B2, int TC>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 2 : 1) pac_queue_kernel(const PassDesc* __restrict__ descs,
                                                        const long long* __restrict__ starts,
                                                        const int* __restrict__ item_desc,
                                                        long long total,
                                                        unsigned long long* counter) {
  extern __shared__ __align__(16) unsigned char pac_smem[];
  __shared__ PassDesc sd;
  __shared__ long long s_lb[128];
  __shared__ long long s_item;
  __shared__ int s_k;
  static_assert(sizeof(PassDesc) % sizeof(int) == 0, "descriptor copy in words");
  int have = -1;  // pass whose descriptor sd holds
  for (;;) {
    if (threadIdx.x == 0) {
      const long long it = (long long)atomicAdd(counter, 1ULL);
      s_item = it;
      s_k = it < total ? item_desc[it] : 0;
    }
    __syncthreads();
    const long long it = s_item;
    if (it >= total) break;
    const int k = s_k;
    if (k != have) {
      const int* src = reinterpret_cast<const int*>(descs + k);
      int* dst = reinterpret_cast<int*>(&sd);
      for (int i = threadIdx.x; i < (int)(sizeof(PassDesc) / sizeof(int)); i += blockDim.x)
        dst[i] = src[i];
      have = k;
    }
    __syncthreads();
    const long long cta = it - starts[k];
    T* sre = reinterpret_cast<T*>(pac_smem);
    T* sim = sre + (size_t)sd.W * sd.pitch;
    if ((int)threadIdx.x < sd.W) {
      const long long g = cta * sd.W + threadIdx.x;
      s_lb[threadIdx.x] = line_base(sd, g);
      s_lb[64 + threadIdx.x] = s_lb[threadIdx.x];
    }
    __syncthreads();
    queue_pass_body<T, B2, TC>(sd, cta, sre, sim, s_lb, s_lb + 64);
    __syncthreads();  // sd, s_lb and the tile are reused by the next item
  }
}

// A column pass whose tile is shared by a cluster of 2^LOGC CTAs
// (pac_special.h, PAC_CLUSTER_LIST): CTA `rank` of the cluster holds rows
// [rank * L/C, (rank + 1) * L/C) of the tile's W columns.  Barriers across
// the cluster separate the phases of pass_body_cl: the first one also
// guarantees that every CTA of the cluster runs before any distributed
// shared-memory access, and in DIT the last one keeps each CTA's tile alive
// while its peers still read it.
template <typename T, int B2, int MODE, int SIGN, int LOGL, int LOGW, int LOGC, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) pac_cluster_kernel(const PassDesc d) {
  constexpr int C = 1 << LOGC, W = 1 << LOGW;
  constexpr int PITCH = pitch_for((int)sizeof(T), LOGL - LOGC, W);
  using SP = Shape<LOGL, LOGW, PITCH, 1>;
  using RS = RadsFor<LOGL, B2>;
  extern __shared__ __align__(16) unsigned char pac_smem[];
  __shared__ long long s_lb[W];
  T* sre = reinterpret_cast<T*>(pac_smem);
  T* sim = sre + (size_t)W * PITCH;
  cg::cluster_group cl = cg::this_cluster();
  ClView<T, C> cv;
  cv.rank = (int)cl.block_rank();
#pragma unroll
  for (int r = 0; r < C; ++r) {
    cv.re[r] = cl.map_shared_rank(sre, r);
    cv.im[r] = cl.map_shared_rank(sim, r);
  }
  const long long cta = (long long)(blockIdx.x >> LOGC);
  if ((int)threadIdx.x < W) s_lb[threadIdx.x] = line_base(d, cta * W + threadIdx.x);
  cl.sync();
  pass_body_cl<T, B2, MODE, SIGN, SP, NT, RS, LOGC>(d, cta, sre, sim, cv, s_lb, 0);
  cl.sync();
  pass_body_cl<T, B2, MODE, SIGN, SP, NT, RS, LOGC>(d, cta, sre, sim, cv, s_lb, 1);
  if constexpr (MODE == MODE_DIT) cl.sync();
}

// A pipelined column pass (ColPipe): persistent CTAs walk the tiles
// blockIdx.x, blockIdx.x + gridDim.x, ...; thread 0 issues the tensor
// copies of a CTA's next tile as soon as the current one is in registers.
// Every wait is bounded: on a timeout all threads leave together (after a
// CTA-wide vote) and the pass reports PAC_ERROR_TIMEOUT in d.status.
template <typename T, int B2, int MODE, int SIGN, int LOGL, int LOGW, int NT>
__global__ void __launch_bounds__(NT, 1)
    pac_pipe_kernel(const PassDesc d, const __grid_constant__ CUtensorMap tin_re,
                    const __grid_constant__ CUtensorMap tin_im) {
  using CP = ColPipe<T, B2, MODE, SIGN, LOGL, LOGW, NT>;
  constexpr int W = CP::W, L = CP::L, BOXR = CP::BOXR, NS = CP::NS;
  extern __shared__ unsigned char pac_smem_raw[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ long long s_lb[W];
  // dense tile (tensor-copy destination, 1024-byte aligned), then the
  // exchange array
  T* Are = reinterpret_cast<T*>(smem_align1024(pac_smem_raw));
  T* Aim = Are + W * L;
  T* X = Aim + W * L;
  const int t = threadIdx.x;
  const long long ntiles = d.nlines >> LOGW;
  auto issue = [&](long long tl) {
    const long long g0 = tl << LOGW;
    const int i0 = (int)(g0 & ((1LL << d.logS) - 1));
    const int o = (int)(g0 >> d.logS);
    mbar_arrive_expect_tx(&bar, (uint32_t)(2 * W * L * sizeof(T)));
    for (int k = 0; k < L / BOXR; ++k) {
      tma_load_3d(Are + k * BOXR * W, &tin_re, &bar, i0, k * BOXR, o);
      tma_load_3d(Aim + k * BOXR * W, &tin_im, &bar, i0, k * BOXR, o);
    }
  };
  if (t == 0) {
    mbar_init(&bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  long long tile = blockIdx.x;
  if (t == 0 && tile < ntiles) issue(tile);
  uint32_t phase = 0;
  Cx<T> x[CP::TPT];
  for (; tile < ntiles; tile += gridDim.x) {
    if (t < W) s_lb[t] = line_base(d, tile * W + t);
    const bool ok = mbar_wait_bounded(&bar, phase, wait_limit_of(d));
    if (!__syncthreads_and(ok)) {
      // a wait gave up: report it, issue nothing more, and keep the CTA (its
      // shared memory) alive until the copies in flight have landed
      if (t == 0) {
        report_timeout(d);
        mbar_wait_bounded(&bar, phase);
      }
      break;
    }
    phase ^= 1;
    CP::load_tile(t, Are, Aim, x);
    __syncthreads();  // the tile is in registers: the buffer may be refilled
    if (t == 0 && tile + gridDim.x < ntiles) {
      fence_proxy_async();
      issue(tile + gridDim.x);
    }
    if constexpr (MODE == MODE_DIT) {
      CP::template xw<-1, 0>(t, X, x);
      __syncthreads();
      CP::template xr<-1, 0>(t, X, x);
      __syncthreads();
      CP::template xw<-1, 1>(t, X, x);
      __syncthreads();
      CP::template xr<-1, 1>(t, X, x);
    }
    static_for<NS>([&](auto ss) {
      constexpr int S = ss.value;
      if constexpr (S > 0) {
        __syncthreads();
        CP::template xw<S - 1, 0>(t, X, x);
        __syncthreads();
        CP::template xr<S - 1, 0>(t, X, x);
        __syncthreads();
        CP::template xw<S - 1, 1>(t, X, x);
        __syncthreads();
        CP::template xr<S - 1, 1>(t, X, x);
      }
      CP::template compute<S>(d, tile, t, x);
    });
    CP::store(d, t, s_lb, x);
    __syncthreads();  // s_lb and the exchange array are reused by the next tile
  }
}

template <typename T>
__global__ void fill_stage_tw_kernel(Cx<T>* dst, int logK, int logR) {
  const long long R1 = (1LL << logR) - 1;
  const long long n = (1LL << (logK - logR)) * R1;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x) {
    // s-major: entry (s-1)*ell + j = w_K^{j s}
    const long long ell = 1LL << (logK - logR);
    long long s = idx / ell + 1, j = idx % ell;
    long long E = (j * s) & ((1LL << logK) - 1);
    double x = -2.0 * (double)E / (double)(1LL << logK);
    double sn, cs;
    sincospi(x, &sn, &cs);
    dst[idx] = Cx<T>{T(cs), T(sn)};
  }
}

template <typename T>
__global__ void fill_pow_tw_kernel(Cx<T>* dst, long long count, long long stride, int logN) {
  const long long mask = (1LL << logN) - 1;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < count;
       k += (long long)gridDim.x * blockDim.x) {
    long long E = (k * stride) & mask;
    double x = -2.0 * (double)E / (double)(1LL << logN);
    double sn, cs;
    sincospi(x, &sn, &cs);
    dst[k] = Cx<T>{T(cs), T(sn)};
  }
}

// reference layout: level q at offset r^q - 1, entry (m-1)*ell + j = w_k^{m j}
__global__ void fill_ref_tw_kernel(int r, int t, double* re, double* im) {
  long long total = 1;
  for (int q = 0; q < t; ++q) total *= r;
  total -= 1;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    long long ell = 1;
    while (idx >= ell * r - 1) ell *= r;
    long long local = idx - (ell - 1);
    long long m = local / ell + 1, j = local % ell;
    long long k = ell * r;
    long long E = (m * j) % k;
    double sn, cs;
    sincospi(-2.0 * (double)E / (double)k, &sn, &cs);
    re[idx] = cs;
    im[idx] = sn;
  }
}

// P order -> plan order, one line per CTA iteration through shared memory
// (the whole line is read before any of it is written, so in == out works)
template <typename Tout>
__global__ void plan_order_kernel(const double* in_re, const double* in_im, Tout* out_re,
                                  Tout* out_im, int logL, int logR, long long nlines,
                                  double scale) {
  extern __shared__ double pbuf[];
  const int L = 1 << logL, lq = logL - logR;
  for (long long line = blockIdx.x; line < nlines; line += gridDim.x) {
    const long long base = line << logL;
    for (int q = threadIdx.x; q < L; q += blockDim.x) {
      pbuf[q] = in_re[base + q];
      pbuf[L + q] = in_im[base + q];
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < L; idx += blockDim.x) {
      const int t = idx >> lq, blk = idx & ((1 << lq) - 1);
      const int q = (blk << logR) + t;
      out_re[base + idx] = (Tout)(pbuf[q] * scale);
      out_im[base + idx] = (Tout)(pbuf[L + q] * scale);
    }
    __syncthreads();
  }
}

__global__ void round_f32_kernel(const double* src, float* dst, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    dst[i] = (float)src[i];
}

template <typename T>
__global__ void pointwise_kernel(long long n, const T* xr, const T* xi, const T* hr, const T* hi,
                                 long long hmask, T* yr, T* yi, T scale) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    T ar = xr[i], ai = xi[i];
    long long k = i & hmask;
    T br = hr[k], bi = hi[k];
    yr[i] = (ar * br - ai * bi) * scale;
    yi[i] = (ar * bi + ai * br) * scale;
  }
}

template <typename T>
__global__ void scale_copy_kernel(long long n, const T* xr, const T* xi, T* yr, T* yi, T scale) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    yr[i] = xr[i] * scale;
    yi[i] = xi[i] * scale;
  }
}

// swap-based permutation by an involution (index_reversals.c:74-94); with
// im == nullptr `re` holds interleaved (re, im) pairs
__global__ void permute_kernel(long long n, const int* rho, double* re, double* im) {
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    long long p = rho[j];
    if (j < p && p < n) {
      if (im) {
        double a = re[j], b = im[j];
        re[j] = re[p];
        im[j] = im[p];
        re[p] = a;
        im[p] = b;
      } else {
        double2* z = reinterpret_cast<double2*>(re);
        double2 a = z[j];
        z[j] = z[p];
        z[p] = a;
      }
    }
  }
}

static int grid_for(long long n) {
  long long g = (n + 255) / 256;
  if (g > 148 * 32) g = 148 * 32;
  if (g < 1) g = 1;
  return (int)g;
}

// ---------------------------------------------------------------------------
// backend interface
// ---------------------------------------------------------------------------
int be_init() {
  static std::once_flag once;
  static int status = PAC_SUCCESS;
  static char msg[256];
  std::call_once(once, [] {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
      status = PAC_ERROR_NO_DEVICE;
      snprintf(msg, sizeof(msg), "no CUDA device (%s)", cudaGetErrorString(e));
      return;
    }
    int dev = 0, major = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    if (major != 10) {
      status = PAC_ERROR_NO_DEVICE;
      snprintf(msg, sizeof(msg), "device %d is sm_%d0, this library is built for sm_100a", dev,
               major);
    }
  });
  if (status != PAC_SUCCESS) return set_error(status, "%s", msg);
  return PAC_SUCCESS;
}

int be_device_name(char* buf, int n) {
  int dev = 0;
  PAC_CU(cudaGetDevice(&dev), "cudaGetDevice");
  cudaDeviceProp prop;
  PAC_CU(cudaGetDeviceProperties(&prop, dev), "cudaGetDeviceProperties");
  snprintf(buf, (size_t)n, "%s", prop.name);
  return PAC_SUCCESS;
}

int be_num_sms() {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1)
    return 1;
  return n;
}

int be_malloc(void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
  if (e != cudaSuccess) {
    *p = nullptr;
    return set_error(PAC_ERROR_ALLOC, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
  }
  return PAC_SUCCESS;
}

int be_free(void* p) {
  if (p) PAC_CU(cudaFree(p), "cudaFree");
  return PAC_SUCCESS;
}

int be_memcpy(void* dst, const void* src, size_t bytes, int kind, void* stream) {
  if (!bytes) return PAC_SUCCESS;
  cudaMemcpyKind k = kind == CPY_H2D   ? cudaMemcpyHostToDevice
                     : kind == CPY_D2H ? cudaMemcpyDeviceToHost
                                       : cudaMemcpyDeviceToDevice;
  PAC_CU(cudaMemcpyAsync(dst, src, bytes, k, (cudaStream_t)stream), "cudaMemcpyAsync");
  return PAC_SUCCESS;
}

int be_memset(void* dst, int value, size_t bytes, void* stream) {
  PAC_CU(cudaMemsetAsync(dst, value, bytes, (cudaStream_t)stream), "cudaMemsetAsync");
  return PAC_SUCCESS;
}

int be_stream_create(void** s) {
  cudaStream_t st;
  PAC_CU(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
  *s = st;
  return PAC_SUCCESS;
}
int be_stream_destroy(void* s) {
  if (s) PAC_CU(cudaStreamDestroy((cudaStream_t)s), "cudaStreamDestroy");
  return PAC_SUCCESS;
}
int be_stream_sync(void* s) {
  PAC_CU(cudaStreamSynchronize((cudaStream_t)s), "cudaStreamSynchronize");
  return PAC_SUCCESS;
}
long long be_l2_bytes() {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&n, cudaDevAttrL2CacheSize, dev) != cudaSuccess || n < 0)
    return 0;
  return n;
}

int be_l2_persist(void* stream, const void* base, size_t bytes) {
  int dev = 0;
  PAC_CU(cudaGetDevice(&dev), "cudaGetDevice");
  cudaDeviceProp prop;
  PAC_CU(cudaGetDeviceProperties(&prop, dev), "cudaGetDeviceProperties");
  cudaStreamAttrValue v;
  memset(&v, 0, sizeof(v));
  if (bytes > 0 && prop.persistingL2CacheMaxSize > 0) {
    size_t limit = bytes < (size_t)prop.persistingL2CacheMaxSize ? bytes
                                                                  : (size_t)prop.persistingL2CacheMaxSize;
    PAC_CU(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, limit), "cudaDeviceSetLimit");
    size_t win = bytes < (size_t)prop.accessPolicyMaxWindowSize ? bytes
                                                                : (size_t)prop.accessPolicyMaxWindowSize;
    v.accessPolicyWindow.base_ptr = const_cast<void*>(base);
    v.accessPolicyWindow.num_bytes = win;
    v.accessPolicyWindow.hitRatio = (float)((double)limit / (double)win > 1.0 ? 1.0 : (double)limit / (double)win);
    v.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    v.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
  }
  PAC_CU(cudaStreamSetAttribute((cudaStream_t)stream, cudaStreamAttributeAccessPolicyWindow, &v),
         "cudaStreamSetAttribute");
  if (bytes == 0) {
    // back to no set-aside: persisting lines become normal lines and the
    // whole L2 serves normal accesses again
    cudaCtxResetPersistingL2Cache();
    if (prop.persistingL2CacheMaxSize > 0)
      PAC_CU(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, 0), "cudaDeviceSetLimit");
  }
  return PAC_SUCCESS;
}

int be_event_create(void** ev) {
  cudaEvent_t e;
  PAC_CU(cudaEventCreate(&e), "cudaEventCreate");
  *ev = e;
  return PAC_SUCCESS;
}
int be_event_destroy(void* ev) {
  if (ev) cudaEventDestroy((cudaEvent_t)ev);
  return PAC_SUCCESS;
}
int be_event_record(void* ev, void* stream) {
  PAC_CU(cudaEventRecord((cudaEvent_t)ev, (cudaStream_t)stream), "cudaEventRecord");
  return PAC_SUCCESS;
}
int be_event_elapsed(void* a, void* b, float* ms) {
  PAC_CU(cudaEventSynchronize((cudaEvent_t)b), "cudaEventSynchronize");
  PAC_CU(cudaEventElapsedTime(ms, (cudaEvent_t)a, (cudaEvent_t)b), "cudaEventElapsedTime");
  return PAC_SUCCESS;
}
int be_stream_wait(void* waiter, void* waitee) {
  cudaEvent_t ev;
  PAC_CU(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "cudaEventCreate");
  cudaError_t e = cudaEventRecord(ev, (cudaStream_t)waitee);
  if (e == cudaSuccess) e = cudaStreamWaitEvent((cudaStream_t)waiter, ev, 0);
  cudaEventDestroy(ev);
  if (e != cudaSuccess) return cuda_fail(e, "stream wait");
  return PAC_SUCCESS;
}

template <typename T, int B2, int TC = 0>
static int launch_pass_t(const PassDesc& d, long long grid, int threads, size_t smem,
                         void* stream) {
  // opt the kernel into the device's whole shared-memory budget once per
  // device, so that every pass geometry (<= 200 KiB) launches
  static std::mutex mu;
  static std::set<int> configured;
  auto kern = pac_pass_kernel<T, B2, TC>;
  if (smem > 48 * 1024) {
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> g(mu);
    if (!configured.count(dev)) {
      int optin = 0;
      PAC_CU(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev),
             "cudaDeviceGetAttribute");
      cudaFuncAttributes fa;
      PAC_CU(cudaFuncGetAttributes(&fa, kern), "cudaFuncGetAttributes");
      PAC_CU(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  optin - (int)fa.sharedSizeBytes),
             "cudaFuncSetAttribute");
      configured.insert(dev);
    }
  }
  if (grid > 0x7fffffffLL) return set_error(PAC_ERROR_SIZE, "pass grid too large");
  kern<<<(unsigned)grid, threads, smem, (cudaStream_t)stream>>>(d);
  PAC_CU(cudaGetLastError(), "pac_pass_kernel launch");
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return PAC_SUCCESS;
}

template <typename K>
static int launch_kernel(K kern, const PassDesc& d, long long grid, int threads, size_t smem,
                         void* stream, std::set<int>& configured, std::mutex& mu) {
  if (smem > 48 * 1024) {
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> g(mu);
    if (!configured.count(dev)) {
      int optin = 0;
      PAC_CU(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev),
             "cudaDeviceGetAttribute");
      cudaFuncAttributes fa;
      PAC_CU(cudaFuncGetAttributes(&fa, kern), "cudaFuncGetAttributes");
      PAC_CU(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  optin - (int)fa.sharedSizeBytes),
             "cudaFuncSetAttribute");
      configured.insert(dev);
    }
  }
  if (grid > 0x7fffffffLL) return set_error(PAC_ERROR_SIZE, "pass grid too large");
  kern<<<(unsigned)grid, threads, smem, (cudaStream_t)stream>>>(d);
  PAC_CU(cudaGetLastError(), "pac_special_kernel launch");
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return PAC_SUCCESS;
}

static int launch_special(const PassDesc& d, int elem_bytes, int b2, long long grid, int threads,
                          size_t smem, void* stream, bool* done) {
  *done = false;
  const int cols = d.logS > 0 ? 1 : 0;
  int seen = 0;  // candidates of this geometry so far; d.spec - 1 picks one
#define PAC_X(T, BY, B2_, MO, SG, LL, CO, LW, NT_, MB, TC_, RC_)                              \
  if (!*done && elem_bytes == BY && b2 == B2_ && d.mode == MO &&                           \
      (MO == MODE_CONV || d.sign == SG) && d.logL == LL && cols == CO && d.tc == TC_ &&    \
      rads_match(d, LL, B2_, RC_) && seen++ == d.spec - 1 && d.W == (1 << LW) &&           \
      threads == NT_) {                                                                    \
    static std::mutex mu;                                                                  \
    static std::set<int> configured;                                                       \
    *done = true;                                                                          \
    return launch_kernel(pac_special_kernel<T, B2_, MO, SG, LL, CO, LW, NT_, MB, TC_, RC_>, \
                         d, grid, threads, smem, stream, configured, mu);                  \
  }
  PAC_SPECIAL_LIST(PAC_X)
#undef PAC_X
  return set_error(PAC_ERROR_INTERNAL, "no specialised kernel for a pass marked special");
}

// A cluster pass: grid = tiles x 2^logC CTAs, launched with a cluster shape
// of (2^logC, 1, 1), so the CTAs of one tile are consecutive blocks.
static int launch_cluster(const PassDesc& d, int elem_bytes, int b2, long long grid, int threads,
                          size_t smem, void* stream) {
#define PAC_X(T, BY, B2_, MO, SG, LL, LW, LC, NT_, MB)                                         \
  if (elem_bytes == BY && b2 == B2_ && d.mode == MO && d.sign == SG && d.logL == LL &&      \
      d.W == (1 << LW) && d.logC == LC && threads == NT_) {                                 \
    static std::mutex mu;                                                                   \
    static std::set<int> configured;                                                        \
    auto kern = pac_cluster_kernel<T, B2_, MO, SG, LL, LW, LC, NT_, MB>;                    \
    if (smem > 48 * 1024) {                                                                 \
      int dev = 0;                                                                          \
      PAC_CU(cudaGetDevice(&dev), "cudaGetDevice");                                         \
      std::lock_guard<std::mutex> g(mu);                                                    \
      if (!configured.count(dev)) {                                                         \
        PAC_CU(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,      \
                                    (int)smem),                                             \
               "cudaFuncSetAttribute");                                                     \
        configured.insert(dev);                                                             \
      }                                                                                     \
    }                                                                                       \
    if (grid > 0x7fffffffLL || (grid & ((1LL << LC) - 1)) != 0)                             \
      return set_error(PAC_ERROR_INTERNAL, "cluster pass grid %lld", grid);                 \
    cudaLaunchConfig_t cfg = {};                                                            \
    cfg.gridDim = dim3((unsigned)grid);                                                     \
    cfg.blockDim = dim3((unsigned)threads);                                                 \
    cfg.dynamicSmemBytes = smem;                                                            \
    cfg.stream = (cudaStream_t)stream;                                                      \
    cudaLaunchAttribute at[1];                                                              \
    at[0].id = cudaLaunchAttributeClusterDimension;                                         \
    at[0].val.clusterDim.x = 1u << LC;                                                      \
    at[0].val.clusterDim.y = 1;                                                             \
    at[0].val.clusterDim.z = 1;                                                             \
    cfg.attrs = at;                                                                         \
    cfg.numAttrs = 1;                                                                       \
    PAC_CU(cudaLaunchKernelEx(&cfg, kern, d), "pac_cluster_kernel launch");                 \
    g_launches.fetch_add(1, std::memory_order_relaxed);                                     \
    return PAC_SUCCESS;                                                                     \
  }
  PAC_CLUSTER_LIST(PAC_X)
#undef PAC_X
  return set_error(PAC_ERROR_INTERNAL, "no cluster kernel for a pass marked clustered");
}

// ---------------------------------------------------------------------------
// work-queue launches and graphs (pac_multi.cpp)
// ---------------------------------------------------------------------------
template <typename T, int B2, int TC = 0>
static int queue_prepare_t(size_t smem, int* grid_per_sm) {
  static std::mutex mu;
  static std::set<int> configured;
  auto kern = pac_queue_kernel<T, B2, TC>;
  int dev = 0;
  PAC_CU(cudaGetDevice(&dev), "cudaGetDevice");
  {
    std::lock_guard<std::mutex> g(mu);
    if (!configured.count(dev)) {
      int optin = 0;
      PAC_CU(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev),
             "cudaDeviceGetAttribute");
      cudaFuncAttributes fa;
      PAC_CU(cudaFuncGetAttributes(&fa, kern), "cudaFuncGetAttributes");
      PAC_CU(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  optin - (int)fa.sharedSizeBytes),
             "cudaFuncSetAttribute");
      configured.insert(dev);
    }
  }
  if (grid_per_sm) {
    int nb = 0;
    PAC_CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, 256, smem),
           "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (nb < 1) return set_error(PAC_ERROR_SIZE, "work-queue pass needs %zu bytes of shared memory", smem);
    *grid_per_sm = nb;
  }
  return PAC_SUCCESS;
}

static int queue_prepare(int elem_bytes, int b2, int tc, size_t smem, int* grid_per_sm) {
  if (tc && b2 != 3) {  // (base-8 schedules have no radix-16 stage)
    if (b2 == 1) return queue_prepare_t<float, 1, 1>(smem, grid_per_sm);
    return queue_prepare_t<float, 2, 1>(smem, grid_per_sm);
  }
  if (elem_bytes == 8) {
    if (b2 == 1) return queue_prepare_t<double, 1>(smem, grid_per_sm);
    if (b2 == 2) return queue_prepare_t<double, 2>(smem, grid_per_sm);
    return queue_prepare_t<double, 3>(smem, grid_per_sm);
  }
  if (b2 == 1) return queue_prepare_t<float, 1>(smem, grid_per_sm);
  if (b2 == 2) return queue_prepare_t<float, 2>(smem, grid_per_sm);
  return queue_prepare_t<float, 3>(smem, grid_per_sm);
}

int be_queue_prepare(int elem_bytes, int b2, int tc, size_t smem) {
  return queue_prepare(elem_bytes, b2, tc, smem, nullptr);
}

int be_launch_queue(const PassDesc* descs, const long long* starts, const int* item_desc,
                    int ndesc, long long total, unsigned long long* counter, int elem_bytes,
                    int b2, int tc, size_t smem, void* stream) {
  (void)ndesc;
  if (total <= 0) return PAC_SUCCESS;
  int per_sm = 0;
  PAC_TRY_BE(queue_prepare(elem_bytes, b2, tc, smem, &per_sm));
  long long grid = (long long)per_sm * be_num_sms();
  if (grid > total) grid = total;
  cudaStream_t s = (cudaStream_t)stream;
#define PAC_Q(T, B, TC_)                                                                \
  pac_queue_kernel<T, B, TC_><<<(unsigned)grid, 256, smem, s>>>(descs, starts, item_desc, \
                                                                  total, counter)
  if (tc && b2 != 3) {
    if (b2 == 1) PAC_Q(float, 1, 1);
    else PAC_Q(float, 2, 1);
  } else if (elem_bytes == 8) {
    if (b2 == 1) PAC_Q(double, 1, 0);
    else if (b2 == 2) PAC_Q(double, 2, 0);
    else PAC_Q(double, 3, 0);
  } else {
    if (b2 == 1) PAC_Q(float, 1, 0);
    else if (b2 == 2) PAC_Q(float, 2, 0);
    else PAC_Q(float, 3, 0);
  }
#undef PAC_Q
  PAC_CU(cudaGetLastError(), "pac_queue_kernel launch");
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return PAC_SUCCESS;
}

int be_graph_supported() { return 1; }

int be_graph_begin(void* stream) {
  PAC_CU(cudaStreamBeginCapture((cudaStream_t)stream, cudaStreamCaptureModeThreadLocal),
         "cudaStreamBeginCapture");
  return PAC_SUCCESS;
}

int be_graph_end(void* stream, void** exec) {
  cudaGraph_t g = nullptr;
  PAC_CU(cudaStreamEndCapture((cudaStream_t)stream, &g), "cudaStreamEndCapture");
  cudaGraphExec_t e = nullptr;
  cudaError_t err = cudaGraphInstantiate(&e, g, 0);
  cudaGraphDestroy(g);
  if (err != cudaSuccess) return cuda_fail(err, "cudaGraphInstantiate");
  *exec = (void*)e;
  return PAC_SUCCESS;
}

int be_graph_launch(void* exec, void* stream) {
  PAC_CU(cudaGraphLaunch((cudaGraphExec_t)exec, (cudaStream_t)stream), "cudaGraphLaunch");
  return PAC_SUCCESS;
}

int be_graph_destroy(void* exec) {
  if (exec) PAC_CU(cudaGraphExecDestroy((cudaGraphExec_t)exec), "cudaGraphExecDestroy");
  return PAC_SUCCESS;
}

// 3D view (S columns, L rows, O = nlines / S outer) of a column pass's input
// array; box W x boxr x 1, unswizzled, so a box lands as dense rows of W
// elements
static int col_tensor_map(CUtensorMap* m, const void* base, int esz, const PassDesc& d,
                          int boxr) {
  auto enc = tensor_map_encoder();
  if (!enc) return set_error(PAC_ERROR_CUDA, "cuTensorMapEncodeTiled unavailable");
  const cuuint64_t S = 1ull << d.logS, L = 1ull << d.logL;
  cuuint64_t dims[3] = {S, L, (cuuint64_t)(d.nlines >> d.logS)};
  cuuint64_t strides[2] = {S * esz, S * L * esz};
  cuuint32_t box[3] = {(cuuint32_t)d.W, (cuuint32_t)boxr, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(m, esz == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                   3, const_cast<void*>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return set_error(PAC_ERROR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return PAC_SUCCESS;
}

static int launch_pipe(const PassDesc& d, int elem_bytes, int b2, long long grid, int threads,
                       size_t smem, void* stream) {
#define PAC_X(T, BY, B2_, MO, SG, LL, LW, NT_)                                               \
  if (elem_bytes == BY && b2 == B2_ && d.mode == MO && d.sign == SG && d.logL == LL &&      \
      d.W == (1 << LW) && threads == NT_) {                                                 \
    using CP = ColPipe<T, B2_, MO, SG, LL, LW, NT_>;                                        \
    static std::mutex mu;                                                                   \
    static std::set<int> configured;                                                        \
    auto kern = pac_pipe_kernel<T, B2_, MO, SG, LL, LW, NT_>;                               \
    CUtensorMap m[2];                                                                       \
    PAC_TRY_BE(col_tensor_map(&m[0], d.in_re, BY, d, CP::BOXR));                            \
    PAC_TRY_BE(col_tensor_map(&m[1], d.in_im, BY, d, CP::BOXR));                            \
    {                                                                                       \
      int dev = 0;                                                                          \
      PAC_CU(cudaGetDevice(&dev), "cudaGetDevice");                                         \
      std::lock_guard<std::mutex> g(mu);                                                    \
      if (!configured.count(dev)) {                                                         \
        PAC_CU(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,      \
                                    (int)smem),                                             \
               "cudaFuncSetAttribute");                                                     \
        configured.insert(dev);                                                             \
      }                                                                                     \
    }                                                                                       \
    if (grid > 0x7fffffffLL) return set_error(PAC_ERROR_SIZE, "pass grid too large");       \
    kern<<<(unsigned)grid, threads, smem, (cudaStream_t)stream>>>(d, m[0], m[1]);           \
    PAC_CU(cudaGetLastError(), "pac_pipe_kernel launch");                                   \
    g_launches.fetch_add(1, std::memory_order_relaxed);                                     \
    return PAC_SUCCESS;                                                                     \
  }
  PAC_PIPE_LIST(PAC_X)
#undef PAC_X
  return set_error(PAC_ERROR_INTERNAL, "no pipelined kernel for a pass marked pipelined");
}

int be_launch_pass(const PassDesc& d, int elem_bytes, int b2, long long grid, int threads,
                   size_t smem, void* stream) {
  if (d.plane) return launch_plane(d, elem_bytes, b2, grid, threads, smem, stream);
  if (d.tma) return launch_coltma(d, elem_bytes, b2, grid, threads, smem, stream);
  if (d.pipe) return launch_pipe(d, elem_bytes, b2, grid, threads, smem, stream);
  if (d.logC > 0) return launch_cluster(d, elem_bytes, b2, grid, threads, smem, stream);
  if (d.spec) {
    bool done = false;
    return launch_special(d, elem_bytes, b2, grid, threads, smem, stream, &done);
  }
  if (d.tc) {
    // tensor-core form: FP32 storage, radix-16 stages (digit bases 2 and 4;
    // base-8 schedules have no radix-16 stage)
    if (b2 == 1) return launch_pass_t<float, 1, 1>(d, grid, threads, smem, stream);
    if (b2 == 2) return launch_pass_t<float, 2, 1>(d, grid, threads, smem, stream);
    return launch_pass_t<float, 3>(d, grid, threads, smem, stream);
  }
  if (elem_bytes == 8) {
    if (b2 == 1) return launch_pass_t<double, 1>(d, grid, threads, smem, stream);
    if (b2 == 2) return launch_pass_t<double, 2>(d, grid, threads, smem, stream);
    return launch_pass_t<double, 3>(d, grid, threads, smem, stream);
  }
  if (b2 == 1) return launch_pass_t<float, 1>(d, grid, threads, smem, stream);
  if (b2 == 2) return launch_pass_t<float, 2>(d, grid, threads, smem, stream);
  return launch_pass_t<float, 3>(d, grid, threads, smem, stream);
}

#define PAC_LAUNCHED(what)                  \
  do {                                      \
    PAC_CU(cudaGetLastError(), what);       \
    g_launches.fetch_add(1);                \
  } while (0)

__global__ void fill_tc_const_kernel(TcConst* t) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < TC_CONST_SETS * 32) tc_const_fill(i >> 5, i & 31, t[i]);
}

int be_fill_tc_const(void* dst, void* stream) {
  fill_tc_const_kernel<<<TC_CONST_SETS, 32, 0, (cudaStream_t)stream>>>((TcConst*)dst);
  PAC_LAUNCHED("fill_tc_const");
  return PAC_SUCCESS;
}

int be_fill_stage_tw(void* dst, int elem_bytes, int logK, int logR, void* stream) {
  long long n = (1LL << (logK - logR)) * ((1LL << logR) - 1);
  if (elem_bytes == 8)
    fill_stage_tw_kernel<double><<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(
        (Cx<double>*)dst, logK, logR);
  else
    fill_stage_tw_kernel<float><<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(
        (Cx<float>*)dst, logK, logR);
  PAC_LAUNCHED("fill_stage_tw");
  return PAC_SUCCESS;
}

int be_fill_pow_tw(void* dst, int elem_bytes, long long count, long long stride, int logN,
                   void* stream) {
  if (elem_bytes == 8)
    fill_pow_tw_kernel<double><<<grid_for(count), 256, 0, (cudaStream_t)stream>>>(
        (Cx<double>*)dst, count, stride, logN);
  else
    fill_pow_tw_kernel<float><<<grid_for(count), 256, 0, (cudaStream_t)stream>>>(
        (Cx<float>*)dst, count, stride, logN);
  PAC_LAUNCHED("fill_pow_tw");
  return PAC_SUCCESS;
}

int be_fill_ref_tw(int r, int t, double* re, double* im, void* stream) {
  long long total = 1;
  for (int q = 0; q < t; ++q) total *= r;
  fill_ref_tw_kernel<<<grid_for(total), 256, 0, (cudaStream_t)stream>>>(r, t, re, im);
  PAC_LAUNCHED("fill_ref_tw");
  return PAC_SUCCESS;
}

int be_plan_order(const double* in_re, const double* in_im, void* out_re, void* out_im,
                  int elem_bytes, int logL, int logR, long long nlines, double scale,
                  void* stream) {
  static std::mutex mu;
  static std::set<std::pair<int, int>> configured;
  const size_t smem = (size_t)2 * sizeof(double) << logL;
  long long grid = nlines < 148 * 8 ? nlines : 148 * 8;
  if (grid < 1) grid = 1;
  int dev = 0;
  cudaGetDevice(&dev);
  if (elem_bytes == 8) {
    if (smem > 48 * 1024) {
      std::lock_guard<std::mutex> g(mu);
      if (!configured.count({dev, 8})) {
        PAC_CU(cudaFuncSetAttribute(plan_order_kernel<double>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024),
               "cudaFuncSetAttribute");
        configured.insert({dev, 8});
      }
    }
    plan_order_kernel<double><<<(unsigned)grid, 256, smem, (cudaStream_t)stream>>>(
        in_re, in_im, (double*)out_re, (double*)out_im, logL, logR, nlines, scale);
  } else {
    if (smem > 48 * 1024) {
      std::lock_guard<std::mutex> g(mu);
      if (!configured.count({dev, 4})) {
        PAC_CU(cudaFuncSetAttribute(plan_order_kernel<float>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024),
               "cudaFuncSetAttribute");
        configured.insert({dev, 4});
      }
    }
    plan_order_kernel<float><<<(unsigned)grid, 256, smem, (cudaStream_t)stream>>>(
        in_re, in_im, (float*)out_re, (float*)out_im, logL, logR, nlines, scale);
  }
  PAC_LAUNCHED("plan_order");
  return PAC_SUCCESS;
}

int be_round_to_f32(const double* src, float* dst, long long n, void* stream) {
  round_f32_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(src, dst, n);
  PAC_LAUNCHED("round_f32");
  return PAC_SUCCESS;
}

int be_pointwise(long long n, int elem_bytes, const void* xr, const void* xi, const void* hr,
                 const void* hi, long long hmask, void* yr, void* yi, double scale,
                 void* stream) {
  if (elem_bytes == 8)
    pointwise_kernel<double><<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(
        n, (const double*)xr, (const double*)xi, (const double*)hr, (const double*)hi, hmask,
        (double*)yr, (double*)yi, scale);
  else
    pointwise_kernel<float><<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(
        n, (const float*)xr, (const float*)xi, (const float*)hr, (const float*)hi, hmask,
        (float*)yr, (float*)yi, (float)scale);
  PAC_LAUNCHED("pointwise");
  return PAC_SUCCESS;
}

int be_scale_copy(long long n, int elem_bytes, const void* xr, const void* xi, void* yr,
                  void* yi, double scale, void* stream) {
  if (elem_bytes == 8)
    scale_copy_kernel<double><<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(
        n, (const double*)xr, (const double*)xi, (double*)yr, (double*)yi, scale);
  else
    scale_copy_kernel<float><<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(
        n, (const float*)xr, (const float*)xi, (float*)yr, (float*)yi, (float)scale);
  PAC_LAUNCHED("scale_copy");
  return PAC_SUCCESS;
}

int be_permute(long long n, const int* rho, double* re, double* im, void* stream) {
  permute_kernel<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(n, rho, re, im);
  PAC_LAUNCHED("permute");
  return PAC_SUCCESS;
}

long long be_launch_count() { return g_launches.load(); }

// 8 independent FMA chains per thread; the result is stored only if it takes
// a value the chains cannot reach, which keeps them live
template <typename T>
__global__ void __launch_bounds__(256) fma_peak_kernel(T* out, int iters, T a, T b) {
  T x[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) x[k] = T(threadIdx.x + k) * T(1e-3);
#pragma unroll 16
  for (int i = 0; i < iters; ++i) {  // unrolled: loop control is a small share of issue slots
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = fma(x[k], a, b);
  }
  T s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += x[k];
  if (s == T(-1)) out[blockIdx.x] = s;
}

template <typename T>
static int fma_peak_t(cudaStream_t st, double* tflops) {
  const int iters = sizeof(T) == 8 ? 256 : 1024;
  const long long blocks = 8LL * be_num_sms();
  T* out = nullptr;
  PAC_CU(cudaMalloc(&out, sizeof(T) * blocks), "cudaMalloc");
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  double best = 0;
  cudaError_t err = cudaSuccess;
  for (int r = 0; r < 4 && err == cudaSuccess; ++r) {
    cudaEventRecord(e0, st);
    fma_peak_kernel<T><<<(unsigned)blocks, 256, 0, st>>>(out, iters, T(0.999999), T(1e-7));
    cudaEventRecord(e1, st);
    err = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
    const double fl = 2.0 * 8.0 * iters * 256.0 * (double)blocks;
    if (r > 0 && err == cudaSuccess && ms > 0.f) best = std::max(best, fl / (ms * 1e-3) / 1e12);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  PAC_CU(err, "fma_peak_kernel");
  g_launches.fetch_add(4, std::memory_order_relaxed);
  *tflops = best;
  return PAC_SUCCESS;
}

int be_fma_peak(int elem_bytes, void* stream, double* tflops) {
  if (elem_bytes == 8) return fma_peak_t<double>((cudaStream_t)stream, tflops);
  return fma_peak_t<float>((cudaStream_t)stream, tflops);
}

}  // namespace pac
