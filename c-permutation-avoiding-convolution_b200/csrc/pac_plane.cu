// pac_plane.cu -- the plane pass of 3D convolutions (pac_plane.cuh): the
// sm_100a cluster kernel and its launcher.  A translation unit of its own,
// beside pac_cuda.cu.
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdio.h>

#include <mutex>
#include <set>

#include "pac.h"
#include "pac_backend.h"
#include "pac_special.h"

namespace cg = cooperative_groups;

namespace pac {

int set_error(int status, const char* fmt, ...);
void count_launch();

// One cluster of 2^LOGC CTAs per plane (grid = planes x 2^LOGC, cluster
// shape (2^LOGC, 1, 1)): CTA `rank` holds rows [rank * RC, (rank + 1) * RC)
// of plane blockIdx.x >> LOGC.  The first cluster barrier also guarantees
// that every CTA of the cluster runs before any distributed shared-memory
// access; the last keeps each CTA's rows alive while its peers read them.
template <typename T, int B2, int LOGN1, int LOGN2, int LOGC, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) pac_plane_kernel(const PassDesc d) {
  using G = PlaneGeo<T, B2, LOGN1, LOGN2, LOGC, NT>;
  extern __shared__ __align__(16) unsigned char pac_smem[];
  __shared__ long long s_lb[G::RC];
  T* sre = reinterpret_cast<T*>(pac_smem);
  T* sim = sre + (size_t)G::RC * G::P2;
  cg::cluster_group cl = cg::this_cluster();
  ClView<T, G::C> cv;
  cv.rank = (int)cl.block_rank();
#pragma unroll
  for (int r = 0; r < G::C; ++r) {
    cv.re[r] = cl.map_shared_rank(sre, r);
    cv.im[r] = cl.map_shared_rank(sim, r);
  }
  const long long plane = (long long)(blockIdx.x >> LOGC);
  for (int r = threadIdx.x; r < G::RC; r += NT)
    s_lb[r] = (plane << (LOGN1 + LOGN2)) + ((long long)(cv.rank * G::RC + r) << LOGN2);
  cl.sync();
  plane_body<T, B2, LOGN1, LOGN2, LOGC, NT>(d, plane, sre, sim, cv, s_lb, 0);
  cl.sync();
  plane_body<T, B2, LOGN1, LOGN2, LOGC, NT>(d, plane, sre, sim, cv, s_lb, 1);
  cl.sync();
  plane_body<T, B2, LOGN1, LOGN2, LOGC, NT>(d, plane, sre, sim, cv, s_lb, 2);
  cl.sync();
}

// grid = planes x 2^logC CTAs, launched with a cluster shape of (2^logC, 1, 1)
int launch_plane(const PassDesc& d, int elem_bytes, int b2, long long grid, int threads,
                 size_t smem, void* stream) {
#define PAC_X(T, BY, B2_, L1, L2, LC, NT_, MB)                                              \
  if (elem_bytes == BY && b2 == B2_ && d.plane_logN1 == L1 && d.plane_logN2 == L2 &&      \
      threads == NT_) {                                                                   \
    static std::mutex mu;                                                                 \
    static std::set<int> configured;                                                      \
    auto kern = pac_plane_kernel<T, B2_, L1, L2, LC, NT_, MB>;                            \
    if (smem > 48 * 1024) {                                                               \
      int dev = 0;                                                                        \
      cudaError_t e = cudaGetDevice(&dev);                                                \
      std::lock_guard<std::mutex> g(mu);                                                  \
      if (e == cudaSuccess && !configured.count(dev)) {                                   \
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,       \
                                 (int)smem);                                              \
        if (e == cudaSuccess) configured.insert(dev);                                     \
      }                                                                                   \
      if (e != cudaSuccess)                                                               \
        return set_error(PAC_ERROR_CUDA, "plane kernel set-up: %s", cudaGetErrorString(e)); \
    }                                                                                     \
    if (grid > 0x7fffffffLL || (grid & ((1LL << LC) - 1)) != 0)                           \
      return set_error(PAC_ERROR_INTERNAL, "plane pass grid %lld", grid);                 \
    cudaLaunchConfig_t cfg = {};                                                          \
    cfg.gridDim = dim3((unsigned)grid);                                                   \
    cfg.blockDim = dim3((unsigned)threads);                                               \
    cfg.dynamicSmemBytes = smem;                                                          \
    cfg.stream = (cudaStream_t)stream;                                                    \
    cudaLaunchAttribute at[1];                                                            \
    at[0].id = cudaLaunchAttributeClusterDimension;                                       \
    at[0].val.clusterDim.x = 1u << LC;                                                    \
    at[0].val.clusterDim.y = 1;                                                           \
    at[0].val.clusterDim.z = 1;                                                           \
    cfg.attrs = at;                                                                       \
    cfg.numAttrs = 1;                                                                     \
    cudaError_t e = cudaLaunchKernelEx(&cfg, kern, d);                                    \
    if (e != cudaSuccess)                                                                 \
      return set_error(PAC_ERROR_CUDA, "pac_plane_kernel launch: %s", cudaGetErrorString(e)); \
    count_launch();                                                                       \
    return PAC_SUCCESS;                                                                   \
  }
  PAC_PLANE_LIST(PAC_X)
#undef PAC_X
  return set_error(PAC_ERROR_INTERNAL, "no plane kernel for a pass marked plane");
}

}  // namespace pac
