// pac_coltma.cu -- the column passes staged by tensor copies (ColTma,
// pac_coltma.cuh): the sm_100a kernel, its tensor maps and its launcher.
// A translation unit of its own, beside pac_cuda.cu.
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdio.h>

#include <atomic>
#include <mutex>
#include <set>

#include "pac.h"
#include "pac_backend.h"
#include "pac_special.h"
#include "pac_tma.cuh"

namespace pac {

int set_error(int status, const char* fmt, ...);
void count_launch();

#define PAC_CU(call, what)                                                             \
  do {                                                                                 \
    cudaError_t _e = (call);                                                           \
    if (_e != cudaSuccess)                                                             \
      return set_error(PAC_ERROR_CUDA, "%s: %s", what, cudaGetErrorString(_e));        \
  } while (0)
#define PAC_TRY_BE(expr)                 \
  do {                                   \
    int _st = (expr);                    \
    if (_st != PAC_SUCCESS) return _st;  \
  } while (0)

// A column pass staged by tensor copies (ColTma, pac_coltma.cuh): persistent
// CTAs walk the tiles blockIdx.x, blockIdx.x + gridDim.x, ...  Thread 0
// loads a tile into shared memory (dense rows for DIF, the transposed view
// for DIT), all threads run the stages on it, thread 0 stores it (transposed
// view for DIF, dense rows for DIT) and, once the store has read the buffer,
// loads the next tile.  The wait for a load is bounded: on a timeout the
// CTA reports PAC_ERROR_TIMEOUT in the plan's status word, waits (bounded)
// for the copy in flight to land and leaves.
//
// TC = 1 (the tensor-core form): the radix-16 steps run on the 5th-generation
// tensor cores (ColTma::tc_prep / tc_finish): every warpgroup writes its 128
// butterflies' A rows after the tile, one of its threads issues the MMAs
// into the warpgroup's 32 tensor-memory columns and commits them to the
// warpgroup's mbarrier, and each thread reads its butterfly's row back.
// Warp 0 allocates the tensor memory at the start and frees it at the end.
template <typename T, int B2, int MODE, int SIGN, int LOGL, int LOGW, int NT, int MINB,
          int TC = 0>
__global__ void __launch_bounds__(NT, MINB)
    pac_coltma_kernel(const PassDesc d, const __grid_constant__ CUtensorMap tin_re,
                      const __grid_constant__ CUtensorMap tin_im,
                      const __grid_constant__ CUtensorMap tout_re,
                      const __grid_constant__ CUtensorMap tout_im) {
  using CT = ColTma<T, B2, MODE, SIGN, LOGL, LOGW, NT, TC>;
  constexpr int W = CT::W, TILE = CT::TILE, NS = CT::NS;
  constexpr bool DIF = CT::DIF;
  extern __shared__ unsigned char pac_smem_raw[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ __align__(8) uint64_t tbar[TC ? CT::NWG : 1];
  __shared__ uint32_t tmem_slot;
  T* Bre = reinterpret_cast<T*>(smem_align1024(pac_smem_raw));
  T* Bim = Bre + TILE;
  // tensor-core form: per warpgroup the hi and lo A tiles, then the DFT
  // operand's hi and lo tiles (32-bit words of two halves)
  uint32_t* Aop = reinterpret_cast<uint32_t*>(Bim + TILE);
  uint32_t* Vh = Aop + (TC ? CT::NWG * CT::UTILE : 0);
  uint32_t* Vl = Vh + 512;
  uint32_t tbase = 0, tph = 0;
  const int t = threadIdx.x;
  const long long ntiles = d.nlines >> LOGW;
  auto issue_load = [&](long long tl) {
    int i0, o;
    CT::tile_coords(d, tl, i0, o);
    mbar_arrive_expect_tx(&bar, (uint32_t)(2 * TILE * sizeof(T)));
    if constexpr (DIF) {
      for (int k = 0; k < CT::L / CT::BOXR; ++k) {
        tma_load_3d(Bre + k * CT::BOXR * W, &tin_re, &bar, i0, k * CT::BOXR, o);
        tma_load_3d(Bim + k * CT::BOXR * W, &tin_im, &bar, i0, k * CT::BOXR, o);
      }
    } else {
      for (int k = 0; k < CT::NBLK / CT::BOXB; ++k) {
        tma_load_4d(Bre + k * CT::BOXB * CT::RIN * W, &tin_re, &bar, i0, k * CT::BOXB, 0, o);
        tma_load_4d(Bim + k * CT::BOXB * CT::RIN * W, &tin_im, &bar, i0, k * CT::BOXB, 0, o);
      }
    }
  };
  auto issue_store = [&](long long tl) {
    int i0, o;
    CT::tile_coords(d, tl, i0, o);
    if constexpr (DIF) {
      for (int k = 0; k < CT::NBLK / CT::BOXB; ++k) {
        tma_store_4d(&tout_re, Bre + k * CT::BOXB * CT::RIN * W, i0, k * CT::BOXB, 0, o);
        tma_store_4d(&tout_im, Bim + k * CT::BOXB * CT::RIN * W, i0, k * CT::BOXB, 0, o);
      }
    } else {
      for (int k = 0; k < CT::L / CT::BOXR; ++k) {
        tma_store_3d(&tout_re, Bre + k * CT::BOXR * W, i0, k * CT::BOXR, o);
        tma_store_3d(&tout_im, Bim + k * CT::BOXR * W, i0, k * CT::BOXR, o);
      }
    }
    bulk_commit();
  };
  if (t == 0) {
    mbar_init(&bar, 1);
    if constexpr (TC) {
      for (int g = 0; g < CT::NWG; ++g) mbar_init(&tbar[g], 1);
    }
    fence_barrier_init();
  }
  if constexpr (TC) {
    for (int i = t; i < 512; i += NT) CT::tc_fill_v(i, Vh, Vl);
    fence_proxy_async();  // the operand is read by the tensor cores
    if (t < 32) tmem_alloc(&tmem_slot, 32 * CT::NWG);
    tc5_fence_before();
  }
  __syncthreads();
  if constexpr (TC) {
    tc5_fence_after();
    tbase = tmem_slot;
  }
  long long tile = blockIdx.x;
  if (t == 0 && tile < ntiles) issue_load(tile);
  uint32_t phase = 0;
  Cx<T> x[CT::TPT];
  for (; tile < ntiles; tile += gridDim.x) {
    const bool ok = mbar_wait_bounded(&bar, phase, wait_limit_of(d));
    if (!__syncthreads_and(ok)) {
      if (t == 0) {
        report_timeout(d);
        mbar_wait_bounded(&bar, phase);  // the copy in flight lands first
      }
      break;
    }
    phase ^= 1;
    static_for<NS>([&](auto ss) {
      constexpr int S = ss.value;
      CT::template read<S>(t, Bre, Bim, x);
      if constexpr (CT::tc_step(S)) {
        const int g = t >> 7;
        uint32_t* Ah = Aop + g * CT::UTILE;
        uint32_t* Al = Ah + CT::UTILE / 2;
        static_for<CT::TPW>([&](auto kk) {
          int E = 0;
          CT::template tc_prep<S>(d, t, kk.value, x, Ah, Al, E);
          fence_proxy_async();  // the A rows are read by the tensor cores
          warpgroup_sync(g);
          if ((t & 127) == 0) {
            tc5_fence_after();
            const uint32_t idesc = umma_idesc_f16(CT::UM, CT::UN);
            // Xlo.Vhi + Xhi.Vlo + Xhi.Vhi (small products first), K = 32 in
            // two steps of 16
#pragma unroll
            for (int pr = 0; pr < 3; ++pr) {
              const uint32_t* A = pr == 0 ? Al : Ah;
              const uint32_t* B = pr == 1 ? Vl : Vh;
#pragma unroll
              for (int ks = 0; ks < 2; ++ks)
                umma_f16(tbase + 32 * g, umma_desc((const char*)A + 256 * ks, 128, 512),
                         umma_desc((const char*)B + 256 * ks, 128, 512), idesc,
                         (pr | ks) != 0);
            }
            umma_commit(&tbar[g]);
          }
          if (!mbar_wait_bounded(&tbar[g], tph)) report_timeout(d);
          tph ^= 1;
          tc5_fence_after();
          float D[32];
          tmem_ld32(tbase + ((uint32_t)(32 * ((t >> 5) & 3)) << 16) + 32 * g, D);
          CT::template tc_finish<S>(d, t, kk.value, D, E, x);
          tc5_fence_before();
        });
      } else {
        CT::template compute<S>(d, tile, t, x);
      }
      if constexpr (CT::split_step(S)) __syncthreads();
      CT::template write<S>(d, t, Bre, Bim, x);
      if constexpr (S == NS - 1) fence_proxy_async();  // visible to the tensor store
      __syncthreads();
    });
    if (t == 0) {
      issue_store(tile);
      bulk_wait_read();  // the buffer is free again
      if (tile + gridDim.x < ntiles) issue_load(tile + gridDim.x);
    }
  }
  if (t == 0) bulk_wait_all();
  if constexpr (TC) {
    tc5_fence_before();
    __syncthreads();
    if (t < 32) {
      tc5_fence_after();
      tmem_dealloc(tbase, 32 * CT::NWG);
    }
  }
}

// The pipelined variant: the tile lives in registers while it computes, so
// the tile buffer A is free as soon as every thread has read its first
// stage's inputs, and thread 0 issues the next tile's tensor load right
// then -- the load runs under this tile's arithmetic.  The stages exchange
// through X, a buffer of one component in the swizzled layout (real parts,
// then imaginary parts), and each component of the result leaves by a
// tensor store from X (transposed view for DIF, dense rows for DIT).  With
// GST the result leaves the registers by plain stores instead (ColTma::
// store_g), so the tensor-copy unit carries only the loads and the last step
// needs no exchange.  Shared memory: A (both components) + X.  Waits bounded
// as above.
template <typename T, int B2, int MODE, int SIGN, int LOGL, int LOGW, int NT, int MINB,
          bool GST>
__global__ void __launch_bounds__(NT, MINB)
    pac_coltma_pipe_kernel(const PassDesc d, const __grid_constant__ CUtensorMap tin_re,
                           const __grid_constant__ CUtensorMap tin_im,
                           const __grid_constant__ CUtensorMap tout_re,
                           const __grid_constant__ CUtensorMap tout_im) {
  using CT = ColTma<T, B2, MODE, SIGN, LOGL, LOGW, NT>;
  constexpr int W = CT::W, TILE = CT::TILE, NS = CT::NS;
  constexpr bool DIF = CT::DIF;
  constexpr int LOUT = DIF ? LAY_TRANS : LAY_DENSE;
  extern __shared__ unsigned char pac_smem_raw[];
  __shared__ __align__(8) uint64_t bar;
  T* Are = reinterpret_cast<T*>(smem_align1024(pac_smem_raw));
  T* Aim = Are + TILE;
  T* X = Aim + TILE;
  Cx<T>* tws = reinterpret_cast<Cx<T>*>(X + TILE);  // the stage twiddles (CT::TWSM)
  const int t = threadIdx.x;
  const long long ntiles = d.nlines >> LOGW;
  auto issue_load = [&](long long tl) {
    int i0, o;
    CT::tile_coords(d, tl, i0, o);
    mbar_arrive_expect_tx(&bar, (uint32_t)(2 * TILE * sizeof(T)));
    if constexpr (DIF) {
      for (int k = 0; k < CT::L / CT::BOXR; ++k) {
        tma_load_3d(Are + k * CT::BOXR * W, &tin_re, &bar, i0, k * CT::BOXR, o);
        tma_load_3d(Aim + k * CT::BOXR * W, &tin_im, &bar, i0, k * CT::BOXR, o);
      }
    } else {
      for (int k = 0; k < CT::NBLK / CT::BOXB; ++k) {
        tma_load_4d(Are + k * CT::BOXB * CT::RIN * W, &tin_re, &bar, i0, k * CT::BOXB, 0, o);
        tma_load_4d(Aim + k * CT::BOXB * CT::RIN * W, &tin_im, &bar, i0, k * CT::BOXB, 0, o);
      }
    }
  };
  auto issue_store = [&](const CUtensorMap* map, long long tl) {
    int i0, o;
    CT::tile_coords(d, tl, i0, o);
    if constexpr (DIF) {
      for (int k = 0; k < CT::NBLK / CT::BOXB; ++k)
        tma_store_4d(map, X + k * CT::BOXB * CT::RIN * W, i0, k * CT::BOXB, 0, o);
    } else {
      for (int k = 0; k < CT::L / CT::BOXR; ++k)
        tma_store_3d(map, X + k * CT::BOXR * W, i0, k * CT::BOXR, o);
    }
    bulk_commit();
  };
  if (t == 0) {
    mbar_init(&bar, 1);
    fence_barrier_init();
  }
  CT::tw_fill(d, t, tws);
  __syncthreads();
  long long tile = blockIdx.x;
  if (t == 0 && tile < ntiles) issue_load(tile);
  uint32_t phase = 0;
  Cx<T> x[CT::TPT];
  for (; tile < ntiles; tile += gridDim.x) {
    const bool ok = mbar_wait_bounded(&bar, phase, wait_limit_of(d));
    if (!__syncthreads_and(ok)) {
      if (t == 0) {
        report_timeout(d);
        mbar_wait_bounded(&bar, phase);  // the copy in flight lands first
      }
      break;
    }
    phase ^= 1;
    CT::template read<0>(t, Are, Aim, x);
    fence_proxy_async();  // these reads precede the next tensor load into A
    __syncthreads();      // A is free; X too (thread 0 waited for the last store)
    if (t == 0 && tile + gridDim.x < ntiles) issue_load(tile + gridDim.x);
    static_for<NS>([&](auto ss) {
      constexpr int S = ss.value;
      CT::template compute<S>(d, tile, t, x, tws);
      if constexpr (S < NS - 1) {
        CT::template write_c<S, 0, LAY_SWZ>(d, t, X, x);
        __syncthreads();
        CT::template read_c<S + 1, 0, LAY_SWZ>(t, X, x);
        __syncthreads();
        CT::template write_c<S, 1, LAY_SWZ>(d, t, X, x);
        __syncthreads();
        CT::template read_c<S + 1, 1, LAY_SWZ>(t, X, x);
        __syncthreads();
      }
    });
    if constexpr (GST) {
      CT::template store_g<NS - 1>(d, tile, t, x);
    } else {
      CT::template write_c<NS - 1, 0, LOUT>(d, t, X, x);
      fence_proxy_async();
      __syncthreads();
      if (t == 0) {
        issue_store(&tout_re, tile);
        bulk_wait_read();
      }
      __syncthreads();
      CT::template write_c<NS - 1, 1, LOUT>(d, t, X, x);
      fence_proxy_async();
      __syncthreads();
      if (t == 0) {
        issue_store(&tout_im, tile);
        bulk_wait_read();
      }
    }
  }
  if (t == 0) bulk_wait_all();
}

// Tensor maps of a ColTma pass over the row array [O][L][S] of one
// component: the dense rows (3D {S, L, O}, boxes of W x boxr rows) and the
// transposed view (4D {S, L/R, R, O}: row e = blk * R + m, boxes of W x boxb
// blocks x R) that lands as [m][blk][w].  Unswizzled; plain copies.
static int coltma_map(CUtensorMap* m, const void* base, int esz, const PassDesc& d, int W,
                      int boxr, bool trans, int vin, int boxb) {
  auto enc = tensor_map_encoder();
  if (!enc) return set_error(PAC_ERROR_CUDA, "cuTensorMapEncodeTiled unavailable");
  const cuuint64_t S = 1ull << d.logS, L = 1ull << d.logL, R = 1ull << vin;
  const cuuint64_t O = (cuuint64_t)(d.nlines >> d.logS);
  const CUtensorMapDataType ty =
      esz == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  CUresult r;
  if (!trans) {
    cuuint64_t dims[3] = {S, L, O};
    cuuint64_t strides[2] = {S * esz, S * L * esz};
    cuuint32_t box[3] = {(cuuint32_t)W, (cuuint32_t)boxr, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    r = enc(m, ty, 3, const_cast<void*>(base), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  } else {
    cuuint64_t dims[4] = {S, L / R, R, O};
    cuuint64_t strides[3] = {S * R * esz, S * esz, S * L * esz};
    cuuint32_t box[4] = {(cuuint32_t)W, (cuuint32_t)boxb, (cuuint32_t)R, 1};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    r = enc(m, ty, 4, const_cast<void*>(base), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  }
  if (r != CUDA_SUCCESS)
    return set_error(PAC_ERROR_CUDA, "cuTensorMapEncodeTiled (%s view) failed (%d)",
                     trans ? "transposed" : "dense", (int)r);
  return PAC_SUCCESS;
}

int launch_coltma(const PassDesc& d, int elem_bytes, int b2, long long grid, int threads,
                         size_t smem, void* stream) {
  int seen = 0;  // candidates of this geometry so far; d.tma - 1 picks one
#define PAC_X(T, BY, B2_, MO, SG, LL, LW, NT_, MB, PP, DF, TC_)                                   \
  if (elem_bytes == BY && b2 == B2_ && d.mode == MO && d.sign == SG && d.logL == LL &&     \
      d.tc == TC_ && seen++ == d.tma - 1) {                                                \
    using CT = ColTma<T, B2_, MO, SG, LL, LW, NT_>;                                        \
    if (d.W != (1 << LW) || threads != NT_)                                                \
      return set_error(PAC_ERROR_INTERNAL, "tensor-copy column pass geometry mismatch");   \
    static std::mutex mu;                                                                  \
    static std::set<int> configured;                                                       \
    /* the pipelined kernel keeps a copy of the stage twiddles after its buffers */        \
    const size_t sm = smem + (PP ? (size_t)CT::TWSM * 2 * sizeof(T) : 0);                  \
    auto kern = PP ? pac_coltma_pipe_kernel<T, B2_, MO, SG, LL, LW, NT_, MB, PP == 2>      \
                   : pac_coltma_kernel<T, B2_, MO, SG, LL, LW, NT_, MB, TC_>;              \
    CUtensorMap m[4];                                                                      \
    const bool tin = MO == MODE_DIT, tout = MO == MODE_DIF;                                \
    PAC_TRY_BE(coltma_map(&m[0], d.in_re, BY, d, CT::W, CT::BOXR, tin, CT::VIN, CT::BOXB)); \
    PAC_TRY_BE(coltma_map(&m[1], d.in_im, BY, d, CT::W, CT::BOXR, tin, CT::VIN, CT::BOXB)); \
    PAC_TRY_BE(coltma_map(&m[2], d.out_re, BY, d, CT::W, CT::BOXR, tout, CT::VIN, CT::BOXB)); \
    PAC_TRY_BE(coltma_map(&m[3], d.out_im, BY, d, CT::W, CT::BOXR, tout, CT::VIN, CT::BOXB)); \
    {                                                                                      \
      int dev = 0;                                                                         \
      PAC_CU(cudaGetDevice(&dev), "cudaGetDevice");                                        \
      std::lock_guard<std::mutex> g(mu);                                                   \
      if (!configured.count(dev)) {                                                        \
        PAC_CU(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,     \
                                    (int)sm),                                              \
               "cudaFuncSetAttribute");                                                    \
        configured.insert(dev);                                                            \
      }                                                                                    \
    }                                                                                      \
    if (grid > 0x7fffffffLL) return set_error(PAC_ERROR_SIZE, "pass grid too large");      \
    kern<<<(unsigned)grid, threads, sm, (cudaStream_t)stream>>>(d, m[0], m[1], m[2], m[3]); \
    PAC_CU(cudaGetLastError(), "pac_coltma_kernel launch");                                \
    count_launch();                                    \
    return PAC_SUCCESS;                                                                    \
  }
  PAC_COLTMA_LIST(PAC_X)
#undef PAC_X
  return set_error(PAC_ERROR_INTERNAL, "no tensor-copy kernel for a pass marked so");
}

}  // namespace pac
