// pac_emu.cpp -- TEST-ONLY host implementation of the backend interface.
//
// Built only into libpac_emu.so, which only tests/ load.  The product
// library (libpac.so) never contains this file and has no host fallback.
//
// "Device" memory is host memory and a pass is replayed CTA by CTA, phase by
// phase, through the same pass_body<T, B2> the sm_100a kernel runs, so the
// plan layer, the pass geometry and the kernels' index arithmetic can be
// checked against the oracle on a machine without a GPU.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <limits>
#include <chrono>
#include <vector>

#include "pac.h"
#include "pac_backend.h"
#include "pac_special.h"

namespace pac {

int set_error(int status, const char* fmt, ...);
static std::atomic<long long> g_launches{0};

int be_init() { return PAC_SUCCESS; }
// a few "SMs", so that persistent kernels replay CTAs that walk several tiles
int be_num_sms() { return 3; }

int be_malloc(void** p, size_t bytes) {
  *p = aligned_alloc(256, ((bytes ? bytes : 16) + 255) / 256 * 256);
  if (!*p) return set_error(PAC_ERROR_ALLOC, "host allocation failed");
  return PAC_SUCCESS;
}
int be_free(void* p) {
  free(p);
  return PAC_SUCCESS;
}
int be_memcpy(void* dst, const void* src, size_t bytes, int, void*) {
  if (bytes && dst != src) memmove(dst, src, bytes);
  return PAC_SUCCESS;
}
int be_memset(void* dst, int value, size_t bytes, void*) {
  memset(dst, value, bytes);
  return PAC_SUCCESS;
}
int be_stream_create(void** s) {
  *s = nullptr;
  return PAC_SUCCESS;
}
int be_stream_destroy(void*) { return PAC_SUCCESS; }
int be_stream_sync(void*) { return PAC_SUCCESS; }
int be_stream_wait(void*, void*) { return PAC_SUCCESS; }
int be_l2_persist(void*, const void*, size_t) { return PAC_SUCCESS; }
long long be_l2_bytes() { return 0; }
// events: host clock readings (the replay runs synchronously, so two
// readings bracket the work issued between them)
int be_event_create(void** ev) {
  *ev = new double(0.0);
  return PAC_SUCCESS;
}
int be_event_destroy(void* ev) {
  delete (double*)ev;
  return PAC_SUCCESS;
}
int be_event_record(void* ev, void*) {
  if (ev)
    *(double*)ev = std::chrono::duration<double, std::milli>(
                       std::chrono::steady_clock::now().time_since_epoch())
                       .count();
  return PAC_SUCCESS;
}
int be_event_elapsed(void* a, void* b, float* ms) {
  *ms = (a && b) ? (float)(*(double*)b - *(double*)a) : 0.f;
  return PAC_SUCCESS;
}
int be_device_name(char* buf, int n) {
  snprintf(buf, (size_t)n, "host replay");
  return PAC_SUCCESS;
}

template <typename T, int B2, int TC = 0>
static void replay(const PassDesc& d, long long grid) {
  std::vector<T> sm((size_t)2 * d.W * d.pitch);
  std::vector<long long> lb(128);
  for (long long cta = 0; cta < grid; ++cta) {
    for (int w = 0; w < d.W; ++w) {
      long long g = cta * d.W + w;
      if (d.nat) nat_line<B2>(d, g, &lb[w], &lb[64 + w]);
      else lb[w] = lb[64 + w] = line_base(d, g);
    }
    pass_body<T, B2, TC>(d, cta, sm.data(), sm.data() + (size_t)d.W * d.pitch, lb.data(),
                         lb.data() + 64);
  }
}

// replay of a specialised kernel (pac_special.h): the compile-time body
template <typename T, int B2, int MODE, int SIGN, int LOGL, int COLS, int LOGW, int NT, int TC,
          int RC>
static void replay_special(const PassDesc& d, long long grid) {
  constexpr int W = 1 << LOGW;
  constexpr int PITCH = pitch_for((int)sizeof(T), LOGL, W, COLS, TC);
  using SP = Shape<LOGL, LOGW, PITCH, COLS, TC>;
  std::vector<T> sm((size_t)2 * W * PITCH);
  std::vector<long long> lb(W);
  for (long long cta = 0; cta < grid; ++cta) {
    for (int w = 0; w < W; ++w) lb[w] = line_base(d, cta * W + w);
    pass_body_ct<T, B2, MODE, SIGN, SP, NT, RadsCap<LOGL, B2, RC>, TC>(
        d, cta, sm.data(), sm.data() + (size_t)W * PITCH, lb.data(), lb.data());
  }
}

// The replay models a tensor copy as landing kCopyCycles SM cycles after it
// is issued: a pass whose wait limit is below that gives up on its first
// tile in every CTA, as on the device -- it reports PAC_ERROR_TIMEOUT in the
// plan's status word and writes no output.
static const long long kCopyCycles = 1000;
static bool copy_wait_gives_up(const PassDesc& d) {
  if (d.wait_limit <= 0 || d.wait_limit >= kCopyCycles) return false;
  if (d.status) *d.status = PAC_ERROR_TIMEOUT;
  return true;
}

// replay of a pipelined column kernel: the CTAs of the persistent launch
// visit their tiles in order; the tensor copy becomes a plain copy of the
// tile into the dense buffer, and each step between two barriers runs for
// every thread in turn, with the per-thread registers kept in an array.
// The exchange array starts every tile as NaN.
template <typename T, int B2, int MODE, int SIGN, int LOGL, int LOGW, int NT>
static void replay_pipe(const PassDesc& d, long long grid) {
  using CP = ColPipe<T, B2, MODE, SIGN, LOGL, LOGW, NT>;
  constexpr int W = CP::W, L = CP::L, NS = CP::NS;
  if (copy_wait_gives_up(d)) return;
  struct Regs {
    Cx<T> v[CP::TPT];
  };
  std::vector<T> A((size_t)2 * W * L), X((size_t)W * CP::PITCH);
  std::vector<Regs> xs(NT);
  std::vector<long long> lb(W);
  const T* ire = (const T*)d.in_re;
  const T* iim = (const T*)d.in_im;
  const long long ntiles = d.nlines >> LOGW;
  auto each = [&](auto&& f) {
    for (int t = 0; t < NT; ++t) f(t, xs[t].v);
  };
  for (long long c = 0; c < grid; ++c)
    for (long long tile = c; tile < ntiles; tile += grid) {
      for (int w = 0; w < W; ++w) lb[w] = line_base(d, tile * W + w);
      for (int e = 0; e < L; ++e)
        for (int w = 0; w < W; ++w) {
          const long long gi = lb[w] + ((long long)e << d.logS);
          A[(size_t)e * W + w] = ire[gi];
          A[(size_t)W * L + (size_t)e * W + w] = iim[gi];
        }
      std::fill(X.begin(), X.end(), std::numeric_limits<T>::quiet_NaN());
      each([&](int t, Cx<T>(&x)[CP::TPT]) { CP::load_tile(t, A.data(), A.data() + W * L, x); });
      if constexpr (MODE == MODE_DIT) {
        each([&](int t, Cx<T>(&x)[CP::TPT]) { CP::template xw<-1, 0>(t, X.data(), x); });
        each([&](int t, Cx<T>(&x)[CP::TPT]) { CP::template xr<-1, 0>(t, X.data(), x); });
        each([&](int t, Cx<T>(&x)[CP::TPT]) { CP::template xw<-1, 1>(t, X.data(), x); });
        each([&](int t, Cx<T>(&x)[CP::TPT]) { CP::template xr<-1, 1>(t, X.data(), x); });
      }
      static_for<NS>([&](auto ss) {
        constexpr int S = ss.value;
        if constexpr (S > 0) {
          each([&](int t, Cx<T>(&x)[CP::TPT]) { CP::template xw<S - 1, 0>(t, X.data(), x); });
          each([&](int t, Cx<T>(&x)[CP::TPT]) { CP::template xr<S - 1, 0>(t, X.data(), x); });
          each([&](int t, Cx<T>(&x)[CP::TPT]) { CP::template xw<S - 1, 1>(t, X.data(), x); });
          each([&](int t, Cx<T>(&x)[CP::TPT]) { CP::template xr<S - 1, 1>(t, X.data(), x); });
        }
        each([&](int t, Cx<T>(&x)[CP::TPT]) { CP::template compute<S>(d, tile, t, x); });
      });
      each([&](int t, Cx<T>(&x)[CP::TPT]) { CP::store(d, t, lb.data(), x); });
    }
}

// replay of a cluster column kernel: each tile's C CTAs get their own
// shared-memory image; every phase of pass_body_cl runs for all C ranks
// before the next one starts, as the cluster barriers order them on the
// device.  The images start as NaN so that a read of an element no stage
// wrote shows up in the results.
template <typename T, int B2, int MODE, int SIGN, int LOGL, int LOGW, int LOGC, int NT>
static void replay_cluster(const PassDesc& d, long long grid) {
  constexpr int C = 1 << LOGC, W = 1 << LOGW;
  constexpr int PITCH = pitch_for((int)sizeof(T), LOGL - LOGC, W);
  using SP = Shape<LOGL, LOGW, PITCH, 1>;
  const size_t per = (size_t)2 * W * PITCH;
  std::vector<T> sm(per * C);
  std::vector<long long> lb(W);
  ClView<T, C> cv;
  for (int r = 0; r < C; ++r) {
    cv.re[r] = sm.data() + per * r;
    cv.im[r] = cv.re[r] + (size_t)W * PITCH;
  }
  for (long long cta = 0; cta < (grid >> LOGC); ++cta) {
    std::fill(sm.begin(), sm.end(), std::numeric_limits<T>::quiet_NaN());
    for (int w = 0; w < W; ++w) lb[w] = line_base(d, cta * W + w);
    for (int phase = 0; phase < 2; ++phase)
      for (int r = 0; r < C; ++r) {
        cv.rank = r;
        pass_body_cl<T, B2, MODE, SIGN, SP, NT, RadsFor<LOGL, B2>, LOGC>(
            d, cta, cv.re[r], cv.im[r], cv, lb.data(), phase);
      }
  }
}

// replay of a tensor-copy column kernel (ColTma): the CTAs of the
// persistent launch visit their tiles in order; the tensor load and store
// become plain copies through the same layout maps (dense rows or the
// transposed view), and every step runs its reads, its arithmetic and its
// writes for all threads in turn -- the order the kernel's barriers impose.
// The buffer starts every tile as NaN, so a read of a slot that no copy or
// stage wrote shows up in the results.
// Host model of the tensor-core step's MMA for one warpgroup: D = Xlo.Vhi +
// Xhi.Vlo + Xhi.Vhi over the operand tiles (FP16 halves in the K-major core-
// matrix layout), each product summed over K in FP64 and the three sums
// added in FP32 in that order.
template <class CT>
static void tc_mma_warpgroup(const uint32_t* Ah, const uint32_t* Al, const uint32_t* Vh,
                             const uint32_t* Vl, float (*D)[32]) {
  auto half = [](const uint32_t* m, int row, int k) {
    const uint32_t w = m[CT::umma_off(row, k) >> 1];
    float lo, hi;
    tc_unpack(w, lo, hi);
    return (k & 1) ? hi : lo;
  };
  for (int r = 0; r < CT::UM; ++r)
    for (int n = 0; n < CT::UN; ++n) {
      double p[3] = {0.0, 0.0, 0.0};
      for (int k = 0; k < CT::UK; ++k) {
        const double ah = half(Ah, r, k), al = half(Al, r, k);
        const double vh = half(Vh, n, k), vl = half(Vl, n, k);
        p[0] += al * vh;
        p[1] += ah * vl;
        p[2] += ah * vh;
      }
      D[r][n] = ((float)p[0] + (float)p[1]) + (float)p[2];
    }
}

template <typename T, int B2, int MODE, int SIGN, int LOGL, int LOGW, int NT, int PIPE, int TC>
static int replay_coltma(const PassDesc& d, long long grid) {
  using CT = ColTma<T, B2, MODE, SIGN, LOGL, LOGW, NT, TC>;
  constexpr int W = CT::W, L = CT::L, NS = CT::NS, TILE = CT::TILE;
  if (copy_wait_gives_up(d)) return PAC_SUCCESS;
  struct Regs {
    Cx<T> v[CT::TPT];
  };
  std::vector<T> B((size_t)2 * TILE);
  std::vector<Regs> xs(NT);
  T* Bre = B.data();
  T* Bim = B.data() + TILE;
  const T* ire = (const T*)d.in_re;
  const T* iim = (const T*)d.in_im;
  T* ore = (T*)d.out_re;
  T* oim = (T*)d.out_im;
  const long long S = 1LL << d.logS;
  const long long ntiles = d.nlines >> LOGW;
  auto each = [&](auto&& f) {
    for (int t = 0; t < NT; ++t) f(t, xs[t].v);
  };
  // every layout map is a bijection of the tile onto [0, TILE)
  {
    std::vector<char> seen(3 * TILE, 0);
    for (int e = 0; e < L; ++e)
      for (int w = 0; w < W; ++w) {
        const int q[3] = {CT::template pos<LAY_DENSE>(e, w), CT::template pos<LAY_TRANS>(e, w),
                          CT::template pos<LAY_SWZ>(e, w)};
        for (int k = 0; k < 3; ++k) {
          if (q[k] < 0 || q[k] >= TILE || seen[k * TILE + q[k]]++)
            return set_error(PAC_ERROR_INTERNAL, "tensor-copy layout %d is not a bijection", k);
        }
      }
  }
  if (d.nlines % W || (1LL << d.logS) % W)
    return set_error(PAC_ERROR_INTERNAL, "tensor-copy tiles do not cover the lines");
  for (long long c = 0; c < grid; ++c)
    for (long long tile = c; tile < ntiles; tile += grid) {
      int i0, o;
      CT::tile_coords(d, tile, i0, o);
      const long long base = (long long)o * L * S + i0;
      std::fill(B.begin(), B.end(), std::numeric_limits<T>::quiet_NaN());
      for (int e = 0; e < L; ++e)
        for (int w = 0; w < W; ++w) {
          const int q = CT::DIF ? CT::template pos<LAY_DENSE>(e, w)
                                : CT::template pos<LAY_TRANS>(e, w);
          Bre[q] = ire[base + e * S + w];
          Bim[q] = iim[base + e * S + w];
        }
      if constexpr (PIPE) {
        // registers between the steps, one-component exchanges through X,
        // the result written into X component by component for the stores
        constexpr int LOUT = CT::DIF ? LAY_TRANS : LAY_DENSE;
        std::vector<T> X((size_t)TILE, std::numeric_limits<T>::quiet_NaN());
        const T qn = std::numeric_limits<T>::quiet_NaN();
        std::vector<Cx<T>> tws((size_t)CT::TWSM + 1, Cx<T>{qn, qn});
        for (int t = 0; t < NT; ++t) CT::tw_fill(d, t, tws.data());
        each([&](int t, Cx<T>(&x)[CT::TPT]) { CT::template read<0>(t, Bre, Bim, x); });
        std::fill(B.begin(), B.end(), std::numeric_limits<T>::quiet_NaN());
        static_for<NS>([&](auto ss) {
          constexpr int St = ss.value;
          each([&](int t, Cx<T>(&x)[CT::TPT]) { CT::template compute<St>(d, tile, t, x, tws.data()); });
          if constexpr (St < NS - 1) {
            each([&](int t, Cx<T>(&x)[CT::TPT]) { CT::template write_c<St, 0, LAY_SWZ>(d, t, X.data(), x); });
            each([&](int t, Cx<T>(&x)[CT::TPT]) { CT::template read_c<St + 1, 0, LAY_SWZ>(t, X.data(), x); });
            each([&](int t, Cx<T>(&x)[CT::TPT]) { CT::template write_c<St, 1, LAY_SWZ>(d, t, X.data(), x); });
            each([&](int t, Cx<T>(&x)[CT::TPT]) { CT::template read_c<St + 1, 1, LAY_SWZ>(t, X.data(), x); });
          }
        });
        if constexpr (PIPE == 2) {
          each([&](int t, Cx<T>(&x)[CT::TPT]) { CT::template store_g<NS - 1>(d, tile, t, x); });
          continue;
        }
        each([&](int t, Cx<T>(&x)[CT::TPT]) { CT::template write_c<NS - 1, 0, LOUT>(d, t, Bre, x); });
        each([&](int t, Cx<T>(&x)[CT::TPT]) { CT::template write_c<NS - 1, 1, LOUT>(d, t, Bim, x); });
      } else {
        static_for<NS>([&](auto ss) {
          constexpr int St = ss.value;
          each([&](int t, Cx<T>(&x)[CT::TPT]) { CT::template read<St>(t, Bre, Bim, x); });
          if constexpr (CT::tc_step(St)) {
            // per warpgroup: every thread's A rows, the MMA, every thread's
            // D row -- round by round
            constexpr int NWG = CT::NWG;
            std::vector<uint32_t> A((size_t)NWG * CT::UTILE), V(1024);
            for (int i = 0; i < 512; ++i) CT::tc_fill_v(i, V.data(), V.data() + 512);
            std::vector<int> E(NT);
            std::vector<float> D((size_t)NWG * CT::UM * 32);
            static_for<CT::TPW>([&](auto kk) {
              std::fill(A.begin(), A.end(), 0xffffffffu);  // NaN halves
              each([&](int t, Cx<T>(&x)[CT::TPT]) {
                uint32_t* Ah = A.data() + (size_t)(t >> 7) * CT::UTILE;
                CT::template tc_prep<St>(d, t, kk.value, x, Ah, Ah + CT::UTILE / 2, E[t]);
              });
              for (int g = 0; g < NWG; ++g) {
                const uint32_t* Ah = A.data() + (size_t)g * CT::UTILE;
                tc_mma_warpgroup<CT>(Ah, Ah + CT::UTILE / 2, V.data(), V.data() + 512,
                                     (float(*)[32])(D.data() + (size_t)g * CT::UM * 32));
              }
              each([&](int t, Cx<T>(&x)[CT::TPT]) {
                float row[32];
                for (int c = 0; c < 32; ++c) row[c] = D[(size_t)t * 32 + c];
                CT::template tc_finish<St>(d, t, kk.value, row, E[t], x);
              });
            });
          } else {
            each([&](int t, Cx<T>(&x)[CT::TPT]) { CT::template compute<St>(d, tile, t, x); });
          }
          each([&](int t, Cx<T>(&x)[CT::TPT]) { CT::template write<St>(d, t, Bre, Bim, x); });
        });
      }
      for (int e = 0; e < L; ++e)
        for (int w = 0; w < W; ++w) {
          const int q = CT::DIF ? CT::template pos<LAY_TRANS>(e, w)
                                : CT::template pos<LAY_DENSE>(e, w);
          ore[base + e * S + w] = Bre[q];
          oim[base + e * S + w] = Bim[q];
        }
    }
  return PAC_SUCCESS;
}

// replay of a plane pass (pac_plane.cuh): each cluster's CTAs get their own
// shared-memory image (NaN at the start, so that a read of a slot no stage
// wrote shows up in the results); every phase runs for all ranks of the
// cluster before the next one starts, as the cluster barriers order them.
template <typename T, int B2, int L1, int L2, int LC, int NT>
static int replay_plane(const PassDesc& d, long long grid) {
  using G = PlaneGeo<T, B2, L1, L2, LC, NT>;
  constexpr int C = G::C;
  const size_t per = (size_t)2 * G::RC * G::P2;
  std::vector<T> sm(per * C);
  std::vector<long long> lb((size_t)G::RC * C);
  ClView<T, C> cv;
  for (int r = 0; r < C; ++r) {
    cv.re[r] = sm.data() + per * r;
    cv.im[r] = cv.re[r] + (size_t)G::RC * G::P2;
  }
  if (grid % C) return set_error(PAC_ERROR_INTERNAL, "plane pass grid %lld", grid);
  for (long long plane = 0; plane < grid / C; ++plane) {
    std::fill(sm.begin(), sm.end(), std::numeric_limits<T>::quiet_NaN());
    for (int r = 0; r < C; ++r)
      for (int i = 0; i < G::RC; ++i)
        lb[(size_t)r * G::RC + i] = (plane << (L1 + L2)) + ((long long)(r * G::RC + i) << L2);
    for (int phase = 0; phase < 3; ++phase)
      for (int r = 0; r < C; ++r) {
        cv.rank = r;
        plane_body<T, B2, L1, L2, LC, NT>(d, plane, cv.re[r], cv.im[r], cv,
                                          lb.data() + (size_t)r * G::RC, phase);
      }
  }
  return PAC_SUCCESS;
}

int be_launch_pass(const PassDesc& d, int elem_bytes, int b2, long long grid, int threads,
                   size_t, void*) {
  if (d.plane) {
#define PAC_X(T, BY, B2_, L1_, L2_, LC, NT_, MB)                                           \
  if (elem_bytes == BY && b2 == B2_ && d.plane_logN1 == L1_ && d.plane_logN2 == L2_ &&   \
      threads == NT_) {                                                                  \
    g_launches++;                                                                        \
    return replay_plane<T, B2_, L1_, L2_, LC, NT_>(d, grid);                             \
  }
    PAC_PLANE_LIST(PAC_X)
#undef PAC_X
    return set_error(PAC_ERROR_INTERNAL, "no plane replay for a pass marked plane");
  }
  if (d.tma) {
    int seen = 0;  // candidates of this geometry so far; d.tma - 1 picks one
#define PAC_X(T, BY, B2_, MO, SG, LL, LW, NT_, MB, PP, DF, TC_)                                   \
  if (elem_bytes == BY && b2 == B2_ && d.mode == MO && d.sign == SG && d.logL == LL &&     \
      d.tc == TC_ && seen++ == d.tma - 1 && d.W == (1 << LW) && threads == NT_) {          \
    g_launches++;                                                                          \
    return replay_coltma<T, B2_, MO, SG, LL, LW, NT_, PP, TC_>(d, grid);                   \
  }
    PAC_COLTMA_LIST(PAC_X)
#undef PAC_X
    return set_error(PAC_ERROR_INTERNAL, "no tensor-copy replay for a pass marked so");
  }
  if (d.pipe) {
#define PAC_X(T, BY, B2_, MO, SG, LL, LW, NT_)                                               \
  if (elem_bytes == BY && b2 == B2_ && d.mode == MO && d.sign == SG && d.logL == LL &&      \
      d.W == (1 << LW) && threads == NT_) {                                                 \
    replay_pipe<T, B2_, MO, SG, LL, LW, NT_>(d, grid);                                      \
    g_launches++;                                                                           \
    return PAC_SUCCESS;                                                                     \
  }
    PAC_PIPE_LIST(PAC_X)
#undef PAC_X
    return set_error(PAC_ERROR_INTERNAL, "no pipelined replay for a pass marked pipelined");
  }
  if (d.logC > 0) {
#define PAC_X(T, BY, B2_, MO, SG, LL, LW, LC, NT_, MB)                                      \
  if (elem_bytes == BY && b2 == B2_ && d.mode == MO && d.sign == SG && d.logL == LL &&   \
      d.W == (1 << LW) && d.logC == LC && threads == NT_) {                              \
    replay_cluster<T, B2_, MO, SG, LL, LW, LC, NT_>(d, grid);                            \
    g_launches++;                                                                        \
    return PAC_SUCCESS;                                                                  \
  }
    PAC_CLUSTER_LIST(PAC_X)
#undef PAC_X
    return set_error(PAC_ERROR_INTERNAL, "no cluster replay for a pass marked clustered");
  }
  if (d.spec) {
    const int cols = d.logS > 0 ? 1 : 0;
    int seen = 0;  // candidates of this geometry so far; d.spec - 1 picks one
#define PAC_X(T, BY, B2_, MO, SG, LL, CO, LW, NT_, MB, TC_, RC_)                              \
  if (elem_bytes == BY && b2 == B2_ && d.mode == MO && (MO == MODE_CONV || d.sign == SG) && \
      d.logL == LL && cols == CO && d.tc == TC_ && rads_match(d, LL, B2_, RC_) &&          \
      seen++ == d.spec - 1 && d.W == (1 << LW) && threads == NT_) {                         \
    replay_special<T, B2_, MO, SG, LL, CO, LW, NT_, TC_, RC_>(d, grid);                              \
    g_launches++;                                                                          \
    return PAC_SUCCESS;                                                                    \
  }
    PAC_SPECIAL_LIST(PAC_X)
#undef PAC_X
    return set_error(PAC_ERROR_INTERNAL, "no specialised replay for a pass marked special");
  }
  if (d.W > 64) return set_error(PAC_ERROR_INTERNAL, "W > 64");
  if (d.tc && b2 != 3) {
    if (b2 == 1) replay<float, 1, 1>(d, grid);
    else replay<float, 2, 1>(d, grid);
  } else if (elem_bytes == 8) {
    if (b2 == 1) replay<double, 1>(d, grid);
    else if (b2 == 2) replay<double, 2>(d, grid);
    else replay<double, 3>(d, grid);
  } else {
    if (b2 == 1) replay<float, 1>(d, grid);
    else if (b2 == 2) replay<float, 2>(d, grid);
    else replay<float, 3>(d, grid);
  }
  g_launches++;
  return PAC_SUCCESS;
}

// exp(-2 pi i E / N) evaluated in long double and rounded once
static void root(long long E, long long N, double* c, double* s) {
  long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)E / (long double)N;
  *c = (double)cosl(a);
  *s = (double)sinl(a);
}

template <typename T>
static void put(void* dst, long long i, double c, double s) {
  T* p = (T*)dst;
  p[2 * i] = (T)c;
  p[2 * i + 1] = (T)s;
}

int be_fill_tc_const(void* dst, void*) {
  TcConst* t = (TcConst*)dst;
  for (int set = 0; set < TC_CONST_SETS; ++set)
    for (int lane = 0; lane < 32; ++lane) tc_const_fill(set, lane, t[set * 32 + lane]);
  return PAC_SUCCESS;
}

int be_fill_stage_tw(void* dst, int elem_bytes, int logK, int logR, void*) {
  long long R1 = (1LL << logR) - 1, K = 1LL << logK;
  long long n = (K >> logR) * R1;
  for (long long idx = 0; idx < n; ++idx) {
    long long ell = K >> logR;  // s-major: entry (s-1)*ell + j = w_K^{j s}
    long long s = idx / ell + 1, j = idx % ell;
    (void)R1;
    double c, sn;
    root((j * s) % K, K, &c, &sn);
    if (elem_bytes == 8) put<double>(dst, idx, c, sn);
    else put<float>(dst, idx, c, sn);
  }
  g_launches++;
  return PAC_SUCCESS;
}

int be_fill_pow_tw(void* dst, int elem_bytes, long long count, long long stride, int logN, void*) {
  long long N = 1LL << logN;
  for (long long k = 0; k < count; ++k) {
    double c, sn;
    root((k * stride) & (N - 1), N, &c, &sn);
    if (elem_bytes == 8) put<double>(dst, k, c, sn);
    else put<float>(dst, k, c, sn);
  }
  g_launches++;
  return PAC_SUCCESS;
}

int be_fill_ref_tw(int r, int t, double* re, double* im, void*) {
  long long off = 0, ell = 1;
  for (int q = 0; q < t; ++q) {
    long long k = ell * r;
    for (long long m = 1; m < r; ++m)
      for (long long j = 0; j < ell; ++j) {
        root((m * j) % k, k, &re[off + (m - 1) * ell + j], &im[off + (m - 1) * ell + j]);
      }
    off += (r - 1) * ell;
    ell = k;
  }
  g_launches++;
  return PAC_SUCCESS;
}

int be_plan_order(const double* in_re, const double* in_im, void* out_re, void* out_im,
                  int elem_bytes, int logL, int logR, long long nlines, double scale, void*) {
  const int L = 1 << logL, lq = logL - logR;
  std::vector<double> br(L), bi(L);
  for (long long line = 0; line < nlines; ++line) {
    const long long base = line << logL;
    for (int q = 0; q < L; ++q) {
      br[q] = in_re[base + q];
      bi[q] = in_im[base + q];
    }
    for (int idx = 0; idx < L; ++idx) {
      const int t = idx >> lq, blk = idx & ((1 << lq) - 1);
      const int q = (blk << logR) + t;
      if (elem_bytes == 8) {
        ((double*)out_re)[base + idx] = br[q] * scale;
        ((double*)out_im)[base + idx] = bi[q] * scale;
      } else {
        ((float*)out_re)[base + idx] = (float)(br[q] * scale);
        ((float*)out_im)[base + idx] = (float)(bi[q] * scale);
      }
    }
  }
  g_launches++;
  return PAC_SUCCESS;
}

int be_round_to_f32(const double* src, float* dst, long long n, void*) {
  for (long long i = 0; i < n; ++i) dst[i] = (float)src[i];
  g_launches++;
  return PAC_SUCCESS;
}

template <typename T>
static void pointwise_t(long long n, const T* xr, const T* xi, const T* hr, const T* hi,
                        long long hmask, T* yr, T* yi, T scale) {
  for (long long i = 0; i < n; ++i) {
    T ar = xr[i], ai = xi[i];
    long long k = i & hmask;
    T br = hr[k], bi = hi[k];
    yr[i] = (ar * br - ai * bi) * scale;
    yi[i] = (ar * bi + ai * br) * scale;
  }
}

int be_pointwise(long long n, int elem_bytes, const void* xr, const void* xi, const void* hr,
                 const void* hi, long long hmask, void* yr, void* yi, double scale, void*) {
  if (elem_bytes == 8)
    pointwise_t<double>(n, (const double*)xr, (const double*)xi, (const double*)hr,
                        (const double*)hi, hmask, (double*)yr, (double*)yi, scale);
  else
    pointwise_t<float>(n, (const float*)xr, (const float*)xi, (const float*)hr, (const float*)hi,
                       hmask, (float*)yr, (float*)yi, (float)scale);
  g_launches++;
  return PAC_SUCCESS;
}

int be_scale_copy(long long n, int elem_bytes, const void* xr, const void* xi, void* yr, void* yi,
                  double scale, void*) {
  for (long long i = 0; i < n; ++i) {
    if (elem_bytes == 8) {
      ((double*)yr)[i] = ((const double*)xr)[i] * scale;
      ((double*)yi)[i] = ((const double*)xi)[i] * scale;
    } else {
      ((float*)yr)[i] = ((const float*)xr)[i] * (float)scale;
      ((float*)yi)[i] = ((const float*)xi)[i] * (float)scale;
    }
  }
  g_launches++;
  return PAC_SUCCESS;
}

int be_permute(long long n, const int* rho, double* re, double* im, void*) {
  for (long long j = 0; j < n; ++j) {
    long long p = rho[j];
    if (j < p && p < n) {
      if (im) {
        double a = re[j], b = im[j];
        re[j] = re[p];
        im[j] = im[p];
        re[p] = a;
        im[p] = b;
      } else {
        double a = re[2 * j], b = re[2 * j + 1];
        re[2 * j] = re[2 * p];
        re[2 * j + 1] = re[2 * p + 1];
        re[2 * p] = a;
        re[2 * p + 1] = b;
      }
    }
  }
  g_launches++;
  return PAC_SUCCESS;
}

long long be_launch_count() { return g_launches.load(); }
int be_fma_peak(int, void*, double*) {
  return set_error(PAC_ERROR_NO_DEVICE, "pac_fma_peak: the host replay has no device to measure");
}

// work-queue launch: the items in queue order, one CTA each (the queue's
// order is the one a single persistent CTA would take)
template <typename T, int B2, int TC = 0>
static void replay_queue(const PassDesc* descs, const long long* starts, const int* item_desc,
                         long long total) {
  std::vector<long long> lb(128);
  for (long long it = 0; it < total; ++it) {
    const int k = item_desc[it];
    const PassDesc& d = descs[k];
    const long long cta = it - starts[k];
    std::vector<T> sm((size_t)2 * d.W * d.pitch, std::numeric_limits<T>::quiet_NaN());
    for (int w = 0; w < d.W; ++w) lb[w] = lb[64 + w] = line_base(d, cta * d.W + w);
    queue_pass_body<T, B2, TC>(d, cta, sm.data(), sm.data() + (size_t)d.W * d.pitch, lb.data(),
                               lb.data() + 64);
  }
}

int be_queue_prepare(int, int, int, size_t) { return PAC_SUCCESS; }

int be_launch_queue(const PassDesc* descs, const long long* starts, const int* item_desc, int,
                    long long total, unsigned long long* counter, int elem_bytes, int b2, int tc,
                    size_t, void*) {
  if (tc && b2 != 3) {
    if (b2 == 1) replay_queue<float, 1, 1>(descs, starts, item_desc, total);
    else replay_queue<float, 2, 1>(descs, starts, item_desc, total);
  } else if (elem_bytes == 8) {
    if (b2 == 1) replay_queue<double, 1>(descs, starts, item_desc, total);
    else if (b2 == 2) replay_queue<double, 2>(descs, starts, item_desc, total);
    else replay_queue<double, 3>(descs, starts, item_desc, total);
  } else {
    if (b2 == 1) replay_queue<float, 1>(descs, starts, item_desc, total);
    else if (b2 == 2) replay_queue<float, 2>(descs, starts, item_desc, total);
    else replay_queue<float, 3>(descs, starts, item_desc, total);
  }
  if (total > 0) *counter += (unsigned long long)total;
  g_launches++;
  return PAC_SUCCESS;
}

int be_graph_supported() { return 0; }
int be_graph_begin(void*) { return set_error(PAC_ERROR_INTERNAL, "no graphs in the host replay"); }
int be_graph_end(void*, void**) {
  return set_error(PAC_ERROR_INTERNAL, "no graphs in the host replay");
}
int be_graph_launch(void*, void*) {
  return set_error(PAC_ERROR_INTERNAL, "no graphs in the host replay");
}
int be_graph_destroy(void*) { return PAC_SUCCESS; }

}  // namespace pac
