// pac_engine.cuh -- per-CTA radix-2^k butterfly engine of the permutation-
// avoiding FFT convolution (sm_100a).
//
// One "pass" transforms W lines of length L (a power of two) that lie in
// global memory at element stride S.  Inside the CTA a line is split into
// radix-R register butterflies (R in {2,4,8,16}); the stages exchange data
// through padded shared memory.  The first stage reads global memory
// directly into registers and the last stage writes registers directly to
// global memory, so a pass costs one HBM read and one HBM write of the tile.
//
// Orders (the reference's factorisation F = A P, butterflies.c):
//   DIF stages  (A^T, forward):  natural input  -> output in base-b digit-
//               reversed order P_b (apply_transposed_butterflies_r*)
//   DIT stages  (A / conj(A)):   P_b input      -> natural output
//               (apply_butterflies_r*, apply_conjugate_butterflies_r*)
// Each register butterfly relabels its outputs so that stages of any radix
// R = b^k compose to the exact base-b digit reversal of the whole line, so
// the device spectrum order is bit-identical to the reference's P_r F x.
//
// The stage code is written as __host__ __device__ phase functions over a
// butterfly index so that a host build (PAC_EMULATE) can replay a CTA
// phase by phase; the device kernel runs the same code with one butterfly
// per thread and __syncthreads() between phases.
#pragma once

#include <stdint.h>

#include <utility>

#if defined(__CUDACC__)
#define PAC_HD __host__ __device__ __forceinline__
#define PAC_HDC __host__ __device__ constexpr
#else
#define PAC_HD inline
#define PAC_HDC constexpr
#endif

namespace pac {

// ---------------------------------------------------------------------------
// Pass descriptor (host fills, kernel reads by value)
// ---------------------------------------------------------------------------
enum PassMode { MODE_DIF = 0, MODE_DIT = 1, MODE_CONV = 2 };
enum { PAC_MAX_STAGES = 8, PAC_MAX_FACTORS = 4 };

struct PassDesc {
  const void* in_re;
  const void* in_im;
  void* out_re;
  void* out_im;
  // CONV: filter spectrum in P_b order, same layout as one problem
  const void* h_re;
  const void* h_im;
  long long h_mask;   // element index mask applied before reading h (N-1 broadcasts)
  double scale;       // CONV: product scale; DIF/DIT: final store scale
  int use_scale;
  int mode;
  int sign;           // -1 forward twiddles, +1 conjugate (DIF/DIT passes)
  int L, logL;        // line length
  int W, logW;        // lines per CTA
  int logS;           // element stride along the line = 1 << logS
  long long nlines;   // lines in the whole launch
  int pitch;          // shared-memory line pitch (elements)
  int nthreads;
  // stages, DIF order (outermost block first); DIT passes run them reversed
  int nst;
  int rlog[PAC_MAX_STAGES];
  int tw_off[PAC_MAX_STAGES];  // offset (in complex entries) of table (K_i, R_i)
  const void* tw;              // stage twiddle pool, forward sign, Cx<T>
  // 4-step twiddle between the factors of a split axis:
  //   w_N^{sign * iG * rev_b(e)},  iG = (i >> tw4_shift) & tw4_mask
  // DIF: after the last stage (post); DIT: before the first stage (pre)
  int tw4;
  int tw4_shift;
  long long tw4_mask;
  int tw4_lolog;
  const void* tw4_lo;  // w_N^{0 .. 2^lolog - 1}
  const void* tw4_hi;  // w_N^{k * 2^lolog}
  // natural-order store (fft / ifft): this pass is the last factor of its
  // axis group; the earlier factors' lengths are nat_flog[0..nat_nf-1]
  // (outermost first), their product is M = 2^nat_Mlog.
  int nat;
  int nat_nf;
  int nat_flog[PAC_MAX_FACTORS];
  int nat_Mlog;
  // device status word of the plan: a bounded wait that gives up writes
  // PAC_ERROR_TIMEOUT here; may be null
  int* status;
  // spin limit of the pass's bounded waits, in SM clock cycles (<= 0: the
  // default, 2^31 cycles, about a second)
  long long wait_limit;
  // 1: this pass runs the kernel specialised for its geometry (pac_special.h)
  int spec;
  // > 0: a cluster of 2^logC CTAs shares each tile of this specialised
  // column pass (pac_special.h, PAC_CLUSTER_LIST)
  int logC;
  // 1: pipelined column pass, one persistent CTA per SM with tensor-copy
  // prefetch of the next tile (pac_special.h, PAC_PIPE_LIST; ColPipe)
  int pipe;
  // k > 0: column pass staged through shared memory by tensor copies, the
  // k-th geometry of its kind on PAC_COLTMA_LIST (pac_special.h; ColTma)
  int tma;
  // 1: plane pass of a 3D convolution (pac_plane.cuh): axes 1 and 2 of
  // every plane, whose stages are rlog[0 .. plane_n1s-1] (axis 1) then
  // rlog[plane_n1s .. nst-1] (axis 2), on a cluster of 2^logC CTAs
  int plane;
  int plane_n1s;
  int plane_logN1;
  int plane_logN2;
  // 1: tensor-core form, radix-16 stages on the tensor cores (pac_tc.cuh);
  // tcc: their DFT operands, per stage kind and lane (tc_const_set)
  int tc;
  const void* tcc;
};

// ---------------------------------------------------------------------------
// Complex arithmetic
// ---------------------------------------------------------------------------
template <typename T>
struct alignas(2 * sizeof(T)) Cx {
  T re, im;
};

template <typename T>
PAC_HD Cx<T> cadd(Cx<T> a, Cx<T> b) {
  return {a.re + b.re, a.im + b.im};
}
template <typename T>
PAC_HD Cx<T> csub(Cx<T> a, Cx<T> b) {
  return {a.re - b.re, a.im - b.im};
}
template <typename T>
PAC_HD Cx<T> cmul(Cx<T> a, Cx<T> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
// a * conj(b)
template <typename T>
PAC_HD Cx<T> cmulc(Cx<T> a, Cx<T> b) {
  return {a.re * b.re + a.im * b.im, a.im * b.re - a.re * b.im};
}
// a * w or a * conj(w) by the sign of the pass
template <typename T>
PAC_HD Cx<T> ctw(Cx<T> a, Cx<T> w, int sign) {
  return sign < 0 ? cmul(a, w) : cmulc(a, w);
}

// ---------------------------------------------------------------------------
// Integer helpers (compile-time label permutations, runtime digit reversal)
// ---------------------------------------------------------------------------
PAC_HDC int brev_c(int x, int bits) {
  int r = 0;
  for (int i = 0; i < bits; ++i) r = (r << 1) | ((x >> i) & 1);
  return r;
}
// reverse the base-2^dbits digits of a bits-wide number
PAC_HDC int drev_c(int x, int bits, int dbits) {
  int r = 0;
  for (int i = 0; i < bits; i += dbits) r = (r << dbits) | ((x >> i) & ((1 << dbits) - 1));
  return r;
}

PAC_HD uint32_t brev32(uint32_t x) {
#if defined(__CUDA_ARCH__)
  return __brev(x);
#else
  x = ((x >> 1) & 0x55555555u) | ((x & 0x55555555u) << 1);
  x = ((x >> 2) & 0x33333333u) | ((x & 0x33333333u) << 2);
  x = ((x >> 4) & 0x0F0F0F0Fu) | ((x & 0x0F0F0F0Fu) << 4);
  x = ((x >> 8) & 0x00FF00FFu) | ((x & 0x00FF00FFu) << 8);
  return (x >> 16) | (x << 16);
#endif
}

// base-2^B2 digit reversal of a bits-wide index (bits a multiple of B2):
// a full bit reversal reverses the digit order and the bits inside every
// digit; the second step restores the bit order inside the digits.
template <int B2>
PAC_HD uint32_t drev(uint32_t x, int bits) {
  if (bits == 0) return 0;
  uint32_t r = brev32(x) >> (32 - bits);
  if (B2 == 2) {
    r = ((r & 0x55555555u) << 1) | ((r >> 1) & 0x55555555u);
  } else if (B2 == 3) {
    r = (r & 0x92492492u) | ((r & 0x49249249u) << 2) | ((r & 0x24924924u) >> 2);
  }
  return r;
}


// ---------------------------------------------------------------------------
// Compile-time loops
// ---------------------------------------------------------------------------
template <int V>
struct IC {
  static constexpr int value = V;
  PAC_HDC operator int() const { return V; }
};
template <int N, int I = 0, class F>
PAC_HD void static_for(F&& f) {
  if constexpr (I < N) {
    f(IC<I>{});
    static_for<N, I + 1>(f);
  }
}
PAC_HDC int ilog2(int x) { return x <= 1 ? 0 : 1 + ilog2(x >> 1); }

// ---------------------------------------------------------------------------
// In-register DFTs.  d * exp(SIGN * 2*pi*i * K16 / 16) with exact handling of
// the multiples of pi/4; the remaining angles use cos(pi/8), sin(pi/8).
// ---------------------------------------------------------------------------
template <typename T, int SIGN, int K16>
PAC_HD Cx<T> rot16(Cx<T> d) {
  constexpr double H = 0.70710678118654752440;   // cos(pi/4)
  constexpr double C1 = 0.92387953251128675613;  // cos(pi/8)
  constexpr double S1 = 0.38268343236508977173;  // sin(pi/8)
  if constexpr (K16 == 0) {
    return d;
  } else if constexpr (K16 == 4) {
    // exp(SIGN i pi/2) = SIGN i
    if constexpr (SIGN < 0) return Cx<T>{d.im, -d.re};
    else return Cx<T>{-d.im, d.re};
  } else if constexpr (K16 == 2) {
    // (1 + SIGN i) / sqrt 2
    if constexpr (SIGN < 0) return Cx<T>{T(H) * (d.re + d.im), T(H) * (d.im - d.re)};
    else return Cx<T>{T(H) * (d.re - d.im), T(H) * (d.im + d.re)};
  } else if constexpr (K16 == 6) {
    // (-1 + SIGN i) / sqrt 2
    if constexpr (SIGN < 0) return Cx<T>{T(H) * (d.im - d.re), T(-H) * (d.im + d.re)};
    else return Cx<T>{T(-H) * (d.re + d.im), T(H) * (d.re - d.im)};
  } else {
    constexpr double c = K16 == 1 ? C1 : K16 == 3 ? S1 : K16 == 5 ? -S1 : -C1;
    constexpr double sn = (K16 == 1 || K16 == 7) ? S1 : C1;
    constexpr double s = SIGN < 0 ? -sn : sn;
    return Cx<T>{d.re * T(c) - d.im * T(s), d.re * T(s) + d.im * T(c)};
  }
}

// R-point DFT in registers, radix-2 decimation in frequency: natural input,
// output X[s] left in register brev(s).  SIGN -1 forward, +1 inverse.
template <typename T, int R, int SIGN>
PAC_HD void dft_reg(Cx<T> (&x)[R]) {
  static_assert(R >= 2 && R <= 16 && (R & (R - 1)) == 0, "radix");
  static_for<ilog2(R)>([&](auto lev) {
    constexpr int h = R >> (lev.value + 1);
    static_for<R / (2 * h)>([&](auto bb) {
      constexpr int b = bb.value * 2 * h;
      static_for<h>([&](auto jj) {
        constexpr int j = jj.value;
        Cx<T> a = x[b + j], c = x[b + j + h];
        x[b + j] = cadd(a, c);
        x[b + j + h] = rot16<T, SIGN, j * (16 / (2 * h))>(csub(a, c));
      });
    });
  });
}

// ---------------------------------------------------------------------------
// Memory helpers
// ---------------------------------------------------------------------------
template <typename T>
struct Pad;
template <>
struct Pad<double> {
  static constexpr int SH = 4;   // one pad element every 16 (8-byte banks)
  static constexpr int NB = 16;  // 8-byte slots per 128-byte bank row
};
template <>
struct Pad<float> {
  static constexpr int SH = 5;
  static constexpr int NB = 32;
};

template <typename T>
PAC_HD int sidx(int e) {
  return e + (e >> Pad<T>::SH);
}

template <typename T>
PAC_HD Cx<T> ld_tw(const Cx<T>* p) {
#if defined(__CUDA_ARCH__)
  if constexpr (sizeof(T) == 8) {
    double2 v = __ldg(reinterpret_cast<const double2*>(p));
    return Cx<T>{v.x, v.y};
  } else {
    float2 v = __ldg(reinterpret_cast<const float2*>(p));
    return Cx<T>{v.x, v.y};
  }
#else
  return *p;
#endif
}

template <typename T>
PAC_HD T ld_g(const T* p) {
#if defined(__CUDA_ARCH__)
  return __ldg(p);
#else
  return *p;
#endif
}

// ---------------------------------------------------------------------------
// Line addressing
// ---------------------------------------------------------------------------
// Base element index of line g for an ordinary pass: the axis of this pass
// has stride S = 2^logS; lines are (outer, inner) with inner fastest.
PAC_HD long long line_base(const PassDesc& d, long long g) {
  long long S1 = (1LL << d.logS) - 1;
  return ((g >> d.logS) << (d.logL + d.logS)) + (g & S1);
}

// Natural-order store: split line g into (o_real, c, i) and its input base.
// c is the natural index contributed by the earlier factors of the axis.
template <int B2>
PAC_HD void nat_line(const PassDesc& d, long long g, long long* in_base, long long* out_base) {
  const int Mlog = d.nat_Mlog;
  long long o_real, i = 0;
  uint32_t c = 0, packed = 0;
  if (d.logS == 0 && d.nat_nf > 0) {
    c = (uint32_t)(g & ((1LL << Mlog) - 1));
    o_real = g >> Mlog;
    // c = sum_f rev(p_f) * (L_1 .. L_{f-1}), first factor least significant
    uint32_t cc = c;
    for (int f = 0; f < d.nat_nf; ++f) {
      int fl = d.nat_flog[f];
      uint32_t k = cc & ((1u << fl) - 1);
      cc >>= fl;
      packed = (packed << fl) | drev<B2>(k, fl);
    }
  } else {
    i = g & ((1LL << d.logS) - 1);
    long long outer = g >> d.logS;
    packed = (uint32_t)(outer & ((1LL << Mlog) - 1));
    o_real = outer >> Mlog;
    // packed = p_1 * (L_2..L_{g-1}) + ... + p_{g-1}; unpack last factor first
    uint32_t pk = packed;
    int shift_acc[PAC_MAX_FACTORS];
    int acc = 0;
    for (int f = 0; f < d.nat_nf; ++f) {
      shift_acc[f] = acc;
      acc += d.nat_flog[f];
    }
    for (int f = d.nat_nf - 1; f >= 0; --f) {
      int fl = d.nat_flog[f];
      uint32_t p = pk & ((1u << fl) - 1);
      pk >>= fl;
      c |= drev<B2>(p, fl) << shift_acc[f];
    }
  }
  long long outer_in = (o_real << Mlog) + packed;
  *in_base = (outer_in << (d.logL + d.logS)) + i;
  *out_base = (o_real << (Mlog + d.logL + d.logS)) + ((long long)c << d.logS) + i;
}

}  // namespace pac
#include "pac_stages.cuh"
#include "pac_coltma.cuh"
#include "pac_plane.cuh"
