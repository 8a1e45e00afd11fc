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
  // device status word (bounded waits report here); may be null
  int* status;
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

// ---------------------------------------------------------------------------
// One radix-R butterfly of a stage.
//   DIF: load x[m] @ j + ell*m, DFT, twiddle output s by w_K^{j s},
//        store @ j + ell*sigma_b(s)
//   DIT: load x[s] @ j + ell*sigma_b(s), twiddle by w_K^{j s}, DFT,
//        store @ j + ell*m
// Global-facing stages read (first) or write (last) the line in global
// memory; all other accesses go to the padded shared-memory line.
// ---------------------------------------------------------------------------
enum { IO_SMEM = 0, IO_GLOBAL = 1 };

struct StageGeo {
  int logK, logR, logell;
  int twoff;
};

// butterfly index -> (w, blk, j)
PAC_HD void bf_coords(const PassDesc& d, const StageGeo& st, bool global_facing, int u, int* w,
                      int* blk, int* j) {
  const int lbf = d.logL - st.logR;  // butterflies per line (log)
  int v;
  if (global_facing && d.logS > 0) {
    *w = u & (d.W - 1);
    v = u >> d.logW;
  } else {
    v = u & ((1 << lbf) - 1);
    *w = u >> lbf;
  }
  *blk = v >> st.logell;
  *j = v & ((1 << st.logell) - 1);
}

template <typename T, int B2, int R, int SIGN, bool DIF>
PAC_HD void stage_bf(const PassDesc& d, long long cta, T* sre, T* sim, const StageGeo& st,
                     int src, int dst, int u, const long long* lbase_in,
                     const long long* lbase_out) {
  constexpr int LR = ilog2(R);
  static_assert(LR % B2 == 0, "radix must be a power of the digit base");
  int w, blk, j;
  bf_coords(d, st, src == IO_GLOBAL || dst == IO_GLOBAL, u, &w, &blk, &j);
  const int ell = 1 << st.logell;
  const int e0 = (blk << st.logK) + j;
  const T* ire = (const T*)d.in_re;
  const T* iim = (const T*)d.in_im;
  Cx<T> x[R];
  // ---- load
  static_for<R>([&](auto mm) {
    constexpr int m = mm.value;
    constexpr int slot = DIF ? m : drev_c(m, LR, B2);
    const int e = e0 + ell * slot;
    if (src == IO_GLOBAL) {
      long long gi = lbase_in[w] + ((long long)e << d.logS);
      x[m] = Cx<T>{ld_g(ire + gi), ld_g(iim + gi)};
    } else {
      int si = w * d.pitch + sidx<T>(e);
      x[m] = Cx<T>{sre[si], sim[si]};
    }
  });
  const Cx<T>* tw = (const Cx<T>*)d.tw + st.twoff + j * (R - 1);
  const bool twiddle = st.logell > 0 && j > 0;
  // ---- DIT: 4-step pre-twiddle (first DIT stage only, ell == 1) and
  //      stage twiddle on the inputs
  if constexpr (!DIF) {
    if (d.tw4 == 2 && st.logell == 0) {
      long long g = (long long)cta * d.W + w;
      long long i = g & ((1LL << d.logS) - 1);
      uint32_t iG = (uint32_t)((i >> d.tw4_shift) & d.tw4_mask);
      const Cx<T>* lo = (const Cx<T>*)d.tw4_lo;
      const Cx<T>* hi = (const Cx<T>*)d.tw4_hi;
      static_for<R>([&](auto mm) {
        constexpr int m = mm.value;
        constexpr int slot = drev_c(m, LR, B2);
        uint32_t E = iG * drev<B2>((uint32_t)(e0 + slot), d.logL);
        Cx<T> wv = cmul(ld_tw(lo + (E & ((1u << d.tw4_lolog) - 1))), ld_tw(hi + (E >> d.tw4_lolog)));
        x[m] = ctw(x[m], wv, SIGN);
      });
    }
    if (twiddle) {
      static_for<R - 1>([&](auto ss) {
        constexpr int s = ss.value + 1;
        x[s] = ctw(x[s], ld_tw(tw + (s - 1)), SIGN);
      });
    }
  }
  dft_reg<T, R, SIGN>(x);
  // register p now holds output index brev(p)
  if constexpr (DIF) {
    if (twiddle) {
      static_for<R>([&](auto pp) {
        constexpr int s = brev_c(pp.value, LR);
        if constexpr (s > 0) x[pp.value] = ctw(x[pp.value], ld_tw(tw + (s - 1)), SIGN);
      });
    }
    if (d.tw4 == 1 && st.logell == 0) {
      long long g = (long long)cta * d.W + w;
      long long i = g & ((1LL << d.logS) - 1);
      uint32_t iG = (uint32_t)((i >> d.tw4_shift) & d.tw4_mask);
      const Cx<T>* lo = (const Cx<T>*)d.tw4_lo;
      const Cx<T>* hi = (const Cx<T>*)d.tw4_hi;
      static_for<R>([&](auto pp) {
        constexpr int slot = drev_c(brev_c(pp.value, LR), LR, B2);
        uint32_t E = iG * drev<B2>((uint32_t)(e0 + ell * slot), d.logL);
        Cx<T> wv = cmul(ld_tw(lo + (E & ((1u << d.tw4_lolog) - 1))), ld_tw(hi + (E >> d.tw4_lolog)));
        x[pp.value] = ctw(x[pp.value], wv, SIGN);
      });
    }
  }
  // ---- store
  T* ore = (T*)d.out_re;
  T* oim = (T*)d.out_im;
  static_for<R>([&](auto pp) {
    constexpr int p = pp.value;
    constexpr int slot = DIF ? drev_c(brev_c(p, LR), LR, B2) : brev_c(p, LR);
    const int e = e0 + ell * slot;
    Cx<T> v = x[p];
    if (dst == IO_GLOBAL) {
      if (d.use_scale) {
        v.re *= T(d.scale);
        v.im *= T(d.scale);
      }
      long long gi = lbase_out[w] + ((long long)e << d.logS);
      ore[gi] = v.re;
      oim[gi] = v.im;
    } else {
      int si = w * d.pitch + sidx<T>(e);
      sre[si] = v.re;
      sim[si] = v.im;
    }
  });
}

// Convolution middle: the last DIF stage (ell == 1), the pointwise product
// with the filter spectrum at the same P_b positions, and the first DIT
// stage, all in registers.
template <typename T, int B2, int R>
PAC_HD void middle_bf(const PassDesc& d, long long cta, T* sre, T* sim, const StageGeo& st,
                      int src, int dst, int u, const long long* lbase) {
  constexpr int LR = ilog2(R);
  int w, blk, j;
  bf_coords(d, st, src == IO_GLOBAL || dst == IO_GLOBAL, u, &w, &blk, &j);
  const int e0 = blk << st.logK;  // ell == 1, j == 0
  const T* ire = (const T*)d.in_re;
  const T* iim = (const T*)d.in_im;
  const T* hre = (const T*)d.h_re;
  const T* him = (const T*)d.h_im;
  Cx<T> x[R];
  static_for<R>([&](auto mm) {
    constexpr int m = mm.value;
    const int e = e0 + m;
    if (src == IO_GLOBAL) {
      long long gi = lbase[w] + ((long long)e << d.logS);
      x[m] = Cx<T>{ld_g(ire + gi), ld_g(iim + gi)};
    } else {
      int si = w * d.pitch + sidx<T>(e);
      x[m] = Cx<T>{sre[si], sim[si]};
    }
  });
  dft_reg<T, R, -1>(x);
  // register p holds the spectrum at slot sigma_b(brev(p)); the DIT stage
  // wants register s = the value at slot sigma_b(s), i.e. register brev(s).
  Cx<T> y[R];
  const T sc = T(d.scale);
  static_for<R>([&](auto ss) {
    constexpr int s = ss.value;
    constexpr int p = brev_c(s, LR);
    const int e = e0 + drev_c(s, LR, B2);
    long long hi = (lbase[w] + ((long long)e << d.logS)) & d.h_mask;
    Cx<T> hv = Cx<T>{ld_g(hre + hi) * sc, ld_g(him + hi) * sc};
    y[s] = cmul(x[p], hv);
  });
  dft_reg<T, R, +1>(y);
  T* ore = (T*)d.out_re;
  T* oim = (T*)d.out_im;
  static_for<R>([&](auto pp) {
    constexpr int p = pp.value;
    const int e = e0 + brev_c(p, LR);
    if (dst == IO_GLOBAL) {
      long long gi = lbase[w] + ((long long)e << d.logS);
      ore[gi] = y[p].re;
      oim[gi] = y[p].im;
    } else {
      int si = w * d.pitch + sidx<T>(e);
      sre[si] = y[p].re;
      sim[si] = y[p].im;
    }
  });
}

// ---------------------------------------------------------------------------
// Runtime -> compile-time dispatch of one butterfly
// ---------------------------------------------------------------------------
template <typename T, int B2, bool DIF>
PAC_HD void stage_dispatch(const PassDesc& d, long long cta, T* sre, T* sim, const StageGeo& st,
                           int sign, int src, int dst, int u, const long long* lbi,
                           const long long* lbo) {
#define PAC_ST(RR)                                                                          \
  if (sign < 0) stage_bf<T, B2, RR, -1, DIF>(d, cta, sre, sim, st, src, dst, u, lbi, lbo); \
  else stage_bf<T, B2, RR, +1, DIF>(d, cta, sre, sim, st, src, dst, u, lbi, lbo);
  if constexpr (B2 == 1) {
    switch (st.logR) {
      case 1: PAC_ST(2) break;
      case 2: PAC_ST(4) break;
      case 3: PAC_ST(8) break;
      default: PAC_ST(16) break;
    }
  } else if constexpr (B2 == 2) {
    if (st.logR == 2) { PAC_ST(4) } else { PAC_ST(16) }
  } else {
    PAC_ST(8)
  }
#undef PAC_ST
}

template <typename T, int B2>
PAC_HD void middle_dispatch(const PassDesc& d, long long cta, T* sre, T* sim, const StageGeo& st,
                            int src, int dst, int u, const long long* lb) {
  if constexpr (B2 == 1) {
    switch (st.logR) {
      case 1: middle_bf<T, B2, 2>(d, cta, sre, sim, st, src, dst, u, lb); break;
      case 2: middle_bf<T, B2, 4>(d, cta, sre, sim, st, src, dst, u, lb); break;
      case 3: middle_bf<T, B2, 8>(d, cta, sre, sim, st, src, dst, u, lb); break;
      default: middle_bf<T, B2, 16>(d, cta, sre, sim, st, src, dst, u, lb); break;
    }
  } else if constexpr (B2 == 2) {
    if (st.logR == 2) middle_bf<T, B2, 4>(d, cta, sre, sim, st, src, dst, u, lb);
    else middle_bf<T, B2, 16>(d, cta, sre, sim, st, src, dst, u, lb);
  } else {
    middle_bf<T, B2, 8>(d, cta, sre, sim, st, src, dst, u, lb);
  }
}

// ---------------------------------------------------------------------------
// Pass body: a sequence of phases separated by CTA barriers.  A phase is a
// loop over butterflies; the device runs it with one butterfly per thread,
// the host emulator with a plain loop.  Barrier placement: every phase that
// reads shared memory is preceded by a barrier after the phase that wrote it.
// ---------------------------------------------------------------------------
#if defined(__CUDA_ARCH__)
#define PAC_FOR_BF(n, u) for (int u = (int)threadIdx.x; u < (n); u += (int)blockDim.x)
#define PAC_SYNC() __syncthreads()
#else
#define PAC_FOR_BF(n, u) for (int u = 0; u < (n); ++u)
#define PAC_SYNC() ((void)0)
#endif

PAC_HD StageGeo geo_of(const PassDesc& d, int i) {
  // stage i of the DIF order: K_i = L / (R_0 ... R_{i-1})
  int logK = d.logL;
  for (int q = 0; q < i; ++q) logK -= d.rlog[q];
  StageGeo g;
  g.logK = logK;
  g.logR = d.rlog[i];
  g.logell = logK - d.rlog[i];
  g.twoff = d.tw_off[i];
  return g;
}

template <typename T, int B2>
PAC_HD void pass_body(const PassDesc& d, long long cta, T* sre, T* sim, long long* lbi,
                      long long* lbo) {
  // per-line global bases (W <= 64); every thread computes them
  const bool nat = d.nat != 0;
  for (int w = 0; w < d.W; ++w) {
    long long g = cta * d.W + w;
    if (nat) {
      nat_line<B2>(d, g, &lbi[w], &lbo[w]);
    } else {
      lbi[w] = line_base(d, g);
      lbo[w] = lbi[w];
    }
  }
  const int nst = d.nst;
  if (d.mode == MODE_DIF) {
    for (int i = 0; i < nst; ++i) {
      StageGeo st = geo_of(d, i);
      int src = (i == 0) ? IO_GLOBAL : IO_SMEM;
      int dst = (i == nst - 1 && !nat) ? IO_GLOBAL : IO_SMEM;
      int nbf = d.W << (d.logL - st.logR);
      if (i > 0) PAC_SYNC();
      PAC_FOR_BF(nbf, u) {
        stage_dispatch<T, B2, true>(d, cta, sre, sim, st, d.sign, src, dst, u, lbi, lbo);
      }
    }
    if (nat) {
      // natural-order store out of shared memory
      PAC_SYNC();
      T* ore = (T*)d.out_re;
      T* oim = (T*)d.out_im;
      const int n = d.W << d.logL;
      const bool lines_fast = d.logS > 0 || d.nat_nf > 0;
      PAC_FOR_BF(n, u) {
        int w, q;
        if (lines_fast) {
          w = u & (d.W - 1);
          q = u >> d.logW;
        } else {
          w = u >> d.logL;
          q = u & (d.L - 1);
        }
        // q is the natural index inside this factor: it sits at slot rev(q)
        int e = (int)drev<B2>((uint32_t)q, d.logL);
        int si = w * d.pitch + sidx<T>(e);
        T vr = sre[si], vi = sim[si];
        if (d.use_scale) {
          vr *= T(d.scale);
          vi *= T(d.scale);
        }
        long long gi = lbo[w] + ((long long)q << (d.nat_Mlog + d.logS));
        ore[gi] = vr;
        oim[gi] = vi;
      }
    }
  } else if (d.mode == MODE_DIT) {
    for (int k = 0; k < nst; ++k) {
      int i = nst - 1 - k;
      StageGeo st = geo_of(d, i);
      int src = (k == 0) ? IO_GLOBAL : IO_SMEM;
      int dst = (k == nst - 1) ? IO_GLOBAL : IO_SMEM;
      int nbf = d.W << (d.logL - st.logR);
      if (k > 0) PAC_SYNC();
      PAC_FOR_BF(nbf, u) {
        stage_dispatch<T, B2, false>(d, cta, sre, sim, st, d.sign, src, dst, u, lbi, lbo);
      }
    }
  } else {  // MODE_CONV
    for (int i = 0; i < nst - 1; ++i) {
      StageGeo st = geo_of(d, i);
      int src = (i == 0) ? IO_GLOBAL : IO_SMEM;
      int nbf = d.W << (d.logL - st.logR);
      if (i > 0) PAC_SYNC();
      PAC_FOR_BF(nbf, u) {
        stage_dispatch<T, B2, true>(d, cta, sre, sim, st, -1, src, IO_SMEM, u, lbi, lbo);
      }
    }
    {
      StageGeo st = geo_of(d, nst - 1);
      int src = (nst == 1) ? IO_GLOBAL : IO_SMEM;
      int dst = (nst == 1) ? IO_GLOBAL : IO_SMEM;
      int nbf = d.W << (d.logL - st.logR);
      if (nst > 1) PAC_SYNC();
      PAC_FOR_BF(nbf, u) { middle_dispatch<T, B2>(d, cta, sre, sim, st, src, dst, u, lbi); }
    }
    for (int i = nst - 2; i >= 0; --i) {
      StageGeo st = geo_of(d, i);
      int dst = (i == 0) ? IO_GLOBAL : IO_SMEM;
      int nbf = d.W << (d.logL - st.logR);
      PAC_SYNC();
      PAC_FOR_BF(nbf, u) {
        stage_dispatch<T, B2, false>(d, cta, sre, sim, st, +1, IO_SMEM, dst, u, lbi, lbo);
      }
    }
  }
}

}  // namespace pac
