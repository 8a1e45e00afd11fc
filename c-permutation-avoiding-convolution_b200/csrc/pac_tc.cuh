// pac_tc.cuh -- radix-16 stages on the tensor cores (PAC_FORM_TC).
//
// In the tensor-core form every radix-16 stage of an FP32 pass runs as
// dense 16 x 16 complex DFT products on warp-level tensor-core MMAs
// (mma.sync m16n8k16: FP16 operands, FP32 accumulation).  A warp takes a
// tile of 16 butterflies of the stage:
//
//   Y (16 butterflies x 16 outputs) = X (16 x 16 inputs) . V,
//   V[k][c] = exp(SIGN 2 pi i m(k) f(c) / 16)
//
// where input column k is the element at slot s_in(k) of the butterfly
// (input index m(k): DIF s_in(k), DIT rev(s_in(k))) and output column c is
// stored at slot s_out(c) (frequency f(c): DIF rev(s_out(c)), DIT s_out(c)),
// rev the base-b digit reversal of 4 bits -- the same loads, outputs and
// stores as the register butterfly (stage_bf), so the two are
// interchangeable stage by stage.  A complex product is four real ones
// (Yr = Xr Vr - Xi Vi, Yi = Xr Vi + Xi Vr), and each real product is
// compensated: an operand a splits into a_hi = fp16(a) and
// a_lo = fp16(a - a_hi), and A.B ~ A_lo.B_hi + A_hi.B_lo + A_hi.B_hi
// (A_lo.B_lo, ~2^-22 relative, dropped), 24 MMAs per tile.  Before the
// split the 16 inputs of a butterfly are scaled by a power of two that puts
// their largest magnitude in [2^14, 2^15) -- the FP16 parts neither overflow
// nor, for all but the smallest elements, lose bits to subnormals -- and the
// outputs are scaled back exactly.  Stage and 4-step twiddles stay FP32 on
// the CUDA cores, before the DFT (DIT) or after it (DIF), as in bf_math.
//
// Fragment layouts (PTX ISA, mma.m16n8k16 with .f16 A/B and .f32 C/D;
// lane = 4 g + q; an f16x2 register holds the lower column in its low half):
//   A 16x16: reg 0 (row g, cols 2q, 2q+1)    reg 1 (row g+8, cols 2q, 2q+1)
//            reg 2 (row g, cols 2q+8, 2q+9)  reg 3 (row g+8, cols 2q+8, 2q+9)
//   B 16x8:  reg 0 (rows 2q, 2q+1, col g)    reg 1 (rows 2q+8, 2q+9, col g)
//   D 16x8:  d0, d1 (row g, cols 2q, 2q+1)   d2, d3 (row g+8, cols 2q, 2q+1)
// So lane (g, q) loads inputs k in {2q, 2q+1, 2q+8, 2q+9} of butterflies g
// and g+8 of the tile and stores outputs c in {2q, 2q+1} (+8 for the second
// MMA column half) of the same two butterflies: a butterfly never leaves its
// quad of lanes, and its scale needs only a two-step quad reduction.
//
// Slot maps: with the identity map the lanes of one load or store hit slots
// 2q + const; with the quad map (tc_qmap) they hit q + const.  Which of the
// two keeps the 32 lanes on 32 distinct shared-memory banks depends on the
// stage stride ell: the quad map for ell in {4, 8, 16}, the identity
// otherwise (for 2048-point lines: ell = 128 and 8, both conflict-free on
// rows with one pad element per 32, and on 8-line column tiles with the
// same pad and an odd line pitch).
//
// The lane code (loads, scaling, fragment packing, epilogue) is shared by
// the device, which runs one lane per thread with shuffles and mma.sync, and
// the host replay, which runs the 32 lanes of a warp in turn around an MMA
// emulated from the fragment layouts above.
#pragma once

#if defined(__CUDA_ARCH__)
#include <cuda_fp16.h>
#else
#include <math.h>
#include <string.h>
#endif

namespace pac {

PAC_HD uint32_t f32_bits(float f) {
#if defined(__CUDA_ARCH__)
  return __float_as_uint(f);
#else
  uint32_t u;
  memcpy(&u, &f, 4);
  return u;
#endif
}
PAC_HD float bits_f32(uint32_t u) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float f;
  memcpy(&f, &u, 4);
  return f;
#endif
}

#if !defined(__CUDA_ARCH__)
// IEEE binary16 (1 sign, 5 exponent, 10 fraction bits) from binary32,
// rounded to nearest even, with subnormals, overflow to infinity and NaN.
inline uint32_t f16_rn_host(float f) {
  const uint32_t x = f32_bits(f);
  const uint32_t sign = (x >> 16) & 0x8000u;
  const uint32_t ax = x & 0x7fffffffu;
  if (ax >= 0x7f800000u) return sign | (ax > 0x7f800000u ? 0x7e00u : 0x7c00u);
  const int e = (int)(ax >> 23) - 127;
  if (e > 15) return sign | 0x7c00u;
  if (e >= -14) {
    const uint32_t mant = ax & 0x7fffffu;
    uint32_t h = ((uint32_t)(e + 15) << 10) | (mant >> 13);
    const uint32_t rem = mant & 0x1fffu;
    if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) ++h;  // a carry may reach infinity
    return sign | h;
  }
  if (e < -25) return sign;
  // subnormal: the result counts units of 2^-24
  const uint32_t mant = (ax & 0x7fffffu) | 0x800000u;
  const int shift = -e - 1;  // 14 .. 24
  uint32_t h = mant >> shift;
  const uint32_t rem = mant & ((1u << shift) - 1u), half = 1u << (shift - 1);
  if (rem > half || (rem == half && (h & 1u))) ++h;
  return sign | h;
}
inline float f16_value_host(uint32_t h) {
  const uint32_t sign = (h & 0x8000u) << 16;
  const int e = (int)((h >> 10) & 0x1fu);
  const uint32_t m = h & 0x3ffu;
  if (e == 31) return bits_f32(sign | 0x7f800000u | (m << 13));
  if (e == 0) {
    const float v = ldexpf((float)m, -24);
    return sign ? -v : v;
  }
  return bits_f32(sign | ((uint32_t)(e - 15 + 127) << 23) | (m << 13));
}
#endif

// two floats -> f16x2 (a in the low half), rounded to nearest even
PAC_HD uint32_t tc_pack(float a, float b) {
#if defined(__CUDA_ARCH__)
  union {
    __half2 h;
    uint32_t u;
  } v;
  v.h = __floats2half2_rn(a, b);
  return v.u;
#else
  return f16_rn_host(a) | (f16_rn_host(b) << 16);
#endif
}
PAC_HD void tc_unpack(uint32_t x, float& a, float& b) {
#if defined(__CUDA_ARCH__)
  union {
    uint32_t u;
    __half2 h;
  } v;
  v.u = x;
  const float2 f = __half22float2(v.h);
  a = f.x;
  b = f.y;
#else
  a = f16_value_host(x & 0xffffu);
  b = f16_value_host(x >> 16);
#endif
}
// (a, b) -> hi = fp16(a, b), lo = fp16(a - hi_a, b - hi_b); the differences
// are exact in FP32
PAC_HD void tc_split2(float a, float b, uint32_t& hi, uint32_t& lo) {
  hi = tc_pack(a, b);
  float ha, hb;
  tc_unpack(hi, ha, hb);
  lo = tc_pack(a - ha, b - hb);
}

// 2^E for |E| <= 126, exact
PAC_HD float tc_pow2(int E) { return bits_f32((uint32_t)(127 + E) << 23); }

PAC_HDC int tc_qmap(int x) { return ((x >> 1) & 3) + 4 * ((x & 1) + 2 * (x >> 3)); }
PAC_HD int tc_slot(int x, bool useq) { return useq ? tc_qmap(x) : x; }
PAC_HDC bool tc_useq(int logell) { return logell >= 2 && logell <= 4; }

// cos and sin of 2 pi t / 16: the first-octant values of rot16 rotated by
// whole quarter turns
PAC_HD void tc_cs16(int t, float& c, float& s) {
  constexpr float H = 0.70710678118654752440f;   // cos(pi/4)
  constexpr float C1 = 0.92387953251128675613f;  // cos(pi/8)
  constexpr float S1 = 0.38268343236508977173f;  // sin(pi/8)
  const int r = t & 3, qd = (t >> 2) & 3;
  const float c0 = r == 0 ? 1.f : r == 1 ? C1 : r == 2 ? H : S1;
  const float s0 = r == 0 ? 0.f : r == 1 ? S1 : r == 2 ? H : C1;
  c = qd == 0 ? c0 : qd == 1 ? -s0 : qd == 2 ? -c0 : s0;
  s = qd == 0 ? s0 : qd == 1 ? c0 : qd == 2 ? -s0 : -c0;
}

// The DFT operand V of one lane, both MMA column halves h (columns 8h..8h+7):
// B registers of Re V, Im V and -Im V, hi and lo parts.
struct TcConst {
  uint32_t rh[2][2], rl[2][2];
  uint32_t ih[2][2], il[2][2];
  uint32_t nh[2][2], nl[2][2];
};

template <int B2, int SIGN, bool DIF>
PAC_HD void tc_const(int lane, bool useq, TcConst& wc) {
  const int g = lane >> 2, q = lane & 3;
  for (int h = 0; h < 2; ++h) {
    for (int r = 0; r < 2; ++r) {
      float vr[2], vi[2];
      for (int e = 0; e < 2; ++e) {
        const int sk = tc_slot(2 * q + e + 8 * r, useq);
        const int sc = tc_slot(g + 8 * h, useq);
        const int m = DIF ? sk : (int)drev<B2>((uint32_t)sk, 4);
        const int f = DIF ? (int)drev<B2>((uint32_t)sc, 4) : sc;
        float c, s;
        tc_cs16((m * f) & 15, c, s);
        vr[e] = c;
        vi[e] = SIGN < 0 ? -s : s;
      }
      tc_split2(vr[0], vr[1], wc.rh[h][r], wc.rl[h][r]);
      tc_split2(vi[0], vi[1], wc.ih[h][r], wc.il[h][r]);
      wc.nh[h][r] = wc.ih[h][r] ^ 0x80008000u;
      wc.nl[h][r] = wc.il[h][r] ^ 0x80008000u;
    }
  }
}

// The operands of every stage kind, built once per plan by tc_const into a
// device table (PassDesc.tcc, be_fill_tc_const): set (digit base 2 or 4,
// sign, DIF/DIT, slot map) x 32 lanes.  A stage loads its lane's 96 bytes
// instead of rebuilding them.
enum { TC_CONST_SETS = 16 };
PAC_HDC int tc_const_set(int b2, int sign, bool dif, bool useq) {
  return (((b2 - 1) * 2 + (sign > 0 ? 1 : 0)) * 2 + (dif ? 1 : 0)) * 2 + (useq ? 1 : 0);
}
// inverse of tc_const_set: fill entry `set` of the table for `lane`
PAC_HD void tc_const_fill(int set, int lane, TcConst& wc) {
  const bool useq = set & 1, dif = (set >> 1) & 1, pos = (set >> 2) & 1;
  const int b2 = (set >> 3) + 1;
  if (b2 == 1) {
    if (pos) dif ? tc_const<1, +1, true>(lane, useq, wc) : tc_const<1, +1, false>(lane, useq, wc);
    else dif ? tc_const<1, -1, true>(lane, useq, wc) : tc_const<1, -1, false>(lane, useq, wc);
  } else {
    if (pos) dif ? tc_const<2, +1, true>(lane, useq, wc) : tc_const<2, +1, false>(lane, useq, wc);
    else dif ? tc_const<2, -1, true>(lane, useq, wc) : tc_const<2, -1, false>(lane, useq, wc);
  }
}
PAC_HD void tc_const_load(const PassDesc& d, int set, int lane, TcConst& wc) {
  const TcConst* p = (const TcConst*)d.tcc + set * 32 + lane;
#if defined(__CUDA_ARCH__)
  static_assert(sizeof(TcConst) == 96, "6 x 16 bytes, one per member");
  const uint4* v = reinterpret_cast<const uint4*>(p);
  auto put = [](uint32_t(&m)[2][2], uint4 x) {
    m[0][0] = x.x;
    m[0][1] = x.y;
    m[1][0] = x.z;
    m[1][1] = x.w;
  };
  put(wc.rh, __ldg(v + 0));
  put(wc.rl, __ldg(v + 1));
  put(wc.ih, __ldg(v + 2));
  put(wc.il, __ldg(v + 3));
  put(wc.nh, __ldg(v + 4));
  put(wc.nl, __ldg(v + 5));
#else
  wc = *p;
#endif
}

// Shared-memory offset of the element ell * s past a butterfly's first
// element e0, for lines padded one element per 32 (sidx<float>, the layout
// of every tensor-core tile): sidx(e0 + ell s) = sidx(e0) + tc_soff(ell s),
// because e0 mod 32 + (ell s) mod 32 < 32 for the butterflies of a
// radix-16 stage: e0 = blk * 16 ell + j with j < ell; for ell >= 32 the
// second term is 0; for 2 <= ell < 32, e0 mod 32 = j <= ell - 1 and
// (ell s) mod 32 <= 32 - ell; for ell = 1, e0 mod 32 is 0 or 16 and s <= 15.
PAC_HD int tc_soff(int x) { return x + (x >> 5); }

// Per-lane state of one tile: butterflies g (bh = 0) and g + 8 (bh = 1).
struct TcLane {
  float xr[2][4], xi[2][4];  // inputs k = 2q + (kk & 1) + 8 (kk >> 1), kk = 0..3
  float mx[2];               // largest |re|, |im| of the butterfly's inputs
  int E[2];                  // input scale exponent
  uint32_t arh[4], arl[4], aih[4], ail[4];  // A registers: reg = bh + 2 * (kk >> 1)
  float yr[2][4], yi[2][4];  // D registers of column half h
  int w[2], e0[2], j[2];
  int sb[2];  // shared-memory index of the butterfly's first element
  bool ok[2];
};

// Load the lane's 8 inputs (global memory or shared), DIT pre-twiddles.
template <int B2, int SIGN, bool DIF, class SP>
PAC_HD void tc_load(const PassDesc& d, long long cta, const float* sre, const float* sim,
                    int logK, int twoff, int src, int dst, int lane, int tile, int nbf,
                    const long long* lbi, TcLane& t) {
  const int g = lane >> 2, q = lane & 3;
  const int logell = logK - 4, ell = 1 << logell;
  const bool useq = tc_useq(logell);
  const bool gf = src == IO_GLOBAL || dst == IO_GLOBAL;
  const float* ire = (const float*)d.in_re;
  const float* iim = (const float*)d.in_im;
  const Cx<float>* tw = (const Cx<float>*)d.tw + twoff;
  for (int bh = 0; bh < 2; ++bh) {
    const int u = tile * 16 + g + 8 * bh;
    int w = 0, blk = 0, j = 0;
    t.ok[bh] = u < nbf;
    if (t.ok[bh]) bf_coords<SP>(d, logK, 4, gf, u, &w, &blk, &j);
    const int e0 = (blk << logK) + j;
    t.w[bh] = w;
    t.j[bh] = j;
    t.e0[bh] = e0;
    t.sb[bh] = SP::template sm<float>(d, w, e0);
    float mx = 0.f;
    for (int kk = 0; kk < 4; ++kk) {
      const int s = tc_slot(2 * q + (kk & 1) + 8 * (kk >> 1), useq);
      Cx<float> v{0.f, 0.f};
      if (t.ok[bh]) {
        const int e = e0 + ell * s;
        if (src == IO_GLOBAL) {
          const long long gi = lbi[w] + ((long long)e << d.logS);
          v = Cx<float>{ld_g(ire + gi), ld_g(iim + gi)};
        } else {
          const int si = t.sb[bh] + tc_soff(ell * s);
          v = Cx<float>{sre[si], sim[si]};
        }
        if constexpr (!DIF) {
          const int m = (int)drev<B2>((uint32_t)s, 4);
          if (d.tw4 == 2 && logell == 0) v = ctw(v, tw4_value<float, B2, SP>(d, cta, w, e), SIGN);
          if (logell > 0 && j > 0 && m > 0) v = ctw(v, ld_tw(tw + j + (m - 1) * ell), SIGN);
        }
      }
      t.xr[bh][kk] = v.re;
      t.xi[bh][kk] = v.im;
      mx = fmaxf(mx, fmaxf(fabsf(v.re), fabsf(v.im)));
    }
    t.mx[bh] = mx;
  }
}

// Scale (after the quad reduction of mx) and split into the A registers.
PAC_HD void tc_split_lane(TcLane& t) {
  for (int bh = 0; bh < 2; ++bh) {
    const int ex = (int)((f32_bits(t.mx[bh]) >> 23) & 0xffu) - 127;  // -127 for 0 / subnormal
    int E = 14 - ex;
    E = E < -100 ? -100 : E > 100 ? 100 : E;
    t.E[bh] = E;
    const float sc = tc_pow2(E);
    for (int p = 0; p < 2; ++p) {
      const int r = bh + 2 * p;
      tc_split2(t.xr[bh][2 * p] * sc, t.xr[bh][2 * p + 1] * sc, t.arh[r], t.arl[r]);
      tc_split2(t.xi[bh][2 * p] * sc, t.xi[bh][2 * p + 1] * sc, t.aih[r], t.ail[r]);
    }
  }
}

// Unscale, DIF post-twiddles, store the lane's 8 outputs.
template <int B2, int SIGN, bool DIF, class SP>
PAC_HD void tc_store(const PassDesc& d, long long cta, float* sre, float* sim, int logK,
                     int twoff, int dst, int lane, const TcLane& t, const long long* lbo) {
  const int q = lane & 3;
  const int logell = logK - 4, ell = 1 << logell;
  const bool useq = tc_useq(logell);
  float* ore = (float*)d.out_re;
  float* oim = (float*)d.out_im;
  const Cx<float>* tw = (const Cx<float>*)d.tw + twoff;
  for (int h = 0; h < 2; ++h) {
    for (int i = 0; i < 4; ++i) {
      const int bh = i >> 1;
      if (!t.ok[bh]) continue;
      const int s = tc_slot(2 * q + (i & 1) + 8 * h, useq);
      const float us = tc_pow2(-t.E[bh]);
      Cx<float> v{t.yr[h][i] * us, t.yi[h][i] * us};
      const int w = t.w[bh], j = t.j[bh];
      const int e = t.e0[bh] + ell * s;
      if constexpr (DIF) {
        const int f = (int)drev<B2>((uint32_t)s, 4);
        if (logell > 0 && j > 0 && f > 0) v = ctw(v, ld_tw(tw + j + (f - 1) * ell), SIGN);
        if (d.tw4 == 1 && logell == 0) v = ctw(v, tw4_value<float, B2, SP>(d, cta, w, e), SIGN);
      }
      if (dst == IO_GLOBAL) {
        if (d.use_scale) {
          v.re *= float(d.scale);
          v.im *= float(d.scale);
        }
        const long long gi = lbo[w] + ((long long)e << d.logS);
        ore[gi] = v.re;
        oim[gi] = v.im;
      } else {
        const int si = t.sb[bh] + tc_soff(ell * s);
        sre[si] = v.re;
        sim[si] = v.im;
      }
    }
  }
}

#if defined(__CUDA_ARCH__)
__device__ __forceinline__ void tc_mma(float (&c)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Y = X V for one lane: small products first
__device__ __forceinline__ void tc_mma_lane(TcLane& t, const TcConst& wc) {
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    float(&yr)[4] = t.yr[h];
    float(&yi)[4] = t.yi[h];
#pragma unroll
    for (int i = 0; i < 4; ++i) yr[i] = yi[i] = 0.f;
    tc_mma(yr, t.arl, wc.rh[h]);
    tc_mma(yr, t.arh, wc.rl[h]);
    tc_mma(yr, t.ail, wc.nh[h]);
    tc_mma(yr, t.aih, wc.nl[h]);
    tc_mma(yr, t.arh, wc.rh[h]);
    tc_mma(yr, t.aih, wc.nh[h]);
    tc_mma(yi, t.arl, wc.ih[h]);
    tc_mma(yi, t.arh, wc.il[h]);
    tc_mma(yi, t.ail, wc.rh[h]);
    tc_mma(yi, t.aih, wc.rl[h]);
    tc_mma(yi, t.arh, wc.ih[h]);
    tc_mma(yi, t.aih, wc.rh[h]);
  }
}
#else
// Host model of one warp-wide m16n8k16 MMA, D = A B + D, from the fragment
// layouts: products exact, each MMA's sum formed in FP64 and rounded once.
template <int N>
inline void tc_mma_host(TcLane (&t)[32], const TcConst (&wc)[32], uint32_t (TcLane::*A)[N],
                             uint32_t (TcConst::*B)[2][2], int h, float (TcLane::*D)[2][4]) {
  float a[16][16], b[16][8];
  for (int lane = 0; lane < 32; ++lane) {
    const int g = lane >> 2, q = lane & 3;
    const uint32_t* ar = t[lane].*A;
    for (int r = 0; r < 4; ++r) {
      float lo, hi;
      tc_unpack(ar[r], lo, hi);
      const int row = g + 8 * (r & 1), col = 2 * q + 8 * (r >> 1);
      a[row][col] = lo;
      a[row][col + 1] = hi;
    }
    for (int r = 0; r < 2; ++r) {
      float lo, hi;
      tc_unpack((wc[lane].*B)[h][r], lo, hi);
      b[2 * q + 8 * r][g] = lo;
      b[2 * q + 8 * r + 1][g] = hi;
    }
  }
  for (int lane = 0; lane < 32; ++lane) {
    const int g = lane >> 2, q = lane & 3;
    float* dd = (t[lane].*D)[h];
    for (int i = 0; i < 4; ++i) {
      const int row = g + 8 * (i >> 1), col = 2 * q + (i & 1);
      double acc = dd[i];
      for (int k = 0; k < 16; ++k) acc += (double)a[row][k] * (double)b[k][col];
      dd[i] = (float)acc;
    }
  }
}

inline void tc_mma_warp_host(TcLane (&t)[32], const TcConst (&wc)[32]) {
  for (int h = 0; h < 2; ++h) {
    for (int lane = 0; lane < 32; ++lane)
      for (int i = 0; i < 4; ++i) t[lane].yr[h][i] = t[lane].yi[h][i] = 0.f;
    tc_mma_host(t, wc, &TcLane::arl, &TcConst::rh, h, &TcLane::yr);
    tc_mma_host(t, wc, &TcLane::arh, &TcConst::rl, h, &TcLane::yr);
    tc_mma_host(t, wc, &TcLane::ail, &TcConst::nh, h, &TcLane::yr);
    tc_mma_host(t, wc, &TcLane::aih, &TcConst::nl, h, &TcLane::yr);
    tc_mma_host(t, wc, &TcLane::arh, &TcConst::rh, h, &TcLane::yr);
    tc_mma_host(t, wc, &TcLane::aih, &TcConst::nh, h, &TcLane::yr);
    tc_mma_host(t, wc, &TcLane::arl, &TcConst::ih, h, &TcLane::yi);
    tc_mma_host(t, wc, &TcLane::arh, &TcConst::il, h, &TcLane::yi);
    tc_mma_host(t, wc, &TcLane::ail, &TcConst::rh, h, &TcLane::yi);
    tc_mma_host(t, wc, &TcLane::aih, &TcConst::rl, h, &TcLane::yi);
    tc_mma_host(t, wc, &TcLane::arh, &TcConst::ih, h, &TcLane::yi);
    tc_mma_host(t, wc, &TcLane::aih, &TcConst::rh, h, &TcLane::yi);
  }
}
#endif

// One radix-16 stage of nbf butterflies on the tensor cores.  Device: warp
// k of the CTA takes tiles k, k + nwarps, ...; every lane of a warp runs
// the same number of tiles (the MMAs are warp-wide), and lanes whose
// butterfly lies beyond nbf load zeros and store nothing.  Host: the tiles
// in turn, the 32 lanes of each emulated.
template <int B2, int SIGN, bool DIF, class SP, int CLOGK>
PAC_HD void stage_tc(const PassDesc& d, long long cta, float* sre, float* sim, int logK_rt,
                     int twoff, int src, int dst, int nbf, const long long* lbi,
                     const long long* lbo) {
  const int logK = CLOGK >= 0 ? CLOGK : logK_rt;
  const bool useq = tc_useq(logK - 4);
  const int ntiles = (nbf + 15) >> 4;
#if defined(__CUDA_ARCH__)
  const int lane = (int)threadIdx.x & 31;
  TcConst wc;
  tc_const_load(d, tc_const_set(B2, SIGN, DIF, useq), lane, wc);
  for (int tile = (int)threadIdx.x >> 5; tile < ntiles; tile += (int)blockDim.x >> 5) {
    TcLane t;
    tc_load<B2, SIGN, DIF, SP>(d, cta, sre, sim, logK, twoff, src, dst, lane, tile, nbf, lbi, t);
#pragma unroll
    for (int bh = 0; bh < 2; ++bh) {
      t.mx[bh] = fmaxf(t.mx[bh], __shfl_xor_sync(0xffffffffu, t.mx[bh], 1));
      t.mx[bh] = fmaxf(t.mx[bh], __shfl_xor_sync(0xffffffffu, t.mx[bh], 2));
    }
    tc_split_lane(t);
    tc_mma_lane(t, wc);
    tc_store<B2, SIGN, DIF, SP>(d, cta, sre, sim, logK, twoff, dst, lane, t, lbo);
  }
#else
  TcConst wc[32];
  for (int lane = 0; lane < 32; ++lane)
    tc_const_load(d, tc_const_set(B2, SIGN, DIF, useq), lane, wc[lane]);
  for (int tile = 0; tile < ntiles; ++tile) {
    TcLane t[32];
    for (int lane = 0; lane < 32; ++lane)
      tc_load<B2, SIGN, DIF, SP>(d, cta, sre, sim, logK, twoff, src, dst, lane, tile, nbf, lbi,
                                 t[lane]);
    for (int g = 0; g < 8; ++g)
      for (int bh = 0; bh < 2; ++bh) {
        float m = 0.f;
        for (int q = 0; q < 4; ++q) m = fmaxf(m, t[4 * g + q].mx[bh]);
        for (int q = 0; q < 4; ++q) t[4 * g + q].mx[bh] = m;
      }
    for (int lane = 0; lane < 32; ++lane) tc_split_lane(t[lane]);
    tc_mma_warp_host(t, wc);
    for (int lane = 0; lane < 32; ++lane)
      tc_store<B2, SIGN, DIF, SP>(d, cta, sre, sim, logK, twoff, dst, lane, t[lane], lbo);
  }
#endif
}

}  // namespace pac
