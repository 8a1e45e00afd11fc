// pac_stages.cuh -- butterfly stages and pass bodies of the engine.
//
// One radix-R butterfly of a stage:
//   DIF: load x[m] @ j + ell*m, DFT, twiddle output s by w_K^{j s},
//        store @ j + ell*sigma_b(s)
//   DIT: load x[s] @ j + ell*sigma_b(s), twiddle by w_K^{j s}, DFT,
//        store @ j + ell*m
// Global-facing stages read (first) or write (last) the line in global
// memory; all other accesses go to the padded shared-memory line.
//
// The same stage code serves two kinds of kernels through a shape policy:
// the generic kernel reads every geometry value (line length, tile width,
// pitch, stride kind) from the PassDesc at run time; a specialised kernel
// fixes them at compile time together with its radix schedule, so the index
// arithmetic folds into constants.
#pragma once

namespace pac {

enum { IO_SMEM = 0, IO_GLOBAL = 1 };

// FP32 column tiles of 8 lines pad every line by one element per 8 plus 8
// per 128 (sidx_col32): their three stage patterns -- 8 lines x 4
// consecutive rows (the stage next to global memory), 4 blocks of 128 x 8
// butterflies of one line (the middle stage), 8 lines x 4 blocks of 8 (the
// innermost stage) -- then fall on 32 distinct banks, which one pad element
// per 32 leaves 2-way conflicted.
PAC_HDC bool col_pad32(int bytes, int cols, int W) { return bytes == 4 && cols == 1 && W == 8; }
PAC_HD int sidx_col32(int e) { return e + (e >> 3) + 8 * (e >> 7); }

// FP32 row tiles of 256-point lines (2 <= W <= 16) pad every line by one element
// per 16 and start each line 16 banks after the previous one (pitch 272):
// both radix-16 stages give a warp 16 butterflies of each of two lines --
// 16 consecutive elements per line (j + 16m) in the outer stage, a stride of
// 16 (16 blk + m) in the inner one -- and with this pad and pitch the two
// lines fall on complementary halves of the 32 banks in both, where the
// one-per-32 pad left every access 2-way conflicted.  (Not for the plane
// pass's 32-row tiles, whose transposed stages read 32 consecutive columns
// of a row and keep the one-per-32 pad.)
PAC_HDC bool row_pad16(int bytes, int cols, int logL, int W) {
  return bytes == 4 && cols == 0 && logL == 8 && W >= 2 && W <= 16;
}
PAC_HD int sidx_row16(int e) { return e + (e >> 4); }

// FP32 row tiles of 128-point lines (2 <= W <= 16): the radix-16 stage gives
// a warp 8 butterflies of each of four lines (j + 8m), the radix-8 stage 16
// of each of two lines (8 blk + m).  Lines of pitch 136 with the one-per-32
// pad, and bit 2 of the element index flipped in odd lines, put every such
// access on 32 distinct banks (the pitch alone left the first stage 4-way
// conflicted; no pitch does better than 2-way without the flip).
PAC_HDC bool row_swz128(int bytes, int cols, int logL, int W) {
  return bytes == 4 && cols == 0 && logL == 7 && W >= 2 && W <= 16;
}

// FP32 columns of 512 points in 16-line tiles (schedule 8, 8, 8; pitch 546,
// two banks per line): the middle stage gives a warp 8 consecutive j in each
// of 4 blocks of 64 of one line (4-way conflicted with the one-per-32 pad),
// the last stage 2 consecutive blocks of 8 in each of the 16 lines (2-way).
// Bit 0 flipped by bit 3, then bits 3-4 by bits 6-7 (the middle stage's block
// index), make all three stages conflict-free; the generic pad's pitch is
// kept.
PAC_HDC bool col_swz512(int bytes, int cols, int logL, int W) {
  return bytes == 4 && cols == 1 && logL == 9 && W == 16;
}
PAC_HD int sidx_col512(int e) {
  const int t = e ^ ((e >> 3) & 1);
  return t ^ (((t >> 6) & 3) << 3);
}

// geometry policy; -1 = read from the PassDesc at run time.  TCL_ = 1: a
// tile of the tensor-core form, whose column tiles keep the one-per-32 pad
// (pitch_for gives them an odd pitch instead of sidx_col32).  TR_ = 1: the
// lines are the columns of a row-major shared-memory tile (element e of
// line w at e * PITCH + sidx(w)), and consecutive threads always take
// consecutive lines (the plane passes' local axis-1 stages)
template <int LOGL_ = -1, int LOGW_ = -1, int PITCH_ = -1, int COLS_ = -1, int TCL_ = 0,
          int TR_ = 0>
struct Shape {
  static constexpr int kLogL = LOGL_;
  static constexpr int kLogW = LOGW_;
  static constexpr int kPitch = PITCH_;
  static constexpr int kCols = COLS_;
  static PAC_HD int logL(const PassDesc& d) {
    if constexpr (LOGL_ >= 0) return LOGL_;
    else return d.logL;
  }
  static PAC_HD int logW(const PassDesc& d) {
    if constexpr (LOGW_ >= 0) return LOGW_;
    else return d.logW;
  }
  static PAC_HD int W(const PassDesc& d) { return 1 << logW(d); }
  static PAC_HD int pitch(const PassDesc& d) {
    if constexpr (PITCH_ >= 0) return PITCH_;
    else return d.pitch;
  }
  // lines of the tile are consecutive columns (element stride S > 1)
  static PAC_HD bool cols(const PassDesc& d) {
    if constexpr (COLS_ >= 0) return COLS_ != 0;
    else return d.logS > 0;
  }
  // threads take consecutive lines first: only where a stage touches global
  // memory of a column tile (coalesced rows of W elements)
  static PAC_HD bool wfast(const PassDesc& d, bool global_facing) {
    if constexpr (TR_) return true;
    else return global_facing && cols(d);
  }
  // shared-memory index of element e of line w: padded lines
  template <typename T>
  static PAC_HD int sm(const PassDesc& d, int w, int e) {
    if constexpr (TR_)
      return e * pitch(d) + sidx<T>(w);
    else if constexpr (!TCL_ && col_pad32((int)sizeof(T), COLS_, LOGW_ >= 0 ? 1 << LOGW_ : 0))
      return w * pitch(d) + sidx_col32(e);
    else if constexpr (!TCL_ && row_pad16((int)sizeof(T), COLS_, LOGL_, LOGW_ >= 0 ? 1 << LOGW_ : 0))
      return w * pitch(d) + sidx_row16(e);
    else if constexpr (!TCL_ && row_swz128((int)sizeof(T), COLS_, LOGL_, LOGW_ >= 0 ? 1 << LOGW_ : 0))
      return w * pitch(d) + sidx<T>(e ^ ((w & 1) << 2));
    else if constexpr (!TCL_ && col_swz512((int)sizeof(T), COLS_, LOGL_, LOGW_ >= 0 ? 1 << LOGW_ : 0))
      return w * pitch(d) + sidx_col512(e);
    else
      return w * pitch(d) + sidx<T>(e);
  }
};
using RtShape = Shape<>;

// butterfly index -> (w, blk, j) for a stage of block 2^logK, radix 2^logR
template <class SP>
PAC_HD void bf_coords(const PassDesc& d, int logK, int logR, bool global_facing, int u, int* w,
                      int* blk, int* j) {
  const int lbf = SP::logL(d) - logR;  // butterflies per line (log)
  const int logell = logK - logR;
  int v;
  if (SP::wfast(d, global_facing)) {
    // consecutive threads take consecutive columns: coalesced rows of W
    *w = u & (SP::W(d) - 1);
    v = u >> SP::logW(d);
  } else {
    v = u & ((1 << lbf) - 1);
    *w = u >> lbf;
  }
  *blk = v >> logell;
  *j = v & ((1 << logell) - 1);
}

// The 4-step twiddle w_N^{iG * rev_b(e)} of line w at element e.
template <typename T, int B2, class SP>
PAC_HD Cx<T> tw4_value(const PassDesc& d, long long cta, int w, int e) {
  long long g = cta * SP::W(d) + w;
  long long i = g & ((1LL << d.logS) - 1);
  uint32_t iG = (uint32_t)((i >> d.tw4_shift) & d.tw4_mask);
  uint32_t E = iG * drev<B2>((uint32_t)e, SP::logL(d));
  const Cx<T>* lo = (const Cx<T>*)d.tw4_lo;
  const Cx<T>* hi = (const Cx<T>*)d.tw4_hi;
  return cmul(ld_tw(lo + (E & ((1u << d.tw4_lolog) - 1))), ld_tw(hi + (E >> d.tw4_lolog)));
}

// The stage twiddles w_K^{j s}, s = 1 .. R-1, of a butterfly with index j
// (tw points at entry j of the stage table, which is s-major: entry
// (s-1)*ell + j).  FP64 reads only the powers of two w^j, w^2j, w^4j, w^8j
// and forms every other power as a product of two already formed ones
// (w^s = w^hb * w^(s-hb), hb the highest power of two in s: at most three
// roundings deep, ~1e-15 relative) -- a load per twiddle costs more issue
// slots and load-queue space than the FP64 product, whose pipe the passes
// leave mostly idle.  FP32 reads every entry: its table values are rounded
// once from FP64 and are used as they are.
template <typename T, int R>
PAC_HD void stage_twiddles(const Cx<T>* tw, int ell, Cx<T> (&w)[R]) {
  if constexpr (sizeof(T) == 8 && R >= 4) {
    static_for<ilog2(R)>([&](auto b) {
      constexpr int s = 1 << b.value;
      w[s] = ld_tw(tw + (s - 1) * ell);
    });
    static_for<R>([&](auto ss) {
      constexpr int s = ss.value;
      if constexpr (s > 2 && (s & (s - 1)) != 0) {
        constexpr int hb = 1 << ilog2(s);
        w[s] = cmul(w[hb], w[s - hb]);
      }
    });
  } else {
    static_for<R - 1>([&](auto ss) {
      constexpr int s = ss.value + 1;
      w[s] = ld_tw(tw + (s - 1) * ell);
    });
  }
}

// The same twiddles from a compact copy of the table's rows (a CTA's
// shared-memory copy, see ColTma::tw_fill): row r holds w_K^{j s(r)} for
// the ell values of j, s(r) = 2^r in FP64 at radix >= 4 (the rows
// stage_twiddles reads; the other factors are products), else r + 1.
template <typename T, int R>
PAC_HD void stage_twiddles_c(const Cx<T>* tws, int ell, Cx<T> (&w)[R]) {
  if constexpr (sizeof(T) == 8 && R >= 4) {
    static_for<ilog2(R)>([&](auto b) { w[1 << b.value] = tws[b.value * ell]; });
    static_for<R>([&](auto ss) {
      constexpr int s = ss.value;
      if constexpr (s > 2 && (s & (s - 1)) != 0) {
        constexpr int hb = 1 << ilog2(s);
        w[s] = cmul(w[hb], w[s - hb]);
      }
    });
  } else {
    static_for<R - 1>([&](auto ss) { w[ss.value + 1] = tws[ss.value * ell]; });
  }
}

// The arithmetic of one radix-R butterfly on registers x: DIT pre-twiddles,
// the R-point DFT, DIF post-twiddles.  x[m] holds the element at input slot
// m (DIF: m, DIT: sigma_b(m)); afterwards register p holds output index
// brev(p).  e0 is the butterfly's first element, j its index in the block,
// w its line, ell = 2^logell the element stride.  With tws the stage
// twiddles come from that compact copy of the stage's rows instead of the
// table in global memory.
template <typename T, int B2, int R, int SIGN, bool DIF, class SP>
PAC_HD void bf_math(const PassDesc& d, long long cta, Cx<T> (&x)[R], int w, int e0, int j,
                    int logell, int twoff, const Cx<T>* tws = nullptr) {
  constexpr int LR = ilog2(R);
  const int ell = 1 << logell;
  // stage table, s-major: entry (s-1)*ell + j = w_K^{j s}; for one s the
  // threads of a warp read consecutive j (coalesced)
  const Cx<T>* tw = (const Cx<T>*)d.tw + twoff + j;
  const bool twiddle = logell > 0 && j > 0;
  if constexpr (!DIF) {
    // 4-step pre-twiddle: only the innermost stage (ell == 1) of a DIT pass
    if (d.tw4 == 2 && logell == 0) {
      static_for<R>([&](auto mm) {
        constexpr int slot = drev_c(mm.value, LR, B2);
        x[mm.value] = ctw(x[mm.value], tw4_value<T, B2, SP>(d, cta, w, e0 + slot), SIGN);
      });
    }
    if (twiddle) {
      Cx<T> wv[R];
      if (tws) stage_twiddles_c<T, R>(tws + j, ell, wv);
      else stage_twiddles<T, R>(tw, ell, wv);
      static_for<R - 1>([&](auto ss) {
        constexpr int s = ss.value + 1;
        x[s] = ctw(x[s], wv[s], SIGN);
      });
    }
  }
  dft_reg<T, R, SIGN>(x);
  // register p now holds output index brev(p)
  if constexpr (DIF) {
    if (twiddle) {
      Cx<T> wv[R];
      if (tws) stage_twiddles_c<T, R>(tws + j, ell, wv);
      else stage_twiddles<T, R>(tw, ell, wv);
      static_for<R>([&](auto pp) {
        constexpr int s = brev_c(pp.value, LR);
        if constexpr (s > 0) x[pp.value] = ctw(x[pp.value], wv[s], SIGN);
      });
    }
    // 4-step post-twiddle: only the innermost stage of a DIF pass
    if (d.tw4 == 1 && logell == 0) {
      static_for<R>([&](auto pp) {
        constexpr int slot = drev_c(brev_c(pp.value, LR), LR, B2);
        x[pp.value] = ctw(x[pp.value], tw4_value<T, B2, SP>(d, cta, w, e0 + slot), SIGN);
      });
    }
  }
}

// One butterfly.  CLOGK >= 0 fixes the stage's block size at compile time.
template <typename T, int B2, int R, int SIGN, bool DIF, class SP, int CLOGK>
PAC_HD void stage_bf(const PassDesc& d, long long cta, T* sre, T* sim, int logK_rt, int twoff,
                     int src, int dst, int u, const long long* lbase_in,
                     const long long* lbase_out) {
  constexpr int LR = ilog2(R);
  static_assert(LR % B2 == 0, "radix must be a power of the digit base");
  const int logK = CLOGK >= 0 ? CLOGK : logK_rt;
  const int logell = logK - LR;
  int w, blk, j;
  bf_coords<SP>(d, logK, LR, src == IO_GLOBAL || dst == IO_GLOBAL, u, &w, &blk, &j);
  if constexpr (sizeof(T) == 4 && SP::kCols == 0 && CLOGK >= 0) {
    // FP32 rows, shared-memory stages of stride 8: a warp takes 8 blocks x 4
    // butterflies instead of 4 x 8, so that its addresses 128 blk + j + 8 m
    // (pad one per 32) fall on the distinct banks j + 4 blk
    if constexpr (CLOGK - LR == 3 && SP::kLogL - CLOGK >= 3) {
      if (src != IO_GLOBAL && dst != IO_GLOBAL) {
        const int lbf = SP::kLogL - LR;
        const int v = u & ((1 << lbf) - 1), hi = v >> 5;
        w = u >> lbf;
        j = (v & 3) + 4 * (hi & 1);
        blk = ((v >> 2) & 7) + 8 * (hi >> 1);
      }
    }
  }
  const int ell = 1 << logell;
  const int e0 = (blk << logK) + j;
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
      int si = SP::template sm<T>(d, w, e);
      x[m] = Cx<T>{sre[si], sim[si]};
    }
  });
  bf_math<T, B2, R, SIGN, DIF, SP>(d, cta, x, w, e0, j, logell, twoff);
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
      int si = SP::template sm<T>(d, w, e);
      sre[si] = v.re;
      sim[si] = v.im;
    }
  });
}

// Convolution middle: the last DIF stage (ell == 1), the pointwise product
// with the filter spectrum at the same P_b positions, and the first DIT
// stage, all in registers.
template <typename T, int B2, int R, class SP>
PAC_HD void middle_bf(const PassDesc& d, T* sre, T* sim, int src, int dst, int u,
                      const long long* lbase) {
  constexpr int LR = ilog2(R);
  int w, blk, j;
  bf_coords<SP>(d, LR, LR, src == IO_GLOBAL || dst == IO_GLOBAL, u, &w, &blk, &j);
  const int e0 = blk << LR;  // ell == 1, j == 0
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
      int si = SP::template sm<T>(d, w, e);
      x[m] = Cx<T>{sre[si], sim[si]};
    }
  });
  dft_reg<T, R, -1>(x);
  // register p holds the spectrum at slot sigma_b(brev(p)); the DIT stage
  // wants register s = the value at slot sigma_b(s), i.e. register brev(s).
  Cx<T> y[R];
  const T sc = T(d.scale);
  // The filter spectrum is in plan order: P_b order of the line with every
  // block of R positions transposed to stride L/R, i.e. P-order slot
  // blk*R + t sits at t*(L/R) + blk.  For a fixed register s the threads of
  // a warp (consecutive blk) then read consecutive addresses.  This pass
  // always runs on the contiguous innermost factor (element stride 1).
  const int lq = SP::logL(d) - LR;
  static_for<R>([&](auto ss) {
    constexpr int s = ss.value;
    constexpr int p = brev_c(s, LR);
    constexpr int t = drev_c(s, LR, B2);
    long long hi = (lbase[w] + ((long long)t << lq) + (e0 >> LR)) & d.h_mask;
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
      int si = SP::template sm<T>(d, w, e);
      sre[si] = y[p].re;
      sim[si] = y[p].im;
    }
  });
}

}  // namespace pac
#include "pac_tc.cuh"
namespace pac {

// ---------------------------------------------------------------------------
// Phases: a loop over butterflies; the device runs it with one butterfly per
// thread, the host emulator with a plain loop.  Barriers separate a phase
// that writes shared memory from the next phase that reads it.
// ---------------------------------------------------------------------------
#if defined(__CUDA_ARCH__)
#define PAC_FOR_BF(n, u) for (int u = (int)threadIdx.x; u < (n); u += (int)blockDim.x)
#define PAC_SYNC() __syncthreads()
#else
#define PAC_FOR_BF(n, u) for (int u = 0; u < (n); ++u)
#define PAC_SYNC() ((void)0)
#endif

// ---------------------------------------------------------------------------
// Generic pass body: geometry and radix schedule at run time
// ---------------------------------------------------------------------------
template <typename T, int B2, bool DIF>
PAC_HD void stage_dispatch(const PassDesc& d, long long cta, T* sre, T* sim, int logK, int logR,
                           int twoff, int sign, int src, int dst, int u, const long long* lbi,
                           const long long* lbo) {
#define PAC_ST(RR)                                                                     \
  if (sign < 0)                                                                        \
    stage_bf<T, B2, RR, -1, DIF, RtShape, -1>(d, cta, sre, sim, logK, twoff, src, dst, u, \
                                              lbi, lbo);                               \
  else                                                                                 \
    stage_bf<T, B2, RR, +1, DIF, RtShape, -1>(d, cta, sre, sim, logK, twoff, src, dst, u, \
                                              lbi, lbo);
  if constexpr (B2 == 1) {
    switch (logR) {
      case 1: PAC_ST(2) break;
      case 2: PAC_ST(4) break;
      case 3: PAC_ST(8) break;
      default: PAC_ST(16) break;
    }
  } else if constexpr (B2 == 2) {
    if (logR == 2) {
      PAC_ST(4)
    } else {
      PAC_ST(16)
    }
  } else {
    PAC_ST(8)
  }
#undef PAC_ST
}

template <typename T, int B2>
PAC_HD void middle_dispatch(const PassDesc& d, T* sre, T* sim, int logR, int src, int dst, int u,
                            const long long* lb) {
  if constexpr (B2 == 1) {
    switch (logR) {
      case 1: middle_bf<T, B2, 2, RtShape>(d, sre, sim, src, dst, u, lb); break;
      case 2: middle_bf<T, B2, 4, RtShape>(d, sre, sim, src, dst, u, lb); break;
      case 3: middle_bf<T, B2, 8, RtShape>(d, sre, sim, src, dst, u, lb); break;
      default: middle_bf<T, B2, 16, RtShape>(d, sre, sim, src, dst, u, lb); break;
    }
  } else if constexpr (B2 == 2) {
    if (logR == 2) middle_bf<T, B2, 4, RtShape>(d, sre, sim, src, dst, u, lb);
    else middle_bf<T, B2, 16, RtShape>(d, sre, sim, src, dst, u, lb);
  } else {
    middle_bf<T, B2, 8, RtShape>(d, sre, sim, src, dst, u, lb);
  }
}

// Tensor-core form (PassDesc.tc; the generic kernels are instantiated with
// TC = 1 for it): radix-16 stages of FP32 passes run on the tensor cores
// (stage_tc); every other stage and the convolution middle stay on the CUDA
// cores.
template <typename T, int TC>
PAC_HD bool tc_stage(int logR) {
  return TC && sizeof(T) == 4 && logR == 4;
}
template <typename T, int B2, bool DIF>
PAC_HD void stage_tc_rt(const PassDesc& d, long long cta, T* sre, T* sim, int logK, int twoff,
                        int sign, int src, int dst, int nbf, const long long* lbi,
                        const long long* lbo) {
  if constexpr (sizeof(T) == 4 && B2 != 3) {
    if (sign < 0)
      stage_tc<B2, -1, DIF, RtShape, -1>(d, cta, sre, sim, logK, twoff, src, dst, nbf, lbi, lbo);
    else
      stage_tc<B2, +1, DIF, RtShape, -1>(d, cta, sre, sim, logK, twoff, src, dst, nbf, lbi, lbo);
  }
}

// block size (log) of stage i of the DIF order: L / (R_0 ... R_{i-1})
PAC_HD int stage_logK(const PassDesc& d, int i) {
  int logK = d.logL;
  for (int q = 0; q < i; ++q) logK -= d.rlog[q];
  return logK;
}

template <typename T, int B2, int TC = 0>
PAC_HD void pass_body(const PassDesc& d, long long cta, T* sre, T* sim, const long long* lbi,
                      const long long* lbo) {
  const bool nat = d.nat != 0;
  const int nst = d.nst;
  if (d.mode == MODE_DIF) {
    for (int i = 0; i < nst; ++i) {
      int logK = stage_logK(d, i), logR = d.rlog[i];
      int src = (i == 0) ? IO_GLOBAL : IO_SMEM;
      int dst = (i == nst - 1 && !nat) ? IO_GLOBAL : IO_SMEM;
      int nbf = d.W << (d.logL - logR);
      if (i > 0) PAC_SYNC();
      if (tc_stage<T, TC>(logR)) {
        stage_tc_rt<T, B2, true>(d, cta, sre, sim, logK, d.tw_off[i], d.sign, src, dst, nbf, lbi,
                                 lbo);
        continue;
      }
      PAC_FOR_BF(nbf, u) {
        stage_dispatch<T, B2, true>(d, cta, sre, sim, logK, logR, d.tw_off[i], d.sign, src, dst, u,
                                    lbi, lbo);
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
      int logK = stage_logK(d, i), logR = d.rlog[i];
      int src = (k == 0) ? IO_GLOBAL : IO_SMEM;
      int dst = (k == nst - 1) ? IO_GLOBAL : IO_SMEM;
      int nbf = d.W << (d.logL - logR);
      if (k > 0) PAC_SYNC();
      if (tc_stage<T, TC>(logR)) {
        stage_tc_rt<T, B2, false>(d, cta, sre, sim, logK, d.tw_off[i], d.sign, src, dst, nbf, lbi,
                                  lbo);
        continue;
      }
      PAC_FOR_BF(nbf, u) {
        stage_dispatch<T, B2, false>(d, cta, sre, sim, logK, logR, d.tw_off[i], d.sign, src, dst,
                                     u, lbi, lbo);
      }
    }
  } else {  // MODE_CONV
    for (int i = 0; i < nst - 1; ++i) {
      int logK = stage_logK(d, i), logR = d.rlog[i];
      int src = (i == 0) ? IO_GLOBAL : IO_SMEM;
      int nbf = d.W << (d.logL - logR);
      if (i > 0) PAC_SYNC();
      if (tc_stage<T, TC>(logR)) {
        stage_tc_rt<T, B2, true>(d, cta, sre, sim, logK, d.tw_off[i], -1, src, IO_SMEM, nbf, lbi,
                                 lbo);
        continue;
      }
      PAC_FOR_BF(nbf, u) {
        stage_dispatch<T, B2, true>(d, cta, sre, sim, logK, logR, d.tw_off[i], -1, src, IO_SMEM,
                                    u, lbi, lbo);
      }
    }
    {
      int logR = d.rlog[nst - 1];
      int src = (nst == 1) ? IO_GLOBAL : IO_SMEM;
      int dst = (nst == 1) ? IO_GLOBAL : IO_SMEM;
      int nbf = d.W << (d.logL - logR);
      if (nst > 1) PAC_SYNC();
      PAC_FOR_BF(nbf, u) { middle_dispatch<T, B2>(d, sre, sim, logR, src, dst, u, lbi); }
    }
    for (int i = nst - 2; i >= 0; --i) {
      int logK = stage_logK(d, i), logR = d.rlog[i];
      int dst = (i == 0) ? IO_GLOBAL : IO_SMEM;
      int nbf = d.W << (d.logL - logR);
      PAC_SYNC();
      if (tc_stage<T, TC>(logR)) {
        stage_tc_rt<T, B2, false>(d, cta, sre, sim, logK, d.tw_off[i], +1, IO_SMEM, dst, nbf, lbi,
                                  lbo);
        continue;
      }
      PAC_FOR_BF(nbf, u) {
        stage_dispatch<T, B2, false>(d, cta, sre, sim, logK, logR, d.tw_off[i], +1, IO_SMEM, dst,
                                     u, lbi, lbo);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Specialised pass body: shape and radix schedule fixed at compile time
// (RL = radix logs in DIF order, outermost first).  DIF, DIT and CONV.
// ---------------------------------------------------------------------------
template <int... RL>
struct Rads {
  static constexpr int n = sizeof...(RL);
  static constexpr int v[n] = {RL...};
  // block size (log) of stage i
  static PAC_HDC int logK(int logL, int i) {
    int k = logL;
    for (int q = 0; q < i; ++q) k -= v[q];
    return k;
  }
};

#if defined(__CUDA_ARCH__)
#define PAC_FOR_BF_CT(n, NT, u)                                        \
  _Pragma("unroll") for (int u##_base = 0; u##_base < (n); u##_base += (NT)) \
    for (int u = u##_base + (int)threadIdx.x; u < u##_base + (NT) && u < (n); u += (NT))
#else
#define PAC_FOR_BF_CT(n, NT, u) for (int u = 0; u < (n); ++u)
#endif

template <typename T, int B2, int MODE, int SIGN, class SP, int NT, class RS, int TC = 0>
PAC_HD void pass_body_ct(const PassDesc& d, long long cta, T* sre, T* sim, const long long* lbi,
                         const long long* lbo) {
  static_assert(!TC || sizeof(T) == 4, "the tensor-core form stores FP32");
  constexpr int GIO = IO_GLOBAL;
  constexpr int LOGL = SP::kLogL;
  constexpr int LOGW = SP::kLogW;
  static_assert(LOGL >= 0 && LOGW >= 0 && SP::kPitch >= 0 && SP::kCols >= 0, "fixed shape");
  constexpr int n = RS::n;
  if constexpr (MODE == MODE_DIF) {
    static_for<n>([&](auto ii) {
      constexpr int i = ii.value;
      constexpr int LK = RS::logK(LOGL, i);
      constexpr int LRr = RS::v[i];
      constexpr int nbf = 1 << (LOGW + LOGL - LRr);
      if constexpr (i > 0) PAC_SYNC();
      if constexpr (TC && LRr == 4) {
        stage_tc<B2, SIGN, true, SP, LK>(d, cta, sre, sim, LK, d.tw_off[i],
                                         i == 0 ? GIO : IO_SMEM, i == n - 1 ? GIO : IO_SMEM, nbf,
                                         lbi, lbo);
      } else {
        PAC_FOR_BF_CT(nbf, NT, u) {
          stage_bf<T, B2, (1 << LRr), SIGN, true, SP, LK>(
              d, cta, sre, sim, LK, d.tw_off[i], i == 0 ? GIO : IO_SMEM,
              i == n - 1 ? GIO : IO_SMEM, u, lbi, lbo);
        }
      }
    });
  } else if constexpr (MODE == MODE_DIT) {
    static_for<n>([&](auto kk) {
      constexpr int k = kk.value;
      constexpr int i = n - 1 - k;
      constexpr int LK = RS::logK(LOGL, i);
      constexpr int LRr = RS::v[i];
      constexpr int nbf = 1 << (LOGW + LOGL - LRr);
      if constexpr (k > 0) PAC_SYNC();
      if constexpr (TC && LRr == 4) {
        stage_tc<B2, SIGN, false, SP, LK>(d, cta, sre, sim, LK, d.tw_off[i],
                                          k == 0 ? GIO : IO_SMEM, k == n - 1 ? GIO : IO_SMEM, nbf,
                                          lbi, lbo);
      } else {
        PAC_FOR_BF_CT(nbf, NT, u) {
          stage_bf<T, B2, (1 << LRr), SIGN, false, SP, LK>(
              d, cta, sre, sim, LK, d.tw_off[i], k == 0 ? GIO : IO_SMEM,
              k == n - 1 ? GIO : IO_SMEM, u, lbi, lbo);
        }
      }
    });
  } else {
    static_for<n - 1>([&](auto ii) {
      constexpr int i = ii.value;
      constexpr int LK = RS::logK(LOGL, i);
      constexpr int LRr = RS::v[i];
      constexpr int nbf = 1 << (LOGW + LOGL - LRr);
      if constexpr (i > 0) PAC_SYNC();
      if constexpr (TC && LRr == 4) {
        stage_tc<B2, -1, true, SP, LK>(d, cta, sre, sim, LK, d.tw_off[i], i == 0 ? GIO : IO_SMEM,
                                       IO_SMEM, nbf, lbi, lbo);
      } else {
        PAC_FOR_BF_CT(nbf, NT, u) {
          stage_bf<T, B2, (1 << LRr), -1, true, SP, LK>(
              d, cta, sre, sim, LK, d.tw_off[i], i == 0 ? GIO : IO_SMEM, IO_SMEM, u, lbi, lbo);
        }
      }
    });
    {
      constexpr int LRr = RS::v[n - 1];
      constexpr int nbf = 1 << (LOGW + LOGL - LRr);
      constexpr int io = n == 1 ? GIO : IO_SMEM;
      if constexpr (n > 1) PAC_SYNC();
      PAC_FOR_BF_CT(nbf, NT, u) { middle_bf<T, B2, (1 << LRr), SP>(d, sre, sim, io, io, u, lbi); }
    }
    static_for<n - 1>([&](auto kk) {
      constexpr int i = n - 2 - kk.value;
      constexpr int LK = RS::logK(LOGL, i);
      constexpr int LRr = RS::v[i];
      constexpr int nbf = 1 << (LOGW + LOGL - LRr);
      PAC_SYNC();
      if constexpr (TC && LRr == 4) {
        stage_tc<B2, +1, false, SP, LK>(d, cta, sre, sim, LK, d.tw_off[i], IO_SMEM,
                                        i == 0 ? GIO : IO_SMEM, nbf, lbi, lbo);
      } else {
        PAC_FOR_BF_CT(nbf, NT, u) {
          stage_bf<T, B2, (1 << LRr), +1, false, SP, LK>(
              d, cta, sre, sim, LK, d.tw_off[i], IO_SMEM, i == 0 ? GIO : IO_SMEM, u, lbi, lbo);
        }
      }
    });
  }
}

// ---------------------------------------------------------------------------
// Cluster column tiles.  C = 2^LOGC CTAs of a thread-block cluster share one
// tile of W lines of L = 2^LOGL elements: CTA `rank` keeps elements
// [rank * Lc, (rank + 1) * Lc) of every line in its shared memory (Lc = L/C).
// A tile then needs 1/C of the shared memory of a one-CTA tile, and several
// tiles stay resident per SM, so one tile's global loads overlap another's
// arithmetic.  Only the outermost stage (block L, radix R0 >= C) has
// butterflies that span CTAs: in DIF it reads global memory and stores each
// output into the shared memory of the CTA that owns its position
// (distributed shared memory); in DIT it reads the owners' shared memory and
// writes global memory.  Every other stage has blocks of at most
// L / R0 <= Lc elements, which lie inside one CTA.
// ---------------------------------------------------------------------------
template <typename T, int C>
struct ClView {
  T* re[C];  // shared-memory tile bases of the cluster's CTAs (generic addresses)
  T* im[C];
  int rank;  // this CTA's rank in the cluster
};

// One butterfly of a cluster tile.  XSM: the outermost stage, whose shared-
// memory side (DIF store, DIT load) addresses the owner CTA of each element.
template <typename T, int B2, int R, int SIGN, bool DIF, class SP, int LOGK, int LOGC, bool XSM>
PAC_HD void stage_cl(const PassDesc& d, long long cta, T* sre, T* sim,
                     const ClView<T, (1 << LOGC)>& cv, int twoff, int src, int dst, int u,
                     const long long* lbase) {
  constexpr int LR = ilog2(R);
  static_assert(LR % B2 == 0, "radix must be a power of the digit base");
  constexpr int LOGL = SP::kLogL, LOGW = SP::kLogW, PITCH = SP::kPitch;
  constexpr int LOGLC = LOGL - LOGC;
  constexpr int logell = LOGK - LR;
  constexpr int ell = 1 << logell;
  constexpr int LBF = LOGLC - LR;  // butterflies per line and CTA (log)
  static_assert(XSM ? LOGK == LOGL : LOGK <= LOGLC, "only the outermost stage spans CTAs");
  constexpr int OSH = LOGLC - logell;  // XSM: owner of slot s is s >> OSH
  // global-facing stages: consecutive threads take consecutive lines
  // (coalesced rows of W elements); others: consecutive butterflies
  const bool gf = src == IO_GLOBAL || dst == IO_GLOBAL;
  int w, v;
  if (gf) {
    w = u & ((1 << LOGW) - 1);
    v = u >> LOGW;
  } else {
    v = u & ((1 << LBF) - 1);
    w = u >> LBF;
  }
  v += cv.rank << LBF;
  const int blk = v >> logell;
  const int j = v & (ell - 1);
  const int e0 = (blk << LOGK) + j;
  const T* ire = (const T*)d.in_re;
  const T* iim = (const T*)d.in_im;
  Cx<T> x[R];
  static_for<R>([&](auto mm) {
    constexpr int m = mm.value;
    constexpr int slot = DIF ? m : drev_c(m, LR, B2);
    const int e = e0 + ell * slot;
    if (src == IO_GLOBAL) {
      long long gi = lbase[w] + ((long long)e << d.logS);
      x[m] = Cx<T>{ld_g(ire + gi), ld_g(iim + gi)};
    } else if constexpr (XSM) {
      constexpr int o = slot >> OSH;
      const int si = w * PITCH + sidx<T>(((slot & ((1 << OSH) - 1)) << logell) + j);
      x[m] = Cx<T>{cv.re[o][si], cv.im[o][si]};
    } else {
      const int si = w * PITCH + sidx<T>(e & ((1 << LOGLC) - 1));
      x[m] = Cx<T>{sre[si], sim[si]};
    }
  });
  bf_math<T, B2, R, SIGN, DIF, SP>(d, cta, x, w, e0, j, logell, twoff);
  T* ore = (T*)d.out_re;
  T* oim = (T*)d.out_im;
  static_for<R>([&](auto pp) {
    constexpr int p = pp.value;
    constexpr int slot = DIF ? drev_c(brev_c(p, LR), LR, B2) : brev_c(p, LR);
    const int e = e0 + ell * slot;
    Cx<T> val = x[p];
    if (dst == IO_GLOBAL) {
      if (d.use_scale) {
        val.re *= T(d.scale);
        val.im *= T(d.scale);
      }
      long long gi = lbase[w] + ((long long)e << d.logS);
      ore[gi] = val.re;
      oim[gi] = val.im;
    } else if constexpr (XSM) {
      constexpr int o = slot >> OSH;
      const int si = w * PITCH + sidx<T>(((slot & ((1 << OSH) - 1)) << logell) + j);
      cv.re[o][si] = val.re;
      cv.im[o][si] = val.im;
    } else {
      const int si = w * PITCH + sidx<T>(e & ((1 << LOGLC) - 1));
      sre[si] = val.re;
      sim[si] = val.im;
    }
  });
}

// Phases of a cluster pass; the caller puts a cluster-wide barrier between
// consecutive phases (and, for DIT, after the last one: the peers read this
// CTA's tile in phase 1).
//   DIF  phase 0: outermost stage, global -> owners' shared memory
//        phase 1: the other stages, local; the last one writes global memory
//   DIT  phase 0: every stage but the outermost, local; the first reads global
//        phase 1: outermost stage, owners' shared memory -> global
template <typename T, int B2, int MODE, int SIGN, class SP, int NT, class RS, int LOGC>
PAC_HD void pass_body_cl(const PassDesc& d, long long cta, T* sre, T* sim,
                         const ClView<T, (1 << LOGC)>& cv, const long long* lb, int phase) {
  constexpr int LOGL = SP::kLogL;
  constexpr int LOGW = SP::kLogW;
  constexpr int LOGLC = LOGL - LOGC;
  constexpr int n = RS::n;
  static_assert(MODE == MODE_DIF || MODE == MODE_DIT, "cluster passes are DIF or DIT");
  static_assert(n >= 2 && RS::v[0] >= LOGC, "the outermost stage must span the cluster");
  if constexpr (MODE == MODE_DIF) {
    if (phase == 0) {
      constexpr int LRr = RS::v[0];
      constexpr int nbf = 1 << (LOGW + LOGLC - LRr);
      PAC_FOR_BF_CT(nbf, NT, u) {
        stage_cl<T, B2, (1 << LRr), SIGN, true, SP, LOGL, LOGC, true>(
            d, cta, sre, sim, cv, d.tw_off[0], IO_GLOBAL, IO_SMEM, u, lb);
      }
    } else {
      static_for<n - 1>([&](auto ii) {
        constexpr int i = ii.value + 1;
        constexpr int LK = RS::logK(LOGL, i);
        constexpr int LRr = RS::v[i];
        constexpr int nbf = 1 << (LOGW + LOGLC - LRr);
        if constexpr (i > 1) PAC_SYNC();
        PAC_FOR_BF_CT(nbf, NT, u) {
          stage_cl<T, B2, (1 << LRr), SIGN, true, SP, LK, LOGC, false>(
              d, cta, sre, sim, cv, d.tw_off[i], IO_SMEM, i == n - 1 ? IO_GLOBAL : IO_SMEM, u,
              lb);
        }
      });
    }
  } else {
    if (phase == 0) {
      static_for<n - 1>([&](auto kk) {
        constexpr int k = kk.value;
        constexpr int i = n - 1 - k;
        constexpr int LK = RS::logK(LOGL, i);
        constexpr int LRr = RS::v[i];
        constexpr int nbf = 1 << (LOGW + LOGLC - LRr);
        if constexpr (k > 0) PAC_SYNC();
        PAC_FOR_BF_CT(nbf, NT, u) {
          stage_cl<T, B2, (1 << LRr), SIGN, false, SP, LK, LOGC, false>(
              d, cta, sre, sim, cv, d.tw_off[i], k == 0 ? IO_GLOBAL : IO_SMEM, IO_SMEM, u, lb);
        }
      });
    } else {
      constexpr int LRr = RS::v[0];
      constexpr int nbf = 1 << (LOGW + LOGLC - LRr);
      PAC_FOR_BF_CT(nbf, NT, u) {
        stage_cl<T, B2, (1 << LRr), SIGN, false, SP, LOGL, LOGC, true>(
            d, cta, sre, sim, cv, d.tw_off[0], IO_SMEM, IO_GLOBAL, u, lb);
      }
    }
  }
}

// Radix schedule of one factor of length 2^lg, digit base 2^b2: the fewest
// stages of at most 4 bits (radix 16), bits spread evenly, larger stages
// first; every stage a multiple of b2 bits.
PAC_HDC int sched_n(int lg, int b2) {
  if (b2 == 3) return lg / 3;
  int digits = lg / b2, per = 4 / b2;  // digits per stage at most
  return (digits + per - 1) / per;
}
PAC_HDC int sched_v(int lg, int b2, int i) {
  if (b2 == 3) return 3;
  int n = sched_n(lg, b2);
  int digits = lg / b2;
  int base = digits / n, extra = digits % n;
  return (base + (i < extra ? 1 : 0)) * b2;
}

// The same rule with stages of at most RC bits (RC = 3: radix 8, fewer
// registers per butterfly); RC >= 4 is sched_n / sched_v.
PAC_HDC int sched_n_cap(int lg, int b2, int rc) {
  if (b2 == 3 || rc >= 4) return sched_n(lg, b2);
  const int per = rc / b2 > 0 ? rc / b2 : 1;  // digits per stage at most
  return (lg / b2 + per - 1) / per;
}
PAC_HDC int sched_v_cap(int lg, int b2, int rc, int i) {
  if (b2 == 3 || rc >= 4) return sched_v(lg, b2, i);
  const int n = sched_n_cap(lg, b2, rc), digits = lg / b2;
  return (digits / n + (i < digits % n ? 1 : 0)) * b2;
}
// does pass d run the RC-capped schedule of a 2^logL line?
PAC_HD bool rads_match(const PassDesc& d, int logL, int b2, int rc) {
  if (d.nst != sched_n_cap(logL, b2, rc)) return false;
  for (int i = 0; i < d.nst; ++i)
    if (d.rlog[i] != sched_v_cap(logL, b2, rc, i)) return false;
  return true;
}

template <int LG, int B2, int RC, class IS>
struct RadsImpl;
template <int LG, int B2, int RC, int... I>
struct RadsImpl<LG, B2, RC, std::integer_sequence<int, I...>> {
  using type = Rads<sched_v_cap(LG, B2, RC, I)...>;
};
template <int LG, int B2, int RC>
using RadsCap =
    typename RadsImpl<LG, B2, RC, std::make_integer_sequence<int, sched_n_cap(LG, B2, RC)>>::type;
template <int LG, int B2>
using RadsFor = RadsCap<LG, B2, 4>;

// shared-memory line pitch: one pad element every 16 (FP64) / 32 (FP32)
// (FP32 8-line column tiles: sidx_col32), then skewed so that the W lines
// of a column tile start in different banks
PAC_HDC int pitch_for(int bytes, int logL, int W, int cols = 0, int tc = 0) {
  const int L = 1 << logL;
  const int SH = bytes == 8 ? 4 : 5, NB = bytes == 8 ? 16 : 32;
  if (tc && cols && W > 1) {
    // tensor-core column tiles: one pad per 32 and an odd pitch, so that the
    // 8 lines x 4 slots of a tile load or store fall on distinct banks
    const int p = L + (L >> SH);
    return p + ((1 - p % NB) % NB + NB) % NB;
  }
  if (!tc && row_pad16(bytes, cols, logL, W)) return L + (L >> 4);
  if (!tc && row_swz128(bytes, cols, logL, W)) return L + (L >> 5) + 4;
  int pitch = !tc && col_pad32(bytes, cols, W) ? L + (L >> 3) + 8 * (L >> 7) : L + (L >> SH);
  if (W > 1) {
    int want = (NB / (W < NB ? W : NB)) % NB;
    pitch += ((want - pitch % NB) % NB + NB) % NB;
  }
  return pitch;
}

// ---------------------------------------------------------------------------
// Pipelined column passes.  One CTA per SM walks over the column tiles
// (W columns x L rows) of a launch; the tile lives in registers, TPT
// elements per thread.  A tensor copy (TMA) brings the next tile into a
// dense shared buffer while the current one runs its stages, so the SM keeps
// HBM reads in flight while it computes -- a one-CTA-per-SM pass that loads
// through the LSU path alternates between loading and computing instead, and
// loads in flight are bounded by the L1 left beside a large shared tile.
// The stages exchange data through one padded shared array, real parts
// first and then imaginary parts, which needs half the shared memory of a
// complex tile.  Global stores go out from registers in the last stage.
//
// The members below are per-thread steps between two CTA barriers; the
// device kernel runs them with __syncthreads() in between, the host replay
// runs each step for every thread in turn.  "Step" s is the s-th stage in
// the order of execution (DIF: stage s, DIT: stage NS-1-s).
// ---------------------------------------------------------------------------
template <typename T, int B2, int MODE, int SIGN, int LOGL, int LOGW, int NT>
struct ColPipe {
  static constexpr int L = 1 << LOGL;
  static constexpr int W = 1 << LOGW;
  static constexpr int TPT = (W << LOGL) / NT;  // tile elements per thread
  static constexpr int PITCH = pitch_for((int)sizeof(T), LOGL, W);
  static constexpr int BOXR = L < 256 ? L : 256;  // rows of one tensor-copy box
  using SP = Shape<LOGL, LOGW, PITCH, 1>;
  using RS = RadsFor<LOGL, B2>;
  static constexpr int NS = RS::n;
  static constexpr bool DIF = MODE == MODE_DIF;
  static_assert(MODE == MODE_DIF || MODE == MODE_DIT, "column passes are DIF or DIT");
  static_assert(TPT * NT == (W << LOGL), "the tile must split evenly over the threads");
  static_assert(NS >= 2 && L % BOXR == 0, "at least two stages");

  static PAC_HDC int stage_at(int s) { return DIF ? s : NS - 1 - s; }
  // threads take consecutive lines first (rows of W elements) in the stage
  // that stores to global memory and in the DIF stage that reads the dense
  // tensor-copy tile; the exchange-only stages take consecutive butterflies
  static PAC_HDC bool wfast(int I) { return DIF ? (I == 0 || I == NS - 1) : I == 0; }

  // line w and element e of register K of thread t in stage I, as the
  // stage's input (IN) or output
  template <int I, bool IN, int K>
  static PAC_HD void where(int t, int& w, int& e) {
    constexpr int LR = RS::v[I], R = 1 << LR;
    constexpr int LK = RS::logK(LOGL, I), logell = LK - LR;
    constexpr int LBF = LOGL - LR;
    constexpr int b = K >> LR, r = K & (R - 1);
    constexpr int slot = IN ? (DIF ? r : drev_c(r, LR, B2))
                            : (DIF ? drev_c(brev_c(r, LR), LR, B2) : brev_c(r, LR));
    const int u = t + b * NT;
    int v;
    if constexpr (wfast(I)) {
      w = u & (W - 1);
      v = u >> LOGW;
    } else {
      v = u & ((1 << LBF) - 1);
      w = u >> LBF;
    }
    const int blk = v >> logell, j = v & ((1 << logell) - 1);
    e = (blk << LK) + j + (slot << logell);
  }
  // positions after step S; S = -1 is the copy order of a DIT tile
  // (register K of thread t holds element t + K*NT of the dense tile)
  template <int S, int K>
  static PAC_HD void after(int t, int& w, int& e) {
    if constexpr (S < 0) {
      const int q = t + K * NT;
      w = q & (W - 1);
      e = q >> LOGW;
    } else {
      where<stage_at(S), false, K>(t, w, e);
    }
  }

  // registers from the dense tile A ([e][w], rows of W elements): DIF in
  // stage 0's input order, DIT in copy order.  A warp reads whole rows.
  static PAC_HD void load_tile(int t, const T* Are, const T* Aim, Cx<T> (&x)[TPT]) {
    static_for<TPT>([&](auto kk) {
      constexpr int K = kk.value;
      int w, e;
      if constexpr (DIF) where<0, true, K>(t, w, e);
      else after<-1, K>(t, w, e);
      x[K] = Cx<T>{Are[e * W + w], Aim[e * W + w]};
    });
  }

  // the butterflies of step S on the registers
  template <int S>
  static PAC_HD void compute(const PassDesc& d, long long tile, int t, Cx<T> (&x)[TPT]) {
    constexpr int I = stage_at(S);
    constexpr int LR = RS::v[I], R = 1 << LR;
    constexpr int LK = RS::logK(LOGL, I), logell = LK - LR;
    constexpr int LBF = LOGL - LR;
    static_for<TPT / R>([&](auto bb) {
      constexpr int b = bb.value;
      const int u = t + b * NT;
      int w, v;
      if constexpr (wfast(I)) {
        w = u & (W - 1);
        v = u >> LOGW;
      } else {
        v = u & ((1 << LBF) - 1);
        w = u >> LBF;
      }
      const int blk = v >> logell, j = v & ((1 << logell) - 1);
      Cx<T> y[R];
      static_for<R>([&](auto rr) { y[rr.value] = x[b * R + rr.value]; });
      bf_math<T, B2, R, SIGN, DIF, SP>(d, tile, y, w, (blk << LK) + j, j, logell, d.tw_off[I]);
      static_for<R>([&](auto rr) { x[b * R + rr.value] = y[rr.value]; });
    });
  }

  // exchange halves: write component C (0 re, 1 im) at the positions after
  // step S, read it at the input positions of step S + 1
  template <int S, int C>
  static PAC_HD void xw(int t, T* X, const Cx<T> (&x)[TPT]) {
    static_for<TPT>([&](auto kk) {
      constexpr int K = kk.value;
      int w, e;
      after<S, K>(t, w, e);
      if constexpr (C == 0) X[w * PITCH + sidx<T>(e)] = x[K].re;
      else X[w * PITCH + sidx<T>(e)] = x[K].im;
    });
  }
  template <int S, int C>
  static PAC_HD void xr(int t, const T* X, Cx<T> (&x)[TPT]) {
    static_for<TPT>([&](auto kk) {
      constexpr int K = kk.value;
      int w, e;
      where<stage_at(S + 1), true, K>(t, w, e);
      if constexpr (C == 0) x[K].re = X[w * PITCH + sidx<T>(e)];
      else x[K].im = X[w * PITCH + sidx<T>(e)];
    });
  }

  // the last step's outputs to global memory (lb: line bases of the tile)
  static PAC_HD void store(const PassDesc& d, int t, const long long* lb, const Cx<T> (&x)[TPT]) {
    T* ore = (T*)d.out_re;
    T* oim = (T*)d.out_im;
    static_for<TPT>([&](auto kk) {
      constexpr int K = kk.value;
      int w, e;
      after<NS - 1, K>(t, w, e);
      Cx<T> v = x[K];
      if (d.use_scale) {
        v.re *= T(d.scale);
        v.im *= T(d.scale);
      }
      const long long gi = lb[w] + ((long long)e << d.logS);
      ore[gi] = v.re;
      oim[gi] = v.im;
    });
  }
};

}  // namespace pac
