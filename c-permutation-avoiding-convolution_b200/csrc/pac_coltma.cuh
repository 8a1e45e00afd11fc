// pac_coltma.cuh -- column passes staged through shared memory by tensor
// copies (TMA), in and out.
//
// A column pass transforms W adjacent columns of L rows (a "tile"); every
// row of the tile is a W-element piece of a global row (32 bytes for FP64
// W = 4 and FP32 W = 8).  Read through the load/store units, each such piece
// costs an L1 wavefront and a cache-line slot for the whole time it is in
// flight, which limits the bytes in flight per SM while a 128 KB tile fills
// shared memory.  Here one elected thread moves the whole tile between global
// and shared memory with tensor copies instead, and the threads only ever
// touch shared memory:
//
//   tensor load -> stage 0 -> stage 1 -> ... -> stage n-1 -> tensor store
//
// Every stage reads its butterflies' elements from shared memory into
// registers, computes them (bf_math: twiddles and the in-register DFT of the
// stage engine) and writes them back.  Three layouts of the tile keep all
// these accesses free of bank conflicts (a group of 128 bytes of a warp's
// access -- 16 lanes in FP64, 32 in FP32 -- takes 2^SB = 128 / (W * bytes)
// different rows, which must fall on different banks):
//   dense       (e, w) -> e*W + w: what a tensor copy of the rows writes;
//               conflict-free for every stage whose butterflies are strided
//               (the lanes of a bank group take consecutive j = low bits of e)
//   transposed  (e, w) -> m*(L/R)*W + blk*W + w with e = blk*R + m, R the
//               innermost radix: a tensor copy through a 4D view of the rows
//               (blk, m) writes this; conflict-free for the innermost stage,
//               whose butterflies are R consecutive rows (the lanes of a
//               bank group take consecutive blk)
//   swizzled    (e, w) -> (e ^ ((e >> VIN) & (2^SB - 1)))*W + w: conflict-free
//               for every stage; the working layout between the first and the
//               last stage.
// DIF passes load dense and store transposed, DIT passes load transposed and
// store dense (their first stage is the innermost one).  A stage that reads
// one layout and writes another waits at a CTA barrier between its reads and
// its writes; every other stage writes exactly the slots it read.
//
// A pipelined variant (pac_coltma_pipe_kernel) keeps the tile in registers
// while it computes: the tensor load of the CTA's next tile lands in the
// tile buffer meanwhile, the stages exchange through a buffer of one
// component (real parts, then imaginary parts, in the swizzled layout), and
// each component of the result goes out by a tensor store from that buffer.
//
// The step functions below are per-thread work between two CTA barriers;
// the sm_100a kernel (pac_coltma_kernel, pac_cuda.cu) runs them with
// __syncthreads() between, the host replay (pac_emu.cpp) for every thread in
// turn, with the tensor copies replaced by plain copies through the same
// layout maps.
#pragma once

namespace pac {

enum { LAY_DENSE = 0, LAY_TRANS = 1, LAY_SWZ = 2 };

template <typename T, int B2, int MODE, int SIGN, int LOGL, int LOGW, int NT, int TC = 0>
struct ColTma {
  using RS = RadsFor<LOGL, B2>;
  static constexpr int L = 1 << LOGL;
  static constexpr int W = 1 << LOGW;
  static constexpr int NS = RS::n;
  static constexpr int TILE = W << LOGL;   // elements of one component
  static constexpr int TPT = TILE / NT;    // elements per thread
  static constexpr int VIN = RS::v[NS - 1];  // innermost stage radix (log)
  static constexpr int RIN = 1 << VIN;
  static constexpr int SB = ilog2(128 / (W * (int)sizeof(T)));  // rows per bank group (log)
  static constexpr bool DIF = MODE == MODE_DIF;
  // tensor-copy boxes: dense rows in boxes of BOXR rows; the transposed
  // view in boxes of BOXB blocks x RIN rows
  static constexpr int BOXR = L < 256 ? L : 256;
  static constexpr int NBLK = L >> VIN;
  static constexpr int BOXB = NBLK < 256 ? NBLK : 256;
  using SP = Shape<LOGL, LOGW, 0, 1>;
  static_assert(MODE == MODE_DIF || MODE == MODE_DIT, "column passes are DIF or DIT");
  static_assert(NS >= 2, "at least two stages (one-stage passes need no shared memory)");
  static_assert(TPT * NT == TILE && TPT % 16 == 0, "whole butterflies per thread");
  static_assert(VIN >= SB && VIN + SB <= LOGL, "the swizzle bits lie above the innermost stage");
  static_assert(W * (int)sizeof(T) >= 16, "tensor-copy rows of at least 16 bytes");

  // the stage run in step S
  static PAC_HDC int stage_at(int s) { return DIF ? s : NS - 1 - s; }
  static PAC_HDC int lay_in(int s) { return s > 0 ? LAY_SWZ : (DIF ? LAY_DENSE : LAY_TRANS); }
  static PAC_HDC int lay_out(int s) {
    return s < NS - 1 ? LAY_SWZ : (DIF ? LAY_TRANS : LAY_DENSE);
  }
  // a step whose reads and writes use different layouts waits between them
  static PAC_HDC bool split_step(int s) { return lay_in(s) != lay_out(s); }

  template <int LAY>
  static PAC_HD int pos(int e, int w) {
    if constexpr (LAY == LAY_DENSE) {
      return (e << LOGW) + w;
    } else if constexpr (LAY == LAY_TRANS) {
      // box k of BOXB blocks lands as [m][block in box][w]
      const int blk = e >> VIN;
      const int k = blk / BOXB, bl = blk % BOXB;
      return ((((k << VIN) + (e & (RIN - 1))) * BOXB + bl) << LOGW) + w;
    } else {
      return ((e ^ ((e >> VIN) & ((1 << SB) - 1))) << LOGW) + w;
    }
  }

  // butterfly k of thread t in stage I: line w, first element e0, index j
  // in its block.  Consecutive lanes take consecutive lines, then consecutive
  // j (strided stages) or consecutive blocks (the innermost stage).
  template <int I>
  static PAC_HD void coords(int t, int k, int& w, int& e0, int& j) {
    constexpr int LR = RS::v[I];
    constexpr int LK = RS::logK(LOGL, I), logell = LK - LR;
    const int u = t + k * NT;
    w = u & (W - 1);
    const int v = u >> LOGW;
    const int blk = v >> logell;
    j = v & ((1 << logell) - 1);
    e0 = (blk << LK) + j;
  }

  // element slots of register m (input) / p (output) of a butterfly
  template <int LR, int M>
  static PAC_HDC int in_slot() {
    return DIF ? M : drev_c(M, LR, B2);
  }
  template <int LR, int P>
  static PAC_HDC int out_slot() {
    return DIF ? drev_c(brev_c(P, LR), LR, B2) : brev_c(P, LR);
  }

  // step S, part 1: read every butterfly of this thread into x
  template <int S>
  static PAC_HD void read(int t, const T* Bre, const T* Bim, Cx<T> (&x)[TPT]) {
    constexpr int I = stage_at(S);
    constexpr int LR = RS::v[I], R = 1 << LR;
    constexpr int logell = RS::logK(LOGL, I) - LR;
    constexpr int LAY = lay_in(S);
    static_for<TPT / R>([&](auto kk) {
      int w, e0, j;
      coords<I>(t, kk.value, w, e0, j);
      static_for<R>([&](auto mm) {
        constexpr int m = mm.value;
        const int q = pos<LAY>(e0 + (in_slot<LR, m>() << logell), w);
        x[kk.value * R + m] = Cx<T>{Bre[q], Bim[q]};
      });
    });
  }

  // ---- stage twiddles in shared memory (the pipelined variant) ----------
  // Every tile of a pass reads the same stage-table entries, so a persistent
  // CTA copies the rows that the butterflies read once, at its start, and
  // the stages read them from shared memory: for stage I with ell > 1, rows
  // r < tw_rows(I) of ell entries, row r = table row tw_s(I, r) - 1
  // (stage_twiddles_c's layout).  2048-point FP64: 544 entries (8.5 KB).
  static PAC_HDC int tw_ell(int I) { return 1 << (RS::logK(LOGL, I) - RS::v[I]); }
  static PAC_HDC int tw_rows(int I) {
    return (sizeof(T) == 8 && RS::v[I] >= 2) ? RS::v[I] : (1 << RS::v[I]) - 1;
  }
  static PAC_HDC int tw_s(int I, int r) {
    return (sizeof(T) == 8 && RS::v[I] >= 2) ? 1 << r : r + 1;
  }
  static PAC_HDC int tw_base(int I) {
    int o = 0;
    for (int i = 0; i < I; ++i)
      if (tw_ell(i) > 1) o += tw_rows(i) * tw_ell(i);
    return o;
  }
  static constexpr int TWSM = tw_base(NS);  // entries
  // thread t's share of the copy
  static PAC_HD void tw_fill(const PassDesc& d, int t, Cx<T>* tws) {
    static_for<NS>([&](auto ii) {
      constexpr int I = ii.value;
      constexpr int ell = tw_ell(I), n = tw_rows(I) * ell;
      if constexpr (ell > 1) {
        constexpr int base = tw_base(I);
        const Cx<T>* src = (const Cx<T>*)d.tw + d.tw_off[I];
        for (int q = t; q < n; q += NT) {
          const int r = q / ell, j = q - r * ell;
          constexpr bool pow2 = tw_s(I, 2) == 4;  // rows of s = 2^r
          tws[base + q] = src[((pow2 ? 1 << r : r + 1) - 1) * ell + j];
        }
      }
    });
  }

  // step S, part 2: the butterflies' arithmetic on the registers (stage
  // twiddles from tws, the shared-memory copy, when given)
  template <int S>
  static PAC_HD void compute(const PassDesc& d, long long tile, int t, Cx<T> (&x)[TPT],
                             const Cx<T>* tws = nullptr) {
    constexpr int I = stage_at(S);
    constexpr int LR = RS::v[I], R = 1 << LR;
    constexpr int logell = RS::logK(LOGL, I) - LR;
    constexpr int tb = tw_base(I);
    const Cx<T>* twi = tws ? tws + tb : nullptr;
    static_for<TPT / R>([&](auto kk) {
      int w, e0, j;
      coords<I>(t, kk.value, w, e0, j);
      Cx<T> y[R];
      static_for<R>([&](auto mm) { y[mm.value] = x[kk.value * R + mm.value]; });
      bf_math<T, B2, R, SIGN, DIF, SP>(d, tile, y, w, e0, j, logell, d.tw_off[I], twi);
      static_for<R>([&](auto mm) { x[kk.value * R + mm.value] = y[mm.value]; });
    });
  }

  // step S, part 3: write the outputs back (the last step applies the
  // pass's store scale)
  template <int S>
  static PAC_HD void write(const PassDesc& d, int t, T* Bre, T* Bim, const Cx<T> (&x)[TPT]) {
    constexpr int I = stage_at(S);
    constexpr int LR = RS::v[I], R = 1 << LR;
    constexpr int logell = RS::logK(LOGL, I) - LR;
    constexpr int LAY = lay_out(S);
    const bool scale = S == NS - 1 && d.use_scale;
    const T sc = T(d.scale);
    static_for<TPT / R>([&](auto kk) {
      int w, e0, j;
      coords<I>(t, kk.value, w, e0, j);
      static_for<R>([&](auto pp) {
        constexpr int p = pp.value;
        const int q = pos<LAY>(e0 + (out_slot<LR, p>() << logell), w);
        Cx<T> v = x[kk.value * R + p];
        if (scale) {
          v.re *= sc;
          v.im *= sc;
        }
        Bre[q] = v.re;
        Bim[q] = v.im;
      });
    });
  }

  // ---- one component at a time (the pipelined variant, whose exchange
  // buffer holds one component of the tile) --------------------------------
  // step S's inputs of component C (0 re, 1 im) from buffer B in layout LAY
  template <int S, int C, int LAY>
  static PAC_HD void read_c(int t, const T* B, Cx<T> (&x)[TPT]) {
    constexpr int I = stage_at(S);
    constexpr int LR = RS::v[I], R = 1 << LR;
    constexpr int logell = RS::logK(LOGL, I) - LR;
    static_for<TPT / R>([&](auto kk) {
      int w, e0, j;
      coords<I>(t, kk.value, w, e0, j);
      static_for<R>([&](auto mm) {
        constexpr int m = mm.value;
        const T v = B[pos<LAY>(e0 + (in_slot<LR, m>() << logell), w)];
        if constexpr (C == 0) x[kk.value * R + m].re = v;
        else x[kk.value * R + m].im = v;
      });
    });
  }
  // step S's outputs of component C into buffer B in layout LAY (the last
  // step applies the pass's store scale)
  template <int S, int C, int LAY>
  static PAC_HD void write_c(const PassDesc& d, int t, T* B, const Cx<T> (&x)[TPT]) {
    constexpr int I = stage_at(S);
    constexpr int LR = RS::v[I], R = 1 << LR;
    constexpr int logell = RS::logK(LOGL, I) - LR;
    const bool scale = S == NS - 1 && d.use_scale;
    const T sc = T(d.scale);
    static_for<TPT / R>([&](auto kk) {
      int w, e0, j;
      coords<I>(t, kk.value, w, e0, j);
      static_for<R>([&](auto pp) {
        constexpr int p = pp.value;
        T v = C == 0 ? x[kk.value * R + p].re : x[kk.value * R + p].im;
        if (scale) v *= sc;
        B[pos<LAY>(e0 + (out_slot<LR, p>() << logell), w)] = v;
      });
    });
  }

  // the last step's outputs straight from the registers to the pass's output
  // rows (the pipelined variant's direct-store form): four (FP64) or eight
  // (FP32) consecutive lanes hold the W columns of one row, so every warp
  // store fills eight whole 32-byte sectors and the tensor-copy unit only
  // carries the loads
  template <int S>
  static PAC_HD void store_g(const PassDesc& d, long long tile, int t, const Cx<T> (&x)[TPT]) {
    constexpr int I = stage_at(S);
    constexpr int LR = RS::v[I], R = 1 << LR;
    constexpr int logell = RS::logK(LOGL, I) - LR;
    const bool scale = d.use_scale;
    const T sc = T(d.scale);
    int i0, o;
    tile_coords(d, tile, i0, o);
    const long long base = ((long long)o << (LOGL + d.logS)) + i0;
    T* ore = (T*)d.out_re;
    T* oim = (T*)d.out_im;
    static_for<TPT / R>([&](auto kk) {
      int w, e0, j;
      coords<I>(t, kk.value, w, e0, j);
      static_for<R>([&](auto pp) {
        constexpr int p = pp.value;
        const long long gi = base + ((long long)(e0 + (out_slot<LR, p>() << logell)) << d.logS) + w;
        Cx<T> v = x[kk.value * R + p];
        if (scale) {
          v.re *= sc;
          v.im *= sc;
        }
        ore[gi] = v.re;
        oim[gi] = v.im;
      });
    });
  }

  // ---- tensor-core radix-16 steps (TC = 1, the FP32 tensor-core form) ----
  // Every radix-16 butterfly is one row of a real MMA on the 5th-generation
  // tensor cores (tcgen05.mma kind::f16, FP32 accumulation in tensor
  // memory): the 128 threads of a warpgroup put their butterflies' inputs
  // into rows 0..127 of A (M = 128, K = 32: the 16 real parts, then the 16
  // imaginary parts), B holds the real 32 x 32 form of the 16-point DFT
  // (N = 32 outputs: 16 real parts, then 16 imaginary parts), and row r of
  // D -- read back by the thread that wrote row r (tcgen05.ld 32x32b: warp
  // w of the warpgroup reads lanes 32w..32w+31) -- holds its butterfly's
  // outputs in the register order dft_reg leaves (register p = frequency
  // brev(p)).  Each product is compensated as in the warp-MMA form: inputs
  // scaled by a power of two into [2^14, 2^15), split into FP16 hi and lo
  // parts, Y = Xlo.Vhi + Xhi.Vlo + Xhi.Vhi (small products first).  Operand
  // tiles sit in shared memory K-major without swizzle: core matrices of 8
  // rows x 8 halves (16 bytes a row, 128 bytes each), core matrix
  // (row/8, k/8) at ((row/8) * 4 + k/8) * 128 bytes.
  static constexpr int UM = 128, UK = 32, UN = 32;
  static constexpr int NWG = NT / 128;   // warpgroups
  static constexpr int TPW = TPT / 16;   // radix-16 butterflies of a thread per step
  static constexpr int UTILE = UM * UK;  // halves of one operand tile (8 KB)
  static_assert(!TC || (sizeof(T) == 4 && NT % 128 == 0), "tensor-core steps: FP32, warpgroups");
  static PAC_HDC int umma_off(int row, int k) {
    return ((((row >> 3) << 2) + (k >> 3)) << 6) + ((row & 7) << 3) + (k & 7);
  }
  // the DFT operand (hi and lo halves of Vt[n][k], n-major rows, K
  // contiguous), words of two halves at umma_off(n, k) / 2 for even k
  static PAC_HD void tc_fill_v(int idx, uint32_t* Vh, uint32_t* Vl) {
    const int n = idx >> 4, k = (idx & 15) << 1;  // 32 rows x 16 words
    float v[2];
    for (int e = 0; e < 2; ++e) {
      const int kk = k + e;
      const int c = n & 15, m = kk & 15;
      const int f = brev_c(c, 4);
      float cr, ci;
      tc_cs16((m * f) & 15, cr, ci);
      if (SIGN < 0) ci = -ci;
      // Re y_c = sum xr cr - xi ci ; Im y_c = sum xr ci + xi cr
      v[e] = n < 16 ? (kk < 16 ? cr : -ci) : (kk < 16 ? ci : cr);
    }
    uint32_t hi, lo;
    tc_split2(v[0], v[1], hi, lo);
    Vh[umma_off(n, k) >> 1] = hi;
    Vl[umma_off(n, k) >> 1] = lo;
  }
  // step S, radix-16 butterfly kk of thread t: DIT pre-twiddles, scale, and
  // the hi / lo rows (row t mod 128) of this warpgroup's A tiles
  template <int S>
  static PAC_HD void tc_prep(const PassDesc& d, int t, int kk, const Cx<T> (&x)[TPT], uint32_t* Ah,
                             uint32_t* Al, int& E) {
    constexpr int I = stage_at(S);
    constexpr int logell = RS::logK(LOGL, I) - 4;
    static_assert(RS::v[I] == 4, "radix-16 steps only");
    int w, e0, j;
    coords<I>(t, kk, w, e0, j);
    Cx<T> y[16];
    static_for<16>([&](auto mm) { y[mm.value] = x[kk * 16 + mm.value]; });
    if constexpr (!DIF) {
      if (logell > 0 && j > 0) {
        Cx<T> wv[16];
        stage_twiddles<T, 16>((const Cx<T>*)d.tw + d.tw_off[I] + j, 1 << logell, wv);
        static_for<15>([&](auto ss) { y[ss.value + 1] = ctw(y[ss.value + 1], wv[ss.value + 1], SIGN); });
      }
    }
    float mx = 0.f;
    static_for<16>([&](auto mm) {
      mx = fmaxf(mx, fmaxf(fabsf(y[mm.value].re), fabsf(y[mm.value].im)));
    });
    const int ex = (int)((f32_bits(mx) >> 23) & 0xffu) - 127;  // -127 for 0 / subnormal
    E = 14 - ex;
    E = E < -100 ? -100 : E > 100 ? 100 : E;
    const float sc = tc_pow2(E);
    const int r = t & 127;
    static_for<8>([&](auto pp) {  // words of k = 2p, 2p + 1 (real parts) and 16 + 2p, 17 + 2p
      constexpr int p2 = 2 * pp.value;
      uint32_t hi, lo;
      tc_split2(y[p2].re * sc, y[p2 + 1].re * sc, hi, lo);
      Ah[umma_off(r, p2) >> 1] = hi;
      Al[umma_off(r, p2) >> 1] = lo;
      tc_split2(y[p2].im * sc, y[p2 + 1].im * sc, hi, lo);
      Ah[umma_off(r, 16 + p2) >> 1] = hi;
      Al[umma_off(r, 16 + p2) >> 1] = lo;
    });
  }
  // step S, radix-16 butterfly kk of thread t: D row (32 floats) unscaled,
  // DIF post-twiddles, back into x
  template <int S>
  static PAC_HD void tc_finish(const PassDesc& d, int t, int kk, const float (&D)[32], int E,
                               Cx<T> (&x)[TPT]) {
    constexpr int I = stage_at(S);
    constexpr int logell = RS::logK(LOGL, I) - 4;
    int w, e0, j;
    coords<I>(t, kk, w, e0, j);
    const float us = tc_pow2(-E);
    Cx<T> y[16];
    static_for<16>([&](auto pp) { y[pp.value] = Cx<T>{D[pp.value] * us, D[16 + pp.value] * us}; });
    if constexpr (DIF) {
      if (logell > 0 && j > 0) {
        Cx<T> wv[16];
        stage_twiddles<T, 16>((const Cx<T>*)d.tw + d.tw_off[I] + j, 1 << logell, wv);
        static_for<16>([&](auto pp) {
          constexpr int s = brev_c(pp.value, 4);
          if constexpr (s > 0) y[pp.value] = ctw(y[pp.value], wv[s], SIGN);
        });
      }
    }
    static_for<16>([&](auto pp) { x[kk * 16 + pp.value] = y[pp.value]; });
  }
  // does step S run on the tensor cores?
  static PAC_HDC bool tc_step(int s) { return TC && RS::v[stage_at(s)] == 4; }

  // tile -> tensor coordinates: column i0 of the row array, outer index o
  static PAC_HD void tile_coords(const PassDesc& d, long long tile, int& i0, int& o) {
    const long long g0 = tile << LOGW;
    i0 = (int)(g0 & ((1LL << d.logS) - 1));
    o = (int)(g0 >> d.logS);
  }
};

}  // namespace pac
