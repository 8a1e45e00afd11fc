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

template <typename T, int B2, int MODE, int SIGN, int LOGL, int LOGW, int NT>
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

  // step S, part 2: the butterflies' arithmetic on the registers
  template <int S>
  static PAC_HD void compute(const PassDesc& d, long long tile, int t, Cx<T> (&x)[TPT]) {
    constexpr int I = stage_at(S);
    constexpr int LR = RS::v[I], R = 1 << LR;
    constexpr int logell = RS::logK(LOGL, I) - LR;
    static_for<TPT / R>([&](auto kk) {
      int w, e0, j;
      coords<I>(t, kk.value, w, e0, j);
      Cx<T> y[R];
      static_for<R>([&](auto mm) { y[mm.value] = x[kk.value * R + mm.value]; });
      bf_math<T, B2, R, SIGN, DIF, SP>(d, tile, y, w, e0, j, logell, d.tw_off[I]);
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

  // tile -> tensor coordinates: column i0 of the row array, outer index o
  static PAC_HD void tile_coords(const PassDesc& d, long long tile, int& i0, int& o) {
    const long long g0 = tile << LOGW;
    i0 = (int)(g0 & ((1LL << d.logS) - 1));
    o = (int)(g0 >> d.logS);
  }
};

}  // namespace pac
