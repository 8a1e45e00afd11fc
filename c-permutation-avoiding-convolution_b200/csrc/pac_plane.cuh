// pac_plane.cuh -- the plane pass of a 3D convolution: axes 1 and 2 of every
// plane in one launch.
//
// A 3D convolution over N0 x N1 x N2 runs, with the line schedule, five
// passes over HBM (DIF axis 0, DIF axis 1, fused axis 2, DIT axis 1, DIT
// axis 0).  The plane schedule runs three: DIF axis 0, one plane pass, DIT
// axis 0.  The plane pass transforms each N1 x N2 plane (contiguous in
// memory) forward along axes 1 and 2, multiplies by the filter spectrum and
// transforms back, so the plane makes one HBM read and one HBM write.
//
// A plane is larger than one CTA's shared memory (256 x 256 complex FP32 is
// 512 KB), so a thread-block cluster of C = 2^LOGC CTAs holds it: CTA `rank`
// keeps rows [rank * RC, (rank + 1) * RC) of the plane (RC = N1 / C), row-
// major with padded rows.  Only the outermost axis-1 stage (radix R0 >= C,
// stride N1 / R0 rows) has butterflies whose rows lie in several CTAs; it
// runs between global memory and the owners' shared memory (distributed
// shared memory), every other stage inside one CTA:
//   phase 0  axis-1 stage 0 (DIF): global rows -> owners' shared memory
//   phase 1  axis-1 stages 1.. (DIF), axis-2 stages (DIF), the product with
//            the filter spectrum (fused with the last axis-2 DIF stage and
//            the first axis-2 DIT stage, as in the fused row pass), axis-2
//            DIT stages, axis-1 DIT stages down to 1 -- all local
//   phase 2  axis-1 stage 0 (DIT): owners' shared memory -> global rows
// with a cluster barrier between the phases (and after phase 2, while the
// peers still read this CTA's rows).  The axes commute, so this order gives
// the spectrum positions of the line schedule: the filter spectrum keeps the
// plan order of the fused row pass.
//
// The phase functions run the same code on the device (one butterfly per
// thread, __syncthreads between stages) and in the host replay (every
// butterfly in turn, the cluster's CTAs phase by phase).
#pragma once

namespace pac {

template <typename T, int B2, int LOGN1, int LOGN2, int LOGC, int NT>
struct PlaneGeo {
  static constexpr int kLogN1 = LOGN1, kLogN2 = LOGN2;
  static constexpr int N1 = 1 << LOGN1, N2 = 1 << LOGN2, C = 1 << LOGC;
  static constexpr int LOGRC = LOGN1 - LOGC, RC = 1 << LOGRC;
  // padded rows of N2 elements; the RC rows start in different banks
  static constexpr int P2 = pitch_for((int)sizeof(T), LOGN2, RC);
  using R1 = RadsFor<LOGN1, B2>;
  using R2 = RadsFor<LOGN2, B2>;
  static constexpr int N1S = R1::n, N2S = R2::n;
  // local stages: rows (RC lines of N2) and columns (N2 lines of RC, the
  // transposed view of the same row-major tile)
  using SPR = Shape<LOGN2, LOGRC, P2, 0>;
  using SPC = Shape<LOGRC, LOGN2, P2, 1, 0, 1>;
  static constexpr int R0L = R1::v[0];                 // outermost axis-1 stage (log radix)
  static constexpr int NBX = (N1 >> R0L) * N2 / C;     // its butterflies per CTA
  static constexpr size_t SMEM = (size_t)2 * RC * P2 * sizeof(T);
  static_assert(R0L >= LOGC, "the outermost axis-1 stage must span the cluster");
  static_assert(N1S >= 2 && N2S >= 2, "two stages per axis at least");
  static_assert(N1S + N2S <= PAC_MAX_STAGES, "stage count");
  static_assert(NBX % NT == 0 || NT % NBX == 0, "cross-CTA butterflies per thread");
};

// One butterfly of the outermost axis-1 stage.  Butterfly b of the cluster
// (b = rank * NBX + u) is column col = b mod N2, index j = b / N2 in the
// stage's block (the stage has one block: K = N1, ell = N1 / R0).  DIF: its
// R0 inputs come from global rows j + ell*m and its outputs go to the
// shared memory of the CTAs that own rows j + ell*slot; DIT: the reverse.
template <typename T, int B2, int R, int SIGN, bool DIF, class G>
PAC_HD void plane_xstage(const PassDesc& d, long long plane, const ClView<T, G::C>& cv, int u,
                         int twoff) {
  constexpr int LR = ilog2(R);
  constexpr int logell = G::kLogN1 - LR;
  const int b = cv.rank * G::NBX + u;
  const int col = b & (G::N2 - 1);
  const int j = b >> G::kLogN2;
  const long long base = plane << (G::kLogN1 + G::kLogN2);
  Cx<T> x[R];
  static_for<R>([&](auto mm) {
    constexpr int m = mm.value;
    constexpr int slot = DIF ? m : drev_c(m, LR, B2);
    if constexpr (DIF) {
      const int row = j + (slot << logell);
      const long long gi = base + ((long long)row << G::kLogN2) + col;
      x[m] = Cx<T>{ld_g((const T*)d.in_re + gi), ld_g((const T*)d.in_im + gi)};
    } else {
      // j < ell <= RC: the owner and the row offset are compile-time
      constexpr int o = (slot << logell) >> G::LOGRC;
      constexpr int roff = (slot << logell) & (G::RC - 1);
      const int si = (j + roff) * G::P2 + sidx<T>(col);
      x[m] = Cx<T>{cv.re[o][si], cv.im[o][si]};
    }
  });
  bf_math<T, B2, R, SIGN, DIF, typename G::SPR>(d, plane, x, col, j, j, logell, twoff);
  static_for<R>([&](auto pp) {
    constexpr int p = pp.value;
    constexpr int slot = DIF ? drev_c(brev_c(p, LR), LR, B2) : brev_c(p, LR);
    if constexpr (DIF) {
      constexpr int o = (slot << logell) >> G::LOGRC;
      constexpr int roff = (slot << logell) & (G::RC - 1);
      const int si = (j + roff) * G::P2 + sidx<T>(col);
      cv.re[o][si] = x[p].re;
      cv.im[o][si] = x[p].im;
    } else {
      const int row = j + (slot << logell);
      const long long gi = base + ((long long)row << G::kLogN2) + col;
      ((T*)d.out_re)[gi] = x[p].re;
      ((T*)d.out_im)[gi] = x[p].im;
    }
  });
}

// Phase `phase` of the plane pass for CTA cv.rank of the cluster that holds
// plane `plane`.  lb[r] is the global element index of the start of local
// row r (the fused product reads the filter spectrum by it).
template <typename T, int B2, int LOGN1, int LOGN2, int LOGC, int NT>
PAC_HD void plane_body(const PassDesc& d, long long plane, T* sre, T* sim,
                       const ClView<T, (1 << LOGC)>& cv, const long long* lb, int phase) {
  using G = PlaneGeo<T, B2, LOGN1, LOGN2, LOGC, NT>;
  using R1 = typename G::R1;
  using R2 = typename G::R2;
  using SPR = typename G::SPR;
  using SPC = typename G::SPC;
  constexpr int N1S = G::N1S, N2S = G::N2S;
  constexpr int LOGRC = G::LOGRC;
  if (phase == 0) {
    PAC_FOR_BF_CT(G::NBX, NT, u) {
      plane_xstage<T, B2, (1 << R1::v[0]), -1, true, G>(d, plane, cv, u, d.tw_off[0]);
    }
    return;
  }
  if (phase == 2) {
    PAC_FOR_BF_CT(G::NBX, NT, u) {
      plane_xstage<T, B2, (1 << R1::v[0]), +1, false, G>(d, plane, cv, u, d.tw_off[0]);
    }
    return;
  }
  // phase 1: everything local.  Axis-1 DIF stages 1 .. N1S-1 (block sizes
  // of the N1-point schedule; blocks lie inside the CTA's RC rows)
  static_for<N1S - 1>([&](auto ii) {
    constexpr int i = ii.value + 1;
    constexpr int LK = R1::logK(LOGN1, i);
    constexpr int LRr = R1::v[i];
    constexpr int nbf = 1 << (LOGN2 + LOGRC - LRr);
    if constexpr (i > 1) PAC_SYNC();
    PAC_FOR_BF_CT(nbf, NT, u) {
      stage_bf<T, B2, (1 << LRr), -1, true, SPC, LK>(d, plane, sre, sim, LK, d.tw_off[i],
                                                     IO_SMEM, IO_SMEM, u, lb, lb);
    }
  });
  // axis-2 DIF stages but the last
  static_for<N2S - 1>([&](auto ii) {
    constexpr int i = ii.value;
    constexpr int LK = R2::logK(LOGN2, i);
    constexpr int LRr = R2::v[i];
    constexpr int nbf = 1 << (LOGRC + LOGN2 - LRr);
    PAC_SYNC();
    PAC_FOR_BF_CT(nbf, NT, u) {
      stage_bf<T, B2, (1 << LRr), -1, true, SPR, LK>(d, plane, sre, sim, LK,
                                                     d.tw_off[N1S + i], IO_SMEM, IO_SMEM, u,
                                                     lb, lb);
    }
  });
  // last axis-2 DIF stage, product with the filter spectrum, first DIT stage
  {
    constexpr int LRr = R2::v[N2S - 1];
    constexpr int nbf = 1 << (LOGRC + LOGN2 - LRr);
    PAC_SYNC();
    PAC_FOR_BF_CT(nbf, NT, u) {
      middle_bf<T, B2, (1 << LRr), SPR>(d, sre, sim, IO_SMEM, IO_SMEM, u, lb);
    }
  }
  // axis-2 DIT stages
  static_for<N2S - 1>([&](auto kk) {
    constexpr int i = N2S - 2 - kk.value;
    constexpr int LK = R2::logK(LOGN2, i);
    constexpr int LRr = R2::v[i];
    constexpr int nbf = 1 << (LOGRC + LOGN2 - LRr);
    PAC_SYNC();
    PAC_FOR_BF_CT(nbf, NT, u) {
      stage_bf<T, B2, (1 << LRr), +1, false, SPR, LK>(d, plane, sre, sim, LK,
                                                      d.tw_off[N1S + i], IO_SMEM, IO_SMEM, u,
                                                      lb, lb);
    }
  });
  // axis-1 DIT stages N1S-1 .. 1
  static_for<N1S - 1>([&](auto kk) {
    constexpr int i = N1S - 1 - kk.value;
    constexpr int LK = R1::logK(LOGN1, i);
    constexpr int LRr = R1::v[i];
    constexpr int nbf = 1 << (LOGN2 + LOGRC - LRr);
    PAC_SYNC();
    PAC_FOR_BF_CT(nbf, NT, u) {
      stage_bf<T, B2, (1 << LRr), +1, false, SPC, LK>(d, plane, sre, sim, LK, d.tw_off[i],
                                                      IO_SMEM, IO_SMEM, u, lb, lb);
    }
  });
}

}  // namespace pac
