// pac_special.h -- the specialised pass kernels and the radix schedules.
//
// A pass whose (element type, digit base, mode, sign, line length, stride
// kind) appears in PAC_SPECIAL_LIST runs a kernel compiled for exactly that
// geometry (pass_body_ct): tile width W = 2^logW, NT threads per CTA and a
// register bound that leaves MINB CTAs per SM.  Every other pass runs the
// generic kernel.  The planner, the CUDA backend and the test-only host
// replay all read this one list, so the replay checks the specialised code.
#pragma once

#include <utility>

#include "pac_engine.cuh"

namespace pac {

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

template <int LG, int B2, class IS>
struct RadsImpl;
template <int LG, int B2, int... I>
struct RadsImpl<LG, B2, std::integer_sequence<int, I...>> {
  using type = Rads<sched_v(LG, B2, I)...>;
};
template <int LG, int B2>
using RadsFor = typename RadsImpl<LG, B2, std::make_integer_sequence<int, sched_n(LG, B2)>>::type;

// shared-memory line pitch: one pad element every 16 (FP64) / 32 (FP32),
// then skewed so that the W lines of a column tile start in different banks
PAC_HDC int pitch_for(int bytes, int logL, int W) {
  const int L = 1 << logL;
  const int SH = bytes == 8 ? 4 : 5, NB = bytes == 8 ? 16 : 32;
  int pitch = L + (L >> SH);
  if (W > 1) {
    int want = (NB / (W < NB ? W : NB)) % NB;
    pitch += ((want - pitch % NB) % NB + NB) % NB;
  }
  return pitch;
}

// fields: element type, bytes, log2 digit base, mode, sign (DIF/DIT), log2 L,
// column tile (element stride > 1), log2 W, threads, min CTAs per SM
#define PAC_SPECIAL_LIST(X)                                \
  X(double, 8, 1, MODE_CONV, 0, 11, 0, 0, 128, 4)          \
  X(double, 8, 1, MODE_DIF, -1, 11, 1, 2, 512, 1)          \
  X(double, 8, 1, MODE_DIT, +1, 11, 1, 2, 512, 1)          \
  X(float, 4, 1, MODE_CONV, 0, 11, 0, 1, 256, 2)           \
  X(float, 4, 1, MODE_DIF, -1, 11, 1, 3, 512, 1)           \
  X(float, 4, 1, MODE_DIT, +1, 11, 1, 3, 512, 1)           \
  X(double, 8, 1, MODE_DIF, -1, 11, 1, 1, 256, 2)          \
  X(double, 8, 1, MODE_DIT, +1, 11, 1, 1, 256, 2)          \
  X(float, 4, 1, MODE_DIF, -1, 11, 1, 2, 512, 1)           \
  X(float, 4, 1, MODE_DIT, +1, 11, 1, 2, 512, 1)
// Measured on C3 (2048^2): FP64 columns W=4 (32-byte rows) 53 us vs W=2
// 68 us; FP32 columns W=8 34 us vs W=4 45 us -- row width, not occupancy,
// bounds these passes.
// (a geometry may have several candidates; the first is the default and
// PAC_SPECIAL_VARIANT=k selects the k-th, for tuning)

// Column passes whose tile is shared by a cluster of 2^logC CTAs
// (PassDesc.logC, pass_body_cl): each CTA holds L / 2^logC rows of the
// W-column tile, so 32- or 64-byte row pieces fit in ~64 KB of shared
// memory per CTA and two tiles stay resident per SM.  Opt-in
// (PAC_CLUSTER_VARIANT=k): on 2048^2 FP64 the 2-CTA tiles (W = 4) ran
// 57 / 59 us per DIF / DIT pass against 54 / 51 us for the one-CTA tiles,
// and the 4-CTA tiles (W = 8) 69 / 78 us -- the two CTAs of an SM start
// together, so they load and compute in step, and the exchange through
// distributed shared memory and the cluster barriers come on top.
// fields: element type, bytes, log2 digit base, mode, sign, log2 L, log2 W,
// log2 cluster size, threads, min CTAs per SM
#define PAC_CLUSTER_LIST(X)                          \
  X(double, 8, 1, MODE_DIF, -1, 11, 2, 1, 256, 2)    \
  X(double, 8, 1, MODE_DIT, +1, 11, 2, 1, 256, 2)    \
  X(float, 4, 1, MODE_DIF, -1, 11, 3, 1, 256, 2)     \
  X(float, 4, 1, MODE_DIT, +1, 11, 3, 1, 256, 2)     \
  X(double, 8, 1, MODE_DIF, -1, 11, 3, 2, 256, 2)    \
  X(double, 8, 1, MODE_DIT, +1, 11, 3, 2, 256, 2)    \
  X(float, 4, 1, MODE_DIF, -1, 11, 4, 2, 256, 2)     \
  X(float, 4, 1, MODE_DIT, +1, 11, 4, 2, 256, 2)

inline bool cluster_geometry(int bytes, int b2, int mode, int sign, int logL, int* logW,
                             int* logC, int* nt, int variant = 0) {
  int seen = 0;
#define PAC_X(T, BY, B2_, MO, SG, LL, LW, LC, NT_, MB)                                    \
  if (bytes == BY && b2 == B2_ && mode == MO && sign == SG && logL == LL &&            \
      seen++ == variant) {                                                             \
    *logW = LW;                                                                        \
    *logC = LC;                                                                        \
    *nt = NT_;                                                                         \
    return true;                                                                       \
  }
  PAC_CLUSTER_LIST(PAC_X)
#undef PAC_X
  return false;
}

inline bool special_geometry(int bytes, int b2, int mode, int sign, int logL, int cols,
                             int* logW, int* nt, int variant = 0) {
  int seen = 0;
#define PAC_X(T, BY, B2_, MO, SG, LL, CO, LW, NT_, MB)                                    \
  if (bytes == BY && b2 == B2_ && mode == MO && (MO == MODE_CONV || sign == SG) &&     \
      logL == LL && cols == CO && seen++ == variant) {                                 \
    *logW = LW;                                                                        \
    *nt = NT_;                                                                         \
    return true;                                                                       \
  }
  PAC_SPECIAL_LIST(PAC_X)
#undef PAC_X
  return false;
}

}  // namespace pac
