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

// (the radix schedules sched_n / sched_v / RadsFor and the line pitch
// pitch_for are defined with the stage engine, pac_stages.cuh)

// fields: element type, bytes, log2 digit base, mode, sign (DIF/DIT), log2 L,
// column tile (element stride > 1), log2 W, threads, min CTAs per SM,
// tensor-core form (radix-16 stages on the tensor cores, pac_tc.cuh), log2
// of the largest stage radix (4: the default schedule RadsFor; 3: radix 8,
// for plans tuned with max_radix_log = 3, RadsCap)
#define PAC_SPECIAL_LIST(X)                                \
  X(double, 8, 1, MODE_CONV, 0, 11, 0, 0, 128, 4, 0, 4)          \
  X(double, 8, 1, MODE_DIF, -1, 11, 1, 2, 512, 1, 0, 4)          \
  X(double, 8, 1, MODE_DIT, +1, 11, 1, 2, 512, 1, 0, 4)          \
  X(float, 4, 1, MODE_CONV, 0, 11, 0, 0, 128, 7, 0, 4)           \
  X(float, 4, 1, MODE_DIF, -1, 11, 1, 3, 512, 1, 0, 4)           \
  X(float, 4, 1, MODE_DIT, +1, 11, 1, 3, 512, 1, 0, 4)           \
  /* 3D FP32: 256-point rows and columns (256^3, and the middle axis of */ \
  /* 512 x 256 x 128), 512-point columns and 128-point rows */           \
  X(float, 4, 1, MODE_CONV, 0, 8, 0, 3, 128, 6, 0, 4)            \
  X(float, 4, 1, MODE_DIF, -1, 8, 1, 4, 256, 2, 0, 4)            \
  X(float, 4, 1, MODE_DIT, +1, 8, 1, 4, 256, 2, 0, 4)            \
  X(float, 4, 1, MODE_DIF, -1, 9, 1, 4, 512, 2, 0, 4)            \
  X(float, 4, 1, MODE_DIT, +1, 9, 1, 4, 512, 2, 0, 4)            \
  X(float, 4, 1, MODE_CONV, 0, 7, 0, 4, 128, 8, 0, 4)            \
  /* 3D FP64: fused 256- and 128-point rows */                          \
  X(double, 8, 1, MODE_CONV, 0, 8, 0, 3, 128, 4, 0, 4)           \
  X(double, 8, 1, MODE_CONV, 0, 7, 0, 4, 128, 4, 0, 4)           \
  /* 1D batches: 16-point columns (one radix-16 stage, no shared memory) */ \
  X(float, 4, 1, MODE_DIF, -1, 4, 1, 8, 256, 4, 0, 4)            \
  X(float, 4, 1, MODE_DIT, +1, 4, 1, 8, 256, 4, 0, 4)            \
  X(double, 8, 1, MODE_DIF, -1, 4, 1, 8, 256, 2, 0, 4)           \
  X(double, 8, 1, MODE_DIT, +1, 4, 1, 8, 256, 2, 0, 4)           \
  /* 1D batches: fused 4096-point rows (2^16-point lines split 16 x 4096) */ \
  X(float, 4, 1, MODE_CONV, 0, 12, 0, 1, 256, 3, 0, 4)           \
  X(double, 8, 1, MODE_CONV, 0, 12, 0, 0, 256, 2, 0, 4)          \
  /* further candidates (PAC_SPECIAL_VARIANT=k, tuner knob special = k): */ \
  /* the fused 2048-point FP32 pass: one line per 128-thread CTA at */     \
  /* seven CTAs per SM (72 registers) is the default: 2048 lines over */    \
  /* 148 SMs are 13.8 lines per SM, so seven resident lines leave */         \
  /* almost no idle last round where eight (four CTAs of two lines) */      \
  /* leave 14%; on 2048^2 it ran 31.6 us against 34.3 for two lines per */  \
  /* 256-thread CTA at four CTAs per SM (64 registers), eight one-line */    \
  /* CTAs 32.5; two lines at three and two CTAs per SM ran 34.9 and */        \
  /* 37.2.  The FP64 pass at three CTAs per SM ran 49.1 us against 45.9 */  \
  /* at four; at five CTAs per SM it spills 144 bytes and ran */              \
  /* 53.2 us against 47.2 at four, and with two lines per 256-thread CTA */  \
  /* (two CTAs per SM) 51.4 against 46.5 */                                  \
  X(float, 4, 1, MODE_CONV, 0, 11, 0, 1, 256, 4, 0, 4)           \
  X(float, 4, 1, MODE_CONV, 0, 11, 0, 1, 256, 3, 0, 4)           \
  X(float, 4, 1, MODE_CONV, 0, 11, 0, 1, 256, 2, 0, 4)           \
  X(float, 4, 1, MODE_CONV, 0, 11, 0, 0, 128, 8, 0, 4)           \
  /* the 3D passes at the other occupancy: on 512 x 256 x 128 the */     \
  /* 512-point columns at 2 CTAs per SM ran 145 / 135 us against 149 / */ \
  /* 151 at one, the fused 128-point rows at 3 CTAs 155 against 160 us; */ \
  /* 256-point columns at 3 CTAs were 2-7% slower (not kept) */           \
  /* the fused 256-point rows: FP32 eight lines per 128-thread CTA at */  \
  /* six CTAs per SM (the default) ran 89.5 us on 256^3, sixteen lines */    \
  /* per 256-thread CTA at three 97.6, at two 106.5, eight lines at */       \
  /* eight CTAs 96.9; FP64 eight lines per 128-thread CTA at four CTAs */   \
  /* (the default) 134 us, sixteen per 256-thread CTA at two 153 (the */     \
  /* generic kernel took 254) */                                             \
  X(float, 4, 1, MODE_CONV, 0, 8, 0, 4, 256, 3, 0, 4)            \
  X(float, 4, 1, MODE_CONV, 0, 8, 0, 4, 256, 2, 0, 4)            \
  X(float, 4, 1, MODE_CONV, 0, 8, 0, 3, 128, 8, 0, 4)            \
  X(double, 8, 1, MODE_CONV, 0, 8, 0, 4, 256, 2, 0, 4)           \
  /* the fused 4096-point FP32 rows at one line per 256-thread CTA */   \
  X(float, 4, 1, MODE_CONV, 0, 12, 0, 0, 256, 4, 0, 4)           \
  X(float, 4, 1, MODE_CONV, 0, 12, 0, 0, 256, 3, 0, 4)           \
  /* the fused 128-point FP32 rows: sixteen lines per 128-thread CTA at */ \
  /* eight CTAs per SM (the default) 107.1 us on 512 x 256 x 128, at six */  \
  /* 109.3, thirty-two lines per 256-thread CTA at three 118.4 */            \
  X(float, 4, 1, MODE_CONV, 0, 7, 0, 5, 256, 3, 0, 4)            \
  X(float, 4, 1, MODE_CONV, 0, 7, 0, 4, 128, 6, 0, 4)            \
  X(float, 4, 1, MODE_DIF, -1, 9, 1, 4, 512, 1, 0, 4)            \
  X(float, 4, 1, MODE_DIT, +1, 9, 1, 4, 512, 1, 0, 4)            \
  X(float, 4, 1, MODE_CONV, 0, 7, 0, 5, 256, 2, 0, 4)            \
  /* tensor-core form, 2048-point rows and 8-line columns */             \
  X(float, 4, 1, MODE_CONV, 0, 11, 0, 0, 128, 5, 1, 4)           \
  X(float, 4, 1, MODE_DIF, -1, 11, 1, 3, 512, 1, 1, 4)           \
  X(float, 4, 1, MODE_DIT, +1, 11, 1, 3, 512, 1, 1, 4)           \
  /* (the fused pass with one line per 128-thread CTA at five CTAs per */ \
  /* SM, 96 registers, ran 55.2 us against 59.1 for two lines per */       \
  /* 256-thread CTA at three CTAs per SM (80 registers; 62.7 us at two), */ \
  /* one line at seven CTAs per SM (72 registers, 12 bytes of spills) */   \
  /* 55.6 us) */                                                             \
  X(float, 4, 1, MODE_CONV, 0, 11, 0, 1, 256, 3, 1, 4)           \
  X(float, 4, 1, MODE_CONV, 0, 11, 0, 1, 256, 2, 1, 4)           \
  X(float, 4, 1, MODE_CONV, 0, 11, 0, 0, 128, 7, 1, 4)
// Measured on C3 (2048^2): FP64 columns W=4 (32-byte rows) 53 us vs W=2
// 68 us; FP32 columns W=8 34 us vs W=4 45 us -- row width, not occupancy,
// bounds these passes (the narrower tiles were dropped from the list), and
// neither do more warps: FP32 columns at 1024 threads per CTA (64 registers,
// no spills) ran 30.0 / 30.6 us against 31.2 / 30.1 us.  Radix-8 schedules
// for 2048-point FP64 lines (RC = 3: fused pass at three 256-thread CTAs per
// SM, 80 registers; columns at 1024 threads, 64 registers) ran 67 / 62 / 63
// us against 54 / 47 / 51 us: the fourth stage's shared-memory round trip
// costs more than the extra warps recover.  On 3D 512 x 256 x 128 FP32 the specialised passes
// gain 4% over the generic kernel (256^3: 1%); specialising FP64 256-point
// passes and the base-4 4096/16-point passes of 1D 2^16 measured 2-5%
// slower than the generic kernel, so those shapes stay generic.
// (a geometry may have several candidates; the first is the default and
// PAC_SPECIAL_VARIANT=k or the tuner knob special = k selects the k-th; the
// pass descriptor records it as spec = 1 + k)

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

// Pipelined column passes (PassDesc.pipe, ColPipe): one persistent CTA per
// SM, the tile in registers, the next tile brought in by tensor copies
// while the current one computes.  Rows of W elements are 32 bytes, which
// keeps every tensor-copy x coordinate a multiple of 16 bytes.  Opt-in
// (PAC_PIPE=1): on 2048^2 the pass takes 57 / 55 us (FP64 DIF / DIT) and
// 38 / 36 us (FP32) against 54 / 51 and 36 / 33 us for the one-CTA tiles.
// Taking the loads off the critical path does not help while 16 warps per
// SM run each tile's stages in lockstep: the SM issues in ~17% of its
// cycles, waiting at the barriers between stages and on the exchanges.
// fields: element type, bytes, log2 digit base, mode, sign, log2 L, log2 W,
// threads
#define PAC_PIPE_LIST(X)                            \
  X(double, 8, 1, MODE_DIF, -1, 11, 2, 512)         \
  X(double, 8, 1, MODE_DIT, +1, 11, 2, 512)         \
  X(float, 4, 1, MODE_DIF, -1, 11, 3, 512)          \
  X(float, 4, 1, MODE_DIT, +1, 11, 3, 512)

// Column passes staged by tensor copies (PassDesc.tma, ColTma in
// pac_coltma.cuh): persistent CTAs, the tile moved between global and shared
// memory by tensor copies in both directions, conflict-free layouts in
// shared memory.  PIPE = 1: the pipelined variant (tile in registers, the
// next tile's tensor load in flight meanwhile, exchanges through a
// one-component buffer).  For each geometry the first entry is candidate 1,
// the next candidate 2, ... (PassDesc.tma = candidate); PAC_COLTMA=k picks
// the k-th, 0 none, and without it a geometry runs its DEF = 1 entry.
// Measured on 2048^2 (per DIF / DIT pass): FP64 one-CTA tiles 61.8 / 55.5 us,
// W = 2 at two CTAs per SM 62.0 / 54.0, pipelined 53.1 / 47.6, against
// 54.9 / 51.0 for the load/store-unit kernel (pac_special.h above): the
// pipelined FP64 variant is the default.  FP32: 36.8 / 32.8, 41.2 / 34.8
// and 47.4 / 36.9 (the pipelined FP32 tile spills) against 32.0 / 30.1: the
// FP32 passes kept the load/store-unit kernel.  Then the pipelined kernel
// took the stage twiddles from shared memory (ColTma::tw_fill): FP64 DIF
// 53.1 -> 50.9 us, DIT 48.1.  And its tile pointers, rounded to 1024 bytes
// as integers before, became offsets of the shared array (smem_align1024),
// so its shared accesses compile to shared rather than generic loads and
// stores: FP64 pipelined 49.6 / 45.8 us, FP32 pipelined 31.3 / 29.5 and,
// storing the result from the registers (PP = 2: the tensor-copy unit
// carries only the loads), 31.6 / 28.5 against 32.3 / 30.1 for the
// load/store-unit kernel, so PP = 2 at 512 threads is the FP32 default.
// fields: element type, bytes, log2 digit base, mode, sign, log2 L, log2 W,
// threads, CTAs per SM, pipelined, default
#define PAC_COLTMA_LIST(X)                                     \
  X(double, 8, 1, MODE_DIF, -1, 11, 2, 512, 1, 0, 0, 0)        \
  X(double, 8, 1, MODE_DIT, +1, 11, 2, 512, 1, 0, 0, 0)        \
  X(float, 4, 1, MODE_DIF, -1, 11, 3, 512, 1, 0, 0, 0)         \
  X(float, 4, 1, MODE_DIT, +1, 11, 3, 512, 1, 0, 0, 0)         \
  X(double, 8, 1, MODE_DIF, -1, 11, 1, 256, 2, 0, 0, 0)        \
  X(double, 8, 1, MODE_DIT, +1, 11, 1, 256, 2, 0, 0, 0)        \
  X(float, 4, 1, MODE_DIF, -1, 11, 2, 256, 2, 0, 0, 0)         \
  X(float, 4, 1, MODE_DIT, +1, 11, 2, 256, 2, 0, 0, 0)         \
  X(double, 8, 1, MODE_DIF, -1, 11, 2, 512, 1, 1, 1, 0)        \
  X(double, 8, 1, MODE_DIT, +1, 11, 2, 512, 1, 1, 1, 0)        \
  X(float, 4, 1, MODE_DIF, -1, 11, 3, 512, 1, 1, 0, 0)         \
  X(float, 4, 1, MODE_DIT, +1, 11, 3, 512, 1, 1, 0, 0)         \
  X(float, 4, 1, MODE_DIF, -1, 11, 3, 1024, 1, 1, 0, 0)        \
  X(float, 4, 1, MODE_DIT, +1, 11, 3, 1024, 1, 1, 0, 0)        \
  X(float, 4, 1, MODE_DIF, -1, 11, 3, 1024, 1, 0, 0, 0)        \
  X(float, 4, 1, MODE_DIT, +1, 11, 3, 1024, 1, 0, 0, 0)        \
  /* pipelined, the result stored from the registers (PP = 2) */ \
  X(double, 8, 1, MODE_DIF, -1, 11, 2, 512, 1, 2, 0, 0)        \
  X(double, 8, 1, MODE_DIT, +1, 11, 2, 512, 1, 2, 0, 0)        \
  X(float, 4, 1, MODE_DIF, -1, 11, 3, 512, 1, 2, 1, 0)         \
  X(float, 4, 1, MODE_DIT, +1, 11, 3, 512, 1, 2, 1, 0)         \
  X(float, 4, 1, MODE_DIF, -1, 11, 3, 1024, 1, 2, 0, 0)        \
  X(float, 4, 1, MODE_DIT, +1, 11, 3, 1024, 1, 2, 0, 0)        \
  /* 3D FP32: 256- and 512-point columns of 16 lines (64-byte rows), */ \
  /* pipelined at three (256) and two (512) CTAs per SM.  On 256^3 (line */ \
  /* schedule) the four column passes took 59 / 51 / 54 / 51 us with */     \
  /* tensor stores (the default), 59 / 53 / 53 / 53 with direct stores, */  \
  /* against 75 / 70 / 73 / 72 for the load/store-unit kernel */            \
  X(float, 4, 1, MODE_DIF, -1, 8, 4, 256, 3, 2, 0, 0)          \
  X(float, 4, 1, MODE_DIT, +1, 8, 4, 256, 3, 2, 0, 0)          \
  X(float, 4, 1, MODE_DIF, -1, 8, 4, 256, 3, 1, 1, 0)          \
  X(float, 4, 1, MODE_DIT, +1, 8, 4, 256, 3, 1, 1, 0)          \
  X(float, 4, 1, MODE_DIF, -1, 9, 4, 512, 2, 2, 0, 0)          \
  X(float, 4, 1, MODE_DIT, +1, 9, 4, 512, 2, 2, 0, 0)          \
  X(float, 4, 1, MODE_DIF, -1, 9, 4, 512, 2, 1, 1, 0)          \
  X(float, 4, 1, MODE_DIT, +1, 9, 4, 512, 2, 1, 1, 0)          \
  /* 3D FP64: 256- and 512-point columns of 8 lines (64-byte rows) */ \
  /* (on 256^3 98-112 against 183-193 us per pass for the */        \
  /* load/store-unit kernel; direct stores 100-138 us) */                \
  X(double, 8, 1, MODE_DIF, -1, 8, 3, 128, 3, 1, 1, 0)         \
  X(double, 8, 1, MODE_DIT, +1, 8, 3, 128, 3, 1, 1, 0)         \
  X(double, 8, 1, MODE_DIF, -1, 9, 3, 256, 2, 1, 1, 0)         \
  X(double, 8, 1, MODE_DIT, +1, 9, 3, 256, 2, 1, 1, 0)         \
  X(double, 8, 1, MODE_DIF, -1, 8, 3, 128, 3, 2, 0, 0)         \
  X(double, 8, 1, MODE_DIT, +1, 8, 3, 128, 3, 2, 0, 0)         \
  X(double, 8, 1, MODE_DIF, -1, 9, 3, 256, 2, 2, 0, 0)         \
  X(double, 8, 1, MODE_DIT, +1, 9, 3, 256, 2, 2, 0, 0)         \
  /* tensor-core form: radix-16 steps on tcgen05 MMAs */         \
  X(float, 4, 1, MODE_DIF, -1, 11, 3, 512, 1, 0, 0, 1)         \
  X(float, 4, 1, MODE_DIT, +1, 11, 3, 512, 1, 0, 0, 1)

// the variant-th candidate of a geometry (variant < 0: its default entry);
// *cand returns its 1-based candidate number
inline bool coltma_geometry(int bytes, int b2, int mode, int sign, int logL, int tc, int* logW,
                            int* nt, int* minb, int* pipe, int variant, int* cand) {
  int seen = 0;
#define PAC_X(T, BY, B2_, MO, SG, LL, LW, NT_, MB, PP, DF, TC_)                           \
  if (bytes == BY && b2 == B2_ && mode == MO && sign == SG && logL == LL && tc == TC_ && \
      (variant < 0 ? (++seen, DF == 1) : seen++ == variant)) {                         \
    *logW = LW;                                                                        \
    *nt = NT_;                                                                         \
    *minb = MB;                                                                        \
    *pipe = PP;                                                                        \
    *cand = variant < 0 ? seen : variant + 1;                                          \
    return true;                                                                       \
  }
  PAC_COLTMA_LIST(PAC_X)
#undef PAC_X
  return false;
}

// Plane passes of 3D convolutions (PassDesc.plane, pac_plane.cuh): axes 1
// and 2 of every N1 x N2 plane in one launch on a cluster of 2^LOGC CTAs.
// fields: element type, bytes, log2 digit base, log2 N1, log2 N2, log2
// cluster size, threads, CTAs per SM
#define PAC_PLANE_LIST(X)                          \
  X(float, 4, 1, 8, 8, 3, 256, 2)                  \
  X(float, 4, 1, 8, 7, 2, 256, 2)                  \
  X(double, 8, 1, 8, 8, 3, 256, 1)                 \
  X(double, 8, 1, 8, 7, 2, 256, 1)

inline bool plane_geometry(int bytes, int b2, int logN1, int logN2, int* logC, int* nt) {
#define PAC_X(T, BY, B2_, L1, L2, LC, NT_, MB)                                        \
  if (bytes == BY && b2 == B2_ && logN1 == L1 && logN2 == L2) {                     \
    *logC = LC;                                                                     \
    *nt = NT_;                                                                      \
    return true;                                                                    \
  }
  PAC_PLANE_LIST(PAC_X)
#undef PAC_X
  return false;
}

// Work-queue fast paths (pac_queue_kernel, 256 threads): multi-plan passes
// of these geometries get their tile width and run the compile-time body
// (pass_body_ct) inside the persistent queue kernel; all others run the
// generic body.  The FP32 base-2 geometries that carry most of the elements
// of uneven 1D/2D batches (fused 2048-point rows; 512-, 256- and 128-point
// columns, the outer factors of 2^18..2^20-point lines).
// fields: element type, bytes, log2 digit base, mode, sign, log2 L, column
// tile, log2 W, tensor-core form
#define PAC_QUEUE_LIST(X)                            \
  X(float, 4, 1, MODE_CONV, 0, 11, 0, 2, 0)          \
  X(float, 4, 1, MODE_DIF, -1, 9, 1, 4, 0)           \
  X(float, 4, 1, MODE_DIT, +1, 9, 1, 4, 0)           \
  X(float, 4, 1, MODE_DIF, -1, 8, 1, 5, 0)           \
  X(float, 4, 1, MODE_DIT, +1, 8, 1, 5, 0)           \
  X(float, 4, 1, MODE_DIF, -1, 7, 1, 6, 0)           \
  X(float, 4, 1, MODE_DIT, +1, 7, 1, 6, 0)
enum { PAC_QUEUE_THREADS = 256 };

inline bool queue_geometry(int bytes, int b2, int mode, int sign, int logL, int cols, int tc,
                           int* logW) {
#define PAC_X(T, BY, B2_, MO, SG, LL, CO, LW, TC_)                                     \
  if (bytes == BY && b2 == B2_ && mode == MO && (MO == MODE_CONV || sign == SG) &&  \
      logL == LL && cols == CO && tc == TC_) {                                      \
    *logW = LW;                                                                     \
    return true;                                                                    \
  }
  PAC_QUEUE_LIST(PAC_X)
#undef PAC_X
  return false;
}

// One work item of the queue kernel (device) or of its host replay: the
// compile-time body when the descriptor is marked special and its geometry
// is on PAC_QUEUE_LIST, else the generic body.
template <typename T, int B2, int TC>
PAC_HD void queue_pass_body(const PassDesc& d, long long cta, T* sre, T* sim, const long long* lbi,
                            const long long* lbo) {
  if (d.spec) {
#define PAC_X(T_, BY, B2_, MO, SG, LL, CO, LW, TC_)                                          \
    if constexpr (sizeof(T) == BY && B2 == B2_ && TC == TC_) {                            \
      if (d.mode == MO && (MO == MODE_CONV || d.sign == SG) && d.logL == LL &&            \
          (d.logS > 0 ? 1 : 0) == CO && d.logW == LW) {                                   \
        constexpr int P_ = pitch_for(BY, LL, 1 << LW, CO, TC_);                           \
        pass_body_ct<T, B2, MO, SG, Shape<LL, LW, P_, CO, TC_>, PAC_QUEUE_THREADS,        \
                     RadsFor<LL, B2>, TC_>(d, cta, sre, sim, lbi, lbo);                   \
        return;                                                                           \
      }                                                                                   \
    }
    PAC_QUEUE_LIST(PAC_X)
#undef PAC_X
  }
  pass_body<T, B2, TC>(d, cta, sre, sim, lbi, lbo);
}

inline bool pipe_geometry(int bytes, int b2, int mode, int sign, int logL, int* logW, int* nt) {
#define PAC_X(T, BY, B2_, MO, SG, LL, LW, NT_)                                      \
  if (bytes == BY && b2 == B2_ && mode == MO && sign == SG && logL == LL) {      \
    *logW = LW;                                                                  \
    *nt = NT_;                                                                   \
    return true;                                                                 \
  }
  PAC_PIPE_LIST(PAC_X)
#undef PAC_X
  return false;
}

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

inline bool special_geometry(int bytes, int b2, int mode, int sign, int logL, int cols, int tc,
                             int rc, int* logW, int* nt, int variant = 0) {
  int seen = 0;
#define PAC_X(T, BY, B2_, MO, SG, LL, CO, LW, NT_, MB, TC_, RC_)                          \
  if (bytes == BY && b2 == B2_ && mode == MO && (MO == MODE_CONV || sign == SG) &&     \
      logL == LL && cols == CO && tc == TC_ && rc == RC_ && seen++ == variant) {       \
    *logW = LW;                                                                        \
    *nt = NT_;                                                                         \
    return true;                                                                       \
  }
  PAC_SPECIAL_LIST(PAC_X)
#undef PAC_X
  return false;
}

}  // namespace pac
