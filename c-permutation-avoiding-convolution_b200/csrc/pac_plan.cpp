// pac_plan.cpp -- plans and pass schedules behind pac.h.
//
// A plan splits every axis of the problem into "virtual axes" (factors) no
// longer than one CTA can hold in shared memory, and turns each operator
// into a sequence of passes (one kernel launch each):
//
//   A^T  (forward):  DIF passes over the factors in memory order; the outer
//                    factor of a split axis multiplies by the 4-step twiddle
//                    w_N^{i * rev(e)} after its stages.  Output: P_b order.
//   A, conj(A):      DIT passes in reverse order, 4-step twiddle before the
//                    stages of an outer factor.  Input: P_b order.
//   convolution:     DIF passes over all factors but the innermost, one fused
//                    pass (DIF stages, product with the filter spectrum at the
//                    same P_b positions, DIT stages) on the innermost factor,
//                    then the DIT passes back.  2m-1 launches for m factors;
//                    no pass ever permutes data in HBM.
//   fft / ifft:      DIF passes whose last factor per axis stores in natural
//                    order (self-sorting store of that pass).
//
// The reference performs the same factorisation with one stage per memory
// sweep (butterflies.c) and per-axis gather/scatter (butterflies_2d.c,
// butterflies_3d.c); the plan keeps its digit-reversal convention so the
// spectrum order is the reference's P_r F x.
#include <math.h>
#include <stdarg.h>
#include <stdlib.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "pac.h"
#include "pac_backend.h"
#include "pac_special.h"

namespace pac {

// ---------------------------------------------------------------------------
// error reporting
// ---------------------------------------------------------------------------
static thread_local char t_err[512];

int set_error(int status, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(t_err, sizeof(t_err), fmt, ap);
  va_end(ap);
  return status;
}

#define PAC_TRY(expr)                  \
  do {                                 \
    int _st = (expr);                  \
    if (_st != PAC_SUCCESS) return _st; \
  } while (0)

// ---------------------------------------------------------------------------
// schedules
// ---------------------------------------------------------------------------
struct VAx {
  int log;      // factor length 2^log
  int axis;     // real axis index
  int first;    // first factor of its axis
  int last;     // last (innermost) factor of its axis
  int b2;       // log2 of its axis's digit base
};

struct Schedule {
  int bytes = 8;  // element bytes of one real component
  int b2 = 1;     // log2 of the digit base
  int tc = 0;     // tensor-core form: radix-16 stages on the tensor cores
  // knobs (pac_tune_t): factor cap (0: built-in), largest stage radix (log2),
  // specialised kernels (-1 off, 0 default, k > 0 k-th candidate), tile shift
  int flog_cap = 0;
  int rlog_cap = 4;
  int special = 0;
  int w_shift = 0;
  int plane = 0;        // 3D: 1 plane schedule, -1 line schedule, 0 built-in
  void* tcc = nullptr;  // its DFT operand table (tensor-core form)
  std::vector<VAx> vax;
  std::vector<std::vector<int>> rad;  // per factor: stage radix logs, DIF order
  void* pool = nullptr;               // stage twiddle tables
  std::map<std::pair<int, int>, int> tw_off;
  struct Tw4 {
    void* lo = nullptr;
    void* hi = nullptr;
    int lolog = 0;
  };
  std::map<int, Tw4> tw4;  // keyed by log N
  ~Schedule() {
    if (pool) be_free(pool);
    if (tcc) be_free(tcc);
    for (auto& kv : tw4) {
      be_free(kv.second.lo);
      be_free(kv.second.hi);
    }
  }
};

static const int kSmemBudget = 200 * 1024;

// stage radices of one factor of length 2^lg for digit base 2^b2: with
// stages of at most 4 bits the schedule the specialised kernels are compiled
// with (sched_n / sched_v, pac_stages.cuh); a tuned plan may cap them at 3
// bits (the same rule: fewest stages, bits spread evenly, larger first)
static std::vector<int> radix_schedule(int lg, int b2, int rlog_cap = 4) {
  std::vector<int> r;
  for (int i = 0; i < sched_n_cap(lg, b2, rlog_cap); ++i)
    r.push_back(sched_v_cap(lg, b2, rlog_cap, i));
  return r;
}

// Longest factor one CTA holds: 2^12 complex FP64 / 2^13 complex FP32
// (64 KiB per line).  PAC_MAX_FACTOR_LOG lowers it, which forces more
// factors per axis (used by the tests to reach 3- and 4-factor splits at
// small sizes).
static int max_factor_log(int bytes, int b2, int cap = 0) {
  int lmax = bytes == 8 ? 12 : 13;
  const char* env = getenv("PAC_MAX_FACTOR_LOG");
  if (cap > 0) {
    if (cap >= b2 && cap < lmax) lmax = cap;
  } else if (env) {
    int v = atoi(env);
    if (v >= b2 && v < lmax) lmax = v;
  }
  return lmax - lmax % b2;
}

// Device memory for a schedule's tables: cudaMalloc'd (freed by the
// Schedule), or carved out of caller-supplied scratch (Arena; nothing to
// free).
struct Arena {
  char* cur;
  char* end;
  void* take(size_t bytes) {
    size_t a = (bytes + 255) & ~(size_t)255;
    if (cur + a > end) return nullptr;
    void* p = cur;
    cur += a;
    return p;
  }
};
static int table_alloc(Arena* ar, void** p, size_t bytes) {
  if (!ar) return be_malloc(p, bytes);
  *p = ar->take(bytes);
  return *p ? PAC_SUCCESS : set_error(PAC_ERROR_SIZE, "no-allocation scratch too small");
}

// The factors of every axis and their stage radices -- the one rule every
// plan follows (allocating plans and the no-allocation entry point alike).
static int split_axes(Schedule& s, int rank, const int* logs, const int* b2s, int bytes) {
  s.bytes = bytes;
  s.b2 = b2s[rank - 1];
  for (int a = 0; a < rank; ++a) {
    int lg = logs[a];
    if (lg == 0) continue;
    const int b2 = b2s[a];
    const int lmax = max_factor_log(bytes, b2, s.flog_cap);
    int digits = lg / b2;
    int dmax = lmax / b2;
    int nf = (digits + dmax - 1) / dmax;
    if (nf > PAC_MAX_FACTORS)
      return set_error(PAC_ERROR_SIZE, "axis %d needs %d factors (at most %d)", a, nf,
                       (int)PAC_MAX_FACTORS);
    // the innermost factor (contiguous lines, the fused pass of a
    // convolution) as long as one CTA holds; the outer factors (column
    // passes, whose tiles grow with the column length) share the rest evenly
    std::vector<int> parts(nf, 0);
    parts[nf - 1] = nf == 1 ? digits : dmax;
    const int rest = digits - parts[nf - 1];
    for (int f = 0; f < nf - 1; ++f) parts[f] = rest / (nf - 1) + (f < rest % (nf - 1) ? 1 : 0);
    for (int f = 0; f < nf; ++f) s.vax.push_back({parts[f] * b2, a, f == 0, f == nf - 1, b2});
  }
  for (auto& v : s.vax) {
    s.rad.push_back(radix_schedule(v.log, v.b2, s.rlog_cap));
    if (s.rad.back().size() > (size_t)PAC_MAX_STAGES)
      return set_error(PAC_ERROR_UNSUPPORTED_RADIX,
                       "a factor of 2^%d needs %zu stages of radix <= 2^%d (at most %d)", v.log,
                       s.rad.back().size(), s.rlog_cap, (int)PAC_MAX_STAGES);
  }
  return PAC_SUCCESS;
}

// Stage and 4-step twiddle tables of a split schedule, in memory from
// table_alloc, generated on `stream`.
static int build_tables(Schedule& s, Arena* ar, void* stream) {
  const int bytes = s.bytes;
  std::vector<std::pair<int, int>> specs;
  long long total = 0;
  for (size_t i = 0; i < s.vax.size(); ++i) {
    int logK = s.vax[i].log;
    for (int rl : s.rad[i]) {
      std::pair<int, int> key(logK, rl);
      if (!s.tw_off.count(key) && logK > rl) {
        s.tw_off[key] = (int)total;
        specs.push_back(key);
        total += (1LL << (logK - rl)) * ((1LL << rl) - 1);
      }
      logK -= rl;
    }
  }
  if (total > 0) {
    PAC_TRY(table_alloc(ar, &s.pool, (size_t)total * 2 * bytes));
    for (auto& k : specs) {
      char* dst = (char*)s.pool + (size_t)s.tw_off[k] * 2 * bytes;
      PAC_TRY(be_fill_stage_tw(dst, bytes, k.first, k.second, stream));
    }
  }
  // 4-step twiddles: for every non-last factor, N = L * (later factors of its axis)
  for (size_t i = 0; i < s.vax.size(); ++i) {
    if (s.vax[i].last) continue;
    int logN = 0;
    for (size_t j = i; j < s.vax.size() && s.vax[j].axis == s.vax[i].axis; ++j) logN += s.vax[j].log;
    if (s.tw4.count(logN)) continue;
    Schedule::Tw4 t;
    t.lolog = (logN + 1) / 2;
    long long nlo = 1LL << t.lolog, nhi = 1LL << (logN - t.lolog);
    PAC_TRY(table_alloc(ar, &t.lo, (size_t)nlo * 2 * bytes));
    int st = table_alloc(ar, &t.hi, (size_t)nhi * 2 * bytes);
    if (st != PAC_SUCCESS) {
      if (!ar) be_free(t.lo);
      return st;
    }
    s.tw4[logN] = t;
    PAC_TRY(be_fill_pow_tw(t.lo, bytes, nlo, 1, logN, stream));
    PAC_TRY(be_fill_pow_tw(t.hi, bytes, nhi, nlo, logN, stream));
  }
  return PAC_SUCCESS;
}

static int build_schedule(Schedule& s, int rank, const int* logs, const int* b2s, int bytes) {
  PAC_TRY(split_axes(s, rank, logs, b2s, bytes));
  PAC_TRY(build_tables(s, nullptr, nullptr));
  // the tables are filled on the legacy stream, which does not order against
  // non-blocking streams: finish them before the plan is handed out
  return be_stream_sync(nullptr);
}

}  // namespace pac

// ---------------------------------------------------------------------------
// the plan object
// ---------------------------------------------------------------------------
struct pac_plan_s {
  int rank = 0;
  int dims[3] = {1, 1, 1};
  int logs[3] = {0, 0, 0};
  long long batch = 1;
  int b2 = 1;                // axis 0's digit base (log2)
  int b2s[3] = {1, 1, 1};    // every axis's
  int form = PAC_FORM_F64;
  long long N = 1;
  pac_tune_t tune = {0, 0, 0, 0, 0};      // knobs the plan was built with
  pac::Schedule main;                     // storage type of the form
  std::unique_ptr<pac::Schedule> s64;     // FP64 schedule (F32 form: filter spectrum)
  std::mutex ws_mu;
  void* ws = nullptr;  // workspace: 2 arrays of batch*N elements of the storage type
  size_t ws_bytes = 0;
  void* tmp64 = nullptr;  // FP64 temporary for the F32 filter spectrum
  size_t tmp64_bytes = 0;
  // device status word of the bounded waits (pac_plan_check_status) and
  // their spin limit in SM cycles (0: the kernels' default)
  int* status = nullptr;
  long long wait_limit = 0;
  // per-pass timing (pac_plan_set_pass_timing)
  int timing = 0;
  std::mutex t_mu;
  std::vector<void*> t_ev;
  std::vector<double> t_ms;
  long long t_calls = 0;
  ~pac_plan_s() {
    if (ws) pac::be_free(ws);
    if (tmp64) pac::be_free(tmp64);
    if (status) pac::be_free(status);
    for (void* e : t_ev) pac::be_event_destroy(e);
  }
};

namespace pac {

struct PassSpec {
  PassDesc d;
  long long grid;
  int threads;
  size_t smem;
  bool oop;  // cannot run in place
  int b2;    // log2 digit base of the pass's axis
};

// geometry of a pass over factor vi for `batch` problems
static PassSpec make_pass(const Schedule& s, int vi, long long batch, long long N) {
  PassSpec p;
  PassDesc& d = p.d;
  memset(&d, 0, sizeof(d));
  const VAx& v = s.vax[vi];
  const int esz = s.bytes;
  const int SH = esz == 8 ? 4 : 5, NB = esz == 8 ? 16 : 32;
  d.L = 1 << v.log;
  d.logL = v.log;
  int logS = 0;
  for (size_t j = vi + 1; j < s.vax.size(); ++j) logS += s.vax[j].log;
  d.logS = logS;
  d.nlines = (batch * N) >> v.log;
  const int base_pitch = d.L + (d.L >> SH);
  long long target = (esz == 8 ? 4096 : 8192) >> v.log;
  long long W = target < 1 ? 1 : target;
  if (logS > 0) {
    if (W < 16) W = 16;
    if (W > (1LL << logS)) W = 1LL << logS;
  }
  if (s.w_shift > 0) W <<= s.w_shift;
  if (s.w_shift < 0) W >>= -s.w_shift;
  if (W < 1) W = 1;
  long long wmax = kSmemBudget / (2LL * esz * (base_pitch + NB));
  if (wmax < 1) wmax = 1;
  while (W > wmax) W >>= 1;
  if (W > 64) W = 64;
  // tiles must cover the lines exactly: W divides nlines (a batch that is
  // not a power of two makes nlines odd-factored)
  const long long lowbit = d.nlines & -d.nlines;
  if (W > lowbit) W = lowbit;
  if (W < 1) W = 1;
  d.W = (int)W;
  d.logW = 0;
  while ((1 << d.logW) < d.W) ++d.logW;
  d.pitch = pitch_for(esz, v.log, d.W);
  d.tc = s.tc;
  d.tcc = s.tcc;
  const std::vector<int>& rad = s.rad[vi];
  d.nst = (int)rad.size();
  int logK = v.log;
  int min_rl = 4;
  for (int i = 0; i < d.nst; ++i) {
    d.rlog[i] = rad[i];
    auto it = s.tw_off.find(std::make_pair(logK, rad[i]));
    d.tw_off[i] = it == s.tw_off.end() ? 0 : it->second;
    logK -= rad[i];
    if (rad[i] < min_rl) min_rl = rad[i];
  }
  d.tw = s.pool;
  long long bf = (long long)d.W << (v.log - 4 > 0 ? v.log - 4 : 0);
  int threads = (int)(bf < 32 ? 32 : bf > 256 ? 256 : bf);
  threads = (threads + 31) / 32 * 32;
  d.nthreads = threads;
  if (!v.last) {
    int logGin = 0, logSreal = 0;
    for (size_t j = vi + 1; j < s.vax.size(); ++j) {
      if (s.vax[j].axis == v.axis) logGin += s.vax[j].log;
      else logSreal += s.vax[j].log;
    }
    int logN = v.log + logGin;
    auto& t = s.tw4.at(logN);
    d.tw4_shift = logSreal;
    d.tw4_mask = (1LL << logGin) - 1;
    d.tw4_lolog = t.lolog;
    d.tw4_lo = t.lo;
    d.tw4_hi = t.hi;
  }
  p.grid = d.nlines / d.W;
  p.threads = threads;
  p.smem = (size_t)2 * d.W * d.pitch * esz;
  p.oop = false;
  p.b2 = v.b2;
  return p;
}

// Switch a pass to its specialised kernel when pac_special.h has one for its
// geometry and the tile fits the lines (W divides nlines and the stride).
static void apply_special(const Schedule& s, PassSpec& p) {
  PassDesc& d = p.d;
  int logW = 0, nt = 0;
  if (d.nat || d.plane) return;
  if (s.special < 0) return;  // tuned off
  // column pass whose tile a CTA cluster shares (W columns within the
  // stride, whole tiles), opt-in: PAC_CLUSTER_VARIANT=k picks the k-th
  // candidate geometry of the cluster list
  // (the cluster and pipelined variants have no tensor-core stages)
  // (the cluster and pipelined variants run the radix-16 schedule only)
  const char* cvar = d.tc || s.rlog_cap < 4 ? nullptr : getenv("PAC_CLUSTER_VARIANT");
  if (d.logS > 0 && cvar != nullptr) {
    int logC = 0;
    if (cluster_geometry(s.bytes, p.b2, d.mode, d.sign, d.logL, &logW, &logC, &nt, atoi(cvar)) &&
        logW <= d.logS && (d.nlines & ((1LL << logW) - 1)) == 0) {
      d.W = 1 << logW;
      d.logW = logW;
      d.logC = logC;
      d.pitch = pitch_for(s.bytes, d.logL - logC, d.W);
      d.nthreads = nt;
      d.spec = 1;
      p.threads = nt;
      p.grid = (d.nlines >> logW) << logC;
      p.smem = (size_t)2 * d.W * d.pitch * s.bytes;
      return;
    }
  }
  // pipelined column pass, opt-in (PAC_PIPE=1): persistent CTAs, one per
  // SM, tensor-copy prefetch of the next tile (16-byte aligned input arrays
  // for the tensor maps)
  const char* pipe = d.tc || s.rlog_cap < 4 ? nullptr : getenv("PAC_PIPE");
  if (d.logS > 0 && cvar == nullptr && pipe != nullptr && atoi(pipe) != 0 &&
      pipe_geometry(s.bytes, p.b2, d.mode, d.sign, d.logL, &logW, &nt) && logW <= d.logS &&
      (d.nlines & ((1LL << logW) - 1)) == 0 && (d.nlines >> d.logS) < (1LL << 31) &&
      ((uintptr_t)d.in_re | (uintptr_t)d.in_im) % 16 == 0) {
    d.W = 1 << logW;
    d.logW = logW;
    d.pitch = pitch_for(s.bytes, d.logL, d.W);
    d.nthreads = nt;
    d.spec = 1;
    d.pipe = 1;
    const long long tiles = d.nlines >> logW;
    const long long sms = be_num_sms();
    p.threads = nt;
    p.grid = tiles < sms ? tiles : sms;
    p.smem = (size_t)2 * d.W * d.L * s.bytes + (size_t)d.W * d.pitch * s.bytes + 1024;
    return;
  }
  // column pass staged by tensor copies: PAC_COLTMA=k picks the k-th
  // candidate of its geometry, 0 none; unset, the geometry's default entry.
  // Plain DIF / DIT passes of the default radix schedule, 16-byte aligned
  // arrays; not with specialised kernels tuned off.
  const char* tv = getenv("PAC_COLTMA");
  const int tvar = (s.rlog_cap < 4 || s.special < 0) ? 0 : tv ? atoi(tv) : -1;
  int tminb = 1, tpipe = 0, tcand = 0;
  if (d.logS > 0 && cvar == nullptr && tvar != 0 && d.tw4 == 0 &&
      (d.mode == MODE_DIF || d.mode == MODE_DIT) &&
      coltma_geometry(s.bytes, p.b2, d.mode, d.sign, d.logL, d.tc, &logW, &nt, &tminb, &tpipe,
                      tvar > 0 ? tvar - 1 : -1, &tcand) &&
      rads_match(d, d.logL, p.b2, 4) && logW <= d.logS &&
      (d.nlines & ((1LL << logW) - 1)) == 0 && (d.nlines >> d.logS) < (1LL << 31) &&
      ((uintptr_t)d.in_re | (uintptr_t)d.in_im | (uintptr_t)d.out_re | (uintptr_t)d.out_im) %
              16 == 0) {
    d.W = 1 << logW;
    d.logW = logW;
    d.nthreads = nt;
    d.spec = 1;
    d.tma = tcand;
    const long long tiles = d.nlines >> logW;
    const long long slots = (long long)be_num_sms() * tminb;
    p.threads = nt;
    p.grid = tiles < slots ? tiles : slots;
    p.smem = (size_t)(tpipe ? 3 : 2) * d.W * d.L * s.bytes + 1024;
    // tensor-core form: per warpgroup two 8 KB operand tiles, and the DFT
    // operand's two 2 KB tiles
    if (d.tc) p.smem += (size_t)(nt / 128) * 16384 + 4096;
    return;
  }
  const char* var = getenv("PAC_SPECIAL_VARIANT");
  int variant = s.special > 0 ? s.special : var ? atoi(var) : 0;
  const int cols = d.logS > 0 ? 1 : 0;
  const int rc = s.rlog_cap < 4 ? s.rlog_cap : 4;
  if (!special_geometry(s.bytes, p.b2, d.mode, d.sign, d.logL, cols, d.tc, rc, &logW, &nt,
                        variant)) {
    variant = 0;
    if (!special_geometry(s.bytes, p.b2, d.mode, d.sign, d.logL, cols, d.tc, rc, &logW, &nt))
      return;
  }
  const long long W = 1LL << logW;
  if ((d.nlines & (W - 1)) != 0) return;
  if (d.logS > 0 && logW > d.logS) return;
  d.W = (int)W;
  d.logW = logW;
  d.pitch = pitch_for(s.bytes, d.logL, d.W, cols, d.tc);
  d.nthreads = nt;
  d.spec = 1 + variant;
  p.threads = nt;
  p.grid = d.nlines / W;
  p.smem = (size_t)2 * d.W * d.pitch * s.bytes;
}

// A multi-plan pass whose geometry has a work-queue fast path
// (PAC_QUEUE_LIST): its tile width, and the mark that selects the
// compile-time body inside pac_queue_kernel.
static void apply_queue_special(const Schedule& s, PassSpec& p) {
  PassDesc& d = p.d;
  int logW = 0;
  const int cols = d.logS > 0 ? 1 : 0;
  if (d.nat || s.special < 0 || s.rlog_cap < 4) return;
  if (!queue_geometry(s.bytes, p.b2, d.mode, d.sign, d.logL, cols, d.tc, &logW)) return;
  const long long W = 1LL << logW;
  if ((d.nlines & (W - 1)) != 0 || (cols && logW > d.logS)) return;
  d.W = (int)W;
  d.logW = logW;
  d.pitch = pitch_for(s.bytes, d.logL, d.W, cols, d.tc);
  d.nthreads = PAC_QUEUE_THREADS;
  d.spec = 1;
  p.threads = PAC_QUEUE_THREADS;
  p.grid = d.nlines / W;
  p.smem = (size_t)2 * d.W * d.pitch * s.bytes;
}

// A pass of one stage reads global memory into registers and writes them
// back (no exchange through shared memory, unless it stores in natural order
// out of shared memory): it reserves none, so more CTAs fit per SM.
static size_t pass_smem(const PassSpec& p) {
  const PassDesc& d = p.d;
  return (d.nst == 1 && !d.nat && !d.pipe && d.logC == 0) ? 0 : p.smem;
}

// NVTX range name of a pass: its mode and line length, as bench.py names
// the passes of its per-pass breakdown ("DIF factor k", "fused innermost",
// "DIT factor k")
static void pass_range_name(const PassDesc& d, int index, char* buf, size_t n) {
  const char* mode = d.mode == MODE_CONV ? "fused innermost: DIF, x Hhat, DIT"
                     : d.mode == MODE_DIF ? "DIF" : "DIT";
  snprintf(buf, n, "pac pass %d %s 2^%d%s%s", index, mode, d.logL, d.logS > 0 ? " columns" : "",
           d.tma ? " (tensor copies)" : "");
}

static int launch(const Schedule& s, PassSpec& p, void* stream, int index = 0) {
  p.smem = pass_smem(p);
  char name[96];
  pass_range_name(p.d, index, name, sizeof(name));
  nvtxRangePushA(name);
  const int st = be_launch_pass(p.d, s.bytes, p.b2, p.grid, p.threads, p.smem, stream);
  nvtxRangePop();
  return st;
}

// Launch a pass list; with pass timing enabled, bracket every pass with
// events and accumulate the per-pass milliseconds in the plan.
static int exec_passes(pac_plan_s* pl, const Schedule& s, std::vector<PassSpec>& passes,
                       void* stream) {
  for (auto& p : passes) {
    p.d.status = pl->status;
    p.d.wait_limit = pl->wait_limit;
    apply_special(s, p);
  }
  if (!pl->timing) {
    for (size_t i = 0; i < passes.size(); ++i) PAC_TRY(launch(s, passes[i], stream, (int)i));
    return PAC_SUCCESS;
  }
  std::lock_guard<std::mutex> g(pl->t_mu);
  const size_t n = passes.size();
  while (pl->t_ev.size() < n + 1) {
    void* ev = nullptr;
    PAC_TRY(be_event_create(&ev));
    pl->t_ev.push_back(ev);
  }
  if (pl->t_ms.size() != n) {
    pl->t_ms.assign(n, 0.0);
    pl->t_calls = 0;
  }
  PAC_TRY(be_event_record(pl->t_ev[0], stream));
  for (size_t i = 0; i < n; ++i) {
    PAC_TRY(launch(s, passes[i], stream, (int)i));
    PAC_TRY(be_event_record(pl->t_ev[i + 1], stream));
  }
  for (size_t i = 0; i < n; ++i) {
    float ms = 0.f;
    PAC_TRY(be_event_elapsed(pl->t_ev[i], pl->t_ev[i + 1], &ms));
    pl->t_ms[i] += ms;
  }
  pl->t_calls++;
  return PAC_SUCCESS;
}

static int get_ws(pac_plan_s* pl, size_t bytes, void** out) {
  if (pl->ws_bytes < bytes) {
    if (pl->ws) be_free(pl->ws);
    pl->ws = nullptr;
    pl->ws_bytes = 0;
    PAC_TRY(be_malloc(&pl->ws, bytes));
    pl->ws_bytes = bytes;
  }
  *out = pl->ws;
  return PAC_SUCCESS;
}

// Run one operator of schedule s over `batch` problems.
static int run_transform(pac_plan_s* pl, const Schedule& s, int op, long long batch,
                         const void* in_re, const void* in_im, void* out_re, void* out_im,
                         double scale, int use_scale, void* stream) {
  const long long N = pl->N;
  const int m = (int)s.vax.size();
  const long long total = batch * N;
  if (m == 0) {
    double sc = use_scale ? scale : 1.0;
    return be_scale_copy(total, s.bytes, in_re, in_im, out_re, out_im, sc, stream);
  }
  std::vector<PassSpec> passes;
  if (op == PAC_OP_AT || op == PAC_OP_FFT || op == PAC_OP_IFFT) {
    int sign = (op == PAC_OP_IFFT) ? +1 : -1;
    for (int vi = 0; vi < m; ++vi) {
      PassSpec p = make_pass(s, vi, batch, N);
      p.d.mode = MODE_DIF;
      p.d.sign = sign;
      p.d.tw4 = s.vax[vi].last ? 0 : 1;
      if (op != PAC_OP_AT && s.vax[vi].last) {
        // natural-order store of this axis
        p.d.nat = 1;
        int nf = 0, Mlog = 0;
        for (int j = vi - 1; j >= 0 && s.vax[j].axis == s.vax[vi].axis; --j) ++nf;
        for (int f = 0; f < nf; ++f) {
          p.d.nat_flog[f] = s.vax[vi - nf + f].log;
          Mlog += s.vax[vi - nf + f].log;
        }
        p.d.nat_nf = nf;
        p.d.nat_Mlog = Mlog;
        p.oop = nf > 0;
      }
      passes.push_back(p);
    }
  } else {
    int sign = (op == PAC_OP_A || op == PAC_OP_UFFT) ? -1 : +1;
    for (int vi = m - 1; vi >= 0; --vi) {
      PassSpec p = make_pass(s, vi, batch, N);
      p.d.mode = MODE_DIT;
      p.d.sign = sign;
      p.d.tw4 = s.vax[vi].last ? 0 : 2;
      passes.push_back(p);
    }
  }
  if (use_scale) {
    passes.back().d.use_scale = 1;
    passes.back().d.scale = scale;
  }
  // buffer sequence: the last pass must write `out`
  const size_t arr_bytes = (size_t)total * s.bytes;
  int flips = 0;
  for (size_t i = 1; i < passes.size(); ++i) flips += passes[i].oop ? 1 : 0;
  void* ws = nullptr;
  bool need_ws = flips > 0 || (passes[0].oop && in_re == out_re);
  std::unique_lock<std::mutex> lk(pl->ws_mu, std::defer_lock);
  if (need_ws) {
    lk.lock();
    PAC_TRY(get_ws(pl, 2 * arr_bytes, &ws));
  }
  void* bre[2] = {out_re, ws};
  void* bim[2] = {out_im, ws ? (char*)ws + arr_bytes : nullptr};
  int cur = (flips % 2 == 0) ? 0 : 1;
  if (passes[0].oop && in_re == bre[cur]) cur ^= 1;  // only when in == out
  const void* src_re = in_re;
  const void* src_im = in_im;
  for (size_t i = 0; i < passes.size(); ++i) {
    PassSpec& p = passes[i];
    int dst = cur;
    if (i > 0 && p.oop) dst = cur ^ 1;
    p.d.in_re = src_re;
    p.d.in_im = src_im;
    p.d.out_re = bre[dst];
    p.d.out_im = bim[dst];
    cur = dst;
    src_re = bre[cur];
    src_im = bim[cur];
  }
  PAC_TRY(exec_passes(pl, s, passes, stream));
  if (cur != 0) PAC_TRY(be_memcpy(out_re, bre[cur], arr_bytes, CPY_D2D, stream));
  if (cur != 0) PAC_TRY(be_memcpy(out_im, bim[cur], arr_bytes, CPY_D2D, stream));
  return PAC_SUCCESS;
}

// The passes of one convolution call (2m - 1 for m factors): DIF over the
// outer factors, the fused innermost pass, DIT back; all in place in y.
// The plane schedule of a 3D convolution (pac_plane.cuh): the knob plane
// (or, at its built-in 0, PAC_PLANE=1/0; unset: off), one factor per axis,
// the default radix schedules, and a plane kernel compiled for the (N1, N2)
// planes.  Measured on FP32 256^3: 35% fewer DRAM bytes per convolution;
// against the line schedule with load/store-unit column passes the same
// time (and 13% faster on 512 x 256 x 128), but with the tensor-copy column
// passes the line schedule is faster on both (0.297 against 0.345 ms, 0.333
// against 0.350 ms), so it is the built-in choice and the tuner may still
// pick the plane schedule.
static bool plane_active(const Schedule& s, int* logC = nullptr, int* nt = nullptr) {
  int want = s.plane;
  if (want == 0) {
    const char* e = getenv("PAC_PLANE");
    want = e ? (atoi(e) ? 1 : -1) : -1;
  }
  if (want <= 0 || s.tc || s.rlog_cap < 4 || s.vax.size() != 3) return false;
  for (int i = 0; i < 3; ++i)
    if (!s.vax[i].first || !s.vax[i].last || s.vax[i].axis != i) return false;
  const int b2 = s.vax[1].b2;
  if (s.vax[2].b2 != b2) return false;
  int lc = 0, n = 0;
  if (!plane_geometry(s.bytes, b2, s.vax[1].log, s.vax[2].log, &lc, &n)) return false;
  if (s.rad[1] != radix_schedule(s.vax[1].log, b2) || s.rad[2] != radix_schedule(s.vax[2].log, b2))
    return false;
  if (logC) *logC = lc;
  if (nt) *nt = n;
  return true;
}

// The plane pass of a 3D plan over `batch` problems, in place in y: axes 1
// and 2 of every plane, stages of axis 1 then axis 2 in rlog / tw_off.
static PassSpec make_plane_pass(const Schedule& s, long long batch, long long N) {
  int logC = 0, nt = 0;
  plane_active(s, &logC, &nt);
  PassSpec p = make_pass(s, 2, batch, N);
  PassDesc& d = p.d;
  const int log1 = s.vax[1].log, log2 = s.vax[2].log;
  d.plane = 1;
  d.plane_logN1 = log1;
  d.plane_logN2 = log2;
  d.plane_n1s = (int)s.rad[1].size();
  d.nst = (int)(s.rad[1].size() + s.rad[2].size());
  int k = 0;
  for (int a = 1; a <= 2; ++a) {
    int logK = s.vax[a].log;
    for (int rl : s.rad[a]) {
      d.rlog[k] = rl;
      auto it = s.tw_off.find(std::make_pair(logK, rl));
      d.tw_off[k] = it == s.tw_off.end() ? 0 : it->second;
      logK -= rl;
      ++k;
    }
  }
  const int rc = 1 << (log1 - logC);
  d.W = rc;
  d.logW = log1 - logC;
  d.pitch = pitch_for(s.bytes, log2, rc);
  d.nthreads = nt;
  p.threads = nt;
  p.grid = ((batch * N) >> (log1 + log2)) << logC;
  p.smem = (size_t)2 * rc * d.pitch * s.bytes;
  return p;
}

static void build_conv_passes(pac_plan_s* pl, const void* x_re, const void* x_im,
                              const void* h_re, const void* h_im, int per_problem, void* y_re,
                              void* y_im, double scale, std::vector<PassSpec>& passes,
                              bool allow_plane = true) {
  const Schedule& s = pl->main;
  const long long N = pl->N;
  const int m = (int)s.vax.size();
  const long long hmask = per_problem ? -1LL : (N - 1);
  if (allow_plane && plane_active(s)) {
    // DIF axis 0, the plane pass, DIT axis 0
    PassSpec a = make_pass(s, 0, pl->batch, N);
    a.d.mode = MODE_DIF;
    a.d.sign = -1;
    a.d.in_re = x_re;
    a.d.in_im = x_im;
    a.d.out_re = y_re;
    a.d.out_im = y_im;
    passes.push_back(a);
    PassSpec p = make_plane_pass(s, pl->batch, N);
    p.d.mode = MODE_CONV;
    p.d.h_re = h_re;
    p.d.h_im = h_im;
    p.d.h_mask = hmask;
    p.d.scale = scale;
    p.d.in_re = y_re;
    p.d.in_im = y_im;
    p.d.out_re = y_re;
    p.d.out_im = y_im;
    passes.push_back(p);
    PassSpec c = make_pass(s, 0, pl->batch, N);
    c.d.mode = MODE_DIT;
    c.d.sign = +1;
    c.d.in_re = y_re;
    c.d.in_im = y_im;
    c.d.out_re = y_re;
    c.d.out_im = y_im;
    passes.push_back(c);
    return;
  }
  for (int vi = 0; vi < m - 1; ++vi) {
    PassSpec p = make_pass(s, vi, pl->batch, N);
    p.d.mode = MODE_DIF;
    p.d.sign = -1;
    p.d.tw4 = s.vax[vi].last ? 0 : 1;
    p.d.in_re = vi == 0 ? x_re : y_re;
    p.d.in_im = vi == 0 ? x_im : y_im;
    p.d.out_re = y_re;
    p.d.out_im = y_im;
    passes.push_back(p);
  }
  {
    PassSpec p = make_pass(s, m - 1, pl->batch, N);
    p.d.mode = MODE_CONV;
    p.d.h_re = h_re;
    p.d.h_im = h_im;
    p.d.h_mask = hmask;
    p.d.scale = scale;
    p.d.in_re = m == 1 ? x_re : y_re;
    p.d.in_im = m == 1 ? x_im : y_im;
    p.d.out_re = y_re;
    p.d.out_im = y_im;
    passes.push_back(p);
  }
  for (int vi = m - 2; vi >= 0; --vi) {
    PassSpec p = make_pass(s, vi, pl->batch, N);
    p.d.mode = MODE_DIT;
    p.d.sign = +1;
    p.d.tw4 = s.vax[vi].last ? 0 : 2;
    p.d.in_re = y_re;
    p.d.in_im = y_im;
    p.d.out_re = y_re;
    p.d.out_im = y_im;
    passes.push_back(p);
  }
}

static int run_conv(pac_plan_s* pl, const void* x_re, const void* x_im, const void* h_re,
                    const void* h_im, int per_problem, void* y_re, void* y_im, double scale,
                    void* stream) {
  const Schedule& s = pl->main;
  if (s.vax.empty()) {
    const long long hmask = per_problem ? -1LL : (pl->N - 1);
    return be_pointwise(pl->batch * pl->N, s.bytes, x_re, x_im, h_re, h_im, hmask, y_re, y_im,
                        scale, stream);
  }
  std::vector<PassSpec> passes;
  build_conv_passes(pl, x_re, x_im, h_re, h_im, per_problem, y_re, y_im, scale, passes);
  return exec_passes(pl, s, passes, stream);
}

// For a batch of plans (pac_multi.cpp): the convolution pass descriptors of
// one problem in the generic kernel's geometry, with their CTA counts and
// shared-memory sizes.  A problem of one element (no factors) has none.
int plan_conv_descs(pac_plan_s* pl, const void* x_re, const void* x_im, const void* h_re,
                    const void* h_im, void* y_re, void* y_im, std::vector<PassDesc>& descs,
                    std::vector<long long>& ctas, std::vector<size_t>& smem) {
  std::vector<PassSpec> passes;
  if (!pl->main.vax.empty())  // (the work queue runs line passes only)
    build_conv_passes(pl, x_re, x_im, h_re, h_im, 0, y_re, y_im, 1.0, passes, false);
  for (auto& p : passes) apply_queue_special(pl->main, p);
  for (auto& p : passes) {
    p.smem = pass_smem(p);
    descs.push_back(p.d);
    ctas.push_back(p.grid);
    smem.push_back(p.smem);
  }
  return PAC_SUCCESS;
}
int plan_bytes(pac_plan_s* pl) { return pl->main.bytes; }
// the factor lengths and stage radices of the plan (the autotuner skips a
// knob set whose schedule it has already timed)
std::string plan_signature(pac_plan_s* pl) {
  std::string sig = plane_active(pl->main) ? "plane|" : "";
  for (size_t i = 0; i < pl->main.vax.size(); ++i) {
    sig += std::to_string(pl->main.vax[i].log) + ":";
    for (int r : pl->main.rad[i]) sig += std::to_string(r) + ",";
    sig += ";";
  }
  return sig;
}
int plan_b2(pac_plan_s* pl) { return pl->b2; }

// P-order FP64 spectrum -> the plan's spectrum storage: every block of R
// positions (R the last stage radix of the innermost factor, the one the
// fused pass multiplies in) transposed to stride L/R, scaled, and rounded
// once to the plan's element type.  Plan set-up work, never part of a
// convolution.
static int to_plan_order(pac_plan_s* pl, const double* in_re, const double* in_im, int nfilters,
                         void* out_re, void* out_im, double scale, void* stream) {
  const Schedule& s = pl->main;
  const long long total = (long long)nfilters * pl->N;
  if (s.vax.empty()) {
    if (s.bytes == 8)
      return be_scale_copy(total, 8, in_re, in_im, out_re, out_im, scale, stream);
    PAC_TRY(be_round_to_f32(in_re, (float*)out_re, total, stream));
    return be_round_to_f32(in_im, (float*)out_im, total, stream);
  }
  const int logL = s.vax.back().log;
  const int logR = s.rad.back().back();
  return be_plan_order(in_re, in_im, out_re, out_im, s.bytes, logL, logR, total >> logL, scale,
                       stream);
}

// ---------------------------------------------------------------------------
// 1D convolution in caller-supplied device scratch (pac_convolve_1d_noalloc).
// The twiddle tables and the filter spectrum are carved out of `scratch` in
// 256-byte aligned pieces and regenerated on `stream` by every call, so a
// call never depends on what an earlier call left there.  Nothing here
// allocates device memory.
// ---------------------------------------------------------------------------
static int build_schedule_in_arena(Schedule& s, int logn, Arena& ar, void* stream) {
  const int logs[1] = {logn}, b2s[1] = {1};
  if (logn > 0) PAC_TRY(split_axes(s, 1, logs, b2s, 8));
  return build_tables(s, &ar, stream);
}

int conv_in_scratch(void* scratch, size_t scratch_bytes, int logn, int batch, const double* x_re,
                    const double* x_im, const double* h_re, const double* h_im, double* y_re,
                    double* y_im, void* stream) {
  pac_plan_s pl;
  pl.rank = 1;
  pl.dims[0] = 1 << logn;
  pl.logs[0] = logn;
  pl.batch = batch;
  pl.b2 = 1;
  pl.form = PAC_FORM_F64;
  pl.N = 1LL << logn;
  Arena ar{(char*)scratch, (char*)scratch + scratch_bytes};
  int st = build_schedule_in_arena(pl.main, logn, ar, stream);
  double* hre = (double*)ar.take((size_t)pl.N * 8);
  double* him = (double*)ar.take((size_t)pl.N * 8);
  if (st == PAC_SUCCESS && (!hre || !him))
    st = set_error(PAC_ERROR_SIZE, "no-allocation scratch too small");
  if (st == PAC_SUCCESS)
    st = run_transform(&pl, pl.main, PAC_OP_AT, 1, h_re, h_im, hre, him, 1.0 / (double)pl.N, 1,
                       stream);
  if (st == PAC_SUCCESS) st = to_plan_order(&pl, hre, him, 1, hre, him, 1.0, stream);
  if (st == PAC_SUCCESS) st = run_conv(&pl, x_re, x_im, hre, him, 0, y_re, y_im, 1.0, stream);
  // the tables live in the caller's scratch: nothing to free
  pl.main.pool = nullptr;
  pl.main.tw4.clear();
  return st;
}

}  // namespace pac

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
using namespace pac;

static int ilog2_exact(long long v, int b2) {
  if (v < 1) return -1;
  int lg = 0;
  while ((1LL << lg) < v) ++lg;
  if ((1LL << lg) != v) return -1;
  if (lg % b2) return -1;
  return lg;
}

namespace pac {
// pac_tune.cpp: the knobs PAC_TUNE_CACHE holds for this device and problem
bool tune_from_env_cache(int rank, const int* dims, const int* bases, int batch, int form,
                         pac_tune_t* tune);
}  // namespace pac

extern "C" {

static int create_plan(pac_plan_t* plan, int rank, const int* dims, const int* digit_bases,
                       int batch, int form, const pac_tune_t* tune) {
  if (!plan || !dims || !digit_bases || rank < 1 || rank > 3 || batch < 1)
    return set_error(PAC_ERROR_INVALID_VALUE, "pac_plan_create: invalid rank/dims/batch");
  const pac_tune_t knobs = tune ? *tune : pac_tune_t{0, 0, 0, 0, 0};
  if (knobs.max_factor_log < 0 || knobs.max_factor_log > 13 || knobs.max_radix_log < 0 ||
      knobs.max_radix_log > 4 || knobs.special < -1 || knobs.w_shift < -6 || knobs.w_shift > 6 ||
      knobs.plane < -1 || knobs.plane > 1)
    return set_error(PAC_ERROR_INVALID_VALUE,
                     "pac_plan_create: knobs out of range (factor log %d, radix log %d, "
                     "special %d, w shift %d)",
                     knobs.max_factor_log, knobs.max_radix_log, knobs.special, knobs.w_shift);
  int b2s[3] = {1, 1, 1};
  for (int a = 0; a < rank; ++a) {
    const int base = digit_bases[a] == 0 ? 2 : digit_bases[a];
    b2s[a] = base == 2 ? 1 : base == 4 ? 2 : base == 8 ? 3 : 0;
    if (!b2s[a])
      return set_error(PAC_ERROR_UNSUPPORTED_RADIX,
                       "pac_plan_create: digit base %d (axis %d) not in {2,4,8}", base, a);
  }
  if (form != PAC_FORM_F64 && form != PAC_FORM_F32 && form != PAC_FORM_TC)
    return set_error(PAC_ERROR_INVALID_VALUE, "pac_plan_create: unknown form %d", form);
  int st = be_init();
  if (st != PAC_SUCCESS) return st;
  std::unique_ptr<pac_plan_s> p(new pac_plan_s());
  p->rank = rank;
  p->batch = batch;
  p->b2 = b2s[0];
  p->form = form;
  long long N = 1;
  for (int a = 0; a < rank; ++a) {
    int lg = ilog2_exact(dims[a], b2s[a]);
    if (lg < 0)
      return set_error(PAC_ERROR_NOT_POWER, "pac_plan_create: axis %d length %d is not a power of %d",
                       a, dims[a], 1 << b2s[a]);
    p->dims[a] = dims[a];
    p->logs[a] = lg;
    p->b2s[a] = b2s[a];
    N *= dims[a];
  }
  if (N * (long long)batch > (1LL << 40) || N > (1LL << 31))
    return set_error(PAC_ERROR_SIZE, "pac_plan_create: problem too large");
  p->N = N;
  p->tune = knobs;
  p->main.flog_cap = knobs.max_factor_log;
  p->main.rlog_cap = knobs.max_radix_log > 0 ? knobs.max_radix_log : 4;
  p->main.special = knobs.special;
  p->main.w_shift = knobs.w_shift;
  p->main.plane = knobs.plane;
  int bytes = form == PAC_FORM_F64 ? 8 : 4;
  st = build_schedule(p->main, rank, p->logs, b2s, bytes);
  if (st != PAC_SUCCESS) return st;
  p->main.tc = form == PAC_FORM_TC;
  if (p->main.tc) {
    st = be_malloc(&p->main.tcc, sizeof(TcConst) * TC_CONST_SETS * 32);
    if (st == PAC_SUCCESS) st = be_fill_tc_const(p->main.tcc, nullptr);
    if (st != PAC_SUCCESS) return st;
  }
  if (bytes != 8) {
    p->s64.reset(new Schedule());
    st = build_schedule(*p->s64, rank, p->logs, b2s, 8);
    if (st != PAC_SUCCESS) return st;
  }
  st = be_malloc((void**)&p->status, sizeof(int));
  if (st == PAC_SUCCESS) st = be_memset(p->status, 0, sizeof(int), nullptr);
  if (st == PAC_SUCCESS) st = be_stream_sync(nullptr);
  if (st != PAC_SUCCESS) return st;
  *plan = p.release();
  return PAC_SUCCESS;
}

PAC_API int pac_plan_create_tuned(pac_plan_t* plan, int rank, const int* dims,
                                  const int* digit_bases, int batch, int form,
                                  const pac_tune_t* tune) {
  return create_plan(plan, rank, dims, digit_bases, batch, form, tune);
}

PAC_API int pac_plan_create_axes(pac_plan_t* plan, int rank, const int* dims,
                                 const int* digit_bases, int batch, int form) {
  pac_tune_t t;
  if (dims && digit_bases && rank >= 1 && rank <= 3 &&
      tune_from_env_cache(rank, dims, digit_bases, batch, form, &t))
    return create_plan(plan, rank, dims, digit_bases, batch, form, &t);
  return create_plan(plan, rank, dims, digit_bases, batch, form, nullptr);
}

PAC_API int pac_plan_create(pac_plan_t* plan, int rank, const int* dims, int batch,
                            int digit_base, int form) {
  const int bases[3] = {digit_base, digit_base, digit_base};
  return pac_plan_create_axes(plan, rank, dims, bases, batch, form);
}

PAC_API int pac_plan_destroy(pac_plan_t plan) {
  delete plan;
  return PAC_SUCCESS;
}

PAC_API int pac_plan_get_info(pac_plan_t plan, pac_plan_info_t* info) {
  if (!plan || !info) return set_error(PAC_ERROR_INVALID_VALUE, "pac_plan_get_info: NULL");
  memset(info, 0, sizeof(*info));
  info->n_elements = plan->N;
  info->batch = plan->batch;
  info->rank = plan->rank;
  for (int a = 0; a < 3; ++a) info->dims[a] = plan->dims[a];
  info->digit_base = 1 << plan->b2;
  for (int a = 0; a < 3; ++a) info->digit_bases[a] = a < plan->rank ? 1 << plan->b2s[a] : 0;
  info->form = plan->form;
  info->element_bytes = plan->main.bytes;
  int m = (int)plan->main.vax.size();
  info->conv_passes = m == 0 ? 1 : plane_active(plan->main) ? 3 : 2 * m - 1;
  info->transform_passes = m == 0 ? 1 : m;
  info->workspace_bytes = plan->ws_bytes + plan->tmp64_bytes;
  info->tune = plan->tune;
  return PAC_SUCCESS;
}

PAC_API int pac_filter_spectrum(pac_plan_t plan, const double* h_re, const double* h_im,
                                int nfilters, void* hhat_re, void* hhat_im, double scale,
                                pac_stream_t stream) {
  if (!plan || !h_re || !h_im || !hhat_re || !hhat_im)
    return set_error(PAC_ERROR_INVALID_VALUE, "pac_filter_spectrum: NULL argument");
  if (nfilters != 1 && nfilters != plan->batch)
    return set_error(PAC_ERROR_INVALID_VALUE, "pac_filter_spectrum: nfilters must be 1 or batch");
  if (plan->form == PAC_FORM_F64) {
    // A^T h in P order straight into hhat, then reordered in place
    PAC_TRY(run_transform(plan, plan->main, PAC_OP_AT, nfilters, h_re, h_im, hhat_re, hhat_im,
                          scale, 1, stream));
    return to_plan_order(plan, (const double*)hhat_re, (const double*)hhat_im, nfilters, hhat_re,
                         hhat_im, 1.0, stream);
  }
  // F32 form: FP64 transform into a temporary, reordered and rounded once
  std::lock_guard<std::mutex> g(plan->ws_mu);
  size_t need = (size_t)nfilters * plan->N * 2 * sizeof(double);
  if (plan->tmp64_bytes < need) {
    if (plan->tmp64) be_free(plan->tmp64);
    plan->tmp64 = nullptr;
    plan->tmp64_bytes = 0;
    PAC_TRY(be_malloc(&plan->tmp64, need));
    plan->tmp64_bytes = need;
  }
  double* tre = (double*)plan->tmp64;
  double* tim = tre + (size_t)nfilters * plan->N;
  // the FP64 schedule never needs the workspace for A^T
  PAC_TRY(run_transform(plan, *plan->s64, PAC_OP_AT, nfilters, h_re, h_im, tre, tim, scale, 1,
                        stream));
  return to_plan_order(plan, tre, tim, nfilters, hhat_re, hhat_im, 1.0, stream);
}

PAC_API int pac_spectrum_to_plan_order(pac_plan_t plan, const double* p_re, const double* p_im,
                                       int nfilters, void* hhat_re, void* hhat_im, double scale,
                                       pac_stream_t stream) {
  if (!plan || !p_re || !p_im || !hhat_re || !hhat_im)
    return set_error(PAC_ERROR_INVALID_VALUE, "pac_spectrum_to_plan_order: NULL argument");
  if (nfilters != 1 && nfilters != plan->batch)
    return set_error(PAC_ERROR_INVALID_VALUE,
                     "pac_spectrum_to_plan_order: nfilters must be 1 or batch");
  if (plan->form != PAC_FORM_F64 && (p_re == hhat_re || p_im == hhat_im))
    return set_error(PAC_ERROR_INVALID_VALUE,
                     "pac_spectrum_to_plan_order: in place only for PAC_FORM_F64");
  return to_plan_order(plan, p_re, p_im, nfilters, hhat_re, hhat_im, scale, stream);
}

PAC_API int pac_convolve(pac_plan_t plan, const void* x_re, const void* x_im, const void* hhat_re,
                         const void* hhat_im, int hhat_per_problem, void* y_re, void* y_im,
                         double scale, pac_stream_t stream) {
  if (!plan || !x_re || !x_im || !hhat_re || !hhat_im || !y_re || !y_im)
    return set_error(PAC_ERROR_INVALID_VALUE, "pac_convolve: NULL argument");
  return run_conv(plan, x_re, x_im, hhat_re, hhat_im, hhat_per_problem ? 1 : 0, y_re, y_im, scale,
                  stream);
}

PAC_API int pac_transform(pac_plan_t plan, int op, const void* in_re, const void* in_im,
                          void* out_re, void* out_im, pac_stream_t stream) {
  if (!plan || !in_re || !in_im || !out_re || !out_im)
    return set_error(PAC_ERROR_INVALID_VALUE, "pac_transform: NULL argument");
  if (op < PAC_OP_AT || op > PAC_OP_UIFFT)
    return set_error(PAC_ERROR_INVALID_VALUE, "pac_transform: unknown op %d", op);
  bool scaled = op == PAC_OP_IFFT || op == PAC_OP_UIFFT;
  return run_transform(plan, plan->main, op, plan->batch, in_re, in_im, out_re, out_im,
                       scaled ? 1.0 / (double)plan->N : 1.0, scaled ? 1 : 0, stream);
}

PAC_API int pac_pointwise_product(long long n, const double* x_re, const double* x_im,
                                  const double* h_re, const double* h_im, double* y_re,
                                  double* y_im, double scale, pac_stream_t stream) {
  if (n < 0 || (n > 0 && (!x_re || !x_im || !h_re || !h_im || !y_re || !y_im)))
    return set_error(PAC_ERROR_INVALID_VALUE, "pac_pointwise_product: bad argument");
  if (n == 0) return PAC_SUCCESS;
  PAC_TRY(be_init());
  return be_pointwise(n, 8, x_re, x_im, h_re, h_im, -1LL, y_re, y_im, scale, stream);
}

PAC_API int pac_scale(long long n, const double* x_re, const double* x_im, double* y_re,
                      double* y_im, double scale, pac_stream_t stream) {
  if (n < 0 || (n > 0 && (!x_re || !x_im || !y_re || !y_im)))
    return set_error(PAC_ERROR_INVALID_VALUE, "pac_scale: bad argument");
  if (n == 0) return PAC_SUCCESS;
  PAC_TRY(be_init());
  return be_scale_copy(n, 8, x_re, x_im, y_re, y_im, scale, stream);
}

PAC_API int pac_permute(long long n, const int* rho, double* re, double* im, pac_stream_t stream) {
  if (n < 0 || (n > 0 && (!rho || !re)))
    return set_error(PAC_ERROR_INVALID_VALUE, "pac_permute: bad argument");
  if (n == 0) return PAC_SUCCESS;
  PAC_TRY(be_init());
  return be_permute(n, rho, re, im, stream);
}

PAC_API int pac_reference_twiddles(int r, int n, double* re, double* im, pac_stream_t stream) {
  if ((r != 2 && r != 4 && r != 8) || n < 1 || !re || !im)
    return set_error(PAC_ERROR_INVALID_VALUE, "pac_reference_twiddles: bad argument");
  PAC_TRY(be_init());
  // the reference's level count (twiddle_factors.c:18, :40-45, :77-82)
  int t = 0;
  if (r == 2) {
    while (!((n >> t) & 1)) ++t;
  } else {
    int sh = r == 4 ? 2 : 3;
    for (int v = n; v > 1; v >>= sh) ++t;
  }
  if (t == 0) return PAC_SUCCESS;
  return be_fill_ref_tw(r, t, re, im, stream);
}

PAC_API int pac_malloc(void** ptr, size_t bytes) {
  if (!ptr) return set_error(PAC_ERROR_INVALID_VALUE, "pac_malloc: NULL");
  PAC_TRY(be_init());
  return be_malloc(ptr, bytes);
}
PAC_API int pac_free(void* ptr) { return ptr ? be_free(ptr) : PAC_SUCCESS; }
PAC_API int pac_memcpy_h2d(void* dst, const void* src, size_t bytes, pac_stream_t s) {
  return be_memcpy(dst, src, bytes, CPY_H2D, s);
}
PAC_API int pac_memcpy_d2h(void* dst, const void* src, size_t bytes, pac_stream_t s) {
  return be_memcpy(dst, src, bytes, CPY_D2H, s);
}
PAC_API int pac_memcpy_d2d(void* dst, const void* src, size_t bytes, pac_stream_t s) {
  return be_memcpy(dst, src, bytes, CPY_D2D, s);
}
PAC_API int pac_stream_create(pac_stream_t* s) {
  if (!s) return set_error(PAC_ERROR_INVALID_VALUE, "pac_stream_create: NULL");
  PAC_TRY(be_init());
  return be_stream_create(s);
}
PAC_API int pac_stream_destroy(pac_stream_t s) { return be_stream_destroy(s); }
PAC_API int pac_stream_synchronize(pac_stream_t s) { return be_stream_sync(s); }
PAC_API int pac_stream_set_l2_persisting(pac_stream_t stream, const void* base, size_t bytes) {
  if (bytes > 0 && !base)
    return set_error(PAC_ERROR_INVALID_VALUE, "pac_stream_set_l2_persisting: NULL base");
  PAC_TRY(be_init());
  return be_l2_persist(stream, base, bytes);
}
PAC_API int pac_stream_wait_stream(pac_stream_t waiter, pac_stream_t waitee) {
  return be_stream_wait(waiter, waitee);
}
PAC_API long long pac_launch_count(void) { return be_launch_count(); }
PAC_API int pac_fma_peak(int elem_bytes, pac_stream_t stream, double* tflops) {
  if (!tflops || (elem_bytes != 8 && elem_bytes != 4))
    return set_error(PAC_ERROR_INVALID_VALUE, "pac_fma_peak: elem_bytes 8 or 4, tflops non-NULL");
  PAC_TRY(be_init());
  return be_fma_peak(elem_bytes, stream, tflops);
}

PAC_API int pac_plan_set_pass_timing(pac_plan_t plan, int enable) {
  if (!plan) return set_error(PAC_ERROR_INVALID_VALUE, "pac_plan_set_pass_timing: NULL");
  std::lock_guard<std::mutex> g(plan->t_mu);
  plan->timing = enable ? 1 : 0;
  plan->t_ms.clear();
  plan->t_calls = 0;
  return PAC_SUCCESS;
}

PAC_API int pac_plan_get_pass_timing(pac_plan_t plan, int max_passes, double* ms, long long* calls,
                                     int* npasses) {
  if (!plan || !npasses) return set_error(PAC_ERROR_INVALID_VALUE, "pac_plan_get_pass_timing: NULL");
  std::lock_guard<std::mutex> g(plan->t_mu);
  *npasses = (int)plan->t_ms.size();
  for (int i = 0; i < *npasses && i < max_passes; ++i) {
    if (ms) ms[i] = plan->t_ms[i];
  }
  if (calls) *calls = plan->t_calls;
  std::fill(plan->t_ms.begin(), plan->t_ms.end(), 0.0);
  plan->t_calls = 0;
  return PAC_SUCCESS;
}

PAC_API int pac_plan_set_wait_limit(pac_plan_t plan, long long cycles) {
  if (!plan) return set_error(PAC_ERROR_INVALID_VALUE, "pac_plan_set_wait_limit: NULL plan");
  plan->wait_limit = cycles > 0 ? cycles : 0;
  return PAC_SUCCESS;
}

PAC_API int pac_plan_check_status(pac_plan_t plan, pac_stream_t stream) {
  if (!plan) return set_error(PAC_ERROR_INVALID_VALUE, "pac_plan_check_status: NULL plan");
  int word = 0;
  PAC_TRY(be_stream_sync(stream));
  PAC_TRY(be_memcpy(&word, plan->status, sizeof(int), CPY_D2H, stream));
  PAC_TRY(be_stream_sync(stream));
  if (word == PAC_SUCCESS) return PAC_SUCCESS;
  PAC_TRY(be_memset(plan->status, 0, sizeof(int), stream));
  PAC_TRY(be_stream_sync(stream));
  return set_error(word, "a bounded device wait of this plan gave up (status %d); the output "
                         "of the call it belongs to is incomplete", word);
}

PAC_API const char* pac_status_string(int status) {
  switch (status) {
    case PAC_SUCCESS: return "success";
    case PAC_ERROR_INVALID_VALUE: return "invalid value";
    case PAC_ERROR_NOT_POWER: return "axis length is not a power of the radix";
    case PAC_ERROR_UNSUPPORTED_RADIX: return "unsupported radix";
    case PAC_ERROR_SIZE: return "problem too large";
    case PAC_ERROR_CUDA: return "CUDA error";
    case PAC_ERROR_NO_DEVICE: return "no usable sm_100 device";
    case PAC_ERROR_ALLOC: return "allocation failed";
    case PAC_ERROR_TIMEOUT: return "device wait timed out";
    default: return "internal error";
  }
}

PAC_API const char* pac_last_error(void) { return t_err; }

}  // extern "C"
