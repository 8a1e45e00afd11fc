// pac_tune.cpp -- the autotuner of the plan knobs (pac_tune_t) and its cache.
//
// A problem's knobs are found by timing it: convolutions of device buffers
// the tuner allocates (contents irrelevant to the time: zeros), one plan per
// candidate knob set, each timed with device events as the best of three
// rounds of enough calls to fill ~10 ms.  The search is a coordinate
// descent from the built-in knobs over (radix 8 stages, the plane or line
// schedule of 3D problems, shorter factors, then -- once the factors that
// the kernels serve are fixed -- specialised kernels off or their second to
// fifth candidates, and narrower / wider generic tiles); a step is kept
// only if it is at least 2% faster, so timing noise does not move a plan
// off the built-in choices.  Candidates that build the same schedule as one
// already timed (a factor cap that splits no axis differently) are skipped.
//
// The cache is a text file of JSON objects, one per line, appended to; the
// last line for a key wins.  The key names the device and the problem
// (form, batch, dims, digit bases; for a multi-plan the problem count and a
// 64-bit FNV-1a hash of every problem's shape).
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#include "pac.h"
#include "pac_backend.h"

namespace pac {

int set_error(int status, const char* fmt, ...);
std::string plan_signature(pac_plan_t plan);
std::string multi_signature(pac_multi_t multi);

enum { TUNE_DUPLICATE = -1 };  // a candidate whose schedule was already timed

#define PAC_TUNE_TRY(expr)               \
  do {                                   \
    int _st = (expr);                    \
    if (_st != PAC_SUCCESS) return _st;  \
  } while (0)

static int device_prefix(std::string* out) {
  char dev[160];
  PAC_TUNE_TRY(be_init());
  PAC_TUNE_TRY(be_device_name(dev, (int)sizeof(dev)));
  for (char* c = dev; *c; ++c)
    if (*c == '"' || *c == '\\' || *c == '|') *c = '_';
  *out = dev;
  return PAC_SUCCESS;
}

static int plan_key(int rank, const int* dims, const int* bases, int batch, int form,
                    std::string* key) {
  PAC_TUNE_TRY(device_prefix(key));
  char buf[160];
  int n = snprintf(buf, sizeof(buf), "|form %d|batch %d|dims", form, batch);
  for (int a = 0; a < rank; ++a) n += snprintf(buf + n, sizeof(buf) - n, "%s%d", a ? "x" : " ", dims[a]);
  n += snprintf(buf + n, sizeof(buf) - n, "|bases");
  for (int a = 0; a < rank; ++a)
    n += snprintf(buf + n, sizeof(buf) - n, "%s%d", a ? "," : " ", bases[a] ? bases[a] : 2);
  *key += buf;
  return PAC_SUCCESS;
}

static int multi_key(int nprob, const int* ranks, const int* dims, int base, int form,
                     std::string* key) {
  PAC_TUNE_TRY(device_prefix(key));
  unsigned long long h = 1469598103934665603ULL;
  auto mix = [&](long long v) {
    for (int i = 0; i < 8; ++i) {
      h ^= (unsigned long long)((v >> (8 * i)) & 0xff);
      h *= 1099511628211ULL;
    }
  };
  for (int p = 0; p < nprob; ++p) {
    mix(ranks[p]);
    for (int a = 0; a < ranks[p]; ++a) mix(dims[3 * p + a]);
  }
  char buf[160];
  snprintf(buf, sizeof(buf), "|multi|form %d|base %d|problems %d|shapes fnv %016llx", form,
           base ? base : 2, nprob, h);
  *key += buf;
  return PAC_SUCCESS;
}

static bool json_int(const char* line, const char* name, long long* v) {
  char pat[64];
  snprintf(pat, sizeof(pat), "\"%s\": ", name);
  const char* p = strstr(line, pat);
  if (!p) return false;
  *v = strtoll(p + strlen(pat), nullptr, 10);
  return true;
}
static bool json_num(const char* line, const char* name, double* v) {
  char pat[64];
  snprintf(pat, sizeof(pat), "\"%s\": ", name);
  const char* p = strstr(line, pat);
  if (!p) return false;
  *v = strtod(p + strlen(pat), nullptr);
  return true;
}

// the last entry for `key` in the cache file
static bool cache_lookup(const char* path, const std::string& key, pac_tune_result_t* r) {
  FILE* f = path ? fopen(path, "r") : nullptr;
  if (!f) return false;
  const std::string want = "{\"key\": \"" + key + "\",";
  bool found = false;
  std::vector<char> line(4096);
  while (fgets(line.data(), (int)line.size(), f)) {
    if (strncmp(line.data(), want.c_str(), want.size()) != 0) continue;
    long long a, b, c, d, e = 0;
    double ms = 0, dms = 0;
    if (!json_int(line.data(), "max_factor_log", &a) || !json_int(line.data(), "max_radix_log", &b) ||
        !json_int(line.data(), "special", &c) || !json_int(line.data(), "w_shift", &d))
      continue;
    json_int(line.data(), "plane", &e);  // absent in lines of older caches: 0
    json_num(line.data(), "ms", &ms);
    json_num(line.data(), "default_ms", &dms);
    memset(r, 0, sizeof(*r));
    r->tune = pac_tune_t{(int)a, (int)b, (int)c, (int)d, (int)e};
    r->ms = ms;
    r->default_ms = dms;
    r->cached = 1;
    found = true;
  }
  fclose(f);
  return found;
}

static int cache_append(const char* path, const std::string& key, const pac_tune_result_t& r) {
  if (!path) return PAC_SUCCESS;
  FILE* f = fopen(path, "a");
  if (!f) return set_error(PAC_ERROR_INVALID_VALUE, "pac_autotune: cannot write %s", path);
  fprintf(f,
          "{\"key\": \"%s\", \"max_factor_log\": %d, \"max_radix_log\": %d, \"special\": %d, "
          "\"w_shift\": %d, \"plane\": %d, \"ms\": %.6g, \"default_ms\": %.6g, "
          "\"candidates\": %d}\n",
          key.c_str(), r.tune.max_factor_log, r.tune.max_radix_log, r.tune.special,
          r.tune.w_shift, r.tune.plane, r.ms, r.default_ms, r.candidates);
  fclose(f);
  return PAC_SUCCESS;
}

bool tune_from_env_cache(int rank, const int* dims, const int* bases, int batch, int form,
                         pac_tune_t* tune) {
  const char* path = getenv("PAC_TUNE_CACHE");
  if (!path || !*path) return false;
  std::string key;
  if (plan_key(rank, dims, bases, batch, form, &key) != PAC_SUCCESS) return false;
  pac_tune_result_t r;
  if (!cache_lookup(path, key, &r)) return false;
  *tune = r.tune;
  return true;
}

// false if sig is in seen (a schedule already timed), else records it
static bool note_signature(const std::string& sig, std::vector<std::string>* seen) {
  for (auto& x : *seen)
    if (x == sig) return false;
  seen->push_back(sig);
  return true;
}

// device buffers of a timing run: x, hhat (re, im) of `bytes` each and y
// (re and im back to back).  The timing runs keep y -- the output and the
// passes' intermediate -- persisting in L2 when it fits in three quarters of
// L2, the policy of the timed runs of bench.py, so that schedules whose extra
// passes would run out of L2 there are timed that way here too.
struct TuneBufs {
  void* p[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  void* window = nullptr;
  void* stream = nullptr;
  ~TuneBufs() {
    if (window) be_l2_persist(stream, nullptr, 0);
    for (int i = 0; i < 5; ++i)
      if (p[i]) be_free(p[i]);
  }
  int alloc(size_t bytes, void* s) {
    stream = s;
    for (int i = 0; i < 5; ++i) {
      const size_t n = i == 4 ? 2 * bytes : bytes;
      PAC_TUNE_TRY(be_malloc(&p[i], n));
      PAC_TUNE_TRY(be_memset(p[i], 0, n, stream));
    }
    p[5] = (char*)p[4] + bytes;
    const long long l2 = be_l2_bytes();
    if (l2 > 0 && 2.0 * (double)bytes <= 0.75 * (double)l2) {
      PAC_TUNE_TRY(be_l2_persist(stream, p[4], 2 * bytes));
      window = p[4];
    }
    return PAC_SUCCESS;
  }
};

// milliseconds per call of `run`: best of three rounds of enough calls to
// fill ~10 ms (so microsecond-scale problems average over many launches),
// after two warm-up calls
template <class F>
static int time_calls(F run, void* stream, double* ms) {
  void* e0 = nullptr;
  void* e1 = nullptr;
  int st = be_event_create(&e0);
  if (st == PAC_SUCCESS) st = be_event_create(&e1);
  float t = 0.f;
  for (int i = 0; i < 2 && st == PAC_SUCCESS; ++i) st = run();
  if (st == PAC_SUCCESS) st = be_event_record(e0, stream);
  if (st == PAC_SUCCESS) st = run();
  if (st == PAC_SUCCESS) st = be_event_record(e1, stream);
  if (st == PAC_SUCCESS) st = be_event_elapsed(e0, e1, &t);
  int reps = (int)ceil(10.0 / (t > 1e-3f ? t : 1e-3f));
  reps = reps < 3 ? 3 : reps > 2000 ? 2000 : reps;
  double best = 1e30;
  for (int round = 0; round < 3 && st == PAC_SUCCESS; ++round) {
    st = be_event_record(e0, stream);
    for (int i = 0; i < reps && st == PAC_SUCCESS; ++i) st = run();
    if (st == PAC_SUCCESS) st = be_event_record(e1, stream);
    if (st == PAC_SUCCESS) st = be_event_elapsed(e0, e1, &t);
    if (st == PAC_SUCCESS && t / reps < best) best = t / reps;
  }
  if (e0) be_event_destroy(e0);
  if (e1) be_event_destroy(e1);
  *ms = best;
  return st;
}

// coordinate descent.  measure(t, seen, &ms) builds the plan of knob set
// t; if `seen` is given and the plan's schedule signature is in it, it
// returns TUNE_DUPLICATE without timing, else it adds the signature and
// times the plan.  Any other error (a knob set that builds no plan) skips
// the candidate.
template <class M>
static void descend(M measure, bool search_special, int bytes, pac_tune_result_t* r) {
  pac_tune_t cur = {0, 0, 0, 0, 0};
  double cur_ms = 0;
  std::vector<std::string> seen;
  r->candidates = 0;
  if (measure(cur, &seen, &cur_ms) != PAC_SUCCESS) return;
  r->candidates = 1;
  r->default_ms = cur_ms;
  auto consider = [&](pac_tune_t t, bool dedupe) {
    double ms = 0;
    if (measure(t, dedupe ? &seen : nullptr, &ms) != PAC_SUCCESS) return false;
    r->candidates++;
    if (ms < 0.98 * cur_ms) {
      cur = t;
      cur_ms = ms;
      return true;
    }
    return false;
  };
  {
    pac_tune_t t = cur;
    t.max_radix_log = 3;
    consider(t, false);
  }
  {
    // 3D: the other of the plane and line schedules (a knob set that builds
    // the same schedule as the current one is not timed twice)
    pac_tune_t t = cur;
    t.plane = 1;
    consider(t, true);
    t.plane = -1;
    consider(t, true);
  }
  {
    const int lmax = bytes == 8 ? 12 : 13;
    const pac_tune_t base = cur;
    for (int c = lmax - 1; c >= lmax - 3; --c) {
      pac_tune_t t = base;
      t.max_factor_log = c;
      consider(t, true);
    }
  }
  // the kernel candidates after the factor split, whose geometries they serve
  if (search_special) {
    const pac_tune_t base = cur;
    for (int sp : {-1, 1, 2, 3, 4}) {  // generic kernels only; the k-th specialised candidates
      pac_tune_t t = base;
      t.special = sp;
      consider(t, false);
    }
  }
  {
    const pac_tune_t base = cur;
    for (int w : {-1, 1}) {
      pac_tune_t t = base;
      t.w_shift = w;
      consider(t, false);
    }
  }
  r->tune = cur;
  r->ms = cur_ms;
}

}  // namespace pac

using namespace pac;

extern "C" {

PAC_API int pac_autotune(int rank, const int* dims, const int* digit_bases, int batch, int form,
                         pac_stream_t stream, const char* cache_path, pac_tune_result_t* result) {
  if (!dims || !digit_bases || !result || rank < 1 || rank > 3 || batch < 1)
    return set_error(PAC_ERROR_INVALID_VALUE, "pac_autotune: invalid arguments");
  std::string key;
  PAC_TUNE_TRY(plan_key(rank, dims, digit_bases, batch, form, &key));
  memset(result, 0, sizeof(*result));
  if (cache_lookup(cache_path, key, result)) return PAC_SUCCESS;
  // the problem must build with the built-in knobs
  pac_plan_t probe = nullptr;
  PAC_TUNE_TRY(pac_plan_create_tuned(&probe, rank, dims, digit_bases, batch, form, nullptr));
  pac_plan_info_t info;
  pac_plan_get_info(probe, &info);
  pac_plan_destroy(probe);
  const size_t bytes = (size_t)info.element_bytes * (size_t)(info.n_elements * batch);
  TuneBufs b;
  PAC_TUNE_TRY(b.alloc(bytes, stream));
  auto measure = [&](const pac_tune_t& t, std::vector<std::string>* seen, double* ms) {
    pac_plan_t pl = nullptr;
    int st = pac_plan_create_tuned(&pl, rank, dims, digit_bases, batch, form, &t);
    if (st != PAC_SUCCESS) return st;
    if (seen && !note_signature(plan_signature(pl), seen)) {
      pac_plan_destroy(pl);
      return (int)TUNE_DUPLICATE;
    }
    st = time_calls(
        [&] {
          return pac_convolve(pl, b.p[0], b.p[1], b.p[2], b.p[3], 0, b.p[4], b.p[5], 1.0, stream);
        },
        stream, ms);
    pac_plan_destroy(pl);
    return st;
  };
  descend(measure, true, info.element_bytes, result);
  if (result->candidates == 0)
    return set_error(PAC_ERROR_INTERNAL, "pac_autotune: the built-in knobs could not be timed");
  PAC_TUNE_TRY(be_stream_sync(stream));
  return cache_append(cache_path, key, *result);
}

PAC_API int pac_multi_autotune(int nprob, const int* ranks, const int* dims, int digit_base,
                               int form, pac_stream_t stream, const char* cache_path,
                               pac_tune_result_t* result) {
  if (nprob < 1 || !ranks || !dims || !result)
    return set_error(PAC_ERROR_INVALID_VALUE, "pac_multi_autotune: invalid arguments");
  std::string key;
  PAC_TUNE_TRY(multi_key(nprob, ranks, dims, digit_base, form, &key));
  memset(result, 0, sizeof(*result));
  if (cache_lookup(cache_path, key, result)) return PAC_SUCCESS;
  pac_multi_t probe = nullptr;
  PAC_TUNE_TRY(pac_multi_create_tuned(&probe, nprob, ranks, dims, digit_base, form, nullptr));
  std::vector<long long> off(nprob + 1);
  pac_multi_offsets(probe, off.data());
  pac_multi_destroy(probe);
  const int esz = form == PAC_FORM_F64 ? 8 : 4;
  TuneBufs b;
  PAC_TUNE_TRY(b.alloc((size_t)esz * (size_t)off[nprob], stream));
  auto measure = [&](const pac_tune_t& t, std::vector<std::string>* seen, double* ms) {
    pac_multi_t m = nullptr;
    int st = pac_multi_create_tuned(&m, nprob, ranks, dims, digit_base, form, &t);
    if (st != PAC_SUCCESS) return st;
    if (seen && !note_signature(multi_signature(m), seen)) {
      pac_multi_destroy(m);
      return (int)TUNE_DUPLICATE;
    }
    st = time_calls(
        [&] { return pac_multi_convolve(m, b.p[0], b.p[1], b.p[2], b.p[3], b.p[4], b.p[5], stream); },
        stream, ms);
    pac_multi_destroy(m);
    return st;
  };
  descend(measure, false, esz, result);
  if (result->candidates == 0)
    return set_error(PAC_ERROR_INTERNAL, "pac_multi_autotune: the built-in knobs could not be timed");
  PAC_TUNE_TRY(be_stream_sync(stream));
  return cache_append(cache_path, key, *result);
}

}  // extern "C"
