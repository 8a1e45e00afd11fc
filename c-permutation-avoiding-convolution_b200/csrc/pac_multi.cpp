// pac_multi.cpp -- many convolutions of uneven shapes per call (pac.h,
// pac_multi_*): one plan per distinct shape, every problem's passes grouped
// into levels (the k-th pass of every problem), each level run by
// persistent work-queue launches, the launches of a buffer set captured once
// into a CUDA graph.
//
// A work-queue launch reserves the largest shared-memory tile of its passes
// for every CTA, so a level is split by tile size into groups: passes with
// tiles up to kSmallSmem go to one launch (several CTAs per SM), larger ones
// to another, and the two run side by side on two streams (two branches of
// the graph).
#include <stdlib.h>
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

namespace pac {
int set_error(int status, const char* fmt, ...);
int plan_conv_descs(pac_plan_s* pl, const void* x_re, const void* x_im, const void* h_re,
                    const void* h_im, void* y_re, void* y_im, std::vector<PassDesc>& descs,
                    std::vector<long long>& ctas, std::vector<size_t>& smem);
int plan_bytes(pac_plan_s* pl);
}  // namespace pac

using namespace pac;

#define PAC_TRY(expr)                    \
  do {                                   \
    int _st = (expr);                    \
    if (_st != PAC_SUCCESS) return _st;  \
  } while (0)

namespace {

enum { kMaxLevels = 8, kGroups = 2 };
const size_t kSmallSmem = 72 * 1024;

// one work-queue launch: passes of one level and one tile-size class
struct Group {
  int ndesc = 0;
  long long total = 0;  // work items (CTAs)
  size_t smem = 0;
  size_t desc_off = 0;   // byte offsets into the device block
  size_t start_off = 0;
  size_t item_off = 0;
};

size_t round256(size_t v) { return (v + 255) / 256 * 256; }

}  // namespace

struct pac_multi_s {
  int nprob = 0;
  int bytes = 8;
  int b2 = 1;
  int tc = 0;  // tensor-core form
  std::vector<long long> off;       // nprob + 1
  std::vector<int> shape_of;        // problem -> plan index
  std::vector<pac_plan_t> plans;    // one per distinct shape
  std::vector<long long> nelem;     // per plan: elements of one problem
  // launch state of the last buffer set
  std::mutex mu;
  const void* key[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  bool built = false;
  std::vector<std::vector<Group>> levels;  // per level: its non-empty groups
  void* dev = nullptr;  // descriptors, starts, item tables and counters
  size_t dev_bytes = 0;
  size_t counter_off = 0;
  void* side = nullptr;  // second stream for the small-tile groups
  void* graph = nullptr;
  void* graph_stream = nullptr;
  // level timing (pac_multi_set_level_timing)
  int timing = 0;
  std::vector<void*> ev;
  double level_ms[kMaxLevels] = {};
  long long timed_calls = 0;
  long long fast_items = 0;  // work items of descriptors marked special
  ~pac_multi_s() {
    for (void* e : ev) be_event_destroy(e);
    if (graph) be_graph_destroy(graph);
    if (side) be_stream_destroy(side);
    if (dev) be_free(dev);
    for (pac_plan_t p : plans) pac_plan_destroy(p);
  }
};

// Gather every problem's pass list for the buffer set, group the passes by
// level and tile size, order each group's passes by tile size (largest
// first: the queue hands out the long CTAs early) and upload descriptors,
// item starts and the item -> pass tables.
static int build_levels(pac_multi_s* m, const void* x_re, const void* x_im, const void* h_re,
                        const void* h_im, void* y_re, void* y_im, void* stream) {
  struct Item {
    PassDesc d;
    long long ctas;
    size_t smem;
    long long work;  // elements per CTA
  };
  std::vector<std::vector<Item>> lv[kGroups];
  const size_t B = (size_t)m->bytes;
  size_t nlev = 0;
  for (int p = 0; p < m->nprob; ++p) {
    const size_t o = (size_t)m->off[p] * B;
    std::vector<PassDesc> descs;
    std::vector<long long> ctas;
    std::vector<size_t> smem;
    PAC_TRY(plan_conv_descs(m->plans[m->shape_of[p]], (const char*)x_re + o,
                            (const char*)x_im + o, (const char*)h_re + o, (const char*)h_im + o,
                            (char*)y_re + o, (char*)y_im + o, descs, ctas, smem));
    if (descs.size() > (size_t)kMaxLevels)
      return set_error(PAC_ERROR_SIZE, "problem %d needs %zu passes (at most %d)", p,
                       descs.size(), (int)kMaxLevels);
    nlev = std::max(nlev, descs.size());
    for (int g = 0; g < kGroups; ++g)
      if (lv[g].size() < nlev) lv[g].resize(nlev);
    for (size_t k = 0; k < descs.size(); ++k) {
      const int g = smem[k] <= kSmallSmem ? 1 : 0;
      lv[g][k].push_back({descs[k], ctas[k], smem[k], (long long)descs[k].W << descs[k].logL});
    }
  }
  m->levels.assign(nlev, {});
  long long fast = 0;
  size_t bytes = 0;
  for (size_t k = 0; k < nlev; ++k)
    for (int g = 0; g < kGroups; ++g) {
      auto& items = lv[g][k];
      if (items.empty()) continue;
      std::stable_sort(items.begin(), items.end(),
                       [](const Item& a, const Item& b) { return a.work > b.work; });
      Group G;
      G.ndesc = (int)items.size();
      for (auto& it : items) {
        G.total += it.ctas;
        G.smem = std::max(G.smem, it.smem);
        if (it.d.spec) fast += it.ctas;
      }
      G.desc_off = bytes;
      bytes += round256(sizeof(PassDesc) * G.ndesc);
      G.start_off = bytes;
      bytes += round256(sizeof(long long) * (G.ndesc + 1));
      G.item_off = bytes;
      bytes += round256(sizeof(int) * (size_t)G.total);
      m->levels[k].push_back(G);
    }
  m->fast_items = fast;
  m->counter_off = bytes;
  bytes += round256(sizeof(unsigned long long) * kMaxLevels * kGroups);
  std::vector<unsigned char> host(bytes, 0);
  for (size_t k = 0; k < nlev; ++k) {
    size_t gi = 0;
    for (int g = 0; g < kGroups; ++g) {
      const auto& items = lv[g][k];
      if (items.empty()) continue;
      const Group& G = m->levels[k][gi++];
      PassDesc* d = (PassDesc*)(host.data() + G.desc_off);
      long long* st = (long long*)(host.data() + G.start_off);
      int* tab = (int*)(host.data() + G.item_off);
      long long acc = 0;
      for (int i = 0; i < G.ndesc; ++i) {
        d[i] = items[i].d;
        st[i] = acc;
        for (long long c = 0; c < items[i].ctas; ++c) tab[acc + c] = i;
        acc += items[i].ctas;
      }
      st[G.ndesc] = acc;
    }
  }
  if (m->dev_bytes < bytes) {
    if (m->dev) PAC_TRY(be_free(m->dev));
    m->dev = nullptr;
    m->dev_bytes = 0;
    PAC_TRY(be_malloc(&m->dev, bytes));
    m->dev_bytes = bytes;
  }
  PAC_TRY(be_memcpy(m->dev, host.data(), bytes, CPY_H2D, stream));
  // the host staging vector dies here: wait for the copy
  PAC_TRY(be_stream_sync(stream));
  for (auto& groups : m->levels)
    for (auto& G : groups) PAC_TRY(be_queue_prepare(m->bytes, m->b2, m->tc, G.smem));
  if (!m->side) PAC_TRY(be_stream_create(&m->side));
  return PAC_SUCCESS;
}

static int launch_group(pac_multi_s* m, const Group& G, unsigned long long* cnt, void* stream) {
  char* dev = (char*)m->dev;
  return be_launch_queue((const PassDesc*)(dev + G.desc_off),
                         (const long long*)(dev + G.start_off), (const int*)(dev + G.item_off),
                         G.ndesc, G.total, cnt, m->bytes, m->b2, m->tc, G.smem, stream);
}

// counters to zero, then every level: its groups side by side (the second
// group on the side stream, forked from and joined back into `stream`);
// with `ev`, event k is recorded on `stream` before level k and the last
// one after the last level
static int issue_levels(pac_multi_s* m, void* stream, void** ev = nullptr) {
  unsigned long long* cnt = (unsigned long long*)((char*)m->dev + m->counter_off);
  PAC_TRY(be_memset(cnt, 0, sizeof(unsigned long long) * kMaxLevels * kGroups, stream));
  for (size_t k = 0; k < m->levels.size(); ++k) {
    const auto& groups = m->levels[k];
    unsigned long long* c = cnt + k * kGroups;
    if (ev) PAC_TRY(be_event_record(ev[k], stream));
    // one NVTX range per level, named as bench.py's per-level breakdown
    char name[48];
    snprintf(name, sizeof(name), "pac multi level %d", (int)k);
    nvtxRangePushA(name);
    int st = PAC_SUCCESS;
    if (groups.size() == 1) {
      st = launch_group(m, groups[0], c, stream);
    } else {
      st = be_stream_wait(m->side, stream);
      if (st == PAC_SUCCESS) st = launch_group(m, groups[0], c, stream);
      if (st == PAC_SUCCESS) st = launch_group(m, groups[1], c + 1, m->side);
      if (st == PAC_SUCCESS) st = be_stream_wait(stream, m->side);
    }
    nvtxRangePop();
    PAC_TRY(st);
  }
  if (ev) PAC_TRY(be_event_record(ev[m->levels.size()], stream));
  return PAC_SUCCESS;
}

// a timed call: levels issued directly with events around them
static int issue_timed(pac_multi_s* m, void* stream) {
  const size_t n = m->levels.size();
  while (m->ev.size() < n + 1) {
    void* e = nullptr;
    PAC_TRY(be_event_create(&e));
    m->ev.push_back(e);
  }
  PAC_TRY(issue_levels(m, stream, m->ev.data()));
  for (size_t k = 0; k < n; ++k) {
    float ms = 0.f;
    PAC_TRY(be_event_elapsed(m->ev[k], m->ev[k + 1], &ms));
    m->level_ms[k] += ms;
  }
  m->timed_calls++;
  return PAC_SUCCESS;
}

static int ilog_exact(int v, int b2) {
  if (v < 1 || (v & (v - 1))) return -1;
  int lg = 0;
  while ((1 << lg) < v) ++lg;
  return lg % b2 ? -1 : lg;
}

// tune NULL: every shape's plan as pac_plan_create makes it (with the
// knobs PAC_TUNE_CACHE holds for it, if any); else these knobs for all
static int create_multi(pac_multi_t* multi, int nprob, const int* ranks, const int* dims,
                        int digit_base, int form, const pac_tune_t* tune) {
  if (!multi || nprob < 1 || !ranks || !dims)
    return set_error(PAC_ERROR_INVALID_VALUE, "pac_multi_create: invalid arguments");
  if (digit_base == 0) digit_base = 2;
  const int b2 = digit_base == 2 ? 1 : digit_base == 4 ? 2 : digit_base == 8 ? 3 : 0;
  if (!b2)
    return set_error(PAC_ERROR_UNSUPPORTED_RADIX, "pac_multi_create: digit base %d not in {2,4,8}",
                     digit_base);
  std::unique_ptr<pac_multi_s> m(new pac_multi_s());
  m->nprob = nprob;
  m->b2 = b2;
  m->tc = form == PAC_FORM_TC;
  m->off.assign(nprob + 1, 0);
  m->shape_of.assign(nprob, 0);
  std::map<std::vector<int>, int> seen;
  for (int p = 0; p < nprob; ++p) {
    const int r = ranks[p];
    if (r < 1 || r > 3) return set_error(PAC_ERROR_INVALID_VALUE, "problem %d: rank %d", p, r);
    std::vector<int> key(dims + 3 * p, dims + 3 * p + r);
    long long n = 1;
    for (int a = 0; a < r; ++a) {
      if (ilog_exact(key[a], b2) < 0)
        return set_error(PAC_ERROR_NOT_POWER, "problem %d: axis %d length %d is not a power of %d",
                         p, a, key[a], digit_base);
      n *= key[a];
    }
    if (n < 2) return set_error(PAC_ERROR_SIZE, "problem %d has a single element", p);
    auto it = seen.find(key);
    if (it == seen.end()) {
      pac_plan_t pl = nullptr;
      const int bases[3] = {digit_base, digit_base, digit_base};
      int st = tune ? pac_plan_create_tuned(&pl, r, key.data(), bases, 1, form, tune)
                    : pac_plan_create(&pl, r, key.data(), 1, digit_base, form);
      if (st != PAC_SUCCESS) return st;
      it = seen.emplace(key, (int)m->plans.size()).first;
      m->plans.push_back(pl);
      m->nelem.push_back(n);
    }
    m->shape_of[p] = it->second;
    m->off[p + 1] = m->off[p] + n;
  }
  m->bytes = plan_bytes(m->plans[0]);
  *multi = m.release();
  return PAC_SUCCESS;
}

namespace pac {
std::string plan_signature(pac_plan_s* pl);
// every shape's plan schedule (pac_tune.cpp)
std::string multi_signature(pac_multi_s* m) {
  std::string sig;
  for (auto* pl : m->plans) sig += plan_signature(pl) + "|";
  return sig;
}
}  // namespace pac

extern "C" {

PAC_API int pac_multi_create(pac_multi_t* multi, int nprob, const int* ranks, const int* dims,
                             int digit_base, int form) {
  return create_multi(multi, nprob, ranks, dims, digit_base, form, nullptr);
}

PAC_API int pac_multi_create_tuned(pac_multi_t* multi, int nprob, const int* ranks,
                                   const int* dims, int digit_base, int form,
                                   const pac_tune_t* tune) {
  static const pac_tune_t built_in = {0, 0, 0, 0};
  return create_multi(multi, nprob, ranks, dims, digit_base, form, tune ? tune : &built_in);
}

PAC_API int pac_multi_destroy(pac_multi_t multi) {
  delete multi;
  return PAC_SUCCESS;
}

PAC_API int pac_multi_offsets(pac_multi_t m, long long* offsets) {
  if (!m || !offsets) return set_error(PAC_ERROR_INVALID_VALUE, "pac_multi_offsets: NULL");
  memcpy(offsets, m->off.data(), sizeof(long long) * m->off.size());
  return PAC_SUCCESS;
}

PAC_API int pac_multi_filter_spectra(pac_multi_t m, const double* h_re, const double* h_im,
                                     void* hhat_re, void* hhat_im, pac_stream_t stream) {
  if (!m || !h_re || !h_im || !hhat_re || !hhat_im)
    return set_error(PAC_ERROR_INVALID_VALUE, "pac_multi_filter_spectra: NULL");
  const size_t B = (size_t)m->bytes;
  for (int p = 0; p < m->nprob; ++p) {
    const long long o = m->off[p];
    const int s = m->shape_of[p];
    PAC_TRY(pac_filter_spectrum(m->plans[s], h_re + o, h_im + o, 1, (char*)hhat_re + o * B,
                                (char*)hhat_im + o * B, 1.0 / (double)m->nelem[s], stream));
  }
  return PAC_SUCCESS;
}

PAC_API int pac_multi_convolve(pac_multi_t m, const void* x_re, const void* x_im,
                               const void* hhat_re, const void* hhat_im, void* y_re, void* y_im,
                               pac_stream_t stream) {
  if (!m || !x_re || !x_im || !hhat_re || !hhat_im || !y_re || !y_im)
    return set_error(PAC_ERROR_INVALID_VALUE, "pac_multi_convolve: NULL");
  std::lock_guard<std::mutex> g(m->mu);
  const void* key[6] = {x_re, x_im, hhat_re, hhat_im, y_re, y_im};
  if (!m->built || memcmp(key, m->key, sizeof(key)) != 0) {
    if (m->graph) {
      be_graph_destroy(m->graph);
      m->graph = nullptr;
    }
    m->built = false;
    PAC_TRY(build_levels(m, x_re, x_im, hhat_re, hhat_im, y_re, y_im, stream));
    memcpy(m->key, key, sizeof(key));
    m->built = true;
  }
  if (m->timing) return issue_timed(m, stream);
  if (stream == nullptr || !be_graph_supported()) return issue_levels(m, stream);
  if (m->graph && m->graph_stream != stream) {
    be_graph_destroy(m->graph);
    m->graph = nullptr;
  }
  if (!m->graph) {
    PAC_TRY(be_graph_begin(stream));
    int st = issue_levels(m, stream);
    void* exec = nullptr;
    int st2 = be_graph_end(stream, &exec);
    if (st != PAC_SUCCESS) {
      if (exec) be_graph_destroy(exec);
      return st;
    }
    PAC_TRY(st2);
    m->graph = exec;
    m->graph_stream = stream;
  }
  return be_graph_launch(m->graph, stream);
}

PAC_API int pac_multi_get_info(pac_multi_t m, pac_multi_info_t* info) {
  if (!m || !info) return set_error(PAC_ERROR_INVALID_VALUE, "pac_multi_get_info: NULL");
  memset(info, 0, sizeof(*info));
  info->nprob = m->nprob;
  info->nshapes = (int)m->plans.size();
  info->nlevels = (int)m->levels.size();
  for (size_t k = 0; k < m->levels.size() && k < kMaxLevels; ++k)
    for (auto& G : m->levels[k]) info->items[k] += G.total;
  info->elements = m->off[m->nprob];
  info->graph = m->graph ? 1 : 0;
  info->timed_calls = m->timed_calls;
  info->fast_items = m->fast_items;
  for (size_t k = 0; k < m->levels.size() && k < kMaxLevels; ++k)
    info->level_ms[k] = m->timed_calls ? m->level_ms[k] / (double)m->timed_calls : 0.0;
  return PAC_SUCCESS;
}

PAC_API int pac_multi_set_level_timing(pac_multi_t m, int enable) {
  if (!m) return set_error(PAC_ERROR_INVALID_VALUE, "pac_multi_set_level_timing: NULL");
  std::lock_guard<std::mutex> g(m->mu);
  m->timing = enable ? 1 : 0;
  if (enable) {
    for (auto& v : m->level_ms) v = 0.0;
    m->timed_calls = 0;
  }
  return PAC_SUCCESS;
}

}  // extern "C"
