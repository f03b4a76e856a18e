// schedule.cu -- insert schedules, batch features and the schedule selector.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "mlp.h"
#include "schedule.h"

namespace gmpt {

namespace {

// name, PhaseNU, persistent, local build, local sort, LockNU ways, LockNU
// dedup, persistent grid, warp-per-branch hash levels
const Schedule kSchedules[] = {
    {"phasenu", true, false, 1, 1, 4, 1, 0, 4096},
    {"phasenu-global-build", true, false, 0, 1, 4, 1, 0, 4096},
    {"locknu-4", false, false, 1, 1, 4, 1, 0, 4096},
    {"locknu-2", false, false, 1, 1, 2, 1, 0, 4096},
    {"locknu-1", false, false, 1, 1, 1, 1, 0, 4096},
    // LockNU insert + PhaseHC + root read in one graph-replayed persistent
    // launch, with all co-resident CTAs or one CTA per SM
    {"persistent-2cta", false, true, 1, 1, 4, 1, 0, 4096},
    {"persistent-1cta", false, true, 1, 1, 4, 1, 148, 4096},
    {"locknu-4-nodedup", false, false, 1, 1, 4, 0, 0, 4096},
    {"phasenu-global-sort", true, false, 1, 0, 4, 1, 0, 4096},
    {"phasenu-warp-hash", true, false, 1, 1, 4, 1, 0, 65536},
};
constexpr int kNumSchedules = (int)(sizeof(kSchedules) / sizeof(kSchedules[0]));
static_assert(kNumSchedules <= kMlpMaxOut, "one network output per schedule");

constexpr int kPhaseNU = 0, kLockNU4 = 2, kPersistent1 = 6;

}  // namespace

int schedule_count() { return kNumSchedules; }

const Schedule *schedule_at(int k) { return (k >= 0 && k < kNumSchedules) ? &kSchedules[k] : nullptr; }

int apply_schedule(Trie &t, int k) {
  const Schedule *s = schedule_at(k);
  if (!s) return E_ARG;
  int rc = OK;
  if (!rc) rc = t.set_option("local_build", s->local_build);
  if (!rc) rc = t.set_option("local_sort", s->local_sort);
  if (!rc) rc = t.set_option("latch_ways", s->latch_ways);
  if (!rc) rc = t.set_option("latch_dedup", s->latch_dedup);
  if (!rc) rc = t.set_option("warp_full_max", s->warp_full_max);
  if (!rc && s->persistent) rc = t.set_option("block_grid", s->block_grid);
  return rc;
}

int put_schedule(Trie &t, int k, const BatchIn &b) {
  int rc = apply_schedule(t, k);
  if (rc) return rc;
  const Schedule *s = schedule_at(k);
  // the persistent launch takes hex keys whose index pairs tile the stream
  // and no caller host pointers; other batches run as LockNU with its knobs
  if (s->persistent && (b.raw_keys || b.values_hps)) return t.put_latching(b);
  if (!s->persistent) return s->two_phase ? t.put_2phase(b) : t.put_latching(b);
  // every key in stage 0 of one persistent launch (no roots read back)
  BlockIn bl;
  bl.keys_hexs = b.keys_hexs;
  bl.keys_indexs = b.keys_indexs;
  bl.values = b.values;
  bl.values_indexs = b.values_indexs;
  bl.trie_ids = b.trie_ids;  // null: every key in trie 0
  bl.n = b.n;
  bl.n0 = b.n;
  bl.keys_bytes = b.keys_bytes;
  bl.values_bytes = b.values_bytes;
  bl.device = b.device;
  rc = t.block_update(bl, nullptr, nullptr);
  // a rejected block applied nothing (e.g. pairs that do not tile the key
  // stream): LockNU takes the batch, and reports any malformed key itself
  if (rc == E_ARG) rc = t.put_latching(b);
  return rc;
}

// ---------------------------------------------------------------------------
// features

namespace {

// The statistics k_sample_features computes on the device, restated on the
// host: over s = min(n, 64) keys at positions j * n / s, the mean key length,
// its spread (population standard deviation), the share of samples equal to
// an earlier sample, and the mean longest common prefix of a sample with any
// other sample over the mean length.
void host_sample_stats(const uint8_t *keys, const int *kidx, int n, int64_t keys_bytes, float out[4]) {
  const int s = std::min(n, 64);
  std::vector<int64_t> off(s);
  std::vector<int> len(s);
  for (int j = 0; j < s; ++j) {
    const int64_t i = (int64_t)j * n / s;
    const int a = kidx[2 * i], z = kidx[2 * i + 1];
    const bool ok = a >= 0 && z >= a && (int64_t)z < keys_bytes;
    off[j] = ok ? a : 0;
    len[j] = ok ? z - a + 1 : 0;
  }
  double tl = 0, dup = 0, lcp = 0;
  for (int j = 0; j < s; ++j) {
    int best = 0;
    bool earlier = false;
    for (int k = 0; k < s; ++k) {
      if (k == j) continue;
      const int m = std::min(len[j], len[k]);
      int l = 0;
      while (l < m && keys[off[j] + l] == keys[off[k] + l]) ++l;
      if (l == m && len[j] == len[k] && k < j) earlier = true;
      best = std::max(best, l);
    }
    tl += len[j];
    dup += earlier ? 1 : 0;
    lcp += best;
  }
  const double mean = s ? tl / s : 0.0;
  double var = 0;
  for (int j = 0; j < s; ++j) var += (len[j] - mean) * (len[j] - mean);
  out[0] = (float)mean;
  out[1] = s ? (float)std::sqrt(var / s) : 0.f;
  out[2] = s ? (float)(dup / s) : 0.f;
  out[3] = mean > 0 ? (float)(lcp / s / mean) : 0.f;
}

}  // namespace

int batch_features(Trie &t, const BatchIn &b, float out[kNumFeatures], std::string &err) {
  const int n = b.n;
  if (n <= 0 || !b.keys_hexs || !b.keys_indexs || (!b.device && !b.values_indexs)) {
    err = "batch_features: empty batch or null arrays";
    return E_ARG;
  }
  int64_t kb = b.keys_bytes, vb = b.values_bytes;
  float st[4];
  if (b.device) {
    if (kb < 0 || vb < 0) {
      err = "batch_features: device batches need keys_bytes and values_bytes";
      return E_ARG;
    }
    if (kb == 0) {
      err = "batch_features: empty key stream";
      return E_ARG;
    }
    int rc = batch_features_device(b.keys_hexs, b.keys_indexs, n, kb, st, t.stream(), err);
    if (rc) return rc;
  } else {
    if (kb < 0) kb = (int64_t)b.keys_indexs[2 * n - 1] + 1;
    if (vb < 0) vb = (int64_t)b.values_indexs[2 * n - 1] + 1;
    host_sample_stats(b.keys_hexs, b.keys_indexs, n, kb, st);
  }
  int touched = 1;
  if (b.trie_ids && !b.device) {
    std::vector<int> ids(b.trie_ids, b.trie_ids + n);
    std::sort(ids.begin(), ids.end());
    touched = (int)(std::unique(ids.begin(), ids.end()) - ids.begin());
  }
  out[0] = (float)std::log2((double)n + 1.0);
  out[1] = (float)((double)kb / n / 64.0);
  out[2] = st[1] / 64.f;
  out[3] = st[2];
  out[4] = (float)std::log2((double)t.value_nodes() + 1.0);
  out[5] = (float)std::log2((double)vb / n + 1.0);
  out[6] = st[3];
  out[7] = (float)std::log2((double)std::max(touched, 1));
  return OK;
}

Bucket bucket_of(const float f[kNumFeatures]) {
  // the Python rule's buckets (gmpt/tuner.py bucket): size by 4x steps,
  // trie size (empty, then 64x steps), repeated-key share
  const double log2_n = f[0], log2_trie = f[4], dup = f[3];
  Bucket b;
  b.n = (int)(std::floor(std::min(std::max(log2_n, 10.0), 24.0) / 2.0));
  b.trie = log2_trie < 1.0 ? 0 : 1 + std::min(3, (int)std::floor(log2_trie / 6.0));
  b.dup = dup < 0.05 ? 0 : (dup < 0.3 ? 1 : 2);
  return b;
}

// ---------------------------------------------------------------------------
// selector

Selector::Selector(int device) : dev_(device) {}
Selector::~Selector() = default;

int Selector::rule_choice(const float f[kNumFeatures]) const {
  if (rules_.empty()) {
    if (default_k_ >= 0) return default_k_;
    if (f[4] < 1.0f) return kPhaseNU;           // empty trie: bulk load
    if (f[0] <= 16.0f) return kPersistent1;     // up to 64K keys: one launch
    return kLockNU4;
  }
  const Bucket b = bucket_of(f);
  int best = -1, dist = 1 << 30;
  for (const auto &r : rules_) {
    if (r.first == b) return r.second;
    const int d = std::abs(r.first.n - b.n) + std::abs(r.first.trie - b.trie) + std::abs(r.first.dup - b.dup);
    if (d < dist) {  // the first of equally near buckets, in file order
      dist = d;
      best = r.second;
    }
  }
  return best;
}

int Selector::choose(const float f[kNumFeatures], int *k, bool *used_net) {
  ++choices_;
  *used_net = false;
  bool in_range = use_net_ && net_ && !cols_.empty();
  for (int i = 0; in_range && i < kNumFeatures; ++i) {
    const float span = std::max(hi_[i] - lo_[i], 1e-6f);
    if (f[i] < lo_[i] - margin_ * span || f[i] > hi_[i] + margin_ * span) in_range = false;
  }
  if (!in_range) {
    ++fallbacks_;
    *k = rule_choice(f);
    return OK;
  }
  float z[kNumFeatures], y[kMlpMaxOut];
  for (int i = 0; i < kNumFeatures; ++i) z[i] = (f[i] - mean_[i]) / std_[i];
  if (net_->forward(z, 1, y)) {
    err_ = net_->error();
    return E_CUDA;
  }
  int best = cols_[0];
  for (int c : cols_)
    if (y[c] < y[best]) best = c;
  *k = best;
  *used_net = true;
  return OK;
}

// Selector file (text, whitespace separated), as gmpt.tuner.Selector.save
// writes it:
//   gmpt-selector 1
//   schedules K            (must equal the library's schedule count)
//   default k              (-1: the built-in default rule)
//   rules R   then R lines "bucket_n bucket_trie bucket_dup k"
//   net use I H O          (use 0/1; I = 8, O = K)
//   margin m
//   mean I floats / std I floats / lo I floats / hi I floats
//   cols C k...
//   params P floats        (W1 b1 W2 b2 W3 b3, gmpt_mlp layout)
// A file whose net line has I = 0 holds only the rule.
int Selector::load(const std::string &path) {
  std::ifstream in(path);
  if (!in) {
    err_ = "cannot open selector file " + path;
    return E_ARG;
  }
  auto bad = [&](const std::string &what) {
    err_ = "selector file " + path + ": " + what;
    return E_ARG;
  };
  std::string tag, word;
  int version = 0, K = 0, R = 0;
  if (!(in >> tag >> version) || tag != "gmpt-selector" || version != 1) return bad("not a gmpt-selector 1 file");
  if (!(in >> word >> K) || word != "schedules") return bad("schedules");
  if (K != kNumSchedules) return bad("written for " + std::to_string(K) + " schedules, the library has " +
                                     std::to_string(kNumSchedules));
  int dflt = -1;
  if (!(in >> word >> dflt) || word != "default" || dflt < -1 || dflt >= K) return bad("default");
  if (!(in >> word >> R) || word != "rules" || R < 0 || R > 100000) return bad("rules");
  std::vector<std::pair<Bucket, int>> rules;
  for (int r = 0; r < R; ++r) {
    Bucket b;
    int k;
    if (!(in >> b.n >> b.trie >> b.dup >> k) || k < 0 || k >= K) return bad("rule line");
    rules.push_back({b, k});
  }
  int use = 0, I = 0, H = 0, O = 0;
  if (!(in >> word >> use >> I >> H >> O) || word != "net") return bad("net");
  std::vector<float> mean, sd, lo, hi, params;
  std::vector<int> cols;
  float margin = 0.5f;
  std::unique_ptr<Mlp> net;
  if (I > 0) {
    if (I != kNumFeatures || O != K || H < 1 || H > kMlpMaxHidden) return bad("network shape");
    if (!(in >> word >> margin) || word != "margin") return bad("margin");
    auto vec = [&](const char *name, std::vector<float> &v, int count) {
      std::string w;
      if (!(in >> w) || w != name) return false;
      v.resize(count);
      for (auto &x : v)
        if (!(in >> x)) return false;
      return true;
    };
    if (!vec("mean", mean, I) || !vec("std", sd, I) || !vec("lo", lo, I) || !vec("hi", hi, I))
      return bad("normalisation");
    for (float s : sd)
      if (!(s > 0)) return bad("std must be positive");
    int C = 0;
    if (!(in >> word >> C) || word != "cols" || C < 1 || C > K) return bad("cols");
    cols.resize(C);
    for (auto &c : cols)
      if (!(in >> c) || c < 0 || c >= K) return bad("cols");
    net.reset(new Mlp(dev_, I, H, O, 1));
    if (!net->error().empty()) return bad(net->error());
    int P = 0;
    if (!(in >> word >> P) || word != "params" || P != net->n_params()) return bad("params");
    params.resize(P);
    for (auto &x : params)
      if (!(in >> x)) return bad("params");
    if (net->set_params(params.data())) return bad(net->error());
  }
  default_k_ = dflt;
  rules_ = std::move(rules);
  use_net_ = use != 0 && net != nullptr;
  margin_ = margin;
  mean_ = std::move(mean);
  std_ = std::move(sd);
  lo_ = std::move(lo);
  hi_ = std::move(hi);
  cols_ = std::move(cols);
  net_ = std::move(net);
  return OK;
}

}  // namespace gmpt
