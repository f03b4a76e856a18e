// schedule.h -- insert schedules and the schedule selector of the library.
//
// A put batch can run under several schedules that all give the same trie
// (the MPT is canonical in its key set, and every schedule applies the batch
// as if in index order, the last write of a key winning): PhaseNU (sort +
// level build) or LockNU (CAS insert), each with launch-shape knobs, or the
// persistent graph-replayed launch that inserts, hashes and reads the root
// in one kernel.  Choosing among them only changes time.
//
// The reference fixes the strategy (LockNU in lib/libgmpt.cu:107-111,
// 192-196, 299-303) and fits its cost model offline
// (test/experiments.cu:3250-3348); here the choice is made per batch at run
// time, by an autotuned rule table (coarse batch buckets -> the schedule
// measured fastest there) or by a small MLP whose inference runs on the
// library's own CUDA kernel (k_mlp_forward), with the rule as its fallback.
#pragma once
#include <stdint.h>

#include <memory>
#include <string>
#include <vector>

#include "trie.h"

namespace gmpt {

class Mlp;

struct Schedule {
  const char *name;
  bool two_phase;     // PhaseNU (else LockNU)
  bool persistent;    // one persistent launch: LockNU insert + PhaseHC + roots
  int local_build;    // PhaseNU: finish small build segments in one CTA
  int local_sort;     // PhaseNU: finish small tied sort runs in one CTA
  int latch_ways;     // LockNU keys per thread (1, 2, 4)
  int latch_dedup;    // LockNU repeated-key drop: 0 off, 1 batches >= 64K keys, 2 always
  int block_grid;     // persistent kernel CTAs (0 = all co-resident)
  int warp_full_max;  // hash levels with at most this many branches: a warp per branch
};

int schedule_count();
const Schedule *schedule_at(int k);

// Set every knob of schedule k on the trie.
int apply_schedule(Trie &t, int k);
// Insert batch b under schedule k (a persistent schedule also hashes; the
// caller's gmpt_hash_onepass then finds nothing left to do).
int put_schedule(Trie &t, int k, const BatchIn &b);

// Selector features of a put batch (kNumFeatures floats):
//   0 log2(n + 1)                    4 log2(keys in the trie object + 1)
//   1 mean key nibbles / 64          5 log2(mean value bytes + 1)
//   2 key-length spread / 64         6 mean longest common prefix of a
//   3 repeated-key share                sampled key with the other samples,
//                                       over the mean key length
//                                     7 log2(tries the batch touches)
// Items 2, 3, 6 come from 64 evenly spaced sampled keys (j * n / 64):
// k_sample_features on the device for device batches, the same statistics
// on the host for host batches.
constexpr int kNumFeatures = 8;
int batch_features(Trie &t, const BatchIn &b, float out[kNumFeatures], std::string &err);

// The rule's coarse bucket of a feature vector.
struct Bucket {
  int n, trie, dup;
  bool operator==(const Bucket &o) const { return n == o.n && trie == o.trie && dup == o.dup; }
};
Bucket bucket_of(const float f[kNumFeatures]);

class Selector {
 public:
  // A selector with only the built-in default rule (no measurements yet):
  // an empty trie is bulk-loaded by PhaseNU, batches of at most 64K keys run
  // as one persistent launch, larger ones as LockNU with 4 keys per thread.
  explicit Selector(int device);
  ~Selector();
  Selector(const Selector &) = delete;
  Selector &operator=(const Selector &) = delete;

  // Read a selector file (written by gmpt.tuner.Selector.save).
  int load(const std::string &path);
  int choose(const float f[kNumFeatures], int *k, bool *used_net);
  const std::string &error() const { return err_; }
  uint64_t choices() const { return choices_; }
  uint64_t fallbacks() const { return fallbacks_; }

 private:
  int dev_;
  int default_k_ = -1;  // -1: the built-in default rule
  std::vector<std::pair<Bucket, int>> rules_;
  bool use_net_ = false;
  float margin_ = 0.5f;
  std::vector<float> mean_, std_, lo_, hi_;
  std::vector<int> cols_;
  std::unique_ptr<Mlp> net_;
  uint64_t choices_ = 0, fallbacks_ = 0;
  std::string err_;
  int rule_choice(const float f[kNumFeatures]) const;
};

}  // namespace gmpt
