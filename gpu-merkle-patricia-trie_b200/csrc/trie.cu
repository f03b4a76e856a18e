// trie.cu -- host orchestration of the B200 MPT update path.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <mutex>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "trie.h"
#include "trie_kernels.cuh"
#include "latch_kernels.cuh"
#include "export_kernels.cuh"
#include "keccak_batch.cuh"
#include "local_build.cuh"
#include "local_sort.cuh"
#include "block_update.cuh"
#include "delete_kernels.cuh"
#include "gen_kernels.cuh"

namespace gmpt {

namespace {

constexpr int kThreads = 256;
constexpr int kHashThreads = kHashLevelThreads;
// k_hash_level_wide (132 registers: three CTAs per SM) for launches that
// cannot place more than three CTAs on each of B200's 148 SMs anyway
constexpr unsigned kWideGrid = 3 * 148;
// branch hash class (blocks - 1) from which a branch is hashed by a warp
constexpr uint32_t kWarpMinClass = 4;
constexpr uint32_t kMaxDepths = kMaxKeyNibbles + 2;  // nibble depths a dirty node can have
// LockNU batches of at least this many keys drop repeated keys first
constexpr int kDedupMinKeys = 1 << 16;

inline unsigned blocks_for(int64_t n, int t = kThreads) { return (unsigned)((n + t - 1) / t); }

// managed: unified memory (the trie may then exceed the device's memory,
// pages migrating on demand -- the reference's UMMPT, mpt/um_mpt.cuh:13-52),
// preferring the device the trie lives on
template <typename T>
cudaError_t grow_array(T *&p, size_t old_n, size_t new_n, cudaStream_t st, bool managed = false, int dev = 0) {
  T *q = nullptr;
  const size_t bytes = new_n * sizeof(T) + 64;
  cudaError_t e = managed ? cudaMallocManaged(&q, bytes) : cudaMalloc(&q, bytes);
  if (e != cudaSuccess) return e;
  if (managed) {
    e = cudaMemAdvise(q, bytes, cudaMemAdviseSetPreferredLocation, dev);
    if (e == cudaSuccess) e = cudaMemAdvise(q, bytes, cudaMemAdviseSetAccessedBy, dev);
    if (e != cudaSuccess) {
      cudaFree(q);
      return e;
    }
  }
  if (p && old_n) {
    e = cudaMemcpyAsync(q, p, old_n * sizeof(T), cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
  }
  if (p) cudaFree(p);
  p = q;
  return cudaSuccess;
}

template <typename T>
T *wsp(DevBlock &b, size_t n, cudaError_t &e) {
  if (e != cudaSuccess) return nullptr;
  e = b.ensure(n * sizeof(T) + 64);
  return b.as<T>();
}

}  // namespace

// ---------------------------------------------------------------------------

Trie::Trie(int device, int geth_mode, int max_tries, bool unified)
    : dev_(device), geth_(geth_mode ? 1 : 0), managed_(unified),
      n_tries_(max_tries > 1 ? (uint32_t)max_tries : 1u) {
  cudaError_t e = cudaSetDevice(dev_);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&roots_, sizeof(uint32_t) * n_tries_ + 64);
  if (e == cudaSuccess) e = cudaMalloc(&ctr_, sizeof(Counters));
  if (e == cudaSuccess) e = cudaMallocHost(&h_ctr_, sizeof(Counters));
  if (e == cudaSuccess) e = cudaMallocHost(&h_small_, 256);
  if (e == cudaSuccess) e = cudaMemset(roots_, 0, sizeof(uint32_t) * n_tries_ + 64);
  if (e == cudaSuccess) e = cudaMemset(ctr_, 0, sizeof(Counters));
  if (e != cudaSuccess) {
    err_ = std::string("trie init: ") + cudaGetErrorString(e);
    return;
  }
  tv_.roots = roots_;
  tv_.n_tries = n_tries_;
  tv_.ctr = ctr_;
  tv_.geth_mode = geth_;
  ensure_capacity(1024, 1024, 1024, 1024, 4096, 4096);
}

Trie::~Trie() {
  cudaSetDevice(dev_);
  if (st_) cudaStreamSynchronize(st_);
  void *ptrs[] = {tv_.full_child, tv_.full_epoch, tv_.full_depth, tv_.full_hash, tv_.full_hlen, tv_.full_dead, fl_refs_,
                  tv_.short_key, tv_.short_klen, tv_.short_child, tv_.short_epoch, tv_.short_depth,
                  tv_.short_dead, tv_.short_hash, tv_.short_hlen, tv_.short_claim, tv_.short_pseudo,
                  tv_.value_vid, tv_.rec, tv_.rec_hp, (void *)tv_.keys, (void *)tv_.vals,
                  roots_, ctr_, dirty_ref_, dirty_depth_};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  DevBlock *blocks[] = {&ws_.koff, &ws_.klen, &ws_.ki, &ws_.vi, &ws_.hp, &ws_.kin, &ws_.order, &ws_.eqprev,
                        &ws_.flags, &ws_.pos, &ws_.act, &ws_.skey, &ws_.sval, &ws_.uord, &ws_.w_status,
                        &ws_.w_code, &ws_.w_d0, &ws_.w_slot, &ws_.w_short, &ws_.w_after, &ws_.p_short,
                        &ws_.p_d0, &ws_.p_slot, &ws_.p_amin, &ws_.p_max, &ws_.it_key, &ws_.it_id,
                        &ws_.it_base, &ws_.it_len, &ws_.it_ref, &ws_.it_d0, &ws_.it_slot, &ws_.sb_base,
                        &ws_.sb_len, &ws_.sb_ref, &ws_.sb_d0, &ws_.sb_slot, &ws_.sb_code, &ws_.lcp,
                        &ws_.act2, &ws_.aseg, &ws_.aseg2, &ws_.kflags, &ws_.knib, &ws_.bins, &ws_.cursor,
                        &ws_.sorted_dirty, &ws_.g_keys, &ws_.g_idx, &ws_.g_hp, &ws_.g_len, &ws_.g_tid,
                        &ws_.tid, &ws_.dd_hash, &ws_.dd_pos, &ws_.dd_sel, &ws_.dd_slot, &ws_.raw, &ws_.dirty_cls, &ws_.rw_flags,
                        &ws_.rw_a, &ws_.rw_b, &ws_.rw_c, &ws_.rw_d, &ws_.rw_e, &ws_.rw_wpos, &ws_.rw_hp,
                        &ws_.rw_len, &ws_.rw_tot, &ws_.rw_kept, &ws_.rw_koff, &ws_.rw_klen, &ws_.rw_tid,
                        &ws_.del_hslot, &ws_.del_hext, &ws_.del_stamp,
                        &ws_.misc};
  for (DevBlock *b : blocks) b->release();
  for (int k = 0; k < 2; ++k) {
    ws_.s_start[k].release();
    ws_.s_end[k].release();
    ws_.s_depth[k].release();
    ws_.s_slot[k].release();
    ws_.s_D[k].release();
    ws_.s_branch[k].release();
  }
  sorter_.release();
  scan_ws_.release();
  DevBlock *bblocks[] = {&blk_.keys, &blk_.kidx, &blk_.vals, &blk_.vidx, &blk_.tid, &blk_.ptrie, &blk_.poff,
                         &blk_.out_ids, &blk_.out, &blk_.koff, &blk_.klen, &blk_.bins, &blk_.sorted};
  for (DevBlock *b : bblocks) b->release();
  for (auto &c : blk_.graphs) {
    if (c.exec) cudaGraphExecDestroy(c.exec);
    if (c.graph) cudaGraphDestroy(c.graph);
  }
  for (auto &ps : pipe_) {
    DevBlock *pb[] = {&ps.keys, &ps.kidx, &ps.vals, &ps.vidx, &ps.hp, &ps.tid};
    for (DevBlock *b : pb) b->release();
    if (ps.ready) cudaEventDestroy(ps.ready);
    if (ps.free) cudaEventDestroy(ps.free);
  }
  if (copy_st_) cudaStreamDestroy(copy_st_);
  if (blk_.d_desc) cudaFree(blk_.d_desc);
  if (blk_.h_desc) cudaFreeHost(blk_.h_desc);
  if (h_ctr_) cudaFreeHost(h_ctr_);
  if (h_small_) cudaFreeHost(h_small_);
  if (st_) cudaStreamDestroy(st_);
}

int Trie::fail(int code, const std::string &msg) {
  err_ = msg;
  return code;
}

int Trie::check_cuda(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return OK;
  return fail(E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

int Trie::sync_counters() {
  cudaError_t e = cudaMemcpyAsync(h_ctr_, ctr_, sizeof(Counters), cudaMemcpyDeviceToHost, st_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st_);
  if (e != cudaSuccess) return check_cuda(e, "sync counters");
  return apply_counters();
}

// Node counts and the error word from the pinned copy in h_ctr_.
int Trie::apply_counters() {
  n_full_ = h_ctr_->n_full;
  n_short_ = h_ctr_->n_short;
  n_value_ = h_ctr_->n_value;
  uint32_t err = h_ctr_->error;
  if (err) {
    cudaMemsetAsync(&ctr_->error, 0, 4, st_);
    if (err & ERR_CAPACITY) return fail(E_CAPACITY, "node pool capacity exceeded");
    if (err & ERR_RETRY_LIMIT) return fail(E_RETRY_LIMIT, "insert retry limit exceeded");
    if (err & ERR_KEY_TOO_LONG) return fail(E_BAD_KEY, "key longer than the supported maximum");
    if (err & ERR_BAD_TRIE) return fail(E_ARG, "trie id outside [0, max_tries)");
    if (err & ERR_BARRIER) return fail(E_INTERNAL, "grid barrier wait gave up");
    if (err & ERR_BAD_FLAG) return fail(E_ARG, "read/write flag other than 0 (read) or 1 (write)");
    if (err & ERR_BAD_KEY)
      return fail(E_BAD_KEY, "malformed key: nibble > 16, terminator not last, or a key that is a prefix of another");
    return fail(E_INTERNAL, "internal consistency check failed");
  }
  return OK;
}

uint64_t Trie::read_u64(const void *dptr) {
  cudaMemcpyAsync(h_small_, dptr, 8, cudaMemcpyDeviceToHost, st_);
  cudaStreamSynchronize(st_);
  return h_small_[0];
}

int Trie::ensure_capacity(uint64_t add_full, uint64_t add_short, uint64_t add_value, uint64_t add_rec,
                          uint64_t add_key_bytes, uint64_t add_val_bytes, bool exact) {
  cudaError_t e = cudaSuccess;
  auto grow_to = [exact](uint64_t need, uint64_t cap) {
    if (exact) return std::max<uint64_t>(need, 1024);
    uint64_t c = cap ? cap : 1024;
    while (c < need) c = c + c / 2 + 1024;
    return c;
  };
  uint64_t need_full = (uint64_t)n_full_ + add_full;
  if (need_full > kMaxNodes) return fail(E_CAPACITY, "branch node count exceeds 2^30");
  // a branch-pool cap: the pool stops growing there and a kernel that runs
  // out of branch nodes reports ERR_CAPACITY (the batch is then cut short)
  if (opt_max_full_ && need_full > opt_max_full_) need_full = std::max<uint64_t>(opt_max_full_, n_full_);
  if (need_full > cap_full_) {
    uint64_t nc = std::min<uint64_t>(grow_to(need_full, cap_full_), kMaxNodes);
    if (opt_max_full_) nc = std::min<uint64_t>(nc, std::max<uint64_t>(opt_max_full_, need_full));
    size_t o = n_full_;
    if (e == cudaSuccess) e = grow_array(tv_.full_child, o * 17, nc * 17, st_, managed_, dev_);
    if (e == cudaSuccess) e = grow_array(tv_.full_epoch, o, nc, st_, managed_, dev_);
    if (e == cudaSuccess) e = grow_array(tv_.full_depth, o, nc, st_, managed_, dev_);
    if (e == cudaSuccess) e = grow_array(tv_.full_hash, o * 32, nc * 32, st_, managed_, dev_);
    if (e == cudaSuccess) e = grow_array(tv_.full_hlen, o, nc, st_, managed_, dev_);
    if (e == cudaSuccess) e = grow_array(tv_.full_dead, o, nc, st_, managed_, dev_);
    if (e != cudaSuccess) return check_cuda(e, "grow branch pool");
    cap_full_ = (uint32_t)nc;
  }
  uint64_t need_short = (uint64_t)n_short_ + add_short;
  if (need_short > kMaxNodes) return fail(E_CAPACITY, "short node count exceeds 2^30");
  if (need_short > cap_short_) {
    uint64_t nc = std::min<uint64_t>(grow_to(need_short, cap_short_), kMaxNodes);
    size_t o = n_short_;
    if (e == cudaSuccess) e = grow_array(tv_.short_key, o, nc, st_, managed_, dev_);
    if (e == cudaSuccess) e = grow_array(tv_.short_klen, o, nc, st_, managed_, dev_);
    if (e == cudaSuccess) e = grow_array(tv_.short_child, o, nc, st_, managed_, dev_);
    if (e == cudaSuccess) e = grow_array(tv_.short_epoch, o, nc, st_, managed_, dev_);
    if (e == cudaSuccess) e = grow_array(tv_.short_depth, o, nc, st_, managed_, dev_);
    if (e == cudaSuccess) e = grow_array(tv_.short_dead, o, nc, st_, managed_, dev_);
    if (e == cudaSuccess) e = grow_array(tv_.short_hash, o * 32, nc * 32, st_, managed_, dev_);
    if (e == cudaSuccess) e = grow_array(tv_.short_hlen, o, nc, st_, managed_, dev_);
    if (e == cudaSuccess) e = grow_array(tv_.short_claim, o, nc, st_, managed_, dev_);
    if (e == cudaSuccess) e = grow_array(tv_.short_pseudo, o, nc, st_, managed_, dev_);
    if (e != cudaSuccess) return check_cuda(e, "grow short pool");
    cap_short_ = (uint32_t)nc;
  }
  uint64_t need_value = (uint64_t)n_value_ + add_value;
  if (need_value > kMaxNodes) return fail(E_CAPACITY, "value node count exceeds 2^30");
  if (need_value > cap_value_) {
    uint64_t nc = std::min<uint64_t>(grow_to(need_value, cap_value_), kMaxNodes);
    if ((e = grow_array(tv_.value_vid, n_value_, nc, st_, managed_, dev_)) != cudaSuccess) return check_cuda(e, "grow values");
    cap_value_ = (uint32_t)nc;
  }
  uint64_t need_rec = n_rec_ + add_rec;
  if (need_rec > cap_rec_) {
    uint64_t nc = grow_to(need_rec, cap_rec_);
    if (e == cudaSuccess) e = grow_array(tv_.rec, n_rec_, nc, st_, managed_, dev_);
    if (e == cudaSuccess) e = grow_array(tv_.rec_hp, n_rec_, nc, st_, managed_, dev_);
    if (e != cudaSuccess) return check_cuda(e, "grow value records");
    cap_rec_ = nc;
  }
  uint64_t need_keys = key_used_ + add_key_bytes + 64;
  if (need_keys > cap_keys_) {
    uint64_t nc = grow_to(need_keys, cap_keys_);
    uint8_t *p = const_cast<uint8_t *>(tv_.keys);
    if ((e = grow_array(p, key_used_, nc + 64, st_, managed_, dev_)) != cudaSuccess) return check_cuda(e, "grow key arena");
    tv_.keys = p;
    cap_keys_ = nc;
  }
  uint64_t need_vals = val_used_ + add_val_bytes + 64;
  if (need_vals > cap_vals_) {
    uint64_t nc = grow_to(need_vals, cap_vals_);
    uint8_t *p = const_cast<uint8_t *>(tv_.vals);
    if ((e = grow_array(p, val_used_, nc + 64, st_, managed_, dev_)) != cudaSuccess) return check_cuda(e, "grow value arena");
    tv_.vals = p;
    cap_vals_ = nc;
  }
  // every node is pushed to the dirty list at most once per hash generation
  uint64_t need_dirty = (uint64_t)cap_full_ + cap_short_;
  if (need_dirty > cap_dirty_) {
    uint64_t nc = need_dirty;
    uint32_t nd = 0;
    if (cap_dirty_) {
      cudaMemcpyAsync(h_small_, &ctr_->n_dirty, 4, cudaMemcpyDeviceToHost, st_);
      cudaStreamSynchronize(st_);
      nd = (uint32_t)(h_small_[0] & 0xFFFFFFFFu);
    }
    if (e == cudaSuccess) e = grow_array(dirty_ref_, nd, nc, st_, managed_, dev_);
    if (e == cudaSuccess) e = grow_array(dirty_depth_, nd, nc, st_, managed_, dev_);
    if (e != cudaSuccess) return check_cuda(e, "grow dirty list");
    cap_dirty_ = nc;
  }
  tv_.cap_full = cap_full_;
  tv_.cap_short = cap_short_;
  tv_.cap_value = cap_value_;
  stats_.device_bytes = (uint64_t)cap_full_ * (68 + 4 + 2 + 32 + 1 + 1) + (uint64_t)cap_short_ * (8 + 4 + 4 + 4 + 2 + 1 + 32 + 1 + 8) +
                        (uint64_t)cap_value_ * 8 + cap_rec_ * 24 + cap_keys_ + cap_vals_ + cap_dirty_ * 6;
  return OK;
}

// Copy the batch into the arenas and build per-key records.
int Trie::stage(const BatchIn &b, uint64_t &key_base, uint64_t &vid_base, uint64_t **koff, uint32_t **klen,
                uint32_t *maxlen, const int **tid_out) {
  const int n = b.n;
  cudaError_t e = cudaSuccess;
  const cudaMemcpyKind kind = b.device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  int64_t kbytes = b.keys_bytes, vbytes = b.values_bytes;
  if (kbytes < 0 || vbytes < 0) {
    if (b.device) return fail(E_ARG, "device batches must give keys_bytes and values_bytes");
    kbytes = (int64_t)b.keys_indexs[2 * n - 1] + 1;
    vbytes = (int64_t)b.values_indexs[2 * n - 1] + 1;
  }
  const int64_t raw_bytes = b.raw_keys ? kbytes : 0;
  unsigned long long *raw_pos = nullptr;
  if (b.raw_keys) {
    // pass 1: hex length of every key (pairs may overlap, so the expanded
    // stream is sized by a scan, not by the raw byte count)
    int *ki = wsp<int>(ws_.ki, 2 * (size_t)n, e);
    unsigned long long *lens = wsp<unsigned long long>(ws_.flags, (size_t)n, e);
    raw_pos = wsp<unsigned long long>(ws_.pos, (size_t)n, e);
    unsigned long long *d_tot = wsp<unsigned long long>(ws_.misc, 16, e) + 2;
    if (e == cudaSuccess) e = scan_ws_.ensure(scan_ws_bytes<unsigned long long>(n));
    if (e == cudaSuccess) e = cudaMemcpyAsync(ki, b.keys_indexs, sizeof(int) * 2 * (size_t)n, kind, st_);
    if (e != cudaSuccess) return check_cuda(e, "stage raw lengths");
    count_launch(), k_raw_lens<<<blocks_for(n), kThreads, 0, st_>>>(tv_, ki, n, raw_bytes, lens);
    if ((e = exclusive_scan<unsigned long long>(lens, raw_pos, n, d_tot, scan_ws_, st_)) != cudaSuccess ||
        (e = cudaMemcpyAsync(h_small_, d_tot, 8, cudaMemcpyDeviceToHost, st_)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st_)) != cudaSuccess)
      return check_cuda(e, "stage raw scan");
    kbytes = (int64_t)h_small_[0];
    // malformed pairs are reported (and the error word cleared) before any
    // other early return, so the next call does not inherit them
    if (int rc0 = sync_counters()) return rc0;
    if (kbytes >= (1ll << 31)) return fail(E_ARG, "key stream exceeds the int32 index range");
  }
  int rc = ensure_capacity(2ull * n, 4ull * n, (uint64_t)n, (uint64_t)n, (uint64_t)kbytes, (uint64_t)vbytes);
  if (rc) return rc;
  key_base = key_used_;
  vid_base = n_rec_;
  uint64_t val_base = val_used_;
  uint8_t *karena = const_cast<uint8_t *>(tv_.keys);
  uint8_t *varena = const_cast<uint8_t *>(tv_.vals);
  int *ki = wsp<int>(ws_.ki, 2 * (size_t)n, e);
  int64_t *vi = wsp<int64_t>(ws_.vi, 2 * (size_t)n, e);
  uint64_t *hp = b.values_hps ? wsp<uint64_t>(ws_.hp, (size_t)n, e) : nullptr;
  *koff = wsp<uint64_t>(ws_.koff, (size_t)n, e);
  *klen = wsp<uint32_t>(ws_.klen, (size_t)n, e);
  uint32_t *d_max = wsp<uint32_t>(ws_.misc, 32, e);  // same block size as the scan totals
  int *tid = b.trie_ids ? wsp<int>(ws_.tid, (size_t)n, e) : nullptr;
  if (e != cudaSuccess) return check_cuda(e, "stage alloc");
  *tid_out = tid;
  if (b.raw_keys) {
    // pass 2: nibbles + terminator written straight into the arena (device
    // batches are read where they lie; host bytes cross once)
    const uint8_t *raw = b.device ? b.keys_hexs : wsp<uint8_t>(ws_.raw, (size_t)raw_bytes + 8, e);
    if (e == cudaSuccess && raw_bytes && !b.device)
      e = cudaMemcpyAsync(const_cast<uint8_t *>(raw), b.keys_hexs, (size_t)raw_bytes, kind, st_);
    if (e != cudaSuccess) return check_cuda(e, "stage raw keys");
    count_launch(), k_raw_expand<<<blocks_for(n), kThreads, 0, st_>>>(raw, ki, raw_pos, n, raw_bytes,
                                                                     karena + key_base);
  } else {
    e = cudaMemcpyAsync(karena + key_base, b.keys_hexs, (size_t)kbytes, kind, st_);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ki, b.keys_indexs, sizeof(int) * 2 * (size_t)n, kind, st_);
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(varena + val_base, b.values, (size_t)vbytes, kind, st_);
  if (e == cudaSuccess) e = cudaMemcpyAsync(vi, b.values_indexs, sizeof(int64_t) * 2 * (size_t)n, kind, st_);
  if (e == cudaSuccess && hp) e = cudaMemcpyAsync(hp, b.values_hps, sizeof(uint64_t) * (size_t)n, kind, st_);
  if (e == cudaSuccess && tid) e = cudaMemcpyAsync(tid, b.trie_ids, sizeof(int) * (size_t)n, kind, st_);
  if (e == cudaSuccess) e = cudaMemsetAsync(karena + key_base + kbytes, 0, 64, st_);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_max, 0, 8, st_);
  if (e != cudaSuccess) return check_cuda(e, "stage copy");
  if ((e = cudaMemsetAsync(&ctr_->stream_terms, 0, 24, st_)) != cudaSuccess) return check_cuda(e, "stage reset");
  count_launch(), k_stage<<<std::min<unsigned>(blocks_for(n), 148 * 8), kThreads, 0, st_>>>(tv_, ki, vi, hp, n, key_base, val_base, vid_base, kbytes, vbytes,
                                                *koff, *klen, d_max, tid);
  if (kbytes > 0 && !b.raw_keys)  // expanded raw keys are well formed by construction
    count_launch(), k_stage_stream<<<std::min<unsigned>(blocks_for(kbytes / 8 + 1), 148 * 8), kThreads, 0, st_>>>(
        tv_, karena + key_base, kbytes);
  e = cudaMemcpyAsync(h_small_, d_max, 8, cudaMemcpyDeviceToHost, st_);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h_ctr_, ctr_, sizeof(Counters), cudaMemcpyDeviceToHost, st_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st_);
  if (e != cudaSuccess) return check_cuda(e, "stage");
  *maxlen = (uint32_t)(h_small_[0] & 0xFFFFFFFFu);
  max_key_nibbles_ = std::max(max_key_nibbles_, *maxlen);
  max_value_len_ = std::max(max_value_len_, (uint32_t)(h_small_[0] >> 32));
  if (b.raw_keys) {
    // nothing to check beyond k_raw_lens (errors come back with the counters)
  } else if (h_ctr_->noncontig) {
    // index pairs do not tile the stream: check every key's interior
    count_launch(), k_stage_keys<<<blocks_for(n), kThreads, 0, st_>>>(tv_, *koff, *klen, n);
  } else if (h_ctr_->bad_byte || h_ctr_->stream_terms != h_ctr_->key_terms) {
    return fail(E_BAD_KEY, "malformed key: nibble > 16 or a terminator inside a key");
  }
  // keys are 8-aligned in the arena so chunk loads start aligned more often
  key_used_ += ((uint64_t)kbytes + 7) & ~7ull;
  val_used_ += (uint64_t)vbytes;
  n_rec_ += (uint64_t)n;
  stats_.key_bytes = key_used_;
  stats_.value_bytes = val_used_;
  stats_.n_records = n_rec_;
  return OK;
}

// Lexicographic order of keys koff/klen[0..n) (terminator before nibble 0;
// a forest orders by trie first), stable: order[0..n) are positions, and
// eqprev[p] = 1 when key p equals key p - 1.
int Trie::sort_batch(int n, const uint64_t *koff, const uint32_t *klen, uint32_t maxlen, const int *tid,
                     uint32_t **order_out, uint8_t **eqprev_out) {
  cudaError_t e = cudaSuccess;
  uint32_t *order = wsp<uint32_t>(ws_.order, (size_t)n, e);
  uint8_t *eqprev = wsp<uint8_t>(ws_.eqprev, (size_t)n + 1, e);
  unsigned long long *flags = wsp<unsigned long long>(ws_.flags, (size_t)n, e);
  unsigned long long *pos = wsp<unsigned long long>(ws_.pos, (size_t)n, e);
  uint32_t *act = wsp<uint32_t>(ws_.act, (size_t)n, e);
  uint64_t *skey = wsp<uint64_t>(ws_.skey, (size_t)n, e);
  uint32_t *sval = wsp<uint32_t>(ws_.sval, (size_t)n, e);
  unsigned long long *d_tot = wsp<unsigned long long>(ws_.misc, 16, e) + 2;
  if (e == cudaSuccess) e = scan_ws_.ensure(scan_ws_bytes<unsigned long long>(n));
  if (e != cudaSuccess) return check_cuda(e, "sort alloc");
  count_launch(), k_init_order<<<blocks_for(n + 1), kThreads, 0, st_>>>(order, eqprev, n);
  int nchunks = (int)((maxlen + 7) / 8);
  stats_.sort_passes = 0;
  // leading chunks that every key shares sort nothing: skip their passes
  int c_first = tid ? -1 : 0;
  if (!tid && n > 1) {
    uint32_t *differs = reinterpret_cast<uint32_t *>(d_tot + 1);
    for (; c_first < nchunks; ++c_first) {
      if ((e = cudaMemsetAsync(differs, 0, 4, st_)) != cudaSuccess) return check_cuda(e, "sort prefix");
      count_launch(), k_chunk_shared<<<blocks_for(n), kThreads, 0, st_>>>(tv_.keys, koff, klen, n, c_first, differs);
      if ((e = cudaMemcpyAsync(h_small_, differs, 4, cudaMemcpyDeviceToHost, st_)) != cudaSuccess ||
          (e = cudaStreamSynchronize(st_)) != cudaSuccess)
        return check_cuda(e, "sort prefix");
      if (h_small_[0] & 0xFFFFFFFFu) break;
    }
  }
  // forest batches: a first pass orders by trie id
  for (int c = c_first; c <= nchunks; ++c) {
    int cc = (c == nchunks) ? -1 : (c < 0 ? -2 : c);  // final pass: key length
    count_launch(), k_sort_flags<<<blocks_for(n), kThreads, 0, st_>>>(eqprev, n, flags);
    e = exclusive_scan<unsigned long long>(flags, pos, n, d_tot, scan_ws_, st_);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_small_, d_tot, 8, cudaMemcpyDeviceToHost, st_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st_);
    if (e != cudaSuccess) return check_cuda(e, "sort flags");
    int K = (int)(h_small_[0] & 0xFFFFFFFFu);
    int S = (int)(h_small_[0] >> 32);
    if (K == 0) break;
    if (opt_local_sort_ && c >= 0) {
      // still-tied runs; if the largest fits one CTA, finish every run there
      uint32_t *rs = wsp<uint32_t>(ws_.it_id, (size_t)S, e);
      uint32_t *re = wsp<uint32_t>(ws_.it_len, (size_t)S, e);
      uint32_t *d_max = reinterpret_cast<uint32_t *>(d_tot + 1);
      if (e == cudaSuccess) e = cudaMemsetAsync(d_max, 0, 4, st_);
      if (e != cudaSuccess) return check_cuda(e, "sort runs alloc");
      count_launch(), k_sort_runs<<<blocks_for(n), kThreads, 0, st_>>>(flags, pos, eqprev, n, rs, re);
      count_launch(), k_run_max<<<blocks_for(S), kThreads, 0, st_>>>(rs, re, S, d_max);
      if ((e = cudaMemcpyAsync(h_small_, d_max, 4, cudaMemcpyDeviceToHost, st_)) != cudaSuccess ||
          (e = cudaStreamSynchronize(st_)) != cudaSuccess)
        return check_cuda(e, "sort runs");
      uint32_t maxrun = (uint32_t)(h_small_[0] & 0xFFFFFFFFu);
      const uint32_t cap = opt_local_sort_cap_ > 0 ? (uint32_t)opt_local_sort_cap_ : (uint32_t)kSortLocalCap;
      if (maxrun <= cap) {
        const size_t smem = sizeof(LocalSortSmem);
        if ((e = cudaFuncSetAttribute(k_local_sort, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
            cudaSuccess)
          return check_cuda(e, "local sort attr");
        count_launch(), k_local_sort<<<S, kSortLocalThreads, smem, st_>>>(tv_, rs, re, c, order, eqprev, koff, klen);
        if ((e = cudaGetLastError()) != cudaSuccess) return check_cuda(e, "local sort");
        break;
      }
    }
    count_launch(), k_sort_build<<<blocks_for(n), kThreads, 0, st_>>>(tv_, flags, pos, order, koff, klen, n, cc, act, skey, sval,
                                                                       tid);
    int passes = 0;
    if ((e = sorter_.sort(skey, sval, K, st_, &passes)) != cudaSuccess) return check_cuda(e, "radix sort");
    stats_.sort_passes += passes;
    count_launch(), k_sort_scatter<<<blocks_for(K), kThreads, 0, st_>>>(act, skey, sval, K, order, eqprev);
  }
  *order_out = order;
  *eqprev_out = eqprev;
  return OK;
}

// Lexicographic order of the batch with the last occurrence of every key
// kept: uord[0..m) are batch indices.  A mixed read/write batch (rw_ set)
// goes through sort_rw instead.
int Trie::sort_unique(int n, const uint64_t *koff, const uint32_t *klen, uint32_t maxlen, const int *tid,
                      uint32_t **uord_out, int *m_out) {
  if (rw_) return sort_rw(n, koff, klen, maxlen, tid, uord_out, m_out);
  if (opt_sort_dedup_ && n >= kDedupMinKeys) {
    bool done = false;
    int rc = sort_unique_dedup(n, koff, klen, maxlen, tid, uord_out, m_out, &done);
    if (rc || done) return rc;
  }
  uint32_t *order;
  uint8_t *eqprev;
  int rc = sort_batch(n, koff, klen, maxlen, tid, &order, &eqprev);
  if (rc) return rc;
  cudaError_t e = cudaSuccess;
  unsigned long long *flags = wsp<unsigned long long>(ws_.flags, (size_t)n, e);
  unsigned long long *pos = wsp<unsigned long long>(ws_.pos, (size_t)n, e);
  uint32_t *uord = wsp<uint32_t>(ws_.uord, (size_t)n, e);
  unsigned long long *d_tot = wsp<unsigned long long>(ws_.misc, 16, e) + 2;
  if (e != cudaSuccess) return check_cuda(e, "unique alloc");
  count_launch(), k_keep_flags<<<blocks_for(n), kThreads, 0, st_>>>(eqprev, n, flags);
  e = exclusive_scan<unsigned long long>(flags, pos, n, d_tot, scan_ws_, st_);
  if (e == cudaSuccess) count_launch(), k_keep_scatter<<<blocks_for(n), kThreads, 0, st_>>>(flags, pos, order, n, uord);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h_small_, d_tot, 8, cudaMemcpyDeviceToHost, st_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st_);
  if (e != cudaSuccess) return check_cuda(e, "unique");
  *m_out = (int)(h_small_[0] & 0xFFFFFFFFu);
  *uord_out = uord;
  return OK;
}


// PhaseNU with repeated keys: keep each key's last occurrence (the LockNU
// repeat table, k_dedup_*), then sort only the distinct keys.  Runs of one
// key repeated never untie in the chunked sort, so a batch with many
// repeats would run it to the last chunk of its longest key; distinct keys
// leave it after a few chunks.  Taken when an evenly spaced sample of 2^16
// keys holds more than 1 % repeats (or always, sort_dedup = 2); *done stays
// false (the caller sorts the whole batch) when it is not taken or when two
// different keys share a 64-bit hash.
int Trie::sort_unique_dedup(int n, const uint64_t *koff, const uint32_t *klen, uint32_t maxlen, const int *tid,
                            uint32_t **uord_out, int *m_out, bool *done) {
  cudaError_t e = cudaSuccess;
  *done = false;
  if (opt_sort_dedup_ == 1) {
    const int samples = std::min(n, 1 << 16);
    const uint32_t tsize = 1u << 17;
    unsigned long long *table = wsp<unsigned long long>(ws_.dd_hash, tsize, e);
    uint32_t *dups = reinterpret_cast<uint32_t *>(wsp<unsigned long long>(ws_.misc, 16, e) + 2);
    if (e == cudaSuccess) e = cudaMemsetAsync(table, 0, sizeof(unsigned long long) * tsize, st_);
    if (e == cudaSuccess) e = cudaMemsetAsync(dups, 0, 4, st_);
    if (e != cudaSuccess) return check_cuda(e, "repeat sample alloc");
    count_launch(), k_dup_sample<<<blocks_for(samples), kThreads, 0, st_>>>(tv_.keys, koff, klen, tid, samples,
                                                                              n / samples, table, tsize - 1, dups);
    if ((e = cudaMemcpyAsync(h_small_, dups, 4, cudaMemcpyDeviceToHost, st_)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st_)) != cudaSuccess)
      return check_cuda(e, "repeat sample");
    if ((uint64_t)(h_small_[0] & 0xFFFFFFFFu) * 100 <= (uint64_t)samples) return OK;
  }
  uint64_t size = 1024;
  while (size < 2ull * (uint64_t)n) size <<= 1;
  unsigned long long *table = wsp<unsigned long long>(ws_.dd_hash, 2 * size, e);
  uint32_t *sel = wsp<uint32_t>(ws_.dd_sel, (size_t)n, e);
  unsigned long long *keep = wsp<unsigned long long>(ws_.flags, (size_t)n, e);
  unsigned long long *rank = wsp<unsigned long long>(ws_.pos, (size_t)n, e);
  unsigned long long *d_tot = wsp<unsigned long long>(ws_.misc, 16, e) + 2;
  uint32_t *collision = reinterpret_cast<uint32_t *>(d_tot + 1);
  uint32_t *slot_of = wsp<uint32_t>(ws_.dd_slot, (size_t)n, e);
  if (e == cudaSuccess) e = scan_ws_.ensure(scan_ws_bytes<unsigned long long>(n));
  if (e == cudaSuccess) e = cudaMemsetAsync(table, 0, 2 * sizeof(unsigned long long) * size, st_);
  if (e == cudaSuccess) e = cudaMemsetAsync(collision, 0, 4, st_);
  if (e != cudaSuccess) return check_cuda(e, "repeat table alloc");
  const uint64_t hmask = opt_dedup_bits_ >= 64 ? ~0ull : ((1ull << opt_dedup_bits_) - 1);
  DedupTable tab{table, size - 1, hmask};
  count_launch(), k_dedup_insert<<<blocks_for(n), kThreads, 0, st_>>>(tv_, koff, klen, tid, n, tab, slot_of);
  count_launch(), k_dedup_mark<<<blocks_for(n), kThreads, 0, st_>>>(tv_, koff, klen, tid, n, tab, slot_of, keep,
                                                                    collision);
  if ((e = exclusive_scan<unsigned long long>(keep, rank, n, d_tot, scan_ws_, st_)) != cudaSuccess)
    return check_cuda(e, "repeat scan");
  count_launch(), k_dedup_compact<<<blocks_for(n), kThreads, 0, st_>>>(keep, rank, n, sel);
  if ((e = cudaMemcpyAsync(h_small_, d_tot, 16, cudaMemcpyDeviceToHost, st_)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st_)) != cudaSuccess)
    return check_cuda(e, "repeat count");
  if (h_small_[1] & 0xFFFFFFFFu) return OK;  // a hash shared by two keys: sort the whole batch
  const int m = (int)(h_small_[0] & 0xFFFFFFFFu);
  uint64_t *koff2 = wsp<uint64_t>(ws_.rw_koff, (size_t)m, e);
  uint32_t *klen2 = wsp<uint32_t>(ws_.rw_klen, (size_t)m, e);
  int *tid2 = tid ? wsp<int>(ws_.rw_tid, (size_t)m, e) : nullptr;
  uint32_t *uord = wsp<uint32_t>(ws_.uord, (size_t)m, e);
  if (e != cudaSuccess) return check_cuda(e, "repeat gather alloc");
  count_launch(), k_rw_gather<<<blocks_for(m), kThreads, 0, st_>>>(sel, m, koff, klen, tid, koff2, klen2, tid2);
  uint32_t *order2;
  uint8_t *eqprev2;
  int rc = sort_batch(m, koff2, klen2, maxlen, tid2, &order2, &eqprev2);
  if (rc) return rc;
  count_launch(), k_rw_map<<<blocks_for(m), kThreads, 0, st_>>>(order2, sel, m, uord);
  *uord_out = uord;
  *m_out = m;
  *done = true;
  return OK;
}

// Mixed read/write batch: group equal keys in batch order (hash-table slots
// + a stable radix sort of the slots; full-key sort if two keys share a
// 64-bit hash), answer the reads, keep the last write of every key; PhaseNU
// then gets the kept writes in key order.
int Trie::sort_rw(int n, const uint64_t *koff, const uint32_t *klen, uint32_t maxlen, const int *tid,
                  uint32_t **uord_out, int *m_out) {
  cudaError_t e = cudaSuccess;
  uint64_t size = 1024;
  while (size < 2ull * (uint64_t)n) size <<= 1;
  unsigned long long *table = wsp<unsigned long long>(ws_.dd_hash, 2 * size, e);
  uint64_t *skey = wsp<uint64_t>(ws_.skey, (size_t)n, e);
  uint32_t *sval = wsp<uint32_t>(ws_.sval, (size_t)n, e);
  uint32_t *order = wsp<uint32_t>(ws_.order, (size_t)n, e);
  uint8_t *eqprev = wsp<uint8_t>(ws_.eqprev, (size_t)n + 1, e);
  unsigned long long *tot = wsp<unsigned long long>(ws_.rw_tot, 8, e);
  uint32_t *collision = reinterpret_cast<uint32_t *>(tot + 5);
  if (e == cudaSuccess) e = cudaMemsetAsync(table, 0, 2 * sizeof(unsigned long long) * size, st_);
  if (e == cudaSuccess) e = cudaMemsetAsync(tot, 0, 64, st_);
  if (e != cudaSuccess) return check_cuda(e, "rw group alloc");
  const uint64_t hmask = opt_dedup_bits_ >= 64 ? ~0ull : ((1ull << opt_dedup_bits_) - 1);
  DedupTable tab{table, size - 1, hmask};
  uint32_t *slot_of = wsp<uint32_t>(ws_.dd_slot, (size_t)n, e);
  if (e != cudaSuccess) return check_cuda(e, "rw group alloc");
  count_launch(), k_dedup_insert<<<blocks_for(n), kThreads, 0, st_>>>(tv_, koff, klen, tid, n, tab, slot_of);
  count_launch(), k_rw_slots<<<blocks_for(n), kThreads, 0, st_>>>(tv_, koff, klen, tid, n, tab, slot_of, skey, sval,
                                                                  collision);
  if ((e = cudaMemcpyAsync(h_small_, collision, 4, cudaMemcpyDeviceToHost, st_)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st_)) != cudaSuccess)
    return check_cuda(e, "rw group");
  const bool grouped = (h_small_[0] & 0xFFFFFFFFu) == 0;
  int rc = OK;
  if (grouped) {
    int passes = 0;
    if ((e = sorter_.sort(skey, sval, n, st_, &passes)) != cudaSuccess) return check_cuda(e, "rw group sort");
    stats_.sort_passes = (uint32_t)passes;
    count_launch(), k_rw_groups<<<blocks_for(n + 1), kThreads, 0, st_>>>(skey, sval, n, order, eqprev);
  } else if ((rc = sort_batch(n, koff, klen, maxlen, tid, &order, &eqprev))) {
    return rc;
  }
  uint32_t *kept;
  int m = 0;
  if ((rc = resolve_rw(n, order, eqprev, koff, klen, tid, &kept, &m))) return rc;
  *m_out = m;
  *uord_out = kept;
  if (!rw_->key_order || !grouped || m <= 1) return OK;
  uint64_t *koff2 = wsp<uint64_t>(ws_.rw_koff, (size_t)m, e);
  uint32_t *klen2 = wsp<uint32_t>(ws_.rw_klen, (size_t)m, e);
  int *tid2 = tid ? wsp<int>(ws_.rw_tid, (size_t)m, e) : nullptr;
  uint32_t *uord = wsp<uint32_t>(ws_.uord, (size_t)m, e);
  if (e != cudaSuccess) return check_cuda(e, "rw key order alloc");
  count_launch(), k_rw_gather<<<blocks_for(m), kThreads, 0, st_>>>(kept, m, koff, klen, tid, koff2, klen2, tid2);
  uint32_t *order2;
  uint8_t *eqprev2;
  if ((rc = sort_batch(m, koff2, klen2, maxlen, tid2, &order2, &eqprev2))) return rc;
  count_launch(), k_rw_map<<<blocks_for(m), kThreads, 0, st_>>>(order2, kept, m, uord);
  *uord_out = uord;
  return OK;
}

// Mixed read/write batch after the sort: answer every read (k_rw_resolve)
// and keep the last write of every run, in sorted order, as uord[0..m).
int Trie::resolve_rw(int n, const uint32_t *order, const uint8_t *eqprev, const uint64_t *koff,
                     const uint32_t *klen, const int *tid, uint32_t **uord_out, int *m_out) {
  cudaError_t e = cudaSuccess;
  unsigned long long *A = wsp<unsigned long long>(ws_.rw_a, (size_t)n, e);  // is_write, then is_read
  unsigned long long *wrank = wsp<unsigned long long>(ws_.rw_b, (size_t)n, e);
  unsigned long long *head = wsp<unsigned long long>(ws_.rw_c, (size_t)n, e);
  unsigned long long *hbefore = wsp<unsigned long long>(ws_.rw_d, (size_t)n, e);
  unsigned long long *rrank = wsp<unsigned long long>(ws_.rw_e, (size_t)n, e);
  uint32_t *wpos = wsp<uint32_t>(ws_.rw_wpos, (size_t)n, e);
  unsigned long long *keep = wsp<unsigned long long>(ws_.flags, (size_t)n, e);
  unsigned long long *pos = wsp<unsigned long long>(ws_.pos, (size_t)n, e);
  uint32_t *uord = wsp<uint32_t>(ws_.rw_kept, (size_t)n, e);
  unsigned long long *tot = wsp<unsigned long long>(ws_.rw_tot, 8, e);  // writes, heads, reads, kept
  if (e == cudaSuccess) e = scan_ws_.ensure(scan_ws_bytes<unsigned long long>(n));
  if (e == cudaSuccess) e = cudaMemsetAsync(tot, 0, 64, st_);  // tot[4]: LockNU's (unused) collision word
  if (e != cudaSuccess) return check_cuda(e, "rw alloc");
  count_launch(), k_rw_sorted_flags<<<blocks_for(n), kThreads, 0, st_>>>(eqprev, order, rw_->flags, n, A, head);
  if ((e = exclusive_scan<unsigned long long>(A, wrank, n, tot + 0, scan_ws_, st_)) != cudaSuccess)
    return check_cuda(e, "rw scan");
  count_launch(), k_rw_wpos<<<blocks_for(n), kThreads, 0, st_>>>(A, wrank, n, wpos);
  if ((e = exclusive_scan<unsigned long long>(head, hbefore, n, tot + 1, scan_ws_, st_)) != cudaSuccess)
    return check_cuda(e, "rw scan");
  count_launch(), k_rw_read_flags<<<blocks_for(n), kThreads, 0, st_>>>(tv_, rw_->flags, n, A);
  if ((e = exclusive_scan<unsigned long long>(A, rrank, n, tot + 2, scan_ws_, st_)) != cudaSuccess)
    return check_cuda(e, "rw scan");
  count_launch(), k_rw_resolve<<<blocks_for(n), kThreads, 0, st_>>>(tv_, order, rw_->flags, head, hbefore, wrank, wpos,
                                                                     tot + 0, rrank, koff, klen, tid, rw_->vid_base, n,
                                                                     rw_->hp, rw_->len, keep);
  if ((e = exclusive_scan<unsigned long long>(keep, pos, n, tot + 3, scan_ws_, st_)) != cudaSuccess)
    return check_cuda(e, "rw scan");
  count_launch(), k_keep_scatter<<<blocks_for(n), kThreads, 0, st_>>>(keep, pos, order, n, uord);
  if ((e = cudaMemcpyAsync(h_small_, tot, 32, cudaMemcpyDeviceToHost, st_)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st_)) != cudaSuccess)
    return check_cuda(e, "rw resolve");
  rw_->reads = h_small_[2];
  *m_out = (int)h_small_[3];
  *uord_out = uord;
  return sync_counters();  // a bad flag rejects the batch before any insert
}

// A mixed batch was staged whole into the key arena, but after the reads
// are answered only the kept writes' keys are referenced (by the leaves the
// insert makes): move them to the start of the batch's region and give the
// rest back, so a read-heavy stream does not fill the arena with keys
// nothing points to.
int Trie::compact_rw_keys(int m, const uint32_t *kept, uint64_t *koff, const uint32_t *klen, uint64_t key_base) {
  cudaError_t e = cudaSuccess;
  uint8_t *arena = const_cast<uint8_t *>(tv_.keys);
  uint64_t total = 0;
  if (m > 0) {
    unsigned long long *sizes = wsp<unsigned long long>(ws_.rw_a, (size_t)m, e);
    unsigned long long *offs = wsp<unsigned long long>(ws_.rw_b, (size_t)m, e);
    unsigned long long *d_tot = wsp<unsigned long long>(ws_.rw_tot, 8, e) + 6;
    if (e == cudaSuccess) e = scan_ws_.ensure(scan_ws_bytes<unsigned long long>(m));
    if (e != cudaSuccess) return check_cuda(e, "rw compact alloc");
    count_launch(), k_rw_kept_sizes<<<blocks_for(m), kThreads, 0, st_>>>(kept, m, klen, sizes);
    if ((e = exclusive_scan<unsigned long long>(sizes, offs, m, d_tot, scan_ws_, st_)) != cudaSuccess)
      return check_cuda(e, "rw compact scan");
    total = read_u64(d_tot);
    uint8_t *tmp = wsp<uint8_t>(ws_.raw, (size_t)total + 8, e);
    if (e != cudaSuccess) return check_cuda(e, "rw compact alloc");
    count_launch(), k_rw_kept_copy<<<blocks_for(m), kThreads, 0, st_>>>(tv_.keys, koff, klen, kept, offs, m, tmp);
    if ((e = cudaMemcpyAsync(arena + key_base, tmp, (size_t)total, cudaMemcpyDeviceToDevice, st_)) != cudaSuccess)
      return check_cuda(e, "rw compact copy");
    count_launch(), k_rw_kept_offsets<<<blocks_for(m), kThreads, 0, st_>>>(kept, offs, m, key_base, koff);
  }
  if ((e = cudaMemsetAsync(arena + key_base + total, 0, 64, st_)) != cudaSuccess) return check_cuda(e, "rw compact tail");
  key_used_ = key_base + ((total + 7) & ~7ull);
  stats_.key_bytes = key_used_;
  return OK;
}

// Level-synchronous construction over the T sorted items in ws_.sb_*.
int Trie::build_levels(int T) {
  cudaError_t e = cudaSuccess;
  SortedItems si{ws_.sb_base.as<uint64_t>(), ws_.sb_len.as<uint32_t>(), ws_.sb_ref.as<uint32_t>(),
                 ws_.sb_d0.as<uint32_t>(),   ws_.sb_slot.as<uint64_t>(), ws_.sb_code.as<uint64_t>(),
                 ws_.lcp.as<uint16_t>()};
  DirtyList dl{dirty_ref_, dirty_depth_};
  uint8_t *kflags = wsp<uint8_t>(ws_.kflags, (size_t)T, e);
  uint8_t *knib = wsp<uint8_t>(ws_.knib, (size_t)T, e);
  unsigned long long *flags = wsp<unsigned long long>(ws_.flags, (size_t)T, e);
  unsigned long long *pos = wsp<unsigned long long>(ws_.pos, (size_t)T, e);
  uint32_t *act[2] = {wsp<uint32_t>(ws_.act, (size_t)T, e), wsp<uint32_t>(ws_.act2, (size_t)T, e)};
  uint32_t *aseg[2] = {wsp<uint32_t>(ws_.aseg, (size_t)T, e), wsp<uint32_t>(ws_.aseg2, (size_t)T, e)};
  SegArrays sg[2];
  for (int k = 0; k < 2; ++k) {
    sg[k].start = wsp<uint32_t>(ws_.s_start[k], (size_t)T, e);
    sg[k].end = wsp<uint32_t>(ws_.s_end[k], (size_t)T, e);
    sg[k].depth = wsp<uint32_t>(ws_.s_depth[k], (size_t)T, e);
    sg[k].D = wsp<uint32_t>(ws_.s_D[k], (size_t)T, e);
    sg[k].branch = wsp<uint32_t>(ws_.s_branch[k], (size_t)T, e);
    sg[k].slot = wsp<uint64_t>(ws_.s_slot[k], (size_t)T, e);
  }
  unsigned long long *d_tot = wsp<unsigned long long>(ws_.misc, 16, e) + 2;
  if (e == cudaSuccess) e = scan_ws_.ensure(scan_ws_bytes<unsigned long long>(T));
  if (e != cudaSuccess) return check_cuda(e, "build alloc");
  count_launch(), k_groups_init<<<blocks_for(T), kThreads, 0, st_>>>(tv_, dl, si, T, gen_, kflags, flags);
  e = exclusive_scan<unsigned long long>(flags, pos, T, d_tot, scan_ws_, st_);
  if (e != cudaSuccess) return check_cuda(e, "groups scan");
  count_launch(), k_groups_scatter<<<blocks_for(T), kThreads, 0, st_>>>(si, kflags, pos, T, act[0], aseg[0], sg[0]);
  uint32_t *d_max = reinterpret_cast<uint32_t *>(d_tot + 1);
  auto read_level = [&](int S_now, int cur_now) -> cudaError_t {
    cudaError_t x = cudaMemsetAsync(d_max, 0, 4, st_);
    if (x == cudaSuccess && S_now > 0 && opt_local_build_)
      count_launch(), k_seg_max<<<blocks_for(S_now), kThreads, 0, st_>>>(sg[cur_now], S_now, d_max);
    if (x == cudaSuccess) x = cudaMemcpyAsync(h_small_, d_tot, 16, cudaMemcpyDeviceToHost, st_);
    if (x == cudaSuccess) x = cudaStreamSynchronize(st_);
    return x;
  };
  if ((e = cudaMemcpyAsync(h_small_, d_tot, 8, cudaMemcpyDeviceToHost, st_)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st_)) != cudaSuccess)
    return check_cuda(e, "groups");
  int K = (int)(h_small_[0] & 0xFFFFFFFFu);
  int S = (int)(h_small_[0] >> 32);
  if ((e = read_level(S, 0)) != cudaSuccess) return check_cuda(e, "groups max");
  uint32_t maxseg = (uint32_t)(h_small_[1] & 0xFFFFFFFFu);
  int cur = 0, levels = 0;
  while (K > 0) {
    ++levels;
    if (levels > kMaxKeyNibbles + 2) return fail(E_INTERNAL, "builder did not converge");
    const uint32_t lcap = opt_local_build_cap_ > 0 ? (uint32_t)opt_local_build_cap_ : (uint32_t)kLocalCap;
    if (opt_local_build_ && maxseg <= lcap) {
      // every remaining segment fits one CTA: finish all subtries there
      const size_t smem = sizeof(LocalSmem);
      if ((e = cudaFuncSetAttribute(k_local_build, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
          cudaSuccess)
        return check_cuda(e, "local build attr");
      count_launch(), k_local_build<<<S, kLocalThreads, smem, st_>>>(tv_, dl, si, sg[cur], gen_);
      if ((e = cudaGetLastError()) != cudaSuccess) return check_cuda(e, "local build");
      break;
    }
    count_launch(), k_level_min<<<blocks_for(K), kThreads, 0, st_>>>(si, act[cur], aseg[cur], K, sg[cur]);
    count_launch(), k_level_nodes<<<blocks_for(S), kThreads, 0, st_>>>(tv_, dl, si, S, sg[cur], gen_);
    count_launch(), k_level_children<<<blocks_for(K), kThreads, 0, st_>>>(tv_, dl, si, act[cur], aseg[cur], K, sg[cur], gen_,
                                                          kflags, knib, flags);
    e = exclusive_scan<unsigned long long>(flags, pos, K, d_tot, scan_ws_, st_);
    if (e != cudaSuccess) return check_cuda(e, "level scan");
    count_launch(), k_level_scatter<<<blocks_for(K), kThreads, 0, st_>>>(act[cur], aseg[cur], kflags, knib, pos, K, sg[cur],
                                                         act[cur ^ 1], aseg[cur ^ 1], sg[cur ^ 1]);
    K = 0;
    cur ^= 1;
    // K, S of the next level are in d_tot; the largest segment comes with them
    if ((e = cudaMemcpyAsync(h_small_, d_tot, 8, cudaMemcpyDeviceToHost, st_)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st_)) != cudaSuccess)
      return check_cuda(e, "level");
    K = (int)(h_small_[0] & 0xFFFFFFFFu);
    S = (int)(h_small_[0] >> 32);
    if (K > 0 && opt_local_build_) {
      if ((e = read_level(S, cur)) != cudaSuccess) return check_cuda(e, "level max");
      maxseg = (uint32_t)(h_small_[1] & 0xFFFFFFFFu);
    }
  }
  stats_.build_levels = levels;
  return OK;
}

int Trie::put_2phase(const BatchIn &b) {
  err_.clear();
  if (b.n < 0 || b.n > (1 << 26)) return fail(E_ARG, "batch size must be in [0, 2^26]");
  if (b.n == 0) return OK;
  if (!b.keys_hexs || !b.keys_indexs || !b.values || !b.values_indexs) return fail(E_ARG, "null batch array");
  cudaSetDevice(dev_);
  cudaEvent_t ev[6];
  if (timing_)
    for (auto &x : ev) cudaEventCreate(&x);
  if (timing_) cudaEventRecord(ev[0], st_);
  ++epoch_;
  tv_.epoch = epoch_;
  tv_.gen = gen_;
  uint64_t key_base, vid_base;
  uint64_t *koff;
  uint32_t *klen;
  uint32_t maxlen = 0;
  const int *tid = nullptr;
  int rc = stage(b, key_base, vid_base, &koff, &klen, &maxlen, &tid);
  if (rc) return rc;
  if ((rc = sync_counters())) return rc;  // key validation
  if (timing_) cudaEventRecord(ev[1], st_);
  const int n = b.n;
  uint32_t *uord;
  int m = 0;
  if (rw_) rw_->vid_base = vid_base;
  if ((rc = sort_unique(n, koff, klen, maxlen, tid, &uord, &m))) return rc;
  if (rw_ && (rc = compact_rw_keys(m, uord, koff, klen, key_base))) return rc;
  stats_.last_unique = (uint64_t)m;
  if (timing_) cudaEventRecord(ev[2], st_);
  cudaError_t e = cudaSuccess;
  if (m == 0) {  // a mixed batch of reads only
    if (timing_)
      for (auto &x : ev) cudaEventDestroy(x);
    return sync_counters();
  }

  if (empty_) {
    // bulk load: one group (the root), items already sorted, no walk
    uint64_t *sb_base = wsp<uint64_t>(ws_.sb_base, (size_t)m, e);
    uint32_t *sb_len = wsp<uint32_t>(ws_.sb_len, (size_t)m, e);
    uint32_t *sb_ref = wsp<uint32_t>(ws_.sb_ref, (size_t)m, e);
    uint32_t *sb_d0 = wsp<uint32_t>(ws_.sb_d0, (size_t)m, e);
    uint64_t *sb_slot = wsp<uint64_t>(ws_.sb_slot, (size_t)m, e);
    uint64_t *sb_code = wsp<uint64_t>(ws_.sb_code, (size_t)m, e);
    uint16_t *lcp = wsp<uint16_t>(ws_.lcp, (size_t)m + 1, e);
    if (e != cudaSuccess) return check_cuda(e, "bulk alloc");
    if ((uint64_t)n_value_ + (uint64_t)m > cap_value_) return fail(E_CAPACITY, "value pool bound");
    count_launch(), k_items_bulk<<<blocks_for(m), kThreads, 0, st_>>>(tv_, uord, m, koff, klen, vid_base, n_value_,
                                                                      sb_base, sb_len, sb_ref, sb_d0, sb_slot, sb_code,
                                                                      tid);
    count_launch(), k_items_lcp<<<blocks_for(m), kThreads, 0, st_>>>(tv_, sb_base, sb_len, sb_d0, sb_code, m, lcp);
    stats_.last_new = (uint64_t)m;
    stats_.last_pseudo = 0;
    if (timing_) cudaEventRecord(ev[3], st_);
    if ((rc = build_levels(m))) return rc;
  } else {
  // walk
  WalkOut wo;
  wo.status = wsp<uint8_t>(ws_.w_status, (size_t)m, e);
  wo.code = wsp<uint64_t>(ws_.w_code, (size_t)m, e);
  wo.d0 = wsp<uint32_t>(ws_.w_d0, (size_t)m, e);
  wo.slot = wsp<uint64_t>(ws_.w_slot, (size_t)m, e);
  wo.short_id = wsp<uint32_t>(ws_.w_short, (size_t)m, e);
  wo.after = wsp<uint8_t>(ws_.w_after, (size_t)m, e);
  wo.p_short = wsp<uint32_t>(ws_.p_short, (size_t)m, e);
  wo.p_d0 = wsp<uint32_t>(ws_.p_d0, (size_t)m, e);
  wo.p_slot = wsp<uint64_t>(ws_.p_slot, (size_t)m, e);
  wo.p_amin = wsp<uint32_t>(ws_.p_amin, (size_t)m, e);
  wo.p_max = wsp<uint32_t>(ws_.p_max, (size_t)m, e);
  unsigned long long *flags = wsp<unsigned long long>(ws_.flags, (size_t)m, e);
  unsigned long long *pos = wsp<unsigned long long>(ws_.pos, (size_t)m, e);
  unsigned long long *d_tot = wsp<unsigned long long>(ws_.misc, 16, e) + 2;
  if (e == cudaSuccess) e = cudaMemsetAsync(&ctr_->n_pseudo, 0, 4, st_);
  if (e != cudaSuccess) return check_cuda(e, "walk alloc");
  DirtyList dl{dirty_ref_, dirty_depth_};
  count_launch(), k_walk<<<blocks_for((m + kWalkWays - 1) / kWalkWays), kThreads, 0, st_>>>(tv_, dl, uord, m, koff,
                                                                                             klen, vid_base, wo, tid);
  count_launch(), k_pseudo_ranks<<<blocks_for(m), kThreads, 0, st_>>>(tv_, wo, m);
  count_launch(), k_new_flags<<<blocks_for(m), kThreads, 0, st_>>>(wo.status, m, flags);
  e = exclusive_scan<unsigned long long>(flags, pos, m, d_tot, scan_ws_, st_);
  if (e != cudaSuccess) return check_cuda(e, "walk scan");
  if ((rc = sync_counters())) return rc;
  uint32_t n_pseudo = h_ctr_->n_pseudo;
  int n_new = (int)(read_u64(d_tot) & 0xFFFFFFFFu);
  stats_.last_new = (uint64_t)n_new;
  stats_.last_pseudo = n_pseudo;
  if (timing_) cudaEventRecord(ev[3], st_);
  int T = n_new + (int)n_pseudo;
  if (T > 0) {
    Items it;
    it.key = wsp<uint64_t>(ws_.it_key, (size_t)T, e);
    it.id = wsp<uint32_t>(ws_.it_id, (size_t)T, e);
    it.base = wsp<uint64_t>(ws_.it_base, (size_t)T, e);
    it.len = wsp<uint32_t>(ws_.it_len, (size_t)T, e);
    it.ref = wsp<uint32_t>(ws_.it_ref, (size_t)T, e);
    it.d0 = wsp<uint32_t>(ws_.it_d0, (size_t)T, e);
    it.slot = wsp<uint64_t>(ws_.it_slot, (size_t)T, e);
    uint64_t *sb_base = wsp<uint64_t>(ws_.sb_base, (size_t)T, e);
    uint32_t *sb_len = wsp<uint32_t>(ws_.sb_len, (size_t)T, e);
    uint32_t *sb_ref = wsp<uint32_t>(ws_.sb_ref, (size_t)T, e);
    uint32_t *sb_d0 = wsp<uint32_t>(ws_.sb_d0, (size_t)T, e);
    uint64_t *sb_slot = wsp<uint64_t>(ws_.sb_slot, (size_t)T, e);
    uint64_t *sb_code = wsp<uint64_t>(ws_.sb_code, (size_t)T, e);
    uint16_t *lcp = wsp<uint16_t>(ws_.lcp, (size_t)T + 1, e);
    if (e != cudaSuccess) return check_cuda(e, "items alloc");
    if (n_new > 0)
      count_launch(), k_items_new<<<blocks_for(m), kThreads, 0, st_>>>(tv_, wo, pos, m, uord, koff, klen, vid_base, it);
    if (n_pseudo > 0) {
      count_launch(), k_items_pseudo<<<blocks_for(n_pseudo), kThreads, 0, st_>>>(tv_, wo, (int)n_pseudo, n_new, it);
      int passes = 0;
      if ((e = sorter_.sort(it.key, it.id, T, st_, &passes)) != cudaSuccess) return check_cuda(e, "group sort");
    }
    count_launch(), k_items_gather<<<blocks_for(T), kThreads, 0, st_>>>(it, n_pseudo > 0 ? it.id : nullptr, T, sb_base, sb_len,
                                                        sb_ref, sb_d0, sb_slot, sb_code);
    count_launch(), k_items_lcp<<<blocks_for(T), kThreads, 0, st_>>>(tv_, sb_base, sb_len, sb_d0, sb_code, T, lcp);
    if ((rc = build_levels(T))) return rc;
  }
  }
  if ((rc = sync_counters())) return rc;
  if (timing_) {
    cudaEventRecord(ev[4], st_);
    cudaEventSynchronize(ev[4]);
    cudaEventElapsedTime(&stats_.t_stage_ms, ev[0], ev[1]);
    cudaEventElapsedTime(&stats_.t_sort_ms, ev[1], ev[2]);
    cudaEventElapsedTime(&stats_.t_walk_ms, ev[2], ev[3]);
    cudaEventElapsedTime(&stats_.t_build_ms, ev[3], ev[4]);
    for (auto &x : ev) cudaEventDestroy(x);
  }
  stats_.n_full = n_full_;
  stats_.n_short = n_short_;
  stats_.n_value = n_value_;
  empty_ = false;
  return OK;
}

// Counting sort of the nd dirty nodes by (depth, kind, hash class) into
// ws_.sorted_dirty; off[b] .. off[b + 1] is bin b (dirty_bin).
int Trie::bucket_dirty(uint32_t nd, uint32_t **sorted_out, std::vector<uint32_t> &off) {
  cudaError_t e = cudaSuccess;
  const uint32_t nbins = level_bin(kMaxDepths);
  uint32_t *bins = wsp<uint32_t>(ws_.bins, nbins, e);
  uint32_t *cursor = wsp<uint32_t>(ws_.cursor, nbins, e);
  uint32_t *sorted = wsp<uint32_t>(ws_.sorted_dirty, nd, e);
  uint8_t *cls = wsp<uint8_t>(ws_.dirty_cls, nd, e);
  if (e == cudaSuccess) e = cudaMemsetAsync(bins, 0, sizeof(uint32_t) * nbins, st_);
  if (e != cudaSuccess) return check_cuda(e, "hash alloc");
  // a leaf can take two or more Keccak blocks: order leaves by block count
  const int leaf_classes = (uint64_t)max_value_len_ + max_key_nibbles_ / 2 + 8 > 135 ? 1 : 0;
  int grid = std::min<int>(blocks_for(nd), 148 * 4);
  count_launch(), k_dirty_hist<<<grid, kThreads, sizeof(uint32_t) * nbins, st_>>>(
                      tv_, dirty_ref_, dirty_depth_, (int)nd, bins, (int)nbins, leaf_classes, cls);
  std::vector<uint32_t> hb(nbins);
  off.assign((size_t)nbins + 1, 0);
  if ((e = cudaMemcpyAsync(hb.data(), bins, sizeof(uint32_t) * nbins, cudaMemcpyDeviceToHost, st_)) !=
          cudaSuccess ||
      (e = cudaStreamSynchronize(st_)) != cudaSuccess)
    return check_cuda(e, "hash bins");
  for (uint32_t i = 0; i < nbins; ++i) off[i + 1] = off[i] + hb[i];
  if ((e = cudaMemcpyAsync(cursor, off.data(), sizeof(uint32_t) * nbins, cudaMemcpyHostToDevice, st_)) !=
      cudaSuccess)
    return check_cuda(e, "hash cursor");
  count_launch(), k_dirty_scatter<<<std::min<unsigned>(blocks_for(nd), 148 * 8), kThreads, 0, st_>>>(
                      dirty_ref_, dirty_depth_, cls, (int)nd, cursor, sorted, ctr_);
  *sorted_out = sorted;
  return OK;
}

// PhaseHC over every node marked dirty since the last hash.
int Trie::bucket_and_hash() {
  cudaError_t e = cudaSuccess;
  uint32_t nd = 0;
  if ((e = cudaMemcpyAsync(h_small_, &ctr_->n_dirty, 4, cudaMemcpyDeviceToHost, st_)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st_)) != cudaSuccess)
    return check_cuda(e, "dirty count");
  nd = (uint32_t)(h_small_[0] & 0xFFFFFFFFu);
  stats_.last_dirty = nd;
  stats_.last_hash_levels = 0;
  if (nd == 0) return OK;
  uint32_t *sorted = nullptr;
  std::vector<uint32_t> off;
  int rc = bucket_dirty(nd, &sorted, off);
  if (rc) return rc;
  size_t smem = sizeof(uint64_t) * 17 * kHashThreads;
  int levels = 0;
  if ((e = cudaMemsetAsync(&ctr_->hashed, 0, 4, st_)) != cudaSuccess ||
      (e = cudaMemsetAsync(&ctr_->enc_bytes, 0, 16, st_)) != cudaSuccess)
    return check_cuda(e, "hash counters");
  cudaEvent_t ka = nullptr, kz = nullptr;
  if (timing_) {
    cudaEventCreate(&ka);
    cudaEventCreate(&kz);
    cudaEventRecord(ka, st_);
  }
  const size_t smem_warp = 4 * kWarpMsgBytes;
  tv_.account = timing_ ? 1 : 0;  // per-node accounting atomics only when measuring
  // a launch of at most kWideGrid CTAs cannot fill the SMs at the
  // throughput form's occupancy: it runs the wide form (more registers per
  // thread, no spills, shorter serial chains)
  auto level = [&](const uint32_t *refs, uint32_t cnt) {
    const unsigned grid = blocks_for(cnt, kHashThreads);
    if (grid <= kWideGrid)
      count_launch(), k_hash_level_wide<<<grid, kHashThreads, smem, st_>>>(tv_, refs, (int)cnt);
    else
      count_launch(), k_hash_level<<<grid, kHashThreads, smem, st_>>>(tv_, refs, (int)cnt);
  };
  // every leaf first (one launch), then the levels deepest first
  if (off[kLeafClasses] > 0) {
    ++levels;
    level(sorted, off[kLeafClasses]);
  }
  for (int d = (int)kMaxDepths - 1; d >= 0; --d) {
    uint32_t a = off[level_bin(d)], m = off[level_bin(d) + 1], z = off[level_bin(d + 1)];
    if (z == a) continue;
    ++levels;
    // branches of kWarpMinClass + 1 blocks or more: the level's first branch
    // bins (longest first)
    const uint32_t ml = off[level_bin(d) + 1 + (kHashClasses - kWarpMinClass)];
    if (z - m > 0 && z - m <= (uint32_t)opt_warp_full_max_) {
      // few branches: short nodes thread-wise, branches one warp each
      if (m > a) level(sorted + a, m - a);
      count_launch(), k_hash_full_warp<<<(z - m + 3) / 4, 128, smem_warp, st_>>>(tv_, sorted + m, (int)(z - m));
    } else if (ml > m && ml - m <= (uint32_t)opt_warp_full_max_) {
      // a few branches of many blocks (a key ending at a branch puts its
      // value, up to kilobytes, in slot 16) would set the level's time as
      // one thread's serial chain: one warp each, the rest thread-wise
      count_launch(), k_hash_full_warp<<<(ml - m + 3) / 4, 128, smem_warp, st_>>>(tv_, sorted + m, (int)(ml - m));
      if (m > a) level(sorted + a, m - a);
      level(sorted + ml, z - ml);
    } else {
      level(sorted + a, z - a);
    }
  }
  if (timing_) {
    cudaEventRecord(kz, st_);
    cudaEventSynchronize(kz);
    cudaEventElapsedTime(&stats_.t_hash_kernels_ms, ka, kz);
    cudaEventDestroy(ka);
    cudaEventDestroy(kz);
  }
  tv_.account = 0;
  if (track_dirty_) {  // keep this pass's nodes for flush_dirty
    if (fl_n_ + nd > fl_cap_) {
      uint64_t nc = std::max<uint64_t>(fl_n_ + nd, fl_cap_ + fl_cap_ / 2 + 1024);
      if ((e = grow_array(fl_refs_, fl_n_, nc, st_, managed_, dev_)) != cudaSuccess)
        return check_cuda(e, "grow flush record");
      fl_cap_ = nc;
    }
    if ((e = cudaMemcpyAsync(fl_refs_ + fl_n_, dirty_ref_, 4 * (size_t)nd, cudaMemcpyDeviceToDevice, st_)) !=
        cudaSuccess)
      return check_cuda(e, "flush record");
    fl_n_ += nd;
  }
  stats_.last_hash_levels = levels;
  stats_.hash_launches = levels;
  if ((e = cudaMemsetAsync(&ctr_->n_dirty, 0, 4, st_)) != cudaSuccess) return check_cuda(e, "hash reset");
  if ((e = cudaGetLastError()) != cudaSuccess) return check_cuda(e, "hash launch");
  ++gen_;
  tv_.gen = gen_;
  return OK;
}

int Trie::hash() {
  err_.clear();
  cudaSetDevice(dev_);
  cudaEvent_t a, z;
  if (timing_) {
    cudaEventCreate(&a);
    cudaEventCreate(&z);
    cudaEventRecord(a, st_);
  }
  int rc = bucket_and_hash();
  if (rc) return rc;
  if ((rc = sync_counters())) return rc;
  stats_.last_hashed = h_ctr_->hashed;
  stats_.last_enc_bytes = h_ctr_->enc_bytes;
  stats_.last_keccak_blocks = h_ctr_->keccak_blocks;
  if (timing_) {
    cudaEventRecord(z, st_);
    cudaEventSynchronize(z);
    cudaEventElapsedTime(&stats_.t_hash_ms, a, z);
    cudaEventDestroy(a);
    cudaEventDestroy(z);
  }
  return OK;
}

int Trie::root(uint8_t out[32], int *len, int trie) {
  err_.clear();
  if (trie < 0 || (uint32_t)trie >= n_tries_) return fail(E_ARG, "trie id outside [0, max_tries)");
  cudaSetDevice(dev_);
  cudaError_t e = cudaSuccess;
  uint8_t *d = wsp<uint8_t>(ws_.misc, 256, e) + 128;
  int *did = reinterpret_cast<int *>(d + 64);
  if (e != cudaSuccess) return check_cuda(e, "root alloc");
  if ((e = cudaMemcpyAsync(did, &trie, 4, cudaMemcpyHostToDevice, st_)) != cudaSuccess) return check_cuda(e, "root id");
  count_launch(), k_roots<<<1, 32, 0, st_>>>(tv_, did, 1, d);
  uint8_t h[40];
  if ((e = cudaMemcpyAsync(h_small_, d, 33, cudaMemcpyDeviceToHost, st_)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st_)) != cudaSuccess)
    return check_cuda(e, "root");
  std::memcpy(h, h_small_, 33);
  *len = h[32];
  std::memcpy(out, h, 32);
  return OK;
}

int Trie::roots(const int *ids, int n, uint8_t *out32, int *sizes) {
  err_.clear();
  if (n <= 0) return OK;
  if (ids)
    for (int i = 0; i < n; ++i)
      if (ids[i] < 0 || (uint32_t)ids[i] >= n_tries_) return fail(E_ARG, "trie id outside [0, max_tries)");
  if (!ids && (uint32_t)n > n_tries_) return fail(E_ARG, "more roots than tries");
  cudaSetDevice(dev_);
  cudaError_t e = cudaSuccess;
  int *did = ids ? wsp<int>(ws_.g_tid, (size_t)n, e) : nullptr;
  uint8_t *d = wsp<uint8_t>(ws_.g_keys, 33 * (size_t)n, e);
  if (e == cudaSuccess && ids) e = cudaMemcpyAsync(did, ids, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, st_);
  if (e != cudaSuccess) return check_cuda(e, "roots alloc");
  count_launch(), k_roots<<<blocks_for(32 * (int64_t)n), kThreads, 0, st_>>>(tv_, did, n, d);
  std::vector<uint8_t> h(33 * (size_t)n);
  if ((e = cudaMemcpyAsync(h.data(), d, h.size(), cudaMemcpyDeviceToHost, st_)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st_)) != cudaSuccess)
    return check_cuda(e, "roots");
  for (int i = 0; i < n; ++i) {
    std::memcpy(out32 + 32 * (size_t)i, h.data() + 33 * (size_t)i, 32);
    sizes[i] = h[33 * (size_t)i + 32];
  }
  return OK;
}

int Trie::gets(const uint8_t *keys_hexs, const int *keys_indexs, int n, bool device_inputs, uint64_t *out_hp,
               int *out_len, int64_t keys_bytes, const int *trie_ids, bool device_outputs) {
  err_.clear();
  if (n <= 0) return OK;
  cudaSetDevice(dev_);
  cudaError_t e = cudaSuccess;
  if (keys_bytes < 0) {
    if (device_inputs) return fail(E_ARG, "device lookups need keys_bytes");
    keys_bytes = (int64_t)keys_indexs[2 * n - 1] + 1;
  }
  cudaMemcpyKind kind = device_inputs ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  uint8_t *dk = wsp<uint8_t>(ws_.g_keys, (size_t)keys_bytes + 64, e);
  int *di = wsp<int>(ws_.g_idx, 2 * (size_t)n, e);
  uint64_t *dhp = wsp<uint64_t>(ws_.g_hp, (size_t)n, e);
  int *dlen = wsp<int>(ws_.g_len, (size_t)n, e);
  int *dtid = trie_ids ? wsp<int>(ws_.g_tid, (size_t)n, e) : nullptr;
  // the keys are copied next to a zeroed 64-byte tail (the 8-byte key loads
  // may read past a key's last byte); index pairs and trie ids of device
  // batches are read where they are
  if (e == cudaSuccess) e = cudaMemcpyAsync(dk, keys_hexs, (size_t)keys_bytes, kind, st_);
  if (e == cudaSuccess) e = cudaMemsetAsync(dk + keys_bytes, 0, 64, st_);
  const int *ki = device_inputs ? keys_indexs : di;
  const int *ti = device_inputs ? trie_ids : dtid;
  if (e == cudaSuccess && !device_inputs)
    e = cudaMemcpyAsync(di, keys_indexs, sizeof(int) * 2 * (size_t)n, kind, st_);
  if (e == cudaSuccess && dtid && !device_inputs)
    e = cudaMemcpyAsync(dtid, trie_ids, sizeof(int) * (size_t)n, kind, st_);
  if (e != cudaSuccess) return check_cuda(e, "gets copy");
  if (device_outputs) {
    count_launch(), k_gets<<<blocks_for(n), kThreads, 0, st_>>>(tv_, dk, ki, n, keys_bytes, out_hp, out_len, nullptr,
                                                                ti);
    e = cudaStreamSynchronize(st_);
    return check_cuda(e, "gets");
  }
  count_launch(), k_gets<<<blocks_for(n), kThreads, 0, st_>>>(tv_, dk, ki, n, keys_bytes, dhp, dlen, nullptr, ti);
  e = cudaMemcpyAsync(out_hp, dhp, sizeof(uint64_t) * (size_t)n, cudaMemcpyDeviceToHost, st_);
  if (e == cudaSuccess) e = cudaMemcpyAsync(out_len, dlen, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, st_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st_);
  return check_cuda(e, "gets");
}

int Trie::get_values(const uint8_t *keys_hexs, const int *keys_indexs, int n, std::vector<uint8_t> &vals,
                     std::vector<int64_t> &offs) {
  err_.clear();
  vals.clear();
  offs.assign(2 * (size_t)n, -1);
  if (n <= 0) return OK;
  cudaSetDevice(dev_);
  cudaError_t e = cudaSuccess;
  int64_t keys_bytes = (int64_t)keys_indexs[2 * n - 1] + 1;
  uint8_t *dk = wsp<uint8_t>(ws_.g_keys, (size_t)keys_bytes + 64, e);
  int *di = wsp<int>(ws_.g_idx, 2 * (size_t)n, e);
  uint64_t *dhp = wsp<uint64_t>(ws_.g_hp, (size_t)n, e);
  int *dlen = wsp<int>(ws_.g_len, (size_t)n, e);
  int64_t *dvid = wsp<int64_t>(ws_.misc, (size_t)n + 64, e);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dk, keys_hexs, (size_t)keys_bytes, cudaMemcpyHostToDevice, st_);
  if (e == cudaSuccess) e = cudaMemsetAsync(dk + keys_bytes, 0, 64, st_);
  if (e == cudaSuccess) e = cudaMemcpyAsync(di, keys_indexs, sizeof(int) * 2 * (size_t)n, cudaMemcpyHostToDevice, st_);
  if (e != cudaSuccess) return check_cuda(e, "get_values copy");
  count_launch(), k_gets<<<blocks_for(n), kThreads, 0, st_>>>(tv_, dk, di, n, keys_bytes, dhp, dlen, dvid, nullptr);
  std::vector<int64_t> vid(n);
  std::vector<int> len(n);
  e = cudaMemcpyAsync(vid.data(), dvid, 8 * (size_t)n, cudaMemcpyDeviceToHost, st_);
  if (e == cudaSuccess) e = cudaMemcpyAsync(len.data(), dlen, 4 * (size_t)n, cudaMemcpyDeviceToHost, st_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st_);
  if (e != cudaSuccess) return check_cuda(e, "get_values");
  // value offsets of the found records
  std::vector<uint64_t> roff(n, 0);
  for (int i = 0; i < n; ++i) {
    if (vid[i] < 0) continue;
    e = cudaMemcpyAsync(&roff[i], &tv_.rec[vid[i]].off, 8, cudaMemcpyDeviceToHost, st_);
    if (e != cudaSuccess) return check_cuda(e, "get_values rec");
  }
  cudaStreamSynchronize(st_);
  for (int i = 0; i < n; ++i) {
    if (vid[i] < 0) continue;
    size_t at = vals.size();
    vals.resize(at + (size_t)len[i]);
    if (len[i] > 0) {
      e = cudaMemcpy(vals.data() + at, tv_.vals + roff[i], (size_t)len[i], cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) return check_cuda(e, "get_values bytes");
    }
    offs[2 * i] = (int64_t)at;
    offs[2 * i + 1] = (int64_t)at + len[i] - 1;
  }
  return OK;
}

const uint32_t *Trie::pending_dirty(int *n) const {
  cudaMemcpy(h_small_, &ctr_->n_dirty, 4, cudaMemcpyDeviceToHost);
  *n = (int)(h_small_[0] & 0xFFFFFFFFu);
  return dirty_ref_;
}

int Trie::reset() {
  err_.clear();
  cudaSetDevice(dev_);
  cudaError_t e = cudaMemsetAsync(roots_, 0, sizeof(uint32_t) * n_tries_, st_);
  if (e == cudaSuccess) e = cudaMemsetAsync(ctr_, 0, sizeof(Counters), st_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st_);
  if (e != cudaSuccess) return check_cuda(e, "reset");
  n_full_ = n_short_ = n_value_ = 0;
  n_rec_ = key_used_ = val_used_ = 0;
  max_key_nibbles_ = max_value_len_ = 0;
  fl_n_ = 0;
  empty_ = true;
  ++gen_;
  tv_.gen = gen_;
  return OK;
}

}  // namespace gmpt

namespace gmpt {

// LockNU batch: no sort, every key (duplicates included) inserted concurrently.
int Trie::put_latching(const BatchIn &b) {
  err_.clear();
  if (b.n < 0 || b.n > (1 << 26)) return fail(E_ARG, "batch size must be in [0, 2^26]");
  if (b.n == 0) return OK;
  if (!b.keys_hexs || !b.keys_indexs || !b.values || !b.values_indexs) return fail(E_ARG, "null batch array");
  cudaSetDevice(dev_);
  cudaEvent_t ev[3];
  if (timing_) {
    for (auto &x : ev) cudaEventCreate(&x);
    cudaEventRecord(ev[0], st_);
  }
  ++epoch_;
  tv_.epoch = epoch_;
  tv_.gen = gen_;
  uint64_t key_base, vid_base;
  uint64_t *koff;
  uint32_t *klen;
  uint32_t maxlen = 0;
  const int *tid = nullptr;
  int rc = stage(b, key_base, vid_base, &koff, &klen, &maxlen, &tid);
  if (rc) return rc;
  if ((rc = sync_counters())) return rc;
  if (timing_) cudaEventRecord(ev[1], st_);
  DirtyList dl{dirty_ref_, dirty_depth_};
  KeySelect ks;
  if (rw_) {
    // mixed batch: the sort answers the reads and selects the last write of
    // every key (in key order) for the insert
    rw_->vid_base = vid_base;
    uint32_t *uord;
    int m = 0;
    if ((rc = sort_unique(b.n, koff, klen, maxlen, tid, &uord, &m))) return rc;
    if ((rc = sync_counters())) return rc;
    if ((rc = compact_rw_keys(m, uord, koff, klen, key_base))) return rc;
    if (m == 0) {
      if (timing_)
        for (auto &x : ev) cudaEventDestroy(x);
      return OK;
    }
    ks.sel = uord;
    ks.count = ws_.rw_tot.as<unsigned long long>() + 3;
    ks.collision = reinterpret_cast<const uint32_t *>(ws_.rw_tot.as<unsigned long long>() + 4);  // zeroed
  } else if (opt_latch_dedup_ == 2 || (opt_latch_dedup_ == 1 && b.n >= kDedupMinKeys)) {
    // walk each distinct key once (its last occurrence); see k_dedup_*
    cudaError_t e = cudaSuccess;
    uint64_t size = 1024;
    while (size < 2ull * (uint64_t)b.n) size <<= 1;
    unsigned long long *table = wsp<unsigned long long>(ws_.dd_hash, 2 * size, e);
    uint32_t *sel = wsp<uint32_t>(ws_.dd_sel, (size_t)b.n, e);
    unsigned long long *keep = wsp<unsigned long long>(ws_.flags, (size_t)b.n, e);
    unsigned long long *rank = wsp<unsigned long long>(ws_.pos, (size_t)b.n, e);
    unsigned long long *d_tot = wsp<unsigned long long>(ws_.misc, 16, e) + 2;
    uint32_t *collision = reinterpret_cast<uint32_t *>(d_tot + 1);
    if (e == cudaSuccess) e = scan_ws_.ensure(scan_ws_bytes<unsigned long long>(b.n));
    if (e == cudaSuccess) e = cudaMemsetAsync(table, 0, 2 * sizeof(unsigned long long) * size, st_);
    if (e == cudaSuccess) e = cudaMemsetAsync(collision, 0, 4, st_);
    if (e != cudaSuccess) return check_cuda(e, "dedup alloc");
    const uint64_t hmask = opt_dedup_bits_ >= 64 ? ~0ull : ((1ull << opt_dedup_bits_) - 1);
    DedupTable tab{table, size - 1, hmask};
    uint32_t *slot_of = wsp<uint32_t>(ws_.dd_slot, (size_t)b.n, e);
    if (e != cudaSuccess) return check_cuda(e, "dedup alloc");
    count_launch(), k_dedup_insert<<<blocks_for(b.n), kThreads, 0, st_>>>(tv_, koff, klen, tid, b.n, tab, slot_of);
    count_launch(), k_dedup_mark<<<blocks_for(b.n), kThreads, 0, st_>>>(tv_, koff, klen, tid, b.n, tab, slot_of, keep,
                                                                        collision);
    if ((e = exclusive_scan<unsigned long long>(keep, rank, b.n, d_tot, scan_ws_, st_)) != cudaSuccess)
      return check_cuda(e, "dedup scan");
    count_launch(), k_dedup_compact<<<blocks_for(b.n), kThreads, 0, st_>>>(keep, rank, b.n, sel);
    ks.sel = sel;
    ks.count = d_tot;
    ks.collision = collision;
  }
  const int ways = opt_latch_ways_;
  auto kern = ways == 1 ? k_latch_insert<1> : (ways == 2 ? k_latch_insert<2> : k_latch_insert<4>);
  count_launch(), kern<<<blocks_for((b.n + ways - 1) / ways), kThreads, 0, st_>>>(tv_, dl, koff, klen, b.n, vid_base,
                                                                                 opt_retry_limit_, tid, ks);
  if ((rc = check_cuda(cudaGetLastError(), "latch launch"))) return rc;
  empty_ = false;  // keys may be in even when the batch stops on an error
  if ((rc = sync_counters())) return rc;
  if (timing_) {
    cudaEventRecord(ev[2], st_);
    cudaEventSynchronize(ev[2]);
    cudaEventElapsedTime(&stats_.t_stage_ms, ev[0], ev[1]);
    cudaEventElapsedTime(&stats_.t_build_ms, ev[1], ev[2]);
    stats_.t_sort_ms = stats_.t_walk_ms = 0;
    for (auto &x : ev) cudaEventDestroy(x);
  }
  stats_.n_full = n_full_;
  stats_.n_short = n_short_;
  stats_.n_value = n_value_;
  stats_.last_unique = (uint64_t)b.n;
  empty_ = false;
  return OK;
}

}  // namespace gmpt

namespace gmpt {

int Trie::flush_nodes(const uint8_t *keys_hexs, const int *keys_indexs, int n, std::vector<uint8_t> &hashs,
                      std::vector<uint8_t> &encs, std::vector<unsigned long long> &encs_indexs) {
  err_.clear();
  hashs.clear();
  encs.clear();
  encs_indexs.clear();
  if (n <= 0) return OK;
  cudaSetDevice(dev_);
  cudaError_t e = cudaSuccess;
  int64_t keys_bytes = (int64_t)keys_indexs[2 * n - 1] + 1;
  uint8_t *dk = wsp<uint8_t>(ws_.g_keys, (size_t)keys_bytes + 64, e);
  int *di = wsp<int>(ws_.g_idx, 2 * (size_t)n, e);
  uint32_t *d_cnt = wsp<uint32_t>(ws_.misc, 64, e);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dk, keys_hexs, (size_t)keys_bytes, cudaMemcpyHostToDevice, st_);
  if (e == cudaSuccess) e = cudaMemsetAsync(dk + keys_bytes, 0, 64, st_);
  if (e == cudaSuccess) e = cudaMemcpyAsync(di, keys_indexs, sizeof(int) * 2 * (size_t)n, cudaMemcpyHostToDevice, st_);
  if (e != cudaSuccess) return check_cuda(e, "flush copy");
  uint32_t cap = (uint32_t)std::min<uint64_t>((uint64_t)n * 24 + 64, 0x7FFFFFFFull);
  for (int attempt = 0; attempt < 2; ++attempt) {
    uint64_t *refs = wsp<uint64_t>(ws_.skey, cap, e);
    uint32_t *dummy = wsp<uint32_t>(ws_.sval, cap, e);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_cnt, 0, 4, st_);
    if (e != cudaSuccess) return check_cuda(e, "flush alloc");
    count_launch(), k_flush_collect<<<blocks_for(n), kThreads, 0, st_>>>(tv_, dk, di, n, keys_bytes, refs, d_cnt, cap);
    uint32_t cnt = (uint32_t)(read_u64(d_cnt) & 0xFFFFFFFFu);
    if (cnt > cap) {
      cap = cnt;
      continue;
    }
    if (cnt == 0) return OK;
    if ((e = sorter_.sort(refs, dummy, cnt, st_)) != cudaSuccess) return check_cuda(e, "flush sort");
    unsigned long long *flags = wsp<unsigned long long>(ws_.flags, cnt, e);
    unsigned long long *pos = wsp<unsigned long long>(ws_.pos, cnt, e);
    uint32_t *uref = wsp<uint32_t>(ws_.act, cnt, e);
    unsigned long long *sizes = wsp<unsigned long long>(ws_.it_key, cnt, e);
    unsigned long long *offs = wsp<unsigned long long>(ws_.it_base, cnt, e);
    unsigned long long *d_tot = wsp<unsigned long long>(ws_.misc, 64, e) + 4;
    if (e == cudaSuccess) e = scan_ws_.ensure(scan_ws_bytes<unsigned long long>(cnt));
    if (e != cudaSuccess) return check_cuda(e, "flush alloc2");
    count_launch(), k_flush_unique_flags<<<blocks_for(cnt), kThreads, 0, st_>>>(refs, (int)cnt, flags);
    if ((e = exclusive_scan<unsigned long long>(flags, pos, cnt, d_tot, scan_ws_, st_)) != cudaSuccess)
      return check_cuda(e, "flush scan");
    int m = (int)read_u64(d_tot);
    count_launch(), k_flush_sizes<<<blocks_for(cnt), kThreads, 0, st_>>>(tv_, refs, flags, pos, (int)cnt, uref, sizes);
    if ((e = exclusive_scan<unsigned long long>(sizes, offs, m, d_tot, scan_ws_, st_)) != cudaSuccess)
      return check_cuda(e, "flush scan2");
    uint64_t total = read_u64(d_tot);
    uint8_t *d_encs = wsp<uint8_t>(ws_.sb_base, total + 64, e);
    unsigned long long *d_idx = wsp<unsigned long long>(ws_.sb_slot, 2 * (size_t)m, e);
    uint8_t *d_hash = wsp<uint8_t>(ws_.sb_code, 32 * (size_t)m, e);
    if (e != cudaSuccess) return check_cuda(e, "flush alloc3");
    count_launch(), k_flush_write<<<blocks_for(m), kThreads, 0, st_>>>(tv_, uref, offs, m, d_encs, d_idx, d_hash);
    hashs.resize(32 * (size_t)m);
    encs.resize(total);
    encs_indexs.resize(2 * (size_t)m);
    e = cudaMemcpyAsync(hashs.data(), d_hash, hashs.size(), cudaMemcpyDeviceToHost, st_);
    if (e == cudaSuccess && total) e = cudaMemcpyAsync(encs.data(), d_encs, total, cudaMemcpyDeviceToHost, st_);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(encs_indexs.data(), d_idx, 8 * encs_indexs.size(), cudaMemcpyDeviceToHost, st_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st_);
    return check_cuda(e, "flush read");
  }
  return fail(E_INTERNAL, "flush: node count changed between passes");
}

int Trie::flush_dirty(std::vector<uint8_t> &hashs, std::vector<uint8_t> &encs,
                       std::vector<unsigned long long> &encs_indexs) {
  err_.clear();
  hashs.clear();
  encs.clear();
  encs_indexs.clear();
  if (!track_dirty_) return fail(E_ARG, "flush_dirty needs the track_dirty option (set before the puts)");
  cudaSetDevice(dev_);
  const uint64_t cnt = fl_n_;
  if (cnt == 0) return OK;
  if (cnt > 0x7FFFFFFFull) return fail(E_CAPACITY, "flush record exceeds 2^31 nodes");
  cudaError_t e = cudaSuccess;
  uint64_t *refs = wsp<uint64_t>(ws_.skey, cnt, e);
  uint32_t *dummy = wsp<uint32_t>(ws_.sval, cnt, e);
  unsigned long long *flags = wsp<unsigned long long>(ws_.flags, cnt, e);
  unsigned long long *pos = wsp<unsigned long long>(ws_.pos, cnt, e);
  uint32_t *uref = wsp<uint32_t>(ws_.act, cnt, e);
  unsigned long long *sizes = wsp<unsigned long long>(ws_.it_key, cnt, e);
  unsigned long long *offs = wsp<unsigned long long>(ws_.it_base, cnt, e);
  unsigned long long *d_tot = wsp<unsigned long long>(ws_.misc, 64, e) + 4;
  if (e == cudaSuccess) e = scan_ws_.ensure(scan_ws_bytes<unsigned long long>(cnt));
  if (e != cudaSuccess) return check_cuda(e, "flush dirty alloc");
  count_launch(), k_widen_u32<<<blocks_for((int64_t)cnt), kThreads, 0, st_>>>(fl_refs_, (int64_t)cnt, refs);
  if ((e = sorter_.sort(refs, dummy, (int)cnt, st_)) != cudaSuccess) return check_cuda(e, "flush dirty sort");
  count_launch(), k_flush_dirty_flags<<<blocks_for((int64_t)cnt), kThreads, 0, st_>>>(tv_, refs, (int)cnt, flags);
  if ((e = exclusive_scan<unsigned long long>(flags, pos, cnt, d_tot, scan_ws_, st_)) != cudaSuccess)
    return check_cuda(e, "flush dirty scan");
  const int m = (int)read_u64(d_tot);
  fl_n_ = 0;
  if (m == 0) return OK;
  count_launch(), k_flush_sizes<<<blocks_for((int64_t)cnt), kThreads, 0, st_>>>(tv_, refs, flags, pos, (int)cnt, uref,
                                                                               sizes);
  if ((e = exclusive_scan<unsigned long long>(sizes, offs, m, d_tot, scan_ws_, st_)) != cudaSuccess)
    return check_cuda(e, "flush dirty scan2");
  const uint64_t total = read_u64(d_tot);
  uint8_t *d_encs = wsp<uint8_t>(ws_.sb_base, total + 64, e);
  unsigned long long *d_idx = wsp<unsigned long long>(ws_.sb_slot, 2 * (size_t)m, e);
  uint8_t *d_hash = wsp<uint8_t>(ws_.sb_code, 32 * (size_t)m, e);
  if (e != cudaSuccess) return check_cuda(e, "flush dirty alloc2");
  count_launch(), k_flush_write<<<blocks_for(m), kThreads, 0, st_>>>(tv_, uref, offs, m, d_encs, d_idx, d_hash);
  hashs.resize(32 * (size_t)m);
  encs.resize(total);
  encs_indexs.resize(2 * (size_t)m);
  e = cudaMemcpyAsync(hashs.data(), d_hash, hashs.size(), cudaMemcpyDeviceToHost, st_);
  if (e == cudaSuccess && total) e = cudaMemcpyAsync(encs.data(), d_encs, total, cudaMemcpyDeviceToHost, st_);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(encs_indexs.data(), d_idx, 8 * encs_indexs.size(), cudaMemcpyDeviceToHost, st_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st_);
  return check_cuda(e, "flush dirty read");
}

}  // namespace gmpt

namespace gmpt {

static std::atomic<uint64_t> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
uint64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }

// Keccak-256 of n messages (inclusive [start, end] int64 index pairs into
// data); device pointers, synchronous.
int keccak256_batch_device(const uint8_t *d_data, const int64_t *d_idx, int n, uint8_t *d_out, cudaStream_t st) {
  if (n <= 0) return OK;
  size_t smem = sizeof(uint64_t) * 17 * kHashThreads;
  count_launch(), k_keccak256_batch<<<blocks_for(n, kHashThreads), kHashThreads, smem, st>>>(d_data, d_idx, n, d_out);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return e == cudaSuccess ? OK : E_CUDA;
}

// Permutations per second of the register-only Keccak loop on `device`.
int keccak_peak(int device, double *perm_per_s) {
  cudaError_t e = cudaSetDevice(device);
  int sms = 0;
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  uint64_t *sink = nullptr;
  if (e == cudaSuccess) e = cudaMalloc(&sink, 64);
  cudaEvent_t a, z;
  cudaEventCreate(&a);
  cudaEventCreate(&z);
  const int blocks = sms * 16, threads = 128, iters = 64;
  double best = 0;
  for (int rep = 0; rep < 4 && e == cudaSuccess; ++rep) {
    cudaEventRecord(a);
    count_launch(), k_keccak_peak<<<blocks, threads>>>(sink, iters);
    cudaEventRecord(z);
    e = cudaEventSynchronize(z);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, z);
    double r = (double)blocks * threads * iters / (ms / 1e3);
    if (rep > 0 && r > best) best = r;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(z);
  if (sink) cudaFree(sink);
  if (e != cudaSuccess) return E_CUDA;
  *perm_per_s = best;
  return OK;
}

}  // namespace gmpt

// ---------------------------------------------------------------------------
// Allocation-free batched Keccak-256 for callers that cannot allocate device
// memory.  All device-side staging lives in one file-scope array of fixed
// size that every GPU loading the library keeps until process exit.

#include <mutex>

namespace gmpt {

namespace {

constexpr int64_t kNoAllocMaxMessages = 32768;
constexpr int64_t kNoAllocMaxBytes = 2ll << 20;  // message bytes per call
constexpr int64_t kNoAllocTail = 64;             // zeroed, covers 8-byte over-reads
constexpr int64_t kNoAllocIdxOff = kNoAllocMaxBytes + 256;
constexpr int64_t kNoAllocOutOff = kNoAllocIdxOff + kNoAllocMaxMessages * 16;
constexpr int64_t kNoAllocBytes = kNoAllocOutOff + kNoAllocMaxMessages * 32;  // 3.5 MiB + 256 B

static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocBytes];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
uint8_t *g_noalloc_ptr[kNoAllocMaxDevices] = {};

}  // namespace

int keccak256_batch_noalloc(const uint8_t *data, const int64_t *indexs, int n, uint8_t *out32, std::string &err) {
  if (n < 0 || (n > 0 && (!data || !indexs || !out32))) {
    err = "null argument";
    return E_ARG;
  }
  if (n == 0) return OK;
  if (n > kNoAllocMaxMessages) {
    err = "gmpt_keccak256_batch_noalloc: " + std::to_string(n) + " messages exceed the limit of " +
          std::to_string(kNoAllocMaxMessages);
    return E_ARG;
  }
  int64_t bytes = 0;
  for (int i = 0; i < n; ++i) {
    if (indexs[2 * i] < 0 || indexs[2 * i + 1] < indexs[2 * i] - 1) {
      err = "bad index pair";
      return E_ARG;
    }
    // bounded before the + 1, so an end near INT64_MAX cannot wrap past the check
    if (indexs[2 * i + 1] >= kNoAllocMaxBytes) {
      err = "gmpt_keccak256_batch_noalloc: message bytes up to index " + std::to_string(indexs[2 * i + 1]) +
            " exceed the limit of " + std::to_string(kNoAllocMaxBytes);
      return E_ARG;
    }
    bytes = std::max<int64_t>(bytes, indexs[2 * i + 1] + 1);
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) {
    err = "no usable current device";
    return E_CUDA;
  }
  std::lock_guard<std::mutex> g(g_noalloc_mu);  // calls share the array
  if (!g_noalloc_ptr[dev]) {
    // one-time set-up on this device (the current one): the device address
    // of the array; the host-side symbol is not a device address
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
      return E_CUDA;
    }
    g_noalloc_ptr[dev] = static_cast<uint8_t *>(p);
  }
  uint8_t *base = g_noalloc_ptr[dev];
  uint8_t *d_data = base;
  int64_t *d_idx = reinterpret_cast<int64_t *>(base + kNoAllocIdxOff);
  uint8_t *d_out = base + kNoAllocOutOff;
  // The calling thread's per-thread default stream: it does not wait for the
  // library's own or the caller's non-blocking streams (only for the legacy
  // default stream, if the process uses that one too).
  cudaStream_t st = cudaStreamPerThread;
  if (bytes) e = cudaMemcpyAsync(d_data, data, (size_t)bytes, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_data + bytes, 0, kNoAllocTail, st);  // what the over-reads see
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_idx, indexs, sizeof(int64_t) * 2 * (size_t)n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    size_t smem = sizeof(uint64_t) * 17 * kHashThreads;
    count_launch(),
        k_keccak256_batch<<<blocks_for(n, kHashThreads), kHashThreads, smem, st>>>(d_data, d_idx, n, d_out);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(out32, d_out, 32 * (size_t)n, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    err = std::string("keccak no-alloc: ") + cudaGetErrorString(e);
    return E_CUDA;
  }
  return OK;
}

}  // namespace gmpt

namespace gmpt {

int Trie::set_option(const std::string &name, int64_t value) {
  err_.clear();
  if (name == "local_build") {
    opt_local_build_ = value != 0;
    return OK;
  }
  if (name == "local_sort") {
    opt_local_sort_ = value != 0;
    return OK;
  }
  if (name == "block_grid") {
    if (value < 0 || value > 1 << 20) return fail(E_ARG, "block_grid must be in [0, 2^20]");
    opt_block_grid_ = (int)value;
    return OK;
  }
  if (name == "latch_dedup") {
    if (value < 0 || value > 2) return fail(E_ARG, "latch_dedup must be 0, 1 or 2");
    opt_latch_dedup_ = (int)value;
    return OK;
  }
  if (name == "sort_dedup") {
    if (value < 0 || value > 2) return fail(E_ARG, "sort_dedup must be 0, 1 or 2");
    opt_sort_dedup_ = (int)value;
    return OK;
  }
  if (name == "latch_dedup_bits") {
    if (value < 1 || value > 64) return fail(E_ARG, "latch_dedup_bits must be in [1, 64]");
    opt_dedup_bits_ = (int)value;
    return OK;
  }
  if (name == "latch_ways") {
    if (value != 1 && value != 2 && value != 4) return fail(E_ARG, "latch_ways must be 1, 2 or 4");
    opt_latch_ways_ = (int)value;
    return OK;
  }
  if (name == "block_graph") {
    opt_block_graph_ = value != 0;
    return OK;
  }
  if (name == "warp_full_max") {
    if (value < 0 || value > 1 << 30) return fail(E_ARG, "warp_full_max must be in [0, 2^30]");
    opt_warp_full_max_ = (int)value;
    return OK;
  }
  if (name == "local_build_cap") {
    if (value < 0 || value > kLocalCap) return fail(E_ARG, "local_build_cap must be in [0, 2048]");
    opt_local_build_cap_ = (int)value;
    return OK;
  }
  if (name == "local_sort_cap") {
    if (value < 0 || value > kSortLocalCap) return fail(E_ARG, "local_sort_cap must be in [0, 2048]");
    opt_local_sort_cap_ = (int)value;
    return OK;
  }
  if (name == "track_dirty") {
    track_dirty_ = value != 0;
    if (!track_dirty_) fl_n_ = 0;
    return OK;
  }
  if (name == "block_barrier_ns") {
    if (value < 1 || value > 60000000000ll) return fail(E_ARG, "block_barrier_ns must be in [1, 6e10]");
    opt_barrier_ns_ = (uint64_t)value;
    return OK;
  }
  if (name == "max_branch_nodes") {
    if (value < 0 || value > (int64_t)kMaxNodes) return fail(E_ARG, "max_branch_nodes must be in [0, 2^30)");
    opt_max_full_ = (uint32_t)value;
    return OK;
  }
  if (name == "retry_limit") {
    if (value < 1 || value > (1ll << 30)) return fail(E_ARG, "retry_limit must be in [1, 2^30]");
    opt_retry_limit_ = (uint32_t)value;
    return OK;
  }
  return fail(E_ARG, "unknown option: " + name);
}

}  // namespace gmpt

// ---------------------------------------------------------------------------
// Persistent forest block updates.

namespace gmpt {

namespace {

constexpr int kBlockThreads = 256;
constexpr size_t kBlockSmem = sizeof(uint64_t) * 17 * kBlockThreads + (kBlockThreads / 32) * kWarpMsgBytes;

// everything a captured graph has baked in
struct BlockSig {
  TrieView tv;
  DirtyList dl;
  BlockBufs bb;
  void *h_desc;
  void *h_ctr;
  int grid, stage_grid;
};

}  // namespace

int Trie::block_launch(bool launch) {
  cudaError_t e = cudaSuccess;
  int sms = 0, occ = 0;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev_)) != cudaSuccess ||
      (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_block, kBlockThreads, kBlockSmem)) != cudaSuccess)
    return check_cuda(e, "block occupancy");
  const int max_grid = occ * sms;
  if (max_grid < 1) return fail(E_INTERNAL, "persistent kernel does not fit an SM");
  const int grid = opt_block_grid_ > 0 ? std::min(opt_block_grid_, max_grid) : max_grid;
  const int stage_grid = sms * 4;
  BlockSig sig;
  std::memset(&sig, 0, sizeof(sig));
  sig.tv = tv_;
  sig.tv.gen = 0;    // the kernels take the generation from the descriptor
  sig.tv.epoch = 0;  // (LockNU claims no split epochs)
  sig.dl = DirtyList{dirty_ref_, dirty_depth_};
  uint32_t *bins = blk_.bins.as<uint32_t>();
  sig.bb = BlockBufs{blk_.keys.as<uint8_t>(), blk_.kidx.as<int>(),      blk_.vals.as<uint8_t>(),
                     blk_.vidx.as<int64_t>(), blk_.tid.as<int>(),       blk_.ptrie.as<int>(),
                     blk_.poff.as<int>(),     blk_.out_ids.as<int>(),   blk_.out.as<uint8_t>(),
                     blk_.koff.as<uint64_t>(), blk_.klen.as<uint32_t>(), bins,
                     bins + 4 * (kDepthBins + 1), blk_.sorted.as<uint32_t>(),
                     static_cast<BlockDesc *>(blk_.d_desc)};
  sig.h_desc = blk_.h_desc;
  sig.h_ctr = h_ctr_;
  sig.grid = grid;
  sig.stage_grid = stage_grid;
  auto issue = [&]() -> cudaError_t {
    cudaError_t x = cudaMemcpyAsync(blk_.d_desc, blk_.h_desc, sizeof(BlockDesc), cudaMemcpyHostToDevice, st_);
    if (x != cudaSuccess) return x;
    count_launch(), k_block_stage<<<stage_grid, kBlockThreads, 0, st_>>>(sig.tv, sig.bb);
    if ((x = cudaGetLastError()) != cudaSuccess) return x;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(kBlockThreads);
    cfg.dynamicSmemBytes = kBlockSmem;
    cfg.stream = st_;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;  // all CTAs co-resident, or the launch fails
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    count_launch();
    if ((x = cudaLaunchKernelEx(&cfg, k_block, sig.tv, sig.dl, sig.bb, (uint32_t)(1u << 20))) != cudaSuccess) return x;
    if ((x = cudaMemcpyAsync(blk_.h_desc, blk_.d_desc, sizeof(BlockDesc), cudaMemcpyDeviceToHost, st_)) != cudaSuccess)
      return x;
    return cudaMemcpyAsync(h_ctr_, ctr_, sizeof(Counters), cudaMemcpyDeviceToHost, st_);
  };
  binfo_.grid = grid;
  if (!opt_block_graph_) {
    if (!launch) return OK;
    if ((e = issue()) != cudaSuccess) return check_cuda(e, "block launch");
    ++binfo_.launches;
    return OK;
  }
  const uint8_t *sb = reinterpret_cast<const uint8_t *>(&sig);
  BlockRt::Captured *hit = nullptr;
  for (auto &c : blk_.graphs)
    if (c.sig.size() == sizeof(sig) && std::memcmp(c.sig.data(), sb, sizeof(sig)) == 0) hit = &c;
  if (!hit) {
    constexpr size_t kKeep = 4;
    if (blk_.graphs.size() >= kKeep) {  // drop the least recently used capture
      auto lru = std::min_element(blk_.graphs.begin(), blk_.graphs.end(),
                                  [](const BlockRt::Captured &a, const BlockRt::Captured &b) { return a.used < b.used; });
      if (lru->exec) cudaGraphExecDestroy(lru->exec);
      if (lru->graph) cudaGraphDestroy(lru->graph);
      blk_.graphs.erase(lru);
    }
    BlockRt::Captured c;
    if ((e = cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
      return check_cuda(e, "block graph capture");
    cudaError_t ie = issue();
    e = cudaStreamEndCapture(st_, &c.graph);
    if (ie != cudaSuccess) {
      if (c.graph) cudaGraphDestroy(c.graph);
      return check_cuda(ie, "block graph capture");
    }
    if (e != cudaSuccess) return check_cuda(e, "block graph capture end");
    if ((e = cudaGraphInstantiate(&c.exec, c.graph, 0)) != cudaSuccess) {
      cudaGraphDestroy(c.graph);
      return check_cuda(e, "block graph instantiate");
    }
    c.sig.assign(sb, sb + sizeof(sig));
    blk_.graphs.push_back(std::move(c));
    hit = &blk_.graphs.back();
    ++binfo_.captures;
  }
  hit->used = ++blk_.tick;
  if (!launch) return OK;
  if ((e = cudaGraphLaunch(hit->exec, st_)) != cudaSuccess) return check_cuda(e, "block graph launch");
  count_launch();
  count_launch();
  ++binfo_.launches;
  return OK;
}

int Trie::block_update(const BlockIn &b, uint8_t *out32, int *sizes) {
  err_.clear();
  const int n = b.n;
  if (n < 0 || n > (1 << 26) || b.n0 < 0 || b.n0 > n || b.n_out < 0 || b.n_out > (1 << 26))
    return fail(E_ARG, "block sizes out of range");
  if (n > 0 && (!b.keys_hexs || !b.keys_indexs || !b.values || !b.values_indexs))
    return fail(E_ARG, "null block array");  // trie_ids may be null: every key in trie 0
  if ((b.patch_trie == nullptr) != (b.patch_off == nullptr)) return fail(E_ARG, "patch_trie and patch_off go together");
  if (b.n_out > 0 && (!b.out_ids || !out32 || !sizes)) return fail(E_ARG, "null output array");
  for (int i = 0; i < b.n_out; ++i)
    if (b.out_ids[i] < 0 || (uint32_t)b.out_ids[i] >= n_tries_) return fail(E_ARG, "trie id outside [0, max_tries)");
  cudaSetDevice(dev_);
  cudaEvent_t ev[4] = {};
  if (timing_) {
    for (auto &x : ev) cudaEventCreate(&x);
    cudaEventRecord(ev[0], st_);
  }
  struct EvGuard {
    cudaEvent_t *e;
    ~EvGuard() {
      for (int i = 0; i < 4; ++i)
        if (e[i]) cudaEventDestroy(e[i]);
    }
  } ev_guard{ev};
  int64_t kb = b.keys_bytes, vb = b.values_bytes;
  if (kb < 0 || vb < 0) {
    if (b.device) return fail(E_ARG, "device blocks need keys_bytes and values_bytes");
    kb = n ? (int64_t)b.keys_indexs[2 * n - 1] + 1 : 0;
    vb = n ? (int64_t)b.values_indexs[2 * n - 1] + 1 : 0;
  }
  if (kb < 0 || vb < 0 || kb > 0x7FFFFFFFll) return fail(E_ARG, "bad stream lengths");
  int rc = ensure_capacity((uint64_t)n, 3ull * n, (uint64_t)n, (uint64_t)n, (uint64_t)kb + 64, (uint64_t)vb + 80);
  if (rc) return rc;
  if ((rc = block_buffers(n, kb, vb, b.n_out))) return rc;
  cudaError_t e = cudaSuccess;
  const cudaMemcpyKind kind = b.device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  if (n > 0) {
    e = cudaMemcpyAsync(blk_.keys.p, b.keys_hexs, (size_t)kb, kind, st_);
    if (e == cudaSuccess) e = cudaMemcpyAsync(blk_.kidx.p, b.keys_indexs, 8 * (size_t)n, kind, st_);
    if (e == cudaSuccess && vb) e = cudaMemcpyAsync(blk_.vals.p, b.values, (size_t)vb, kind, st_);
    if (e == cudaSuccess) e = cudaMemcpyAsync(blk_.vidx.p, b.values_indexs, 16 * (size_t)n, kind, st_);
    if (e == cudaSuccess)
      e = b.trie_ids ? cudaMemcpyAsync(blk_.tid.p, b.trie_ids, 4 * (size_t)n, kind, st_)
                     : cudaMemsetAsync(blk_.tid.p, 0, 4 * (size_t)n, st_);
    if (b.patch_trie) {
      if (e == cudaSuccess) e = cudaMemcpyAsync(blk_.ptrie.p, b.patch_trie, 4 * (size_t)n, kind, st_);
      if (e == cudaSuccess) e = cudaMemcpyAsync(blk_.poff.p, b.patch_off, 4 * (size_t)n, kind, st_);
    } else if (e == cudaSuccess) {
      e = cudaMemsetAsync(blk_.ptrie.p, 0xFF, 4 * (size_t)n, st_);  // -1: no patch
    }
  }
  if (e == cudaSuccess && b.n_out > 0)
    e = cudaMemcpyAsync(blk_.out_ids.p, b.out_ids, 4 * (size_t)b.n_out, cudaMemcpyHostToDevice, st_);
  if (e != cudaSuccess) return check_cuda(e, "block inputs");
  BlockDesc *h = static_cast<BlockDesc *>(blk_.h_desc);
  std::memset(h, 0, sizeof(BlockDesc));
  const uint64_t val_base = (val_used_ + 7) & ~7ull;
  h->n = n;
  h->n0 = b.n0;
  h->n_out = b.n_out;
  h->kbytes = kb;
  h->vbytes = vb;
  h->key_base = key_used_;
  h->val_base = val_base;
  h->vid_base = n_rec_;
  h->gen = gen_;
  h->barrier_ns = opt_barrier_ns_;
  if (timing_) cudaEventRecord(ev[1], st_);
  if ((rc = block_launch())) return rc;
  if (timing_) cudaEventRecord(ev[2], st_);
  if ((e = cudaStreamSynchronize(st_)) != cudaSuccess) return check_cuda(e, "block");
  binfo_.levels[0] = h->levels[0];
  binfo_.levels[1] = h->levels[1];
  binfo_.dirty[0] = h->dirty[0];
  binfo_.dirty[1] = h->dirty[1];
  binfo_.n_ts = std::min<uint32_t>(h->n_ts, kBlockMaxTs);
  std::memcpy(binfo_.ts, h->ts, sizeof(uint64_t) * binfo_.n_ts);
  if (h->bad || h->noncontig || h->stream_terms != h->key_terms) {
    cudaMemsetAsync(&ctr_->error, 0, 4, st_);
    if (h->bad & BLOCK_BAD_TRIE) return fail(E_ARG, "trie id outside [0, max_tries)");
    if (h->bad & BLOCK_BAD_PATCH)
      return fail(E_ARG, "patch outside the value, of a stage-0 key, or naming a trie outside [0, max_tries)");
    if (h->bad & BLOCK_BAD_VALUE) return fail(E_ARG, "value index pair outside the value stream");
    if (h->noncontig) return fail(E_ARG, "block key index pairs must tile the key stream");
    return fail(E_BAD_KEY, "malformed key: nibble > 16, terminator not last, or too long");
  }
  // the launch got past staging: the arena bytes and records are in use
  key_used_ += ((uint64_t)kb + 7) & ~7ull;
  val_used_ = val_base + (uint64_t)vb;
  n_rec_ += (uint64_t)n;
  gen_ += 2;
  tv_.gen = gen_;
  if (n > 0) empty_ = false;
  stats_.key_bytes = key_used_;
  stats_.value_bytes = val_used_;
  stats_.n_records = n_rec_;
  if ((rc = apply_counters())) return rc;
  if (h->status & 1u) return fail(E_INTERNAL, "grid barrier wait gave up");
  stats_.n_full = n_full_;
  stats_.n_short = n_short_;
  stats_.n_value = n_value_;
  stats_.last_dirty = (uint64_t)h->dirty[0] + h->dirty[1];
  stats_.last_hash_levels = (uint64_t)h->levels[0] + h->levels[1];
  if (b.n_out > 0) {
    std::vector<uint8_t> o(33 * (size_t)b.n_out);
    if ((e = cudaMemcpyAsync(o.data(), blk_.out.p, o.size(), cudaMemcpyDeviceToHost, st_)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st_)) != cudaSuccess)
      return check_cuda(e, "block roots");
    for (int i = 0; i < b.n_out; ++i) {
      std::memcpy(out32 + 32 * (size_t)i, o.data() + 33 * (size_t)i, 32);
      sizes[i] = o[33 * (size_t)i + 32];
    }
  }
  if (timing_) {
    cudaEventRecord(ev[3], st_);
    cudaEventSynchronize(ev[3]);
    cudaEventElapsedTime(&binfo_.t_inputs_ms, ev[0], ev[1]);
    cudaEventElapsedTime(&binfo_.t_launch_ms, ev[1], ev[2]);
    cudaEventElapsedTime(&binfo_.t_total_ms, ev[0], ev[3]);
  }
  return OK;
}

// Block input / scratch buffers for a block of n keys (grown, never shrunk).
int Trie::block_buffers(int64_t n, int64_t kb, int64_t vb, int64_t n_out) {
  cudaError_t e = cudaSuccess;
  const size_t nn = (size_t)std::max<int64_t>(n, 1), no = (size_t)std::max<int64_t>(n_out, 1);
  if (e == cudaSuccess) e = blk_.keys.ensure((size_t)kb + 128);
  if (e == cudaSuccess) e = blk_.kidx.ensure(8 * nn);
  if (e == cudaSuccess) e = blk_.vals.ensure((size_t)vb + 128);
  if (e == cudaSuccess) e = blk_.vidx.ensure(16 * nn);
  if (e == cudaSuccess) e = blk_.tid.ensure(4 * nn);
  if (e == cudaSuccess) e = blk_.ptrie.ensure(4 * nn);
  if (e == cudaSuccess) e = blk_.poff.ensure(4 * nn);
  if (e == cudaSuccess) e = blk_.out_ids.ensure(4 * no);
  if (e == cudaSuccess) e = blk_.out.ensure(33 * no);
  if (e == cudaSuccess) e = blk_.koff.ensure(8 * nn);
  if (e == cudaSuccess) e = blk_.klen.ensure(4 * nn);
  if (e == cudaSuccess) e = blk_.bins.ensure(sizeof(uint32_t) * (5 * (kDepthBins + 1)));
  if (e == cudaSuccess) e = blk_.sorted.ensure(sizeof(uint32_t) * (cap_dirty_ + 64));
  if (e == cudaSuccess && !blk_.d_desc) e = cudaMalloc(&blk_.d_desc, sizeof(BlockDesc));
  if (e == cudaSuccess && !blk_.h_desc) e = cudaMallocHost(&blk_.h_desc, sizeof(BlockDesc));
  return check_cuda(e, "block buffers");
}

int Trie::reserve_block(int64_t max_keys, int64_t max_key_bytes, int64_t max_value_bytes, int64_t max_out) {
  err_.clear();
  if (max_keys < 0 || max_keys > (1 << 26) || max_key_bytes < 0 || max_value_bytes < 0 || max_out < 0)
    return fail(E_ARG, "reserve_block: bad sizes");
  cudaSetDevice(dev_);
  int rc = sync_counters();
  if (!rc) rc = ensure_capacity((uint64_t)max_keys, 3ull * max_keys, (uint64_t)max_keys, (uint64_t)max_keys,
                                (uint64_t)max_key_bytes + 64, (uint64_t)max_value_bytes + 80);
  if (!rc) rc = block_buffers(max_keys, max_key_bytes, max_value_bytes, max_out);
  if (!rc) rc = block_launch(false);
  return rc;
}

int Trie::reserve_nodes(uint64_t full, uint64_t shorts, uint64_t values, uint64_t records, uint64_t key_bytes,
                        uint64_t value_bytes) {
  err_.clear();
  cudaSetDevice(dev_);
  int rc = sync_counters();
  if (rc) return rc;
  return ensure_capacity(full, shorts, values, records, key_bytes + 64 * 8, value_bytes + 80 * 8, true);
}

int Trie::reserve(uint64_t n_keys, uint64_t key_bytes, uint64_t value_bytes) {
  err_.clear();
  if (n_keys > (1ull << 30)) return fail(E_ARG, "reserve: too many keys");
  cudaSetDevice(dev_);
  int rc = sync_counters();
  if (rc) return rc;
  // LockNU / block bound per key: one branch, three short nodes, one value
  return ensure_capacity(n_keys, 3 * n_keys, n_keys, n_keys, key_bytes + 64 * 8, value_bytes + 80 * 8, true);
}

}  // namespace gmpt

// ---------------------------------------------------------------------------
// Synthetic request batches generated on the device.

namespace gmpt {

namespace {

std::mutex g_gen_mu;
DevBlock g_gen_flags, g_gen_rank, g_gen_scan, g_gen_tot;

ZipfParams zipf_params(int64_t items, double theta) {
  ZipfParams z{};
  z.items = items;
  if (std::fabs(theta - 1.0) < 1e-3) theta = 0.999;  // Gray's constants are singular at 1
  z.theta = theta;
  if (items <= 0 || theta <= 0.0) return z;
  // zeta(items, theta): exact head, midpoint-integral tail
  const int64_t K = std::min<int64_t>(items, 100000);
  double zs = 0;
  for (int64_t i = 1; i <= K; ++i) zs += std::pow((double)i, -theta);
  if (items > K) {
    const double a = (double)K + 0.5, b = (double)items + 0.5;
    zs += (std::pow(b, 1.0 - theta) - std::pow(a, 1.0 - theta)) / (1.0 - theta);
  }
  z.zetan = zs;
  z.alpha = 1.0 / (1.0 - theta);
  z.half_pow = std::pow(0.5, theta);
  const double zeta2 = 1.0 + z.half_pow;
  z.eta = (1.0 - std::pow(2.0 / (double)items, 1.0 - theta)) / (1.0 - zeta2 / zs);
  return z;
}

}  // namespace

int gen_ids(uint64_t seed, int64_t n, int64_t n_existing, int64_t next_new, double p_new, double theta, int64_t *d_ids,
            int64_t *n_new, cudaStream_t st, std::string &err) {
  if (n < 0 || n > (1ll << 30) || n_existing < 0 || next_new < 0 || !d_ids || !n_new) {
    err = "gen_ids: bad arguments";
    return E_ARG;
  }
  *n_new = 0;
  if (n == 0) return OK;
  std::lock_guard<std::mutex> g(g_gen_mu);
  cudaError_t e = g_gen_flags.ensure(sizeof(uint32_t) * n + 64);
  if (e == cudaSuccess) e = g_gen_rank.ensure(sizeof(unsigned long long) * 2 * n + 64);
  if (e == cudaSuccess) e = g_gen_scan.ensure(scan_ws_bytes<unsigned long long>(n));
  if (e == cudaSuccess) e = g_gen_tot.ensure(64);
  if (e != cudaSuccess) {
    err = std::string("gen_ids: ") + cudaGetErrorString(e);
    return E_CUDA;
  }
  const ZipfParams z = zipf_params(n_existing, theta);
  uint32_t *flags = g_gen_flags.as<uint32_t>();
  unsigned long long *f64 = g_gen_rank.as<unsigned long long>(), *rank = f64 + n;
  count_launch(), k_gen_ids<<<blocks_for(n), kThreads, 0, st>>>(seed, n, p_new, z, d_ids, flags);
  count_launch(), k_gen_widen<<<blocks_for(n), kThreads, 0, st>>>(flags, n, f64);
  unsigned long long *tot = g_gen_tot.as<unsigned long long>();
  e = exclusive_scan<unsigned long long>(f64, rank, n, tot, g_gen_scan, st);
  if (e == cudaSuccess) count_launch(), k_gen_new_ids<<<blocks_for(n), kThreads, 0, st>>>(flags, rank, n, next_new, d_ids);
  unsigned long long h = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, tot, 8, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    err = std::string("gen_ids: ") + cudaGetErrorString(e);
    return E_CUDA;
  }
  *n_new = (int64_t)(h & 0xFFFFFFFFull);
  return OK;
}

int gen_keys(uint64_t seed, const int64_t *d_ids, int64_t n, int key_bytes, uint8_t *d_hexs, int *d_idx, cudaStream_t st,
             std::string &err) {
  if (n < 0 || key_bytes < 1 || key_bytes > kMaxKeyNibbles / 2 || (n > 0 && (!d_ids || !d_hexs || !d_idx)) ||
      n * (2 * (int64_t)key_bytes + 1) >= (1ll << 31)) {
    err = "gen_keys: bad arguments";
    return E_ARG;
  }
  if (n == 0) return OK;
  count_launch(), k_gen_keys<<<blocks_for(n), kThreads, 0, st>>>(seed, d_ids, n, key_bytes, d_hexs, d_idx);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    err = std::string("gen_keys: ") + cudaGetErrorString(e);
    return E_CUDA;
  }
  return OK;
}

int gen_values(uint64_t seed, int64_t n, int value_bytes, uint8_t *d_vals, int64_t *d_idx, cudaStream_t st,
               std::string &err) {
  if (n < 0 || value_bytes < 1 || (n > 0 && (!d_vals || !d_idx))) {
    err = "gen_values: bad arguments";
    return E_ARG;
  }
  if (n == 0) return OK;
  count_launch(), k_gen_values<<<blocks_for(n), kThreads, 0, st>>>(seed, n, value_bytes, d_vals, d_idx);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    err = std::string("gen_values: ") + cudaGetErrorString(e);
    return E_CUDA;
  }
  return OK;
}

}  // namespace gmpt

namespace gmpt {

namespace {
static __device__ float g_feat_out[4 * 64];
std::mutex g_feat_mu;
float *g_feat_ptr[64] = {};
}  // namespace

// Sampled key features of a device-resident batch (k_sample_features); no
// allocation per call: a small static device array per device.
int batch_features_device(const uint8_t *d_keys, const int *d_kidx, int n, int64_t keys_bytes, float out[4],
                          cudaStream_t st, std::string &err) {
  if (n <= 0 || keys_bytes <= 0 || !d_keys || !d_kidx || !out) {
    err = "batch_features: bad arguments";
    return E_ARG;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    err = "batch_features: no usable device";
    return E_CUDA;
  }
  std::lock_guard<std::mutex> g(g_feat_mu);
  if (!g_feat_ptr[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_feat_out) != cudaSuccess) {
      err = "batch_features: symbol address";
      return E_CUDA;
    }
    g_feat_ptr[dev] = static_cast<float *>(p);
  }
  count_launch(), k_sample_features<<<1, 64, 0, st>>>(d_keys, d_kidx, n, keys_bytes, g_feat_ptr[dev]);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, g_feat_ptr[dev], 16, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    err = std::string("batch_features: ") + cudaGetErrorString(e);
    return E_CUDA;
  }
  return OK;
}

}  // namespace gmpt

// ---------------------------------------------------------------------------
// Host batches with the copy of the next batch overlapping this one's work
// (the reference's two-stream puts_2phase_pipeline / puts_latching_pipeline_v2,
// gpu_mpt.cuh:1715-1823 and 926-982).

namespace gmpt {

int Trie::del(const uint8_t *keys_hexs, const int *keys_indexs, int n, bool device_inputs, int64_t keys_bytes,
              const int *trie_ids) {
  err_.clear();
  if (n < 0 || n > (1 << 26)) return fail(E_ARG, "batch size must be in [0, 2^26]");
  if (n == 0) return OK;
  if (!keys_hexs || !keys_indexs) return fail(E_ARG, "null batch array");
  cudaSetDevice(dev_);
  cudaError_t e = cudaSuccess;
  if (keys_bytes < 0) {
    if (device_inputs) return fail(E_ARG, "device deletes need keys_bytes");
    keys_bytes = (int64_t)keys_indexs[2 * n - 1] + 1;
  }
  if (keys_bytes < 0) return fail(E_ARG, "bad index pairs");
  int rc = sync_counters();
  if (rc) return rc;
  const cudaMemcpyKind kind = device_inputs ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  uint8_t *dk = wsp<uint8_t>(ws_.g_keys, (size_t)keys_bytes + 64, e);
  int *di = wsp<int>(ws_.g_idx, 2 * (size_t)n, e);
  int *dtid = trie_ids ? wsp<int>(ws_.g_tid, (size_t)n, e) : nullptr;
  const size_t nf = (size_t)n_full_ + 1;
  uint64_t *hslot = wsp<uint64_t>(ws_.del_hslot, nf, e);
  uint32_t *hext = wsp<uint32_t>(ws_.del_hext, nf, e);
  uint8_t *stamp = wsp<uint8_t>(ws_.del_stamp, nf, e);
  unsigned long long *dcnt = wsp<unsigned long long>(ws_.rw_tot, 8, e);  // [0] need, [1] key cursor
  if (e == cudaSuccess) e = cudaMemcpyAsync(dk, keys_hexs, (size_t)keys_bytes, kind, st_);
  if (e == cudaSuccess) e = cudaMemsetAsync(dk + keys_bytes, 0, 64, st_);
  if (e == cudaSuccess) e = cudaMemcpyAsync(di, keys_indexs, sizeof(int) * 2 * (size_t)n, kind, st_);
  if (e == cudaSuccess && dtid) e = cudaMemcpyAsync(dtid, trie_ids, sizeof(int) * (size_t)n, kind, st_);
  if (e == cudaSuccess) e = cudaMemsetAsync(stamp, 0, nf, st_);
  if (e != cudaSuccess) return check_cuda(e, "delete copy");
  DirtyList dl{dirty_ref_, dirty_depth_};
  count_launch(), k_del_walk<<<blocks_for(n), kThreads, 0, st_>>>(tv_, dl, dk, di, n, keys_bytes, dtid, hslot, hext,
                                                                  stamp);
  if ((rc = sync_counters())) return rc;
  const uint32_t nd = h_ctr_->n_dirty;
  if (nd == 0) return OK;
  uint32_t *sorted = nullptr;
  std::vector<uint32_t> off;
  if ((rc = bucket_dirty(nd, &sorted, off))) return rc;
  for (int d = (int)kMaxDepths - 1; d >= 0; --d) {
    const uint32_t a = off[level_bin(d) + 1], z = off[level_bin(d + 1)];  // branches at depth d
    if (z == a) continue;
    const int cnt = (int)(z - a);
    // room for this level's new keys and short nodes, then collapse
    if ((e = cudaMemsetAsync(dcnt, 0, 8, st_)) != cudaSuccess) return check_cuda(e, "delete need");
    count_launch(), k_del_need<<<blocks_for(cnt), kThreads, 0, st_>>>(tv_, sorted + a, cnt, hext, stamp, dcnt);
    if ((e = cudaMemcpyAsync(h_small_, dcnt, 8, cudaMemcpyDeviceToHost, st_)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st_)) != cudaSuccess)
      return check_cuda(e, "delete need");
    const uint64_t need = h_small_[0];
    if ((rc = sync_counters())) return rc;
    if ((rc = ensure_capacity(0, (uint64_t)cnt, 0, 0, need + 64, 0))) return rc;
    dl = DirtyList{dirty_ref_, dirty_depth_};  // the list may have grown with the short pool
    h_small_[1] = key_used_;
    if ((e = cudaMemcpyAsync(dcnt + 1, h_small_ + 1, 8, cudaMemcpyHostToDevice, st_)) != cudaSuccess)
      return check_cuda(e, "delete cursor");
    count_launch(), k_del_collapse<<<blocks_for(cnt), kThreads, 0, st_>>>(tv_, dl, sorted + a, cnt, hslot, hext, stamp,
                                                                          dcnt + 1, cap_keys_);
    if ((e = cudaMemcpyAsync(h_small_, dcnt + 1, 8, cudaMemcpyDeviceToHost, st_)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st_)) != cudaSuccess)
      return check_cuda(e, "delete collapse");
    const uint64_t cursor = h_small_[0];
    // k_del_collapse advances the cursor even when a level's key bytes did
    // not fit (it then raises ERR_CAPACITY): check before the arena is touched
    if ((rc = sync_counters())) return rc;
    if (cursor + 64 > cap_keys_) return fail(E_CAPACITY, "key arena capacity exceeded by a delete collapse");
    key_used_ = (cursor + 7) & ~7ull;
    if ((e = cudaMemsetAsync(const_cast<uint8_t *>(tv_.keys) + cursor, 0, 64, st_)) != cudaSuccess)
      return check_cuda(e, "delete tail");
  }
  if ((rc = sync_counters())) return rc;
  stats_.key_bytes = key_used_;
  stats_.n_full = n_full_;
  stats_.n_short = n_short_;
  return OK;
}

int Trie::put_rw(const BatchIn &b, const uint8_t *rw, bool two_phase, uint64_t *read_hps, int *read_sizes,
                 int *read_num) {
  err_.clear();
  if (b.n < 0 || b.n > (1 << 26)) return fail(E_ARG, "batch size must be in [0, 2^26]");
  if (read_num) *read_num = 0;
  if (b.n == 0) return OK;
  if (!rw || !read_hps || !read_sizes || !read_num) return fail(E_ARG, "null argument");
  cudaSetDevice(dev_);
  cudaError_t e = cudaSuccess;
  const size_t n = (size_t)b.n;
  RwState st;
  st.key_order = two_phase;
  st.flags = wsp<uint8_t>(ws_.rw_flags, n, e);
  st.hp = b.device ? read_hps : wsp<uint64_t>(ws_.rw_hp, n, e);
  st.len = b.device ? read_sizes : wsp<int>(ws_.rw_len, n, e);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(const_cast<uint8_t *>(st.flags), rw, n,
                        b.device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st_);
  if (e != cudaSuccess) return check_cuda(e, "rw flags");
  rw_ = &st;
  int rc = two_phase ? put_2phase(b) : put_latching(b);
  rw_ = nullptr;
  if (rc) return rc;
  *read_num = (int)st.reads;
  if (!b.device && st.reads) {
    e = cudaMemcpyAsync(read_hps, st.hp, 8 * st.reads, cudaMemcpyDeviceToHost, st_);
    if (e == cudaSuccess) e = cudaMemcpyAsync(read_sizes, st.len, 4 * st.reads, cudaMemcpyDeviceToHost, st_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st_);
    if (e != cudaSuccess) return check_cuda(e, "rw results");
  }
  return OK;
}

int Trie::puts_pipeline(const BatchIn *bs, const int *two_phase, int count, uint8_t *roots32, int *sizes) {
  err_.clear();
  if (count < 0 || (count > 0 && (!bs || !two_phase || !roots32 || !sizes))) return fail(E_ARG, "null argument");
  if (count == 0) return OK;
  cudaSetDevice(dev_);
  std::vector<int64_t> kb(count), vb(count);
  int64_t mk = 0, mv = 0;
  int mn = 0;
  for (int i = 0; i < count; ++i) {
    const BatchIn &b = bs[i];
    if (b.device) return fail(E_ARG, "puts_pipeline takes host batches");
    if (b.n < 0 || b.n > (1 << 26)) return fail(E_ARG, "batch size must be in [0, 2^26]");
    if (b.n > 0 && (!b.keys_hexs || !b.keys_indexs || !b.values || !b.values_indexs))
      return fail(E_ARG, "null batch array");
    kb[i] = b.n ? (int64_t)b.keys_indexs[2 * b.n - 1] + 1 : 0;
    vb[i] = b.n ? (int64_t)b.values_indexs[2 * b.n - 1] + 1 : 0;
    if (kb[i] < 0 || vb[i] < 0) return fail(E_ARG, "bad index pairs");
    mk = std::max(mk, kb[i]);
    mv = std::max(mv, vb[i]);
    mn = std::max(mn, b.n);
  }
  cudaError_t e = cudaSuccess;
  if (!copy_st_) e = cudaStreamCreateWithFlags(&copy_st_, cudaStreamNonBlocking);
  for (auto &ps : pipe_) {  // size both slots for the largest batch up front
    if (e == cudaSuccess && !ps.ready) e = cudaEventCreateWithFlags(&ps.ready, cudaEventDisableTiming);
    if (e == cudaSuccess && !ps.free) e = cudaEventCreateWithFlags(&ps.free, cudaEventDisableTiming);
    if (e == cudaSuccess) e = ps.keys.ensure((size_t)mk + 64);
    if (e == cudaSuccess) e = ps.kidx.ensure(8 * (size_t)std::max(mn, 1));
    if (e == cudaSuccess) e = ps.vals.ensure((size_t)mv + 64);
    if (e == cudaSuccess) e = ps.vidx.ensure(16 * (size_t)std::max(mn, 1));
    if (e == cudaSuccess) e = ps.hp.ensure(8 * (size_t)std::max(mn, 1));
    if (e == cudaSuccess) e = ps.tid.ensure(4 * (size_t)std::max(mn, 1));
    if (e == cudaSuccess) e = cudaEventRecord(ps.free, copy_st_);
  }
  if (e != cudaSuccess) return check_cuda(e, "pipeline buffers");
  auto issue = [&](int i) -> cudaError_t {
    const BatchIn &b = bs[i];
    PipeSlot &ps = pipe_[i & 1];
    cudaError_t x = cudaStreamWaitEvent(copy_st_, ps.free, 0);  // its previous batch is staged
    if (x == cudaSuccess && kb[i]) x = cudaMemcpyAsync(ps.keys.p, b.keys_hexs, (size_t)kb[i], cudaMemcpyHostToDevice, copy_st_);
    if (x == cudaSuccess && b.n) x = cudaMemcpyAsync(ps.kidx.p, b.keys_indexs, 8 * (size_t)b.n, cudaMemcpyHostToDevice, copy_st_);
    if (x == cudaSuccess && vb[i]) x = cudaMemcpyAsync(ps.vals.p, b.values, (size_t)vb[i], cudaMemcpyHostToDevice, copy_st_);
    if (x == cudaSuccess && b.n)
      x = cudaMemcpyAsync(ps.vidx.p, b.values_indexs, 16 * (size_t)b.n, cudaMemcpyHostToDevice, copy_st_);
    if (x == cudaSuccess && b.n && b.values_hps)
      x = cudaMemcpyAsync(ps.hp.p, b.values_hps, 8 * (size_t)b.n, cudaMemcpyHostToDevice, copy_st_);
    if (x == cudaSuccess && b.n && b.trie_ids)
      x = cudaMemcpyAsync(ps.tid.p, b.trie_ids, 4 * (size_t)b.n, cudaMemcpyHostToDevice, copy_st_);
    if (x == cudaSuccess) x = cudaEventRecord(ps.ready, copy_st_);
    return x;
  };
  int rc = OK;
  if ((e = issue(0)) != cudaSuccess) return check_cuda(e, "pipeline copy");
  for (int i = 0; i < count && rc == OK; ++i) {
    if (i + 1 < count && (e = issue(i + 1)) != cudaSuccess) {
      rc = check_cuda(e, "pipeline copy");
      break;
    }
    PipeSlot &ps = pipe_[i & 1];
    if ((e = cudaStreamWaitEvent(st_, ps.ready, 0)) != cudaSuccess) {
      rc = check_cuda(e, "pipeline wait");
      break;
    }
    const BatchIn &h = bs[i];
    BatchIn d;
    d.keys_hexs = ps.keys.as<uint8_t>();
    d.keys_indexs = ps.kidx.as<int>();
    d.values = ps.vals.as<uint8_t>();
    d.values_indexs = ps.vidx.as<int64_t>();
    d.values_hps = h.values_hps ? ps.hp.as<uint64_t>() : nullptr;
    d.trie_ids = h.trie_ids ? ps.tid.as<int>() : nullptr;
    d.n = h.n;
    d.keys_bytes = kb[i];
    d.values_bytes = vb[i];
    d.device = true;
    d.raw_keys = h.raw_keys;
    rc = two_phase[i] ? put_2phase(d) : put_latching(d);
    // the put has copied the slot into the arenas (it synchronises its stream)
    if ((e = cudaEventRecord(ps.free, st_)) != cudaSuccess && rc == OK) rc = check_cuda(e, "pipeline event");
    if (rc == OK) rc = hash();
    if (rc == OK) rc = root(roots32 + 32 * (size_t)i, sizes + i);
  }
  cudaStreamSynchronize(copy_st_);
  return rc;
}

}  // namespace gmpt
