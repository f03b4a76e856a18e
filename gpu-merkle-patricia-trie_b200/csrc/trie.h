// trie.h -- host side of the B200 MPT: one device-resident trie per object.
//
// Mirrors GpuMPT::Compress::MPT (mpt-with-compress/include/mpt/gpu_mpt.cuh:18-192):
//   put_2phase   <- puts_2phase_with_valuehp        (gpu_mpt.cuh:1262-1399)
//   put_latching <- puts_latching_with_valuehp_v2   (gpu_mpt.cuh:554-615)
//   hash         <- hash_onepass_v2                 (gpu_mpt.cuh:1162-1191)
//   gets         <- gets_parallel                   (gpu_mpt.cuh:984-1036)
//   root         <- get_root_hash                   (gpu_mpt.cuh:1217-1247)
// Differences that are deliberate: the trie owns copies of key and value
// bytes (the reference keeps pointers into per-call buffers it never frees),
// errors come back as status codes instead of exit(), duplicate keys in a
// batch resolve to the last occurrence (the reference CPU semantics) in both
// insert strategies, and an update to an existing key replaces its value in
// both strategies.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "common.cuh"
#include "prims.cuh"

namespace gmpt {

struct BatchIn {
  const uint8_t *keys_hexs = nullptr;    // nibble bytes
  const int *keys_indexs = nullptr;      // [2n] inclusive
  const uint8_t *values = nullptr;
  const int64_t *values_indexs = nullptr;  // [2n] inclusive
  const uint64_t *values_hps = nullptr;  // [n] caller host pointers, may be null
  const int *trie_ids = nullptr;         // [n] trie of each key (forest), null = trie 0
  int n = 0;
  int64_t keys_bytes = -1;    // total key stream bytes (derived if < 0, host only)
  int64_t values_bytes = -1;  // total value stream bytes
  bool device = false;        // pointers are device memory
  bool raw_keys = false;      // keys_hexs holds raw key bytes, keys_indexs byte ranges
                              // (expanded to nibbles + terminator on the device)
};

// One persistent two-stage update of a forest (Trie::block_update): keys
// [0, n0) are stage 0, keys [n0, n) stage 1; stage 1 runs after stage 0 is
// hashed, and key i of stage 1 with patch_trie[i] >= 0 first gets the 32
// root bytes of that trie (zero-padded below 32) written into its value at
// byte patch_off[i].  Index pairs must tile the key and value streams.
struct BlockIn {
  const uint8_t *keys_hexs = nullptr;
  const int *keys_indexs = nullptr;
  const uint8_t *values = nullptr;
  const int64_t *values_indexs = nullptr;
  const int *trie_ids = nullptr;    // [n]
  const int *patch_trie = nullptr;  // [n] or null (no patches)
  const int *patch_off = nullptr;   // [n] or null
  int n = 0, n0 = 0;
  const int *out_ids = nullptr;     // host array [n_out]: tries whose roots are returned
  int n_out = 0;
  int64_t keys_bytes = -1, values_bytes = -1;  // required for device inputs
  bool device = false;              // key/value/trie/patch arrays are device memory
};

struct TrieStats {
  uint64_t n_full, n_short, n_value, n_records;
  uint64_t key_bytes, value_bytes;
  uint64_t last_unique, last_new, last_pseudo, last_dirty, last_levels, last_hash_levels;
  uint64_t device_bytes;
  uint32_t sort_passes, build_levels;
  float t_stage_ms, t_sort_ms, t_walk_ms, t_build_ms, t_hash_ms;
  uint64_t last_hashed, last_enc_bytes, last_keccak_blocks;  // last hash pass
  float t_hash_kernels_ms;  // hash-level kernels only (timing mode)
  uint32_t hash_launches, pad;
};

enum Status : int {
  OK = 0,
  E_CUDA = 1,
  E_BAD_KEY = 2,
  E_CAPACITY = 3,
  E_RETRY_LIMIT = 4,
  E_ARG = 5,
  E_INTERNAL = 6,
};

class Trie {
 public:
  // max_tries > 1 makes a forest: independent tries sharing the node pools
  // and arenas, addressed by trie id 0..max_tries-1
  // unified: node pools, arenas and the dirty list in unified memory
  Trie(int device, int geth_mode, int max_tries = 1, bool unified = false);
  ~Trie();
  Trie(const Trie &) = delete;
  Trie &operator=(const Trie &) = delete;

  int put_2phase(const BatchIn &b);
  int put_latching(const BatchIn &b);
  // Mixed read/write batch: rw[i] = 0 reads key i, 1 writes it (rw host or
  // device as b.device).  Applied as if in index order: a read sees the last
  // earlier write of its key in the batch, else the trie before the batch.
  // Read i's result lands at its rank among the reads: read_hps / read_sizes
  // (host arrays, or device arrays when b.device), *read_num = reads.
  int put_rw(const BatchIn &b, const uint8_t *rw, bool two_phase, uint64_t *read_hps, int *read_sizes,
             int *read_num);
  // Delete keys (hex keys, as gets; trie ids or null for trie 0; device or
  // host arrays).  Absent keys are ignored.  The trie becomes the canonical
  // trie of the remaining keys after hash().
  int del(const uint8_t *keys_hexs, const int *keys_indexs, int n, bool device_inputs, int64_t keys_bytes = -1,
          const int *trie_ids = nullptr);
  int hash();
  int root(uint8_t out[32], int *len, int trie = 0);
  // roots of tries ids[0..n) (host array; null = tries 0..n-1): out32[32 i..]
  // zero-padded, sizes[i] = length (0 = empty trie)
  int roots(const int *ids, int n, uint8_t *out32, int *sizes);
  // out_hp[i] = host pointer given with the value (0 when absent), out_len[i] its size
  // (device_outputs: out_hp / out_len are device arrays, written by the kernel)
  int gets(const uint8_t *keys_hexs, const int *keys_indexs, int n, bool device_inputs,
           uint64_t *out_hp, int *out_len, int64_t keys_bytes = -1, const int *trie_ids = nullptr,
           bool device_outputs = false);
  // value bytes of the stored value for each key (test/export helper)
  int get_values(const uint8_t *keys_hexs, const int *keys_indexs, int n, std::vector<uint8_t> &vals,
                 std::vector<int64_t> &offs);
  int reset();
  // dirty node refs pending for hash (device array) and their count
  const uint32_t *pending_dirty(int *n) const;
  int flush_nodes(const uint8_t *keys_hexs, const int *keys_indexs, int n, std::vector<uint8_t> &hashs,
                  std::vector<uint8_t> &encs, std::vector<unsigned long long> &encs_indexs);
  // (hash, encoding) of every node hashed since the last flush_dirty that is
  // still in a trie and referenced by hash (encoding >= 32 bytes, or a root),
  // in its current state, ordered by node reference; needs the "track_dirty"
  // option (set before the puts).  Clears the record.
  int flush_dirty(std::vector<uint8_t> &hashs, std::vector<uint8_t> &encs,
                  std::vector<unsigned long long> &encs_indexs);
  const TrieStats &stats() const { return stats_; }
  const std::string &error() const { return err_; }
  cudaStream_t stream() const { return st_; }
  int device() const { return dev_; }
  int max_tries() const { return (int)n_tries_; }
  bool unified() const { return managed_; }
  // value nodes in the pools (the keys stored, deleted ones included)
  uint64_t value_nodes() const { return n_value_; }
  void set_timing(bool on) { timing_ = on; }
  // tuning knobs (names: "local_build", "local_sort", "latch_ways", "latch_dedup", "block_grid",
  // "block_graph", "warp_full_max", "local_build_cap", "local_sort_cap", "retry_limit", ...)
  int set_option(const std::string &name, int64_t value);
  // persistent graph-replayed forest update; out32[32 i..] / sizes[i] = root
  // of trie out_ids[i] after the update
  int block_update(const BlockIn &b, uint8_t *out32, int *sizes);
  // the last block launch: stage levels / dirty counts, CTAs, graph rebuilds
  struct BlockInfo {
    uint32_t levels[2], dirty[2];
    int grid;
    uint32_t captures, launches;
    float t_inputs_ms, t_launch_ms, t_total_ms;  // timing mode: input copies, graph, whole call
    uint32_t n_ts;
    uint64_t ts[64];  // device timeline of the last block (ns): stage start, k_block start, each barrier, end
  };
  // grow the pools and arenas now for n_keys more keys of the given byte
  // totals (no growth stalls, and no block graph rebuild, until then)
  int reserve(uint64_t n_keys, uint64_t key_bytes, uint64_t value_bytes);
  // Host batches applied in order, each followed by PhaseHC and a root read
  // (roots32[32 i..], sizes[i]); batch i+1 is copied to the device on a copy
  // stream while batch i is inserted and hashed.  two_phase[i] picks PhaseNU.
  int puts_pipeline(const BatchIn *batches, const int *two_phase, int count, uint8_t *roots32, int *sizes);
  // the same with explicit headroom per pool
  int reserve_nodes(uint64_t full, uint64_t shorts, uint64_t values, uint64_t records, uint64_t key_bytes,
                    uint64_t value_bytes);
  // size the block buffers for blocks up to these sizes and capture the
  // block graph now (so the first blocks do not pay for it)
  int reserve_block(int64_t max_keys, int64_t max_key_bytes, int64_t max_value_bytes, int64_t max_out);
  const BlockInfo &block_info() const { return binfo_; }

 private:
  int dev_ = 0;
  int geth_ = 0;
  bool managed_ = false;
  cudaStream_t st_ = nullptr;
  std::string err_;
  TrieStats stats_{};
  bool timing_ = false;
  bool opt_local_build_ = true;  // finish small build segments in one CTA each
  bool opt_local_sort_ = true;   // finish small tied sort runs in one CTA each
  int opt_latch_ways_ = 4;       // LockNU keys per thread (1, 2, 4)
  int opt_latch_dedup_ = 1;      // 0 off, 1 batches >= kDedupMinKeys, 2 always
  int opt_sort_dedup_ = 1;       // PhaseNU drops repeats first: 0 never, 1 when a sample shows them, 2 always
  int opt_dedup_bits_ = 64;      // hash bits the dedup keeps (fewer only to test collisions)
  int opt_warp_full_max_ = 4096; // hash levels with at most this many branches: a warp per branch
  int opt_local_build_cap_ = 0;  // largest segment finished in one CTA (0 = the kernel's capacity)
  int opt_local_sort_cap_ = 0;   // largest tied run finished in one CTA (0 = the kernel's capacity)
  uint32_t opt_retry_limit_ = 1u << 20;  // failed CASes per LockNU key before GMPT_E_RETRY_LIMIT
  uint64_t opt_barrier_ns_ = 2000000000ull;  // persistent kernel: longest grid-barrier wait
  uint32_t opt_max_full_ = 0;    // branch pool cap (0 = none)

  // node pools (capacities in elements)
  TrieView tv_{};
  uint32_t cap_full_ = 0, cap_short_ = 0, cap_value_ = 0;
  uint64_t cap_rec_ = 0;
  uint64_t cap_keys_ = 0, cap_vals_ = 0;
  uint32_t n_full_ = 0, n_short_ = 0, n_value_ = 0;
  uint64_t n_rec_ = 0, key_used_ = 0, val_used_ = 0;
  // longest key (nibbles) and value (bytes) staged since the last reset:
  // whether the hash pass orders leaves by Keccak block count
  uint32_t max_key_nibbles_ = 0, max_value_len_ = 0;
  uint32_t *roots_ = nullptr;  // [n_tries_] root words
  uint32_t n_tries_ = 1;
  Counters *ctr_ = nullptr;
  Counters *h_ctr_ = nullptr;  // pinned mirror
  uint32_t epoch_ = 0;         // per put batch (split claims)
  uint32_t gen_ = 1;           // per hash pass (dirty marks)
  bool empty_ = true;

  // nodes hashed since the last flush_dirty (when tracking is on)
  bool track_dirty_ = false;
  uint32_t *fl_refs_ = nullptr;
  uint64_t fl_n_ = 0, fl_cap_ = 0;

  // dirty list pending for hash()
  uint32_t *dirty_ref_ = nullptr;
  uint16_t *dirty_depth_ = nullptr;
  uint64_t cap_dirty_ = 0;

  // persistent block launches
  struct BlockRt {
    DevBlock keys, kidx, vals, vidx, tid, ptrie, poff, out_ids, out, koff, klen, bins, sorted;
    void *d_desc = nullptr, *h_desc = nullptr;  // BlockDesc (device / pinned)
    struct Captured {
      std::vector<uint8_t> sig;  // launch arguments the graph was captured with
      cudaGraph_t graph = nullptr;
      cudaGraphExec_t exec = nullptr;
      uint64_t used = 0;
    };
    std::vector<Captured> graphs;  // a few recent captures (e.g. one per grid size)
    uint64_t tick = 0;
  } blk_;
  BlockInfo binfo_{};
  int opt_block_grid_ = 0;      // CTAs of the persistent kernel (0 = all that fit co-resident)
  bool opt_block_graph_ = true;  // replay a captured graph (else plain launches)
  int block_launch(bool launch = true);
  int block_buffers(int64_t n, int64_t kb, int64_t vb, int64_t n_out);

  // double-buffered host -> device staging of puts_pipeline
  struct PipeSlot {
    DevBlock keys, kidx, vals, vidx, hp, tid;
    cudaEvent_t ready = nullptr, free = nullptr;
  } pipe_[2];
  cudaStream_t copy_st_ = nullptr;

  // per-batch workspaces
  struct Ws {
    DevBlock koff, klen, ki, vi, hp, kin;          // staged batch
    DevBlock order, eqprev, flags, pos, act, skey, sval, uord;  // sort / dedup
    DevBlock w_status, w_code, w_d0, w_slot, w_short, w_after;  // walk
    DevBlock p_short, p_d0, p_slot, p_amin, p_max;              // pseudo items
    DevBlock it_key, it_id, it_base, it_len, it_ref, it_d0, it_slot;  // items
    DevBlock sb_base, sb_len, sb_ref, sb_d0, sb_slot, sb_code, lcp;   // sorted items
    DevBlock act2, aseg, aseg2, kflags, knib;                   // builder levels
    DevBlock s_start[2], s_end[2], s_depth[2], s_slot[2], s_D[2], s_branch[2];
    DevBlock bins, cursor, sorted_dirty;                        // hash buckets
    DevBlock g_keys, g_idx, g_hp, g_len, g_tid;                 // gets
    DevBlock tid;                                               // trie ids of the batch
    DevBlock dd_hash, dd_pos, dd_sel, dd_slot;                  // LockNU batch dedup
    DevBlock raw;                                               // raw key bytes of the batch
    DevBlock dirty_cls;                                         // hash class of each dirty node
    DevBlock rw_flags, rw_a, rw_b, rw_c, rw_d, rw_e, rw_wpos;   // mixed read/write resolution
    DevBlock rw_hp, rw_len, rw_tot, rw_kept, rw_koff, rw_klen, rw_tid;
    DevBlock del_hslot, del_hext, del_stamp;                    // deletes: how each path branch is linked
    DevBlock misc;
  } ws_;
  RadixSorter sorter_;
  DevBlock scan_ws_;
  uint64_t *h_small_ = nullptr;  // pinned scratch for small readbacks
  // set by put_rw for the duration of one put: sort_unique then resolves the
  // reads and keeps the last write of every key
  struct RwState {
    const uint8_t *flags = nullptr;  // device, batch order
    uint64_t *hp = nullptr;          // device, read rank order
    int *len = nullptr;
    uint64_t vid_base = 0;
    bool key_order = false;          // kept writes in key order (PhaseNU)
    uint64_t reads = 0;              // out
  };
  RwState *rw_ = nullptr;

  int fail(int code, const std::string &msg);
  int check_cuda(cudaError_t e, const char *what);
  int sync_counters();
  int apply_counters();
  // exact: grow to exactly what is asked (reservations) instead of by 1.5x steps
  int ensure_capacity(uint64_t add_full, uint64_t add_short, uint64_t add_value, uint64_t add_rec,
                      uint64_t add_key_bytes, uint64_t add_val_bytes, bool exact = false);
  int stage(const BatchIn &b, uint64_t &key_base, uint64_t &vid_base, uint64_t **koff, uint32_t **klen,
            uint32_t *maxlen, const int **tid);
  int bucket_dirty(uint32_t nd, uint32_t **sorted_out, std::vector<uint32_t> &off);
  int sort_unique_dedup(int n, const uint64_t *koff, const uint32_t *klen, uint32_t maxlen, const int *tid,
                        uint32_t **uord_out, int *m_out, bool *done);
  int sort_batch(int n, const uint64_t *koff, const uint32_t *klen, uint32_t maxlen, const int *tid,
                 uint32_t **order_out, uint8_t **eqprev_out);
  int sort_rw(int n, const uint64_t *koff, const uint32_t *klen, uint32_t maxlen, const int *tid, uint32_t **uord_out,
              int *m_out);
  int resolve_rw(int n, const uint32_t *order, const uint8_t *eqprev, const uint64_t *koff, const uint32_t *klen,
                 const int *tid, uint32_t **uord_out, int *m_out);
  int sort_unique(int n, const uint64_t *koff, const uint32_t *klen, uint32_t maxlen, const int *tid,
                  uint32_t **uord, int *m);
  int build_levels(int T);
  // mixed batch: keep only the m kept writes' key bytes in the arena
  int compact_rw_keys(int m, const uint32_t *kept, uint64_t *koff, const uint32_t *klen, uint64_t key_base);
  int bucket_and_hash();
  uint64_t read_u64(const void *dptr);
};

int keccak256_batch_device(const uint8_t *d_data, const int64_t *d_idx, int n, uint8_t *d_out, cudaStream_t st);
int keccak_peak(int device, double *perm_per_s);
int keccak256_batch_noalloc(const uint8_t *data, const int64_t *indexs, int n, uint8_t *out32, std::string &err);
int gen_ids(uint64_t seed, int64_t n, int64_t n_existing, int64_t next_new, double p_new, double theta, int64_t *d_ids,
            int64_t *n_new, cudaStream_t st, std::string &err);
int gen_keys(uint64_t seed, const int64_t *d_ids, int64_t n, int key_bytes, uint8_t *d_hexs, int *d_idx, cudaStream_t st,
             std::string &err);
int gen_values(uint64_t seed, int64_t n, int value_bytes, uint8_t *d_vals, int64_t *d_idx, cudaStream_t st,
               std::string &err);
int batch_features_device(const uint8_t *d_keys, const int *d_kidx, int n, int64_t keys_bytes, float out[4],
                          cudaStream_t st, std::string &err);

}  // namespace gmpt
