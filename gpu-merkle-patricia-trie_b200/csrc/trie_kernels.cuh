// trie_kernels.cuh -- sm_100a kernels of the batched MPT update path.
//
// Pipeline of one PhaseNU batch (puts_2phase_with_valuehp,
// mpt-with-compress/include/mpt/gpu_mpt.cuh:1262-1399):
//   k_stage        key/value records into trie-owned arenas, key validation
//   k_sort_*       lexicographic sort of the batch by 8-nibble chunks with
//                  segment refinement; last occurrence of a key wins
//   k_walk         per unique key: read-only descent from the root, marks
//                  the path dirty, overwrites values of keys that exist,
//                  and finds where new keys attach (anchor)
//   k_items_*      new keys + one "pseudo" item per short node that must be
//                  split, grouped by anchor
//   k_level_*      level-synchronous construction of the compressed
//                  subtries of every group (branch / extension / leaf)
//   k_hash_level   fused RLP encode + Keccak-256 of every dirty node of one
//                  nibble depth, deepest first (PhaseHC)
// The reference instead expands every key into one 240-byte FullNode per
// nibble and recompresses (K:3655, K:4025, K:4643); building the compressed
// form directly from the sorted batch writes each node once.
#pragma once
#include "common.cuh"
#include "keccak.cuh"

namespace gmpt {

// ---------------------------------------------------------------------------
// dirty list

struct DirtyList {
  uint32_t *ref;
  uint16_t *depth;
};

__device__ __forceinline__ void dirty_push(Counters *c, DirtyList d, uint32_t ref, uint32_t depth) {
  uint32_t i = warp_alloc(&c->n_dirty, 1);
  d.ref[i] = ref;
  d.depth[i] = (uint16_t)depth;
}

// First visitor of a node in this hash generation appends it to the dirty
// list.  Reads go through L2 (ld.cg): under LockNU the node may have been
// created by another SM during this launch.
__device__ __forceinline__ void mark_full(const TrieView &tv, DirtyList d, uint32_t f, uint32_t gen) {
  if (__ldcg(tv.full_epoch + f) != gen) {
    if (atomicExch(&tv.full_epoch[f], gen) != gen)
      dirty_push(tv.ctr, d, make_ref(KIND_FULL, f), __ldcg(tv.full_depth + f));
  }
}

__device__ __forceinline__ void mark_short(const TrieView &tv, DirtyList d, uint32_t s, uint32_t gen) {
  if (__ldcg(tv.short_epoch + s) != gen) {
    if (atomicExch(&tv.short_epoch[s], gen) != gen)
      dirty_push(tv.ctr, d, make_ref(KIND_SHORT, s), __ldcg(tv.short_depth + s));
  }
}

__device__ __forceinline__ void write_slot(const TrieView &tv, uint64_t slot, uint32_t ref) {
  if (is_root_slot(slot))
    tv.roots[slot_trie(slot)] = ref;
  else
    tv.full_child[(slot >> 5) * 17 + (slot & 31)] = ref;
}

__device__ __forceinline__ uint32_t new_full(const TrieView &tv, DirtyList d, uint32_t depth, uint32_t gen) {
  uint32_t f = warp_alloc(&tv.ctr->n_full, 1);
  if (f >= tv.cap_full) {
    set_error(tv.ctr, ERR_CAPACITY);
    return 0xFFFFFFFFu;
  }
  uint32_t *ch = tv.full_child + (size_t)f * 17;
#pragma unroll
  for (int i = 0; i < 17; ++i) ch[i] = 0;
  tv.full_depth[f] = (uint16_t)depth;
  tv.full_epoch[f] = gen;
  tv.full_hlen[f] = 0;
  tv.full_dead[f] = 0;
  dirty_push(tv.ctr, d, make_ref(KIND_FULL, f), depth);
  return f;
}

__device__ __forceinline__ uint32_t new_short(const TrieView &tv, DirtyList d, uint64_t key_off, uint32_t klen,
                                              uint32_t child, uint32_t depth, uint32_t gen) {
  uint32_t s = warp_alloc(&tv.ctr->n_short, 1);
  if (s >= tv.cap_short) {
    set_error(tv.ctr, ERR_CAPACITY);
    return 0xFFFFFFFFu;
  }
  tv.short_key[s] = key_off;
  tv.short_klen[s] = klen;
  tv.short_child[s] = child;
  tv.short_depth[s] = (uint16_t)depth;
  tv.short_epoch[s] = gen;
  tv.short_dead[s] = 0;
  tv.short_claim[s] = 0;
  tv.short_hlen[s] = 0;
  dirty_push(tv.ctr, d, make_ref(KIND_SHORT, s), depth);
  return s;
}

// ---------------------------------------------------------------------------
// staging

// Per-key records of a staged batch.  Grid-stride, with the stream counters
// (terminated keys, index-pair gaps; maxlen[0] = longest key, maxlen[1] =
// longest value) reduced per CTA: one atomic per CTA and counter instead of
// one per warp, which serialised on the counter addresses at 16M keys.
__global__ void __launch_bounds__(256) k_stage(TrieView tv, const int *ki, const int64_t *vi, const uint64_t *hp,
                                               int n, uint64_t key_base, uint64_t val_base, uint64_t vid_base,
                                               int64_t kbytes, int64_t vbytes, uint64_t *koff, uint32_t *klen,
                                               uint32_t *maxlen, const int *tid) {
  uint32_t terms = 0, gaps = 0, lmax = 0, vmax = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (tid && (uint32_t)tid[i] >= tv.n_tries) set_error(tv.ctr, ERR_BAD_TRIE);
    int ks = ki[2 * i], ke = ki[2 * i + 1];
    bool bad = ks < 0 || ke < ks || (int64_t)ke >= kbytes;  // index pair outside the key stream
    if (bad) ks = ke = 0;
    int len = ke - ks + 1;
    uint64_t off = key_base + (uint64_t)ks;
    if (len > kMaxKeyNibbles) {
      set_error(tv.ctr, ERR_KEY_TOO_LONG);
      bad = true;
    }
    // Interior nibbles are checked by k_stage_stream over the whole stream
    // when the index pairs tile it (the usual layout), else by k_stage_keys.
    bool term = false;
    if (!bad) {
      uint8_t last = tv.keys[off + len - 1];
      if (last > 16) bad = true;
      term = last == 16;
    }
    const bool gap = (i == 0) ? (ks != 0) : (ks != ki[2 * i - 1] + 1);
    terms += (term && !bad) ? 1u : 0u;
    gaps |= gap ? 1u : 0u;
    if (bad) {
      set_error(tv.ctr, ERR_BAD_KEY);
      len = 1;  // keep later stages in bounds
    }
    koff[i] = off;
    klen[i] = (uint32_t)len;
    lmax = max(lmax, (uint32_t)len);
    int64_t vs = vi[2 * i], ve = vi[2 * i + 1];
    if (vs < 0 || ve < vs - 1 || ve >= vbytes || ve - vs + 1 > 0x7FFFFFFF) {  // empty values allowed
      set_error(tv.ctr, ERR_BAD_KEY);
      vs = 0;
      ve = -1;
    }
    uint64_t vid = vid_base + (uint64_t)i;
    vmax = max(vmax, (uint32_t)(ve - vs + 1));
    tv.rec[vid] = ValueRec{val_base + (uint64_t)vs, (uint32_t)(ve - vs + 1), 0u};
    tv.rec_hp[vid] = hp ? hp[i] : 0ull;
  }
  __shared__ uint32_t red[4][8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  terms = __reduce_add_sync(0xffffffffu, terms);
  gaps = __reduce_or_sync(0xffffffffu, gaps);
  lmax = __reduce_max_sync(0xffffffffu, lmax);
  vmax = __reduce_max_sync(0xffffffffu, vmax);
  if (lane == 0) {
    red[0][warp] = terms;
    red[1][warp] = gaps;
    red[2][warp] = lmax;
    red[3][warp] = vmax;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0, g = 0, m = 0, v = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      t += red[0][w];
      g |= red[1][w];
      m = max(m, red[2][w]);
      v = max(v, red[3][w]);
    }
    if (t) atomicAdd(&tv.ctr->key_terms, t);
    if (g) atomicOr(&tv.ctr->noncontig, 1u);
    if (m) atomicMax(maxlen, m);
    if (v) atomicMax(maxlen + 1, v);  // longest value of the batch
  }
}

// Raw key bytes (the caller skips the hex conversion, util/utils.cuh:340-349
// key_bytes_to_hex).  A pair (s, e) is a key of e - s + 1 bytes, e = s - 1
// the empty key; its hex form is 2 * bytes + 1 nibbles.
__device__ __forceinline__ int raw_key_len(const int *ki, int i, int64_t raw_bytes) {
  const int s = ki[2 * i], e = ki[2 * i + 1];
  const bool bad = s < 0 || e < s - 1 || (int64_t)e >= raw_bytes || 2ll * (e - s + 1) + 1 > kMaxKeyNibbles;
  return bad ? -1 : e - s + 1;
}

// Hex length of every key into flags (for the offset scan); a malformed pair
// sets ERR_BAD_KEY and counts as the empty key so later stages stay in bounds.
__global__ void k_raw_lens(TrieView tv, const int *ki, int n, int64_t raw_bytes, unsigned long long *flags) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int len = raw_key_len(ki, i, raw_bytes);
  if (len < 0) set_error(tv.ctr, ERR_BAD_KEY);
  flags[i] = 2ull * (uint64_t)max(len, 0) + 1ull;
}

// Expand key i to nibbles (high, low per byte) + terminator 16 at hex offset
// pos[i] of `out`, and rewrite its index pair (in place) to the hex range.
__global__ void k_raw_expand(const uint8_t *raw, int *ki, const unsigned long long *pos, int n, int64_t raw_bytes,
                             uint8_t *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int len = max(raw_key_len(ki, i, raw_bytes), 0);
  const int s = ki[2 * i];
  const uint64_t p = pos[i];
  uint8_t *o = out + p;
  for (int b = 0; b < len; ++b) {
    const uint8_t x = raw[s + b];
    o[2 * b] = x >> 4;
    o[2 * b + 1] = x & 15;
  }
  o[2 * len] = 16;
  ki[2 * i] = (int)p;
  ki[2 * i + 1] = (int)(p + 2 * (uint64_t)len);
}

// Coalesced check of a key stream that the index pairs tile: no byte > 16,
// and exactly as many 16s as keys that end in one (so none is interior).
__global__ void k_stage_stream(TrieView tv, const uint8_t *stream, int64_t nbytes) {
  unsigned long long terms = 0;
  uint32_t bad = 0;
  const int64_t nvec = nbytes / 8;
  const uint64_t *v = reinterpret_cast<const uint64_t *>(stream);  // 8-aligned arena base
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nvec; q += (int64_t)gridDim.x * blockDim.x) {
    uint64_t x = __ldg(v + q);
    bad |= (x & 0xE0E0E0E0E0E0E0E0ull) != 0;                    // >= 32
    uint64_t hi = x & 0x1010101010101010ull;                      // bit 4 set: 16..31
    bad |= (x & ((hi >> 4) * 0x0Full)) ? 1u : 0u;                 // 17..31: low nibble != 0
    terms += __popcll(hi);
  }
  if (blockIdx.x == 0 && threadIdx.x < (nbytes & 7)) {
    uint8_t b = stream[nvec * 8 + threadIdx.x];
    bad |= b > 16;
    terms += b == 16;
  }
  unsigned am = __activemask();
  terms = __reduce_add_sync(am, (uint32_t)terms);
  bad = __reduce_or_sync(am, bad);
  if ((int)(threadIdx.x & 31) == __ffs(am) - 1) {
    if (terms) atomicAdd(&tv.ctr->stream_terms, terms);
    if (bad) atomicOr(&tv.ctr->bad_byte, 1u);
  }
}

// Per-key interior check for streams the index pairs do not tile.
__global__ void k_stage_keys(TrieView tv, const uint64_t *koff, const uint32_t *klen, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint8_t *k = tv.keys + koff[i];
  int len = (int)klen[i];
  uint64_t acc = 0;
  for (int j = 0; j < len - 1; j += 8) acc |= load_u64_unaligned(k + j) & low_mask64(min(8, len - 1 - j));
  if (acc & 0xF0F0F0F0F0F0F0F0ull) set_error(tv.ctr, ERR_BAD_KEY);
}

// ---------------------------------------------------------------------------
// sort + dedup (chunked MSD refinement over LSD radix passes)

__device__ __forceinline__ uint32_t key_chunk(const uint8_t *keys, uint64_t off, uint32_t len, int c) {
  uint32_t start = (uint32_t)c * 8;
  if (start >= len) return 0;
  uint64_t x = load_u64_unaligned(keys + off + start);
  uint32_t rem = len - start;
  if (rem < 8) x &= (1ull << (8 * rem)) - 1;  // zero bytes beyond the key
  return pack_nibbles8(x);
}

// *differs = 1 when some key's chunk c is not key 0's (a chunk every key of
// the batch shares needs no sort pass: YCSB keys all begin with "user")
__global__ void k_chunk_shared(const uint8_t *keys, const uint64_t *koff, const uint32_t *klen, int n, int c,
                               uint32_t *differs) {
  // once one warp has found a difference the rest have nothing to add: they
  // read the flag and leave instead of queueing atomics on one address
  if (__any_sync(0xffffffffu, __ldcg(differs) != 0u)) return;  // the whole warp leaves
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool d = i < n && key_chunk(keys, koff[i], klen[i], c) != key_chunk(keys, koff[0], klen[0], c);
  if (__any_sync(0xffffffffu, d) && (threadIdx.x & 31) == 0 && !__ldcg(differs)) atomicOr(differs, 1u);
}

// active = tied with a neighbour; packed: low = active, high = segment start
__global__ void k_sort_flags(const uint8_t *eqprev, int n, unsigned long long *flags) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  uint32_t tl = eqprev[p], tr = eqprev[p + 1];
  uint32_t active = (tl | tr) ? 1u : 0u;
  uint32_t start = (active && !tl) ? 1u : 0u;
  flags[p] = (unsigned long long)active | ((unsigned long long)start << 32);
}

// c >= 0: key chunk c; c == -1: key length; c == -2: trie id (forest batches)
__global__ void k_sort_build(TrieView tv, const unsigned long long *flags, const unsigned long long *pos,
                             const uint32_t *order, const uint64_t *koff, const uint32_t *klen, int n, int c,
                             uint32_t *act, uint64_t *skey, uint32_t *sval, const int *tid) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  unsigned long long f = flags[p];
  if (!(f & 1ull)) return;
  unsigned long long q = pos[p];
  uint32_t k = (uint32_t)q;
  uint32_t seg = (uint32_t)(q >> 32) + (uint32_t)(f >> 32) - 1u;
  uint32_t it = order[p];
  uint32_t ch = c >= 0 ? key_chunk(tv.keys, koff[it], klen[it], c) : (c == -1 ? klen[it] : (uint32_t)tid[it]);
  act[k] = (uint32_t)p;
  skey[k] = ((uint64_t)seg << 32) | ch;
  sval[k] = it;
}

__global__ void k_sort_scatter(const uint32_t *act, const uint64_t *skey, const uint32_t *sval, int K,
                               uint32_t *order, uint8_t *eqprev) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K) return;
  uint32_t p = act[k];
  order[p] = sval[k];
  eqprev[p] = (k > 0 && skey[k] == skey[k - 1]) ? 1 : 0;
}

__global__ void k_init_order(uint32_t *order, uint8_t *eqprev, int n) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p > n) return;
  if (p < n) order[p] = (uint32_t)p;
  eqprev[p] = (p > 0 && p < n) ? 1 : 0;
}

// keep the last of every run of equal keys
__global__ void k_keep_flags(const uint8_t *eqprev, int n, unsigned long long *flags) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  flags[p] = eqprev[p + 1] ? 0ull : 1ull;
}

__global__ void k_keep_scatter(const unsigned long long *flags, const unsigned long long *pos,
                               const uint32_t *order, int n, uint32_t *uord) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  if (flags[p]) uord[(uint32_t)pos[p]] = order[p];
}

// ---------------------------------------------------------------------------
// mixed read/write batches (puts_*_with_read, gpu_mpt.cuh:684-765 and
// 1609-1713).  The sort leaves equal keys (same trie) in runs, in batch
// order; p is a sorted position, order[p] its batch index, rw[i] = 1 for a
// write.  A read takes the last write before it in its run, else the trie
// as it was before the batch; each run keeps its last write for the insert.

__global__ void k_rw_sorted_flags(const uint8_t *eqprev, const uint32_t *order, const uint8_t *rw, int n,
                                  unsigned long long *is_write, unsigned long long *is_head) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  is_write[p] = rw[order[p]] ? 1ull : 0ull;
  is_head[p] = eqprev[p] ? 0ull : 1ull;
}

// sorted slots -> order / eqprev as the full-key sort leaves them
__global__ void k_rw_groups(const uint64_t *skey, const uint32_t *sval, int n, uint32_t *order, uint8_t *eqprev) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p > n) return;
  if (p < n) order[p] = sval[p];
  eqprev[p] = (p > 0 && p < n && skey[p] == skey[p - 1]) ? 1 : 0;
}

// the kept writes' key records, for a key-order sort of them alone
__global__ void k_rw_gather(const uint32_t *kept, int m, const uint64_t *koff, const uint32_t *klen, const int *tid,
                            uint64_t *koff_out, uint32_t *klen_out, int *tid_out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  const uint32_t i = kept[j];
  koff_out[j] = koff[i];
  klen_out[j] = klen[i];
  if (tid) tid_out[j] = tid[i];
}

__global__ void k_rw_map(const uint32_t *order, const uint32_t *kept, int m, uint32_t *uord) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < m) uord[j] = kept[order[j]];
}

// Key bytes of the kept writes of a mixed batch, moved together to the start
// of the batch's region of the key arena (the reads' keys are referenced by
// nothing once the reads are answered).  sizes -> scan -> copy out -> copy
// back -> offsets.
__global__ void k_rw_kept_sizes(const uint32_t *kept, int m, const uint32_t *klen, unsigned long long *sizes) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < m) sizes[j] = klen[kept[j]];
}

__global__ void k_rw_kept_copy(const uint8_t *keys, const uint64_t *koff, const uint32_t *klen, const uint32_t *kept,
                               const unsigned long long *offs, int m, uint8_t *out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  const uint32_t i = kept[j];
  const uint8_t *src = keys + koff[i];
  uint8_t *dst = out + offs[j];
  for (uint32_t b = 0; b < klen[i]; ++b) dst[b] = src[b];
}

__global__ void k_rw_kept_offsets(const uint32_t *kept, const unsigned long long *offs, int m, uint64_t base,
                                  uint64_t *koff) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < m) koff[kept[j]] = base + offs[j];
}

__global__ void k_rw_read_flags(TrieView tv, const uint8_t *rw, int n, unsigned long long *is_read) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (rw[i] > 1) set_error(tv.ctr, ERR_BAD_FLAG);
  is_read[i] = rw[i] ? 0ull : 1ull;
}

// wpos[k] = sorted position of the k-th write in sorted order
__global__ void k_rw_wpos(const unsigned long long *is_write, const unsigned long long *wrank, int n, uint32_t *wpos) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  if (is_write[p]) wpos[wrank[p]] = (uint32_t)p;
}

__device__ __forceinline__ int64_t lookup(const TrieView &tv, uint32_t root, const uint8_t *kb, uint32_t len);

__global__ void k_rw_resolve(TrieView tv, const uint32_t *order, const uint8_t *rw, const unsigned long long *is_head,
                             const unsigned long long *heads_before, const unsigned long long *wrank,
                             const uint32_t *wpos, const unsigned long long *n_writes, const unsigned long long *rrank,
                             const uint64_t *koff, const uint32_t *klen, const int *tid, uint64_t vid_base, int n,
                             uint64_t *out_hp, int *out_len, unsigned long long *keep) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const uint32_t i = order[p];
  // run id of a sorted position: heads up to and including it, minus one
  auto run = [&](uint32_t q) { return heads_before[q] + is_head[q]; };
  const unsigned long long k = wrank[p];  // writes before p in sorted order
  const unsigned long long nw = *n_writes;
  if (rw[i]) {
    keep[p] = (k + 1 >= nw || run(wpos[k + 1]) != run(p)) ? 1ull : 0ull;
    return;
  }
  keep[p] = 0ull;
  int64_t vid = -1;
  if (k > 0) {
    const uint32_t q = wpos[k - 1];
    if (run(q) == run(p)) vid = (int64_t)(vid_base + order[q]);
  }
  if (vid < 0) {
    const uint32_t tr = tid ? (uint32_t)tid[i] : 0u;
    vid = tr < tv.n_tries ? lookup(tv, tv.roots[tr], tv.keys + koff[i], klen[i]) : -1;
  }
  const unsigned long long r = rrank[i];
  out_hp[r] = vid < 0 ? 0ull : tv.rec_hp[vid];
  out_len[r] = vid < 0 ? 0 : (int)tv.rec[vid].len;
}

// ---------------------------------------------------------------------------
// walk (PhaseNU against an existing trie)

enum : uint8_t { W_EXISTS = 0, W_NEW = 1, W_SPLIT = 2, W_ERROR = 3 };

// anchor code: kind(2) | index(30) | child(5)  (37 bits, shifted left 27
// in the item sort key; the low 27 bits hold the rank)
__device__ __forceinline__ uint64_t code_full(uint32_t f, uint32_t c) {
  return (1ull << 35) | ((uint64_t)f << 5) | c;
}
__device__ __forceinline__ uint64_t code_short(uint32_t s) { return (2ull << 35) | ((uint64_t)s << 5) | 31u; }
// the root word of trie t (kind 0)
__device__ __forceinline__ uint64_t code_root(uint32_t t) { return (uint64_t)t << 5; }
__device__ __forceinline__ uint64_t code_slot(uint64_t slot) {
  return is_root_slot(slot) ? code_root(slot_trie(slot)) : code_full((uint32_t)(slot >> 5), (uint32_t)(slot & 31));
}

// nibble order used by the sort: terminator (16) sorts before 0
__device__ __forceinline__ int sym_rank(uint8_t b) { return b == 16 ? -1 : (int)b; }

struct WalkOut {
  uint8_t *status;
  uint64_t *code;
  uint32_t *d0;
  uint64_t *slot;
  uint32_t *short_id;
  uint8_t *after;
  // pseudo items
  uint32_t *p_short;
  uint32_t *p_d0;
  uint64_t *p_slot;
  uint32_t *p_amin;
  uint32_t *p_max;
};

// Thread per kWalkWays unique keys advancing together, so each thread keeps
// several independent pointer chases in flight (the walk is latency bound).
constexpr int kWalkWays = 4;

__global__ void __launch_bounds__(256, 2) k_walk(TrieView tv, DirtyList dl, const uint32_t *uord, int m,
                                                 const uint64_t *koff, const uint32_t *klen, uint64_t vid_base,
                                                 WalkOut wo, const int *tid) {
  const int nthreads = gridDim.x * blockDim.x;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t gen = tv.gen;
  uint32_t ref[kWalkWays], x[kWalkWays], len[kWalkWays], item[kWalkWays];
  uint64_t slot[kWalkWays];
  bool act[kWalkWays];
#pragma unroll
  for (int w = 0; w < kWalkWays; ++w) {
    const int j = t + w * nthreads;
    act[w] = j < m;
    item[w] = act[w] ? uord[j] : 0;
    len[w] = act[w] ? klen[item[w]] : 0;
    const uint32_t tr = (act[w] && tid) ? (uint32_t)tid[item[w]] : 0u;
    ref[w] = act[w] ? tv.roots[tr] : 0u;
    x[w] = 0;
    slot[w] = root_slot(tr);
  }
  for (int round = 0; round < kMaxKeyNibbles + 2; ++round) {
    bool any = false;
#pragma unroll
    for (int w = 0; w < kWalkWays; ++w) {
      if (!act[w]) continue;
      const int j = t + w * nthreads;
      const uint8_t *kb = tv.keys + koff[item[w]];
      const uint32_t kind = ref_kind(ref[w]), idx = ref_idx(ref[w]);
      if (kind == KIND_NULL) {
        wo.status[j] = W_NEW;
        wo.code[j] = code_slot(slot[w]);
        wo.d0[j] = x[w];
        wo.slot[j] = slot[w];
        act[w] = false;
        continue;
      }
      if (kind == KIND_FULL) {
        mark_full(tv, dl, idx, gen);
        if (x[w] >= len[w]) {
          wo.status[j] = W_ERROR;
          set_error(tv.ctr, ERR_BAD_KEY);
          act[w] = false;
          continue;
        }
        const uint32_t c = kb[x[w]];
        slot[w] = ((uint64_t)idx << 5) | c;
        ref[w] = tv.full_child[(size_t)idx * 17 + c];
        ++x[w];
        any = true;
        continue;
      }
      if (kind == KIND_SHORT) {
        const uint8_t *sk = tv.keys + tv.short_key[idx];
        const uint32_t sl = tv.short_klen[idx];
        const uint32_t lim = min(sl, len[w] - x[w]);
        const uint32_t mm = (uint32_t)match_nibbles(sk, kb + x[w], (int)lim);
        if (mm == sl) {
          mark_short(tv, dl, idx, gen);
          ref[w] = tv.short_child[idx];
          x[w] += sl;
          any = true;
          continue;
        }
        act[w] = false;
        if (mm == len[w] - x[w]) {  // key ends inside a stored key: prefix
          wo.status[j] = W_ERROR;
          set_error(tv.ctr, ERR_BAD_KEY);
          continue;
        }
        wo.status[j] = W_SPLIT;
        wo.code[j] = code_short(idx);
        wo.d0[j] = x[w];
        wo.slot[j] = slot[w];
        wo.short_id[j] = idx;
        wo.after[j] = sym_rank(kb[x[w] + mm]) > sym_rank(sk[mm]) ? 1 : 0;
        // the first diverger claims the split and creates the pseudo item
        const uint32_t ep = tv.epoch;
        if (tv.short_claim[idx] != ep) {
          if (atomicExch(&tv.short_claim[idx], ep) != ep) {
            const uint32_t p = atomicAdd(&tv.ctr->n_pseudo, 1u);
            wo.p_short[p] = idx;
            wo.p_d0[p] = x[w];
            wo.p_slot[p] = slot[w];
            wo.p_amin[p] = 0xFFFFFFFFu;
            wo.p_max[p] = 0;
            tv.short_pseudo[idx] = p;
            tv.short_dead[idx] = 1;
          }
        }
        continue;
      }
      // value node
      act[w] = false;
      if (x[w] == len[w]) {
        atomicMax(&tv.value_vid[idx], (unsigned long long)(vid_base + item[w]));
        wo.status[j] = W_EXISTS;
      } else {
        wo.status[j] = W_ERROR;
        set_error(tv.ctr, ERR_BAD_KEY);
      }
    }
    if (!any) break;
  }
}

__global__ void k_new_flags(const uint8_t *status, int m, unsigned long long *flags) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  uint8_t st = status[j];
  flags[j] = (st == W_NEW || st == W_SPLIT) ? 1ull : 0ull;
}

__global__ void k_pseudo_ranks(TrieView tv, const WalkOut wo, int m) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  if (wo.status[j] != W_SPLIT) return;
  uint32_t p = tv.short_pseudo[wo.short_id[j]];
  if (wo.after[j]) atomicMin(&wo.p_amin[p], (uint32_t)j);
  atomicMax(&wo.p_max[p], (uint32_t)j);
}

struct Items {
  uint64_t *key;
  uint32_t *id;
  uint64_t *base;
  uint32_t *len;
  uint32_t *ref;
  uint32_t *d0;
  uint64_t *slot;
};

// new keys (status NEW / SPLIT) -> items [0, n_new)
__global__ void k_items_new(TrieView tv, const WalkOut wo, const unsigned long long *pos, int m,
                            const uint32_t *uord, const uint64_t *koff, const uint32_t *klen, uint64_t vid_base,
                            Items it) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  uint8_t st = wo.status[j];
  if (st != W_NEW && st != W_SPLIT) return;
  uint32_t i = (uint32_t)pos[j];
  uint32_t item = uord[j];
  uint32_t v = warp_alloc(&tv.ctr->n_value, 1);
  if (v >= tv.cap_value) {
    set_error(tv.ctr, ERR_CAPACITY);
    v = 0;
  }
  tv.value_vid[v] = vid_base + item;
  it.key[i] = (wo.code[j] << 27) | (2ull * (uint64_t)j + 1ull);
  it.id[i] = i;
  it.base[i] = koff[item];
  it.len[i] = klen[item];
  it.ref[i] = make_ref(KIND_VALUE, v);
  it.d0[i] = wo.d0[j];
  it.slot[i] = wo.slot[j];
}

// pseudo items [n_new, n_new + n_pseudo): the existing short node re-inserted
// as a key ending in its old child
__global__ void k_items_pseudo(TrieView tv, const WalkOut wo, int n_pseudo, int n_new, Items it) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n_pseudo) return;
  uint32_t s = wo.p_short[p];
  uint32_t d0 = wo.p_d0[p];
  uint32_t amin = wo.p_amin[p];
  // real keys rank 2j+1; the pseudo item sits just before the first key
  // that sorts after the short node's key, else after the last diverger
  uint64_t rank = (amin != 0xFFFFFFFFu) ? (2ull * amin) : (2ull * wo.p_max[p] + 2ull);
  uint32_t i = (uint32_t)n_new + (uint32_t)p;
  it.key[i] = (code_short(s) << 27) | rank;
  it.id[i] = i;
  it.base[i] = tv.short_key[s] - d0;
  it.len[i] = d0 + tv.short_klen[s];
  it.ref[i] = tv.short_child[s];
  it.d0[i] = d0;
  it.slot[i] = wo.p_slot[p];
}

// Empty trie: every unique key is a new item of the single root group, already
// in sorted order (no walk, no grouping sort).  Value node j = vbase + j.
__global__ void k_items_bulk(TrieView tv, const uint32_t *uord, int m, const uint64_t *koff, const uint32_t *klen,
                             uint64_t vid_base, uint32_t vbase, uint64_t *sb_base, uint32_t *sb_len,
                             uint32_t *sb_ref, uint32_t *sb_d0, uint64_t *sb_slot, uint64_t *sb_code,
                             const int *tid) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  if (j == 0) atomicAdd(&tv.ctr->n_value, (uint32_t)m);
  uint32_t item = uord[j];
  uint32_t v = vbase + (uint32_t)j;
  tv.value_vid[v] = vid_base + item;
  sb_base[j] = koff[item];
  sb_len[j] = klen[item];
  sb_ref[j] = make_ref(KIND_VALUE, v);
  sb_d0[j] = 0;
  const uint32_t tr = tid ? (uint32_t)tid[item] : 0u;
  sb_slot[j] = root_slot(tr);
  sb_code[j] = code_root(tr);
}

// gather items into sorted order, group starts, and adjacent LCPs
__global__ void k_items_gather(const Items it, const uint32_t *order, int T, uint64_t *sb_base, uint32_t *sb_len,
                               uint32_t *sb_ref, uint32_t *sb_d0, uint64_t *sb_slot, uint64_t *sb_code) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= T) return;
  uint32_t s = order ? order[i] : (uint32_t)i;
  sb_base[i] = it.base[s];
  sb_len[i] = it.len[s];
  sb_ref[i] = it.ref[s];
  sb_d0[i] = it.d0[s];
  sb_slot[i] = it.slot[s];
  sb_code[i] = it.key[order ? i : s] >> 27;
}

__global__ void k_items_lcp(TrieView tv, const uint64_t *sb_base, const uint32_t *sb_len, const uint32_t *sb_d0,
                            const uint64_t *sb_code, int T, uint16_t *lcp) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= T) return;
  if (i == 0 || sb_code[i] != sb_code[i - 1]) {
    lcp[i] = kLcpInf;
    return;
  }
  uint32_t d0 = sb_d0[i];
  uint32_t la = sb_len[i - 1], lb = sb_len[i];
  uint32_t lim = min(la, lb);
  uint32_t m = d0 + (uint32_t)match_nibbles(tv.keys + sb_base[i - 1] + d0, tv.keys + sb_base[i] + d0, (int)(lim - d0));
  if (m >= lim) {  // equal keys or one is a prefix of the other
    set_error(tv.ctr, ERR_BAD_KEY);
    m = lim - 1;
  }
  lcp[i] = (uint16_t)m;
}

// ---------------------------------------------------------------------------
// level-synchronous subtrie construction

struct SegArrays {
  uint32_t *start, *end, *depth, *D, *branch;
  uint64_t *slot;
};

struct SortedItems {
  const uint64_t *base;
  const uint32_t *len;
  const uint32_t *ref;
  const uint32_t *d0;
  const uint64_t *slot;
  const uint64_t *code;
  const uint16_t *lcp;
};

// leaf for item i whose path is consumed up to nibble depth x
__device__ __forceinline__ void make_leaf(const TrieView &tv, DirtyList dl, const SortedItems &si, uint32_t i,
                                          uint32_t x, uint64_t slot, uint32_t gen) {
  uint32_t len = si.len[i];
  uint32_t child = si.ref[i];
  if (x < len) {
    uint32_t s = new_short(tv, dl, si.base[i] + x, len - x, child, x, gen);
    if (s == 0xFFFFFFFFu) return;
    write_slot(tv, slot, make_ref(KIND_SHORT, s));
  } else {
    write_slot(tv, slot, child);
  }
}

// groups -> leaves (singletons) or first-level segments
// kflags bits: 0 keep, 1 child/segment start, 2 child/segment end
__global__ void k_groups_init(TrieView tv, DirtyList dl, SortedItems si, int T, uint32_t gen, uint8_t *kflags,
                              unsigned long long *flags) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= T) return;
  bool gs = (i == 0) || si.code[i] != si.code[i - 1];
  bool ge = (i + 1 == T) || si.code[i + 1] != si.code[i];
  if (gs && ge) {
    make_leaf(tv, dl, si, i, si.d0[i], si.slot[i], gen);
    kflags[i] = 0;
    flags[i] = 0;
    return;
  }
  kflags[i] = 1 | (gs ? 2 : 0) | (ge ? 4 : 0);
  flags[i] = 1ull | ((unsigned long long)(gs ? 1 : 0) << 32);
}

__global__ void k_groups_scatter(SortedItems si, const uint8_t *kflags, const unsigned long long *pos, int T,
                                 uint32_t *act, uint32_t *aseg, SegArrays sg) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= T) return;
  uint8_t f = kflags[i];
  if (!(f & 1)) return;
  unsigned long long q = pos[i];
  uint32_t k = (uint32_t)q;
  uint32_t s = (uint32_t)(q >> 32) + ((f & 2) ? 1u : 0u) - 1u;
  act[k] = (uint32_t)i;
  aseg[k] = s;
  if (f & 2) {
    sg.start[s] = (uint32_t)i;
    sg.depth[s] = si.d0[i];
    sg.slot[s] = si.slot[i];
    sg.D[s] = 0xFFFFFFFFu;
  }
  if (f & 4) sg.end[s] = (uint32_t)i + 1;
}

// D[s] = min LCP over the interior boundaries of segment s
__global__ void k_level_min(SortedItems si, const uint32_t *act, const uint32_t *aseg, int K, SegArrays sg) {
  __shared__ uint32_t s_first;
  __shared__ uint32_t wmin[32];
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  bool ok = k < K;
  uint32_t s = ok ? aseg[k] : 0xFFFFFFFFu;
  uint32_t v = 0xFFFFFFFFu;
  if (ok) {
    uint32_t i = act[k];
    if (i != sg.start[s]) v = si.lcp[i];
  }
  if (threadIdx.x == 0) s_first = s;
  __syncthreads();
  int same = __syncthreads_and(!ok || s == s_first);
  if (same) {
    uint32_t w = __reduce_min_sync(0xffffffffu, v);
    if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = w;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t b = wmin[0];
      for (int i = 1; i < (int)(blockDim.x >> 5); ++i) b = min(b, wmin[i]);
      if (b != 0xFFFFFFFFu && s_first != 0xFFFFFFFFu) atomicMin(&sg.D[s_first], b);
    }
    return;
  }
  unsigned peers = __match_any_sync(0xffffffffu, s);
  uint32_t w = __reduce_min_sync(peers, v);
  if (ok && (int)(threadIdx.x & 31) == __ffs(peers) - 1 && w != 0xFFFFFFFFu) atomicMin(&sg.D[s], w);
}

// one branch (+ extension) per segment
__global__ void k_level_nodes(TrieView tv, DirtyList dl, SortedItems si, int S, SegArrays sg, uint32_t gen) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  uint32_t D = sg.D[s];
  uint32_t d = sg.depth[s];
  uint32_t i0 = sg.start[s];
  if (D == 0xFFFFFFFFu || D < d || D >= si.len[i0]) {
    set_error(tv.ctr, ERR_INTERNAL);
    sg.branch[s] = 0xFFFFFFFFu;
    return;
  }
  uint32_t f = new_full(tv, dl, D, gen);
  sg.branch[s] = f;
  if (f == 0xFFFFFFFFu) return;
  uint32_t top = make_ref(KIND_FULL, f);
  if (D > d) {
    uint32_t e = new_short(tv, dl, si.base[i0] + d, D - d, top, d, gen);
    if (e == 0xFFFFFFFFu) return;
    top = make_ref(KIND_SHORT, e);
  }
  write_slot(tv, sg.slot[s], top);
}

// children of every branch: leaves now, larger children become segments of
// the next level
__global__ void k_level_children(TrieView tv, DirtyList dl, SortedItems si, const uint32_t *act,
                                 const uint32_t *aseg, int K, SegArrays sg, uint32_t gen, uint8_t *kflags,
                                 uint8_t *knib, unsigned long long *flags) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K) return;
  uint32_t i = act[k];
  uint32_t s = aseg[k];
  uint32_t D = sg.D[s];
  uint32_t f = sg.branch[s];
  if (f == 0xFFFFFFFFu) {
    kflags[k] = 0;
    flags[k] = 0;
    return;
  }
  bool cs = (i == sg.start[s]) || si.lcp[i] == D;
  bool ce = (i + 1 == sg.end[s]) || si.lcp[i + 1] == D;
  // only the first item of a child run names the child slot: the other
  // items skip the gather of their key's nibble
  uint8_t nib = cs ? tv.keys[si.base[i] + D] : 0;
  uint64_t slot = ((uint64_t)f << 5) | nib;
  if (cs && ce) {
    make_leaf(tv, dl, si, i, D + 1, slot, gen);
    kflags[k] = 0;
    flags[k] = 0;
    return;
  }
  kflags[k] = 1 | (cs ? 2 : 0) | (ce ? 4 : 0);
  knib[k] = nib;
  flags[k] = 1ull | ((unsigned long long)(cs ? 1 : 0) << 32);
}

__global__ void k_level_scatter(const uint32_t *act, const uint32_t *aseg, const uint8_t *kflags,
                                const uint8_t *knib, const unsigned long long *pos, int K, SegArrays cur,
                                uint32_t *nact, uint32_t *naseg, SegArrays nxt) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K) return;
  uint8_t f = kflags[k];
  if (!(f & 1)) return;
  unsigned long long q = pos[k];
  uint32_t nk = (uint32_t)q;
  uint32_t ns = (uint32_t)(q >> 32) + ((f & 2) ? 1u : 0u) - 1u;
  uint32_t i = act[k];
  uint32_t s = aseg[k];
  nact[nk] = i;
  naseg[nk] = ns;
  if (f & 2) {
    nxt.start[ns] = i;
    nxt.depth[ns] = cur.D[s] + 1;
    nxt.slot[ns] = ((uint64_t)cur.branch[s] << 5) | knib[k];
    nxt.D[ns] = 0xFFFFFFFFu;
  }
  if (f & 4) nxt.end[ns] = i + 1;
}

// ---------------------------------------------------------------------------
// PhaseHC: dirty leaves first, then the other nodes bucketed by (nibble
// depth, kind), deepest first

// Keccak blocks a dirty branch's encoding is expected to take, minus one,
// capped at kHashClasses - 1: children counted as 33-byte references, and a
// value in slot 16 (a key that ends at the branch) by its length, which can
// be kilobytes.  Branches of a level are binned by it, and k_hash_level
// orders each CTA's nodes by block class, so the lanes of a warp need the
// same number of permutations and none idles through another's extra ones.
constexpr uint32_t kHashClasses = 8;

__device__ __forceinline__ uint32_t full_bytes(const TrieView &tv, uint32_t idx) {
  const uint32_t *c = tv.full_child + (size_t)idx * 17;
  uint32_t cnt = 0;
#pragma unroll
  for (int k = 0; k < 16; ++k) cnt += c[k] != 0u ? 1u : 0u;
  uint32_t bytes = 20u + 32u * cnt;
  const uint32_t v = c[16];
  if (ref_kind(v) == KIND_VALUE) bytes += 3u + load_rec(tv, tv.value_vid[ref_idx(v)]).len;
  return bytes;
}

__device__ __forceinline__ uint32_t full_class(const TrieView &tv, uint32_t idx) {
  return min(full_bytes(tv, idx) / 136u, kHashClasses - 1u);
}

// Finer classes for the order inside one hashing CTA (leaves with values of
// up to kilobytes take 1 to 31 blocks): 1, 2, 3, 4, 5-6, 7-10, 11-18, 19+
// blocks.
constexpr uint32_t kCtaClasses = 8;

__device__ __forceinline__ uint32_t blocks_class(uint32_t blocks_minus_1) {
  const uint32_t b = blocks_minus_1;
  return b < 4u ? b : (b < 6u ? 4u : (b < 10u ? 5u : (b < 18u ? 6u : 7u)));
}

__device__ __forceinline__ uint32_t hash_class(const TrieView &tv, uint32_t r) {
  const uint32_t kind = ref_kind(r), idx = ref_idx(r);
  uint32_t bytes;
  if (kind == KIND_FULL) {
    return blocks_class(full_bytes(tv, idx) / 136u);
  } else {
    if (tv.short_dead[idx]) return 0u;
    const uint32_t ch = tv.short_child[idx];
    bytes = tv.short_klen[idx] / 2u + 8u;
    bytes += ref_kind(ch) == KIND_VALUE ? load_rec(tv, tv.value_vid[ref_idx(ch)]).len : 33u;
  }
  return blocks_class(bytes / 136u);
}

// Leaves (short nodes over a value) depend on nothing below them, so every
// dirty leaf is hashed in one launch ahead of the levels, whatever its
// depth; the levels then hold only branches and extensions.  Leaves are
// ordered by their exact Keccak block count (minus one, capped at
// kLeafClasses - 1) over the whole batch, so a warp's 32 leaves need the
// same number of permutations.  Ordering inside one 128-node CTA alone left
// about half of the lanes idle with values of up to kilobytes (1 to 31
// blocks), and hashing leaves level by level made deep tries a chain of
// small launches, each as long as its slowest leaf.
constexpr uint32_t kLeafClasses = 32;
// bins: the kLeafClasses leaf bins, then per nibble depth one bin of
// extensions and kHashClasses bins of branches; a level is one contiguous
// range of the sorted dirty list
constexpr uint32_t kBinsPerDepth = 1 + kHashClasses;
constexpr uint32_t kLeafBit = 0x80;  // class byte of a leaf

__host__ __device__ __forceinline__ uint32_t level_bin(uint32_t depth) { return kLeafClasses + depth * kBinsPerDepth; }

// class byte of a dirty node: kLeafBit | block class for a leaf, the hash
// class for a branch, 0 for an extension or a dead short node (LockNU's
// splits leave many: among the leaves they would idle lanes of the warps
// that hash live leaves of the same block count)
__device__ __forceinline__ uint32_t dirty_class(const TrieView &tv, uint32_t r, bool leaf_classes) {
  const uint32_t idx = ref_idx(r);
  if (ref_kind(r) == KIND_FULL) return full_class(tv, idx);
  if (tv.short_dead[idx]) return 0u;
  const uint32_t ch = tv.short_child[idx];
  if (ref_kind(ch) != KIND_VALUE) return 0u;
  if (!leaf_classes) return kLeafBit;
  const uint32_t bytes = tv.short_klen[idx] / 2u + 8u + load_rec(tv, tv.value_vid[ref_idx(ch)]).len;
  return kLeafBit | min(bytes / 136u, kLeafClasses - 1u);
}

// bin of a dirty node from its depth, kind and class byte; inside a launch
// the classes run longest first, so the CTAs of the slowest nodes start in
// the first wave instead of forming the last one
__device__ __forceinline__ uint32_t dirty_bin(uint32_t depth, uint32_t r, uint32_t cls) {
  if (cls & kLeafBit) return kLeafClasses - 1u - (cls & ~kLeafBit);
  return level_bin(depth) + (ref_kind(r) == KIND_FULL ? kHashClasses - cls : 0u);
}

// Histogram of the dirty list over the bins (nbins of them, covering every
// depth a node can have).  Leaves are classed by block count only when
// `leaf_classes` is set (a batch held values long enough for a leaf to take
// two or more Keccak blocks).
__global__ void k_dirty_hist(TrieView tv, const uint32_t *ref, const uint16_t *depth, int n, uint32_t *bins,
                             int nbins, int leaf_classes, uint8_t *cls) {
  extern __shared__ uint32_t h[];
  for (int b = threadIdx.x; b < nbins; b += blockDim.x) h[b] = 0;
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t r = ref[i];
    const uint32_t c = dirty_class(tv, r, leaf_classes != 0);
    cls[i] = (uint8_t)c;
    atomicAdd(&h[dirty_bin(depth[i], r, c)], 1u);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < nbins; b += blockDim.x)
    if (h[b]) atomicAdd(&bins[b], h[b]);
}

// Scatter of the dirty list into its bins, 256 entries per CTA pass.  Counts
// are aggregated per warp (match_any) and then per CTA in a shared table of
// the bins the pass touches, so a hot bin (a level of millions of leaves)
// takes one global atomic per CTA pass instead of one per warp.
__global__ void __launch_bounds__(256) k_dirty_scatter(const uint32_t *ref, const uint16_t *depth, const uint8_t *cls,
                                                       int n, uint32_t *cursor, uint32_t *out, Counters *ctr) {
  constexpr uint32_t kEmpty = 0xFFFFFFFFu;
  __shared__ uint32_t tbin[256], tcnt[256], tbase[256];
  const int lane = threadIdx.x & 31;
  for (int c0 = blockIdx.x * 256; c0 < n; c0 += gridDim.x * 256) {
    tbin[threadIdx.x] = kEmpty;
    tcnt[threadIdx.x] = 0;
    __syncthreads();
    const int i = c0 + threadIdx.x;
    const bool ok = i < n;
    const uint32_t r = ok ? ref[i] : 0u;
    const uint32_t b = ok ? dirty_bin(depth[i], r, cls[i]) : kEmpty;
    const unsigned peers = __match_any_sync(0xffffffffu, b);
    const int leader = __ffs(peers) - 1;
    uint32_t slot = 0, off = 0, claimed = 0;
    if (ok && lane == leader) {
      slot = (b * 0x9E3779B1u) >> 24;  // at most 256 bins per pass: a free slot exists
      for (int probe = 0; probe < 256; ++probe) {
        const uint32_t prev = atomicCAS(&tbin[slot], kEmpty, b);
        if (prev == kEmpty || prev == b) {
          claimed = 1;
          break;
        }
        slot = (slot + 1) & 255u;
      }
      // no slot of this bin (cannot happen with <= 256 bins per pass): report
      // it and leave the entries out rather than count them in another bin
      if (claimed)
        off = atomicAdd(&tcnt[slot], (uint32_t)__popc(peers));
      else
        set_error(ctr, ERR_INTERNAL);
    }
    slot = __shfl_sync(0xffffffffu, slot, leader);
    off = __shfl_sync(0xffffffffu, off, leader);
    claimed = __shfl_sync(0xffffffffu, claimed, leader);
    __syncthreads();
    if (tbin[threadIdx.x] != kEmpty) tbase[threadIdx.x] = atomicAdd(&cursor[tbin[threadIdx.x]], tcnt[threadIdx.x]);
    __syncthreads();
    if (ok && claimed) out[tbase[slot] + off + __popc(peers & ((1u << lane) - 1u))] = r;
    __syncthreads();
  }
}

// one message item: <= 8 prefix bytes, then a body read from memory
struct EncItem {
  uint64_t pre;
  uint32_t pren;
  uint32_t nib;  // body holds nibbles, packed in pairs
  const uint8_t *body;
  uint32_t blen;
};

__device__ __forceinline__ int be_size(uint64_t v) {
  int s = 1;
  while (v >>= 8) ++s;
  return s;
}

// RLP header bytes (tag small/large) for a payload of `size`, little-endian
__device__ __forceinline__ void rlp_head(uint64_t size, uint32_t small_tag, uint32_t large_tag, uint64_t &pre,
                                         uint32_t &pren) {
  if (size < 56) {
    pre = small_tag + size;
    pren = 1;
    return;
  }
  int s = be_size(size);
  pre = large_tag + (uint32_t)s;
  for (int k = 0; k < s; ++k) pre |= ((size >> (8 * (s - 1 - k))) & 0xFF) << (8 * (1 + k));
  pren = 1 + s;
}

// Loads of node fields and message bytes.  kCoh = true inside a persistent
// launch, where the data may have been written earlier in the same launch by
// another SM, before a grid barrier (fence, arrive, wait, fence): ordinary
// loads then see those writes, but the non-coherent read-only path
// (ld.global.nc) is not used for them.  Key nibbles are staged by an earlier
// launch and stay on the read-only path in both modes.
template <bool kCoh, typename T>
__device__ __forceinline__ T ldn(const T *p) {
  return *p;
}

template <bool kCoh>
__device__ __forceinline__ uint64_t ld8(const uint8_t *p) {
  if constexpr (kCoh)
    return load_u64_unaligned_cg(p);
  else
    return load_u64_unaligned(p);
}

// the item a parent writes for child `r` (node.cuh:437-450 / 548-557;
// rlp.cuh:132-155 write_bytes; a value node's "hash" is its raw value)
template <bool kCoh = false>
__device__ __forceinline__ EncItem child_item(const TrieView &tv, uint32_t r) {
  EncItem it{0, 0, 0, nullptr, 0};
  uint32_t kind = ref_kind(r), idx = ref_idx(r);
  if (kind == KIND_NULL) {
    it.pre = 0x80;
    it.pren = 1;
    return it;
  }
  const uint8_t *h;
  uint32_t hl;
  if (kind == KIND_VALUE) {
    unsigned long long vid = ldn<kCoh>(tv.value_vid + idx);
    const ValueRec rc = load_rec(tv, vid);
    h = tv.vals + rc.off;
    hl = rc.len;
  } else {
    if (kind == KIND_FULL) {
      h = tv.full_hash + (size_t)idx * 32;
      hl = ldn<kCoh>(tv.full_hlen + idx);
    } else {
      h = tv.short_hash + (size_t)idx * 32;
      hl = ldn<kCoh>(tv.short_hlen + idx);
    }
    if (tv.geth_mode && hl < 32) {  // go-ethereum embeds small nodes
      it.body = h;
      it.blen = hl;
      return it;
    }
  }
  it.body = h;
  it.blen = hl;
  if (hl == 1 && ldn<kCoh>(h) < 0x80) return it;  // single byte is its own encoding
  rlp_head(hl, 0x80, 0xb7, it.pre, it.pren);
  return it;
}

// compact (hex-prefix) key item: utils.cuh:361-396 hex_to_compact
__device__ __forceinline__ EncItem compact_item(const TrieView &tv, uint64_t koff, uint32_t klen) {
  EncItem it{0, 0, 1, nullptr, 0};
  const uint8_t *k = tv.keys + koff;
  uint32_t term = (klen > 0 && k[klen - 1] == 16) ? 1 : 0;
  uint32_t ln = klen - term;
  uint32_t odd = ln & 1;
  uint32_t clen = ln / 2 + 1;
  uint32_t flag = (term << 5) | (odd ? (0x10u | k[0]) : 0u);
  it.body = k + odd;
  it.blen = clen - 1;
  if (clen == 1) {  // one byte < 0x80: written as itself
    it.pre = flag;
    it.pren = 1;
    return it;
  }
  uint64_t h;
  uint32_t hn;
  rlp_head(clen, 0x80, 0xb7, h, hn);
  it.pre = h | ((uint64_t)flag << (8 * hn));
  it.pren = hn + 1;
  return it;
}

// 16 nibble bytes -> 8 bytes (hi << 4 | lo)
__device__ __forceinline__ uint64_t pack_pairs8(const uint8_t *p) {
  uint64_t r = 0;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    uint64_t x = load_u64_unaligned(p + 8 * h);
    uint64_t z = ((x & 0x000F000F000F000Full) << 4) | ((x >> 8) & 0x000F000F000F000Full);
    z = (z | (z >> 8)) & 0x0000FFFF0000FFFFull;
    z = (z | (z >> 16)) & 0x00000000FFFFFFFFull;
    r |= z << (32 * h);
  }
  return r;
}

template <bool kCoh = false>
__device__ __forceinline__ EncItem node_item(const TrieView &tv, bool full, uint32_t idx, int item,
                                             uint64_t payload) {
  EncItem it{0, 0, 0, nullptr, 0};
  if (item == 0) {
    rlp_head(payload, 0xc0, 0xf7, it.pre, it.pren);
    return it;
  }
  if (full) return child_item<kCoh>(tv, ldn<kCoh>(tv.full_child + (size_t)idx * 17 + (item - 1)));
  if (item == 1) return compact_item(tv, ldn<kCoh>(tv.short_key + idx), ldn<kCoh>(tv.short_klen + idx));
  return child_item<kCoh>(tv, ldn<kCoh>(tv.short_child + idx));
}

// Thread per dirty node: RLP-encode straight into the sponge, Keccak-256 if
// the encoding is >= 32 bytes, else keep it raw (gpu_mpt_kernels.cuh:2885-3045
// semantics; cpu_mpt.cuh:380-496).
__device__ __forceinline__ void prefetch_l1(const void *p) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// OR the low n bytes of v into the message at byte position p (the staged
// block is zeroed first); a chunk may straddle two 8-byte words.
__device__ __forceinline__ void or_bytes(uint64_t *st, uint32_t S, uint64_t v, uint32_t n, uint32_t p) {
  if (n == 0) return;
  const uint32_t q = p >> 3, r = p & 7;
  st[q * S] |= v << (8 * r);
  if (r != 0 && r + n > 8) st[(q + 1) * S] |= v >> (64 - 8 * r);
}

// Start the loads of a child item's bytes early (hash line, or the first
// lines of a value) so the encoder's streaming reads hit L1.
__device__ __forceinline__ void prefetch_child(const TrieView &tv, uint32_t r) {
  uint32_t kind = ref_kind(r), idx = ref_idx(r);
  if (kind == KIND_FULL)
    prefetch_l1(tv.full_hash + (size_t)idx * 32);
  else if (kind == KIND_SHORT)
    prefetch_l1(tv.short_hash + (size_t)idx * 32);
}

// Encode + hash one dirty node; `stage` is this thread's 17-word message
// block in shared memory (word w at stage[w * stride]).
template <bool kCoh>
__device__ __forceinline__ void hash_node(const TrieView &tv, uint32_t ref, uint64_t *stage, uint32_t stride) {
  uint32_t kind = ref_kind(ref), idx = ref_idx(ref);
  bool full = kind == KIND_FULL;
  // nodes a split or a delete unlinked are not hashed
  if (ldn<kCoh>((full ? tv.full_dead : tv.short_dead) + idx)) return;
  // depth 0 holds exactly the roots of the forest's tries; go-ethereum
  // hashes a root whatever its size
  bool force = tv.geth_mode && (full ? ldn<kCoh>(tv.full_depth + idx) : ldn<kCoh>(tv.short_depth + idx)) == 0;
  int nitems = full ? 18 : 3;
  // pass 1: payload size (all child loads issued together, sources prefetched)
  uint64_t payload = 0;
  EncItem it1{0, 0, 0, nullptr, 0}, it2{0, 0, 0, nullptr, 0};  // short: key, child
  const uint32_t *chp = tv.full_child + (size_t)idx * 17;
  // branch whose children are all hashed nodes (32-byte references) and whose
  // value slot is empty: its encoding is regular and is generated word by word
  uint32_t present = 0;
  bool regular = full;
  if (full) {
    uint32_t ch[17];
#pragma unroll
    for (int k = 0; k < 17; ++k) ch[k] = ldn<kCoh>(chp + k);
#pragma unroll
    for (int k = 0; k < 17; ++k) prefetch_child(tv, ch[k]);
#pragma unroll
    for (int k = 0; k < 17; ++k) {
      EncItem it = child_item<kCoh>(tv, ch[k]);
      payload += it.pren + it.blen;
      const uint32_t kd = ref_kind(ch[k]);
      if (kd == KIND_VALUE) {  // a key ending here: its value (up to kilobytes) closes the encoding
        prefetch_l1(it.body);
        if (it.blen > 120) prefetch_l1(it.body + 128);
      }
      if (kd != KIND_NULL) {
        present |= 1u << k;
        regular = regular && k < 16 && kd != KIND_VALUE && it.blen == 32 && it.pren == 1;
      }
    }
  } else {
    uint32_t child = ldn<kCoh>(tv.short_child + idx);
    const uint8_t *kp = tv.keys + ldn<kCoh>(tv.short_key + idx);
    prefetch_l1(kp);
    if (ref_kind(child) == KIND_VALUE) {
      unsigned long long vid = tv.value_vid[ref_idx(child)];
      const ValueRec rc = load_rec(tv, vid);
      const uint8_t *vp = tv.vals + rc.off;
      prefetch_l1(vp);
      if (rc.len > 120) prefetch_l1(vp + 128);
    } else {
      prefetch_child(tv, child);
    }
    it1 = node_item<kCoh>(tv, false, idx, 1, 0);
    it2 = node_item<kCoh>(tv, false, idx, 2, 0);
    payload = it1.pren + it1.blen + it2.pren + it2.blen;
  }
  uint64_t hdr;
  uint32_t hn;
  rlp_head(payload, 0xc0, 0xf7, hdr, hn);
  uint64_t total = payload + hn;
  bool raw = total < 32 && !force;
  Sponge sp;
  sp.reset(stage, stride);
  if (!full && total <= 135) {
    // One-block short node (every leaf with a value up to ~100 bytes, every
    // extension): place each segment's 8-byte chunks into the zeroed block
    // with shared-memory OR, pad, and permute once.
    uint64_t *st = sp.stage;
    const uint32_t S = sp.stride;
#pragma unroll
    for (int w = 0; w < 17; ++w) st[w * S] = 0;
    uint32_t p = 0;
    or_bytes(st, S, hdr, hn, p);
    p += hn;
    or_bytes(st, S, it1.pre, it1.pren, p);
    p += it1.pren;
    for (uint32_t o = 0; o < it1.blen; o += 8) {
      uint32_t nb = min(8u, it1.blen - o);
      or_bytes(st, S, pack_pairs8(it1.body + 2 * o) & low_bytes_mask(nb), nb, p + o);
    }
    p += it1.blen;
    or_bytes(st, S, it2.pre, it2.pren, p);
    p += it2.pren;
    for (uint32_t o = 0; o < it2.blen; o += 8) {
      uint32_t nb = min(8u, it2.blen - o);
      or_bytes(st, S, ld8<kCoh>(it2.body + o) & low_bytes_mask(nb), nb, p + o);
    }
    p += it2.blen;
    if (!raw) {
      or_bytes(st, S, 0x01, 1, p);
      st[16 * S] |= 0x8000000000000000ull;
#pragma unroll
      for (int w = 0; w < 17; ++w) sp.a[w] = st[w * S];
      keccak_f1600(sp.a);
    }
  } else if (regular) {
  // regular branch: pending message bytes (little-endian), next slot, words
  // left of the current child's hash
  uint64_t buf = hdr;
  uint32_t nb = hn, slot = 0, hj = 8;
  const uint32_t *hw = nullptr;
  bool last = false;
  while (true) {
    {  // one block: 0x80 per empty slot, 0xa0 + 32 hash bytes per child, then
       // the Keccak padding (rlp.cuh:132-155, node.cuh:46-112)
      uint64_t *st = sp.stage;
      const uint32_t S = sp.stride;
      for (int w = 0; w < 17; ++w) {
        uint64_t word = 0;
#pragma unroll
        for (int half = 0; half < 2; ++half) {
          while (nb < 4) {
            if (hj < 8) {
              buf |= (uint64_t)ldn<kCoh>(hw + hj) << (8 * nb);
              nb += 4;
              ++hj;
            } else if (slot < 17) {
              if ((present >> slot) & 1u) {
                const uint32_t r = ldn<kCoh>(chp + slot);
                hw = reinterpret_cast<const uint32_t *>(
                    (ref_kind(r) == KIND_FULL ? tv.full_hash : tv.short_hash) + (size_t)ref_idx(r) * 32);
                buf |= 0xa0ull << (8 * nb);
                hj = 0;
              } else {
                buf |= 0x80ull << (8 * nb);
              }
              nb += 1;
              ++slot;
            } else if (!last) {
              buf |= 0x01ull << (8 * nb);  // Keccak padding starts here
              nb += 1;
              last = true;
            } else {
              nb = 4;  // zeros to the end of the block
            }
          }
          word |= (buf & 0xFFFFFFFFull) << (32 * half);
          buf >>= 32;
          nb -= 4;
        }
        st[w * S] = word;
      }
      if (last) st[16 * S] |= 0x8000000000000000ull;
    }
    sp.absorb();
    if (last) break;
  }
  } else {
  // pass 2: stream
  int item = 0;
  EncItem cur{hdr, hn, 0, nullptr, 0};
  uint32_t off = 0;
  bool pre_pending = true, last = false;
  while (true) {
    while (!sp.full()) {
      if (pre_pending) {
        pre_pending = false;
        if (cur.pren) sp.push(cur.pre, cur.pren);
        continue;
      }
      if (off < cur.blen) {
        const uint32_t room = 17u - sp.w;  // whole words left in this block
        if (!cur.nib && cur.blen - off >= 8u * room) {
          // the item (a long value) covers the rest of the block: whole
          // words straight from memory, the loads independent of each other
          // (the partial word carried in acc keeps its length)
          const uint8_t *src = cur.body + off;
          const uint32_t ca = 8u * sp.accn;
#pragma unroll 4
          for (uint32_t i = 0; i < room; ++i) {
            const uint64_t x = ld8<kCoh>(src + 8u * i);
            if (ca == 0) {
              sp.emit(x);
            } else {
              sp.emit(sp.acc | (x << ca));
              sp.acc = x >> (64u - ca);
            }
          }
          off += 8u * room;
          continue;
        }
        uint32_t nb = min(8u, cur.blen - off);
        uint64_t v = cur.nib ? pack_pairs8(cur.body + 2 * off) : ld8<kCoh>(cur.body + off);
        sp.push(v & low_bytes_mask(nb), nb);
        off += nb;
        continue;
      }
      if (++item == nitems) {
        sp.pad();
        last = true;
        break;
      }
      cur = node_item<kCoh>(tv, full, idx, item, payload);
      off = 0;
      pre_pending = true;
    }
    if (raw) break;
    // a long body (a value of up to kilobytes) streams through many blocks:
    // start the loads of the next two lines of it before the permutation,
    // so they arrive while it runs (addresses stay inside the body)
    if (cur.body && !cur.nib && off < cur.blen) {
      const uint32_t rest = cur.blen - off - 1;
      prefetch_l1(cur.body + off + min(128u, rest));
      prefetch_l1(cur.body + off + min(256u, rest));
    }
    sp.absorb();
    if (last) break;
  }
  }
  if (tv.account) {  // accounting (timing mode): encoding bytes and absorbed blocks of this pass
    unsigned am = __activemask();
    unsigned long long eb = __reduce_add_sync(am, (uint32_t)total);
    unsigned long long kb = __reduce_add_sync(am, raw ? 0u : (uint32_t)((total + 1 + 135) / 136));
    uint32_t nh = __popc(am);
    if ((int)(threadIdx.x & 31) == __ffs(am) - 1) {
      atomicAdd(&tv.ctr->enc_bytes, eb);
      atomicAdd(&tv.ctr->keccak_blocks, kb);
      atomicAdd(&tv.ctr->hashed, nh);
    }
  }
  uint8_t *hout = (full ? tv.full_hash : tv.short_hash) + (size_t)idx * 32;
  uint64_t *o = reinterpret_cast<uint64_t *>(hout);
  if (raw) {
#pragma unroll
    for (int w = 0; w < 4; ++w) {
      uint64_t v = sp.stage[w * sp.stride];
      int keep = (int)total - 8 * w;
      o[w] = keep >= 8 ? v : (keep <= 0 ? 0ull : (v & ((1ull << (8 * keep)) - 1)));
    }
    (full ? tv.full_hlen : tv.short_hlen)[idx] = (uint8_t)total;
  } else {
    o[0] = sp.a[0];
    o[1] = sp.a[1];
    o[2] = sp.a[2];
    o[3] = sp.a[3];
    (full ? tv.full_hlen : tv.short_hlen)[idx] = 32;
  }
}

// Message buffer of one warp for hash_full_warp (8 Keccak blocks).
constexpr int kWarpMsgBytes = 8 * 136;

// Warp-cooperative encode + hash of branch node idx, for levels with few
// nodes or for branches of many blocks, where one thread's serial chain is
// the latency: the message is built window by window (kWarpMsgBytes, 8
// blocks) in the warp's shared buffer, every lane copying a share of each
// item's bytes (lane k < 17 holds child k's item, the header goes first),
// and absorbed with the warp-spread permutation.  All 32 lanes call it with
// the same idx.
template <bool kCoh>
__device__ __forceinline__ void hash_full_warp(const TrieView &tv, uint32_t idx, uint8_t *msg, const CoopLanes &cl) {
  constexpr unsigned kAll = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  if (ldn<kCoh>(tv.full_dead + idx)) return;  // unlinked by a delete: nothing to hash
  EncItem it{0, 0, 0, nullptr, 0};
  if (lane < 17) it = child_item<kCoh>(tv, ldn<kCoh>(tv.full_child + (size_t)idx * 17 + lane));
  const uint32_t sz = lane < 17 ? it.pren + it.blen : 0u;
  uint32_t incl = sz;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t v = __shfl_up_sync(kAll, incl, o);
    if (lane >= o) incl += v;
  }
  const uint32_t payload = __shfl_sync(kAll, incl, 31);
  uint64_t hdr;
  uint32_t hn;
  rlp_head(payload, 0xc0, 0xf7, hdr, hn);
  const uint32_t total = payload + hn;
  const bool force = tv.geth_mode && ldn<kCoh>(tv.full_depth + idx) == 0;
  const bool raw = total < 32 && !force;
  const uint32_t nblk = raw ? 1u : (total + 1 + 135) / 136;
  const uint32_t padded = nblk * 136;
  const uint32_t my_off = hn + incl - sz;  // message offset of this lane's item
  uint64_t *m64 = reinterpret_cast<uint64_t *>(msg);
  uint64_t a = 0;  // this lane's word of the state
  for (uint32_t b0 = 0; b0 < nblk; b0 += kWarpMsgBytes / 136) {
    const uint32_t wb = min((uint32_t)(kWarpMsgBytes / 136), nblk - b0);
    const uint32_t lo = b0 * 136, hi = lo + wb * 136;
    for (uint32_t w = lane; w < wb * 17; w += 32) m64[w] = 0;
    __syncwarp();
    if (lane == 0)
      for (uint32_t q = 0; q < hn; ++q)
        if (q >= lo && q < hi) msg[q - lo] = (uint8_t)(hdr >> (8 * q));
    // items in order; the lanes share each item's bytes that fall in the window
    for (int k = 0; k < 17; ++k) {
      const uint32_t p = __shfl_sync(kAll, my_off, k);
      const uint32_t pren = __shfl_sync(kAll, it.pren, k);
      const uint32_t blen = __shfl_sync(kAll, it.blen, k);
      const uint64_t pre = __shfl_sync(kAll, it.pre, k);
      const uint8_t *body = reinterpret_cast<const uint8_t *>(
          __shfl_sync(kAll, reinterpret_cast<unsigned long long>(it.body), k));
      const uint32_t n = pren + blen;
      if (p >= hi || p + n <= lo) continue;
      const uint32_t j0 = lo > p ? lo - p : 0u, j1 = min(n, hi - p);
      for (uint32_t j = j0 + (uint32_t)lane; j < j1; j += 32)
        msg[p + j - lo] = j < pren ? (uint8_t)(pre >> (8 * j)) : ldn<kCoh>(body + (j - pren));
    }
    __syncwarp();
    if (raw) break;  // under 32 bytes: the window holds the whole encoding
    if (lane == 0) {  // Keccak padding (pad byte 0x01 ... last byte |= 0x80)
      if (total >= lo && total < hi) msg[total - lo] ^= 0x01;
      if (padded - 1 >= lo && padded - 1 < hi) msg[padded - 1 - lo] ^= 0x80;
    }
    __syncwarp();
    for (uint32_t bb = 0; bb < wb; ++bb) {
      if (lane < 17) a ^= m64[bb * 17 + lane];
      a = keccak_f1600_warp(a, cl, lane);
    }
    __syncwarp();  // the next window reuses the buffer
  }
  uint64_t *o = reinterpret_cast<uint64_t *>(tv.full_hash + (size_t)idx * 32);
  if (raw) {
    if (lane < 4) o[lane] = m64[lane];  // zero beyond total
    if (lane == 0) tv.full_hlen[idx] = (uint8_t)total;
  } else {
    if (lane < 4) o[lane] = a;
    if (lane == 0) tv.full_hlen[idx] = 32;
  }
  if (lane == 0 && tv.account) {
    atomicAdd(&tv.ctr->enc_bytes, (unsigned long long)total);
    atomicAdd(&tv.ctr->keccak_blocks, (unsigned long long)(raw ? 0u : nblk));
    atomicAdd(&tv.ctr->hashed, 1u);
  }
  __syncwarp();
}

// Branch nodes one warp each (a level's branches when it has few, or its
// branches of many blocks): 4 warps per CTA.
__global__ void __launch_bounds__(128) k_hash_full_warp(TrieView tv, const uint32_t *refs, int count) {
  extern __shared__ uint64_t msg_all[];  // one message window per warp
  const int j = blockIdx.x * 4 + (threadIdx.x >> 5);
  if (j >= count) return;  // whole warps leave together
  uint8_t *msg = reinterpret_cast<uint8_t *>(msg_all) + (threadIdx.x >> 5) * kWarpMsgBytes;
  const CoopLanes cl = coop_lanes(threadIdx.x & 31);
  hash_full_warp<false>(tv, ref_idx(refs[j]), msg, cl);
}

// Six 128-thread CTAs per SM (at most 85 registers): the permutation keeps
// its 25 lanes in registers; a few encoder temporaries spill, and the extra
// resident warps hide more of the child / record gathers (measured faster
// than five CTAs at 96 registers without spills).
// One level, thread per node; the CTA's 128 nodes are first reordered by
// hash class (stable counting partition from warp ballots), so warps hold
// nodes of one Keccak block count.
constexpr int kHashLevelThreads = 128;  // k_hash_level's block size (the partition assumes it)

#ifndef GMPT_HASH_CTAS
#define GMPT_HASH_CTAS 6
#endif
__device__ __forceinline__ void hash_level_cta(const TrieView &tv, const uint32_t *refs, int count) {
  extern __shared__ uint64_t stage_all[];
  __shared__ uint32_t s_ref[kHashLevelThreads];
  __shared__ uint32_t s_cnt[kCtaClasses][kHashLevelThreads / 32];  // [class][warp]
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool valid = t < count;
  const uint32_t r = valid ? refs[t] : 0u;
  const uint32_t c = valid ? hash_class(tv, r) : kCtaClasses;
  uint32_t mine = 0;
#pragma unroll
  for (uint32_t v = 0; v < kCtaClasses; ++v) {
    const unsigned b = __ballot_sync(0xffffffffu, c == v);
    if (lane == 0) s_cnt[v][warp] = (uint32_t)__popc(b);
    if (c == v) mine = (uint32_t)__popc(b & ((1u << lane) - 1u));
  }
  __syncthreads();
  if (valid) {
    uint32_t pos = mine;
    for (uint32_t v = 0; v < kCtaClasses; ++v)
      for (int w = 0; w < kHashLevelThreads / 32; ++w)
        if (v < c || (v == c && w < warp)) pos += s_cnt[v][w];
    s_ref[pos] = r;
  }
  __syncthreads();
  if (!valid) return;  // the valid nodes fill s_ref[0 .. valid count)
  hash_node<false>(tv, s_ref[threadIdx.x], stage_all + threadIdx.x, blockDim.x);
}

// The level kernel at the register budget of six resident CTAs per SM (the
// throughput form), and with the whole register file open to one CTA per
// SM: a level too small to fill the SMs is as long as the serial Keccak
// chain of its longest node, which the wider form schedules with more
// permutation state in flight.
__global__ void __launch_bounds__(kHashLevelThreads, GMPT_HASH_CTAS) k_hash_level(TrieView tv, const uint32_t *refs,
                                                                                 int count) {
  hash_level_cta(tv, refs, count);
}

__global__ void __launch_bounds__(kHashLevelThreads, 1) k_hash_level_wide(TrieView tv, const uint32_t *refs, int count) {
  hash_level_cta(tv, refs, count);
}

// ---------------------------------------------------------------------------
// gets (gpu_mpt_kernels.cuh:2267-2340)

__device__ __forceinline__ int64_t lookup(const TrieView &tv, uint32_t root, const uint8_t *kb, uint32_t len) {
  uint32_t ref = root;
  uint32_t x = 0;
  for (uint32_t guard = 0; guard <= len + 1; ++guard) {
    uint32_t kind = ref_kind(ref), idx = ref_idx(ref);
    if (kind == KIND_NULL) return -1;
    if (kind == KIND_VALUE) return x == len ? (int64_t)tv.value_vid[idx] : -1;
    if (kind == KIND_FULL) {
      if (x >= len) return -1;
      uint32_t c = kb[x];
      if (c > 16) return -1;
      ref = tv.full_child[(size_t)idx * 17 + c];
      ++x;
      continue;
    }
    uint32_t sl = tv.short_klen[idx];
    if (len - x < sl) return -1;
    if ((uint32_t)match_nibbles(tv.keys + tv.short_key[idx], kb + x, (int)sl) != sl) return -1;
    x += sl;
    ref = tv.short_child[idx];
  }
  return -1;
}

__global__ void k_gets(TrieView tv, const uint8_t *keys, const int *idx, int n, int64_t keys_bytes,
                       uint64_t *out_hp, int *out_len, int64_t *out_vid, const int *tid) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int ks = idx[2 * i], ke = idx[2 * i + 1];
  int len = ke - ks + 1;
  const uint32_t tr = tid ? (uint32_t)tid[i] : 0u;
  bool ok = ks >= 0 && len > 0 && (int64_t)ke < keys_bytes && tr < tv.n_tries;
  int64_t vid = ok ? lookup(tv, tv.roots[tr], keys + ks, (uint32_t)len) : -1;
  if (out_vid) out_vid[i] = vid;
  if (vid < 0) {
    out_hp[i] = 0;
    out_len[i] = 0;
  } else {
    out_hp[i] = tv.rec_hp[vid];
    out_len[i] = (int)tv.rec[vid].len;
  }
}

// Root bytes of trie ids[i] (or trie i when ids is null) into out[33 i ..]:
// 32 bytes (zero-padded) and the length (0 = empty trie).  Warp per trie.
__global__ void k_roots(TrieView tv, const int *ids, int n, uint8_t *out) {
  const int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (i >= n) return;
  const int t = threadIdx.x & 31;
  const uint32_t tr = ids ? (uint32_t)ids[i] : (uint32_t)i;
  out += 33 * (size_t)i;
  uint32_t r = tr < tv.n_tries ? tv.roots[tr] : 0u;
  uint32_t kind = ref_kind(r), idx = ref_idx(r);
  uint32_t len = 0;
  const uint8_t *h = nullptr;
  if (kind == KIND_FULL) {
    h = tv.full_hash + (size_t)idx * 32;
    len = tv.full_hlen[idx];
  } else if (kind == KIND_SHORT) {
    h = tv.short_hash + (size_t)idx * 32;
    len = tv.short_hlen[idx];
  } else if (kind == KIND_VALUE) {
    unsigned long long vid = tv.value_vid[idx];
    const ValueRec rc = tv.rec[vid];
    h = tv.vals + rc.off;
    len = min(32u, rc.len);
  }
  out[t] = (h && (uint32_t)t < len) ? h[t] : 0;
  if (t == 0) out[32] = (uint8_t)len;
}

}  // namespace gmpt
