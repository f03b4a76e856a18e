// latch_kernels.cuh -- LockNU: concurrent per-key insert on the live trie.
//
// The reference's LockNU (puts_latching_v2, gpu_mpt_kernels.cuh:1573-1605 ->
// put_olc_v2 :971-1228) runs one warp per key with only lane 0 working and
// optimistic lock coupling (version word read-lock / validate / upgrade CAS,
// node.cuh:360-396) with an unbounded restart loop.  Here one thread inserts
// one key and nodes are never modified after they are published, except a
// branch's child slots and a value node's record id:
//   * an empty slot is filled with a CAS from null to a new leaf;
//   * a short node that must be split is replaced as a whole: the new upper
//     extension / branch / remainder / own leaf are built privately and
//     swung into the parent slot with one CAS (the old node is marked dead);
//   * an existing key takes max(record id), i.e. the last batch position of
//     the key wins, whatever order the threads run in.
// A failed CAS re-reads the same slot; the number of failures per key is
// bounded and exceeding it raises ERR_RETRY_LIMIT instead of spinning.
#pragma once
#include "common.cuh"
#include "trie_kernels.cuh"

namespace gmpt {

__device__ __forceinline__ uint32_t load_slot(const uint32_t *p) {
  return *reinterpret_cast<const volatile uint32_t *>(p);
}

// Pool slots are taken warp-aggregated among the lanes that allocate
// together (one atomic per warp on the pool counter, not one per lane).
__device__ __forceinline__ uint32_t alloc_short(const TrieView &tv) {
  uint32_t s = warp_alloc(&tv.ctr->n_short, 1u);
  if (s >= tv.cap_short) {
    set_error(tv.ctr, ERR_CAPACITY);
    return 0xFFFFFFFFu;
  }
  return s;
}

__device__ __forceinline__ uint32_t alloc_full(const TrieView &tv) {
  uint32_t f = warp_alloc(&tv.ctr->n_full, 1u);
  if (f >= tv.cap_full) {
    set_error(tv.ctr, ERR_CAPACITY);
    return 0xFFFFFFFFu;
  }
  return f;
}

__device__ __forceinline__ void init_short(const TrieView &tv, uint32_t s, uint64_t key_off, uint32_t klen,
                                           uint32_t child, uint32_t depth, uint32_t gen) {
  tv.short_key[s] = key_off;
  tv.short_klen[s] = klen;
  tv.short_child[s] = child;
  tv.short_depth[s] = (uint16_t)depth;
  tv.short_epoch[s] = gen;
  tv.short_dead[s] = 0;
  tv.short_claim[s] = 0;
  tv.short_hlen[s] = 0;
}

// Insert key i continuing from slot `sp` at nibble depth `x` (the root and
// depth 0 for a fresh start): CAS-based, retries bounded by retry_limit.
__device__ __noinline__ void latch_from(TrieView tv, DirtyList dl, uint32_t *sp, uint32_t x, uint64_t ko,
                                        uint32_t len, unsigned long long vid, uint32_t retry_limit) {
  const uint32_t gen = tv.gen;
  const uint8_t *kb = tv.keys + ko;
  uint32_t vnode = 0xFFFFFFFFu, leaf = 0xFFFFFFFFu, br = 0xFFFFFFFFu, up = 0xFFFFFFFFu, left = 0xFFFFFFFFu;
  uint32_t fails = 0;
  for (uint32_t guard = 0; guard < len + 2 + retry_limit; ++guard) {
    uint32_t ref = load_slot(sp);
    uint32_t kind = ref_kind(ref), idx = ref_idx(ref);
    if (kind == KIND_NULL) {
      if (vnode == 0xFFFFFFFFu) {
        vnode = warp_alloc(&tv.ctr->n_value, 1u);
        if (vnode >= tv.cap_value) {
          set_error(tv.ctr, ERR_CAPACITY);
          return;
        }
        tv.value_vid[vnode] = vid;
      }
      uint32_t vref = make_ref(KIND_VALUE, vnode);
      uint32_t nref = vref;
      if (x < len) {
        if (leaf == 0xFFFFFFFFu && (leaf = alloc_short(tv)) == 0xFFFFFFFFu) return;
        init_short(tv, leaf, ko + x, len - x, vref, x, gen);
        nref = make_ref(KIND_SHORT, leaf);
      }
      __threadfence();
      if (atomicCAS(sp, 0u, nref) == 0u) {
        if (x < len) dirty_push(tv.ctr, dl, nref, x);
        return;
      }
      if (++fails > retry_limit) break;
      continue;
    }
    if (kind == KIND_FULL) {
      mark_full(tv, dl, idx, gen);
      if (x >= len) break;
      uint32_t c = kb[x];
      sp = tv.full_child + (size_t)idx * 17 + c;
      ++x;
      continue;
    }
    if (kind == KIND_VALUE) {
      if (x != len) break;
      atomicMax(&tv.value_vid[idx], vid);
      return;
    }
    // short node
    const uint64_t sko = __ldcg(tv.short_key + idx);
    const uint32_t sl = __ldcg(tv.short_klen + idx);
    const uint32_t schild = __ldcg(tv.short_child + idx);
    const uint8_t *sk = tv.keys + sko;
    uint32_t lim = min(sl, len - x);
    uint32_t mm = (uint32_t)match_nibbles(sk, kb + x, (int)lim);
    if (mm == sl) {
      mark_short(tv, dl, idx, gen);
      sp = tv.short_child + idx;
      x += sl;
      continue;
    }
    if (mm == len - x) break;  // key is a prefix of a stored key
    // split: [up(key[0..mm))] -> br{ sk[mm]: left/rest, kb[x+mm]: own leaf }
    if (br == 0xFFFFFFFFu && (br = alloc_full(tv)) == 0xFFFFFFFFu) return;
    uint32_t bd = x + mm;
    uint32_t *ch = tv.full_child + (size_t)br * 17;
#pragma unroll
    for (int c = 0; c < 17; ++c) ch[c] = 0;
    tv.full_depth[br] = (uint16_t)bd;
    tv.full_epoch[br] = gen;
    tv.full_hlen[br] = 0;
    tv.full_dead[br] = 0;
    // the old node's remainder
    uint32_t rest = schild;
    bool use_left = sl - mm - 1 > 0;
    if (use_left) {
      if (left == 0xFFFFFFFFu && (left = alloc_short(tv)) == 0xFFFFFFFFu) return;
      init_short(tv, left, sko + mm + 1, sl - mm - 1, schild, bd + 1, gen);
      rest = make_ref(KIND_SHORT, left);
    }
    ch[sk[mm]] = rest;
    // this key's leaf
    if (vnode == 0xFFFFFFFFu) {
      vnode = warp_alloc(&tv.ctr->n_value, 1u);
      if (vnode >= tv.cap_value) {
        set_error(tv.ctr, ERR_CAPACITY);
        return;
      }
      tv.value_vid[vnode] = vid;
    }
    uint32_t own = make_ref(KIND_VALUE, vnode);
    bool use_leaf = bd + 1 < len;
    if (use_leaf) {
      if (leaf == 0xFFFFFFFFu && (leaf = alloc_short(tv)) == 0xFFFFFFFFu) return;
      init_short(tv, leaf, ko + bd + 1, len - bd - 1, own, bd + 1, gen);
      own = make_ref(KIND_SHORT, leaf);
    }
    ch[kb[bd]] = own;
    uint32_t top = make_ref(KIND_FULL, br);
    if (mm > 0) {
      if (up == 0xFFFFFFFFu && (up = alloc_short(tv)) == 0xFFFFFFFFu) return;
      init_short(tv, up, sko, mm, top, x, gen);
      top = make_ref(KIND_SHORT, up);
    }
    __threadfence();
    if (atomicCAS(sp, ref, top) == ref) {
      tv.short_dead[idx] = 1;
      dirty_push(tv.ctr, dl, make_ref(KIND_FULL, br), bd);
      if (use_left) dirty_push(tv.ctr, dl, make_ref(KIND_SHORT, left), bd + 1);
      if (use_leaf) dirty_push(tv.ctr, dl, make_ref(KIND_SHORT, leaf), bd + 1);
      if (mm > 0) dirty_push(tv.ctr, dl, make_ref(KIND_SHORT, up), x);
      return;
    }
    if (++fails > retry_limit) break;
  }
  if (fails > retry_limit)
    set_error(tv.ctr, ERR_RETRY_LIMIT);
  else
    set_error(tv.ctr, ERR_BAD_KEY);
}

// Thread per kLatchWays keys: the keys advance one node per round together,
// so a thread keeps several independent pointer chases in flight.  The
// read-only descent marks the path dirty and resolves keys that exist
// (atomicMax of the record id); a key that needs a new leaf or a split is
// handed to latch_from at the slot where its descent stopped.
constexpr int kLatchWays = 4;

// Which keys a LockNU launch walks: all of [0, n), or (dedup) the positions
// sel[0 .. *count) -- the last occurrence of every distinct key -- unless
// *collision is set, in which case all keys are walked after all.
struct KeySelect {
  const uint32_t *sel = nullptr;
  const unsigned long long *count = nullptr;
  const uint32_t *collision = nullptr;
};

// Keys t + w * nthreads (w < kWays) of koff/klen[0..n) (or of the selected
// positions), record ids vid_base + i, trie ids tid[i] (null: trie 0).
template <int kWays = kLatchWays>
__device__ __forceinline__ void latch_keys(const TrieView &tv, DirtyList dl, const uint64_t *koff,
                                           const uint32_t *klen, int n, uint64_t vid_base, uint32_t retry_limit,
                                           const int *tid, int t, int nthreads, KeySelect ks = KeySelect()) {
  const uint32_t gen = tv.gen;
  const uint32_t *sel = ks.sel;
  int n_eff = n;
  if (sel) {
    if (*ks.collision)
      sel = nullptr;
    else
      n_eff = (int)(*ks.count & 0xFFFFFFFFull);
  }
  uint32_t *sp[kWays];
  uint32_t x[kWays], len[kWays], key[kWays];
  uint64_t ko[kWays];
  uint8_t st[kWays];  // 0 done, 1 walking, 2 hand off to latch_from
#pragma unroll
  for (int w = 0; w < kWays; ++w) {
    const int j = t + w * nthreads;
    const bool on = j < n_eff;
    const int i = on ? (sel ? (int)sel[j] : j) : 0;
    key[w] = (uint32_t)i;
    st[w] = on ? 1 : 0;
    sp[w] = tv.roots + ((on && tid) ? tid[i] : 0);
    x[w] = 0;
    ko[w] = on ? koff[i] : 0;
    len[w] = on ? klen[i] : 0;
  }
  // Each round moves every walking key down one node in phases, so the loads
  // of all ways are in flight together: (1) slot + node fields + dirty
  // epoch, (2) key comparison chunks of short nodes, (3) advance / resolve,
  // (4) dirty marks (their atomics are off the descent's critical path).
  for (int round = 0; round < kMaxKeyNibbles + 2; ++round) {
    uint32_t ref[kWays], ep[kWays], nib[kWays], sl[kWays];
    uint64_t sko[kWays];
#pragma unroll
    for (int w = 0; w < kWays; ++w) ref[w] = st[w] == 1 ? __ldcg(sp[w]) : 0u;
#pragma unroll
    for (int w = 0; w < kWays; ++w) {
      const uint32_t kind = ref_kind(ref[w]), idx = ref_idx(ref[w]);
      ep[w] = gen;
      nib[w] = 0;
      sl[w] = 0;
      sko[w] = 0;
      if (st[w] != 1) continue;
      if (kind == KIND_FULL) {
        ep[w] = __ldcg(tv.full_epoch + idx);
        nib[w] = x[w] < len[w] ? tv.keys[ko[w] + x[w]] : 0u;
      } else if (kind == KIND_SHORT) {
        ep[w] = __ldcg(tv.short_epoch + idx);
        sko[w] = __ldcg(tv.short_key + idx);
        sl[w] = __ldcg(tv.short_klen + idx);
      }
    }
    // short nodes: compare the key chunk by chunk, all ways together
    uint32_t lim[kWays], mm[kWays];
    bool cmp[kWays];
#pragma unroll
    for (int w = 0; w < kWays; ++w) {
      cmp[w] = st[w] == 1 && ref_kind(ref[w]) == KIND_SHORT;
      lim[w] = cmp[w] ? min(sl[w], len[w] - x[w]) : 0u;
      mm[w] = 0;
    }
    for (int c = 0; c < kMaxKeyNibbles / 8 + 1; ++c) {
      bool more = false;
#pragma unroll
      for (int w = 0; w < kWays; ++w) {
        if (!cmp[w]) continue;
        const uint32_t o = 8u * c;
        if (o >= lim[w]) {
          mm[w] = lim[w];
          cmp[w] = false;
          continue;
        }
        uint64_t d = load_u64_unaligned(tv.keys + sko[w] + o) ^ load_u64_unaligned(tv.keys + ko[w] + x[w] + o);
        d &= low_mask64((int)min(8u, lim[w] - o));
        if (d) {
          mm[w] = o + (__ffsll((long long)d) - 1) / 8;
          cmp[w] = false;
        } else {
          more = true;
        }
      }
      if (!more) break;
    }
    bool any = false;
#pragma unroll
    for (int w = 0; w < kWays; ++w) {
      if (st[w] != 1) continue;
      const uint32_t kind = ref_kind(ref[w]), idx = ref_idx(ref[w]);
      if (kind == KIND_FULL) {
        if (x[w] >= len[w]) {
          st[w] = 2;
          continue;
        }
        sp[w] = tv.full_child + (size_t)idx * 17 + nib[w];
        ++x[w];
        any = true;
      } else if (kind == KIND_SHORT) {
        if (mm[w] != sl[w]) {
          st[w] = 2;  // split (or a malformed key): CAS path
          ep[w] = gen;  // a node being replaced is not marked here
          continue;
        }
        sp[w] = tv.short_child + idx;
        x[w] += sl[w];
        any = true;
      } else if (kind == KIND_VALUE && x[w] == len[w]) {
        atomicMax(&tv.value_vid[idx], vid_base + (unsigned long long)key[w]);
        st[w] = 0;
      } else {
        st[w] = 2;  // empty slot (new leaf) or malformed key
      }
    }
#pragma unroll
    for (int w = 0; w < kWays; ++w) {
      if (ep[w] == gen) continue;
      const uint32_t kind = ref_kind(ref[w]), idx = ref_idx(ref[w]);
      if (kind == KIND_FULL) {
        if (atomicExch(&tv.full_epoch[idx], gen) != gen)
          dirty_push(tv.ctr, dl, ref[w], __ldcg(tv.full_depth + idx));
      } else if (kind == KIND_SHORT) {
        if (atomicExch(&tv.short_epoch[idx], gen) != gen)
          dirty_push(tv.ctr, dl, ref[w], __ldcg(tv.short_depth + idx));
      }
    }
    if (!any) break;
  }
#pragma unroll
  for (int w = 0; w < kWays; ++w)
    if (st[w] != 0)
      latch_from(tv, dl, sp[w], x[w], ko[w], len[w], vid_base + (unsigned long long)key[w], retry_limit);
}

#ifndef GMPT_LATCH_CTAS
#define GMPT_LATCH_CTAS 2
#endif

template <int kWays>
__global__ void __launch_bounds__(256, GMPT_LATCH_CTAS) k_latch_insert(TrieView tv, DirtyList dl, const uint64_t *koff,
                                                      const uint32_t *klen, int n, uint64_t vid_base,
                                                      uint32_t retry_limit, const int *tid, KeySelect ks) {
  latch_keys<kWays>(tv, dl, koff, klen, n, vid_base, retry_limit, tid, blockIdx.x * blockDim.x + threadIdx.x,
                    gridDim.x * blockDim.x, ks);
}

// ---------------------------------------------------------------------------
// Batch dedup before LockNU: a duplicate-heavy batch (zipf updates) walks the
// trie once per distinct key instead of once per occurrence.  An
// open-addressing table keyed by a 64-bit hash of (trie, key nibbles) keeps
// the largest batch position per hash (= the occurrence that must win); a
// second pass compares every other occurrence's key with its slot's winner,
// and a mismatch (two different keys with one hash) sets *collision, which
// makes the insert walk every key as if there were no dedup.  Results never
// depend on the hash.

constexpr unsigned long long kDedupEmpty = 0ull;

// Slot s is two 8-byte words, [2s] the key hash (0 = free) and [2s + 1] the
// largest batch position with that hash (low 32 bits), so a probe touches one
// 16-byte pair: one DRAM sector per key instead of one per array.
struct DedupTable {
  unsigned long long *slot;  // [2 * size], zeroed = every slot free
  uint64_t mask;             // size - 1 (size a power of two)
  uint64_t hmask;            // hash bits kept (narrower only to test collisions)
  __device__ __forceinline__ unsigned long long *hash(uint64_t s) const { return slot + 2 * s; }
  __device__ __forceinline__ uint32_t *pos(uint64_t s) const { return reinterpret_cast<uint32_t *>(slot + 2 * s + 1); }
};

__device__ __forceinline__ uint64_t dedup_hash(const uint8_t *k, uint32_t len, uint32_t trie, uint64_t hmask) {
  uint64_t h = 0x9E3779B97F4A7C15ull ^ ((uint64_t)len << 32) ^ trie;
  uint32_t o = 0;
  for (; o + 8 <= len; o += 8) {
    h = (h ^ load_u64_unaligned(k + o)) * 0xFF51AFD7ED558CCDull;
    h ^= h >> 32;
  }
  if (o < len) {
    h = (h ^ (load_u64_unaligned(k + o) & low_mask64((int)(len - o)))) * 0xC4CEB9FE1A85EC53ull;
    h ^= h >> 29;
  }
  h = (h ^ (h >> 31)) * 0x94D049BB133111EBull;
  h ^= h >> 32;
  h &= hmask;
  return h == kDedupEmpty ? 1ull : h;
}

__device__ __forceinline__ uint64_t dedup_home(uint64_t h, uint64_t mask) {
  return ((h ^ (h >> 29)) * 0xBF58476D1CE4E5B9ull >> 17) & mask;
}

constexpr uint32_t kNoSlot = 0xFFFFFFFFu;

// slot_of[i] = the slot key i's hash landed in (kNoSlot if the table was
// full), so the passes after it need not hash and probe again
__global__ void k_dedup_insert(TrieView tv, const uint64_t *koff, const uint32_t *klen, const int *tid, int n,
                               DedupTable t, uint32_t *slot_of) {
  // batch positions from the last one down: CTAs start roughly in order, so
  // a zipf-hot key's latest occurrences claim its slot first and the earlier
  // ones find a larger position there and skip the atomic (front to back,
  // every occurrence of a key repeated a million times would raise the slot
  // in turn, one atomic after another on the same address)
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n) return;
  const int i = n - 1 - u;
  const unsigned long long h = dedup_hash(tv.keys + koff[i], klen[i], tid ? (uint32_t)tid[i] : 0u, t.hmask);
  uint64_t s = dedup_home(h, t.mask);
  for (uint64_t probe = 0; probe <= t.mask; ++probe, s = (s + 1) & t.mask) {
    // read before the atomics: a zipf-hot key repeats up to millions of
    // times, and a CAS or max that cannot change the slot would serialise
    // every one of them on the same address
    unsigned long long old = __ldcg(t.hash(s));
    if (old == kDedupEmpty) old = atomicCAS(t.hash(s), kDedupEmpty, h);
    if (old == kDedupEmpty || old == h) {
      if (__ldcg(t.pos(s)) < (uint32_t)i) atomicMax(t.pos(s), (uint32_t)i);
      slot_of[i] = (uint32_t)s;
      return;
    }
  }
  slot_of[i] = kNoSlot;
}

__global__ void k_dedup_mark(TrieView tv, const uint64_t *koff, const uint32_t *klen, const int *tid, int n,
                             DedupTable t, const uint32_t *slot_of, unsigned long long *keep, uint32_t *collision) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t tr = tid ? (uint32_t)tid[i] : 0u;
  const uint8_t *k = tv.keys + koff[i];
  const uint32_t len = klen[i];
  const uint32_t s = slot_of[i];
  if (s == kNoSlot) {  // cannot happen (the table has 2n slots); walk every key then
    atomicOr(collision, 1u);
    keep[i] = 1ull;
    return;
  }
  const uint32_t w = *t.pos(s);
  bool kept = w == (uint32_t)i;
  if (!kept) {
    const bool same = klen[w] == len && (tid ? (uint32_t)tid[w] == tr : true) &&
                      match_nibbles(tv.keys + koff[w], k, (int)len) == (int)len;
    if (!same) atomicOr(collision, 1u);
  }
  keep[i] = kept ? 1ull : 0ull;
}

// Mixed read/write batches: the hash-table slot of every key (k_dedup_insert
// filled the table) as the sort key of a stable radix sort, which then groups
// equal keys in batch order.  A key unequal to its slot's representative (a
// hash collision) sets *collision: the caller sorts by full keys instead.
__global__ void k_rw_slots(TrieView tv, const uint64_t *koff, const uint32_t *klen, const int *tid, int n,
                           DedupTable t, const uint32_t *slot_of, uint64_t *skey, uint32_t *sval,
                           uint32_t *collision) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t tr = tid ? (uint32_t)tid[i] : 0u;
  const uint8_t *k = tv.keys + koff[i];
  const uint32_t len = klen[i];
  uint32_t s = slot_of[i];
  const bool found = s != kNoSlot;
  if (!found) {
    atomicOr(collision, 1u);
    s = 0;
  } else {
    const uint32_t w = *t.pos(s);
    if (w != (uint32_t)i) {
      const bool same = klen[w] == len && (tid ? (uint32_t)tid[w] == tr : true) &&
                        match_nibbles(tv.keys + koff[w], k, (int)len) == (int)len;
      if (!same) atomicOr(collision, 1u);
    }
  }
  skey[i] = s;
  sval[i] = (uint32_t)i;
}

// Repeated keys in an evenly spaced sample of a batch (key hashes in a small
// open-addressing table of tmask + 1 slots): PhaseNU drops a batch's repeats
// before sorting when the sample shows many (runs of one key repeated
// thousands of times otherwise keep the chunked sort going to the last
// chunk).
__global__ void k_dup_sample(const uint8_t *keys, const uint64_t *koff, const uint32_t *klen, const int *tid,
                             int samples, int stride, unsigned long long *table, uint32_t tmask, uint32_t *dups) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= samples) return;
  const int i = j * stride;
  const unsigned long long h = dedup_hash(keys + koff[i], klen[i], tid ? (uint32_t)tid[i] : 0u, ~0ull);
  uint32_t s = (uint32_t)(h ^ (h >> 32)) & tmask;
  for (uint32_t probe = 0; probe <= tmask; ++probe, s = (s + 1) & tmask) {
    const unsigned long long old = atomicCAS(&table[s], kDedupEmpty, h);
    if (old == kDedupEmpty) return;
    if (old == h) {
      atomicAdd(dups, 1u);
      return;
    }
  }
}

__global__ void k_dedup_compact(const unsigned long long *keep, const unsigned long long *pos, int n, uint32_t *sel) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && keep[i]) sel[pos[i]] = (uint32_t)i;
}

}  // namespace gmpt
