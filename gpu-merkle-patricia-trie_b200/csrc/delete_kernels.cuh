// delete_kernels.cuh -- batched deletes.
//
// The reference has no delete path (no delete anywhere in gpu_mpt.cuh /
// cpu_mpt.cuh); go-ethereum deletes empty accounts and zeroed storage slots,
// so a drop-in for its commits needs one.  The result must be the canonical
// trie of the remaining keys:
//   1. k_del_walk (thread per key): walk to the key; unlink its leaf (or clear
//      the value slot of the branch where it ends); mark every node on the
//      path dirty and stamp each branch on it with how it is linked: the
//      slot holding it (or holding the extension right above it) and that
//      extension.
//   2. k_del_collapse (per nibble depth, deepest first, over the stamped
//      dirty branches): a branch left with no child is unlinked (with its
//      extension); one left with a single child becomes a short node whose
//      key is [extension key] + slot nibble + [the child's key if the child
//      is a short node]: the extension is rewritten in place, else a new
//      short node takes the branch's slot.  Deeper levels finish first, so a
//      branch sees its children's final form.
//   3. PhaseHC rehashes the dirty nodes (dead short nodes are skipped).
#pragma once
#include "trie_kernels.cuh"

namespace gmpt {

constexpr uint32_t kNoExt = 0xFFFFFFFFu;

__global__ void k_del_walk(TrieView tv, DirtyList dl, const uint8_t *keys, const int *idx, int n, int64_t keys_bytes,
                           const int *tid, uint64_t *hslot, uint32_t *hext, uint8_t *stamp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int ks = idx[2 * i], ke = idx[2 * i + 1];
  const int len = ke - ks + 1;
  if (ks < 0 || len <= 0 || (int64_t)ke >= keys_bytes || len > kMaxKeyNibbles) {
    set_error(tv.ctr, ERR_BAD_KEY);
    return;
  }
  const uint32_t tr = tid ? (uint32_t)tid[i] : 0u;
  if (tr >= tv.n_tries) {
    set_error(tv.ctr, ERR_BAD_TRIE);
    return;
  }
  const uint8_t *kb = keys + ks;
  const uint32_t gen = tv.gen;
  uint64_t slot = root_slot(tr);  // holds the current node, or the extension above it
  uint32_t ref = tv.roots[tr];
  uint32_t ext = kNoExt;
  uint32_t x = 0;
  for (int guard = 0; guard <= len + 1; ++guard) {
    const uint32_t kind = ref_kind(ref), id = ref_idx(ref);
    if (kind == KIND_NULL || kind == KIND_VALUE) return;  // absent
    if (kind == KIND_FULL) {
      mark_full(tv, dl, id, gen);
      hslot[id] = slot;
      hext[id] = ext;
      stamp[id] = 1;
      if (x >= (uint32_t)len) return;
      const uint32_t c = kb[x];
      if (c > 16) return;
      if (c == 16) {  // the key ends at this branch: its value slot
        if (x + 1 == (uint32_t)len && ref_kind(tv.full_child[(size_t)id * 17 + 16]) == KIND_VALUE)
          tv.full_child[(size_t)id * 17 + 16] = 0u;
        return;
      }
      slot = ((uint64_t)id << 5) | c;
      ref = tv.full_child[(size_t)id * 17 + c];
      ext = kNoExt;
      ++x;
      continue;
    }
    // short node
    const uint32_t sl = tv.short_klen[id];
    if ((uint32_t)len - x < sl) return;
    if ((uint32_t)match_nibbles(tv.keys + tv.short_key[id], kb + x, (int)sl) != sl) return;
    const uint32_t child = tv.short_child[id];
    if (ref_kind(child) == KIND_VALUE) {
      if (x + sl == (uint32_t)len) {  // found: unlink the leaf
        tv.short_dead[id] = 1;
        write_slot(tv, slot, 0u);
      }
      return;
    }
    mark_short(tv, dl, id, gen);
    ext = id;  // `slot` keeps holding the extension
    x += sl;
    ref = child;
  }
}

// Key bytes the collapses of one level will append (same rule as below).
__global__ void k_del_need(TrieView tv, const uint32_t *refs, int count, const uint32_t *hext, const uint8_t *stamp,
                           unsigned long long *need) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t total = 0;
  if (j < count && ref_kind(refs[j]) == KIND_FULL && stamp[ref_idx(refs[j])]) {
    const uint32_t id = ref_idx(refs[j]);
    const uint32_t *ch = tv.full_child + (size_t)id * 17;
    uint32_t cnt = 0, c1 = 0, r1 = 0;
    for (uint32_t k = 0; k < 17; ++k) {
      const uint32_t v = ch[k];
      if (v) {
        ++cnt;
        c1 = k;
        r1 = v;
      }
    }
    if (cnt == 1) {
      const uint32_t e = hext[id];
      total = 1u + (e != kNoExt ? tv.short_klen[e] : 0u) +
              ((c1 < 16 && ref_kind(r1) == KIND_SHORT) ? tv.short_klen[ref_idx(r1)] : 0u);
    }
  }
  const unsigned long long w = __reduce_add_sync(0xffffffffu, total);
  if ((threadIdx.x & 31) == 0 && w) atomicAdd(need, w);
}

__global__ void k_del_collapse(TrieView tv, DirtyList dl, const uint32_t *refs, int count, const uint64_t *hslot,
                               const uint32_t *hext, const uint8_t *stamp, unsigned long long *key_cursor,
                               uint64_t key_cap) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= count) return;
  const uint32_t r = refs[j];
  if (ref_kind(r) != KIND_FULL) return;
  const uint32_t id = ref_idx(r);
  if (!stamp[id]) return;  // dirty from an earlier put, not on a deleted key's path
  const uint32_t *ch = tv.full_child + (size_t)id * 17;
  uint32_t cnt = 0, c1 = 0, r1 = 0;
  for (uint32_t k = 0; k < 17; ++k) {
    const uint32_t v = ch[k];
    if (v) {
      ++cnt;
      c1 = k;
      r1 = v;
    }
  }
  if (cnt >= 2) return;
  const uint64_t hs = hslot[id];
  const uint32_t e = hext[id];
  tv.full_dead[id] = 1;  // unlinked below, or replaced by a short node
  if (cnt == 0) {  // nothing left below: unlink the branch and its extension
    if (e != kNoExt) tv.short_dead[e] = 1;
    write_slot(tv, hs, 0u);
    return;
  }
  // one child left: key = [extension key] + c1 + [child short node's key]
  uint32_t child = r1, le = 0, ls = 0;
  uint64_t oe = 0, os = 0;
  if (e != kNoExt) {
    oe = tv.short_key[e];
    le = tv.short_klen[e];
  }
  if (c1 < 16 && ref_kind(r1) == KIND_SHORT) {
    const uint32_t s = ref_idx(r1);
    os = tv.short_key[s];
    ls = tv.short_klen[s];
    child = tv.short_child[s];
    tv.short_dead[s] = 1;
  }
  const uint32_t total = le + 1u + ls;
  const unsigned long long off = atomicAdd(key_cursor, (unsigned long long)total);
  if (off + total > key_cap) {
    set_error(tv.ctr, ERR_CAPACITY);
    return;
  }
  uint8_t *dst = const_cast<uint8_t *>(tv.keys) + off;
  for (uint32_t k = 0; k < le; ++k) dst[k] = tv.keys[oe + k];
  dst[le] = (uint8_t)c1;
  for (uint32_t k = 0; k < ls; ++k) dst[le + 1 + k] = tv.keys[os + k];
  if (e != kNoExt) {  // the extension above takes the merged key (it is dirty: on the path)
    tv.short_key[e] = off;
    tv.short_klen[e] = total;
    tv.short_child[e] = child;
  } else {
    const uint32_t ns = new_short(tv, dl, off, total, child, tv.full_depth[id], tv.gen);
    if (ns == 0xFFFFFFFFu) return;
    write_slot(tv, hs, make_ref(KIND_SHORT, ns));
  }
}

}  // namespace gmpt
