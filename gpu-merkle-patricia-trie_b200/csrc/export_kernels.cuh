// export_kernels.cuh -- (hash, RLP encoding) of the nodes on a set of key
// paths: the nodeset a geth commit persists (MPT::flush_dirty_nodes,
// gpu_mpt.cuh:1039-1122; kernels gets_dirty_nodes_count / gets_dirty_nodes,
// gpu_mpt_kernels.cuh:2342-2588).  Nodes are emitted once each, ordered by
// node reference; only nodes referenced by hash (encoding >= 32 bytes, or
// the root) are emitted, since smaller ones live inside their parent's
// encoding.
#pragma once
#include "trie_kernels.cuh"

namespace gmpt {

// every full/short node on each key's path -> refs[] (with repeats)
__global__ void k_flush_collect(TrieView tv, const uint8_t *keys, const int *idx, int n, int64_t keys_bytes,
                                uint64_t *out, uint32_t *count, uint32_t cap) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int ks = idx[2 * i], len = idx[2 * i + 1] - ks + 1;
  if (ks < 0 || len <= 0 || (int64_t)idx[2 * i + 1] >= keys_bytes) return;
  const uint8_t *kb = keys + ks;
  const uint32_t root = tv.roots[0];  // the state trie (trie 0)
  uint32_t ref = root;
  int x = 0;
  for (int guard = 0; guard <= len + 1; ++guard) {
    uint32_t kind = ref_kind(ref), id = ref_idx(ref);
    if (kind == KIND_NULL || kind == KIND_VALUE) return;
    uint8_t hl = kind == KIND_FULL ? tv.full_hlen[id] : tv.short_hlen[id];
    if (hl == 32 || ref == root) {
      uint32_t slot = atomicAdd(count, 1u);
      if (slot < cap) out[slot] = ref;
    }
    if (kind == KIND_FULL) {
      if (x >= len || kb[x] > 16) return;
      ref = tv.full_child[(size_t)id * 17 + kb[x]];
      ++x;
    } else {
      uint32_t sl = tv.short_klen[id];
      if ((uint32_t)(len - x) < sl) return;
      if ((uint32_t)match_nibbles(tv.keys + tv.short_key[id], kb + x, (int)sl) != sl) return;
      x += (int)sl;
      ref = tv.short_child[id];
    }
  }
}

__global__ void k_widen_u32(const uint32_t *in, int64_t n, uint64_t *out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[i];
}

// Sorted refs of the nodes hashed since the last flush -> flags[i] = 1 for
// the first copy of a node that is still in a trie (not unlinked by a split
// or a delete) and referenced by hash (encoding of 32 bytes hashed) or a
// root (nibble depth 0: exactly the roots of the forest's tries).
__global__ void k_flush_dirty_flags(TrieView tv, const uint64_t *refs, int n, unsigned long long *flags) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t r = (uint32_t)refs[i];
  const uint32_t id = ref_idx(r);
  bool keep = i == 0 || refs[i] != refs[i - 1];
  if (keep) {
    if (ref_kind(r) == KIND_FULL)
      keep = !tv.full_dead[id] && (tv.full_hlen[id] == 32 || tv.full_depth[id] == 0);
    else
      keep = ref_kind(r) == KIND_SHORT && !tv.short_dead[id] &&
             (tv.short_hlen[id] == 32 || tv.short_depth[id] == 0);
  }
  flags[i] = keep ? 1ull : 0ull;
}

__global__ void k_flush_unique_flags(const uint64_t *refs, int n, unsigned long long *flags) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  flags[i] = (i == 0 || refs[i] != refs[i - 1]) ? 1ull : 0ull;
}

__global__ void k_flush_sizes(TrieView tv, const uint64_t *refs, const unsigned long long *flags,
                              const unsigned long long *pos, int n, uint32_t *uref, unsigned long long *sizes) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !flags[i]) return;
  uint32_t r = (uint32_t)refs[i];
  uint32_t u = (uint32_t)pos[i];
  uref[u] = r;
  bool full = ref_kind(r) == KIND_FULL;
  uint32_t id = ref_idx(r);
  uint64_t payload = 0;
  for (int k = 1; k < (full ? 18 : 3); ++k) {
    EncItem it = node_item(tv, full, id, k, 0);
    payload += it.pren + it.blen;
  }
  uint64_t h;
  uint32_t hn;
  rlp_head(payload, 0xc0, 0xf7, h, hn);
  sizes[u] = payload + hn;
}

__global__ void k_flush_write(TrieView tv, const uint32_t *uref, const unsigned long long *offs, int m,
                              uint8_t *encs, unsigned long long *encs_idx, uint8_t *hashs) {
  int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= m) return;
  uint32_t r = uref[u];
  bool full = ref_kind(r) == KIND_FULL;
  uint32_t id = ref_idx(r);
  int nitems = full ? 18 : 3;
  uint64_t payload = 0;
  for (int k = 1; k < nitems; ++k) {
    EncItem it = node_item(tv, full, id, k, 0);
    payload += it.pren + it.blen;
  }
  uint8_t *o = encs + offs[u];
  uint64_t w = 0;
  for (int k = 0; k < nitems; ++k) {
    EncItem it = node_item(tv, full, id, k, payload);
    for (uint32_t b = 0; b < it.pren; ++b) o[w++] = (uint8_t)(it.pre >> (8 * b));
    for (uint32_t b = 0; b < it.blen; ++b) {
      if (it.nib)
        o[w++] = (uint8_t)(((it.body[2 * b] & 15) << 4) | (it.body[2 * b + 1] & 15));
      else
        o[w++] = it.body[b];
    }
  }
  encs_idx[2 * u] = offs[u];
  encs_idx[2 * u + 1] = offs[u] + w - 1;
  const uint8_t *h = (full ? tv.full_hash : tv.short_hash) + (size_t)id * 32;
  uint8_t hl = (full ? tv.full_hlen : tv.short_hlen)[id];
  for (int b = 0; b < 32; ++b) hashs[32 * (size_t)u + b] = b < hl ? h[b] : 0;
}

}  // namespace gmpt
