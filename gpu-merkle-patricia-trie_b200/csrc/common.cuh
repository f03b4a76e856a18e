// common.cuh -- shared device definitions for the B200 MPT path.
//
// Trie storage (HBM, structure of arrays, 32-bit node references):
//   ref = kind(2 bits) | index(30 bits); kind 0 = null, 1 = full (branch),
//   2 = short (extension / leaf), 3 = value.
// The reference links 56..240-byte AoS nodes by 64-bit pointers
// (mpt/node.cuh:340-589); here a branch is 17 x 4-byte child refs plus
// separate hash / depth / epoch arrays, so the walk touches 68 bytes per
// branch and the hash stage reads only what it encodes.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace gmpt {

enum : uint32_t { KIND_NULL = 0, KIND_FULL = 1, KIND_SHORT = 2, KIND_VALUE = 3 };

__host__ __device__ __forceinline__ uint32_t ref_kind(uint32_t r) { return r >> 30; }
__host__ __device__ __forceinline__ uint32_t ref_idx(uint32_t r) { return r & 0x3FFFFFFFu; }
__host__ __device__ __forceinline__ uint32_t make_ref(uint32_t k, uint32_t i) { return (k << 30) | i; }

constexpr uint32_t kMaxNodes = 0x3FFFFFFFu;  // per node kind
constexpr int kMaxKeyNibbles = 1024;          // longest accepted hex key
constexpr uint16_t kLcpInf = 0xFFFF;

// Device error word bits (read back by the host after each call).
enum : uint32_t {
  ERR_BAD_KEY = 1u << 0,       // nibble > 16, terminator not last, or prefix key
  ERR_CAPACITY = 1u << 1,      // a node pool ran out (host bound violated)
  ERR_RETRY_LIMIT = 1u << 2,   // LockNU insert exceeded its retry budget
  ERR_KEY_TOO_LONG = 1u << 3,
  ERR_INTERNAL = 1u << 4,
  ERR_BAD_TRIE = 1u << 5,      // trie id outside [0, number of tries)
  ERR_BARRIER = 1u << 6,       // a grid barrier wait gave up (persistent launch)
  ERR_BAD_FLAG = 1u << 7,      // read/write flag other than 0 (read) or 1 (write)
};

// Where a new subtree gets linked: a branch child slot, or the root word of
// one trie of the forest.  slot = (full index << 5) | child (< 2^35), or
// ~trie for the root word of `trie` (>= 2^64 - 2^32).
constexpr uint64_t kSlotRoot = ~0ull;  // root of trie 0
__host__ __device__ __forceinline__ uint64_t root_slot(uint32_t trie) { return ~(uint64_t)trie; }
__host__ __device__ __forceinline__ bool is_root_slot(uint64_t slot) { return slot >= 0xFFFFFFFF00000000ull; }
__host__ __device__ __forceinline__ uint32_t slot_trie(uint64_t slot) { return (uint32_t)~slot; }

struct Counters {
  uint32_t n_full, n_short, n_value, pad0;
  uint32_t n_dirty, n_items, n_groups, error;
  uint64_t key_used, val_used;
  uint32_t n_pseudo, retries_max, hashed, pad2;
  unsigned long long enc_bytes, keccak_blocks;  // last hash pass
  // staging checks of the last batch
  unsigned long long stream_terms;  // bytes == 16 in the key stream
  uint32_t key_terms;               // keys whose last byte is 16
  uint32_t noncontig;               // key index pairs do not tile the stream
  uint32_t bad_byte;                // a byte > 16 in the stream
  uint32_t pad3;
};

// A value record: byte offset into the value arena and length, side by side
// in 16 bytes so one sector holds both (a leaf's hash reads them together).
struct __align__(16) ValueRec {
  uint64_t off;
  uint32_t len;
  uint32_t pad;
};

// Everything a kernel needs to reach the trie; passed by value.
struct TrieView {
  // branch (full) nodes
  uint32_t *full_child;   // [cap_full * 17]
  uint32_t *full_epoch;   // dirty marker
  uint16_t *full_depth;   // nibble depth of the node's path
  uint8_t *full_hash;     // [cap_full * 32]
  uint8_t *full_hlen;
  uint8_t *full_dead;     // 1: unlinked by a delete (no longer in any trie)
  // short nodes
  uint64_t *short_key;    // nibble offset into the key arena
  uint32_t *short_klen;
  uint32_t *short_child;
  uint32_t *short_epoch;
  uint16_t *short_depth;
  uint8_t *short_dead;
  uint8_t *short_hash;    // [cap_short * 32]
  uint8_t *short_hlen;
  uint32_t *short_claim;  // split claim: the batch epoch that claimed it
  uint32_t *short_pseudo; // pseudo item created by that claim
  // value nodes -> value records
  unsigned long long *value_vid;
  ValueRec *rec;          // value records (arena offset + length)
  uint64_t *rec_hp;       // caller's host pointer (echoed by gets)
  // arenas
  const uint8_t *keys;    // nibble arena (one byte per nibble, 16 = term.)
  const uint8_t *vals;    // value byte arena
  uint32_t *roots;        // root ref word of every trie of the forest
  Counters *ctr;
  uint32_t cap_full, cap_short, cap_value;
  uint32_t n_tries;       // entries of roots[]
  uint32_t epoch;         // put batch number (split claims)
  uint32_t gen;           // hash generation (dirty marks)
  int geth_mode;          // 1 = embed <32 B children, hash the root always
  int account;            // 1 = hash kernels count encoding bytes / blocks / nodes (timing mode)
};

// ---------------------------------------------------------------------------
// small device helpers

__device__ __forceinline__ void set_error(Counters *c, uint32_t bits) { atomicOr(&c->error, bits); }

// Warp-aggregated allocation of n (0..7) slots among the currently converged
// lanes: one atomicAdd per warp instead of one per thread.  Returns the first
// slot of this lane's run.
__device__ __forceinline__ uint32_t warp_alloc(uint32_t *counter, uint32_t n) {
  unsigned mask = __activemask();
  unsigned lane = threadIdx.x & 31;
  unsigned lt = (1u << lane) - 1u;
  unsigned b0 = __ballot_sync(mask, n & 1u);
  unsigned b1 = __ballot_sync(mask, n & 2u);
  unsigned b2 = __ballot_sync(mask, n & 4u);
  uint32_t total = __popc(b0) + 2u * __popc(b1) + 4u * __popc(b2);
  uint32_t before = __popc(b0 & lt) + 2u * __popc(b1 & lt) + 4u * __popc(b2 & lt);
  int leader = __ffs(mask) - 1;
  uint32_t base = 0;
  if ((int)lane == leader && total) base = atomicAdd(counter, total);
  base = __shfl_sync(mask, base, leader);
  return base + before;
}

// One value record in a single 16-byte load (records are written by the
// staging launch and never change afterwards: the read-only path is safe).
__device__ __forceinline__ ValueRec load_rec(const TrieView &tv, uint64_t vid) {
  const ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2 *>(tv.rec) + vid);
  return ValueRec{v.x, (uint32_t)v.y, 0u};
}

// Unaligned 8-byte little-endian load from a byte array padded by >= 8 bytes.
__device__ __forceinline__ uint64_t load_u64_unaligned(const uint8_t *p) {
  uintptr_t a = reinterpret_cast<uintptr_t>(p);
  const uint64_t *q = reinterpret_cast<const uint64_t *>(a & ~uintptr_t(7));
  uint32_t sh = (uint32_t)(a & 7) * 8;
  uint64_t lo = __ldg(q);
  if (sh == 0) return lo;
  uint64_t hi = __ldg(q + 1);
  return (lo >> sh) | (hi << (64 - sh));
}

// Same with ordinary loads (data written earlier in this kernel, before a
// grid barrier; never the non-coherent read-only path).
__device__ __forceinline__ uint64_t load_u64_unaligned_cg(const uint8_t *p) {
  uintptr_t a = reinterpret_cast<uintptr_t>(p);
  const uint64_t *q = reinterpret_cast<const uint64_t *>(a & ~uintptr_t(7));
  uint32_t sh = (uint32_t)(a & 7) * 8;
  uint64_t lo = q[0];
  if (sh == 0) return lo;
  uint64_t hi = q[1];
  return (lo >> sh) | (hi << (64 - sh));
}

__device__ __forceinline__ uint64_t low_mask64(int nbytes) {
  return nbytes >= 8 ? ~0ull : ((1ull << (8 * nbytes)) - 1);
}

// 8 nibble bytes (little-endian in a u64, each 0..16) -> 32-bit big-endian
// nibble chunk, terminator mapped to 0 (byte & 15).
__device__ __forceinline__ uint32_t pack_nibbles8(uint64_t x) {
  x &= 0x0F0F0F0F0F0F0F0Full;
  uint64_t be = __byte_perm((uint32_t)(x >> 32), 0, 0x0123) |
                ((uint64_t)__byte_perm((uint32_t)x, 0, 0x0123) << 32);
  be = (be | (be >> 4)) & 0x00FF00FF00FF00FFull;
  be = (be | (be >> 8)) & 0x0000FFFF0000FFFFull;
  be = (be | (be >> 16)) & 0x00000000FFFFFFFFull;
  return (uint32_t)be;
}

// Number of equal leading nibbles of a[0..n) and b[0..n).
__device__ __forceinline__ int match_nibbles(const uint8_t *a, const uint8_t *b, int n) {
  int m = 0;
  while (m + 8 <= n) {
    uint64_t x = load_u64_unaligned(a + m) ^ load_u64_unaligned(b + m);
    if (x) return m + (__ffsll((long long)x) - 1) / 8;
    m += 8;
  }
  while (m < n && a[m] == b[m]) ++m;
  return m;
}

}  // namespace gmpt
