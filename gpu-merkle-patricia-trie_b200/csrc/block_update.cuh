// block_update.cuh -- one persistent launch that updates many tries of a
// forest and hashes them: the Ethereum block shape, where every touched
// account's storage trie is updated and hashed first, its new root is
// written into the account's value, and then the state trie is updated and
// hashed.
//
// The reference runs one MPT object per trie and one puts_latching + one
// hash_onepass (several kernel launches, host synchronisation between them)
// per trie (gpu_mpt.cuh:554-615, 1162-1191).  Here a block is:
//   k_block_stage  copy + validate the key/value streams into the arenas and
//                  build the value records (an ordinary launch, so the arena
//                  bytes are read-only for the next one)
//   k_block        cooperative persistent kernel, for stage 0 then stage 1:
//                    [stage 1 only] patch: value bytes of key i at
//                      patch_off[i] := root of trie patch_trie[i]
//                    LockNU insert of the stage's keys into their tries
//                    bucket the dirty nodes by (nibble depth, kind)
//                    hash them deepest level first
//                  with a grid barrier between phases, then the roots asked
//                  for are written out.
// Both launches plus the descriptor / counter copies are captured once as a
// CUDA graph and replayed per block; sizes come from the device-side
// descriptor, so the graph is rebuilt only when a buffer or pool moves.
#pragma once
#include "latch_kernels.cuh"
#include "trie_kernels.cuh"

namespace gmpt {

constexpr int kDepthBins = 2 * (kMaxKeyNibbles + 2);  // (depth, kind) buckets
constexpr int kBlockMaxTs = 64;
constexpr int kWarpFullPerWarp = 4;  // warp-per-branch hashing up to 4 branches per warp

struct BlockDesc {
  // set by the host for every launch; copying it in also zeroes the fields
  // below that the kernels fill
  int32_t n, n0, n_out, pad0;      // keys; stage 0 = [0, n0), stage 1 = [n0, n)
  int64_t kbytes, vbytes;          // stream lengths
  uint64_t key_base, val_base, vid_base;
  uint32_t gen, pad1;              // dirty generation of stage 0 (stage 1: gen + 1)
  uint64_t barrier_ns;             // longest grid-barrier wait before giving up
  uint32_t bar_count, bar_gen;     // grid barrier
  // filled by k_block_stage
  uint32_t stream_terms, key_terms, noncontig, bad;  // bad: BLOCK_BAD_* bits
  // filled by k_block
  uint32_t levels[2], dirty[2], maxbin[2];
  uint32_t status;                 // 1: a barrier gave up; 2: stopped on bad input
  uint32_t n_ts;                   // phase timeline of CTA 0 (globaltimer, ns)
  uint64_t ts[kBlockMaxTs];
};

enum : uint32_t { BLOCK_BAD_KEY = 1, BLOCK_BAD_TRIE = 2, BLOCK_BAD_PATCH = 4, BLOCK_BAD_VALUE = 8 };

struct BlockBufs {
  const uint8_t *keys;     // key stream (nibble bytes)
  const int *kidx;         // [2n] inclusive pairs; must tile the stream
  const uint8_t *vals;     // value stream
  const int64_t *vidx;     // [2n]
  const int *tid;          // [n] trie of each key
  const int *patch_trie;   // [n] -1 = no patch
  const int *patch_off;    // [n] byte offset of the 32-byte root in the value
  const int *out_ids;      // [n_out] tries whose roots are reported
  uint8_t *out;            // [n_out * 33] root bytes + length
  uint64_t *koff;          // [n] staged key offsets
  uint32_t *klen;          // [n]
  uint32_t *bins;          // [2 stages][2][kDepthBins + 1]: counts, offsets
  uint32_t *cursor;        // [kDepthBins]
  uint32_t *sorted;        // dirty refs bucketed by (depth, kind)
  BlockDesc *desc;
};

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// A barrier wait longer than BlockDesc::barrier_ns (2 s unless the trie's
// "block_barrier_ns" option says otherwise) gives up: the CTA raises
// ERR_BARRIER and leaves the kernel, and so does every CTA at its next
// barrier.

// Grid-wide barrier of a cooperative launch (all CTAs co-resident).
// Returns false when this CTA must stop.
__device__ bool grid_barrier(BlockDesc *D, Counters *ctr) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    volatile uint32_t *vgen = &D->bar_gen;
    const uint32_t g = *vgen;
    __threadfence();
    const uint32_t arrived = atomicAdd(&D->bar_count, 1u);
    if (arrived == gridDim.x - 1) {
      atomicExch(&D->bar_count, 0u);
      __threadfence();
      atomicAdd(&D->bar_gen, 1u);
    } else {
      const uint64_t t0 = global_ns();
      const uint64_t limit = D->barrier_ns;
      uint32_t spins = 0;
      while (*vgen == g) {
        __nanosleep(64);
        if ((++spins & 63) == 0 && global_ns() - t0 > limit) {
          ok = 0;
          break;
        }
      }
    }
    if (!ok) {
      set_error(ctr, ERR_BARRIER);
      atomicOr(&D->status, 1u);
    } else if (*reinterpret_cast<volatile uint32_t *>(&D->status) & 1u) {
      ok = 0;  // another CTA gave up earlier
    }
    __threadfence();
    s_ok = ok;
    if (blockIdx.x == 0 && D->n_ts < kBlockMaxTs) D->ts[D->n_ts++] = global_ns();
  }
  __syncthreads();
  return s_ok != 0;
}

// Copy the streams into the arenas (8-byte words; the last partial word is
// masked and 64 zero bytes follow each stream), validate keys and pairs, and
// build the value records.  Grid-stride; every thread runs to the end.
__global__ void __launch_bounds__(256) k_block_stage(TrieView tv, BlockBufs bb) {
  BlockDesc *D = bb.desc;
  const int n = D->n, n0 = D->n0;
  const int64_t kb = D->kbytes, vb = D->vbytes;
  const uint64_t key_base = D->key_base, val_base = D->val_base, vid_base = D->vid_base;
  const int64_t T = (int64_t)gridDim.x * blockDim.x, t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t0 == 0) D->ts[D->n_ts++] = global_ns();
  uint32_t terms = 0, bad = 0, kterms = 0, gap = 0;
  {
    uint64_t *dst = reinterpret_cast<uint64_t *>(const_cast<uint8_t *>(tv.keys) + key_base);
    const uint64_t *src = reinterpret_cast<const uint64_t *>(bb.keys);
    const int64_t words = (kb + 7) / 8 + 8;
    for (int64_t w = t0; w < words; w += T) {
      uint64_t x = 0;
      if (8 * w < kb) {
        x = src[w];
        const int64_t rem = kb - 8 * w;
        if (rem < 8) x &= (1ull << (8 * rem)) - 1;
        if (x & 0xE0E0E0E0E0E0E0E0ull) bad |= BLOCK_BAD_KEY;  // >= 32
        const uint64_t hi = x & 0x1010101010101010ull;        // 16..31
        if (x & ((hi >> 4) * 0x0Full)) bad |= BLOCK_BAD_KEY;  // 17..31
        terms += __popcll(hi);
      }
      dst[w] = x;
    }
  }
  {
    uint64_t *dst = reinterpret_cast<uint64_t *>(const_cast<uint8_t *>(tv.vals) + val_base);
    const uint64_t *src = reinterpret_cast<const uint64_t *>(bb.vals);
    const int64_t words = (vb + 7) / 8 + 8;
    for (int64_t w = t0; w < words; w += T) {
      uint64_t x = 0;
      if (8 * w < vb) {
        x = src[w];
        const int64_t rem = vb - 8 * w;
        if (rem < 8) x &= (1ull << (8 * rem)) - 1;
      }
      dst[w] = x;
    }
  }
  for (int64_t w = t0; w < 2 * (kDepthBins + 1) * 2; w += T) bb.bins[w] = 0;
  for (int64_t i = t0; i < n; i += T) {
    int ks = bb.kidx[2 * i], ke = bb.kidx[2 * i + 1];
    bool badk = ks < 0 || ke < ks || (int64_t)ke >= kb || ke - ks + 1 > kMaxKeyNibbles;
    if (!badk) {
      const uint8_t last = bb.keys[ke];
      if (last > 16) badk = true;
      kterms += last == 16 ? 1u : 0u;
    }
    if (i == 0 ? ks != 0 : ks != bb.kidx[2 * i - 1] + 1) gap = 1;
    if (i + 1 == n && (int64_t)ke + 1 != kb) gap = 1;
    if (badk) {
      bad |= BLOCK_BAD_KEY;
      ks = ke = 0;
    }
    bb.koff[i] = key_base + (uint64_t)ks;
    bb.klen[i] = (uint32_t)(ke - ks + 1);
    if ((uint32_t)bb.tid[i] >= tv.n_tries) bad |= BLOCK_BAD_TRIE;
    int64_t vs = bb.vidx[2 * i], ve = bb.vidx[2 * i + 1];
    if (vs < 0 || ve < vs - 1 || ve >= vb) {
      bad |= BLOCK_BAD_VALUE;
      vs = 0;
      ve = -1;
    }
    const int pt = bb.patch_trie[i];
    if (pt >= 0 && ((uint32_t)pt >= tv.n_tries || i < n0 || bb.patch_off[i] < 0 ||
                    (int64_t)bb.patch_off[i] + 32 > ve - vs + 1))
      bad |= BLOCK_BAD_PATCH;
    const uint64_t vid = vid_base + (uint64_t)i;
    tv.rec[vid] = ValueRec{val_base + (uint64_t)vs, (uint32_t)(ve - vs + 1), 0u};
    tv.rec_hp[vid] = 0;
  }
  terms = __reduce_add_sync(0xffffffffu, terms);
  kterms = __reduce_add_sync(0xffffffffu, kterms);
  bad = __reduce_or_sync(0xffffffffu, bad);
  gap = __reduce_or_sync(0xffffffffu, gap);
  if ((threadIdx.x & 31) == 0) {
    if (terms) atomicAdd(&D->stream_terms, terms);
    if (kterms) atomicAdd(&D->key_terms, kterms);
    if (bad) atomicOr(&D->bad, bad);
    if (gap) atomicOr(&D->noncontig, 1u);
  }
}

// 33 bytes for the root of trie tr (warp-wide: lane b writes byte b)
__device__ __forceinline__ void write_root(const TrieView &tv, uint32_t tr, uint8_t *out, int lane) {
  const uint32_t r = tr < tv.n_tries ? __ldcg(tv.roots + tr) : 0u;
  const uint32_t kind = ref_kind(r), idx = ref_idx(r);
  const uint8_t *h = nullptr;
  uint32_t len = 0;
  if (kind == KIND_FULL) {
    h = tv.full_hash + (size_t)idx * 32;
    len = __ldcg(tv.full_hlen + idx);
  } else if (kind == KIND_SHORT) {
    h = tv.short_hash + (size_t)idx * 32;
    len = __ldcg(tv.short_hlen + idx);
  }
  out[lane] = (h && (uint32_t)lane < len) ? __ldcg(h + lane) : 0;
  if (lane == 0) out[32] = (uint8_t)len;
}

__global__ void __launch_bounds__(256, 2) k_block(TrieView tv0, DirtyList dl, BlockBufs bb, uint32_t retry_limit) {
  extern __shared__ uint64_t smem[];  // 17 message words per thread; histogram
  BlockDesc *D = bb.desc;
  const int n = D->n, n0 = D->n0, n_out = D->n_out;
  const uint64_t vid_base = D->vid_base;
  const int t = blockIdx.x * blockDim.x + threadIdx.x, T = gridDim.x * blockDim.x;
  TrieView tv = tv0;
  if (t == 0) D->ts[D->n_ts++] = global_ns();
  // Spread mapping: warps are numbered CTA-fastest (consecutive warp ids sit
  // on different SMs) and item j goes to warp j % W, lane j / W, so a level
  // of a few hundred nodes, or the keys of one storage trie, use one lane in
  // each of many warps instead of all lanes of a few (divergent Keccak, CAS
  // retries on one slot serialised inside a warp).
  const int lane = threadIdx.x & 31;
  const int W = T >> 5;
  const int gw = (threadIdx.x >> 5) * gridDim.x + blockIdx.x;
  const int t_spread = lane * W + gw;
  // this warp's message buffer for hash_full_warp, after the staging words
  uint8_t *wmsg = reinterpret_cast<uint8_t *>(smem + 17 * blockDim.x) + (threadIdx.x >> 5) * kWarpMsgBytes;
  // staging outcome: every CTA reads the same words, so all leave together
  if (D->bad || D->noncontig || D->stream_terms != D->key_terms) {
    if (t == 0) atomicOr(&D->status, 2u);
    return;
  }
  uint32_t *hist = reinterpret_cast<uint32_t *>(smem);
  for (int s = 0; s < 2; ++s) {
    const int i0 = s ? n0 : 0, i1 = s ? n : n0;
    tv.gen = D->gen + (uint32_t)s;
    if (s == 1) {
      // stage-1 values take the roots their stage-0 tries just got
      for (int i = n0 + t; i < n; i += T) {
        const int pt = bb.patch_trie[i];
        if (pt < 0) continue;
        uint8_t *dst = const_cast<uint8_t *>(tv.vals) + tv.rec[vid_base + (uint64_t)i].off + bb.patch_off[i];
        const uint32_t r = __ldcg(tv.roots + pt);
        const uint32_t kind = ref_kind(r), idx = ref_idx(r);
        const uint8_t *h = kind == KIND_FULL ? tv.full_hash + (size_t)idx * 32
                                             : (kind == KIND_SHORT ? tv.short_hash + (size_t)idx * 32 : nullptr);
        const uint32_t hl =
            kind == KIND_FULL ? __ldcg(tv.full_hlen + idx) : (kind == KIND_SHORT ? __ldcg(tv.short_hlen + idx) : 0u);
        for (uint32_t b = 0; b < 32; ++b) dst[b] = (h && b < hl) ? __ldcg(h + b) : 0;
      }
    }
    // insert (LockNU; the patched bytes are only read after the next barrier)
    const int span = T * kLatchWays;
    for (int base = i0; base < i1; base += span)
      latch_keys(tv, dl, bb.koff + base, bb.klen + base, min(span, i1 - base), vid_base + (uint64_t)base, retry_limit,
                 bb.tid + base, t_spread, T);
    if (!grid_barrier(D, tv.ctr)) return;
    // bucket the dirty nodes: histogram
    const uint32_t nd = __ldcg(&tv.ctr->n_dirty);
    uint32_t *cnt = bb.bins + (size_t)s * 2 * (kDepthBins + 1);
    uint32_t *off = cnt + (kDepthBins + 1);
    for (int b = threadIdx.x; b < kDepthBins; b += blockDim.x) hist[b] = 0;
    __syncthreads();
    for (uint32_t i = t; i < nd; i += T) {
      const uint32_t r = __ldcg(dl.ref + i);
      atomicAdd(&hist[2u * __ldcg(dl.depth + i) + (ref_kind(r) == KIND_FULL ? 1u : 0u)], 1u);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < kDepthBins; b += blockDim.x)
      if (hist[b]) atomicAdd(&cnt[b], hist[b]);
    if (!grid_barrier(D, tv.ctr)) return;
    // offsets (CTA 0): per-thread runs, then a serial scan of the run sums
    if (blockIdx.x == 0) {
      constexpr int kPer = (kDepthBins + 255) / 256;
      uint32_t *sums = hist;  // [blockDim.x]
      uint32_t *smax = hist + 256;
      const int b0 = threadIdx.x * kPer;
      uint32_t v[kPer];
      uint32_t sum = 0, top = 0;
#pragma unroll
      for (int k = 0; k < kPer; ++k) {
        const int b = b0 + k;
        v[k] = (b < kDepthBins) ? __ldcg(cnt + b) : 0u;
        sum += v[k];
        if (v[k]) top = (uint32_t)b + 1;
      }
      if (threadIdx.x == 0) *smax = 0;
      sums[threadIdx.x] = sum;
      __syncthreads();
      if (top) atomicMax(smax, top);
      if (threadIdx.x == 0) {
        uint32_t acc = 0;
        for (int k = 0; k < (int)blockDim.x; ++k) {
          const uint32_t x = sums[k];
          sums[k] = acc;
          acc += x;
        }
      }
      __syncthreads();
      uint32_t acc = sums[threadIdx.x];
#pragma unroll
      for (int k = 0; k < kPer; ++k) {
        const int b = b0 + k;
        if (b < kDepthBins) {
          off[b] = acc;
          bb.cursor[b] = acc;
        }
        acc += v[k];
      }
      if (threadIdx.x == blockDim.x - 1) off[kDepthBins] = acc;
      if (threadIdx.x == 0) {
        D->maxbin[s] = *smax;
        D->dirty[s] = nd;
      }
    }
    if (!grid_barrier(D, tv.ctr)) return;
    // scatter into the buckets (warp-aggregated cursor updates)
    for (uint32_t i0s = (uint32_t)(t & ~31); i0s < nd; i0s += (uint32_t)T) {
      const uint32_t i = i0s + (t & 31);
      const bool ok = i < nd;
      const uint32_t r = ok ? __ldcg(dl.ref + i) : 0u;
      const uint32_t b = ok ? 2u * __ldcg(dl.depth + i) + (ref_kind(r) == KIND_FULL ? 1u : 0u) : 0xFFFFFFFFu;
      const unsigned peers = __match_any_sync(0xffffffffu, b);
      const int leader = __ffs(peers) - 1;
      uint32_t pos = 0;
      if (ok && (int)(threadIdx.x & 31) == leader) pos = atomicAdd(&bb.cursor[b], (uint32_t)__popc(peers));
      pos = __shfl_sync(0xffffffffu, pos, leader);
      if (ok) bb.sorted[pos + __popc(peers & ((1u << (threadIdx.x & 31)) - 1u))] = r;
    }
    if (!grid_barrier(D, tv.ctr)) return;
    if (t == 0) atomicExch(&tv.ctr->n_dirty, 0u);  // the list is consumed
    // hash, deepest level first
    const CoopLanes coop = coop_lanes(lane);
    const uint32_t top = __ldcg(&D->maxbin[s]);
    uint32_t levels = 0;
    for (int d = (int)(top + 1) / 2 - 1; d >= 0; --d) {
      const uint32_t a = __ldcg(off + 2 * d), m = __ldcg(off + 2 * d + 1), z = __ldcg(off + 2 * d + 2);
      if (z == a) continue;
      ++levels;
      // short nodes [a, m) from warp 0 up, full nodes [m, z) from warp W-1 down
      for (uint32_t j = (uint32_t)t_spread; j < m - a; j += (uint32_t)T)
        hash_node<true>(tv, __ldcg(bb.sorted + a + j), smem + threadIdx.x, blockDim.x);
      if (z - m <= (uint32_t)(kWarpFullPerWarp * W)) {
        // few branches: a warp per node (latency)
        for (uint32_t j = (uint32_t)(W - 1 - gw); j < z - m; j += (uint32_t)W) {
          hash_full_warp<true>(tv, ref_idx(__ldcg(bb.sorted + m + j)), wmsg, coop);
          __syncwarp();
        }
      } else {
        const uint32_t t_rev = (uint32_t)(lane * W + (W - 1 - gw));
        for (uint32_t j = t_rev; j < z - m; j += (uint32_t)T)
          hash_node<true>(tv, __ldcg(bb.sorted + m + j), smem + threadIdx.x, blockDim.x);
      }
      if (!grid_barrier(D, tv.ctr)) return;
    }
    if (t == 0) D->levels[s] = levels;
    if (!grid_barrier(D, tv.ctr)) return;  // the n_dirty reset is seen by every CTA
  }
  // roots asked for: one warp each
  for (int w = t >> 5; w < n_out; w += T >> 5) write_root(tv, (uint32_t)bb.out_ids[w], bb.out + 33 * (size_t)w, lane);
  __syncthreads();
  if (t == 0 && D->n_ts < kBlockMaxTs) D->ts[D->n_ts++] = global_ns();
}

}  // namespace gmpt
