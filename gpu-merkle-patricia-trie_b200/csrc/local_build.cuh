// local_build.cuh -- CTA-local completion of the level-synchronous build.
//
// Once every active segment of the global build (trie_kernels.cuh
// k_level_*) holds at most kLocalCap sorted items, one CTA per segment
// builds the segment's entire compressed subtrie with its frontier of
// sub-segments in shared memory: per level, min adjacent LCP per segment
// (shared-memory atomics), one branch (+ extension) per segment, leaves for
// singleton children, and one block-wide scan that numbers the next level's
// segments.  Node shapes are exactly those of the global levels; only the
// synchronisation moves from kernel boundaries to __syncthreads.
#pragma once
#include "trie_kernels.cuh"

namespace gmpt {

constexpr int kLocalCap = 2048;     // items per segment
constexpr int kLocalThreads = 256;  // items [tid*8, tid*8+8) per thread
constexpr int kLocalIpt = kLocalCap / kLocalThreads;
constexpr int kLocalSegs = kLocalCap / 2;  // a segment has >= 2 items
// resident CTAs per SM the register allocation is bounded for
#ifndef GMPT_LOCAL_BUILD_CTAS
#define GMPT_LOCAL_BUILD_CTAS 4
#endif

struct LocalSegs {
  uint64_t slot[kLocalSegs];  // where the segment's top node is linked
  uint32_t D[kLocalSegs];     // branch depth (min interior LCP)
  uint32_t branch[kLocalSegs];
  uint16_t start[kLocalSegs];
  uint16_t end[kLocalSegs];
  uint16_t depth[kLocalSegs];
};

struct LocalSmem {
  LocalSegs s[2];
  uint16_t lcp[kLocalCap + 1];
  uint16_t seg[kLocalCap];  // segment of each item at this level, 0xFFFF = done
  uint32_t warp_sums[kLocalThreads / 32 + 1];
  uint32_t nseg;
  uint32_t leaf_base, dirty_base, leaf_ok;  // this level's leaf short nodes
};

__global__ void __launch_bounds__(kLocalThreads, GMPT_LOCAL_BUILD_CTAS) k_local_build(TrieView tv, DirtyList dl, SortedItems si,
                                                               SegArrays gs, uint32_t gen) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  LocalSmem &L = *reinterpret_cast<LocalSmem *>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const uint32_t gseg = blockIdx.x;
  const uint32_t base = gs.start[gseg];
  const int m = (int)(gs.end[gseg] - base);
  if (m > kLocalCap || m < 2) {  // the host launches only 2 <= m <= cap
    if (tid == 0) set_error(tv.ctr, ERR_INTERNAL);
    return;
  }
  for (int k = tid; k < m; k += kLocalThreads) {
    L.lcp[k] = k == 0 ? kLcpInf : si.lcp[base + k];
    L.seg[k] = 0;
  }
  if (tid == 0) {
    L.lcp[m] = kLcpInf;
    L.nseg = 1;
    L.s[0].start[0] = 0;
    L.s[0].end[0] = (uint16_t)m;
    L.s[0].depth[0] = (uint16_t)gs.depth[gseg];
    L.s[0].slot[0] = gs.slot[gseg];
  }
  __syncthreads();
  int cur = 0;
  for (int level = 0; level < kMaxKeyNibbles + 2; ++level) {
    const uint32_t nseg = L.nseg;
    if (nseg == 0) break;
    LocalSegs &S = L.s[cur];
    LocalSegs &N = L.s[cur ^ 1];
    for (uint32_t q = tid; q < nseg; q += kLocalThreads) S.D[q] = 0xFFFFFFFFu;
    __syncthreads();
    // 1. D = min LCP over each segment's interior boundaries
    for (int k = tid; k < m; k += kLocalThreads) {
      uint16_t q = L.seg[k];
      if (q != 0xFFFF && k != S.start[q]) atomicMin(&S.D[q], (uint32_t)L.lcp[k]);
    }
    __syncthreads();
    // 2. one branch (+ extension above it) per segment
    for (uint32_t q = tid; q < nseg; q += kLocalThreads) {
      uint32_t D = S.D[q], d = S.depth[q];
      uint32_t i0 = base + S.start[q];
      uint32_t f = 0xFFFFFFFFu;
      if (D != 0xFFFFFFFFu && D >= d && D < si.len[i0])
        f = new_full(tv, dl, D, gen);
      else
        set_error(tv.ctr, ERR_INTERNAL);
      S.branch[q] = f;
      if (f == 0xFFFFFFFFu) continue;
      uint32_t top = make_ref(KIND_FULL, f);
      if (D > d) {
        uint32_t e = new_short(tv, dl, si.base[i0] + d, D - d, top, d, gen);
        if (e == 0xFFFFFFFFu) continue;
        top = make_ref(KIND_SHORT, e);
      }
      write_slot(tv, S.slot[q], top);
    }
    __syncthreads();
    // 3a. children of each branch: singleton children become leaves (made in
    // 3b, their short nodes allocated once for the whole CTA: one global
    // atomic per level instead of one per warp); count next-level segment
    // starts and leaves
    uint8_t fl[kLocalIpt];
    uint8_t nb[kLocalIpt];
    uint16_t lq[kLocalIpt];
    uint32_t leafbits = 0, my_starts = 0, my_leaves = 0;
#pragma unroll
    for (int r = 0; r < kLocalIpt; ++r) {
      const int k = tid * kLocalIpt + r;
      fl[r] = 0;
      nb[r] = 0;
      lq[r] = 0;
      if (k >= m) continue;
      const uint16_t q = L.seg[k];
      if (q == 0xFFFF) continue;
      const uint32_t D = S.D[q], f = S.branch[q];
      if (f == 0xFFFFFFFFu) {
        L.seg[k] = 0xFFFF;
        continue;
      }
      const bool cs = (k == S.start[q]) || L.lcp[k] == D;
      const bool ce = (k + 1 == S.end[q]) || L.lcp[k + 1] == D;
      if (cs) nb[r] = tv.keys[si.base[base + k] + D];  // a child run's slot nibble
      if (cs && ce) {
        leafbits |= 1u << r;
        lq[r] = q;
        if (D + 1 < si.len[base + k]) ++my_leaves;  // else the value links straight in
        L.seg[k] = 0xFFFF;
        continue;
      }
      fl[r] = 1 | (cs ? 2 : 0) | (ce ? 4 : 0);
      my_starts += cs ? 1u : 0u;
    }
    // block-wide exclusive scan of (leaves << 16 | starts) (items are in
    // thread order; each count is at most kLocalCap < 2^16)
    const uint32_t mine = (my_leaves << 16) | my_starts;
    uint32_t incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane == 31) L.warp_sums[wid] = incl;
    __syncthreads();
    if (tid == 0) {
      uint32_t run = 0;
      for (int w = 0; w < kLocalThreads / 32; ++w) {
        uint32_t c = L.warp_sums[w];
        L.warp_sums[w] = run;
        run += c;
      }
      L.warp_sums[kLocalThreads / 32] = run & 0xFFFFu;
      const uint32_t tl = run >> 16;
      L.leaf_ok = 1;
      if (tl) {
        const uint32_t b0 = atomicAdd(&tv.ctr->n_short, tl);
        if (b0 + tl > tv.cap_short) {  // nothing pushed to the dirty list then
          set_error(tv.ctr, ERR_CAPACITY);
          L.leaf_ok = 0;
        } else {
          L.leaf_base = b0;
          L.dirty_base = atomicAdd(&tv.ctr->n_dirty, tl);
        }
      }
    }
    __syncthreads();
    // 3b. leaves; an item's next-level segment is the latest start at or before it
    const uint32_t before = L.warp_sums[wid] + incl - mine;
    uint32_t run = before & 0xFFFFu;  // starts before this thread
    uint32_t lb = before >> 16;       // leaf short nodes before this thread
#pragma unroll
    for (int r = 0; r < kLocalIpt; ++r) {
      if (!((leafbits >> r) & 1u)) continue;
      const uint32_t q = lq[r], i = base + tid * kLocalIpt + r;
      const uint32_t x = S.D[q] + 1, len = si.len[i];
      const uint64_t slot = ((uint64_t)S.branch[q] << 5) | nb[r];
      if (x >= len) {
        write_slot(tv, slot, si.ref[i]);
        continue;
      }
      const uint32_t j = lb++;
      if (!L.leaf_ok) continue;
      const uint32_t sn = L.leaf_base + j;
      tv.short_key[sn] = si.base[i] + x;
      tv.short_klen[sn] = len - x;
      tv.short_child[sn] = si.ref[i];
      tv.short_depth[sn] = (uint16_t)x;
      tv.short_epoch[sn] = gen;
      tv.short_dead[sn] = 0;
      tv.short_claim[sn] = 0;
      tv.short_hlen[sn] = 0;
      const uint32_t ref = make_ref(KIND_SHORT, sn);
      dl.ref[L.dirty_base + j] = ref;
      dl.depth[L.dirty_base + j] = (uint16_t)x;
      write_slot(tv, slot, ref);
    }
#pragma unroll
    for (int r = 0; r < kLocalIpt; ++r) {
      const int k = tid * kLocalIpt + r;
      if (!(fl[r] & 1)) continue;
      const uint16_t q = L.seg[k];
      if (fl[r] & 2) {
        ++run;
        const uint32_t id = run - 1;
        N.start[id] = (uint16_t)k;
        N.depth[id] = (uint16_t)(S.D[q] + 1);
        N.slot[id] = ((uint64_t)S.branch[q] << 5) | nb[r];
      }
      const uint32_t id = run - 1;
      if (fl[r] & 4) N.end[id] = (uint16_t)(k + 1);
      L.seg[k] = (uint16_t)id;
    }
    __syncthreads();
    if (tid == 0) L.nseg = L.warp_sums[kLocalThreads / 32];
    __syncthreads();
    cur ^= 1;
  }
}

// largest segment of the current global level (decides the switch to local)
__global__ void k_seg_max(const SegArrays sg, int S, uint32_t *out) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t v = s < S ? sg.end[s] - sg.start[s] : 0u;
  uint32_t w = __reduce_max_sync(0xffffffffu, v);
  if ((threadIdx.x & 31) == 0 && w) atomicMax(out, w);
}

}  // namespace gmpt
