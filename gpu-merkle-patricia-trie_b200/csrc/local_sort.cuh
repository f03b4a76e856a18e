// local_sort.cuh -- CTA-local completion of the batch sort.
//
// The device-wide sort (Trie::sort_unique) refines ties one 8-nibble chunk
// at a time.  Once every still-tied run of positions holds at most
// kSortLocalCap keys, one CTA per run finishes it in shared memory: per
// chunk, a stable block radix sort of (tie-group rank << 32 | chunk) on the
// digits that vary, until no ties are left or the key length breaks them.
// Results are identical to continuing device-wide: the order is
// lexicographic (terminator before nibble 0) and equal keys keep their batch
// order, so the last one is the kept occurrence.
#pragma once
#include "trie_kernels.cuh"

namespace gmpt {

constexpr int kSortLocalCap = 2048;
constexpr int kSortLocalThreads = 256;
constexpr int kSortLocalWarps = kSortLocalThreads / 32;
constexpr int kSortLocalPerWarp = kSortLocalCap / kSortLocalWarps;  // 256 items, 8 rounds

// groups no larger than this are ordered by direct counting instead of radix passes
constexpr uint32_t kSortSmallGroup = 32;

struct LocalSortSmem {
  uint64_t key[2][kSortLocalCap];
  uint32_t val[2][kSortLocalCap];
  union {
    uint16_t cnt[kSortLocalWarps][256];  // radix pass: per-warp digit counts, then offsets (<= kSortLocalCap)
    uint16_t gbeg[kSortLocalCap];        // small-group pass: first position of every tied group
  };
  uint32_t warp_tmp[kSortLocalWarps + 1];
  unsigned long long mask;
  uint32_t maxlen;
  uint32_t maxg;
};
static_assert(kSortLocalWarps * 256 == kSortLocalCap, "gbeg shares the radix counters' space");

// block-wide exclusive scan of one value per thread
__device__ __forceinline__ uint32_t cta_excl_scan(uint32_t v, uint32_t *tmp, uint32_t &total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t u = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += u;
  }
  if (lane == 31) tmp[wid] = incl;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t run = 0;
    for (int w = 0; w < kSortLocalWarps; ++w) {
      uint32_t c = tmp[w];
      tmp[w] = run;
      run += c;
    }
    tmp[kSortLocalWarps] = run;
  }
  __syncthreads();
  total = tmp[kSortLocalWarps];
  uint32_t r = tmp[wid] + incl - v;
  __syncthreads();
  return r;
}

// one stable pass on digit `shift` of key[src] -> key[src ^ 1]
__device__ __forceinline__ void cta_radix_pass(LocalSortSmem &L, int src, int m, int shift) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < kSortLocalWarps * 256; i += kSortLocalThreads) (&L.cnt[0][0])[i] = 0;
  static_assert(kSortLocalCap < 65536, "digit offsets are 16-bit");
  __syncthreads();
  const unsigned lt = (1u << lane) - 1u;
  uint32_t rk[kSortLocalPerWarp / 32];
#pragma unroll
  for (int r = 0; r < kSortLocalPerWarp / 32; ++r) {
    int k = wid * kSortLocalPerWarp + r * 32 + lane;
    bool ok = k < m;
    uint32_t d = ok ? (uint32_t)((L.key[src][k] >> shift) & 0xFF) : (256u + lane);
    unsigned peers = __match_any_sync(0xffffffffu, d);
    uint32_t old = ok ? L.cnt[wid][d] : 0;
    __syncwarp();
    if (ok && (int)lane == __ffs(peers) - 1) L.cnt[wid][d] = (uint16_t)(old + __popc(peers));
    __syncwarp();
    rk[r] = old + __popc(peers & lt);
  }
  __syncthreads();
  // digit-major exclusive offsets: thread t owns digit t
  uint32_t tot = 0;
  for (int w = 0; w < kSortLocalWarps; ++w) tot += L.cnt[w][threadIdx.x];
  uint32_t all;
  uint32_t dbase = cta_excl_scan(tot, L.warp_tmp, all);
  {
    uint32_t run = dbase;
    for (int w = 0; w < kSortLocalWarps; ++w) {
      uint32_t c = L.cnt[w][threadIdx.x];
      L.cnt[w][threadIdx.x] = (uint16_t)run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kSortLocalPerWarp / 32; ++r) {
    int k = wid * kSortLocalPerWarp + r * 32 + lane;
    if (k < m) {
      uint64_t kk = L.key[src][k];
      uint32_t d = (uint32_t)((kk >> shift) & 0xFF);
      uint32_t dst = L.cnt[wid][d] + rk[r];
      L.key[src ^ 1][dst] = kk;
      L.val[src ^ 1][dst] = L.val[src][k];
    }
  }
  __syncthreads();
}

// seg_start / seg_end: position runs still tied before chunk c
__global__ void __launch_bounds__(kSortLocalThreads) k_local_sort(TrieView tv, const uint32_t *seg_start,
                                                                  const uint32_t *seg_end, int c0, uint32_t *order,
                                                                  uint8_t *eqprev, const uint64_t *koff,
                                                                  const uint32_t *klen) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  LocalSortSmem &L = *reinterpret_cast<LocalSortSmem *>(smem_raw);
  const uint32_t a = seg_start[blockIdx.x];
  const int m = (int)(seg_end[blockIdx.x] - a);
  if (m > kSortLocalCap || m < 2) {
    if (threadIdx.x == 0) set_error(tv.ctr, ERR_INTERNAL);
    return;
  }
  if (threadIdx.x == 0) L.maxlen = 0;
  __syncthreads();
  for (int k = threadIdx.x; k < m; k += kSortLocalThreads) {
    uint32_t it = order[a + k];
    L.val[0][k] = it;
    atomicMax(&L.maxlen, klen[it]);
  }
  __syncthreads();
  const int nchunks = (int)((L.maxlen + 7) / 8);
  int src = 0;
  // tied[k] == 1: item k equals item k-1 on everything compared so far
  // (all items start tied: they share the chunks before c0)
  for (int c = c0; c <= nchunks; ++c) {
    // group rank of each item = number of group starts before it
    // (thread t owns items [t*8, t*8+8))
    constexpr int ipt = kSortLocalCap / kSortLocalThreads;
    uint32_t starts = 0;
    uint8_t st[ipt], tp[ipt + 1];
#pragma unroll
    for (int r = 0; r <= ipt; ++r) {
      int k = threadIdx.x * ipt + r;  // r == ipt: the next thread's first item
      bool tied_prev;
      if (c == c0)
        tied_prev = k > 0 && k < m;
      else
        tied_prev = k > 0 && k < m && L.key[src][k] == L.key[src][k - 1];
      tp[r] = tied_prev ? 1 : 0;
      if (r == ipt) break;
      st[r] = (k < m && !tied_prev) ? 1 : 0;
      starts += st[r];
    }
    uint32_t ngroups;
    uint32_t rank = cta_excl_scan(starts, L.warp_tmp, ngroups);
    if (ngroups == (uint32_t)m) break;  // every key distinct
    // build (rank, chunk) keys in the current order
    if (threadIdx.x == 0) {
      L.mask = 0;
      L.maxg = 0;
    }
    __syncthreads();
    uint64_t acc = 0, k0 = 0;
    uint16_t gid[ipt];
#pragma unroll
    for (int r = 0; r < ipt; ++r) {
      int k = threadIdx.x * ipt + r;
      gid[r] = 0;
      if (k >= m) continue;
      rank += st[r];
      gid[r] = (uint16_t)(rank - 1);
      if (c > c0 && st[r]) L.gbeg[rank - 1] = (uint16_t)k;
      uint32_t it = L.val[src][k];
      // an item already alone in its group keeps its place whatever its
      // chunk: skip the gather of its key bytes
      const bool single = !tp[r] && !tp[r + 1];
      uint32_t ch = single ? 0u : (c < nchunks ? key_chunk(tv.keys, koff[it], klen[it], c) : klen[it]);
      uint64_t key = ((uint64_t)(rank - 1) << 32) | ch;
      L.key[src][k] = key;
    }
    if (c > c0 && threadIdx.x == 0) L.gbeg[ngroups] = (uint16_t)m;  // ngroups < m <= kSortLocalCap
    __syncthreads();
    if (c > c0) {
      // Largest tied group: when every group is small (the usual tail, a
      // few pairs among singletons), each item finds its place in its group
      // by counting the members that order before it -- one pass instead
      // of one radix pass per varying byte of (rank, chunk).
      uint32_t gmax = 0;
#pragma unroll
      for (int r = 0; r < ipt; ++r) {
        const int k = threadIdx.x * ipt + r;
        if (k < m && st[r]) gmax = max(gmax, (uint32_t)(L.gbeg[gid[r] + 1] - L.gbeg[gid[r]]));
      }
      gmax = __reduce_max_sync(0xffffffffu, gmax);
      if ((threadIdx.x & 31) == 0 && gmax) atomicMax(&L.maxg, gmax);
      __syncthreads();
      if (L.maxg <= kSortSmallGroup) {
#pragma unroll
        for (int r = 0; r < ipt; ++r) {
          const int k = threadIdx.x * ipt + r;
          if (k >= m) continue;
          const uint64_t key = L.key[src][k];
          const uint32_t b = L.gbeg[gid[r]], e = L.gbeg[gid[r] + 1];
          uint32_t pos = b;
          for (uint32_t j = b; j < e; ++j) {  // stable: equal chunks keep their order
            const uint64_t kj = L.key[src][j];
            pos += (kj < key || (kj == key && j < (uint32_t)k)) ? 1u : 0u;
          }
          L.key[src ^ 1][pos] = key;
          L.val[src ^ 1][pos] = L.val[src][k];
        }
        src ^= 1;
        __syncthreads();
        continue;
      }
    }
    k0 = L.key[src][0];
    for (int k = threadIdx.x; k < m; k += kSortLocalThreads) acc |= L.key[src][k] ^ k0;
    for (int o = 16; o; o >>= 1) acc |= __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc) atomicOr(&L.mask, (unsigned long long)acc);
    __syncthreads();
    uint64_t mask = L.mask;
    {
      // nibbles that vary move to the low end of every key when that saves
      // digit passes (the order and the equalities between keys are kept;
      // the keys are rebuilt from scratch for the next chunk)
      uint64_t nmask = 0;
      int nv = 0, bytes = 0;
      for (int k = 0; k < 16; ++k)
        if ((mask >> (4 * k)) & 0xFull) {
          nmask |= 0xFull << (4 * k);
          ++nv;
        }
      for (int b = 0; b < 8; ++b) bytes += ((mask >> (8 * b)) & 0xFFull) ? 1 : 0;
      if ((4 * nv + 7) / 8 < bytes) {
        for (int k = threadIdx.x; k < m; k += kSortLocalThreads) {
          const uint64_t x = L.key[src][k];
          uint64_t out = 0;
          for (int q = 15; q >= 0; --q)
            if ((nmask >> (4 * q)) & 0xFull) out = (out << 4) | ((x >> (4 * q)) & 0xFull);
          L.key[src][k] = out;
        }
        mask = nv >= 16 ? ~0ull : ((1ull << (4 * nv)) - 1);
        __syncthreads();
      }
    }
    for (int shift = 0; shift < 64; shift += 8) {
      if (((mask >> shift) & 0xFF) == 0) continue;
      cta_radix_pass(L, src, m, shift);
      src ^= 1;
    }
  }
  // final ties are exact duplicates (every chunk and the length equal)
  __syncthreads();
  for (int k = threadIdx.x; k < m; k += kSortLocalThreads) {
    order[a + k] = L.val[src][k];
    eqprev[a + k] = (k > 0 && L.key[src][k] == L.key[src][k - 1]) ? 1 : 0;
  }
}

// positions of each still-tied run (called with the sort_flags scan)
__global__ void k_sort_runs(const unsigned long long *flags, const unsigned long long *pos, const uint8_t *eqprev,
                            int n, uint32_t *seg_start, uint32_t *seg_end) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  unsigned long long f = flags[p];
  if (!(f & 1ull)) return;
  uint32_t seg = (uint32_t)(pos[p] >> 32) + (uint32_t)(f >> 32) - 1u;
  if (f >> 32) seg_start[seg] = (uint32_t)p;
  if (!eqprev[p + 1]) seg_end[seg] = (uint32_t)p + 1;
}

__global__ void k_run_max(const uint32_t *start, const uint32_t *end, int S, uint32_t *out) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t v = s < S ? end[s] - start[s] : 0u;
  uint32_t w = __reduce_max_sync(0xffffffffu, v);
  if ((threadIdx.x & 31) == 0 && w) atomicMax(out, w);
}

}  // namespace gmpt
