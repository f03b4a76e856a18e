// prims.cuh -- device-wide scan and stable radix sort used by the batch
// pipeline (sort/dedup of keys, grouping by anchor, level compaction).
//
// Both are written for sm_100a without any library: the scan is
// reduce-then-scan (three launches, no CTA ever waits on another), the sort
// is a least-significant-digit radix sort on 8-bit digits that skips every
// digit in which no key differs (the OR of key ^ key[0] is computed first),
// so a batch of keys with long shared prefixes pays only for the bits that
// vary.  Stability comes from per-warp match_any ranking in item order.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "common.cuh"

namespace gmpt {

// Kernel launches issued by this library (process-wide, host side).
uint64_t launch_count();
void count_launch();

// ---------------------------------------------------------------------------
// device buffer with grow-on-demand (workspace)

struct DevBlock {
  void *p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t need) {
    if (need <= bytes) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    size_t nb = need + need / 4 + 256;
    cudaError_t e = cudaMalloc(&p, nb);
    if (e == cudaSuccess) bytes = nb;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <typename T>
  T *as() const { return static_cast<T *>(p); }
};

// ---------------------------------------------------------------------------
// scan

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;

template <typename T>
__device__ __forceinline__ T block_excl_scan(T v, T *smem_warp, T &total) {
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  T incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T u = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += u;
  }
  if (lane == 31) smem_warp[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    int nw = blockDim.x >> 5;
    T x = lane < nw ? smem_warp[lane] : T(0);
    T xi = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T u = __shfl_up_sync(0xffffffffu, xi, o);
      if (lane >= o) xi += u;
    }
    if (lane < nw) smem_warp[lane] = xi - x;
    if (lane == nw - 1) smem_warp[32] = xi;
  }
  __syncthreads();
  total = smem_warp[32];
  T r = smem_warp[wid] + incl - v;
  __syncthreads();
  return r;
}

template <typename T>
__global__ void k_scan_reduce(const T *in, T *tile_sums, int64_t n) {
  __shared__ T sw[33];
  int64_t base = (int64_t)blockIdx.x * kScanTile;
  T s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    int64_t idx = base + (int64_t)i * kScanThreads + threadIdx.x;
    if (idx < n) s += in[idx];
  }
  T tot;
  block_excl_scan<T>(s, sw, tot);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = tot;
}

// exclusive scan of one tile per CTA, adding tile_offsets[blockIdx.x]
template <typename T>
__global__ void k_scan_tiles(const T *in, T *out, const T *tile_offsets, int64_t n, T *total_out) {
  __shared__ T sw[33];
  int64_t base = (int64_t)blockIdx.x * kScanTile;
  T v[kScanItems];
  T s = 0;
  // each thread owns a contiguous run of kScanItems elements
  int64_t my = base + (int64_t)threadIdx.x * kScanItems;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    int64_t idx = my + i;
    v[i] = idx < n ? in[idx] : T(0);
    s += v[i];
  }
  T tot;
  T run = block_excl_scan<T>(s, sw, tot);
  T off = tile_offsets ? tile_offsets[blockIdx.x] : T(0);
  run += off;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    int64_t idx = my + i;
    if (idx < n) out[idx] = run;
    run += v[i];
  }
  if (total_out && blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) *total_out = off + tot;
}

// Exclusive scan of n elements; *total_out (device) receives the sum.
// `ws` holds the tile sums of every recursion level.
template <typename T>
cudaError_t exclusive_scan(const T *in, T *out, int64_t n, T *total_out, DevBlock &ws,
                           cudaStream_t st, size_t ws_off = 0) {
  if (n <= 0) {
    if (total_out) return cudaMemsetAsync(total_out, 0, sizeof(T), st);
    return cudaSuccess;
  }
  int64_t tiles = (n + kScanTile - 1) / kScanTile;
  if (tiles == 1) {
    count_launch(), k_scan_tiles<T><<<1, kScanThreads, 0, st>>>(in, out, nullptr, n, total_out);
    return cudaGetLastError();
  }
  size_t need = ws_off + (size_t)(2 * tiles + 64) * sizeof(T);
  if (ws.bytes < need) return cudaErrorMemoryAllocation;  // caller sizes ws
  T *sums = reinterpret_cast<T *>(static_cast<char *>(ws.p) + ws_off);
  T *offs = sums + tiles;
  count_launch(), k_scan_reduce<T><<<(unsigned)tiles, kScanThreads, 0, st>>>(in, sums, n);
  cudaError_t e = exclusive_scan<T>(sums, offs, tiles, (T *)nullptr, ws, st,
                                    ws_off + (size_t)(2 * tiles + 32) * sizeof(T));
  if (e != cudaSuccess) return e;
  count_launch(), k_scan_tiles<T><<<(unsigned)tiles, kScanThreads, 0, st>>>(in, out, offs, n, total_out);
  return cudaGetLastError();
}

// workspace bytes needed by exclusive_scan<T>(n)
template <typename T>
size_t scan_ws_bytes(int64_t n) {
  size_t b = 0;
  while (n > kScanTile) {
    int64_t tiles = (n + kScanTile - 1) / kScanTile;
    b += (size_t)(2 * tiles + 64) * sizeof(T);
    n = tiles;
  }
  return b + 1024;
}

// ---------------------------------------------------------------------------
// radix sort of (u64 key, u32 value) pairs

constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096
constexpr int kSortWarps = kSortThreads / 32;

static __global__ void k_or_diff(const uint64_t *keys, int64_t n, unsigned long long *mask) {
  __shared__ unsigned long long s;
  if (threadIdx.x == 0) s = 0;
  __syncthreads();
  uint64_t k0 = keys[0];
  uint64_t acc = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    acc |= keys[i] ^ k0;
  for (int o = 16; o; o >>= 1) acc |= __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0 && acc) atomicOr(&s, (unsigned long long)acc);
  __syncthreads();
  if (threadIdx.x == 0 && s) atomicOr(mask, s);
}

// Nibble packing around the digit passes: the nibbles that vary across the
// keys (nmask) move, in order, to the low end of each key, so a key whose
// varying bits are spread over many bytes (one nibble in each of several
// bytes, as in nibble-per-byte keys) sorts in fewer 8-bit passes.  Packing
// keeps the order (it drops only nibbles that are equal in every key), and
// unpacking puts them back next to the common nibbles of key k0.
static __global__ void k_nibble_pack(uint64_t *keys, int64_t n, uint64_t nmask) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t x = keys[i];
  uint64_t out = 0;
  for (int k = 15; k >= 0; --k)
    if ((nmask >> (4 * k)) & 0xFull) out = (out << 4) | ((x >> (4 * k)) & 0xFull);
  keys[i] = out;
}

static __global__ void k_nibble_unpack(uint64_t *keys, int64_t n, uint64_t nmask, uint64_t k0) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint64_t p = keys[i];
  uint64_t x = k0 & ~nmask;
  for (int k = 0; k < 16; ++k)
    if ((nmask >> (4 * k)) & 0xFull) {
      x |= (p & 0xFull) << (4 * k);
      p >>= 4;
    }
  keys[i] = x;
}

static __global__ void k_radix_hist(const uint64_t *keys, int64_t n, int shift, uint32_t *counts, int tiles) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  int64_t base = (int64_t)blockIdx.x * kSortTile;
#pragma unroll 4
  for (int i = 0; i < kSortItems; ++i) {
    int64_t idx = base + (int64_t)i * kSortThreads + threadIdx.x;
    if (idx < n) atomicAdd(&h[(keys[idx] >> shift) & 0xFF], 1u);
  }
  __syncthreads();
  counts[(int64_t)threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

static __global__ void __launch_bounds__(kSortThreads)
k_radix_scatter(const uint64_t *keys, const uint32_t *vals, uint64_t *okeys, uint32_t *ovals,
                int64_t n, int shift, const uint32_t *offsets, int tiles) {
  __shared__ uint32_t cnt[kSortWarps][256];
  __shared__ uint32_t gb[256];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < kSortWarps * 256; i += kSortThreads) (&cnt[0][0])[i] = 0;
  gb[threadIdx.x] = offsets[(int64_t)threadIdx.x * tiles + blockIdx.x];
  __syncthreads();
  int64_t base = (int64_t)blockIdx.x * kSortTile + (int64_t)wid * (kSortTile / kSortWarps);
  uint64_t k[kSortItems];
  uint32_t v[kSortItems];
  uint32_t rk[kSortItems];
  unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    int64_t idx = base + r * 32 + lane;
    bool ok = idx < n;
    k[r] = ok ? keys[idx] : 0;
    v[r] = ok ? vals[idx] : 0;
    uint32_t d = ok ? (uint32_t)((k[r] >> shift) & 0xFF) : (256u + lane);
    unsigned peers = __match_any_sync(0xffffffffu, d);
    uint32_t old = ok ? cnt[wid][d] : 0;
    __syncwarp();
    if (ok && (int)lane == __ffs(peers) - 1) cnt[wid][d] = old + __popc(peers);
    __syncwarp();
    rk[r] = old + __popc(peers & lt);
  }
  __syncthreads();
  // exclusive prefix over warps, per digit
  {
    uint32_t run = 0;
    for (int w = 0; w < kSortWarps; ++w) {
      uint32_t c = cnt[w][threadIdx.x];
      cnt[w][threadIdx.x] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    int64_t idx = base + r * 32 + lane;
    if (idx < n) {
      uint32_t d = (uint32_t)((k[r] >> shift) & 0xFF);
      uint32_t dst = gb[d] + cnt[wid][d] + rk[r];
      okeys[dst] = k[r];
      ovals[dst] = v[r];
    }
  }
}

// Sorting context: alternate buffers and counters, grown on demand.
struct RadixSorter {
  DevBlock alt_keys, alt_vals, counts, scan_ws, mask;
  unsigned long long *h_mask = nullptr;  // pinned

  cudaError_t init() {
    cudaError_t e = mask.ensure(64);
    if (e != cudaSuccess) return e;
    if (!h_mask) e = cudaMallocHost(&h_mask, 2 * sizeof(unsigned long long));
    return e;
  }
  void release() {
    alt_keys.release();
    alt_vals.release();
    counts.release();
    scan_ws.release();
    mask.release();
    if (h_mask) cudaFreeHost(h_mask);
    h_mask = nullptr;
  }

  // Stable sort of keys/vals (in place: results end in keys/vals).
  // Returns the number of digit passes run in *passes (optional).
  cudaError_t sort(uint64_t *keys, uint32_t *vals, int64_t n, cudaStream_t st, int *passes = nullptr) {
    if (passes) *passes = 0;
    if (n <= 1) return cudaSuccess;
    cudaError_t e;
    if ((e = init()) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(mask.p, 0, 8, st)) != cudaSuccess) return e;
    int grid = (int)((n + 1023) / 1024);
    if (grid > 2048) grid = 2048;
    count_launch(), k_or_diff<<<grid, 256, 0, st>>>(keys, n, mask.as<unsigned long long>());
    // the varying bits and the first key (its nibbles are every key's common ones)
    if ((e = cudaMemcpyAsync(h_mask, mask.p, 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(h_mask + 1, keys, 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
    uint64_t m = h_mask[0];
    const uint64_t k0 = h_mask[1];
    if (m == 0) return cudaSuccess;
    uint64_t nmask = 0;
    int nv = 0, bytes = 0;
    for (int k = 0; k < 16; ++k)
      if ((m >> (4 * k)) & 0xFull) {
        nmask |= 0xFull << (4 * k);
        ++nv;
      }
    for (int b = 0; b < 8; ++b) bytes += ((m >> (8 * b)) & 0xFFull) ? 1 : 0;
    const bool pack = (4 * nv + 7) / 8 < bytes;
    if (pack) {
      count_launch(), k_nibble_pack<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(keys, n, nmask);
      m = nv >= 16 ? ~0ull : ((1ull << (4 * nv)) - 1);
    }
    int tiles = (int)((n + kSortTile - 1) / kSortTile);
    if ((e = alt_keys.ensure((size_t)n * 8)) != cudaSuccess) return e;
    if ((e = alt_vals.ensure((size_t)n * 4)) != cudaSuccess) return e;
    if ((e = counts.ensure((size_t)tiles * 256 * 4 * 2)) != cudaSuccess) return e;
    if ((e = scan_ws.ensure(scan_ws_bytes<uint32_t>((int64_t)tiles * 256))) != cudaSuccess) return e;
    uint64_t *kin = keys, *kout = alt_keys.as<uint64_t>();
    uint32_t *vin = vals, *vout = alt_vals.as<uint32_t>();
    uint32_t *cnt = counts.as<uint32_t>();
    uint32_t *off = cnt + (size_t)tiles * 256;
    int np = 0;
    for (int shift = 0; shift < 64; shift += 8) {
      if (((m >> shift) & 0xFF) == 0) continue;
      count_launch(), k_radix_hist<<<tiles, kSortThreads, 0, st>>>(kin, n, shift, cnt, tiles);
      if ((e = exclusive_scan<uint32_t>(cnt, off, (int64_t)tiles * 256, nullptr, scan_ws, st)) != cudaSuccess)
        return e;
      count_launch(), k_radix_scatter<<<tiles, kSortThreads, 0, st>>>(kin, vin, kout, vout, n, shift, off, tiles);
      std::swap(kin, kout);
      std::swap(vin, vout);
      ++np;
    }
    if (passes) *passes = np;
    if (kin != keys) {
      if ((e = cudaMemcpyAsync(keys, kin, (size_t)n * 8, cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return e;
      if ((e = cudaMemcpyAsync(vals, vin, (size_t)n * 4, cudaMemcpyDeviceToDevice, st)) != cudaSuccess) return e;
    }
    if (pack) count_launch(), k_nibble_unpack<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(keys, n, nmask, k0);
    return cudaGetLastError();
  }
};

}  // namespace gmpt
