// gen_kernels.cuh -- seeded synthetic request batches generated in HBM (the
// request-stream bench and tests), so multi-million-key batches need no host
// generation or copies.  Not part of the update path.
//
//   ids     key i of a batch is a fresh id (next_new + running count) with
//           probability p_new, else an existing id drawn zipf(theta) over
//           [0, n_existing) with Gray et al.'s generator (YCSB
//           ZipfianGenerator), scrambled by FNV-1a so hot ids spread out;
//   keys    id -> key_bytes bytes (splitmix64 stream of (seed, id)) expanded
//           to hex nibbles + terminator, back to back, int32 index pairs;
//   values  (seed, batch position) -> value_bytes random bytes, int64 pairs.
#pragma once
#include <stdint.h>

#include "common.cuh"

namespace gmpt {

__host__ __device__ __forceinline__ uint64_t gen_mix(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

__device__ __forceinline__ uint64_t fnv1a64_u64(uint64_t v) {
  uint64_t h = 0xCBF29CE484222325ull;
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    h ^= v & 0xFF;
    h *= 1099511628211ull;
    v >>= 8;
  }
  return h;
}

struct ZipfParams {
  double theta, alpha, eta, zetan, half_pow;  // Gray et al. constants
  int64_t items;
};

// new-key flags and zipf ranks; ids of new keys are assigned by the host
// after a scan (k_gen_new_ids), so fresh ids stay dense
__global__ void k_gen_ids(uint64_t seed, int64_t n, double p_new, ZipfParams z, int64_t *ids, uint32_t *is_new) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t r0 = gen_mix(seed ^ (0xA24BAED4963EE407ull * (uint64_t)(i + 1)));
  const uint64_t r1 = gen_mix(r0);
  const double u0 = (double)(r0 >> 11) * (1.0 / 9007199254740992.0);
  const bool fresh = z.items <= 0 || u0 < p_new;
  is_new[i] = fresh ? 1u : 0u;
  if (fresh) {
    ids[i] = -1;
    return;
  }
  int64_t rank;
  const double u = (double)(r1 >> 11) * (1.0 / 9007199254740992.0);
  if (z.theta <= 0.0) {
    rank = (int64_t)(u * (double)z.items);
  } else {
    const double uz = u * z.zetan;
    if (uz < 1.0)
      rank = 0;
    else if (uz < 1.0 + z.half_pow)
      rank = 1;
    else
      rank = (int64_t)((double)z.items * pow(z.eta * u - z.eta + 1.0, z.alpha));
  }
  rank = rank < 0 ? 0 : (rank >= z.items ? z.items - 1 : rank);
  ids[i] = (int64_t)(fnv1a64_u64((uint64_t)rank) % (uint64_t)z.items);
}

__global__ void k_gen_widen(const uint32_t *f, int64_t n, unsigned long long *out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = f[i];
}

// ids of fresh keys: next_new + their exclusive rank among fresh keys
__global__ void k_gen_new_ids(const uint32_t *is_new, const unsigned long long *rank, int64_t n, int64_t next_new,
                              int64_t *ids) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (is_new[i]) ids[i] = next_new + (int64_t)rank[i];
}

__global__ void k_gen_keys(uint64_t seed, const int64_t *ids, int64_t n, int key_bytes, uint8_t *hexs, int *idx) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t w = 2 * (int64_t)key_bytes + 1;
  uint8_t *o = hexs + i * w;
  const uint64_t base = gen_mix(seed ^ (0xD6E8FEB86659FD93ull * (uint64_t)(ids[i] + 1)));
  for (int j = 0; j < key_bytes; j += 8) {
    const uint64_t r = gen_mix(base + (uint64_t)j);
    for (int b = 0; b < 8 && j + b < key_bytes; ++b) {
      const uint8_t x = (uint8_t)(r >> (8 * b));
      o[2 * (j + b)] = x >> 4;
      o[2 * (j + b) + 1] = x & 15;
    }
  }
  o[2 * key_bytes] = 16;
  idx[2 * i] = (int)(i * w);
  idx[2 * i + 1] = (int)(i * w + w - 1);
}

__global__ void k_gen_values(uint64_t seed, int64_t n, int value_bytes, uint8_t *vals, int64_t *idx) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint8_t *o = vals + i * value_bytes;
  const uint64_t base = gen_mix(seed ^ (0x9FB21C651E98DF25ull * (uint64_t)(i + 1)));
  for (int j = 0; j < value_bytes; j += 8) {
    const uint64_t r = gen_mix(base + (uint64_t)j);
    for (int b = 0; b < 8 && j + b < value_bytes; ++b) o[j + b] = (uint8_t)(r >> (8 * b));
  }
  idx[2 * i] = i * value_bytes;
  idx[2 * i + 1] = i * value_bytes + value_bytes - 1;
}

}  // namespace gmpt

namespace gmpt {

// Selector features of a staged key batch from 64 evenly spaced keys, one
// CTA: mean and spread of key length (nibbles), share of sampled keys equal
// to an earlier sample, and mean over samples of the longest common prefix
// with any other sample (= with its neighbour in sorted order) over the mean
// length.  out[4].
// Reads only bytes [0, keys_bytes) of `keys` (ranges outside count as empty
// keys) and compares byte by byte, so the caller's buffer needs no padding.
__global__ void __launch_bounds__(64) k_sample_features(const uint8_t *keys, const int *kidx, int n,
                                                        int64_t keys_bytes, float *out) {
  __shared__ int s_off[64], s_len[64];
  __shared__ float red[4][64];
  const int j = threadIdx.x;
  const int s = n < 64 ? n : 64;
  if (j < s) {
    const int64_t i = (int64_t)j * n / s;
    const int a = kidx[2 * i], z = kidx[2 * i + 1];
    const bool ok = a >= 0 && z >= a && (int64_t)z < keys_bytes;
    s_off[j] = ok ? a : 0;
    s_len[j] = ok ? z - a + 1 : 0;
  }
  __syncthreads();
  float len = 0.f, dup = 0.f, lcp = 0.f;
  if (j < s) {
    const uint8_t *a = keys + s_off[j];
    const int la = s_len[j];
    int best = 0;
    bool earlier = false;
    for (int k = 0; k < s; ++k) {
      if (k == j) continue;
      const int lb = s_len[k];
      const int m = la < lb ? la : lb;
      const uint8_t *b = keys + s_off[k];
      int l = 0;
      while (l < m && a[l] == b[l]) ++l;
      if (l == m && la == lb && k < j) earlier = true;
      best = l > best ? l : best;
    }
    len = (float)la;
    dup = earlier ? 1.f : 0.f;
    lcp = (float)best;
  }
  __shared__ float s_mean;
  red[0][j] = len;
  red[2][j] = dup;
  red[3][j] = lcp;
  __syncthreads();
  if (j == 0) {
    float t = 0.f;
    for (int k = 0; k < s; ++k) t += red[0][k];
    s_mean = s > 0 ? t / (float)s : 0.f;
  }
  __syncthreads();
  const float d = len - s_mean;  // two-pass variance (no cancellation)
  red[1][j] = j < s ? d * d : 0.f;
  __syncthreads();
  if (j < 4 && j > 0) {
    float t = 0.f;
    for (int k = 0; k < s; ++k) t += red[j][k];
    red[j][0] = t;  // row j's slot 0 is read only by thread j
  }
  __syncthreads();
  if (j == 0) {
    const float inv = s > 0 ? 1.f / (float)s : 0.f;
    const float mean = s_mean;
    out[0] = mean;
    out[1] = sqrtf(red[1][0] * inv);
    out[2] = red[2][0] * inv;
    out[3] = mean > 0.f ? red[3][0] * inv / mean : 0.f;
  }
}

}  // namespace gmpt
