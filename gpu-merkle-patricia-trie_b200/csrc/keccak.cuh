// keccak.cuh -- Keccak-f[1600] with the 25 lanes in registers, and a
// streaming Keccak-256 sponge (rate 136 bytes, pad 0x01 ... 0x80).
//
// Follows FIPS 202 / the reference's CPUHash::keccakf + keccak
// (hash/cpu_hash.h:35-127) and its warp kernel's parameters
// (hash/batch_mode_hash.cuh:12-87: rate 1088 bits, Keccak padding, first 4
// lanes out).  The reference spreads one state over 25 lanes of a warp with
// the state in shared memory and table-driven indices; here each thread owns
// one whole sponge in registers (thread per node), so a warp hashes 32 nodes
// at once with no shuffles, no shared-memory state and no idle lanes.
#pragma once
#include <stdint.h>

namespace gmpt {

__device__ __forceinline__ uint64_t rotl64(uint64_t x, int n) {
  // a 64-bit rotate is two 32-bit funnel shifts
  uint32_t lo = (uint32_t)x, hi = (uint32_t)(x >> 32);
  if (n == 32) return ((uint64_t)lo << 32) | hi;
  if (n < 32) {
    uint32_t nh = __funnelshift_l(lo, hi, n);
    uint32_t nl = __funnelshift_l(hi, lo, n);
    return ((uint64_t)nh << 32) | nl;
  }
  uint32_t nh = __funnelshift_l(hi, lo, n - 32);
  uint32_t nl = __funnelshift_l(lo, hi, n - 32);
  return ((uint64_t)nh << 32) | nl;
}

__constant__ uint64_t kKeccakRC[24] = {
    0x0000000000000001ULL, 0x0000000000008082ULL, 0x800000000000808aULL,
    0x8000000080008000ULL, 0x000000000000808bULL, 0x0000000080000001ULL,
    0x8000000080008081ULL, 0x8000000000008009ULL, 0x000000000000008aULL,
    0x0000000000000088ULL, 0x0000000080008009ULL, 0x000000008000000aULL,
    0x000000008000808bULL, 0x800000000000008bULL, 0x8000000000008089ULL,
    0x8000000000008003ULL, 0x8000000000008002ULL, 0x8000000000000080ULL,
    0x000000000000800aULL, 0x800000008000000aULL, 0x8000000080008081ULL,
    0x8000000000008080ULL, 0x0000000080000001ULL, 0x8000000080008008ULL};

// One round; lanes a[x + 5y].  rho offsets and the pi lane order are the
// FIPS 202 constants, written out so every index is a compile-time constant.
__device__ __forceinline__ void keccak_round(uint64_t (&a)[25], uint64_t rc) {
  uint64_t c0 = a[0] ^ a[5] ^ a[10] ^ a[15] ^ a[20];
  uint64_t c1 = a[1] ^ a[6] ^ a[11] ^ a[16] ^ a[21];
  uint64_t c2 = a[2] ^ a[7] ^ a[12] ^ a[17] ^ a[22];
  uint64_t c3 = a[3] ^ a[8] ^ a[13] ^ a[18] ^ a[23];
  uint64_t c4 = a[4] ^ a[9] ^ a[14] ^ a[19] ^ a[24];
  uint64_t d0 = c4 ^ rotl64(c1, 1);
  uint64_t d1 = c0 ^ rotl64(c2, 1);
  uint64_t d2 = c1 ^ rotl64(c3, 1);
  uint64_t d3 = c2 ^ rotl64(c4, 1);
  uint64_t d4 = c3 ^ rotl64(c0, 1);
  // theta + rho + pi: b[y + 5((2x + 3y) % 5)] = rot(a[x + 5y] ^ d[x], r[x][y])
  uint64_t b00 = a[0] ^ d0;
  uint64_t b10 = rotl64(a[6] ^ d1, 44);
  uint64_t b20 = rotl64(a[12] ^ d2, 43);
  uint64_t b30 = rotl64(a[18] ^ d3, 21);
  uint64_t b40 = rotl64(a[24] ^ d4, 14);
  uint64_t b01 = rotl64(a[3] ^ d3, 28);
  uint64_t b11 = rotl64(a[9] ^ d4, 20);
  uint64_t b21 = rotl64(a[10] ^ d0, 3);
  uint64_t b31 = rotl64(a[16] ^ d1, 45);
  uint64_t b41 = rotl64(a[22] ^ d2, 61);
  uint64_t b02 = rotl64(a[1] ^ d1, 1);
  uint64_t b12 = rotl64(a[7] ^ d2, 6);
  uint64_t b22 = rotl64(a[13] ^ d3, 25);
  uint64_t b32 = rotl64(a[19] ^ d4, 8);
  uint64_t b42 = rotl64(a[20] ^ d0, 18);
  uint64_t b03 = rotl64(a[4] ^ d4, 27);
  uint64_t b13 = rotl64(a[5] ^ d0, 36);
  uint64_t b23 = rotl64(a[11] ^ d1, 10);
  uint64_t b33 = rotl64(a[17] ^ d2, 15);
  uint64_t b43 = rotl64(a[23] ^ d3, 56);
  uint64_t b04 = rotl64(a[2] ^ d2, 62);
  uint64_t b14 = rotl64(a[8] ^ d3, 55);
  uint64_t b24 = rotl64(a[14] ^ d4, 39);
  uint64_t b34 = rotl64(a[15] ^ d0, 41);
  uint64_t b44 = rotl64(a[21] ^ d1, 2);
  // chi (row y uses b?y) + iota
  a[0] = b00 ^ (~b10 & b20) ^ rc;
  a[1] = b10 ^ (~b20 & b30);
  a[2] = b20 ^ (~b30 & b40);
  a[3] = b30 ^ (~b40 & b00);
  a[4] = b40 ^ (~b00 & b10);
  a[5] = b01 ^ (~b11 & b21);
  a[6] = b11 ^ (~b21 & b31);
  a[7] = b21 ^ (~b31 & b41);
  a[8] = b31 ^ (~b41 & b01);
  a[9] = b41 ^ (~b01 & b11);
  a[10] = b02 ^ (~b12 & b22);
  a[11] = b12 ^ (~b22 & b32);
  a[12] = b22 ^ (~b32 & b42);
  a[13] = b32 ^ (~b42 & b02);
  a[14] = b42 ^ (~b02 & b12);
  a[15] = b03 ^ (~b13 & b23);
  a[16] = b13 ^ (~b23 & b33);
  a[17] = b23 ^ (~b33 & b43);
  a[18] = b33 ^ (~b43 & b03);
  a[19] = b43 ^ (~b03 & b13);
  a[20] = b04 ^ (~b14 & b24);
  a[21] = b14 ^ (~b24 & b34);
  a[22] = b24 ^ (~b34 & b44);
  a[23] = b34 ^ (~b44 & b04);
  a[24] = b44 ^ (~b04 & b14);
}

__device__ __forceinline__ void keccak_f1600(uint64_t (&a)[25]) {
#pragma unroll 4
  for (int r = 0; r < 24; ++r) keccak_round(a, kKeccakRC[r]);
}

// Keccak-f[1600] spread over a warp: lane t < 25 holds lane t = x + 5y of
// the state, the other lanes carry copies that nothing reads.  A round is
// ten 64-bit shuffles (theta's column sums, the two neighbour columns,
// pi's lane permutation, chi's two row neighbours) around a handful of
// integer ops per lane, so one permutation's latency is a few shuffle
// round trips per round instead of one thread's whole serial chain: the
// form for nodes whose many blocks would otherwise set a level's time.
struct CoopLanes {
  uint32_t col[5];   // theta: the lanes of this lane's column
  uint32_t cm1, cp1; // lanes holding column x - 1 and x + 1
  uint32_t rot;      // rho offset of this lane
  uint32_t src;      // pi: the lane whose rotated word lands here
  uint32_t chi1, chi2;
};

__device__ __forceinline__ CoopLanes coop_lanes(int lane) {
  // rho offsets r[x][y] (FIPS 202), indexed x + 5y
  constexpr uint8_t kRho[25] = {0,  1,  62, 28, 27, 36, 44, 6,  55, 20, 3,  10, 43,
                                25, 39, 41, 45, 15, 21, 8,  18, 2,  61, 56, 14};
  const uint32_t t = (uint32_t)lane < 25u ? (uint32_t)lane : (uint32_t)lane - 25u;
  const uint32_t x = t % 5u, y = t / 5u;
  CoopLanes c;
#pragma unroll
  for (int k = 0; k < 5; ++k) c.col[k] = x + 5u * (uint32_t)k;
  c.cm1 = (x + 4u) % 5u;
  c.cp1 = (x + 1u) % 5u;
  c.rot = kRho[t];
  // pi: B[x'][y'] = A[x][y] with x' = y, y' = (2x + 3y) mod 5; here (x', y')
  // = (x, y), so the source has y_s = x and x_s = 3 (y - 3x) mod 5
  const uint32_t xs = (3u * (y + 15u - 3u * x)) % 5u, ys = x;
  c.src = xs + 5u * ys;
  c.chi1 = (x + 1u) % 5u + 5u * y;
  c.chi2 = (x + 2u) % 5u + 5u * y;
  return c;
}

__device__ __forceinline__ uint64_t rotl64_var(uint64_t v, uint32_t r) {
  uint32_t lo = (uint32_t)v, hi = (uint32_t)(v >> 32);
  if (r & 32u) {
    const uint32_t t = lo;
    lo = hi;
    hi = t;
  }
  const uint32_t s = r & 31u;
  const uint32_t nh = __funnelshift_l(lo, hi, s), nl = __funnelshift_l(hi, lo, s);
  return ((uint64_t)nh << 32) | nl;
}

// All 32 lanes call it together; returns this lane's state word after the
// permutation.
__device__ __forceinline__ uint64_t keccak_f1600_warp(uint64_t a, const CoopLanes &c, int lane) {
  constexpr unsigned kAll = 0xffffffffu;
#pragma unroll 1
  for (int r = 0; r < 24; ++r) {
    const uint64_t cs = __shfl_sync(kAll, a, c.col[0]) ^ __shfl_sync(kAll, a, c.col[1]) ^
                        __shfl_sync(kAll, a, c.col[2]) ^ __shfl_sync(kAll, a, c.col[3]) ^
                        __shfl_sync(kAll, a, c.col[4]);
    const uint64_t dm = __shfl_sync(kAll, cs, c.cm1), dp = __shfl_sync(kAll, cs, c.cp1);
    a ^= dm ^ rotl64(dp, 1);
    const uint64_t b = __shfl_sync(kAll, rotl64_var(a, c.rot), c.src);
    const uint64_t b1 = __shfl_sync(kAll, b, c.chi1), b2 = __shfl_sync(kAll, b, c.chi2);
    a = b ^ (~b1 & b2);
    if (lane == 0) a ^= kKeccakRC[r];
  }
  return a;
}

// Streaming sponge.  Message bytes are pushed in little-endian runs of <= 8
// bytes; whole 64-bit words go to this thread's 17-word staging block in
// shared memory (word w at stage[w * stride]), which absorb() folds into the
// register state.  Callers absorb when full() after a push (a push emits at
// most one word), so the permutation has a single call site.
struct Sponge {
  uint64_t a[25];
  uint64_t acc;      // partial word
  uint32_t accn;     // bytes in acc (0..7)
  uint32_t w;        // words staged in this block (0..17)
  uint64_t *stage;
  uint32_t stride;

  __device__ __forceinline__ void reset(uint64_t *st, uint32_t strd) {
#pragma unroll
    for (int i = 0; i < 25; ++i) a[i] = 0;
    acc = 0;
    accn = 0;
    w = 0;
    stage = st;
    stride = strd;
  }
  __device__ __forceinline__ bool full() const { return w == 17; }
  __device__ __forceinline__ void emit(uint64_t word) {
    stage[w * stride] = word;
    ++w;
  }
  // push n (1..8) bytes held little-endian in v; bytes >= n of v are zero
  __device__ __forceinline__ void push(uint64_t v, uint32_t n) {
    if (accn == 0) {
      if (n == 8) {
        emit(v);
      } else {
        acc = v;
        accn = n;
      }
      return;
    }
    uint32_t t = accn + n;
    uint64_t merged = acc | (v << (8 * accn));
    if (t >= 8) {
      emit(merged);
      acc = (t > 8) ? (v >> (8 * (8 - accn))) : 0;
      accn = t - 8;
    } else {
      acc = merged;
      accn = t;
    }
  }
  // Keccak padding of the final block (pad byte 0x01, last byte |= 0x80)
  __device__ __forceinline__ void pad() {
    stage[w * stride] = acc | (0x01ull << (8 * accn));
    for (uint32_t j = w + 1; j < 17; ++j) stage[j * stride] = 0;
    stage[16 * stride] ^= 0x8000000000000000ull;
    w = 17;
    acc = 0;
    accn = 0;
  }
  __device__ __forceinline__ void absorb() {
#pragma unroll
    for (int i = 0; i < 17; ++i) a[i] ^= stage[i * stride];
    keccak_f1600(a);
    w = 0;
  }
};

__device__ __forceinline__ uint64_t low_bytes_mask(uint32_t n) {
  return n >= 8 ? ~0ull : ((1ull << (8 * n)) - 1);
}

}  // namespace gmpt
