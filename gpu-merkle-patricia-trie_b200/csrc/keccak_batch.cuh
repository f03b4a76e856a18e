// keccak_batch.cuh -- standalone batched Keccak-256 and the Keccak
// throughput probe used as the integer-ALU ceiling of the hash stage.
//
// k_keccak256_batch replaces the reference's keccak_kernel_batch
// (hash/batch_mode_hash.cuh:89-115; one warp per message, 25 active lanes,
// state in shared memory): one thread per message, state in registers,
// message words read with unaligned 8-byte loads.
#pragma once
#include "keccak.cuh"

namespace gmpt {

__global__ void __launch_bounds__(128) k_keccak256_batch(const uint8_t *data, const int64_t *offs, int n,
                                                         uint8_t *out) {
  extern __shared__ uint64_t stage_all[];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int64_t s = offs[2 * i], e = offs[2 * i + 1];
  uint64_t len = (e >= s - 1 && s >= 0) ? (uint64_t)(e - s + 1) : 0;
  const uint8_t *p = data + s;
  Sponge sp;
  sp.reset(stage_all + threadIdx.x, blockDim.x);
  uint64_t off = 0;
  bool last = false;
  while (true) {
    while (!sp.full()) {
      if (off < len) {
        uint32_t nb = (len - off) < 8 ? (uint32_t)(len - off) : 8u;
        sp.push(load_u64_unaligned(p + off) & low_bytes_mask(nb), nb);
        off += nb;
        continue;
      }
      sp.pad();
      last = true;
      break;
    }
    sp.absorb();
    if (last) break;
  }
  uint64_t *o = reinterpret_cast<uint64_t *>(out + 32 * (size_t)i);
  o[0] = sp.a[0];
  o[1] = sp.a[1];
  o[2] = sp.a[2];
  o[3] = sp.a[3];
}

// Register-only Keccak-f[1600] loop: no memory traffic inside the loop, so
// its rate is the integer-pipe ceiling for this permutation code.
__global__ void __launch_bounds__(128) k_keccak_peak(uint64_t *sink, int iters) {
  uint64_t a[25];
#pragma unroll
  for (int i = 0; i < 25; ++i) a[i] = (uint64_t)(blockIdx.x * blockDim.x + threadIdx.x) * 0x9E3779B97F4A7C15ull + i;
  for (int r = 0; r < iters; ++r) keccak_f1600(a);
  uint64_t x = 0;
#pragma unroll
  for (int i = 0; i < 25; ++i) x ^= a[i];
  if (x == 0x123456789ull) sink[0] = x;  // keeps the loop live
}

}  // namespace gmpt
