// ref_gpu_driver.cu -- the reference's own C ABI library (lib/libgmpt.cu),
// compiled unmodified from its sources for sm_100a, so its GPU LockNU +
// PhaseHC path (insert_mpt_olc -> puts_latching_with_valuehp_v2 ->
// hash_onepass_v2 -> get_root_hash, lib/libgmpt.cu:248-321) can be timed on
// the same B200 beside this repository's kernels.  BENCH/TEST INFRASTRUCTURE
// ONLY: nothing in the product loads it.
//
// The file only supplies what the reference's build takes from outside its
// tree: the Crypto++ Keccak_256 that cpu_mpt.cuh's hashing names (the shim
// header in ref_shim/ forwards to shim_keccak256, defined here on the
// reference's own CPUHash::keccak1600, rate 136, Keccak padding).
#include <chrono>

#include "libgmpt.cu"

namespace CryptoPP {
void shim_keccak256(const byte *in, std::size_t len, byte *out32) {
  uint8_t st[200];
  CPUHash::keccak1600(in, len, st);
  std::memcpy(out32, st, 32);
}
}  // namespace CryptoPP

// The reference's GPU MPT through its C++ class on the same batch, under the
// insert + hash pairings the reference uses (values_hps pointing at the
// values, as test/trie.cu:1207-1210 makes them); the root goes to out32.
//   variant 0: puts_latching_with_valuehp + hash_onepass (keys walk), the
//              pair test/trie.cu:1282-1293 times and test/trie.cu:1446-1451
//              checks against the CPU MPT
//   variant 1: puts_latching_with_valuehp_v2 + hash_onepass_v2, the pair
//              insert_mpt_olc runs (lib/libgmpt.cu:299-303)
//   variant 2: puts_2phase_with_valuehp + hash_onepass_v2
// Returns the root's size (32, or 0 for no root); -1 for an unknown variant.
// ms_out (optional): wall time of the insert + hash alone (the trie is built
// before the clock starts), with a device synchronisation on both sides.
extern "C" int ref_gpu_variant_root(int variant, const uint8_t *keys_hexs, int *keys_indexs,
                                    const uint8_t *values, int64_t *values_indexs, int n, uint8_t *out32,
                                    double *ms_out) {
  if (variant < 0 || variant > 2) return -1;
  GPUHashMultiThread::load_constants();
  const uint8_t **hps = new const uint8_t *[n];
  for (int i = 0; i < n; ++i) hps[i] = util::element_start(values_indexs, i, values);
  int size = 0;
  {
    GpuMPT::Compress::MPT mpt;
    cudaDeviceSynchronize();
    const auto t0 = std::chrono::steady_clock::now();
    if (variant == 0) {
      mpt.puts_latching_with_valuehp(keys_hexs, keys_indexs, values, values_indexs, hps, n);
      mpt.hash_onepass(keys_hexs, keys_indexs, n);
    } else if (variant == 1) {
      auto [nodes, cnt] = mpt.puts_latching_with_valuehp_v2(keys_hexs, keys_indexs, values, values_indexs, hps, n);
      mpt.hash_onepass_v2(nodes, cnt);
    } else {
      auto [nodes, cnt] = mpt.puts_2phase_with_valuehp(keys_hexs, keys_indexs, values, values_indexs, hps, n);
      mpt.hash_onepass_v2(nodes, cnt);
    }
    cudaDeviceSynchronize();
    if (ms_out)
      *ms_out = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    const uint8_t *h = nullptr;
    mpt.get_root_hash(h, size);
    if (h && size > 0) std::memcpy(out32, h, size < 32 ? size : 32);
    delete[] h;
  }
  delete[] hps;
  return size;
}

// The reference's warp-cooperative GPU Keccak-256 (hash/gpu_hash_kernel.cuh
// call_keccak_basic_kernel over hash/batch_mode_hash.cuh
// batch_keccak_device: one state spread over 25 lanes in shared memory) on
// one message; the digest goes to out32.  Messages whose length is a
// multiple of 8 bytes only: the helper zeroes just the first bytes of its
// last word (gpu_hash_kernel.cuh:198).
extern "C" int ref_gpu_keccak(const uint8_t *in, uint32_t len, uint8_t *out32) {
  if (len == 0 || (len & 7u)) return -1;
  GPUHashMultiThread::load_constants();
  GPUHashMultiThread::call_keccak_basic_kernel(in, len, out32);
  return 0;
}
