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
#include "libgmpt.cu"

namespace CryptoPP {
void shim_keccak256(const byte *in, std::size_t len, byte *out32) {
  uint8_t st[200];
  CPUHash::keccak1600(in, len, st);
  std::memcpy(out32, st, 32);
}
}  // namespace CryptoPP
