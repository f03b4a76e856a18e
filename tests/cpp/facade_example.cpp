// Uses the GpuMPT::Compress::MPT facade the way the reference's tests use
// the reference class (test/trie.cu:1604-1656): the doe/dog/dogglesworth
// batch, PhaseNU, hash, lookups.  Prints the root as hex.
#include <cstdio>
#include <cstring>

#include "gpu_mpt.hpp"

int main() {
  const char *keys[3] = {"doe", "dog", "dogglesworth"};
  const char *vals[3] = {"reindeer", "puppy", "cat"};
  uint8_t hex[64];
  int kidx[6];
  int pos = 0;
  for (int i = 0; i < 3; ++i) {
    int l = (int)std::strlen(keys[i]);
    kidx[2 * i] = pos;
    for (int j = 0; j < l; ++j) {
      hex[pos++] = (uint8_t)keys[i][j] >> 4;
      hex[pos++] = (uint8_t)keys[i][j] & 15;
    }
    hex[pos++] = 16;
    kidx[2 * i + 1] = pos - 1;
  }
  uint8_t vbytes[32];
  int64_t vidx[6];
  int vp = 0;
  const uint8_t *hps[3];
  for (int i = 0; i < 3; ++i) {
    int l = (int)std::strlen(vals[i]);
    vidx[2 * i] = vp;
    std::memcpy(vbytes + vp, vals[i], l);
    hps[i] = reinterpret_cast<const uint8_t *>(vals[i]);
    vp += l;
    vidx[2 * i + 1] = vp - 1;
  }
  GpuMPT::Compress::MPT mpt;
  auto [targets, n] = mpt.puts_2phase_with_valuehp(hex, kidx, vbytes, vidx, hps, 3);
  mpt.hash_onepass_v2(targets, n);
  const uint8_t *out[3];
  int sizes[3];
  mpt.gets_parallel(hex, kidx, 3, out, sizes);
  for (int i = 0; i < 3; ++i)
    if (out[i] != hps[i] || sizes[i] != (int)std::strlen(vals[i])) return 2;
  auto [root, rs] = mpt.get_root_hash();
  for (int i = 0; i < rs; ++i) std::printf("%02x", root[i]);
  std::printf("\n");
  return 0;
}
