// ref_driver.cu -- exposes the reference's own CpuMPT (compiled from its
// sources, unmodified, through the shim headers in ref_shim/) behind a small
// extern "C" surface.  TEST INFRASTRUCTURE: the checker and the timed CPU
// baseline, never part of the shipped library.
//
// Entry points follow the reference's CPU API:
//   ref_puts_baseline  -> CpuMPT::Compress::MPT::puts_baseline  (cpu_mpt.cuh:359)
//   ref_hash_dirty     -> MPT::hashs_dirty_flag                  (cpu_mpt.cuh:498)
//   ref_puts_lock      -> MPT::puts_lock + hashs_onepass         (cpu_mpt.cuh:191,206)
//   ref_puts_2phase    -> MPT::puts_2phase + hashs_onepass       (cpu_mpt.cuh:165,206)
//   ref_gets           -> MPT::gets_baseline                     (cpu_mpt.cuh:568)
//   ref_root           -> MPT::get_root_hash                     (cpu_mpt.cuh:915)
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <tuple>
#include <vector>

#include "util/utils.cuh"
// The node arena is a compile-time capacity in the reference (4 GiB with
// -DGETH) that is zero-filled on construction; the driver picks a size that
// fits its use.  utils.cuh is #pragma once, so this redefinition is what the
// class template below sees.
#undef ALLOC_CAPACITY
#define ALLOC_CAPACITY REF_NODE_ARENA
#undef KEY_ALLOC_CAPACITY
#define KEY_ALLOC_CAPACITY (uint64_t(1) << 24)
// The reference MPT has no destructor that releases its arenas; open its
// members so the driver can release them between timed samples.
#define private public
#include "mpt/cpu_mpt.cuh"
#undef private

namespace CryptoPP {
void shim_keccak256(const byte *in, std::size_t len, byte *out32) {
  uint8_t st[200];
  CPUHash::keccak1600(in, len, st);
  std::memcpy(out32, st, 32);
}
}  // namespace CryptoPP

using RefMPT = CpuMPT::Compress::MPT;

extern "C" {

void ref_set_threads(int n) { tbb::g_shim_threads = n < 1 ? 1 : n; }

void *ref_new() { return new RefMPT(); }

void ref_delete(void *p) {
  RefMPT *m = static_cast<RefMPT *>(p);
  m->allocator_.free_all();
  m->key_allocator_.free_all();
  delete m;
}

void ref_puts_baseline(void *p, const uint8_t *keys_hexs, const int *keys_indexs,
                       const uint8_t *values, const int64_t *values_indexs,
                       int n) {
  static_cast<RefMPT *>(p)->puts_baseline(keys_hexs, keys_indexs, values,
                                          values_indexs, n);
}

void ref_hash_dirty(void *p) { static_cast<RefMPT *>(p)->hashs_dirty_flag(); }

// LockNU on the CPU (TBB parallel_for -> std::thread shim), then one-pass hash.
void ref_puts_lock(void *p, const uint8_t *keys_hexs, int *keys_indexs,
                   const uint8_t *values, int64_t *values_indexs, int n) {
  RefMPT *m = static_cast<RefMPT *>(p);
  auto [targets, num] = m->puts_lock(keys_hexs, keys_indexs, values, values_indexs, n);
  m->hashs_onepass(targets, num);
}

// PhaseNU on the CPU, then one-pass hash.
void ref_puts_2phase(void *p, const uint8_t *keys_hexs, int *keys_indexs,
                     const uint8_t *values, int64_t *values_indexs, int n) {
  RefMPT *m = static_cast<RefMPT *>(p);
  auto [targets, num] = m->puts_2phase(keys_hexs, keys_indexs, values, values_indexs, n);
  m->hashs_onepass(targets, num);
}

// Root reference after hashs_dirty_flag (sequential form).
int ref_root(void *p, uint8_t *out32) {
  const uint8_t *h = nullptr;
  int hs = 0;
  static_cast<RefMPT *>(p)->get_root_hash(h, hs);
  if (h && hs > 0) std::memcpy(out32, h, hs > 32 ? 32 : hs);
  return hs;
}

// Root reference after the parallel (lock / 2phase) forms.
int ref_root_parallel(void *p, uint8_t *out32) {
  const uint8_t *h = nullptr;
  int hs = 0;
  static_cast<RefMPT *>(p)->get_root_hash_parallel(h, hs);
  if (h && hs > 0) std::memcpy(out32, h, hs > 32 ? 32 : hs);
  return hs;
}

void ref_gets(void *p, const uint8_t *keys_hexs, const int *keys_indexs, int n,
              uint64_t *out_ptr, int *out_len) {
  std::vector<const uint8_t *> ptrs(n, nullptr);
  static_cast<RefMPT *>(p)->gets_baseline(keys_hexs, keys_indexs, n, ptrs.data(),
                                          out_len);
  for (int i = 0; i < n; ++i) out_ptr[i] = (uint64_t)(uintptr_t)ptrs[i];
}

void ref_keccak256(const uint8_t *in, uint64_t len, uint8_t *out32) {
  CPUHash::calculate_hash(in, (int)len, out32);
}

}  // extern "C"
