// gpu_mpt.hpp -- the reference's C++ surface GpuMPT::Compress::MPT
// (mpt-with-compress/include/mpt/gpu_mpt.cuh:18-192) for the batched update
// path, header-only over the C ABI in gmpt.h (link with -lgmpt_b200).
//
// Kept from the reference: the class and method names, argument order and
// meaning (hex-nibble keys with inclusive int index pairs, values with
// inclusive int64_t pairs, caller host pointers echoed by lookups), the
// puts returning (device array of hash targets, count) that hash_onepass_v2
// consumes, and get_root_hash's (pointer, size) / tuple forms.
// Changed on purpose: failures throw gmpt_error instead of exit(); the root
// returned by get_root_hash is owned by the object (valid until the next
// call) instead of leaked; hash targets are node references (uint32_t), not
// Node* pointers.
#pragma once
#include <stdint.h>

#include <stdexcept>
#include <string>
#include <tuple>

#include "gmpt.h"

namespace GpuMPT {
namespace Compress {

struct gmpt_error : std::runtime_error {
  int code;
  gmpt_error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

class MPT {
 public:
  explicit MPT(int device = 0, int encode_mode = GMPT_MODE_REF) : t_(gmpt_create(device, encode_mode)) {
    if (!t_) throw gmpt_error(gmpt_last_error(), gmpt_last_error_message());
  }
  ~MPT() { gmpt_destroy(t_); }
  MPT(const MPT &) = delete;
  MPT &operator=(const MPT &) = delete;

  // gpu_mpt.cuh:95-97
  std::tuple<const uint32_t *, int> puts_2phase_with_valuehp(const uint8_t *keys_hexs, int *keys_indexs,
                                                            const uint8_t *values_bytes, int64_t *values_indexs,
                                                            const uint8_t **values_hps, int n) {
    check(gmpt_puts_2phase(t_, keys_hexs, keys_indexs, values_bytes, values_indexs, values_hps, n));
    return targets();
  }

  // gpu_mpt.cuh:69-71
  std::tuple<const uint32_t *, int> puts_latching_with_valuehp_v2(const uint8_t *keys_hexs, int *keys_indexs,
                                                                  const uint8_t *values_bytes,
                                                                  int64_t *values_indexs,
                                                                  const uint8_t **values_hps, int n) {
    check(gmpt_puts_latching(t_, keys_hexs, keys_indexs, values_bytes, values_indexs, values_hps, n));
    return targets();
  }

  // gpu_mpt.cuh:74-77 / 684-765: mixed batch, rw_flags[i] = 0 read, 1 write;
  // reads see the batch's earlier writes of their key (index order)
  std::tuple<const uint32_t *, int> puts_latching_with_valuehp_v2_with_read(
      const uint8_t *keys_hexs, int *keys_indexs, int &read_num, const uint8_t *rw_flags,
      const uint8_t *values_bytes, int64_t *values_indexs, const uint8_t **values_hps, int n,
      const uint8_t **read_values_hps, int *read_values_sizes) {
    check(gmpt_puts_latching_with_read(t_, keys_hexs, keys_indexs, &read_num, rw_flags, values_bytes, values_indexs,
                                       values_hps, n, read_values_hps, read_values_sizes));
    return targets();
  }

  // gpu_mpt.cuh:105-108 / 1609-1713
  std::tuple<const uint32_t *, int> puts_2phase_with_valuehp_with_read(
      const uint8_t *keys_hexs, int *keys_indexs, int &read_num, const uint8_t *rw_flags,
      const uint8_t *values_bytes, int64_t *values_indexs, const uint8_t **values_hps, int n,
      const uint8_t **read_values_hps, int *read_values_sizes) {
    check(gmpt_puts_2phase_with_read(t_, keys_hexs, keys_indexs, &read_num, rw_flags, values_bytes, values_indexs,
                                     values_hps, n, read_values_hps, read_values_sizes));
    return targets();
  }

  // gpu_mpt.cuh:131: hashes every pending dirty node (the targets returned by
  // the puts since the last call)
  void hash_onepass_v2(const uint32_t * /*d_hash_nodes*/ = nullptr, int /*n*/ = 0) {
    check(gmpt_hash_onepass(t_));
  }

  // gpu_mpt.cuh:139-140
  void gets_parallel(const uint8_t *keys_hexs, int *keys_indexs, int n, const uint8_t **values_hps,
                     int *values_sizes) const {
    check(gmpt_gets_parallel(t_, keys_hexs, keys_indexs, n, values_hps, values_sizes));
  }

  // gpu_mpt.cuh:151-152: hash = nullptr / size 0 for an empty trie
  void get_root_hash(const uint8_t *&hash, int &hash_size) const {
    check(gmpt_get_root_hash(t_, root_, &hash_size));
    hash = hash_size ? root_ : nullptr;
  }
  std::tuple<const uint8_t *, int> get_root_hash() const {
    const uint8_t *h;
    int s;
    get_root_hash(h, s);
    return {h, s};
  }

  gmpt_trie *handle() const { return t_; }

 private:
  gmpt_trie *t_;
  mutable uint8_t root_[32] = {};

  static void check(int rc) {
    if (rc) throw gmpt_error(rc, gmpt_last_error_message());
  }
  std::tuple<const uint32_t *, int> targets() {
    const uint32_t *d = nullptr;
    int n = 0;
    check(gmpt_pending_targets(t_, &d, &n));
    return {d, n};
  }
};

}  // namespace Compress
}  // namespace GpuMPT
