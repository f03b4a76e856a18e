// Shim for Crypto++'s Keccak_256 (test checker only).  It buffers the input
// and finishes with shim_keccak256, which the driver defines on top of the
// reference's own CPUHash::keccak1600 (rate 136, Keccak padding).
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>
namespace CryptoPP {
typedef unsigned char byte;
void shim_keccak256(const byte *in, std::size_t len, byte *out32);
class Keccak_256 {
 public:
  void Update(const byte *p, std::size_t n) { buf_.insert(buf_.end(), p, p + n); }
  void Final(byte *out) {
    shim_keccak256(buf_.data(), buf_.size(), out);
    buf_.clear();
  }
 private:
  std::vector<byte> buf_;
};
}  // namespace CryptoPP
