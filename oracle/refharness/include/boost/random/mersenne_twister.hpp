// Test-harness stand-in for boost::mt19937: the MT19937 generator of
// M. Matsumoto and T. Nishimura, ACM TOMACS 8 (1998), written from the paper.
#pragma once
#include <cstdint>
namespace boost {
class mt19937 {
  uint32_t x_[624];
  int i_ = 624;

 public:
  typedef uint32_t result_type;
  explicit mt19937(uint32_t seed = 5489u) {
    x_[0] = seed;
    for (int k = 1; k < 624; ++k) x_[k] = 1812433253u * (x_[k - 1] ^ (x_[k - 1] >> 30)) + (uint32_t)k;
  }
  static constexpr uint32_t min() { return 0u; }
  static constexpr uint32_t max() { return 0xffffffffu; }
  uint32_t operator()() {
    if (i_ >= 624) {
      for (int k = 0; k < 624; ++k) {
        uint32_t y = (x_[k] & 0x80000000u) | (x_[(k + 1) % 624] & 0x7fffffffu);
        x_[k] = x_[(k + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
      }
      i_ = 0;
    }
    uint32_t y = x_[i_++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
  }
};
}  // namespace boost
