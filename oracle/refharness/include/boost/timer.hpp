// Test-harness stand-in for boost::timer (elapsed seconds since restart).
#pragma once
#include <chrono>
namespace boost {
class timer {
  std::chrono::steady_clock::time_point t0_ = std::chrono::steady_clock::now();

 public:
  double elapsed() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
  }
  void restart() { t0_ = std::chrono::steady_clock::now(); }
};
}  // namespace boost
