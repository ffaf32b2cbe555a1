// Test-harness stand-in for boost::uniform_real: a + (b - a) * u with
// u = engine() / 2^32 in [0, 1).  (Its values need not match Boost's: the
// harness compares only the deterministic methods against the oracle.)
#pragma once
namespace boost {
template <class RealType = double>
class uniform_real {
  RealType a_, b_;

 public:
  uniform_real(RealType a = 0, RealType b = 1) : a_(a), b_(b) {}
  template <class Engine>
  RealType operator()(Engine& e) const {
    return a_ + (b_ - a_) * (RealType)((double)e() / 4294967296.0);
  }
};
}  // namespace boost
