// Test-harness stand-in for boost::variate_generator.
#pragma once
namespace boost {
template <class Engine, class Dist>
class variate_generator {
  Engine e_;
  Dist d_;

 public:
  variate_generator(Engine e, Dist d) : e_(e), d_(d) {}
  double operator()() { return d_(e_); }
};
}  // namespace boost
