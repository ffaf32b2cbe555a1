// Test-harness stand-in for the part of boost::multi_array that the
// reference's kd-tree (src/kdtree/kdtree2.hpp, .cpp) and SPH sampler use: a
// dense row-major 2-D float array built from extents[n][m], with shape() and
// a[i][j] access.
#pragma once
#include <cstddef>
#include <vector>

namespace boost {
namespace harness_ma {
struct extent2 {
  std::size_t n0, n1;
};
struct extent1 {
  std::size_t n0;
  extent2 operator[](std::size_t n1) const { return {n0, n1}; }
};
struct extent0 {
  extent1 operator[](std::size_t n0) const { return {n0}; }
};
}  // namespace harness_ma

static const harness_ma::extent0 extents = {};

template <class T, std::size_t D>
class multi_array;

template <class T>
class multi_array<T, 2> {
  std::vector<T> data_;
  std::size_t shape_[2] = {0, 0};

 public:
  multi_array() = default;
  explicit multi_array(const harness_ma::extent2& e) { resize(e); }
  void resize(const harness_ma::extent2& e) {
    shape_[0] = e.n0;
    shape_[1] = e.n1;
    data_.assign(e.n0 * e.n1, T());
  }
  const std::size_t* shape() const { return shape_; }
  T* operator[](std::size_t i) { return data_.data() + i * shape_[1]; }
  const T* operator[](std::size_t i) const { return data_.data() + i * shape_[1]; }
};

template <class T, std::size_t D>
class const_multi_array_ref;
}  // namespace boost
