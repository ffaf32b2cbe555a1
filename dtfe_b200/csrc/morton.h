// Vertex order of a sub-box's point set: a stable Z-order permutation
// (quantisation to 21 bits per axis over the set's bounding box, in double).
// The planner numbers every sub-box's vertices in this order before
// tessellating them (dtfe_plan_build, dtfe_b200/plan.py morton_order), so
// neighbouring vertices sit close in memory for the device walk.
#pragma once

#include <algorithm>
#include <cstdint>
#include <numeric>
#include <vector>

namespace dtfe {

inline uint64_t spread21(uint64_t x) {
  x &= 0x1FFFFFull;
  x = (x | (x << 32)) & 0x1F00000000FFFFull;
  x = (x | (x << 16)) & 0x1F0000FF0000FFull;
  x = (x | (x << 8)) & 0x100F00F00F00F00Full;
  x = (x | (x << 4)) & 0x10C30C30C30C30C3ull;
  x = (x | (x << 2)) & 0x1249249249249249ull;
  return x;
}

// Permutation of n points (3 coordinates each, float values given as T)
// into Z-order; ties keep their input order.
template <class T>
std::vector<int64_t> morton_order(const T* pos, int64_t n) {
  std::vector<int64_t> order(n);
  std::iota(order.begin(), order.end(), 0);
  if (n == 0) return order;
  T mn[3] = {pos[0], pos[1], pos[2]}, mx[3] = {pos[0], pos[1], pos[2]};
  for (int64_t i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) {
      mn[c] = std::min(mn[c], pos[3 * i + c]);
      mx[c] = std::max(mx[c], pos[3 * i + c]);
    }
  double lo[3], ext[3];
  for (int c = 0; c < 3; ++c) {
    lo[c] = (double)mn[c];
    ext[c] = std::max((double)mx[c] - lo[c], 1e-30);
  }
  const double top = (double)((1 << 21) - 1);
  std::vector<uint64_t> key(n);
  for (int64_t i = 0; i < n; ++i) {
    uint64_t q[3];
    for (int c = 0; c < 3; ++c) {
      double v = ((double)pos[3 * i + c] - lo[c]) / ext[c] * top;
      v = v < 0.0 ? 0.0 : (v > top ? top : v);
      q[c] = (uint64_t)v;
    }
    key[i] = spread21(q[0]) | (spread21(q[1]) << 1) | (spread21(q[2]) << 2);
  }
  std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return key[a] < key[b]; });
  return order;
}

}  // namespace dtfe
