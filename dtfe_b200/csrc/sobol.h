// Sobol' quasi-random points in the unit cube (3 dimensions), host only.
//
// The construction of Bratley & Fox, "Algorithm 659: Implementing Sobol's
// quasirandom sequence generator", ACM Trans. Math. Software 14(1):88-100
// (1988), which GSL's gsl_qrng_sobol implements and the reference's
// averaging method 1 draws from (quasiRandomSequence,
// src/CGAL_triangulation/averaged_interpolation_1.cc:32-50):
//   * per dimension a primitive polynomial over GF(2) of degree d with
//     coefficients a_1..a_{d-1} and odd initial integers m_1..m_d
//     (dimension 1: every m_j = 1; dimension 2: x + 1, m_1 = 1;
//     dimension 3: x^2 + x + 1, m_1 = m_2 = 1 — the first entries of the
//     paper's tables);
//   * further integers by Sobol's recurrence
//     m_j = 2 a_1 m_{j-1} ^ 4 a_2 m_{j-2} ^ ... ^ 2^d m_{j-d} ^ m_{j-d};
//   * 30-bit direction numbers V_j = m_j 2^(30-j), j = 1..30;
//   * point k (k = 1, 2, ...) = the previous numerators XOR V_c, where c is
//     one plus the number of trailing one bits of k - 1 (Gray-code order), so
//     the origin is never returned and the first point is (1/2, 1/2, 1/2);
//   * coordinates = numerator / 2^30 (exact in double).
#pragma once

#include <cstddef>
#include <cstdint>

namespace dtfe {

class Sobol3 {
 public:
  static constexpr int kBits = 30;

  Sobol3() {
    // m_j per dimension (index j = 0 .. kBits-1 holds m_{j+1})
    uint32_t m[3][kBits];
    for (int j = 0; j < kBits; ++j) m[0][j] = 1u;
    // dimension 2: x + 1 (degree 1): m_j = 2 m_{j-1} ^ m_{j-1}
    m[1][0] = 1u;
    for (int j = 1; j < kBits; ++j) m[1][j] = (m[1][j - 1] << 1) ^ m[1][j - 1];
    // dimension 3: x^2 + x + 1 (degree 2, a_1 = 1): m_j = 2 m_{j-1} ^ 4 m_{j-2} ^ m_{j-2}
    m[2][0] = 1u;
    m[2][1] = 1u;
    for (int j = 2; j < kBits; ++j) m[2][j] = (m[2][j - 1] << 1) ^ (m[2][j - 2] << 2) ^ m[2][j - 2];
    for (int d = 0; d < 3; ++d)
      for (int j = 0; j < kBits; ++j) v_[d][j] = m[d][j] << (kBits - 1 - j);
    num_[0] = num_[1] = num_[2] = 0u;
    count_ = 0u;
  }

  // Next point; false once the 2^30 - 1 points are used up.
  bool next(double out[3]) {
    int c = 0;
    for (uint32_t k = count_; k & 1u; k >>= 1) ++c;
    if (c >= kBits) return false;
    for (int d = 0; d < 3; ++d) {
      num_[d] ^= v_[d][c];
      out[d] = (double)num_[d] / (double)(1u << kBits);
    }
    ++count_;
    return true;
  }

 private:
  uint32_t v_[3][kBits];
  uint32_t num_[3];
  uint32_t count_;
};

// The reference's method-1 table: the first n Sobol points whose coordinate
// sum, rounded to float, is at most 1 (points of the corner simplex
// x, y, z >= 0, x + y + z <= 1), stored as floats (3 per point).
inline void sobol_simplex_table(size_t n, float* out) {
  Sobol3 q;
  double r[3];
  for (size_t i = 0; i < n;) {
    if (!q.next(r)) return;
    const float sum = (float)(r[0] + r[1] + r[2]);
    if (sum <= 1.0) {
      out[3 * i + 0] = (float)r[0];
      out[3 * i + 1] = (float)r[1];
      out[3 * i + 2] = (float)r[2];
      ++i;
    }
  }
}

}  // namespace dtfe
