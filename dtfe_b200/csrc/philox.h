// Counter-based random offsets for the Monte-Carlo cell average.
//
// The reference draws U(-0.5,0.5) offsets from one sequential boost::mt19937
// stream seeded with randomSeed + 1000*partNo (averaged_interpolation_2.cc:97-102,
// three uni() calls per sample at :144).  A sequential stream cannot be split
// across GPU threads, and its three constructor-argument calls have no
// specified evaluation order, so the reference's offsets are not reproducible
// anyway.  Here every offset is a pure function of (seed, cell, sample, axis):
// Philox4x32 with 10 rounds (J. K. Salmon, M. A. Moraes, R. O. Dror,
// D. E. Shaw, "Parallel Random Numbers: As Easy as 1, 2, 3", SC'11), keyed by
// the seed and counted by (cell index, sample index).  The oracle uses the
// same definition, so GPU and oracle sample identical points.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define DTFE_RNG_HD __host__ __device__ __forceinline__
#else
#define DTFE_RNG_HD inline
#endif

namespace dtfe {

DTFE_RNG_HD void mulhilo32(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
  uint64_t p = (uint64_t)a * (uint64_t)b;
  hi = (uint32_t)(p >> 32);
  lo = (uint32_t)p;
}

// Philox4x32-10 block: counter c[4], key k[2] -> r[4].
DTFE_RNG_HD void philox4x32_10(const uint32_t c[4], const uint32_t k[2], uint32_t r[4]) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  uint32_t x0 = c[0], x1 = c[1], x2 = c[2], x3 = c[3];
  uint32_t k0 = k[0], k1 = k[1];
  for (int round = 0; round < 10; ++round) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(M0, x0, hi0, lo0);
    mulhilo32(M1, x2, hi1, lo1);
    uint32_t y0 = hi1 ^ x1 ^ k0;
    uint32_t y1 = lo1;
    uint32_t y2 = hi0 ^ x3 ^ k1;
    uint32_t y3 = lo0;
    x0 = y0; x1 = y1; x2 = y2; x3 = y3;
    k0 += W0;
    k1 += W1;
  }
  r[0] = x0; r[1] = x1; r[2] = x2; r[3] = x3;
}

// Key of a sub-box: the reference's seed + 1000*partNo (partNo < 0: no offset).
DTFE_RNG_HD uint64_t mc_key(uint64_t seed, int32_t part_no) {
  return part_no >= 0 ? seed + 1000ull * (uint64_t)part_no : seed;
}

// Three offsets in (-0.5, 0.5) for sample w of main-grid cell `cell`.
DTFE_RNG_HD void mc_offsets(uint64_t key, uint64_t cell, uint32_t w, double u[3]) {
  uint32_t c[4] = {(uint32_t)cell, (uint32_t)(cell >> 32), w, 0u};
  uint32_t k[2] = {(uint32_t)key, (uint32_t)(key >> 32)};
  uint32_t r[4];
  philox4x32_10(c, k, r);
  const double inv = 1.0 / 4294967296.0;
  u[0] = ((double)r[0] + 0.5) * inv - 0.5;
  u[1] = ((double)r[1] + 0.5) * inv - 0.5;
  u[2] = ((double)r[2] + 0.5) * inv - 0.5;
}

}  // namespace dtfe
