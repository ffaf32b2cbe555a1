// Driver of the reference's output writers — TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference's own src/input_output.cc (with its io/ readers and
// writers) unmodified against the stand-in headers and exposes
//   writeBinaryFile   src/io/binary_io.cc:185-216
//   writeOutputData   src/input_output.cc:216-275
// through C entry points, so tests can compare the files this project writes
// with the reference's byte for byte.  The HDF5 readers are not built (no
// HDF5 here); the one HDF5 call outside their #ifdef, in the density-file
// header reader, is given a stand-in that reports it.

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "define.h"
#include "particle_data.h"
#include "quantities.h"
#include "user_options.h"

struct Gadget_header;
void HDF5_readGadgetHeader(std::string filename, Gadget_header* gadgetHeader);

#include "input_output.cc"

void HDF5_readGadgetHeader(std::string filename, Gadget_header*) {
  std::fprintf(stderr, "reference IO harness: no HDF5 reader for %s\n", filename.c_str());
  std::abort();
}

namespace {
template <size_t N>
void write_pvectors(const float* data, int64_t n, const std::string& path) {
  std::vector<Pvector<Real, N>> v((size_t)n);
  for (int64_t i = 0; i < n; ++i)
    for (size_t c = 0; c < N; ++c) v[i][c] = data[(size_t)i * N + c];
  User_options opt;
  writeBinaryFile(v, path, "field", opt);
}
}  // namespace

extern "C" {

// writeBinaryFile of n rows of ncomp floats (1: std::vector<Real>; 3, 5, 9:
// std::vector<Pvector<Real, ncomp>>) into `path`.
int ref_write_binary(const char* path, const float* data, int64_t n, int ncomp) {
  const std::string p(path);
  User_options opt;
  switch (ncomp) {
    case 1: {
      std::vector<Real> v(data, data + n);
      writeBinaryFile(v, p, "field", opt);
      return 0;
    }
    case 3: write_pvectors<3>(data, n, p); return 0;
    case 5: write_pvectors<5>(data, n, p); return 0;
    case 9: write_pvectors<9>(data, n, p); return 0;
    default: return 1;
  }
}

// writeOutputData (outputFileType 101, binary) of the fields in the masks
// (bit = field slot: density, velocity, gradient, divergence, shear,
// vorticity, std, scalar, scalar gradient), each with n rows taken from
// u[slot] / a[slot], to `base` + the reference's suffixes.
int ref_write_output(const char* base, int64_t n, uint32_t u_mask, uint32_t a_mask, const float* const* u,
                     const float* const* a) {
  Quantities uq, aq;
  auto fill = [n](Quantities& q, uint32_t mask, const float* const* src, Field& f) {
    if (mask & 1u) { q.density.assign(src[0], src[0] + n); f.density = true; }
    if (mask & 2u) {
      q.velocity.resize(n);
      for (int64_t i = 0; i < n; ++i) for (int c = 0; c < 3; ++c) q.velocity[i][c] = src[1][3 * i + c];
      f.velocity = true;
    }
    if (mask & 4u) {
      q.velocity_gradient.resize(n);
      for (int64_t i = 0; i < n; ++i) for (int c = 0; c < 9; ++c) q.velocity_gradient[i][c] = src[2][9 * i + c];
      f.velocity_gradient = true;
    }
    if (mask & 8u) { q.velocity_divergence.assign(src[3], src[3] + n); f.velocity_divergence = true; }
    if (mask & 16u) {
      q.velocity_shear.resize(n);
      for (int64_t i = 0; i < n; ++i) for (int c = 0; c < 5; ++c) q.velocity_shear[i][c] = src[4][5 * i + c];
      f.velocity_shear = true;
    }
    if (mask & 32u) {
      q.velocity_vorticity.resize(n);
      for (int64_t i = 0; i < n; ++i) for (int c = 0; c < 3; ++c) q.velocity_vorticity[i][c] = src[5][3 * i + c];
      f.velocity_vorticity = true;
    }
    if (mask & 64u) { q.velocity_std.assign(src[6], src[6] + n); f.velocity_std = true; }
    if (mask & 128u) {
      q.scalar.resize(n);
      for (int64_t i = 0; i < n; ++i) q.scalar[i][0] = src[7][i];
      f.scalar = true;
    }
    if (mask & 256u) {
      q.scalar_gradient.resize(n);
      for (int64_t i = 0; i < n; ++i) for (int c = 0; c < 3; ++c) q.scalar_gradient[i][c] = src[8][3 * i + c];
      f.scalar_gradient = true;
    }
  };
  User_options opt;
  opt.outputFileType = 101;
  opt.outputFilename = base;
  fill(uq, u_mask, u, opt.uField);
  fill(aq, a_mask, a, opt.aField);
  writeOutputData(uq, aq, opt);
  return 0;
}

}  // extern "C"
