// Second translation unit of the reference-code harness — TEST INFRASTRUCTURE
// ONLY.  It compiles the reference's own host planning and grid-deposition
// sources (src/subpartition.h, src/quantities.cc, src/NGP_interpolation.cc,
// src/CIC_interpolation.cc, src/TSC_interpolation.cc — included the way
// src/DTFE.cpp includes them) and exposes them through C entry points, so
// tests can compare this project's restatements with the reference's code:
//
//   ref_parallel_grid        parallelGrid            subpartition.h:454-555
//   ref_optimal_partition    optimalPartitionSplit   subpartition.h:215-372
//   ref_select_in_box        findParticlesInBox      subpartition.h:79-154
//   ref_average_density      averageDensity          subpartition.h:437-449
//   ref_deposit              NGP/CIC/TSC_interpolation_regular_grid
//   ref_sph                  SPH_interpolation (src/SPH_interpolation.cc:47-146,
//                            252-474) over the reference's kd-tree
//                            (src/kdtree/kdtree2.cpp, its own translation unit)

#include <cmath>
#include <cstdint>
#include <cstring>
#include <iostream>
#include <list>
#include <vector>

#include "define.h"
#include "particle_data.h"
#include "user_options.h"
#include "quantities.h"
#include "subpartition.h"
#include "miscellaneous.h"
#include "message.h"

using namespace std;
#include "quantities.cc"
#include "NGP_interpolation.cc"
#include "CIC_interpolation.cc"
#include "TSC_interpolation.cc"
#include "SPH_interpolation.cc"

namespace {

std::vector<Particle_data> make_particles(const float* pos, const float* w, const float* vel, int64_t n) {
  std::vector<Particle_data> p(n);
  for (int64_t i = 0; i < n; ++i) {
    for (int k = 0; k < 3; ++k) p[i].pos[k] = pos[3 * i + k];
    p[i].weight() = w ? w[i] : 1.f;
    for (int k = 0; k < 3; ++k) p[i].velocity(k) = vel ? vel[3 * i + k] : 0.f;
  }
  return p;
}

}  // namespace

extern "C" {

void ref_parallel_grid(int64_t n_threads, const int64_t grid[3], int64_t out[3]) {
  User_options opt;
  opt.gridSize.assign(grid, grid + 3);
  size_t g[3];
  parallelGrid((size_t)n_threads, opt, g);
  for (int i = 0; i < 3; ++i) out[i] = (int64_t)g[i];
}

int ref_optimal_partition(const float* pos, int64_t n, const int64_t grid[3], const float region[6],
                          const int64_t parts[3], int64_t* subgrid, float* coords) {
  std::vector<Particle_data> p = make_particles(pos, nullptr, nullptr, n);
  User_options opt;
  opt.gridSize.assign(grid, grid + 3);
  opt.region.coords.assign(region, region + 6);
  std::vector<size_t> part(parts, parts + 3);
  std::vector<std::vector<size_t>> sub;
  std::vector<Box> sc;
  optimalPartitionSplit(p, opt, part, &sub, &sc);
  for (size_t k = 0; k < sub.size(); ++k)
    for (int a = 0; a < 6; ++a) {
      subgrid[6 * k + a] = (int64_t)sub[k][a];
      coords[6 * k + a] = sc[k][a];
    }
  return 0;
}

int64_t ref_select_in_box(const float* pos, int64_t n, const float full_box[6], const float padded[6], int periodic,
                          float* out_pos) {
  std::vector<Particle_data> p = make_particles(pos, nullptr, nullptr, n), o;
  User_options opt;
  opt.periodic = periodic != 0;
  opt.paddedBox.coords.assign(padded, padded + 6);
  opt.boxCoordinates.coords.assign(full_box, full_box + 6);
  findParticlesInBox(p, &o, opt);
  if (out_pos)
    for (size_t i = 0; i < o.size(); ++i)
      for (int k = 0; k < 3; ++k) out_pos[3 * i + k] = o[i].pos[k];
  return (int64_t)o.size();
}

float ref_average_density(const float* w, int64_t n) {
  std::vector<Particle_data> p = make_particles(std::vector<float>(3 * n, 0.f).data(), w, nullptr, n);
  User_options opt;
  return averageDensity(p, opt);
}

// kind: 0 NGP, 1 CIC, 2 TSC.  density: G floats, velocity: 3G floats (may be
// NULL to skip that field).  average_density: the value the reference
// normalises by.
int ref_deposit(int kind, const float* pos, const float* w, const float* vel, int64_t n, const float region[6],
                const int32_t grid[3], double average_density, float* density, float* velocity) {
  std::vector<Particle_data> p = make_particles(pos, w, vel, n);
  User_options opt;
  opt.gridSize.assign(grid, grid + 3);
  opt.region.coords.assign(region, region + 6);
  opt.averageDensity = (Real)average_density;
  opt.aField.density = density != nullptr;
  opt.aField.velocity = velocity != nullptr;
  Quantities q;
  if (kind == 0) NGP_interpolation_regular_grid(p, opt, &q);
  else if (kind == 1) CIC_interpolation_regular_grid(p, opt, &q);
  else if (kind == 2) TSC_interpolation_regular_grid(p, opt, &q);
  else return 1;
  const size_t G = (size_t)grid[0] * grid[1] * grid[2];
  if (density && q.density.size() == G) std::memcpy(density, q.density.data(), G * sizeof(float));
  if (velocity && q.velocity.size() == G) std::memcpy(velocity, q.velocity.data(), 3 * G * sizeof(float));
  return 0;
}

// SPH density (and velocity) of n particles on the grid of one region, with
// n_neighbors neighbours, normalised by average_density.
// scal: one scalar per particle (NO_SCALARS=1) or NULL; extensive selects
// the reference's extensive-scalar convention.
int ref_sph(const float* pos, const float* w, const float* vel, const float* scal, int extensive, int64_t n,
            const float region[6], const int32_t grid[3], double average_density, int n_neighbors, float* density,
            float* velocity, float* scalar) {
  std::vector<Particle_data> p = make_particles(pos, w, vel, n);
  if (scal)
    for (int64_t i = 0; i < n; ++i) p[i].scalar(0) = scal[i];
  User_options opt;
  opt.extensive = extensive != 0;
  opt.aField.scalar = scalar != nullptr;
  opt.DTFE = false;
  opt.SPH = true;
  opt.SPH_neighbors = n_neighbors;
  opt.gridSize.assign(grid, grid + 3);
  opt.region.coords.assign(region, region + 6);
  opt.averageDensity = (Real)average_density;
  opt.aField.density = true;
  opt.aField.velocity = velocity != nullptr;
  std::vector<Sample_point> samples;
  Quantities q;
  SPH_interpolation(&p, samples, opt, &q);
  const size_t G = (size_t)grid[0] * grid[1] * grid[2];
  if (q.density.size() != G) return 2;
  if (density) std::memcpy(density, q.density.data(), G * sizeof(float));
  if (velocity && q.velocity.size() == G) std::memcpy(velocity, q.velocity.data(), 3 * G * sizeof(float));
  if (scalar && q.scalar.size() == G) std::memcpy(scalar, q.scalar.data(), G * sizeof(float));
  return 0;
}

}  // extern "C"
