// Driver of the reference-code harness — TEST INFRASTRUCTURE ONLY.
//
// Links against the reference's own src/CGAL_triangulation/triangulation.cpp
// (compiled unmodified from the reference tree against cgal_facade.h and the
// stand-in headers under include/) and exposes its interpolation functions
// through a C entry point, so tests can run the reference's arithmetic on
// exactly the tessellation the GPU path and the oracle use:
//
//   vertexDensity               triangulation.cpp:200-279
//   interpolateGrid             unaveraged_interpolation.cc:209-369
//   interpolateGrid_averaged_2  averaged_interpolation_2.cc:35-233
//   interpolateGrid_averaged_3  averaged_interpolation_2.cc:664-866
//   interpolateUserSampling     unaveraged_interpolation.cc:560-691
//   interpolateRedshiftCone     unaveraged_interpolation.cc:381-547
//   interpolateUserSampling_averaged_2, interpolateRedshiftCone_averaged_2
//                               averaged_interpolation_2.cc:245-647
//   interpolateGrid_averaged_1  averaged_interpolation_1.cc:197-421 (Sobol points
//                               from dtfe_b200/csrc/sobol.h behind the GSL API)
//
// The reference's command-line layer (user_options.cc, boost::program_options)
// is not built; the User_options constructor below sets the members those
// functions read, with the reference's defaults (src/user_options.cc:39-92).

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <gsl/gsl_qrng.h>

#include "../../dtfe_b200/csrc/sobol.h"

#include "define.h"
#include "CGAL_triangulation/CGAL_include_3D.h"
#include "particle_data.h"
#include "quantities.h"
#include "user_options.h"

void vertexDensity(DT& dt, User_options& userOptions);
void interpolateGrid(DT& dt, User_options& userOptions, Quantities* quantities);
void interpolateGrid_averaged_2(DT& dt, User_options& userOptions, Quantities* quantities);
void interpolateGrid_averaged_3(DT& dt, User_options& userOptions, Quantities* quantities);
void interpolateGrid_averaged_1(DT& dt, User_options& userOptions, Quantities* quantities);
void interpolateUserSampling(DT& dt, std::vector<Sample_point>& samples, User_options& userOptions,
                             Quantities* quantities);
void interpolateRedshiftCone(DT& dt, User_options& userOptions, Quantities* quantities);
void interpolateUserSampling_averaged_2(DT& dt, std::vector<Sample_point>& samples, User_options& userOptions,
                                        Quantities* quantities);
void interpolateRedshiftCone_averaged_2(DT& dt, User_options& userOptions, Quantities* quantities);

User_options::User_options() {
  periodic = false;
  boxCoordinates.assign(0.);
  userGivenBoxCoordinates = false;
  inputFileType = 101;
  outputFileType = 101;
  regionOn = false;
  regionMpcOn = false;
  partitionOn = false;
  partNo = -1;
  paddingOn = false;
  paddingMpcOn = false;
  paddingParticles = Real(5.);
  testPaddedBoundaries = false;
  method = 1;
  noPoints = 100;
  noPointsOn = false;
  averageDensity = Real(-1.);
  randomSeed = 0;
  redshiftConeOn = false;
  DTFE = true;
  NGP = CIC = TSC = SPH = false;
  SPH_neighbors = 32;
  MpcValue = Real(1.);
  extensive = false;
  verboseLevel = 0;
  randomSample = Real(-1.);
  poisson = 0;
  transformToRedshiftSpaceOn = false;
  paddedBox.assign(0.);
  userDefinedSampling = false;
  noProcessors = 1;
  threadId = 0;
  totalTime = Real(0.);
}

extern "C" {

// GSL stand-ins: gsl_standin.cpp (linked into the same library).


// Runs the reference on one (sub-box) tessellation with LOCAL indices.
//   which: 0 cell-centre (interpolateGrid), 1 / 2 / 3 averaging methods.
//   dens_override (may be NULL): vertex densities used for the interpolation
//   instead of the reference's own (float-accumulated) ones.
//   outputs (float, Quantities layout; NULL to skip): vertex densities,
//   density, velocity, gradient, scalar (S = 1), scalar gradient, velocity std.
// seconds (may be NULL) receives the wall time of the reference's own work:
// vertexDensity + the interpolation call (not the facade's loading).
int ref_interpolate_timed(int64_t nv, const float* xyz, const float* w, const float* vel, const float* scal,
                          int64_t nt, const int32_t* tv, const int32_t* tn, const float region[6],
                          const int32_t grid[3], int which, int n_points, uint64_t seed, double rho_bar,
                          const float* dens_override, float* out_vdens, float* out_density, float* out_velocity,
                          float* out_gradient, float* out_scalar, float* out_scalar_gradient, float* out_std,
                          uint32_t extra_fields, double* seconds) {
  DT dt;
  const std::vector<DT::Vertex*>& verts = dt.load_flat(nv, xyz, nt, tv, tn);
  for (int64_t i = 0; i < nv; ++i) {
    vertexData& d = verts[i]->info();
    d.weight() = w[i];
    for (int c = 0; c < 3; ++c) d.velocity(c) = vel ? vel[3 * i + c] : 0.f;
    d.scalar(0) = scal ? scal[i] : 0.f;
  }
  User_options opt;
  opt.averageDensity = (Real)rho_bar;
  opt.gridSize.assign(grid, grid + 3);
  opt.region.coords.assign(region, region + 6);
  opt.method = which;
  opt.noPoints = n_points;
  opt.randomSeed = (size_t)seed;
  const auto t0 = std::chrono::steady_clock::now();
  vertexDensity(dt, opt);
  const auto t1 = std::chrono::steady_clock::now();
  for (int64_t i = 0; i < nv; ++i) {
    if (out_vdens) out_vdens[i] = verts[i]->info().density();
    if (dens_override) verts[i]->info().setDensity(dens_override[i]);
  }
  Quantities q;
  Field f;
  f.density = out_density != nullptr;
  f.velocity = out_velocity != nullptr;
  f.velocity_gradient = out_gradient != nullptr;
  f.scalar = out_scalar != nullptr;
  f.scalar_gradient = out_scalar_gradient != nullptr;
  f.velocity_std = out_std != nullptr && which == 2;
  // extra_fields bit 0..2: velocity divergence, shear, vorticity (computed by
  // the reference from the gradient, src/DTFE.cpp:394-475, outside the timing)
  if (extra_fields & 7u) f.velocity_gradient = true;
  const auto t2 = std::chrono::steady_clock::now();
  if (which == 0) {
    opt.uField = f;
    interpolateGrid(dt, opt, &q);
  } else if (which == 1) {
    opt.aField = f;
    interpolateGrid_averaged_1(dt, opt, &q);
  } else if (which == 2) {
    opt.aField = f;
    interpolateGrid_averaged_2(dt, opt, &q);
  } else if (which == 3) {
    opt.aField = f;
    interpolateGrid_averaged_3(dt, opt, &q);
  } else {
    return 1;
  }
  const auto t3 = std::chrono::steady_clock::now();
  if (seconds)
    *seconds = std::chrono::duration<double>(t1 - t0).count() + std::chrono::duration<double>(t3 - t2).count();
  const size_t G = (size_t)grid[0] * grid[1] * grid[2];
  auto copy = [&](float* dst, const float* src, size_t n, size_t have) {
    if (dst && have == G) std::memcpy(dst, src, n * sizeof(float));
  };
  copy(out_density, q.density.data(), G, q.density.size());
  copy(out_velocity, (const float*)q.velocity.data(), 3 * G, q.velocity.size());
  copy(out_gradient, (const float*)q.velocity_gradient.data(), 9 * G, q.velocity_gradient.size());
  copy(out_scalar, (const float*)q.scalar.data(), G, q.scalar.size());
  copy(out_scalar_gradient, (const float*)q.scalar_gradient.data(), 3 * G, q.scalar_gradient.size());
  copy(out_std, q.velocity_std.data(), G, q.velocity_std.size());
  return 0;
}

// The reference's interpolateUserSampling (unaveraged_interpolation.cc:560-691)
// at n points (3 floats each) in `region`, with the given vertex densities:
// the fields of the points inside the region, in order (*n_out of them).
int ref_interpolate_points(int64_t nv, const float* xyz, const float* w, const float* vel, const float* scal,
                           int64_t nt, const int32_t* tv, const int32_t* tn, const float region[6], int64_t n,
                           const float* pts, const float* dens, float* out_density, float* out_velocity,
                           float* out_gradient, float* out_scalar, float* out_scalar_gradient, int64_t* n_out,
                           double* seconds) {
  DT dt;
  const std::vector<DT::Vertex*>& verts = dt.load_flat(nv, xyz, nt, tv, tn);
  for (int64_t i = 0; i < nv; ++i) {
    vertexData& d = verts[i]->info();
    d.weight() = w[i];
    for (int c = 0; c < 3; ++c) d.velocity(c) = vel ? vel[3 * i + c] : 0.f;
    d.scalar(0) = scal ? scal[i] : 0.f;
    d.setDensity(dens[i]);
  }
  User_options opt;
  opt.region.coords.assign(region, region + 6);
  opt.userDefinedSampling = true;
  std::vector<Sample_point> samples((size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    float p[3] = {pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]};
    samples[i].setPosition(p);
  }
  Quantities q;
  Field f;
  f.density = out_density != nullptr;
  f.velocity = out_velocity != nullptr;
  f.velocity_gradient = out_gradient != nullptr;
  f.scalar = out_scalar != nullptr;
  f.scalar_gradient = out_scalar_gradient != nullptr;
  opt.uField = f;
  const auto t0 = std::chrono::steady_clock::now();
  interpolateUserSampling(dt, samples, opt, &q);
  if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  const size_t m = f.density ? q.density.size() : (f.velocity ? q.velocity.size() : q.velocity_gradient.size());
  *n_out = (int64_t)m;
  if (out_density && q.density.size() == m) std::memcpy(out_density, q.density.data(), m * sizeof(float));
  if (out_velocity && q.velocity.size() == m) std::memcpy(out_velocity, q.velocity.data(), 3 * m * sizeof(float));
  if (out_gradient && q.velocity_gradient.size() == m)
    std::memcpy(out_gradient, q.velocity_gradient.data(), 9 * m * sizeof(float));
  if (out_scalar && q.scalar.size() == m) std::memcpy(out_scalar, q.scalar.data(), m * sizeof(float));
  if (out_scalar_gradient && q.scalar_gradient.size() == m)
    std::memcpy(out_scalar_gradient, q.scalar_gradient.data(), 3 * m * sizeof(float));
  return 0;
}

// interpolateRedshiftCone on one tessellation (LOCAL indices) with the given
// vertex densities: cone = (r_min, r_max, theta_min, theta_max, psi_min,
// psi_max) in Mpc and degrees, dims = (n_r, n_theta, n_psi).  Outputs hold
// dims[0] dims[1] dims[2] rows (NULL to skip a field); *seconds (if not NULL)
// = the wall time of the interpolateRedshiftCone call alone.
int ref_interpolate_cone(int64_t nv, const float* xyz, const float* w, const float* vel, const float* scal,
                         int64_t nt, const int32_t* tv, const int32_t* tn, const float cone[6],
                         const float origin[3], const int32_t dims[3], const float* dens, float* out_density,
                         float* out_velocity, float* out_gradient, float* out_scalar, float* out_scalar_gradient,
                         double* seconds) {
  DT dt;
  const std::vector<DT::Vertex*>& verts = dt.load_flat(nv, xyz, nt, tv, tn);
  for (int64_t i = 0; i < nv; ++i) {
    vertexData& d = verts[i]->info();
    d.weight() = w[i];
    for (int c = 0; c < 3; ++c) d.velocity(c) = vel ? vel[3 * i + c] : 0.f;
    d.scalar(0) = scal ? scal[i] : 0.f;
    d.setDensity(dens[i]);
  }
  User_options opt;
  opt.redshiftConeOn = true;
  opt.redshiftCone.coords.assign(cone, cone + 6);
  opt.originPosition.assign(origin, origin + 3);
  opt.gridSize.assign({(size_t)dims[0], (size_t)dims[1], (size_t)dims[2]});
  Quantities q;
  Field f;
  f.density = out_density != nullptr;
  f.velocity = out_velocity != nullptr;
  f.velocity_gradient = out_gradient != nullptr;
  f.scalar = out_scalar != nullptr;
  f.scalar_gradient = out_scalar_gradient != nullptr;
  opt.uField = f;
  const auto t0 = std::chrono::steady_clock::now();
  interpolateRedshiftCone(dt, opt, &q);
  if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  const size_t m = (size_t)dims[0] * dims[1] * dims[2];
  if (out_density && q.density.size() == m) std::memcpy(out_density, q.density.data(), m * sizeof(float));
  if (out_velocity && q.velocity.size() == m) std::memcpy(out_velocity, q.velocity.data(), 3 * m * sizeof(float));
  if (out_gradient && q.velocity_gradient.size() == m)
    std::memcpy(out_gradient, q.velocity_gradient.data(), 9 * m * sizeof(float));
  if (out_scalar && q.scalar.size() == m) std::memcpy(out_scalar, q.scalar.data(), m * sizeof(float));
  if (out_scalar_gradient && q.scalar_gradient.size() == m)
    std::memcpy(out_scalar_gradient, q.scalar_gradient.data(), 3 * m * sizeof(float));
  return 0;
}

// The reference's Monte-Carlo averages at user points (which 0: samples xyz
// with cell sizes delta, n of them; region = the kept box) or on a redshift
// cone (which 1: cone, origin, dims), noPoints = NN, randomSeed = seed, on one
// tessellation with LOCAL indices and the given vertex densities.  Outputs
// as ref_interpolate_points / ref_interpolate_cone; *n_out = rows written.
int ref_average_samples(int which, int64_t nv, const float* xyz, const float* w, const float* vel,
                        const float* scal, int64_t nt, const int32_t* tv, const int32_t* tn, const float region[6],
                        int64_t n, const float* pts, const float* delta, const float cone[6], const float origin[3],
                        const int32_t dims[3], int NN, uint64_t seed, const float* dens, float* out_density,
                        float* out_velocity, float* out_gradient, float* out_scalar, float* out_scalar_gradient,
                        int64_t* n_out) {
  DT dt;
  const std::vector<DT::Vertex*>& verts = dt.load_flat(nv, xyz, nt, tv, tn);
  for (int64_t i = 0; i < nv; ++i) {
    vertexData& d = verts[i]->info();
    d.weight() = w[i];
    for (int c = 0; c < 3; ++c) d.velocity(c) = vel ? vel[3 * i + c] : 0.f;
    d.scalar(0) = scal ? scal[i] : 0.f;
    d.setDensity(dens[i]);
  }
  User_options opt;
  opt.noPoints = NN;
  opt.randomSeed = (size_t)seed;
  Field f;
  f.density = out_density != nullptr;
  f.velocity = out_velocity != nullptr;
  f.velocity_gradient = out_gradient != nullptr;
  f.scalar = out_scalar != nullptr;
  f.scalar_gradient = out_scalar_gradient != nullptr;
  opt.aField = f;
  Quantities q;
  if (which == 0) {
    opt.region.coords.assign(region, region + 6);
    opt.userDefinedSampling = true;
    std::vector<Sample_point> samples((size_t)n);
    for (int64_t i = 0; i < n; ++i) {
      float p[3] = {pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]};
      float dl[3] = {delta[3 * i], delta[3 * i + 1], delta[3 * i + 2]};
      samples[i].setPosition(p);
      samples[i].setDelta(dl);
    }
    interpolateUserSampling_averaged_2(dt, samples, opt, &q);
  } else {
    opt.redshiftConeOn = true;
    opt.redshiftCone.coords.assign(cone, cone + 6);
    opt.originPosition.assign(origin, origin + 3);
    opt.gridSize.assign({(size_t)dims[0], (size_t)dims[1], (size_t)dims[2]});
    interpolateRedshiftCone_averaged_2(dt, opt, &q);
  }
  const size_t m = f.density ? q.density.size() : (f.velocity ? q.velocity.size() : q.velocity_gradient.size());
  *n_out = (int64_t)m;
  if (out_density && q.density.size() == m) std::memcpy(out_density, q.density.data(), m * sizeof(float));
  if (out_velocity && q.velocity.size() == m) std::memcpy(out_velocity, q.velocity.data(), 3 * m * sizeof(float));
  if (out_gradient && q.velocity_gradient.size() == m)
    std::memcpy(out_gradient, q.velocity_gradient.data(), 9 * m * sizeof(float));
  if (out_scalar && q.scalar.size() == m) std::memcpy(out_scalar, q.scalar.data(), m * sizeof(float));
  if (out_scalar_gradient && q.scalar_gradient.size() == m)
    std::memcpy(out_scalar_gradient, q.scalar_gradient.data(), 3 * m * sizeof(float));
  return 0;
}

int ref_interpolate(int64_t nv, const float* xyz, const float* w, const float* vel, const float* scal,
                    int64_t nt, const int32_t* tv, const int32_t* tn, const float region[6],
                    const int32_t grid[3], int which, int n_points, uint64_t seed, double rho_bar,
                    const float* dens_override, float* out_vdens, float* out_density, float* out_velocity,
                    float* out_gradient, float* out_scalar, float* out_scalar_gradient, float* out_std) {
  return ref_interpolate_timed(nv, xyz, w, vel, scal, nt, tv, tn, region, grid, which, n_points, seed, rho_bar,
                               dens_override, out_vdens, out_density, out_velocity, out_gradient, out_scalar,
                               out_scalar_gradient, out_std, 0u, nullptr);
}

}  // extern "C"
