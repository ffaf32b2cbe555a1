// Test driver of the DTFE() drop-in (dtfe_b200/shim) — TEST INFRASTRUCTURE
// ONLY.  Builds the reference's own types (Particle_data, User_options with
// the harness's default constructor, Quantities) from flat arrays, calls
// DTFE() exactly as a reference caller would (src/DTFE.h:36-40), and copies
// the Quantities vectors back out, so the Python tests can drive the drop-in.

#include <omp.h>

#include <cstdint>
#include <algorithm>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "define.h"
#include "particle_data.h"
#include "quantities.h"
#include "user_options.h"

void DTFE(std::vector<Particle_data>* allParticles, std::vector<Sample_point>& samples, User_options& userOptions,
          Quantities* uQuantities, Quantities* aQuantities);

namespace {
std::string g_error;

// No progress messages, and no padding test (a -DTEST_PADDING diagnostic;
// the reference's own constructor switches it on and updateEntries then
// refuses to run without that macro, src/user_options.cc:1050-1053).
void quiet(User_options& o) {
  o.verboseLevel = 0;
  o.testPaddedBoundaries = false;
}

void set_fields(Field& f, uint32_t m) {
  f.density = m & 1u;
  f.velocity = m & 2u;
  f.velocity_gradient = m & 4u;
  f.velocity_divergence = m & 8u;
  f.velocity_shear = m & 16u;
  f.velocity_vorticity = m & 32u;
  f.velocity_std = m & 64u;
  f.scalar = m & 128u;
  f.scalar_gradient = m & 256u;
}

template <class V>
void copy_out(const V& v, float* out, size_t G, size_t comps) {
  if (out && v.size() == G) std::memcpy(out, v.data(), sizeof(float) * comps * G);
}

void copy_all(const Quantities& q, float* const* out, size_t G) {
  if (!out) return;
  copy_out(q.density, out[0], G, 1);
  copy_out(q.velocity, out[1], G, 3);
  copy_out(q.velocity_gradient, out[2], G, 9);
  copy_out(q.velocity_divergence, out[3], G, 1);
  copy_out(q.velocity_shear, out[4], G, 5);
  copy_out(q.velocity_vorticity, out[5], G, 3);
  copy_out(q.velocity_std, out[6], G, 1);
  copy_out(q.scalar, out[7], G, noScalarComp);
  copy_out(q.scalar_gradient, out[8], G, 3 * noScalarComp);
}

// Options of DTFE() that change its planning (User_options members): region
// (fractions of the box unless region_mpc), partition with part_no (-1: every
// chunk), padding_mode 0 (padding_particles), 1 (padding[6] in box lengths,
// --padding l1..l6) or 2 (--paddingMpc).
struct DriverOptions {
  int32_t region_on, region_mpc;
  float region[6];
  int32_t partition_on;
  int32_t partition[3];
  int32_t part_no;
  int32_t padding_mode;
  float padding_particles;
  float padding[6];
};

size_t rows_of(const Quantities& q) {
  if (!q.density.empty()) return q.density.size();
  if (!q.velocity.empty()) return q.velocity.size();
  if (!q.velocity_gradient.empty()) return q.velocity_gradient.size();
  if (!q.velocity_divergence.empty()) return q.velocity_divergence.size();
  if (!q.scalar.empty()) return q.scalar.size();
  return 0;
}

int run_impl(int estimator, const float* pos, const float* w, const float* vel, const float* scal, int64_t n,
             const float box[6], int periodic, const int32_t grid[3], double average_density, uint32_t u_fields,
             uint32_t a_fields, int method, int n_points, uint64_t seed, int sph_neighbors, int n_threads,
             float* const* u_out, float* const* a_out, double* avg_out, int64_t* particles_left,
             const DriverOptions* x, int64_t cap_rows, int64_t* rows_out, float* region_out) {
  std::vector<Particle_data> p(n);
  for (int64_t i = 0; i < n; ++i) {
    for (int c = 0; c < 3; ++c) p[i].pos[c] = pos[3 * i + c];
    p[i].weight() = w ? w[i] : 1.f;
    for (int c = 0; c < 3; ++c) p[i].velocity(c) = vel ? vel[3 * i + c] : 0.f;
    p[i].scalar(0) = scal ? scal[i] : 0.f;
  }
  User_options o;
  quiet(o);
  o.gridSize.assign(grid, grid + 3);
  o.boxCoordinates.coords.assign(box, box + 6);
  o.periodic = periodic != 0;
  o.averageDensity = (Real)average_density;
  o.DTFE = estimator == 0;
  o.NGP = estimator == 1;
  o.CIC = estimator == 2;
  o.TSC = estimator == 3;
  o.SPH = estimator == 4;
  o.SPH_neighbors = sph_neighbors;
  o.method = method;
  o.noPoints = n_points;
  o.randomSeed = (size_t)seed;
  set_fields(o.uField, u_fields);
  set_fields(o.aField, a_fields);
  if (x) {
    if (x->region_on) {
      o.regionOn = true;
      o.regionMpcOn = x->region_mpc != 0;
      o.region.coords.assign(x->region, x->region + 6);
    }
    if (x->partition_on) {
      o.partitionOn = true;
      o.partition.assign(x->partition, x->partition + 3);
      o.partNo = x->part_no;
    }
    o.paddingParticles = x->padding_particles;
    if (x->padding_mode != 0) {
      o.paddingOn = true;
      o.paddingMpcOn = x->padding_mode == 2;
      o.paddingLength.coords.assign(x->padding, x->padding + 6);
    }
  }
  if (n_threads > 0) omp_set_num_threads(n_threads);
  std::vector<Sample_point> samples;
  Quantities uq, aq;
  try {
    DTFE(&p, samples, o, &uq, &aq);
  } catch (const std::exception& e) {
    g_error = e.what();
    return 1;
  }
  size_t rows = (size_t)grid[0] * grid[1] * grid[2];
  if (x) {
    rows = std::max(rows_of(uq), rows_of(aq));
    if ((int64_t)rows > cap_rows) {
      g_error = "driver: more result rows than the output buffers hold";
      return 2;
    }
    if (rows_out) *rows_out = (int64_t)rows;
    if (region_out)
      for (int i = 0; i < 6; ++i) region_out[i] = o.region.coords.size() == 6 ? o.region.coords[i] : 0.f;
  }
  copy_all(uq, u_out, rows);
  copy_all(aq, a_out, rows);
  if (avg_out) *avg_out = (double)o.averageDensity;
  if (particles_left) *particles_left = (int64_t)p.size();
  return 0;
}

}  // namespace

extern "C" {

const char* dropin_error() { return g_error.c_str(); }

// estimator: 0 DTFE, 1 NGP, 2 CIC, 3 TSC, 4 SPH.  u_fields / a_fields: bit
// i = field slot i (density, velocity, gradient, divergence, shear,
// vorticity, std, scalar, scalar gradient).  average_density < 0: automatic;
// the value used comes back in *avg_out.  Returns 0, or 1 with
// dropin_error() set when DTFE() threw.
int dropin_run(int estimator, const float* pos, const float* w, const float* vel, const float* scal, int64_t n,
               const float box[6], int periodic, const int32_t grid[3], double average_density, uint32_t u_fields,
               uint32_t a_fields, int method, int n_points, uint64_t seed, int sph_neighbors, int n_threads,
               float* const* u_out, float* const* a_out, double* avg_out, int64_t* particles_left) {
  return run_impl(estimator, pos, w, vel, scal, n, box, periodic, grid, average_density, u_fields, a_fields, method,
                  n_points, seed, sph_neighbors, n_threads, u_out, a_out, avg_out, particles_left, nullptr, 0,
                  nullptr, nullptr);
}

// dropin_run with the options of DriverOptions: the results hold *rows_out
// rows (at most cap_rows; the chunk's cells with partNo), region_out
// receives userOptions.region after the call.
int dropin_run_ex(int estimator, const float* pos, const float* w, const float* vel, const float* scal, int64_t n,
                  const float box[6], int periodic, const int32_t grid[3], double average_density, uint32_t u_fields,
                  uint32_t a_fields, int method, int n_points, uint64_t seed, int sph_neighbors, int n_threads,
                  float* const* u_out, float* const* a_out, const DriverOptions* x, int64_t cap_rows,
                  int64_t* rows_out, float* region_out) {
  if (!x) return 3;
  return run_impl(estimator, pos, w, vel, scal, n, box, periodic, grid, average_density, u_fields, a_fields, method,
                  n_points, seed, sph_neighbors, n_threads, u_out, a_out, nullptr, nullptr, x, cap_rows, rows_out,
                  region_out);
}

// DTFE() with user sampling points (n_samples, xyz 3 each, cell sizes sdelta
// 3 each or NULL) for the fields u_fields / a_fields: *n_kept rows (the
// samples inside the box) land in u_out / a_out.  n_points >= 0 sets
// noPoints (noPointsOn), seed randomSeed.
int dropin_run_points(const float* pos, const float* w, const float* vel, const float* scal, int64_t n,
                      const float box[6], int periodic, const int32_t grid[3], double average_density,
                      uint32_t u_fields, int64_t n_samples, const float* sxyz, int n_threads, float* const* u_out,
                      int64_t* n_kept, uint32_t a_fields, const float* sdelta, int n_points, uint64_t seed,
                      float* const* a_out) {
  std::vector<Particle_data> p(n);
  for (int64_t i = 0; i < n; ++i) {
    for (int c = 0; c < 3; ++c) p[i].pos[c] = pos[3 * i + c];
    p[i].weight() = w ? w[i] : 1.f;
    for (int c = 0; c < 3; ++c) p[i].velocity(c) = vel ? vel[3 * i + c] : 0.f;
    p[i].scalar(0) = scal ? scal[i] : 0.f;
  }
  User_options o;
  quiet(o);
  o.gridSize.assign(grid, grid + 3);
  o.boxCoordinates.coords.assign(box, box + 6);
  o.periodic = periodic != 0;
  o.averageDensity = (Real)average_density;
  o.userDefinedSampling = true;
  set_fields(o.uField, u_fields);
  set_fields(o.aField, a_fields);
  if (n_points >= 0) {
    o.noPoints = n_points;
    o.noPointsOn = true;
  }
  o.randomSeed = (size_t)seed;
  if (n_threads > 0) omp_set_num_threads(n_threads);
  std::vector<Sample_point> samples((size_t)n_samples);
  for (int64_t i = 0; i < n_samples; ++i) {
    float q[3] = {sxyz[3 * i], sxyz[3 * i + 1], sxyz[3 * i + 2]};
    samples[i].setPosition(q);
    if (sdelta) {
      float d[3] = {sdelta[3 * i], sdelta[3 * i + 1], sdelta[3 * i + 2]};
      samples[i].setDelta(d);
    }
  }
  Quantities uq, aq;
  try {
    DTFE(&p, samples, o, &uq, &aq);
  } catch (const std::exception& e) {
    g_error = e.what();
    return 1;
  }
  size_t m = uq.density.size() ? uq.density.size() : uq.velocity.size();
  if (!u_fields) m = aq.density.size() ? aq.density.size() : aq.velocity.size();
  *n_kept = (int64_t)m;
  copy_all(uq, u_out, m);
  copy_all(aq, a_out, m);
  return 0;
}

// DTFE() on a redshift-cone grid: cone = (r_min, r_max, theta_min,
// theta_max, psi_min, psi_max), origin = the apex, grid = bins in r, theta,
// psi; u_out / a_out receive grid[0] grid[1] grid[2] rows.
int dropin_run_cone(const float* pos, const float* w, const float* vel, const float* scal, int64_t n,
                    const float box[6], int periodic, const int32_t grid[3], double average_density,
                    uint32_t u_fields, const float cone[6], const float origin[3], int n_threads,
                    float* const* u_out, uint32_t a_fields, int n_points, uint64_t seed, float* const* a_out) {
  std::vector<Particle_data> p(n);
  for (int64_t i = 0; i < n; ++i) {
    for (int c = 0; c < 3; ++c) p[i].pos[c] = pos[3 * i + c];
    p[i].weight() = w ? w[i] : 1.f;
    for (int c = 0; c < 3; ++c) p[i].velocity(c) = vel ? vel[3 * i + c] : 0.f;
    p[i].scalar(0) = scal ? scal[i] : 0.f;
  }
  User_options o;
  quiet(o);
  o.gridSize.assign(grid, grid + 3);
  o.boxCoordinates.coords.assign(box, box + 6);
  o.periodic = periodic != 0;
  o.averageDensity = (Real)average_density;
  o.redshiftConeOn = true;
  o.redshiftCone.coords.assign(cone, cone + 6);
  o.originPosition.assign(origin, origin + 3);
  set_fields(o.uField, u_fields);
  set_fields(o.aField, a_fields);
  if (n_points >= 0) {
    o.noPoints = n_points;
    o.noPointsOn = true;
  }
  o.randomSeed = (size_t)seed;
  if (n_threads > 0) omp_set_num_threads(n_threads);
  std::vector<Sample_point> samples;
  Quantities uq, aq;
  try {
    DTFE(&p, samples, o, &uq, &aq);
  } catch (const std::exception& e) {
    g_error = e.what();
    return 1;
  }
  copy_all(uq, u_out, (size_t)grid[0] * grid[1] * grid[2]);
  copy_all(aq, a_out, (size_t)grid[0] * grid[1] * grid[2]);
  return 0;
}

}  // extern "C"
