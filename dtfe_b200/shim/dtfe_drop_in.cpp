// Drop-in replacement for the reference library's entry point
//
//   void DTFE(std::vector<Particle_data>* allParticles, std::vector<Sample_point>& samples,
//             User_options& userOptions, Quantities* uQuantities, Quantities* aQuantities);
//
// (src/DTFE.h:36-40, src/DTFE.cpp:76-251).  It is compiled against the
// caller's own reference headers (define.h, particle_data.h, user_options.h,
// quantities.h and what they include), so the types are the caller's, and
// it replaces src/DTFE.cpp in the caller's link.  The control flow of DTFE()
// and DTFE_parallel() (average density, padding, periodic images, the
// parallelGrid(omp_get_max_threads()) sub-box split, tessellation) runs on the
// host through dtfe_plan_build (include/dtfe_host.h); vertex densities,
// interpolation, the averaged methods, the velocity derivatives and the
// NGP/CIC/TSC/SPH estimators run on the GPU through include/dtfe_gpu.h, and
// the results are written straight into the caller's Quantities vectors
// (cells x components, x slowest: the layout Quantities uses).
//
// As the reference: allParticles is cleared, userOptions.averageDensity is
// set when it was negative (automatic), uQuantities receives the fields of
// userOptions.uField (cell centres), aQuantities those of
// userOptions.aField (method 1, 2 or 3 averages, or the NGP/CIC/TSC/SPH grids;
// method 1 computes no velocity standard deviation, as the reference).
// User sampling points (the samples vector) give uQuantities at the samples
// inside the box, in order (interpolateUserSampling); a redshift cone
// (redshiftConeOn) gives them on its gridSize bins (interpolateRedshiftCone).
// Volume averages there are Monte-Carlo averages, as the reference forces
// (method 2, 20 points unless noPointsOn; Philox offsets instead of mt19937).
// --region, --partition / --partNo and given padding lengths (--padding
// l1..l6, --paddingMpc) plan as the reference's DTFE() does; the chunks of
// --partition run in one batched GPU step instead of one after another, and
// --partNo returns the chunk's grid only, as the reference.
// Unlike the reference, failures throw std::runtime_error instead of calling
// exit(), and options this path does not cover throw as well: random
// subsamples, Poisson particles, scalar fields with NGP/CIC/TSC,
// NGP/CIC/TSC/SPH at user points or on cones.  The GPU is device 0 unless
// DTFE_GPU_DEVICE names another.

#include <omp.h>

#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "define.h"
#include "particle_data.h"
#include "quantities.h"
#include "user_options.h"

#include "dtfe_gpu.h"
#include "dtfe_host.h"

#if NO_DIM != 3
#error "the GPU path is three-dimensional"
#endif

namespace {

void check(int rc, const char* what) {
  if (rc != DTFE_OK) {
    const char* msg = dtfe_last_error();
    throw std::runtime_error(std::string("DTFE (GPU): ") + what + ": " + (msg ? msg : "error"));
  }
}

void unsupported(bool cond, const char* what) {
  if (cond) throw std::runtime_error(std::string("DTFE (GPU): not supported: ") + what);
}

struct PlanGuard {
  dtfe_plan p = nullptr;
  ~PlanGuard() { dtfe_plan_release(p); }
};

struct HandleGuard {
  dtfe_handle h = nullptr;
  ~HandleGuard() { dtfe_gpu_destroy(h); }
};

template <class V>
float* sized(V& vec, size_t G) {
  vec.resize(G);
  return reinterpret_cast<float*>(vec.data());
}

// Output pointers for the selected fields of one Quantities object.
void outputs(const Field& f, Quantities* q, size_t G, float* out[DTFE_NUM_FIELDS], uint32_t* mask) {
  for (int s = 0; s < DTFE_NUM_FIELDS; ++s) out[s] = nullptr;
  *mask = 0;
  auto set = [&](bool on, int slot, float* p) {
    if (!on) return;
    out[slot] = p;
    *mask |= DTFE_FIELD_BIT(slot);
  };
  set(f.density, DTFE_DENSITY, f.density ? sized(q->density, G) : nullptr);
  set(f.velocity, DTFE_VELOCITY, f.velocity ? sized(q->velocity, G) : nullptr);
  set(f.velocity_gradient, DTFE_VELOCITY_GRADIENT, f.velocity_gradient ? sized(q->velocity_gradient, G) : nullptr);
  set(f.velocity_divergence, DTFE_VELOCITY_DIVERGENCE,
      f.velocity_divergence ? sized(q->velocity_divergence, G) : nullptr);
  set(f.velocity_shear, DTFE_VELOCITY_SHEAR, f.velocity_shear ? sized(q->velocity_shear, G) : nullptr);
  set(f.velocity_vorticity, DTFE_VELOCITY_VORTICITY, f.velocity_vorticity ? sized(q->velocity_vorticity, G) : nullptr);
  set(f.velocity_std, DTFE_VELOCITY_STD, f.velocity_std ? sized(q->velocity_std, G) : nullptr);
  set(f.scalar, DTFE_SCALAR, f.scalar ? sized(q->scalar, G) : nullptr);
  set(f.scalar_gradient, DTFE_SCALAR_GRADIENT, f.scalar_gradient ? sized(q->scalar_gradient, G) : nullptr);
}

// Keeps the first n rows of every selected field (the user samples inside
// the region).
void resize_all(const Field& f, Quantities* q, size_t n) {
  if (f.density) q->density.resize(n);
  if (f.velocity) q->velocity.resize(n);
  if (f.velocity_gradient) q->velocity_gradient.resize(n);
  if (f.velocity_divergence) q->velocity_divergence.resize(n);
  if (f.velocity_shear) q->velocity_shear.resize(n);
  if (f.velocity_vorticity) q->velocity_vorticity.resize(n);
  if (f.scalar) q->scalar.resize(n);
  if (f.scalar_gradient) q->scalar_gradient.resize(n);
}

bool any(const Field& f) {
  return f.density || f.velocity || f.velocity_gradient || f.velocity_divergence || f.velocity_shear ||
         f.velocity_vorticity || f.velocity_std || f.scalar || f.scalar_gradient;
}

}  // namespace

void DTFE(std::vector<Particle_data>* allParticles, std::vector<Sample_point>& samples, User_options& userOptions,
          Quantities* uQuantities, Quantities* aQuantities) {
  User_options& o = userOptions;
  const bool user_points = !samples.empty() || o.userDefinedSampling;
  const bool cone = o.redshiftConeOn && !user_points;  // user samples switch the cone off (user_options.cc:962-964)
  unsupported((user_points || cone) && (o.NGP || o.CIC || o.TSC || o.SPH),
              "NGP/CIC/TSC/SPH at user-defined sampling points or on redshift-cone grids");
  // volume averages there are Monte-Carlo averages (User_options::updateEntries,
  // src/user_options.cc:962-983; DTFE() writes the choice back)
  if ((user_points || cone) && any(o.aField) && o.method != 2) {
    o.method = 2;
    if (!o.noPointsOn) o.noPoints = 20;
  }
  unsupported(cone && (o.redshiftCone.coords.size() != 6 || o.originPosition.size() != 3),
              "redshift cones without 6 limits and a 3-D origin");
  unsupported(o.randomSample >= Real(0.), "random subsamples");
  unsupported(o.poisson != 0, "Poisson particles");
  unsupported(o.gridSize.size() != 3, "grids other than 3-D regular grids");
  unsupported(o.boxCoordinates.coords.size() != 6, "a box without 6 coordinates");
  unsupported(o.regionOn && o.region.coords.size() != 6, "--region without 6 coordinates");
  unsupported(o.partitionOn && o.partition.size() != 3, "--partition without 3 chunk counts");
  unsupported(!o.paddingLength.coords.empty() && o.paddingLength.coords.size() != 6,
              "padding lengths other than 6 values");
  // --partition is not available at user points or on cones
  // (User_options::updateEntries, src/user_options.cc:986-995)
  if (o.partitionOn && (user_points || cone)) {
    o.partitionOn = false;
    for (size_t i = 0; i < o.partition.size(); ++i) o.partition[i] = 1;
    o.partNo = -1;
  }
  const bool dtfe = !(o.NGP || o.CIC || o.TSC || o.SPH);
  unsupported(dtfe && any(o.aField) && (o.method < 1 || o.method > 3), "averaging methods other than 1, 2, 3");
  unsupported(!dtfe && !o.SPH && (o.aField.scalar || o.aField.scalar_gradient), "scalar fields with NGP/CIC/TSC");

  const int64_t n = (int64_t)allParticles->size();
  std::vector<float> pos(3 * n), w(n), vel(3 * n), sc((size_t)noScalarComp * n);
  for (int64_t i = 0; i < n; ++i) {
    Particle_data& p = (*allParticles)[i];
    for (int c = 0; c < 3; ++c) pos[3 * i + c] = p.pos[c];
    w[i] = p.weight();
#ifdef VELOCITY
    for (int c = 0; c < 3; ++c) vel[3 * i + c] = p.velocity(c);
#endif
#ifdef SCALAR
    for (size_t c = 0; c < noScalarComp; ++c) sc[noScalarComp * i + c] = p.scalar(c);
#endif
  }
  allParticles->clear();  // the reference's contract (src/DTFE.cpp:75)
#ifdef VELOCITY
  const float* velp = vel.data();
#else
  const float* velp = nullptr;
#endif
#ifdef SCALAR
  const float* scp = sc.data();
  const int32_t S = (int32_t)noScalarComp;
#else
  const float* scp = nullptr;
  const int32_t S = 0;
#endif

  float box[6];
  for (int i = 0; i < 6; ++i) box[i] = o.boxCoordinates.coords[i];
  const int32_t main_grid[3] = {(int32_t)o.gridSize[0], (int32_t)o.gridSize[1], (int32_t)o.gridSize[2]};
  if (o.averageDensity < Real(0.)) o.averageDensity = dtfe_average_density(w.data(), n);
  const int kind = dtfe || o.SPH ? DTFE_PLAN_DTFE : (o.NGP ? DTFE_PLAN_NGP : (o.CIC ? DTFE_PLAN_CIC : DTFE_PLAN_TSC));

  // the planning options, as User_options::updateEntries / updatePadding
  // read them (src/user_options.cc:926-1089), box fractions converted with
  // the reference's own [i % 2] indexing of the box offset and length
  dtfe_plan_options po;
  std::memset(&po, 0, sizeof(po));
  po.n_parts = user_points || cone ? 1 : omp_get_max_threads();  // no split (src/DTFE.cpp:301)
  po.padding_particles = (float)o.paddingParticles;
  po.padding_mode = DTFE_PAD_PARTICLES;
  if (o.paddingLength.coords.size() == 6) {
    po.padding_mode = o.paddingOn && !o.paddingMpcOn ? DTFE_PAD_RELATIVE : DTFE_PAD_ABSOLUTE;
    for (int i = 0; i < 6; ++i) po.padding[i] = o.paddingLength.coords[i];
  }
  const float off[3] = {box[0], box[2], box[4]}, len[3] = {box[1] - box[0], box[3] - box[2], box[5] - box[4]};
  if (o.regionOn) {
    po.region_on = 1;
    for (int i = 0; i < 6; ++i)
      po.region[i] = o.regionMpcOn ? (float)o.region.coords[i] : off[i % 2] + (float)o.region.coords[i] * len[i % 2];
  }
  if (o.partitionOn) {
    po.partition_on = 1;
    for (int a = 0; a < 3; ++a) po.partition[a] = (int32_t)o.partition[a];
    po.part_no = o.partNo;
  } else {
    po.part_no = -1;
  }
  po.average_density = (double)o.averageDensity;

  PlanGuard plan;
  const int prc = dtfe_plan_build_ex(kind, pos.data(), w.data(), velp, scp, S, n, box, o.periodic ? 1 : 0, main_grid,
                                     &po, &plan.p);
  if (prc == 4)
    throw std::runtime_error("DTFE (GPU): the region is not a valid sub-box of the data box (Box::validSubBox)");
  if (prc) throw std::runtime_error("DTFE (GPU): planning failed (status " + std::to_string(prc) + ")");
  dtfe_plan_view v;
  check(dtfe_plan_get(plan.p, &v), "plan view");
  // what updateEntries and DTFE() leave in userOptions: the padding as
  // absolute lengths, the region in absolute coordinates (the box without
  // --region; the chunk with --partNo, src/DTFE.cpp:151)
  o.paddingLength.coords.assign(v.padding, v.padding + 6);
  o.paddingOn = o.paddingMpcOn = true;
  o.region.coords.assign(v.region, v.region + 6);
  if (o.regionOn) o.regionMpcOn = true;
  // the grid the results cover: the chunk's own with --partNo
  const int32_t grid[3] = {v.grid[0], v.grid[1], v.grid[2]};
  const size_t G = (size_t)grid[0] * grid[1] * grid[2];

  dtfe_config cfg = {0, dtfe || o.SPH ? S : 0, 0, 0};
  if (const char* d = std::getenv("DTFE_GPU_DEVICE")) cfg.device = std::atoi(d);
  HandleGuard gpu;
  check(dtfe_gpu_create(&cfg, &gpu.h), "create");

  if (kind != DTFE_PLAN_DTFE) {
    const int32_t k = kind == DTFE_PLAN_NGP ? DTFE_DEPOSIT_NGP : (kind == DTFE_PLAN_CIC ? DTFE_DEPOSIT_CIC : DTFE_DEPOSIT_TSC);
    float* dens = o.aField.density ? sized(aQuantities->density, G) : nullptr;
    float* velo = o.aField.velocity ? sized(aQuantities->velocity, G) : nullptr;
    check(dtfe_gpu_deposit(gpu.h, k, v.dep_pos, v.dep_weight, velo ? v.dep_velocity : nullptr, v.n_particles,
                           v.n_dep_boxes, v.dep_boxes, grid, v.rho_bar, dens ? dens : sized(aQuantities->density, G),
                           velo),
          "deposit");
    if (!o.aField.density) aQuantities->density.clear();
    return;
  }

  check(dtfe_gpu_upload(gpu.h, v.tet_v, v.tet_n, v.n_tets, v.xyz, v.weight, v.velocity, v.scalar, v.n_verts),
        "upload");
  check(dtfe_gpu_set_subboxes(gpu.h, v.n_boxes, v.boxes, v.xs, v.n_xs, v.ys, v.n_ys, v.zs, v.n_zs, grid),
        "sub-boxes");
  if (v.regions) check(dtfe_gpu_set_regions(gpu.h, v.n_boxes, v.regions), "sub-box regions");
  if (o.SPH) {
    const bool wv = o.aField.velocity, ws = o.aField.scalar;
    uint32_t f = DTFE_FIELD_BIT(DTFE_DENSITY) | (wv ? DTFE_FIELD_BIT(DTFE_VELOCITY) : 0u) |
                 (ws ? DTFE_FIELD_BIT(DTFE_SCALAR) : 0u);
    check(dtfe_gpu_sph(gpu.h, o.SPH_neighbors, f, o.extensive ? 1 : 0, v.rho_bar, sized(aQuantities->density, G),
                       wv ? sized(aQuantities->velocity, G) : nullptr, ws ? sized(aQuantities->scalar, G) : nullptr),
          "SPH");
    if (!o.aField.density) aQuantities->density.clear();
    return;
  }
  check(dtfe_gpu_vertex_density(gpu.h, v.rho_bar), "vertex density");
  dtfe_status st;
  if (any(o.uField) && user_points) {
    // interpolateUserSampling: the samples inside the region (the box), in order
    const size_t m = samples.size();
    std::vector<float> pts(3 * m);
    for (size_t i = 0; i < m; ++i)
      for (int c = 0; c < 3; ++c) pts[3 * i + c] = samples[i].position(c);
    float* out[DTFE_NUM_FIELDS];
    dtfe_interp_opts io = {DTFE_METHOD_CENTRE, 1, 0, 0, 0};
    outputs(o.uField, uQuantities, m, out, &io.fields);
    int64_t kept = 0;
    check(dtfe_gpu_interpolate_points(gpu.h, (int64_t)m, pts.data(), v.region, &io, out, &kept),
          "interpolation at user sampling points");
    resize_all(o.uField, uQuantities, (size_t)kept);
  } else if (any(o.uField) && cone) {
    // interpolateRedshiftCone: gridSize bins in (r, theta, psi)
    float* out[DTFE_NUM_FIELDS];
    dtfe_interp_opts io = {DTFE_METHOD_CENTRE, 1, 0, 0, 0};
    outputs(o.uField, uQuantities, G, out, &io.fields);
    float lim[6], org[3];
    for (int i = 0; i < 6; ++i) lim[i] = o.redshiftCone.coords[i];
    for (int i = 0; i < 3; ++i) org[i] = o.originPosition[i];
    check(dtfe_gpu_interpolate_cone(gpu.h, lim, org, grid, &io, out), "redshift-cone interpolation");
  } else if (any(o.uField)) {
    float* out[DTFE_NUM_FIELDS];
    dtfe_interp_opts io = {DTFE_METHOD_CENTRE, 1, 0, 0, 0};
    outputs(o.uField, uQuantities, G, out, &io.fields);
    check(dtfe_gpu_interpolate(gpu.h, &io, out, &st), "cell-centre interpolation");
  }
  if (any(o.aField) && (user_points || cone)) {
    // interpolateUserSampling_averaged_2 / interpolateRedshiftCone_averaged_2
    // (no velocity standard deviation there)
    Field f = o.aField;
    f.velocity_std = false;
    dtfe_interp_opts io = {DTFE_METHOD_MONTE_CARLO, (int32_t)o.noPoints, (uint64_t)o.randomSeed, 0, 0};
    float* out[DTFE_NUM_FIELDS];
    if (user_points) {
      const size_t m = samples.size();
      std::vector<float> pts(3 * m), dl(3 * m);
      for (size_t i = 0; i < m; ++i)
        for (int c = 0; c < 3; ++c) {
          pts[3 * i + c] = samples[i].position(c);
          dl[3 * i + c] = samples[i].delta(c);
        }
      outputs(f, aQuantities, m, out, &io.fields);
      int64_t kept = 0;
      check(dtfe_gpu_average_points(gpu.h, (int64_t)m, pts.data(), dl.data(), v.region, &io, out, &kept),
            "volume averages at user sampling points");
      resize_all(f, aQuantities, (size_t)kept);
    } else {
      outputs(f, aQuantities, G, out, &io.fields);
      float lim[6], org[3];
      for (int i = 0; i < 6; ++i) lim[i] = o.redshiftCone.coords[i];
      for (int i = 0; i < 3; ++i) org[i] = o.originPosition[i];
      check(dtfe_gpu_interpolate_cone(gpu.h, lim, org, grid, &io, out), "redshift-cone volume averages");
    }
  } else if (any(o.aField)) {
    float* out[DTFE_NUM_FIELDS];
    const int method = o.method == 1 ? DTFE_METHOD_TETRAHEDRA
                                     : (o.method == 2 ? DTFE_METHOD_MONTE_CARLO : DTFE_METHOD_EQUIDISTANT);
    dtfe_interp_opts io = {method, (int32_t)o.noPoints, (uint64_t)o.randomSeed, 0, 0};
    Field f = o.aField;
    // interpolateGrid_averaged_1 warns and leaves the standard deviation out
    // (averaged_interpolation_1.cc:234-238)
    if (method == DTFE_METHOD_TETRAHEDRA) f.velocity_std = false;
    outputs(f, aQuantities, G, out, &io.fields);
    check(dtfe_gpu_interpolate(gpu.h, &io, out, &st), "averaged interpolation");
  }
}
