// CPU oracle for the DTFE interpolation path — TEST INFRASTRUCTURE ONLY.
//
// Only tests, the smoke check and bench.py's CPU-baseline leg may load this
// library, and only as the checker or the timed CPU baseline; the product path
// never calls it.
//
// It restates, function by function, the reference algorithm
// (lrwesterhoek/DTFE, C++/CGAL/OpenMP) on the flat tessellation format:
//   vertexDensity            src/CGAL_triangulation/triangulation.cpp:200-279
//   matrixInverse, minorDeterminant
//                            src/CGAL_triangulation/triangulation_miscellaneous.cc:25,42-96
//   positionMatrix .. scalarGradient
//                            src/CGAL_triangulation/unaveraged_interpolation.cc:34-173
//   interpolateGrid          unaveraged_interpolation.cc:209-369
//   interpolateGrid_averaged_2 / _3
//                            src/CGAL_triangulation/averaged_interpolation_2.cc:35-233,664-866
//   standardDeviation        triangulation_miscellaneous.cc:256-271
//   velocityDivergence/Shear/Vorticity
//                            src/DTFE.cpp:394-433
// in two arithmetic modes:
//   mode 0 "ref":  the reference's precision pattern (double edge matrix and
//                  inverse rounded to float, float gradients and values,
//                  double products of the float offset) without FMA
//                  contraction; vertex-volume sums in FP64;
//   mode 1 "fp64": every quantity in double — the accuracy yardstick.
// Point location is a visibility walk with exact predicates followed by the
// canonical tie rule (the lowest-numbered tetrahedron whose closure holds the
// point), so it is independent of the walk path.
//
// Parity status: the reference cannot be built in this environment (CGAL,
// Boost and GSL are absent) and ships no tests or golden data; the
// restatement is pinned by the analytic known-answer tests in tests/ and by
// agreement with an independent tessellator (scipy Qhull).

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../include/dtfe_gpu.h"
#include "../dtfe_b200/csrc/philox.h"
#include "../dtfe_b200/csrc/fixed_volume.cuh"
#include "../dtfe_b200/csrc/predicates.h"
#include "../dtfe_b200/csrc/sobol.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct Tess {
  int64_t T, V;
  const int32_t* tv;
  const int32_t* tn;
  const float* xyz;
  const float* vel;
  const float* scal;
  int S;
  void P(int32_t v, double out[3]) const {
    for (int k = 0; k < 3; ++k) out[k] = (double)xyz[3 * (int64_t)v + k];
  }
};

// orientation of tetrahedron t with vertex i replaced by p
int face_orient(const Tess& g, int64_t t, int i, const double* p) {
  double q[4][3];
  for (int a = 0; a < 4; ++a) {
    if (a == i) { q[a][0] = p[0]; q[a][1] = p[1]; q[a][2] = p[2]; }
    else g.P(g.tv[4 * t + a], q[a]);
  }
  return dtfe::orient(q[0], q[1], q[2], q[3]);
}

bool contains(const Tess& g, int64_t t, const double* p, int zero[4]) {
  for (int i = 0; i < 4; ++i) {
    int o = face_orient(g, t, i, p);
    if (o < 0) return false;
    zero[i] = (o == 0);
  }
  return true;
}

// Canonical location: walk, then the lowest id among tetrahedra whose closure
// contains p.  Returns -1 when p is outside the hull (an infinite cell in the
// reference), -2 when the walk fails.
int64_t locate(const Tess& g, const double* p, int64_t start, int64_t lo, int64_t hi) {
  // no tetrahedra in the sub-box (fewer than four non-coplanar points): the
  // reference interpolates zeros (triangulation_miscellaneous.cc:121-138)
  if (hi <= lo) return -1;
  int64_t t = start;
  if (t < lo || t >= hi) t = lo;
  int64_t limit = 4 * (hi - lo) + 64;
  for (int64_t step = 0;; ++step) {
    if (step > limit) return -2;
    int moved = -1;
    for (int i = 0; i < 4; ++i) {
      if (face_orient(g, t, i, p) < 0) { moved = i; break; }
    }
    if (moved < 0) break;
    int64_t nb = g.tn[4 * t + moved];
    if (nb < 0) return -1;
    t = nb;
  }
  int zero[4];
  contains(g, t, p, zero);
  if (!zero[0] && !zero[1] && !zero[2] && !zero[3]) return t;
  // tie: explore the tetrahedra around the face/edge/vertex holding p
  std::vector<int64_t> seen{t}, queue{t};
  int64_t best = t;
  while (!queue.empty()) {
    int64_t u = queue.back();
    queue.pop_back();
    int zu[4];
    contains(g, u, p, zu);
    for (int i = 0; i < 4; ++i) {
      if (!zu[i]) continue;
      int64_t nb = g.tn[4 * u + i];
      if (nb < 0) continue;
      if (std::find(seen.begin(), seen.end(), nb) != seen.end()) continue;
      seen.push_back(nb);
      int zn[4];
      if (!contains(g, nb, p, zn)) continue;
      queue.push_back(nb);
      best = std::min(best, nb);
    }
  }
  return best;
}

// ---- the reference's per-cell arithmetic ---------------------------------

// minorDeterminant + matrixInverse (triangulation_miscellaneous.cc:42-96):
// double cofactors divided by det; zero when |det|/sum|m| <= 1e-6.
template <typename R>
void matrix_inverse(const double A[3][3], R out[3][3]) {
  auto minor = [&](int row, int col) {
    int i1 = (row + 1) % 3, i2 = (row + 2) % 3, j1 = (col + 1) % 3, j2 = (col + 2) % 3;
    return A[j1][i1] * A[j2][i2] - A[j1][i2] * A[j2][i1];
  };
  double det = A[0][0] * minor(0, 0) + A[0][1] * minor(1, 0) + A[0][2] * minor(2, 0);
  double tmp[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) tmp[r][c] = minor(r, c) / det;
  // accumulation order of the reference: left-to-right over the 9 entries
  double s = std::fabs(A[0][0]) + std::fabs(A[0][1]) + std::fabs(A[0][2]) + std::fabs(A[1][0]) +
      std::fabs(A[1][1]) + std::fabs(A[1][2]) + std::fabs(A[2][0]) + std::fabs(A[2][1]) +
      std::fabs(A[2][2]);
  bool ok = std::fabs(det / s) > 1.e-6;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) out[r][c] = ok ? (R)tmp[r][c] : (R)0;
}

struct CellEval {
  // results of one sample
  double dens, vel[3], grad[9], sc[DTFE_MAX_SCALARS], scg[3 * DTFE_MAX_SCALARS];
};

// Evaluates the fields of tetrahedron t at point p in the given mode.
// positionMatrix/relativeSamplePoint (unaveraged_interpolation.cc:34-59),
// densityGrad/densityValue (:66-87), velocityGrad/velocityValue (:94-120),
// velocityGradient (:123-130), scalarGrad/scalarValue/scalarGradient (:137-173).
void eval_cell(const Tess& g, const float* dens32, const double* dens64, int64_t t,
               const double* p, int mode, bool fix, bool want_vel, bool want_sc,
               CellEval& e) {
  const int32_t* v = &g.tv[4 * t];
  double X[4][3];
  for (int a = 0; a < 4; ++a) g.P(v[a], X[a]);
  double A[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) A[r][c] = X[r + 1][c] - X[0][c];
  if (mode == 0) {
    float M[3][3];
    matrix_inverse<float>(A, M);
    float rel[3];
    for (int c = 0; c < 3; ++c) rel[c] = (float)(p[c] - X[0][c]);
    // density
    float d0 = dens32[v[0]];
    float dd[3];
    for (int i = 0; i < 3; ++i) dd[i] = dens32[v[i + 1]] - d0;
    float gr[3];
    for (int i = 0; i < 3; ++i) {
      float acc = 0.f;
      for (int j = 0; j < 3; ++j) acc += M[i][j] * dd[j];
      gr[i] = acc;
    }
    double s = (double)rel[0] * gr[0] + (double)rel[1] * gr[1] + (double)rel[2] * gr[2];
    e.dens = (double)(d0 + (float)s);
    if (want_vel && g.vel) {
      float dv[3][3], VG[3][3];
      const float* v0 = &g.vel[3 * (int64_t)v[0]];
      for (int k = 0; k < 3; ++k)
        for (int j = 0; j < 3; ++j) dv[k][j] = g.vel[3 * (int64_t)v[k + 1] + j] - v0[j];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          float acc = 0.f;
          for (int k = 0; k < 3; ++k) acc += M[i][k] * dv[k][j];
          VG[i][j] = acc;
        }
      for (int i = 0; i < 3; ++i) {
        float tmp = 0.f;
        if (fix) {
          for (int j = 0; j < 3; ++j) tmp = (float)((double)tmp + (double)VG[j][i] * (double)rel[j]);
        } else {
          for (int j = 0; j < 3; ++j) tmp = (float)((double)VG[j][i] * (double)rel[j]);
        }
        e.vel[i] = (double)(tmp + v0[i]);
      }
      for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) e.grad[j * 3 + i] = (double)VG[i][j];
    }
    if (want_sc && g.scal && g.S > 0) {
      int S = g.S;
      const float* s0 = &g.scal[(int64_t)S * v[0]];
      for (int q = 0; q < S; ++q) {
        float ds[3], SG[3];
        for (int k = 0; k < 3; ++k) ds[k] = g.scal[(int64_t)S * v[k + 1] + q] - s0[q];
        for (int i = 0; i < 3; ++i) {
          float acc = 0.f;
          for (int k = 0; k < 3; ++k) acc += M[i][k] * ds[k];
          SG[i] = acc;
        }
        float tmp = 0.f;
        if (fix) {
          for (int j = 0; j < 3; ++j) tmp = (float)((double)tmp + (double)SG[j] * (double)rel[j]);
        } else {
          for (int j = 0; j < 3; ++j) tmp = (float)((double)SG[j] * (double)rel[j]);
        }
        e.sc[q] = (double)(tmp + s0[q]);
        for (int i = 0; i < 3; ++i) e.scg[q * 3 + i] = (double)SG[i];
      }
    }
  } else {
    double M[3][3];
    matrix_inverse<double>(A, M);
    double rel[3];
    for (int c = 0; c < 3; ++c) rel[c] = p[c] - X[0][c];
    double d0 = dens64[v[0]];
    double gr[3];
    for (int i = 0; i < 3; ++i) {
      gr[i] = 0;
      for (int j = 0; j < 3; ++j) gr[i] += M[i][j] * (dens64[v[j + 1]] - d0);
    }
    e.dens = d0 + rel[0] * gr[0] + rel[1] * gr[1] + rel[2] * gr[2];
    if (want_vel && g.vel) {
      double VG[3][3];
      const float* v0 = &g.vel[3 * (int64_t)v[0]];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          VG[i][j] = 0;
          for (int k = 0; k < 3; ++k)
            VG[i][j] += M[i][k] * ((double)g.vel[3 * (int64_t)v[k + 1] + j] - (double)v0[j]);
        }
      for (int i = 0; i < 3; ++i) {
        double tmp = 0;
        if (fix) for (int j = 0; j < 3; ++j) tmp += VG[j][i] * rel[j];
        else tmp = VG[2][i] * rel[2];
        e.vel[i] = tmp + (double)v0[i];
      }
      for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) e.grad[j * 3 + i] = VG[i][j];
    }
    if (want_sc && g.scal && g.S > 0) {
      int S = g.S;
      const float* s0 = &g.scal[(int64_t)S * v[0]];
      for (int q = 0; q < S; ++q) {
        double SG[3];
        for (int i = 0; i < 3; ++i) {
          SG[i] = 0;
          for (int k = 0; k < 3; ++k)
            SG[i] += M[i][k] * ((double)g.scal[(int64_t)S * v[k + 1] + q] - (double)s0[q]);
        }
        double tmp = 0;
        if (fix) for (int j = 0; j < 3; ++j) tmp += SG[j] * rel[j];
        else tmp = SG[2] * rel[2];
        e.sc[q] = tmp + (double)s0[q];
        for (int i = 0; i < 3; ++i) e.scg[q * 3 + i] = SG[i];
      }
    }
  }
}

// velocityDivergence / velocityShear / velocityVorticity (src/DTFE.cpp:394-433)
void derived(const double* g9, int mode, double* div, double* shear, double* vort) {
  if (mode == 0) {
    float g[9];
    for (int i = 0; i < 9; ++i) g[i] = (float)g9[i];
    *div = (double)(g[0] + g[4] + g[8]);
    float t[5];
    int idx = 0;
    for (int i = 0; i < 2; ++i)
      for (int j = i; j < 3; ++j) t[idx++] = (float)((double)(g[i * 3 + j] + g[j * 3 + i]) / 2.);
    float trace = (float)((double)(t[0] + t[3] + g[8]) / 3.);
    t[0] -= trace;
    t[3] -= trace;
    for (int i = 0; i < 5; ++i) shear[i] = t[i];
    idx = 0;
    for (int i = 0; i < 3; ++i)
      for (int j = i + 1; j < 3; ++j)
        vort[idx++] = (double)(float)((double)(g[i * 3 + j] - g[j * 3 + i]) / 2.);
  } else {
    const double* g = g9;
    *div = g[0] + g[4] + g[8];
    double t[5];
    int idx = 0;
    for (int i = 0; i < 2; ++i)
      for (int j = i; j < 3; ++j) t[idx++] = (g[i * 3 + j] + g[j * 3 + i]) / 2.;
    double trace = (t[0] + t[3] + g[8]) / 3.;
    t[0] -= trace;
    t[3] -= trace;
    for (int i = 0; i < 5; ++i) shear[i] = t[i];
    idx = 0;
    for (int i = 0; i < 3; ++i)
      for (int j = i + 1; j < 3; ++j) vort[idx++] = (g[i * 3 + j] - g[j * 3 + i]) / 2.;
  }
}

}  // namespace

extern "C" {

// vertexDensity (triangulation.cpp:200-279): rho_v = w_v*(D+1)/(rho_bar*sum V),
// 0 when any incident cell is infinite.  Volumes are the double determinant/6
// (Tetrahedron_3::volume, triangulation_miscellaneous.cc:205-213), summed in
// double in ascending tetrahedron order within each sub-box.  dens32: mode-0 result, float
// factor (D+1)/rho_bar (:220) times the weight, divided by the double sum;
// dens64: all-double result.  Either output may be NULL.
// dens32: the device's arithmetic — per sub-box, each FP64 volume rounded
// to integer units of 2^-62 of the sub-box vertices' bounding-box volume and
// summed exactly (fixed_volume.cuh), then (w * factor) / volume rounded to
// float; dens64 and volsum_out: plain FP64 sums (the FP64 oracle).
int oracle_vertex_density(int64_t T, const int32_t* tv, const int32_t* tn, int64_t V,
                          const float* xyz, const float* w, double rho_bar, float* dens32,
                          double* dens64, double* volsum_out, int K, const dtfe_subbox* boxes,
                          int nthreads) {
  std::vector<double> vol(V, 0.0);
  std::vector<long long> fixed(V, 0);
  std::vector<double> unit(V, 0.0);
  std::vector<char> hull(V, 0);
  // Sub-boxes own disjoint vertex and tetrahedron ranges, so they run in
  // parallel (one host thread each, as the reference's OpenMP threads do).
  const int nb = (K > 0 && boxes) ? K : 1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1)
  for (int b = 0; b < nb; ++b) {
    int64_t lo = (K > 0 && boxes) ? boxes[b].tet_offset : 0;
    int64_t hi = (K > 0 && boxes) ? boxes[b].tet_offset + boxes[b].n_tets : T;
    const int64_t v0 = (K > 0 && boxes) ? boxes[b].vert_offset : 0;
    const int64_t v1 = (K > 0 && boxes) ? boxes[b].vert_offset + boxes[b].n_verts : V;
    int bb[6] = {INT32_MAX, INT32_MIN, INT32_MAX, INT32_MIN, INT32_MAX, INT32_MIN};
    for (int64_t v = v0; v < v1; ++v)
      for (int c = 0; c < 3; ++c) {
        const int k = dtfe::float_order_key(xyz[3 * v + c]);
        bb[2 * c] = std::min(bb[2 * c], k);
        bb[2 * c + 1] = std::max(bb[2 * c + 1], k);
      }
    const dtfe::VolScale sc = v1 > v0 ? dtfe::vol_scale(dtfe::bbox_volume(bb)) : dtfe::VolScale{0.0, 0.0};
    for (int64_t v = v0; v < v1; ++v) unit[v] = sc.unit;
    for (int64_t t = lo; t < hi; ++t) {
      double X[4][3];
      for (int a = 0; a < 4; ++a)
        for (int k = 0; k < 3; ++k) X[a][k] = (double)xyz[3 * (int64_t)tv[4 * t + a] + k];
      double v6 = dtfe::orient_det(X[0], X[1], X[2], X[3]);
      double vt = v6 / 6.0;
      const long long q = std::llrint(vt * sc.inv_q);
      for (int a = 0; a < 4; ++a) {
        vol[tv[4 * t + a]] += vt;
        fixed[tv[4 * t + a]] += q;
      }
      for (int i = 0; i < 4; ++i)
        if (tn[4 * t + i] < 0)
          for (int a = 0; a < 4; ++a)
            if (a != i) hull[tv[4 * t + a]] = 1;
    }
  }
  float rb = (float)rho_bar;
  float factor = (float)(4.0 / (double)rb);
#pragma omp parallel for schedule(static) num_threads(nthreads > 0 ? nthreads : 1)
  for (int64_t v = 0; v < V; ++v) {
    bool zero = hull[v] || vol[v] == 0.0;
    if (dens32) dens32[v] = dtfe::density_from_fixed(fixed[v], unit[v], w[v], factor, hull[v] != 0);
    if (dens64) dens64[v] = zero ? 0.0 : (double)w[v] * 4.0 / ((double)rb * vol[v]);
    if (volsum_out) volsum_out[v] = vol[v];
  }
  return 0;
}

// The reference's own vertexDensity arithmetic (triangulation.cpp:200-279):
// per vertex the float sum `Real vol += volume(cell)` of its incident finite
// cells in ascending cell id (the harness's incident_cells order), each
// volume the double determinant / 6 rounded to float (volume(),
// triangulation_miscellaneous.cc:205-213); 0 when an incident cell is
// infinite; density = (weight * factor) / vol in float, factor =
// (NO_DIM+1.) / averageDensity as a float.
int oracle_vertex_density_ref(int64_t T, const int32_t* tv, const int32_t* tn, int64_t V, const float* xyz,
                              const float* w, double rho_bar, float* dens, int K, const dtfe_subbox* boxes,
                              int nthreads) {
  std::vector<float> vol(V, 0.f);
  std::vector<char> hull(V, 0);
  const int nb = (K > 0 && boxes) ? K : 1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1)
  for (int b = 0; b < nb; ++b) {
    int64_t lo = (K > 0 && boxes) ? boxes[b].tet_offset : 0;
    int64_t hi = (K > 0 && boxes) ? boxes[b].tet_offset + boxes[b].n_tets : T;
    for (int64_t t = lo; t < hi; ++t) {  // ascending: every vertex adds its cells in ascending id
      double X[4][3];
      for (int a = 0; a < 4; ++a)
        for (int k = 0; k < 3; ++k) X[a][k] = (double)xyz[3 * (int64_t)tv[4 * t + a] + k];
      const float vt = (float)(dtfe::orient_det(X[0], X[1], X[2], X[3]) / 6.0);
      for (int a = 0; a < 4; ++a) vol[tv[4 * t + a]] += vt;
      for (int i = 0; i < 4; ++i)
        if (tn[4 * t + i] < 0)
          for (int a = 0; a < 4; ++a)
            if (a != i) hull[tv[4 * t + a]] = 1;
    }
  }
  const float factor = (float)(4.0 / (double)(float)rho_bar);
  for (int64_t v = 0; v < V; ++v) dens[v] = hull[v] ? 0.f : (w[v] * factor) / vol[v];
  return 0;
}

// Canonical location of np points (double xyz) in tetrahedra [lo, hi).
int oracle_locate(int64_t T, const int32_t* tv, const int32_t* tn, const float* xyz,
                  int64_t lo, int64_t hi, int64_t np, const double* pts, int64_t* out) {
  Tess g{T, 0, tv, tn, xyz, nullptr, nullptr, 0};
  int64_t hint = lo;
  for (int64_t i = 0; i < np; ++i) {
    int64_t r = locate(g, &pts[3 * i], hint, lo, hi);
    out[i] = r;
    if (r >= 0) hint = r;
  }
  return 0;
}

// Interpolation over the sub-boxes into double outputs (main-grid layout).
// out[slot] may be NULL for unrequested fields.  loc (optional) receives the
// canonical tetrahedron of every cell centre (-1 outside the hull).
// nthreads > 0 parallelises over x-slabs of each tile.
int oracle_interpolate(int64_t T, const int32_t* tv, const int32_t* tn, int64_t V,
                       const float* xyz, const float* vel, const float* scal, int S,
                       const float* dens32, const double* dens64, int K,
                       const dtfe_subbox* boxes, const float* xs, const float* ys,
                       const float* zs, const int32_t grid[3], const dtfe_interp_opts* o,
                       int mode, double* const out[DTFE_NUM_FIELDS], int64_t* loc,
                       int nthreads, int64_t* n_fail) {
  Tess g{T, V, tv, tn, xyz, vel, scal, S};
  const uint32_t f = o->fields;
  const bool fix = (o->flags & DTFE_FLAG_FIX_VALUE_INTERP) != 0;
  // the reference's cell-centre raster stays on an outside point for the
  // rest of its z pencil (unaveraged_interpolation.cc:304 skips :353)
  const bool stale_after_outside = o->method == DTFE_METHOD_CENTRE && !(o->flags & DTFE_FLAG_FIX_OUTSIDE_RASTER);
  auto has = [&](int s) { return (f & DTFE_FIELD_BIT(s)) != 0 && out[s] != nullptr; };
  const bool want_grad = has(DTFE_VELOCITY_GRADIENT) || has(DTFE_VELOCITY_DIVERGENCE) ||
                         has(DTFE_VELOCITY_SHEAR) || has(DTFE_VELOCITY_VORTICITY);
  const bool want_vel = has(DTFE_VELOCITY) || want_grad || has(DTFE_VELOCITY_STD);
  const bool want_sc = has(DTFE_SCALAR) || has(DTFE_SCALAR_GRADIENT);
  const int method = o->method;
  const int NN = method == DTFE_METHOD_CENTRE ? 1 : o->n_samples;
  if (NN < 1) return DTFE_ERR_ARG;
  if (has(DTFE_VELOCITY_STD) && (method != DTFE_METHOD_MONTE_CARLO || NN > DTFE_MAX_STD_SAMPLES))
    return DTFE_ERR_ARG;
  int nroot = 1;
  if (method == DTFE_METHOD_EQUIDISTANT) {
    nroot = (int)std::lround(std::cbrt((double)NN));
    if (nroot * nroot * nroot != NN) return DTFE_ERR_ARG;
  }
  int64_t fails = 0;
  const int64_t G1 = grid[1], G2 = grid[2];
  for (int b = 0; b < K; ++b) {
    const dtfe_subbox& B = boxes[b];
    const int64_t lo = B.tet_offset, hi = B.tet_offset + B.n_tets;
    const float dx[3] = {B.dx[0], B.dx[1], B.dx[2]};
    const uint64_t key = dtfe::mc_key(o->seed, B.part_no);
    // equidistant offsets (averaged_interpolation_2.cc:726-740)
    std::vector<float> eq(3 * (size_t)NN);
    if (method == DTFE_METHOD_EQUIDISTANT) {
      for (int i1 = 0; i1 < nroot; ++i1)
        for (int i2 = 0; i2 < nroot; ++i2)
          for (int i3 = 0; i3 < nroot; ++i3) {
            int idx = i1 * nroot * nroot + i2 * nroot + i3;
            eq[3 * idx + 2] = (float)((i3 + 0.5) * (double)dx[2] / nroot - (double)dx[2] / 2.);
            eq[3 * idx + 0] = (float)((i1 + 0.5) * (double)dx[0] / nroot - (double)dx[0] / 2.);
            eq[3 * idx + 1] = (float)((i2 + 0.5) * (double)dx[1] / nroot - (double)dx[1] / 2.);
          }
    }
    // Pencils (i, j) run in parallel; each thread carries its walk hint from
    // one pencil to the next (the reference carries it along its raster).
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1) reduction(+ : fails)
    {
      int64_t row_hint = lo;
      std::vector<double> stdv(3 * (size_t)std::max(NN, 1));
#pragma omp for collapse(2) schedule(dynamic, 4)
    for (int i = 0; i < B.tile_dims[0]; ++i) {
      for (int j = 0; j < B.tile_dims[1]; ++j) {
        int64_t hint = row_hint;
        bool stale = false;  // an earlier sample of this pencil was outside
        for (int k = 0; k < B.tile_dims[2]; ++k) {
          const float x = xs[B.coord_offset[0] + i], y = ys[B.coord_offset[1] + j],
                      z = zs[B.coord_offset[2] + k];
          const int64_t cell = ((int64_t)(B.tile_origin[0] + i) * G1 + (B.tile_origin[1] + j)) * G2 +
                               (B.tile_origin[2] + k);
          double pc[3] = {(double)x, (double)y, (double)z};
          int64_t tc = stale ? -1 : locate(g, pc, hint, lo, hi);
          if (tc == -2) { ++fails; tc = -1; }
          if (tc < 0 && stale_after_outside) stale = true;
          if (tc >= 0) {
            hint = tc;
            if (k == 0) row_hint = tc;
          }
          if (loc) loc[cell] = tc;
          // accumulators: float in mode 0, double in mode 1
          float fD = 0.f, fV[3] = {0, 0, 0}, fG[9] = {0}, fS[DTFE_MAX_SCALARS] = {0},
                fSG[3 * DTFE_MAX_SCALARS] = {0};
          double dD = 0, dV[3] = {0, 0, 0}, dG[9] = {0}, dS[DTFE_MAX_SCALARS] = {0},
                 dSG[3 * DTFE_MAX_SCALARS] = {0};
          for (size_t q = 0; q < stdv.size(); ++q) stdv[q] = 0.0;
          for (int w = 0; w < NN; ++w) {
            double p[3];
            int64_t t;
            if (method == DTFE_METHOD_CENTRE) {
              p[0] = pc[0]; p[1] = pc[1]; p[2] = pc[2];
              t = tc;
            } else {
              if (method == DTFE_METHOD_MONTE_CARLO) {
                double u[3];
                dtfe::mc_offsets(key, (uint64_t)cell, (uint32_t)w, u);
                for (int c = 0; c < 3; ++c) p[c] = u[c] * (double)dx[c] + pc[c];
              } else {
                p[0] = (double)(x + eq[3 * w + 0]);
                p[1] = (double)(y + eq[3 * w + 1]);
                p[2] = (double)(z + eq[3 * w + 2]);
              }
              t = locate(g, p, tc >= 0 ? tc : hint, lo, hi);
              if (t == -2) { ++fails; t = -1; }
            }
            if (t < 0) continue;  // infinite cell: contributes nothing
            CellEval e{};
            eval_cell(g, dens32, dens64, t, p, mode, fix, want_vel, want_sc, e);
            if (mode == 0) {
              fD += (float)e.dens;
              for (int c = 0; c < 3; ++c) fV[c] += (float)e.vel[c];
              for (int c = 0; c < 9; ++c) fG[c] += (float)e.grad[c];
              for (int q = 0; q < S; ++q) {
                fS[q] += (float)e.sc[q];
                for (int c = 0; c < 3; ++c) fSG[3 * q + c] += (float)e.scg[3 * q + c];
              }
            } else {
              dD += e.dens;
              for (int c = 0; c < 3; ++c) dV[c] += e.vel[c];
              for (int c = 0; c < 9; ++c) dG[c] += e.grad[c];
              for (int q = 0; q < S; ++q) {
                dS[q] += e.sc[q];
                for (int c = 0; c < 3; ++c) dSG[3 * q + c] += e.scg[3 * q + c];
              }
            }
            if (want_vel)
              for (int c = 0; c < 3; ++c) stdv[3 * w + c] = e.vel[c];
          }
          double D, Vv[3], Gg[9], Ss[DTFE_MAX_SCALARS], SGg[3 * DTFE_MAX_SCALARS], sd = 0;
          if (mode == 0) {
            float fn = (float)NN;
            D = (double)(fD / fn);
            for (int c = 0; c < 3; ++c) Vv[c] = (double)(fV[c] / fn);
            for (int c = 0; c < 9; ++c) Gg[c] = (double)(fG[c] / fn);
            for (int q = 0; q < S; ++q) {
              Ss[q] = (double)(fS[q] / fn);
              for (int c = 0; c < 3; ++c) SGg[3 * q + c] = (double)(fSG[3 * q + c] / fn);
            }
            if (has(DTFE_VELOCITY_STD)) {
              // standardDeviation for Pvector (triangulation_miscellaneous.cc:256-271)
              float mean[3] = {0, 0, 0};
              for (int w = 0; w < NN; ++w)
                for (int c = 0; c < 3; ++c) mean[c] += (float)stdv[3 * w + c];
              for (int c = 0; c < 3; ++c) mean[c] /= (float)NN;
              float r = 0.f;
              for (int w = 0; w < NN; ++w)
                for (int c = 0; c < 3; ++c) {
                  float d = (float)stdv[3 * w + c] - mean[c];
                  r += d * d;
                }
              sd = (double)std::sqrt(r / (float)NN);
            }
          } else {
            D = dD / NN;
            for (int c = 0; c < 3; ++c) Vv[c] = dV[c] / NN;
            for (int c = 0; c < 9; ++c) Gg[c] = dG[c] / NN;
            for (int q = 0; q < S; ++q) {
              Ss[q] = dS[q] / NN;
              for (int c = 0; c < 3; ++c) SGg[3 * q + c] = dSG[3 * q + c] / NN;
            }
            if (has(DTFE_VELOCITY_STD)) {
              double mean[3] = {0, 0, 0};
              for (int w = 0; w < NN; ++w)
                for (int c = 0; c < 3; ++c) mean[c] += stdv[3 * w + c];
              for (int c = 0; c < 3; ++c) mean[c] /= NN;
              double r = 0;
              for (int w = 0; w < NN; ++w)
                for (int c = 0; c < 3; ++c) {
                  double d = stdv[3 * w + c] - mean[c];
                  r += d * d;
                }
              sd = std::sqrt(r / NN);
            }
          }
          if (has(DTFE_DENSITY)) out[DTFE_DENSITY][cell] = D;
          if (has(DTFE_VELOCITY))
            for (int c = 0; c < 3; ++c) out[DTFE_VELOCITY][3 * cell + c] = Vv[c];
          if (has(DTFE_VELOCITY_GRADIENT))
            for (int c = 0; c < 9; ++c) out[DTFE_VELOCITY_GRADIENT][9 * cell + c] = Gg[c];
          if (has(DTFE_VELOCITY_DIVERGENCE) || has(DTFE_VELOCITY_SHEAR) ||
              has(DTFE_VELOCITY_VORTICITY)) {
            double dv, sh[5], vo[3];
            derived(Gg, mode, &dv, sh, vo);
            if (has(DTFE_VELOCITY_DIVERGENCE)) out[DTFE_VELOCITY_DIVERGENCE][cell] = dv;
            if (has(DTFE_VELOCITY_SHEAR))
              for (int c = 0; c < 5; ++c) out[DTFE_VELOCITY_SHEAR][5 * cell + c] = sh[c];
            if (has(DTFE_VELOCITY_VORTICITY))
              for (int c = 0; c < 3; ++c) out[DTFE_VELOCITY_VORTICITY][3 * cell + c] = vo[c];
          }
          if (has(DTFE_VELOCITY_STD)) out[DTFE_VELOCITY_STD][cell] = sd;
          if (has(DTFE_SCALAR))
            for (int q = 0; q < S; ++q) out[DTFE_SCALAR][(int64_t)S * cell + q] = Ss[q];
          if (has(DTFE_SCALAR_GRADIENT))
            for (int q = 0; q < 3 * S; ++q)
              out[DTFE_SCALAR_GRADIENT][(int64_t)3 * S * cell + q] = SGg[q];
        }
      }
    }
    }
  }
  if (n_fail) *n_fail = fails;
  return fails ? DTFE_ERR_WALK : DTFE_OK;
}

// Fields at user sampling points: interpolateUserSampling
// (src/CGAL_triangulation/unaveraged_interpolation.cc:560-691).  Points
// outside `region` (closed, isPointInBox) are dropped; the rest, in order,
// are located (walk hinted by the previous hit, canonical tie rule) in the
// tetrahedra [lo, hi) and evaluated as cell centres are; outside the hull
// zeros.  Divergence, shear and vorticity from the gradient
// (src/DTFE.cpp:394-475).  Returns the number of points kept in *n_out.
int oracle_interpolate_points(int64_t T, const int32_t* tv, const int32_t* tn, int64_t V, const float* xyz,
                              const float* vel, const float* scal, int S, const float* dens32, const double* dens64,
                              int64_t lo, int64_t hi, int64_t n, const float* pts, const float region[6],
                              uint32_t fields, int mode, int fix, double* const out[DTFE_NUM_FIELDS],
                              int64_t* n_out) {
  (void)T;
  (void)V;
  Tess g{T, V, tv, tn, xyz, vel, scal, S};
  auto has = [&](int s) { return (fields & DTFE_FIELD_BIT(s)) != 0 && out[s] != nullptr; };
  if (has(DTFE_VELOCITY_STD)) return DTFE_ERR_ARG;
  const bool want_vel = has(DTFE_VELOCITY) || has(DTFE_VELOCITY_GRADIENT) || has(DTFE_VELOCITY_DIVERGENCE) ||
                        has(DTFE_VELOCITY_SHEAR) || has(DTFE_VELOCITY_VORTICITY);
  const bool want_sc = has(DTFE_SCALAR) || has(DTFE_SCALAR_GRADIENT);
  int64_t m = 0, hint = lo;
  for (int64_t i = 0; i < n; ++i) {
    const float* q = pts + 3 * i;
    bool in = true;
    for (int c = 0; c < 3; ++c) in = in && q[c] >= region[2 * c] && q[c] <= region[2 * c + 1];
    if (!in) continue;
    const double p[3] = {(double)q[0], (double)q[1], (double)q[2]};
    int64_t t = locate(g, p, hint, lo, hi);
    if (t == -2) return DTFE_ERR_WALK;
    CellEval e;
    std::memset(&e, 0, sizeof(e));
    if (t >= 0) {
      hint = t;
      eval_cell(g, dens32, dens64, t, p, mode, fix != 0, want_vel, want_sc, e);
    }
    if (has(DTFE_DENSITY)) out[DTFE_DENSITY][m] = e.dens;
    if (has(DTFE_VELOCITY))
      for (int c = 0; c < 3; ++c) out[DTFE_VELOCITY][3 * m + c] = e.vel[c];
    if (has(DTFE_VELOCITY_GRADIENT))
      for (int c = 0; c < 9; ++c) out[DTFE_VELOCITY_GRADIENT][9 * m + c] = e.grad[c];
    if (has(DTFE_VELOCITY_DIVERGENCE) || has(DTFE_VELOCITY_SHEAR) || has(DTFE_VELOCITY_VORTICITY)) {
      double dv, sh[5], vo[3];
      derived(e.grad, mode, &dv, sh, vo);
      if (has(DTFE_VELOCITY_DIVERGENCE)) out[DTFE_VELOCITY_DIVERGENCE][m] = dv;
      if (has(DTFE_VELOCITY_SHEAR))
        for (int c = 0; c < 5; ++c) out[DTFE_VELOCITY_SHEAR][5 * m + c] = sh[c];
      if (has(DTFE_VELOCITY_VORTICITY))
        for (int c = 0; c < 3; ++c) out[DTFE_VELOCITY_VORTICITY][3 * m + c] = vo[c];
    }
    if (has(DTFE_SCALAR))
      for (int c = 0; c < S; ++c) out[DTFE_SCALAR][(int64_t)S * m + c] = e.sc[c];
    if (has(DTFE_SCALAR_GRADIENT))
      for (int c = 0; c < 3 * S; ++c) out[DTFE_SCALAR_GRADIENT][(int64_t)3 * S * m + c] = e.scg[c];
    ++m;
  }
  *n_out = m;
  return DTFE_OK;
}

// Sample coordinates of a redshift-cone grid (interpolateRedshiftCone,
// unaveraged_interpolation.cc:381-455) in the reference's float arithmetic:
//   * checkAngles (triangulation_miscellaneous.cc:162-197, 3-D): theta limits
//     must lie in [0, 180]; psi limits wrapped by a -= floor(a / 360) 360;
//     psi_max += 360 when psi_min > psi_max; angles times float(PI / 180)
//     with PI = 3.14159265 (define.h:47);
//   * user_options.cc:1000-1009: a psi span of 360 degrees or more is refused;
//   * dx = (hi - lo) / n in float; first value float(lo + dx / 2.) (double
//     sum), then sequential float adds of dx (:435-447, 505-509);
//   * per-axis tables: r, sin(theta), cos(theta), cos(psi), sin(psi) through
//     the float overloads of <cmath> (the reference's `using namespace std`).
// The point is (o0 + r st cp, o1 + r st sp, o2 + r ct), left to right in float.
int oracle_cone_tables(const float cone[6], const int32_t dims[3], float* r, float* st, float* ct, float* cp,
                       float* sp) {
  float b[6];
  for (int i = 0; i < 6; ++i) b[i] = cone[i];
  for (int a = 0; a < 3; ++a)
    if (dims[a] <= 0) return DTFE_ERR_ARG;
  if (b[2] < 0.f || b[2] > 180.f || b[3] < 0.f || b[3] > 180.f) return DTFE_ERR_ARG;
  if (b[5] - b[4] >= 360.f) return DTFE_ERR_ARG;
  b[4] -= std::floor(b[4] / 360.f) * 360.f;
  b[5] -= std::floor(b[5] / 360.f) * 360.f;
  if (b[4] > b[5]) b[5] += 360.f;
  const float rad = (float)(3.14159265 / 180.);
  for (int i = 2; i < 6; ++i) b[i] *= rad;
  float dx[3];
  for (int a = 0; a < 3; ++a) dx[a] = (b[2 * a + 1] - b[2 * a]) / (float)dims[a];
  float x = (float)((double)b[0] + (double)dx[0] / 2.);
  for (int i = 0; i < dims[0]; ++i, x += dx[0]) r[i] = x;
  x = (float)((double)b[2] + (double)dx[1] / 2.);
  for (int j = 0; j < dims[1]; ++j, x += dx[1]) {
    st[j] = std::sin(x);
    ct[j] = std::cos(x);
  }
  x = (float)((double)b[4] + (double)dx[2] / 2.);
  for (int k = 0; k < dims[2]; ++k, x += dx[2]) {
    cp[k] = std::cos(x);
    sp[k] = std::sin(x);
  }
  return DTFE_OK;
}

// Fields on a redshift-cone grid: interpolateRedshiftCone
// (unaveraged_interpolation.cc:381-547).  Raster r slowest, psi fastest; each
// sample located from the previous hit (canonical tie rule) in the
// tetrahedra [lo, hi) and evaluated as a cell centre; outside the hull
// zeros.  An outside sample skips `psi += dx` (the `continue` at :466 jumps
// over :527), so the rest of that psi pencil re-locates the same outside
// point: zeros to its end.  fix_outside advances psi regardless.  Derived
// fields from the gradient (src/DTFE.cpp:394-475).
int oracle_interpolate_cone(int64_t T, const int32_t* tv, const int32_t* tn, int64_t V, const float* xyz,
                            const float* vel, const float* scal, int S, const float* dens32, const double* dens64,
                            int64_t lo, int64_t hi, const float cone[6], const float origin[3],
                            const int32_t dims[3], uint32_t fields, int mode, int fix, int fix_outside,
                            double* const out[DTFE_NUM_FIELDS]) {
  Tess g{T, V, tv, tn, xyz, vel, scal, S};
  auto has = [&](int s) { return (fields & DTFE_FIELD_BIT(s)) != 0 && out[s] != nullptr; };
  if (has(DTFE_VELOCITY_STD)) return DTFE_ERR_ARG;
  std::vector<float> r(dims[0] > 0 ? dims[0] : 1), st(dims[1] > 0 ? dims[1] : 1), ct(st.size()),
      cp(dims[2] > 0 ? dims[2] : 1), sp(cp.size());
  int rc = oracle_cone_tables(cone, dims, r.data(), st.data(), ct.data(), cp.data(), sp.data());
  if (rc) return rc;
  const bool want_vel = has(DTFE_VELOCITY) || has(DTFE_VELOCITY_GRADIENT) || has(DTFE_VELOCITY_DIVERGENCE) ||
                        has(DTFE_VELOCITY_SHEAR) || has(DTFE_VELOCITY_VORTICITY);
  const bool want_sc = has(DTFE_SCALAR) || has(DTFE_SCALAR_GRADIENT);
  int64_t m = 0, hint = lo;
  for (int i = 0; i < dims[0]; ++i)
    for (int j = 0; j < dims[1]; ++j) {
      const float rs = r[i] * st[j];
      const float z = origin[2] + r[i] * ct[j];
      int kp = 0;  // the psi bin the reference's running `psi` holds
      for (int k = 0; k < dims[2]; ++k, ++m) {
        const float q[3] = {origin[0] + rs * cp[kp], origin[1] + rs * sp[kp], z};
        const double p[3] = {(double)q[0], (double)q[1], (double)q[2]};
        const int64_t t = hi > lo ? locate(g, p, hint, lo, hi) : -1;
        if (t == -2) return DTFE_ERR_WALK;
        CellEval e;
        std::memset(&e, 0, sizeof(e));
        if (t >= 0) {
          hint = t;
          eval_cell(g, dens32, dens64, t, p, mode, fix != 0, want_vel, want_sc, e);
        }
        if (t >= 0 || fix_outside) ++kp;
        if (has(DTFE_DENSITY)) out[DTFE_DENSITY][m] = e.dens;
        if (has(DTFE_VELOCITY))
          for (int c = 0; c < 3; ++c) out[DTFE_VELOCITY][3 * m + c] = e.vel[c];
        if (has(DTFE_VELOCITY_GRADIENT))
          for (int c = 0; c < 9; ++c) out[DTFE_VELOCITY_GRADIENT][9 * m + c] = e.grad[c];
        if (has(DTFE_VELOCITY_DIVERGENCE) || has(DTFE_VELOCITY_SHEAR) || has(DTFE_VELOCITY_VORTICITY)) {
          double dv, sh[5], vo[3];
          derived(e.grad, mode, &dv, sh, vo);
          if (has(DTFE_VELOCITY_DIVERGENCE)) out[DTFE_VELOCITY_DIVERGENCE][m] = dv;
          if (has(DTFE_VELOCITY_SHEAR))
            for (int c = 0; c < 5; ++c) out[DTFE_VELOCITY_SHEAR][5 * m + c] = sh[c];
          if (has(DTFE_VELOCITY_VORTICITY))
            for (int c = 0; c < 3; ++c) out[DTFE_VELOCITY_VORTICITY][3 * m + c] = vo[c];
        }
        if (has(DTFE_SCALAR))
          for (int c = 0; c < S; ++c) out[DTFE_SCALAR][(int64_t)S * m + c] = e.sc[c];
        if (has(DTFE_SCALAR_GRADIENT))
          for (int c = 0; c < 3 * S; ++c) out[DTFE_SCALAR_GRADIENT][(int64_t)3 * S * m + c] = e.scg[c];
      }
    }
  return DTFE_OK;
}

}  // extern "C"

namespace {

// Monte-Carlo average of one point sample (averaged_interpolation_2.cc:
// 343-418, 540-637): the centre located from `hint` (its tetrahedron, when
// inside, seeds the sample walks as the reference's `previous`), NN points
// from sample(w, u, q) with u the Philox offsets of (key, index, w), each
// located and evaluated, summed in float (mode 0) or double (mode 1) in
// sample order, outside points skipped but counted; the mean and its derived
// fields written to row m.  Returns -2 on a walk failure.
template <class Sample>
int average_row(const Tess& g, const float* dens32, const double* dens64, const float centre[3], Sample sample,
                uint64_t key, uint64_t index, int NN, int mode, bool fix, bool want_vel, bool want_sc,
                int64_t& hint, int64_t lo, int64_t hi, uint32_t fields, double* const out[DTFE_NUM_FIELDS],
                int64_t m) {
  const int S = g.S;
  auto has = [&](int s) { return (fields & DTFE_FIELD_BIT(s)) != 0 && out[s] != nullptr; };
  float fD = 0.f, fV[3] = {0, 0, 0}, fG[9] = {0}, fS[DTFE_MAX_SCALARS] = {0}, fSG[3 * DTFE_MAX_SCALARS] = {0};
  double dD = 0, dV[3] = {0, 0, 0}, dG[9] = {0}, dS[DTFE_MAX_SCALARS] = {0}, dSG[3 * DTFE_MAX_SCALARS] = {0};
  if (hi > lo) {
    const double pc[3] = {(double)centre[0], (double)centre[1], (double)centre[2]};
    const int64_t tc = locate(g, pc, hint, lo, hi);
    if (tc == -2) return -2;
    if (tc >= 0) hint = tc;
    for (int w = 0; w < NN; ++w) {
      double u[3];
      dtfe::mc_offsets(key, index, (uint32_t)w, u);
      float q[3];
      sample(u, q);
      const double p[3] = {(double)q[0], (double)q[1], (double)q[2]};
      const int64_t t = locate(g, p, hint, lo, hi);
      if (t == -2) return -2;
      if (t < 0) continue;
      CellEval e{};
      eval_cell(g, dens32, dens64, t, p, mode, fix, want_vel, want_sc, e);
      if (mode == 0) {
        fD += (float)e.dens;
        for (int c = 0; c < 3; ++c) fV[c] += (float)e.vel[c];
        for (int c = 0; c < 9; ++c) fG[c] += (float)e.grad[c];
        for (int k = 0; k < S; ++k) {
          fS[k] += (float)e.sc[k];
          for (int c = 0; c < 3; ++c) fSG[3 * k + c] += (float)e.scg[3 * k + c];
        }
      } else {
        dD += e.dens;
        for (int c = 0; c < 3; ++c) dV[c] += e.vel[c];
        for (int c = 0; c < 9; ++c) dG[c] += e.grad[c];
        for (int k = 0; k < S; ++k) {
          dS[k] += e.sc[k];
          for (int c = 0; c < 3; ++c) dSG[3 * k + c] += e.scg[3 * k + c];
        }
      }
    }
  }
  double D, Vv[3], Gg[9], Ss[DTFE_MAX_SCALARS], SGg[3 * DTFE_MAX_SCALARS];
  if (mode == 0) {
    const float fn = (float)NN;
    D = (double)(fD / fn);
    for (int c = 0; c < 3; ++c) Vv[c] = (double)(fV[c] / fn);
    for (int c = 0; c < 9; ++c) Gg[c] = (double)(fG[c] / fn);
    for (int k = 0; k < S; ++k) {
      Ss[k] = (double)(fS[k] / fn);
      for (int c = 0; c < 3; ++c) SGg[3 * k + c] = (double)(fSG[3 * k + c] / fn);
    }
  } else {
    D = dD / NN;
    for (int c = 0; c < 3; ++c) Vv[c] = dV[c] / NN;
    for (int c = 0; c < 9; ++c) Gg[c] = dG[c] / NN;
    for (int k = 0; k < S; ++k) {
      Ss[k] = dS[k] / NN;
      for (int c = 0; c < 3; ++c) SGg[3 * k + c] = dSG[3 * k + c] / NN;
    }
  }
  if (has(DTFE_DENSITY)) out[DTFE_DENSITY][m] = D;
  if (has(DTFE_VELOCITY))
    for (int c = 0; c < 3; ++c) out[DTFE_VELOCITY][3 * m + c] = Vv[c];
  if (has(DTFE_VELOCITY_GRADIENT))
    for (int c = 0; c < 9; ++c) out[DTFE_VELOCITY_GRADIENT][9 * m + c] = Gg[c];
  if (has(DTFE_VELOCITY_DIVERGENCE) || has(DTFE_VELOCITY_SHEAR) || has(DTFE_VELOCITY_VORTICITY)) {
    double dv, sh[5], vo[3];
    derived(Gg, mode, &dv, sh, vo);
    if (has(DTFE_VELOCITY_DIVERGENCE)) out[DTFE_VELOCITY_DIVERGENCE][m] = dv;
    if (has(DTFE_VELOCITY_SHEAR))
      for (int c = 0; c < 5; ++c) out[DTFE_VELOCITY_SHEAR][5 * m + c] = sh[c];
    if (has(DTFE_VELOCITY_VORTICITY))
      for (int c = 0; c < 3; ++c) out[DTFE_VELOCITY_VORTICITY][3 * m + c] = vo[c];
  }
  if (has(DTFE_SCALAR))
    for (int c = 0; c < S; ++c) out[DTFE_SCALAR][(int64_t)S * m + c] = Ss[c];
  if (has(DTFE_SCALAR_GRADIENT))
    for (int c = 0; c < 3 * S; ++c) out[DTFE_SCALAR_GRADIENT][(int64_t)3 * S * m + c] = SGg[c];
  return 0;
}

}  // namespace

extern "C" {

// Volume averages at user sampling points: interpolateUserSampling_averaged_2
// (averaged_interpolation_2.cc:470-647).  Points outside `region` (closed)
// dropped; for each kept point i, NN points float(position + u delta) per
// axis (:545-553), u the Philox offsets of (seed, i, w) in place of the
// reference's mt19937 stream (seed + 1000 partNo with partNo = -1 here).
int oracle_average_points(int64_t T, const int32_t* tv, const int32_t* tn, int64_t V, const float* xyz,
                          const float* vel, const float* scal, int S, const float* dens32, const double* dens64,
                          int64_t lo, int64_t hi, int64_t n, const float* pts, const float* delta,
                          const float region[6], uint32_t fields, int NN, uint64_t seed, int mode, int fix,
                          double* const out[DTFE_NUM_FIELDS], int64_t* n_out) {
  Tess g{T, V, tv, tn, xyz, vel, scal, S};
  if ((fields & DTFE_FIELD_BIT(DTFE_VELOCITY_STD)) || NN < 1) return DTFE_ERR_ARG;
  const bool want_vel = (fields & (DTFE_FIELD_BIT(DTFE_VELOCITY) | DTFE_FIELD_BIT(DTFE_VELOCITY_GRADIENT) |
                                   DTFE_FIELD_BIT(DTFE_VELOCITY_DIVERGENCE) | DTFE_FIELD_BIT(DTFE_VELOCITY_SHEAR) |
                                   DTFE_FIELD_BIT(DTFE_VELOCITY_VORTICITY))) != 0;
  const bool want_sc = (fields & (DTFE_FIELD_BIT(DTFE_SCALAR) | DTFE_FIELD_BIT(DTFE_SCALAR_GRADIENT))) != 0;
  const uint64_t key = dtfe::mc_key(seed, -1);
  int64_t m = 0, hint = lo;
  for (int64_t i = 0; i < n; ++i) {
    const float* q = pts + 3 * i;
    bool in = true;
    for (int c = 0; c < 3; ++c) in = in && q[c] >= region[2 * c] && q[c] <= region[2 * c + 1];
    if (!in) continue;
    const float* dl = delta + 3 * i;
    auto sample = [&](const double u[3], float r[3]) {
      for (int c = 0; c < 3; ++c) r[c] = (float)((double)q[c] + u[c] * (double)dl[c]);
    };
    if (average_row(g, dens32, dens64, q, sample, key, (uint64_t)i, NN, mode, fix != 0, want_vel, want_sc, hint,
                    lo, hi, fields, out, m))
      return DTFE_ERR_WALK;
    ++m;
  }
  *n_out = m;
  return DTFE_OK;
}

// Volume averages on a redshift-cone grid: interpolateRedshiftCone_averaged_2
// (averaged_interpolation_2.cc:245-466).  Bin (i, j, k) centred at the
// oracle_cone_tables values; NN points with r, theta, psi each
// float(centre + u size) (:360-362), sin and cos of the angles evaluated in
// double and rounded to float, then o + (r st) cp ... in float; u the Philox
// offsets of (seed, bin, w).  No stuck psi (the averaged loop has no
// `continue` before its psi += dx).
int oracle_average_cone(int64_t T, const int32_t* tv, const int32_t* tn, int64_t V, const float* xyz,
                        const float* vel, const float* scal, int S, const float* dens32, const double* dens64,
                        int64_t lo, int64_t hi, const float cone[6], const float origin[3], const int32_t dims[3],
                        uint32_t fields, int NN, uint64_t seed, int mode, int fix,
                        double* const out[DTFE_NUM_FIELDS]) {
  Tess g{T, V, tv, tn, xyz, vel, scal, S};
  if ((fields & DTFE_FIELD_BIT(DTFE_VELOCITY_STD)) || NN < 1) return DTFE_ERR_ARG;
  std::vector<float> r(dims[0] > 0 ? dims[0] : 1), st(dims[1] > 0 ? dims[1] : 1), ct(st.size()),
      cp(dims[2] > 0 ? dims[2] : 1), sp(cp.size());
  int rc = oracle_cone_tables(cone, dims, r.data(), st.data(), ct.data(), cp.data(), sp.data());
  if (rc) return rc;
  // the bin centres and sizes of the angles, as oracle_cone_tables computes them
  float b[6];
  for (int i = 0; i < 6; ++i) b[i] = cone[i];
  b[4] -= std::floor(b[4] / 360.f) * 360.f;
  b[5] -= std::floor(b[5] / 360.f) * 360.f;
  if (b[4] > b[5]) b[5] += 360.f;
  const float rad = (float)(3.14159265 / 180.);
  for (int i = 2; i < 6; ++i) b[i] *= rad;
  float dx[3];
  for (int a = 0; a < 3; ++a) dx[a] = (b[2 * a + 1] - b[2 * a]) / (float)dims[a];
  std::vector<float> th(dims[1]), ps(dims[2]);
  float x = (float)((double)b[2] + (double)dx[1] / 2.);
  for (int j = 0; j < dims[1]; ++j, x += dx[1]) th[j] = x;
  x = (float)((double)b[4] + (double)dx[2] / 2.);
  for (int k = 0; k < dims[2]; ++k, x += dx[2]) ps[k] = x;
  const bool want_vel = (fields & (DTFE_FIELD_BIT(DTFE_VELOCITY) | DTFE_FIELD_BIT(DTFE_VELOCITY_GRADIENT) |
                                   DTFE_FIELD_BIT(DTFE_VELOCITY_DIVERGENCE) | DTFE_FIELD_BIT(DTFE_VELOCITY_SHEAR) |
                                   DTFE_FIELD_BIT(DTFE_VELOCITY_VORTICITY))) != 0;
  const bool want_sc = (fields & (DTFE_FIELD_BIT(DTFE_SCALAR) | DTFE_FIELD_BIT(DTFE_SCALAR_GRADIENT))) != 0;
  const uint64_t key = dtfe::mc_key(seed, -1);
  int64_t m = 0, hint = lo;
  for (int i = 0; i < dims[0]; ++i)
    for (int j = 0; j < dims[1]; ++j)
      for (int k = 0; k < dims[2]; ++k, ++m) {
        const float rs = r[i] * st[j];
        const float centre[3] = {origin[0] + rs * cp[k], origin[1] + rs * sp[k], origin[2] + r[i] * ct[j]};
        auto sample = [&](const double u[3], float q[3]) {
          const float R = (float)((double)r[i] + u[0] * (double)dx[0]);
          const float Th = (float)((double)th[j] + u[1] * (double)dx[1]);
          const float Ps = (float)((double)ps[k] + u[2] * (double)dx[2]);
          const float s1 = (float)std::sin((double)Th), c1 = (float)std::cos((double)Th);
          const float c2 = (float)std::cos((double)Ps), s2 = (float)std::sin((double)Ps);
          const float rr = R * s1;
          q[0] = origin[0] + rr * c2;
          q[1] = origin[1] + rr * s2;
          q[2] = origin[2] + R * c1;
        };
        if (average_row(g, dens32, dens64, centre, sample, key, (uint64_t)m, NN, mode, fix != 0, want_vel, want_sc,
                        hint, lo, hi, fields, out, m))
          return DTFE_ERR_WALK;
      }
  return DTFE_OK;
}

// Averaging method 1: interpolateGrid_averaged_1
// (src/CGAL_triangulation/averaged_interpolation_1.cc:197-421), per sub-box
// over its tetrahedra in order.
//   * quasi-random table: the first 100 NN Sobol points of the corner
//     simplex, as floats (quasiRandomSequence :32-50);
//   * a tetrahedron whose bounding box misses the region is skipped
//     (cellOutsideRegion :67-77; closed boxes, double coordinates);
//   * checkCellPosition (:84-118): base = vertex 0, basePosition =
//     float(base - region lo), its cell floor(basePosition / dx) in float,
//     that cell's box [i dx + lo, i dx + lo + dx] in float, one cell when
//     vertices 1..3 lie in it (closed, isPointInBox box.h:63-73);
//     vertexMatrix = double differences to the base;
//   * volume = float(determinant / 6) (triangulation_miscellaneous.cc:205-213),
//     inverse edge matrix as matrixInverse;
//   * one valid cell: vertex averages (float sums / 4) times the volume and
//     the gradients times the volume are added to it (:292-318);
//   * otherwise n = size_t(NN vol / vcell) + 1 points (at most 100 NN) when
//     vol / vcell > 1/6, else NN/6 + 1; point i = q_i vertexMatrix (double);
//     its cell floor((basePosition + p) / dx) (double); densityValue,
//     velocityValue, scalarValue at p and the gradients, each times vol / n,
//     added to that cell (:322-364);
//   * every cell divided by the cell volume dx0 dx1 dx2 (:371-393);
//     divergence, shear and vorticity from the averaged gradient
//     (src/DTFE.cpp:394-475).
// mode 0 is the reference's float arithmetic and accumulation order; mode 1
// evaluates values, volumes and sums in double over the same points and
// cells.
int oracle_method1(int64_t T, const int32_t* tv, int64_t V, const float* xyz, const float* vel,
                   const float* scal, int S, const float* dens32, const double* dens64, int K,
                   const dtfe_subbox* boxes, const float* regions, const int32_t grid[3], int NN,
                   uint32_t fields, int fix, int mode, double* const out[DTFE_NUM_FIELDS]) {
  (void)T;
  (void)V;
  auto has = [&](int s) { return (fields & DTFE_FIELD_BIT(s)) != 0 && out[s] != nullptr; };
  if (NN < 1 || has(DTFE_VELOCITY_STD)) return DTFE_ERR_ARG;
  const bool want_grad = has(DTFE_VELOCITY_GRADIENT) || has(DTFE_VELOCITY_DIVERGENCE) ||
                         has(DTFE_VELOCITY_SHEAR) || has(DTFE_VELOCITY_VORTICITY);
  const bool want_sc = S > 0 && scal && (has(DTFE_SCALAR) || has(DTFE_SCALAR_GRADIENT));
  const size_t maxNN = 100 * (size_t)NN, minNN = (size_t)NN / 6 + 1;
  const float minRatio = (float)(1. / 6.);
  std::vector<float> q(3 * maxNN);
  dtfe::sobol_simplex_table(maxNN, q.data());
  const int64_t G1 = grid[1], G2 = grid[2];
  for (int b = 0; b < K; ++b) {
    const dtfe_subbox& B = boxes[b];
    const float* reg = regions + 6 * b;
    const float lo[3] = {reg[0], reg[2], reg[4]}, hi[3] = {reg[1], reg[3], reg[5]};
    const float dx[3] = {B.dx[0], B.dx[1], B.dx[2]};
    const int n[3] = {B.tile_dims[0], B.tile_dims[1], B.tile_dims[2]};
    const int64_t Gb = (int64_t)n[0] * n[1] * n[2];
    const float gcv = dx[0] * dx[1] * dx[2];
    // accumulators of the tile: float (mode 0) or double (mode 1)
    std::vector<float> fD(Gb, 0.f), fV(3 * Gb, 0.f), fG(9 * Gb, 0.f), fS(S * Gb, 0.f), fSG(3 * S * Gb, 0.f);
    std::vector<double> dD(Gb, 0.), dV(3 * Gb, 0.), dG(9 * Gb, 0.), dS(S * Gb, 0.), dSG(3 * S * Gb, 0.);
    for (int64_t t = B.tet_offset; t < B.tet_offset + B.n_tets; ++t) {
      const int32_t* v = &tv[4 * t];
      double X[4][3];
      for (int a = 0; a < 4; ++a)
        for (int c = 0; c < 3; ++c) X[a][c] = (double)xyz[3 * (int64_t)v[a] + c];
      bool outside = false;
      for (int c = 0; c < 3; ++c) {
        const double mn = std::min(std::min(X[0][c], X[1][c]), std::min(X[2][c], X[3][c]));
        const double mx = std::max(std::max(X[0][c], X[1][c]), std::max(X[2][c], X[3][c]));
        outside = outside || mn > (double)hi[c] || mx < (double)lo[c];
      }
      if (outside) continue;
      float bp[3];
      int bc[3];
      float gl[3], gh[3];
      for (int c = 0; c < 3; ++c) {
        bp[c] = (float)(X[0][c] - (double)lo[c]);
        bc[c] = (int)std::floor(bp[c] / dx[c]);
        gl[c] = (float)bc[c] * dx[c] + lo[c];
        gh[c] = gl[c] + dx[c];
      }
      bool one = true;
      for (int a = 1; a < 4 && one; ++a)
        for (int c = 0; c < 3; ++c)
          one = one && X[a][c] >= (double)gl[c] && X[a][c] <= (double)gh[c];
      double vM[3][3];
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) vM[r][c] = X[r + 1][c] - X[0][c];
      const double vol64 = dtfe::orient_det(X[0], X[1], X[2], X[3]) / 6.0;
      const float vol = (float)vol64;
      // gradients (densityGrad, velocityGrad, scalarGrad): float in mode 0
      float Mf[3][3];
      double Md[3][3];
      matrix_inverse<float>(vM, Mf);
      matrix_inverse<double>(vM, Md);
      float d0 = dens32[v[0]], grf[3], VGf[3][3] = {}, SGf[DTFE_MAX_SCALARS][3] = {};
      double e0 = dens64[v[0]], grd[3], VGd[3][3] = {}, SGd[DTFE_MAX_SCALARS][3] = {};
      for (int i = 0; i < 3; ++i) {
        float acc = 0.f;
        double accd = 0.;
        for (int j = 0; j < 3; ++j) {
          acc += Mf[i][j] * (dens32[v[j + 1]] - d0);
          accd += Md[i][j] * (dens64[v[j + 1]] - e0);
        }
        grf[i] = acc;
        grd[i] = accd;
      }
      const float* v0 = vel ? &vel[3 * (int64_t)v[0]] : nullptr;
      if (vel)
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) {
            float acc = 0.f;
            double accd = 0.;
            for (int k = 0; k < 3; ++k) {
              acc += Mf[i][k] * (vel[3 * (int64_t)v[k + 1] + j] - v0[j]);
              accd += Md[i][k] * ((double)vel[3 * (int64_t)v[k + 1] + j] - (double)v0[j]);
            }
            VGf[i][j] = acc;
            VGd[i][j] = accd;
          }
      const float* s0 = want_sc ? &scal[(int64_t)S * v[0]] : nullptr;
      if (want_sc)
        for (int qq = 0; qq < S; ++qq)
          for (int i = 0; i < 3; ++i) {
            float acc = 0.f;
            double accd = 0.;
            for (int k = 0; k < 3; ++k) {
              acc += Mf[i][k] * (scal[(int64_t)S * v[k + 1] + qq] - s0[qq]);
              accd += Md[i][k] * ((double)scal[(int64_t)S * v[k + 1] + qq] - (double)s0[qq]);
            }
            SGf[qq][i] = acc;
            SGd[qq][i] = accd;
          }
      const bool valid_one =
          one && bc[0] >= 0 && bc[0] < n[0] && bc[1] >= 0 && bc[1] < n[1] && bc[2] >= 0 && bc[2] < n[2];
      if (valid_one) {
        const int64_t idx = ((int64_t)bc[0] * n[1] + bc[1]) * n[2] + bc[2];
        if (mode == 0) {
          float a = 0.f;
          for (int i = 0; i < 4; ++i) a += dens32[v[i]];
          fD[idx] += (a / 4.f) * vol;
          if (vel)
            for (int c = 0; c < 3; ++c) {
              float av = 0.f;
              for (int i = 0; i < 4; ++i) av += vel[3 * (int64_t)v[i] + c];
              fV[3 * idx + c] += (av / 4.f) * vol;
            }
          for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i) fG[9 * idx + j * 3 + i] += VGf[i][j] * vol;
          if (want_sc)
            for (int qq = 0; qq < S; ++qq) {
              float as = 0.f;
              for (int i = 0; i < 4; ++i) as += scal[(int64_t)S * v[i] + qq];
              fS[S * idx + qq] += (as / 4.f) * vol;
              for (int i = 0; i < 3; ++i) fSG[3 * S * idx + 3 * qq + i] += SGf[qq][i] * vol;
            }
        } else {
          double a = 0.;
          for (int i = 0; i < 4; ++i) a += dens64[v[i]];
          dD[idx] += a / 4. * vol64;
          if (vel)
            for (int c = 0; c < 3; ++c) {
              double av = 0.;
              for (int i = 0; i < 4; ++i) av += vel[3 * (int64_t)v[i] + c];
              dV[3 * idx + c] += av / 4. * vol64;
            }
          for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i) dG[9 * idx + j * 3 + i] += VGd[i][j] * vol64;
          if (want_sc)
            for (int qq = 0; qq < S; ++qq) {
              double as = 0.;
              for (int i = 0; i < 4; ++i) as += scal[(int64_t)S * v[i] + qq];
              dS[S * idx + qq] += as / 4. * vol64;
              for (int i = 0; i < 3; ++i) dSG[3 * S * idx + 3 * qq + i] += SGd[qq][i] * vol64;
            }
        }
        continue;
      }
      const size_t tempInt = (size_t)((float)NN * vol / gcv) + 1;
      const size_t np = (vol / gcv > minRatio) ? (tempInt > maxNN ? maxNN : tempInt) : minNN;
      const float factor = vol / (float)np;
      const double factor64 = vol64 / (double)np;
      for (size_t i = 0; i < np; ++i) {
        double p[3];
        for (int c = 0; c < 3; ++c)
          p[c] = (double)q[3 * i] * vM[0][c] + (double)q[3 * i + 1] * vM[1][c] + (double)q[3 * i + 2] * vM[2][c];
        int pos[3];
        bool ok = true;
        for (int c = 0; c < 3 && ok; ++c) {
          pos[c] = (int)std::floor(((double)bp[c] + p[c]) / (double)dx[c]);
          ok = pos[c] >= 0 && pos[c] < n[c];
        }
        if (!ok) continue;
        const int64_t idx = ((int64_t)pos[0] * n[1] + pos[1]) * n[2] + pos[2];
        if (mode == 0) {
          const float temp = (float)(p[0] * grf[0] + p[1] * grf[1] + p[2] * grf[2]);
          fD[idx] += (d0 + temp) * factor;
          if (vel)
            for (int c = 0; c < 3; ++c) {
              float tmp = 0.f;
              for (int j = 0; j < 3; ++j)
                tmp = fix ? (float)((double)tmp + (double)VGf[j][c] * p[j]) : (float)((double)VGf[j][c] * p[j]);
              fV[3 * idx + c] += (tmp + v0[c]) * factor;
            }
          for (int j = 0; j < 3; ++j)
            for (int c = 0; c < 3; ++c) fG[9 * idx + j * 3 + c] += VGf[c][j] * factor;
          if (want_sc)
            for (int qq = 0; qq < S; ++qq) {
              float tmp = 0.f;
              for (int j = 0; j < 3; ++j)
                tmp = fix ? (float)((double)tmp + (double)SGf[qq][j] * p[j]) : (float)((double)SGf[qq][j] * p[j]);
              fS[S * idx + qq] += (tmp + s0[qq]) * factor;
              for (int c = 0; c < 3; ++c) fSG[3 * S * idx + 3 * qq + c] += SGf[qq][c] * factor;
            }
        } else {
          dD[idx] += (e0 + p[0] * grd[0] + p[1] * grd[1] + p[2] * grd[2]) * factor64;
          if (vel)
            for (int c = 0; c < 3; ++c) {
              double tmp = 0.;
              if (fix) for (int j = 0; j < 3; ++j) tmp += VGd[j][c] * p[j];
              else tmp = VGd[2][c] * p[2];
              dV[3 * idx + c] += (tmp + (double)v0[c]) * factor64;
            }
          for (int j = 0; j < 3; ++j)
            for (int c = 0; c < 3; ++c) dG[9 * idx + j * 3 + c] += VGd[c][j] * factor64;
          if (want_sc)
            for (int qq = 0; qq < S; ++qq) {
              double tmp = 0.;
              if (fix) for (int j = 0; j < 3; ++j) tmp += SGd[qq][j] * p[j];
              else tmp = SGd[qq][2] * p[2];
              dS[S * idx + qq] += (tmp + (double)s0[qq]) * factor64;
              for (int c = 0; c < 3; ++c) dSG[3 * S * idx + 3 * qq + c] += SGd[qq][c] * factor64;
            }
        }
      }
    }
    // divide by the cell volume and write the tile into the grid
    for (int i = 0; i < n[0]; ++i)
      for (int j = 0; j < n[1]; ++j)
        for (int k = 0; k < n[2]; ++k) {
          const int64_t idx = ((int64_t)i * n[1] + j) * n[2] + k;
          const int64_t cell = ((int64_t)(B.tile_origin[0] + i) * G1 + (B.tile_origin[1] + j)) * G2 +
                               (B.tile_origin[2] + k);
          auto val = [&](const std::vector<float>& f, const std::vector<double>& d, int64_t at) {
            return mode == 0 ? (double)(f[at] / gcv) : d[at] / (double)gcv;
          };
          double g9[9];
          for (int c = 0; c < 9; ++c) g9[c] = val(fG, dG, 9 * idx + c);
          if (has(DTFE_DENSITY)) out[DTFE_DENSITY][cell] = val(fD, dD, idx);
          if (has(DTFE_VELOCITY))
            for (int c = 0; c < 3; ++c) out[DTFE_VELOCITY][3 * cell + c] = val(fV, dV, 3 * idx + c);
          if (has(DTFE_VELOCITY_GRADIENT))
            for (int c = 0; c < 9; ++c) out[DTFE_VELOCITY_GRADIENT][9 * cell + c] = g9[c];
          if (want_grad) {
            double dv, sh[5], vo[3];
            derived(g9, mode, &dv, sh, vo);
            if (has(DTFE_VELOCITY_DIVERGENCE)) out[DTFE_VELOCITY_DIVERGENCE][cell] = dv;
            if (has(DTFE_VELOCITY_SHEAR))
              for (int c = 0; c < 5; ++c) out[DTFE_VELOCITY_SHEAR][5 * cell + c] = sh[c];
            if (has(DTFE_VELOCITY_VORTICITY))
              for (int c = 0; c < 3; ++c) out[DTFE_VELOCITY_VORTICITY][3 * cell + c] = vo[c];
          }
          if (want_sc && has(DTFE_SCALAR))
            for (int qq = 0; qq < S; ++qq) out[DTFE_SCALAR][(int64_t)S * cell + qq] = val(fS, dS, S * idx + qq);
          if (want_sc && has(DTFE_SCALAR_GRADIENT))
            for (int c = 0; c < 3 * S; ++c)
              out[DTFE_SCALAR_GRADIENT][(int64_t)3 * S * cell + c] = val(fSG, dSG, 3 * S * idx + c);
        }
  }
  return DTFE_OK;
}

// The method-1 quasi-random table (3 floats per point).
void oracle_sobol_simplex(int64_t n, float* out) { dtfe::sobol_simplex_table((size_t)n, out); }

}  // extern "C"
