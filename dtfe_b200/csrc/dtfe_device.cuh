// Device building blocks of the DTFE interpolation path (sm_100a).
//
//  * walk_locate: hinted visibility walk over the flat tetrahedron arrays with
//    filtered FP64 orientation tests and an exact fallback — the device
//    counterpart of CGAL's dt.locate(p, lt, li, lj, hint)
//    (unaveraged_interpolation.cc:289, averaged_interpolation_2.cc:123,145);
//  * canonical_tie: the documented tie rule (lowest tetrahedron id among the
//    tetrahedra whose closure holds p), so the located tetrahedron does not
//    depend on the walk path;
//  * cell_eval: the per-sample field arithmetic of positionMatrix,
//    matrixInverse, densityGrad/Value, velocityGrad/Value, velocityGradient,
//    scalarGrad/Value/Gradient (unaveraged_interpolation.cc:34-173,
//    triangulation_miscellaneous.cc:25,42-96) in the reference's precision
//    pattern: double edge matrix and inverse, rounded to float; float
//    gradients; double products of the float offset.  The translation unit is
//    compiled with -fmad=false so no product is fused into an FMA.
#pragma once

#include <cstdint>
#include "predicates.h"

namespace dtfe {

constexpr int kOutside = -1;
constexpr int kWalkFail = -2;

struct WalkStats {
  int steps;
  int exact;
  int tie;
};

__device__ __forceinline__ void load_posf(const float4* __restrict__ posd, int v, float X[3]) {
  float4 q = __ldg(&posd[v]);
  X[0] = q.x;
  X[1] = q.y;
  X[2] = q.z;
}

__device__ __forceinline__ void load_pos(const float4* __restrict__ posd, int v, double X[3]) {
  float4 q = __ldg(&posd[v]);
  X[0] = (double)q.x;
  X[1] = (double)q.y;
  X[2] = (double)q.z;
}

// Exact sign of orient(tetrahedron with vertex `face` replaced by p).  All
// arguments by value: the caller's arrays stay in registers.
static __device__ __noinline__ int exact_face_sign(float x0, float y0, float z0, float x1, float y1, float z1,
                                            float x2, float y2, float z2, float x3, float y3, float z3,
                                            double px, double py, double pz, int face) {
  double Q[4][3] = {{x0, y0, z0}, {x1, y1, z1}, {x2, y2, z2}, {x3, y3, z3}};
  Q[face][0] = px;
  Q[face][1] = py;
  Q[face][2] = pz;
  return orient_exact(Q[0], Q[1], Q[2], Q[3]);
}

// Sign of one face orientation from a determinant and its permanent; exact
// re-evaluation (orient_exact with the definition's argument order) when the
// filter cannot decide.
__device__ __forceinline__ int filtered_sign(double det, double perm, int face, const float X[4][3],
                                             const double p[3], int& nexact) {
  double b = kOrientErr * perm;
  if (det > b) return 1;
  if (-det > b) return -1;
  ++nexact;
  return exact_face_sign(X[0][0], X[0][1], X[0][2], X[1][0], X[1][1], X[1][2], X[2][0], X[2][1], X[2][2],
                         X[3][0], X[3][1], X[3][2], p[0], p[1], p[2], face);
}

// Face orientations o_i = orient(tetrahedron with vertex i replaced by p) for
// the faces in `need`, evaluated in order 0..3 and stopping at the first
// negative one (returned; -1 if none).  o_0 and o_1 share d2 x d3, o_2 and
// o_3 share d0 x d1 (d_k = X_k - p).  zmask receives the faces through p.
__device__ __forceinline__ int first_exit_face(const float X[4][3], const double p[3], int need,
                                               int& zmask, int& nexact) {
  double d[4][3];
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) d[k][c] = (double)X[k][c] - p[c];
  zmask = 0;
  if (need & 3) {
    double m0 = d[2][1] * d[3][2], m1 = d[2][2] * d[3][1];
    double m2 = d[2][2] * d[3][0], m3 = d[2][0] * d[3][2];
    double m4 = d[2][0] * d[3][1], m5 = d[2][1] * d[3][0];
    double cx = m0 - m1, cy = m2 - m3, cz = m4 - m5;
    double ax = fabs(m0) + fabs(m1), ay = fabs(m2) + fabs(m3), az = fabs(m4) + fabs(m5);
    if (need & 1) {
      double det = d[1][0] * cx + d[1][1] * cy + d[1][2] * cz;
      double perm = fabs(d[1][0]) * ax + fabs(d[1][1]) * ay + fabs(d[1][2]) * az;
      int s = filtered_sign(det, perm, 0, X, p, nexact);
      if (s < 0) return 0;
      if (s == 0) zmask |= 1;
    }
    if (need & 2) {
      double det = -(d[0][0] * cx + d[0][1] * cy + d[0][2] * cz);
      double perm = fabs(d[0][0]) * ax + fabs(d[0][1]) * ay + fabs(d[0][2]) * az;
      int s = filtered_sign(det, perm, 1, X, p, nexact);
      if (s < 0) return 1;
      if (s == 0) zmask |= 2;
    }
  }
  if (need & 12) {
    double m0 = d[0][1] * d[1][2], m1 = d[0][2] * d[1][1];
    double m2 = d[0][2] * d[1][0], m3 = d[0][0] * d[1][2];
    double m4 = d[0][0] * d[1][1], m5 = d[0][1] * d[1][0];
    double cx = m0 - m1, cy = m2 - m3, cz = m4 - m5;
    double ax = fabs(m0) + fabs(m1), ay = fabs(m2) + fabs(m3), az = fabs(m4) + fabs(m5);
    if (need & 4) {
      double det = d[3][0] * cx + d[3][1] * cy + d[3][2] * cz;
      double perm = fabs(d[3][0]) * ax + fabs(d[3][1]) * ay + fabs(d[3][2]) * az;
      int s = filtered_sign(det, perm, 2, X, p, nexact);
      if (s < 0) return 2;
      if (s == 0) zmask |= 4;
    }
    if (need & 8) {
      double det = -(d[2][0] * cx + d[2][1] * cy + d[2][2] * cz);
      double perm = fabs(d[2][0]) * ax + fabs(d[2][1]) * ay + fabs(d[2][2]) * az;
      int s = filtered_sign(det, perm, 3, X, p, nexact);
      if (s < 0) return 3;
      if (s == 0) zmask |= 8;
    }
  }
  return -1;
}

// FP32 stage of the orientation filter for points that are exact floats
// (cell centres, equidistant points).  Same evaluation as first_exit_face in
// single precision; its forward error is below kOrientErr32 times the
// permanent (the FP64 bound's constant applied to the float unit roundoff,
// with a floor against underflow).  Faces the FP32 bound cannot decide are
// re-evaluated by the FP64 filter and, if needed, exactly.
constexpr float kOrientErr32 = 12.0f * 5.9604645e-8f;  // 12 * 2^-24
constexpr float kPermFloor32 = 1e-30f;

// Returns (sign + 1) | (4 if exact arithmetic was needed).
static __device__ __noinline__ int face_sign_fp64(float x0, float y0, float z0, float x1, float y1, float z1,
                                           float x2, float y2, float z2, float x3, float y3, float z3,
                                           double px, double py, double pz, int face) {
  double Q[4][3] = {{x0, y0, z0}, {x1, y1, z1}, {x2, y2, z2}, {x3, y3, z3}};
  Q[face][0] = px;
  Q[face][1] = py;
  Q[face][2] = pz;
  double bax = Q[1][0] - Q[0][0], bay = Q[1][1] - Q[0][1], baz = Q[1][2] - Q[0][2];
  double cax = Q[2][0] - Q[0][0], cay = Q[2][1] - Q[0][1], caz = Q[2][2] - Q[0][2];
  double dax = Q[3][0] - Q[0][0], day = Q[3][1] - Q[0][1], daz = Q[3][2] - Q[0][2];
  double m0 = cay * daz, m1 = caz * day, m2 = caz * dax, m3 = cax * daz, m4 = cax * day, m5 = cay * dax;
  double det = bax * (m0 - m1) + bay * (m2 - m3) + baz * (m4 - m5);
  double perm = fabs(bax) * (fabs(m0) + fabs(m1)) + fabs(bay) * (fabs(m2) + fabs(m3)) +
                fabs(baz) * (fabs(m4) + fabs(m5));
  double b = kOrientErr * perm;
  if (det > b) return 2;
  if (-det > b) return 0;
  return (orient_exact(Q[0], Q[1], Q[2], Q[3]) + 1) | 4;
}

__device__ __forceinline__ int sign32(float det, float perm, int face, const float X[4][3], const float pf[3],
                                      int& nexact) {
  const float b = kOrientErr32 * perm;
  if (perm > kPermFloor32) {
    if (det > b) return 1;
    if (-det > b) return -1;
  }
  const int r = face_sign_fp64(X[0][0], X[0][1], X[0][2], X[1][0], X[1][1], X[1][2], X[2][0], X[2][1],
                               X[2][2], X[3][0], X[3][1], X[3][2], (double)pf[0], (double)pf[1], (double)pf[2],
                               face);
  nexact += r >> 2;
  return (r & 3) - 1;
}

__device__ __forceinline__ int first_exit_face_f32(const float X[4][3], const float pf[3], int need, int& zmask,
                                                   int& nexact) {
  float d[4][3];
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) d[k][c] = X[k][c] - pf[c];
  zmask = 0;
  if (need & 3) {
    float m0 = d[2][1] * d[3][2], m1 = d[2][2] * d[3][1];
    float m2 = d[2][2] * d[3][0], m3 = d[2][0] * d[3][2];
    float m4 = d[2][0] * d[3][1], m5 = d[2][1] * d[3][0];
    float cx = m0 - m1, cy = m2 - m3, cz = m4 - m5;
    float ax = fabsf(m0) + fabsf(m1), ay = fabsf(m2) + fabsf(m3), az = fabsf(m4) + fabsf(m5);
    if (need & 1) {
      float det = d[1][0] * cx + d[1][1] * cy + d[1][2] * cz;
      float perm = fabsf(d[1][0]) * ax + fabsf(d[1][1]) * ay + fabsf(d[1][2]) * az;
      int s = sign32(det, perm, 0, X, pf, nexact);
      if (s < 0) return 0;
      if (s == 0) zmask |= 1;
    }
    if (need & 2) {
      float det = -(d[0][0] * cx + d[0][1] * cy + d[0][2] * cz);
      float perm = fabsf(d[0][0]) * ax + fabsf(d[0][1]) * ay + fabsf(d[0][2]) * az;
      int s = sign32(det, perm, 1, X, pf, nexact);
      if (s < 0) return 1;
      if (s == 0) zmask |= 2;
    }
  }
  if (need & 12) {
    float m0 = d[0][1] * d[1][2], m1 = d[0][2] * d[1][1];
    float m2 = d[0][2] * d[1][0], m3 = d[0][0] * d[1][2];
    float m4 = d[0][0] * d[1][1], m5 = d[0][1] * d[1][0];
    float cx = m0 - m1, cy = m2 - m3, cz = m4 - m5;
    float ax = fabsf(m0) + fabsf(m1), ay = fabsf(m2) + fabsf(m3), az = fabsf(m4) + fabsf(m5);
    if (need & 4) {
      float det = d[3][0] * cx + d[3][1] * cy + d[3][2] * cz;
      float perm = fabsf(d[3][0]) * ax + fabsf(d[3][1]) * ay + fabsf(d[3][2]) * az;
      int s = sign32(det, perm, 2, X, pf, nexact);
      if (s < 0) return 2;
      if (s == 0) zmask |= 4;
    }
    if (need & 8) {
      float det = -(d[2][0] * cx + d[2][1] * cy + d[2][2] * cz);
      float perm = fabsf(d[2][0]) * ax + fabsf(d[2][1]) * ay + fabsf(d[2][2]) * az;
      int s = sign32(det, perm, 3, X, pf, nexact);
      if (s < 0) return 3;
      if (s == 0) zmask |= 8;
    }
  }
  return -1;
}

__device__ __forceinline__ void load_tet(const int4* __restrict__ tet_v, const float4* __restrict__ posd,
                                        int t, int v[4], float X[4][3]) {
  int4 q = __ldg(&tet_v[t]);
  v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
#pragma unroll
  for (int a = 0; a < 4; ++a) load_posf(posd, v[a], X[a]);
}

__device__ __forceinline__ int nb_of(const int4& n, int i) {
  return i == 0 ? n.x : (i == 1 ? n.y : (i == 2 ? n.z : n.w));
}

// True if the closure of tetrahedron t holds p; zmask marks faces through p.
static __device__ __noinline__ bool tet_contains(const int4* __restrict__ tet_v, const float4* __restrict__ posd,
                                          int t, double px, double py, double pz, int& zmask, int& nexact) {
  int v[4];
  float X[4][3];
  load_tet(tet_v, posd, t, v, X);
  const double p[3] = {px, py, pz};
  return first_exit_face(X, p, 15, zmask, nexact) < 0;
}

// Canonical tie rule: the lowest id among the tetrahedra whose closure holds
// p, found by exploring across faces that pass through p.  Bounded: keeps
// the best so far after kTieMax tetrahedra.
constexpr int kTieMax = 96;
static __device__ __noinline__ int canonical_tie(const int4* __restrict__ tet_v, const int4* __restrict__ tet_n,
                                          const float4* __restrict__ posd, int t, int zmask,
                                          double px, double py, double pz) {
  int nexact = 0;  // exact tests inside tie resolution are not counted
  int seen[kTieMax];
  int nseen = 1, head = 0;
  seen[0] = t;
  int best = t;
  int zm = zmask;
  while (head < nseen) {
    int u = seen[head];
    if (head > 0) tet_contains(tet_v, posd, u, px, py, pz, zm, nexact);
    ++head;
    int4 n = __ldg(&tet_n[u]);
    for (int i = 0; i < 4; ++i) {
      if (!(zm & (1 << i))) continue;
      int nb = nb_of(n, i);
      if (nb < 0) continue;
      bool dup = false;
      for (int q = 0; q < nseen; ++q)
        if (seen[q] == nb) { dup = true; break; }
      if (dup) continue;
      int zn;
      if (!tet_contains(tet_v, posd, nb, px, py, pz, zn, nexact)) continue;
      if (nseen >= kTieMax) return best;
      seen[nseen++] = nb;
      if (nb < best) best = nb;
    }
  }
  return best;
}

// Visibility walk from tetrahedron t toward p.  Returns the canonical
// containing tetrahedron, kOutside, or kWalkFail.  On success v/X hold the
// vertices and positions of the returned tetrahedron.  Crossing a face keeps
// the three shared vertices in registers and loads only the new one; the
// face just crossed is not re-tested (p is strictly inside it).
template <bool FLOAT_POINT = false>
__device__ __forceinline__ int walk_locate(const int4* __restrict__ tet_v, const int4* __restrict__ tet_n,
                                           const float4* __restrict__ posd, const double p[3], int t,
                                           int max_steps, int v[4], float X[4][3], WalkStats& st) {
  // FLOAT_POINT: p holds exact float values, so the FP32 filter stage applies
  const float pf[3] = {(float)p[0], (float)p[1], (float)p[2]};
  load_tet(tet_v, posd, t, v, X);
  int came = -1;
  for (int step = 0; step < max_steps; ++step) {
    ++st.steps;
    int need = 15 & ~(came >= 0 ? (1 << came) : 0);
    int zmask;
    int exit_face = FLOAT_POINT ? first_exit_face_f32(X, pf, need, zmask, st.exact)
                                : first_exit_face(X, p, need, zmask, st.exact);
    if (exit_face < 0) {
      if (zmask) {
        ++st.tie;
        int b = canonical_tie(tet_v, tet_n, posd, t, zmask, p[0], p[1], p[2]);
        if (b != t) {
          t = b;
          load_tet(tet_v, posd, t, v, X);
        }
      }
      return t;
    }
    int nb = nb_of(__ldg(&tet_n[t]), exit_face);
    if (nb < 0) return kOutside;
    int4 q = __ldg(&tet_v[nb]);
    int nv[4] = {q.x, q.y, q.z, q.w};
    float NX[4][3];
    came = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      // predicated selection with compile-time indices keeps X in registers
      bool found = false;
#pragma unroll
      for (int c = 0; c < 3; ++c) NX[j][c] = 0.f;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const bool m = (k != exit_face) && (v[k] == nv[j]);
        found = found || m;
#pragma unroll
        for (int c = 0; c < 3; ++c) NX[j][c] = m ? X[k][c] : NX[j][c];
      }
      if (!found) {
        load_posf(posd, nv[j], NX[j]);
        came = j;
      }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      v[j] = nv[j];
#pragma unroll
      for (int c = 0; c < 3; ++c) X[j][c] = NX[j][c];
    }
    t = nb;
  }
  return kWalkFail;
}

// The same walk over interleaved 32-byte tetrahedron records (rec[2t] = the
// vertices, rec[2t+1] = the neighbours of t): a step reads one sector for the
// next tetrahedron's vertices and neighbours together, then the one new
// vertex.  The vertices' densities (posd .w) ride along in D for the
// evaluation.  Same tests in the same order as walk_locate, so the same
// tetrahedron is located (ties resolved by canonical_tie on the plain arrays).
template <bool FLOAT_POINT = false>
__device__ __forceinline__ int walk_locate_rec(const int4* __restrict__ rec, const int4* __restrict__ tet_v,
                                               const int4* __restrict__ tet_n, const float4* __restrict__ posd,
                                               const double p[3], int t, int max_steps, int v[4], float X[4][3],
                                               float D[4], WalkStats& st) {
  const float pf[3] = {(float)p[0], (float)p[1], (float)p[2]};
  int4 q = __ldg(&rec[2 * (int64_t)t]);
  int4 n = __ldg(&rec[2 * (int64_t)t + 1]);
  v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const float4 r = __ldg(&posd[v[a]]);
    X[a][0] = r.x; X[a][1] = r.y; X[a][2] = r.z; D[a] = r.w;
  }
  int came = -1;
  for (int step = 0; step < max_steps; ++step) {
    ++st.steps;
    int need = 15 & ~(came >= 0 ? (1 << came) : 0);
    int zmask;
    int exit_face = FLOAT_POINT ? first_exit_face_f32(X, pf, need, zmask, st.exact)
                                : first_exit_face(X, p, need, zmask, st.exact);
    if (exit_face < 0) {
      if (zmask) {
        ++st.tie;
        int b = canonical_tie(tet_v, tet_n, posd, t, zmask, p[0], p[1], p[2]);
        if (b != t) {
          t = b;
          const int4 qq = __ldg(&rec[2 * (int64_t)t]);
          v[0] = qq.x; v[1] = qq.y; v[2] = qq.z; v[3] = qq.w;
#pragma unroll
          for (int a = 0; a < 4; ++a) {
            const float4 r = __ldg(&posd[v[a]]);
            X[a][0] = r.x; X[a][1] = r.y; X[a][2] = r.z; D[a] = r.w;
          }
        }
      }
      return t;
    }
    const int nb = nb_of(n, exit_face);
    if (nb < 0) return kOutside;
    q = __ldg(&rec[2 * (int64_t)nb]);
    n = __ldg(&rec[2 * (int64_t)nb + 1]);
    int nv[4] = {q.x, q.y, q.z, q.w};
    float NX[4][3], ND[4];
    came = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      bool found = false;
#pragma unroll
      for (int c = 0; c < 3; ++c) NX[j][c] = 0.f;
      ND[j] = 0.f;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const bool m = (k != exit_face) && (v[k] == nv[j]);
        found = found || m;
#pragma unroll
        for (int c = 0; c < 3; ++c) NX[j][c] = m ? X[k][c] : NX[j][c];
        ND[j] = m ? D[k] : ND[j];
      }
      if (!found) {
        const float4 r = __ldg(&posd[nv[j]]);
        NX[j][0] = r.x; NX[j][1] = r.y; NX[j][2] = r.z; ND[j] = r.w;
        came = j;
      }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      v[j] = nv[j];
      D[j] = ND[j];
#pragma unroll
      for (int c = 0; c < 3; ++c) X[j][c] = NX[j][c];
    }
    t = nb;
  }
  return kWalkFail;
}

// ---- per-sample arithmetic (reference precision pattern) -----------------

// minorDeterminant + matrixInverse (triangulation_miscellaneous.cc:42-96).
__device__ __forceinline__ void matrix_inverse_f(const double A[3][3], float M[3][3]) {
#define DTFE_MINOR(row, col)                                                        \
  (A[((col) + 1) % 3][((row) + 1) % 3] * A[((col) + 2) % 3][((row) + 2) % 3] -      \
   A[((col) + 1) % 3][((row) + 2) % 3] * A[((col) + 2) % 3][((row) + 1) % 3])
  double det = A[0][0] * DTFE_MINOR(0, 0) + A[0][1] * DTFE_MINOR(1, 0) + A[0][2] * DTFE_MINOR(2, 0);
  double s = fabs(A[0][0]) + fabs(A[0][1]) + fabs(A[0][2]) + fabs(A[1][0]) + fabs(A[1][1]) +
             fabs(A[1][2]) + fabs(A[2][0]) + fabs(A[2][1]) + fabs(A[2][2]);
  bool ok = fabs(det / s) > 1.e-6;
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) M[r][c] = ok ? (float)(DTFE_MINOR(r, c) / det) : 0.f;
#undef DTFE_MINOR
}

struct CellOut {
  float dens;
  float vel[3];
  float grad[9];
  float sc[8];
  float scg[24];
};

// Evaluates the requested fields of the located tetrahedron at p.
template <int S>
__device__ __forceinline__ void cell_eval(const int v[4], const float X[4][3], const double p[3],
                                          const float4* __restrict__ posd,
                                          const float4* __restrict__ vel4,
                                          const float* __restrict__ scal, bool want_dens,
                                          bool want_vel, bool want_sc, bool fix, CellOut& e,
                                          const float* Dv = nullptr) {
  double A[3][3];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) A[r][c] = (double)X[r + 1][c] - (double)X[0][c];
  float M[3][3];
  matrix_inverse_f(A, M);
  float rel[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) rel[c] = (float)(p[c] - (double)X[0][c]);
  if (want_dens) {
    // vertex densities: carried from the walk (Dv), else read
    float d0 = Dv ? Dv[0] : __ldg(&posd[v[0]]).w;
    float dd[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) dd[i] = (Dv ? Dv[i + 1] : __ldg(&posd[v[i + 1]]).w) - d0;
    float gr[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      float acc = 0.f;
#pragma unroll
      for (int j = 0; j < 3; ++j) acc += M[i][j] * dd[j];
      gr[i] = acc;
    }
    double s = (double)rel[0] * gr[0] + (double)rel[1] * gr[1] + (double)rel[2] * gr[2];
    e.dens = d0 + (float)s;
  }
  if (want_vel) {
    float4 w0 = __ldg(&vel4[v[0]]);
    float v0[3] = {w0.x, w0.y, w0.z};
    float dv[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      float4 wk = __ldg(&vel4[v[k + 1]]);
      dv[k][0] = wk.x - v0[0];
      dv[k][1] = wk.y - v0[1];
      dv[k][2] = wk.z - v0[2];
    }
    float VG[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        float acc = 0.f;
#pragma unroll
        for (int k = 0; k < 3; ++k) acc += M[i][k] * dv[k][j];
        VG[i][j] = acc;
      }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      float tmp = 0.f;
      if (fix) {
#pragma unroll
        for (int j = 0; j < 3; ++j) tmp = (float)((double)tmp + (double)VG[j][i] * (double)rel[j]);
      } else {
        tmp = (float)((double)VG[2][i] * (double)rel[2]);
      }
      e.vel[i] = tmp + v0[i];
    }
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
      for (int i = 0; i < 3; ++i) e.grad[j * 3 + i] = VG[i][j];
  }
  if (S > 0 && want_sc) {
#pragma unroll
    for (int q = 0; q < S; ++q) {
      float s0 = __ldg(&scal[(int64_t)S * v[0] + q]);
      float ds[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) ds[k] = __ldg(&scal[(int64_t)S * v[k + 1] + q]) - s0;
      float SG[3];
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        float acc = 0.f;
#pragma unroll
        for (int k = 0; k < 3; ++k) acc += M[i][k] * ds[k];
        SG[i] = acc;
      }
      float tmp = 0.f;
      if (fix) {
#pragma unroll
        for (int j = 0; j < 3; ++j) tmp = (float)((double)tmp + (double)SG[j] * (double)rel[j]);
      } else {
        tmp = (float)((double)SG[2] * (double)rel[2]);
      }
      e.sc[q] = tmp + s0;
#pragma unroll
      for (int i = 0; i < 3; ++i) e.scg[q * 3 + i] = SG[i];
    }
  }
}

// velocityDivergence / velocityShear / velocityVorticity (src/DTFE.cpp:394-433)
__device__ __forceinline__ void derived_fields(const float g[9], float& div, float sh[5], float vo[3]) {
  div = g[0] + g[4] + g[8];
  int idx = 0;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = i; j < 3; ++j) sh[idx++] = (float)((double)(g[i * 3 + j] + g[j * 3 + i]) / 2.);
  float trace = (float)((double)(sh[0] + sh[3] + g[8]) / 3.);
  sh[0] -= trace;
  sh[3] -= trace;
  idx = 0;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = i + 1; j < 3; ++j) vo[idx++] = (float)((double)(g[i * 3 + j] - g[j * 3 + i]) / 2.);
}

}  // namespace dtfe
