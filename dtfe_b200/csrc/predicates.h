// Exact geometric predicates shared by the host tessellator, the CUDA walk and
// the CPU oracle.
//
// Role in the reference: CGAL's Exact_predicates_inexact_constructions_kernel
// (src/CGAL_triangulation/CGAL_include_3D.h:52) supplies the orientation and
// in-sphere tests behind Delaunay_triangulation_3::insert / locate
// (triangulation.cpp:183, unaveraged_interpolation.cc:289).  CGAL is not a
// dependency here; these are written from the published method of
// J. R. Shewchuk, "Adaptive Precision Floating-Point Arithmetic and Fast
// Robust Geometric Predicates", Discrete Comput. Geom. 18 (1997): evaluate the
// determinant in double precision, accept its sign when |det| exceeds a
// forward error bound times the permanent, otherwise recompute the sign
// exactly with non-overlapping floating-point expansions.
//
// Conventions (same as CGAL's):
//   orient(a,b,c,d) = sign det[b-a; c-a; d-a]; a tetrahedron (v0,v1,v2,v3) is
//   positively oriented when orient(v0,v1,v2,v3) > 0 and its volume is that
//   determinant / 6.
//   insphere(a,b,c,d,e) > 0 when e lies strictly inside the circumsphere of the
//   positively oriented tetrahedron (a,b,c,d).
#pragma once

#include <cmath>
#include <cfloat>

#if defined(__CUDACC__)
#define DTFE_HD __host__ __device__ __forceinline__
#define DTFE_HD_NOINLINE static __host__ __device__ __noinline__
#else
#define DTFE_HD inline
#define DTFE_HD_NOINLINE static inline
#endif

#if !defined(__CUDA_ARCH__)
#include <vector>
#endif

namespace dtfe {

// Unit roundoff of IEEE double.
constexpr double kEps = 1.1102230246251565e-16;  // 2^-53
// Forward error bounds (relative to the permanent) for the double evaluations
// below.  A first-order count of the rounding steps gives 8 eps for orient and
// 17 eps for insphere; the constants carry a safety margin.
constexpr double kOrientErr = 12.0 * kEps;
constexpr double kInsphereErr = 24.0 * kEps;

// ---- error-free transformations -------------------------------------------
DTFE_HD void two_sum(double a, double b, double& x, double& y) {
  x = a + b;
  double bv = x - a;
  double av = x - bv;
  double br = b - bv;
  double ar = a - av;
  y = ar + br;
}

DTFE_HD void two_diff(double a, double b, double& x, double& y) {
  x = a - b;
  double bv = a - x;
  double av = x + bv;
  double br = bv - b;
  double ar = a - av;
  y = ar + br;
}

DTFE_HD void two_prod(double a, double b, double& x, double& y) {
  x = a * b;
  y = fma(a, b, -x);
}

// ---- expansions: arrays of non-overlapping doubles sorted by increasing
// magnitude; zero components are dropped.  The value is the exact sum. --------

// h = e + b.  h must hold m+1 entries.  Returns the length of h.
DTFE_HD int exp_grow(int m, const double* e, double b, double* h) {
  double q = b;
  int n = 0;
  for (int i = 0; i < m; ++i) {
    double s, r;
    two_sum(q, e[i], s, r);
    q = s;
    if (r != 0.0) h[n++] = r;
  }
  if (q != 0.0 || n == 0) h[n++] = q;
  return n;
}

// h = e + f (by repeated growth; quadratic but only used on the rare exact
// path).  h must hold m+n entries, tmp too.
DTFE_HD int exp_sum(int m, const double* e, int n, const double* f, double* h,
                    double* tmp) {
  int len = m;
  for (int i = 0; i < m; ++i) h[i] = e[i];
  for (int j = 0; j < n; ++j) {
    int l2 = exp_grow(len, h, f[j], tmp);
    for (int i = 0; i < l2; ++i) h[i] = tmp[i];
    len = l2;
  }
  return len;
}

// h = e * b.  h must hold 2m entries, tmp too.
DTFE_HD int exp_scale(int m, const double* e, double b, double* h,
                      double* tmp) {
  int len = 0;
  for (int i = 0; i < m; ++i) {
    double p, err;
    two_prod(e[i], b, p, err);
    int l2 = exp_grow(len, h, err, tmp);
    len = exp_grow(l2, tmp, p, h);
  }
  if (len == 0) {
    h[0] = 0.0;
    len = 1;
  }
  return len;
}

DTFE_HD int exp_negate(int m, double* e) {
  for (int i = 0; i < m; ++i) e[i] = -e[i];
  return m;
}

DTFE_HD int exp_sign(int m, const double* e) {
  for (int i = m - 1; i >= 0; --i) {
    if (e[i] > 0.0) return 1;
    if (e[i] < 0.0) return -1;
  }
  return 0;
}

// Product of two 2-component (or shorter) expansions: at most 8 components.
DTFE_HD int exp_mul2(int m, const double* e, int n, const double* f,
                     double* h /*8*/) {
  double s0[4], s1[4], tmp[8];
  int l0 = exp_scale(m, e, f[0], s0, tmp);
  if (n == 1) {
    for (int i = 0; i < l0; ++i) h[i] = s0[i];
    return l0;
  }
  int l1 = exp_scale(m, e, f[1], s1, tmp);
  return exp_sum(l0, s0, l1, s1, h, tmp);
}

// Exact sign of det[b-a; c-a; d-a] with fixed-size buffers (usable on the
// device).  Entries are 2-component expansions of the coordinate differences.
DTFE_HD_NOINLINE int orient_exact(const double* a, const double* b,
                                  const double* c, const double* d) {
  double u[3][2], v[3][2], w[3][2];
  int lu[3], lv[3], lw[3];
  for (int k = 0; k < 3; ++k) {
    double x, y;
    two_diff(b[k], a[k], x, y);
    u[k][0] = y; u[k][1] = x; lu[k] = 2;
    if (y == 0.0) { u[k][0] = x; lu[k] = 1; }
    two_diff(c[k], a[k], x, y);
    v[k][0] = y; v[k][1] = x; lv[k] = 2;
    if (y == 0.0) { v[k][0] = x; lv[k] = 1; }
    two_diff(d[k], a[k], x, y);
    w[k][0] = y; w[k][1] = x; lw[k] = 2;
    if (y == 0.0) { w[k][0] = x; lw[k] = 1; }
  }
  // det = u0 (v1 w2 - v2 w1) + u1 (v2 w0 - v0 w2) + u2 (v0 w1 - v1 w0)
  double acc[192], acc2[192], tmp[192];
  int lacc = 0;
  const int idx[3][2] = {{1, 2}, {2, 0}, {0, 1}};
  for (int r = 0; r < 3; ++r) {
    int i = idx[r][0], j = idx[r][1];
    double p[8], q[8], minor[16], t1[32], t2[32], term[64];
    int lp = exp_mul2(lv[i], v[i], lw[j], w[j], p);
    int lq = exp_mul2(lv[j], v[j], lw[i], w[i], q);
    exp_negate(lq, q);
    int lm = exp_sum(lp, p, lq, q, minor, tmp);
    int l1 = exp_scale(lm, minor, u[r][0], t1, tmp);
    int lt = l1;
    if (lu[r] == 2) {
      int l2 = exp_scale(lm, minor, u[r][1], t2, tmp);
      lt = exp_sum(l1, t1, l2, t2, term, tmp);
    } else {
      for (int k = 0; k < l1; ++k) term[k] = t1[k];
    }
    int ln = exp_sum(lacc, acc, lt, term, acc2, tmp);
    for (int k = 0; k < ln; ++k) acc[k] = acc2[k];
    lacc = ln;
  }
  return exp_sign(lacc, acc);
}

// Filtered orientation: sign of det[b-a; c-a; d-a].
DTFE_HD int orient(const double* a, const double* b, const double* c,
                   const double* d) {
  double bax = b[0] - a[0], bay = b[1] - a[1], baz = b[2] - a[2];
  double cax = c[0] - a[0], cay = c[1] - a[1], caz = c[2] - a[2];
  double dax = d[0] - a[0], day = d[1] - a[1], daz = d[2] - a[2];
  double m0 = cay * daz, m1 = caz * day;
  double m2 = caz * dax, m3 = cax * daz;
  double m4 = cax * day, m5 = cay * dax;
  double det = bax * (m0 - m1) + bay * (m2 - m3) + baz * (m4 - m5);
  double perm = fabs(bax) * (fabs(m0) + fabs(m1)) +
                fabs(bay) * (fabs(m2) + fabs(m3)) +
                fabs(baz) * (fabs(m4) + fabs(m5));
  double bound = kOrientErr * perm;
  if (det > bound) return 1;
  if (-det > bound) return -1;
  return orient_exact(a, b, c, d);
}

// Signed 6x volume of (a,b,c,d) in double (not exact; a construction).
DTFE_HD double orient_det(const double* a, const double* b, const double* c,
                          const double* d) {
  double bax = b[0] - a[0], bay = b[1] - a[1], baz = b[2] - a[2];
  double cax = c[0] - a[0], cay = c[1] - a[1], caz = c[2] - a[2];
  double dax = d[0] - a[0], day = d[1] - a[1], daz = d[2] - a[2];
  return bax * (cay * daz - caz * day) + bay * (caz * dax - cax * daz) +
         baz * (cax * day - cay * dax);
}

#if !defined(__CUDA_ARCH__)
// ---- host-only exact in-sphere with heap expansions -----------------------
struct HExp {
  std::vector<double> c;
  HExp() : c(1, 0.0) {}
  explicit HExp(double x) : c(1, x) {}
  static HExp diff(double a, double b) {
    HExp r;
    double x, y;
    two_diff(a, b, x, y);
    r.c.clear();
    if (y != 0.0) r.c.push_back(y);
    r.c.push_back(x);
    return r;
  }
  int sign() const { return exp_sign((int)c.size(), c.data()); }
};

inline HExp hexp_add(const HExp& e, const HExp& f) {
  HExp r;
  std::vector<double> h(e.c.size() + f.c.size() + 1), t(h.size());
  int n = exp_sum((int)e.c.size(), e.c.data(), (int)f.c.size(), f.c.data(),
                  h.data(), t.data());
  r.c.assign(h.begin(), h.begin() + n);
  return r;
}
inline HExp hexp_neg(const HExp& e) {
  HExp r = e;
  for (double& x : r.c) x = -x;
  return r;
}
inline HExp hexp_sub(const HExp& e, const HExp& f) { return hexp_add(e, hexp_neg(f)); }
inline HExp hexp_mul(const HExp& e, const HExp& f) {
  HExp acc;
  std::vector<double> s(2 * e.c.size() + 2), t(s.size());
  for (double fj : f.c) {
    HExp term;
    int n = exp_scale((int)e.c.size(), e.c.data(), fj, s.data(), t.data());
    term.c.assign(s.begin(), s.begin() + n);
    acc = hexp_add(acc, term);
  }
  return acc;
}

inline HExp hexp_det3(const HExp* u, const HExp* v, const HExp* w) {
  HExp t0 = hexp_mul(u[0], hexp_sub(hexp_mul(v[1], w[2]), hexp_mul(v[2], w[1])));
  HExp t1 = hexp_mul(u[1], hexp_sub(hexp_mul(v[2], w[0]), hexp_mul(v[0], w[2])));
  HExp t2 = hexp_mul(u[2], hexp_sub(hexp_mul(v[0], w[1]), hexp_mul(v[1], w[0])));
  return hexp_add(hexp_add(t0, t1), t2);
}

inline int insphere_exact(const double* a, const double* b, const double* c,
                          const double* d, const double* e) {
  const double* P[4] = {a, b, c, d};
  HExp r[4][3], lift[4];
  for (int i = 0; i < 4; ++i) {
    for (int k = 0; k < 3; ++k) r[i][k] = HExp::diff(P[i][k], e[k]);
    lift[i] = hexp_add(hexp_add(hexp_mul(r[i][0], r[i][0]), hexp_mul(r[i][1], r[i][1])),
                       hexp_mul(r[i][2], r[i][2]));
  }
  // det4 of rows [r_i, lift_i], expanded along the lift column.
  HExp d0 = hexp_det3(r[1], r[2], r[3]);
  HExp d1 = hexp_det3(r[0], r[2], r[3]);
  HExp d2 = hexp_det3(r[0], r[1], r[3]);
  HExp d3 = hexp_det3(r[0], r[1], r[2]);
  HExp det = hexp_add(hexp_add(hexp_neg(hexp_mul(lift[0], d0)), hexp_mul(lift[1], d1)),
                      hexp_add(hexp_neg(hexp_mul(lift[2], d2)), hexp_mul(lift[3], d3)));
  // For a positively oriented tetrahedron an interior point gives det4 < 0.
  return -det.sign();
}

// Filtered in-sphere test.
inline int insphere(const double* a, const double* b, const double* c,
                    const double* d, const double* e) {
  const double* P[4] = {a, b, c, d};
  double r[4][3], lift[4], alift[4];
  for (int i = 0; i < 4; ++i) {
    for (int k = 0; k < 3; ++k) r[i][k] = P[i][k] - e[k];
    lift[i] = r[i][0] * r[i][0] + r[i][1] * r[i][1] + r[i][2] * r[i][2];
    alift[i] = lift[i];
  }
  auto det3 = [](const double* u, const double* v, const double* w, double& perm) {
    double m0 = v[1] * w[2], m1 = v[2] * w[1];
    double m2 = v[2] * w[0], m3 = v[0] * w[2];
    double m4 = v[0] * w[1], m5 = v[1] * w[0];
    perm = fabs(u[0]) * (fabs(m0) + fabs(m1)) + fabs(u[1]) * (fabs(m2) + fabs(m3)) +
           fabs(u[2]) * (fabs(m4) + fabs(m5));
    return u[0] * (m0 - m1) + u[1] * (m2 - m3) + u[2] * (m4 - m5);
  };
  double p0, p1, p2, p3;
  double d0 = det3(r[1], r[2], r[3], p0);
  double d1 = det3(r[0], r[2], r[3], p1);
  double d2 = det3(r[0], r[1], r[3], p2);
  double d3 = det3(r[0], r[1], r[2], p3);
  double det = -lift[0] * d0 + lift[1] * d1 - lift[2] * d2 + lift[3] * d3;
  double perm = alift[0] * p0 + alift[1] * p1 + alift[2] * p2 + alift[3] * p3;
  double bound = kInsphereErr * perm;
  if (det > bound) return -1;
  if (-det > bound) return 1;
  return insphere_exact(a, b, c, d, e);
}
#endif

}  // namespace dtfe
