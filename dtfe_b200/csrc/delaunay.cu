// Delaunay tessellation of float32 point sets on B200 (sm_100a): the device
// counterpart of delaunayTriangulation() (src/CGAL_triangulation/
// triangulation.cpp:162-195), with the output of this library's host
// tessellator (delaunay.cpp): finite tetrahedra only, positively oriented,
// each in the lexicographically smallest of its 12 even vertex rotations,
// sorted by the Morton key of the FP64 centroid over the set's bounding box
// and then by the vertex tuple.  For a point set whose Delaunay tessellation
// is unique (no five points on one sphere, no four on one plane among the
// tests that decide it) the arrays equal the host's bit for bit.
//
// Method: star construction.  Every vertex p is handled by one warp, which
//   1. gathers the points of the 5^3 grid cells around p's cell (a uniform
//      grid of about two points per cell) into shared memory: every point
//      closer to p than the block's faces is a candidate;
//   2. starts from p's nearest neighbour q, the candidate r whose triangle
//      pqr has the smallest circumradius (the smallest sphere through p, q, r
//      is then empty) and the apex s that closes pqr to a tetrahedron;
//   3. grows the star of p across the open edges of its link (the triangles
//      opposite p): across edge (u, v) the apex is the point on the far side
//      of plane (p, v, u) whose circumsphere with p, v, u contains no other
//      such point (gift wrapping; the spheres through p, v, u form a pencil
//      ordered by the position of their centre along the face normal);
//   4. certifies every tetrahedron it adds: its circumsphere is empty of all
//      points of the set.  Spheres inside the candidate ball are covered by
//      step 3 itself; larger ones are checked against every point of the grid
//      cells they touch, and a point found inside replaces the apex.  A link
//      edge without any point beyond it (certified over the whole grid) lies
//      on the convex hull;
//   5. emits the tetrahedra of its star whose smallest vertex is p.
// Orientation and in-sphere signs are exact: a double-precision evaluation
// with a forward error bound (the host predicates' constants), else the
// determinant in 384-bit integers over the float32 inputs at a common binary
// scale.  Any exact zero among the deciding tests (co-spherical or coplanar
// points, duplicates), or an exhausted bound (candidate or star capacity,
// repair iterations), marks the set; the caller then tessellates that set on
// the host, whose insertion order breaks such ties.

#include <cuda_runtime.h>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_segmented_radix_sort.cuh>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/dtfe_gpu.h"

extern "C" int dtfe_internal_set_error(int code, const char* msg);

namespace {

// ---- per-set flags (status of dtfe_gpu_tess_sizes) -----------------------
constexpr int kFlagDegenerate = 1;   // a deciding predicate was exactly zero
constexpr int kFlagCapacity = 2;     // candidate or star capacity exceeded
constexpr int kFlagOverflow = 4;     // output region too small
constexpr int kFlagRepair = 8;       // certification did not converge / inconsistent star
constexpr int kFlagUndecided = 16;   // exact path outside the 384-bit budget
constexpr int kFlagInput = 32;       // non-finite coordinates or flat set

constexpr int kWarps = 4;            // warps per block of the star kernel
constexpr int kCandCap = 512;        // candidates per warp
constexpr int kTriCap = 512;         // link triangles per warp
constexpr size_t kStarSmem = (size_t)kWarps * (kCandCap + kTriCap) * 16;  // dynamic shared memory per block

constexpr double kEps = 1.1102230246251565e-16;  // 2^-53
constexpr double kOrientErr = 12.0 * kEps;        // same bounds as the host predicates
constexpr double kInsphereErr = 24.0 * kEps;
constexpr double kCircErr = 64.0 * kEps;          // circumcentre numerator / denominator
constexpr double kInf = 1e300;

struct TSet {
  int64_t v0, n;           // global vertex range
  double lo[3], h, inv_h;  // grid frame (h: cell size)
  int32_t dims[3];
  int64_t cell0;           // first cell in the global cell arrays
  int64_t out0, cap;       // output region (tetrahedra)
  double mlo[3], mscale[3];  // Morton frame of the host tessellator
  double slack;            // absolute margin of cell-membership tests
};

// ---- float decomposition and the exact integer path ----------------------

__device__ __forceinline__ void fdecomp(float v, int& lsb, long long& mant) {
  const unsigned b = __float_as_uint(v);
  const int E = (int)((b >> 23) & 0xffu);
  unsigned m = b & 0x7fffffu;
  if (E == 0) {
    lsb = m ? -149 : 0x7fffffff;
  } else {
    m |= 0x800000u;
    lsb = E - 150;
  }
  mant = (b >> 31) ? -(long long)m : (long long)m;
}

// 384-bit two's-complement integer: enough for the in-sphere determinant of
// 62-bit coordinate differences (|det| < 2^317).
struct W6 {
  unsigned long long w[6];
};

__device__ __forceinline__ W6 w_from(__int128 x) {
  W6 r;
  const unsigned __int128 u = (unsigned __int128)x;
  r.w[0] = (unsigned long long)u;
  r.w[1] = (unsigned long long)(u >> 64);
  const unsigned long long s = x < 0 ? ~0ull : 0ull;
  for (int i = 2; i < 6; ++i) r.w[i] = s;
  return r;
}

__device__ __forceinline__ W6 w_mul(const W6& a, const W6& b) {
  W6 r;
  for (int i = 0; i < 6; ++i) r.w[i] = 0;
  for (int i = 0; i < 6; ++i) {
    unsigned long long carry = 0;
    for (int j = 0; i + j < 6; ++j) {
      const unsigned __int128 t = (unsigned __int128)a.w[i] * b.w[j] + r.w[i + j] + carry;
      r.w[i + j] = (unsigned long long)t;
      carry = (unsigned long long)(t >> 64);
    }
  }
  return r;
}

__device__ __forceinline__ W6 w_add(const W6& a, const W6& b) {
  W6 r;
  unsigned long long carry = 0;
  for (int i = 0; i < 6; ++i) {
    const unsigned __int128 t = (unsigned __int128)a.w[i] + b.w[i] + carry;
    r.w[i] = (unsigned long long)t;
    carry = (unsigned long long)(t >> 64);
  }
  return r;
}

__device__ __forceinline__ W6 w_neg(const W6& a) {
  W6 r;
  unsigned long long carry = 1;
  for (int i = 0; i < 6; ++i) {
    const unsigned __int128 t = (unsigned __int128)(~a.w[i]) + carry;
    r.w[i] = (unsigned long long)t;
    carry = (unsigned long long)(t >> 64);
  }
  return r;
}

__device__ __forceinline__ int w_sign(const W6& a) {
  if (a.w[5] >> 63) return -1;
  for (int i = 0; i < 6; ++i)
    if (a.w[i]) return 1;
  return 0;
}

// det[u; v; w] of integer rows, in 384 bits.
__device__ W6 det3_int(const long long* u, const long long* v, const long long* w) {
  const __int128 m0 = (__int128)v[1] * w[2] - (__int128)v[2] * w[1];
  const __int128 m1 = (__int128)v[2] * w[0] - (__int128)v[0] * w[2];
  const __int128 m2 = (__int128)v[0] * w[1] - (__int128)v[1] * w[0];
  W6 t = w_mul(w_from(u[0]), w_from(m0));
  t = w_add(t, w_mul(w_from(u[1]), w_from(m1)));
  return w_add(t, w_mul(w_from(u[2]), w_from(m2)));
}

// Integer coordinates of m float points relative to point `base`, at the
// finest binary scale of all their coordinates.  False when a difference
// needs more than 62 bits (the determinant budget).
__device__ bool to_int(const float3* q, int m, int base, long long (*d)[3]) {
  int emin = 0x7fffffff, etop = -0x7fffffff;
  for (int i = 0; i < m; ++i) {
    const float c[3] = {q[i].x, q[i].y, q[i].z};
    for (int k = 0; k < 3; ++k) {
      int l;
      long long mt;
      fdecomp(c[k], l, mt);
      if (mt == 0) continue;
      emin = min(emin, l);
      etop = max(etop, l + 24);
    }
  }
  if (emin == 0x7fffffff) {
    for (int i = 0; i < m; ++i) d[i][0] = d[i][1] = d[i][2] = 0;
    return true;
  }
  if (etop - emin > 125) return false;
  const long long lim = 1ll << 62;
  const float cb[3] = {q[base].x, q[base].y, q[base].z};
  for (int i = 0; i < m; ++i) {
    const float c[3] = {q[i].x, q[i].y, q[i].z};
    for (int k = 0; k < 3; ++k) {
      int l0, l1;
      long long m0, m1;
      fdecomp(c[k], l0, m0);
      fdecomp(cb[k], l1, m1);
      const __int128 a = m0 ? (__int128)m0 * ((__int128)1 << (l0 - emin)) : 0;
      const __int128 b = m1 ? (__int128)m1 * ((__int128)1 << (l1 - emin)) : 0;
      const __int128 x = a - b;
      if (x >= lim || x <= -lim) return false;
      d[i][k] = (long long)x;
    }
  }
  return true;
}

// Exact orient sign of (a, b, c, d) = sign det[b-a; c-a; d-a]; 2 when undecidable.
__device__ __noinline__ int orient_exact_f(float3 a, float3 b, float3 c, float3 e) {
  const float3 q[4] = {a, b, c, e};
  long long d[4][3];
  if (!to_int(q, 4, 0, d)) return 2;
  return w_sign(det3_int(d[1], d[2], d[3]));
}

// Exact in-sphere sign (> 0: e strictly inside the circumsphere of the
// positively oriented (a, b, c, d)); 2 when undecidable.
__device__ __noinline__ int insphere_exact_f(float3 a, float3 b, float3 c, float3 dd, float3 e) {
  const float3 q[5] = {a, b, c, dd, e};
  long long r[5][3];
  if (!to_int(q, 5, 4, r)) return 2;
  __int128 lift[4];
  for (int i = 0; i < 4; ++i)
    lift[i] = (__int128)r[i][0] * r[i][0] + (__int128)r[i][1] * r[i][1] + (__int128)r[i][2] * r[i][2];
  const W6 d0 = det3_int(r[1], r[2], r[3]);
  const W6 d1 = det3_int(r[0], r[2], r[3]);
  const W6 d2 = det3_int(r[0], r[1], r[3]);
  const W6 d3 = det3_int(r[0], r[1], r[2]);
  W6 det = w_neg(w_mul(w_from(lift[0]), d0));
  det = w_add(det, w_mul(w_from(lift[1]), d1));
  det = w_add(det, w_neg(w_mul(w_from(lift[2]), d2)));
  det = w_add(det, w_mul(w_from(lift[3]), d3));
  return -w_sign(det);
}

// Filtered orientation (the host's double evaluation and bound).
__device__ __forceinline__ int orient_f(float3 a, float3 b, float3 c, float3 d) {
  const double bax = (double)b.x - a.x, bay = (double)b.y - a.y, baz = (double)b.z - a.z;
  const double cax = (double)c.x - a.x, cay = (double)c.y - a.y, caz = (double)c.z - a.z;
  const double dax = (double)d.x - a.x, day = (double)d.y - a.y, daz = (double)d.z - a.z;
  const double m0 = cay * daz, m1 = caz * day;
  const double m2 = caz * dax, m3 = cax * daz;
  const double m4 = cax * day, m5 = cay * dax;
  const double det = bax * (m0 - m1) + bay * (m2 - m3) + baz * (m4 - m5);
  const double perm = fabs(bax) * (fabs(m0) + fabs(m1)) + fabs(bay) * (fabs(m2) + fabs(m3)) +
                      fabs(baz) * (fabs(m4) + fabs(m5));
  const double bound = kOrientErr * perm;
  if (det > bound) return 1;
  if (-det > bound) return -1;
  return orient_exact_f(a, b, c, d);
}

__device__ __forceinline__ double det3d(const double* u, const double* v, const double* w, double& perm) {
  const double m0 = v[1] * w[2], m1 = v[2] * w[1];
  const double m2 = v[2] * w[0], m3 = v[0] * w[2];
  const double m4 = v[0] * w[1], m5 = v[1] * w[0];
  perm = fabs(u[0]) * (fabs(m0) + fabs(m1)) + fabs(u[1]) * (fabs(m2) + fabs(m3)) +
         fabs(u[2]) * (fabs(m4) + fabs(m5));
  return u[0] * (m0 - m1) + u[1] * (m2 - m3) + u[2] * (m4 - m5);
}

// Filtered in-sphere test (the host's double evaluation and bound).
__device__ __noinline__ int insphere_f(float3 a, float3 b, float3 c, float3 d, float3 e) {
  const float3 P[4] = {a, b, c, d};
  double r[4][3], lift[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    r[i][0] = (double)P[i].x - e.x;
    r[i][1] = (double)P[i].y - e.y;
    r[i][2] = (double)P[i].z - e.z;
    lift[i] = r[i][0] * r[i][0] + r[i][1] * r[i][1] + r[i][2] * r[i][2];
  }
  double p0, p1, p2, p3;
  const double d0 = det3d(r[1], r[2], r[3], p0);
  const double d1 = det3d(r[0], r[2], r[3], p1);
  const double d2 = det3d(r[0], r[1], r[3], p2);
  const double d3 = det3d(r[0], r[1], r[2], p3);
  const double det = -lift[0] * d0 + lift[1] * d1 - lift[2] * d2 + lift[3] * d3;
  const double perm = lift[0] * p0 + lift[1] * p1 + lift[2] * p2 + lift[3] * p3;
  const double bound = kInsphereErr * perm;
  if (det > bound) return -1;
  if (-det > bound) return 1;
  return insphere_exact_f(a, b, c, d, e);
}

// Circumsphere of (p, a, b, c) in double with a bound on the centre's error:
// the centre is p + N / D with N = |A|^2 (B x C) + |B|^2 (C x A) + |C|^2 (A x B)
// and D = 2 A.(B x C) (A = a - p, ...); both carry at most kCircErr times
// the sums of their terms' magnitudes.  |centre - true centre| <= err and
// |r - true radius| <= err.  ok is false when D is not resolved.
struct Sphere {
  double c[3], r, err;
  bool ok;
};

__device__ Sphere circum(float3 p, float3 a, float3 b, float3 c) {
  Sphere S;
  const double A[3] = {(double)a.x - p.x, (double)a.y - p.y, (double)a.z - p.z};
  const double B[3] = {(double)b.x - p.x, (double)b.y - p.y, (double)b.z - p.z};
  const double C[3] = {(double)c.x - p.x, (double)c.y - p.y, (double)c.z - p.z};
  const double la = A[0] * A[0] + A[1] * A[1] + A[2] * A[2];
  const double lb = B[0] * B[0] + B[1] * B[1] + B[2] * B[2];
  const double lc = C[0] * C[0] + C[1] * C[1] + C[2] * C[2];
  double N[3], Np[3], bc[3], bca[3];
  double D = 0.0, Dp = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int i = (k + 1) % 3, j = (k + 2) % 3;
    const double x1 = B[i] * C[j], x2 = B[j] * C[i];
    const double y1 = C[i] * A[j], y2 = C[j] * A[i];
    const double z1 = A[i] * B[j], z2 = A[j] * B[i];
    bc[k] = x1 - x2;
    bca[k] = fabs(x1) + fabs(x2);
    N[k] = la * bc[k] + lb * (y1 - y2) + lc * (z1 - z2);
    Np[k] = la * bca[k] + lb * (fabs(y1) + fabs(y2)) + lc * (fabs(z1) + fabs(z2));
    D += A[k] * bc[k];
    Dp += fabs(A[k]) * bca[k];
  }
  D *= 2.0;
  Dp *= 2.0;
  const double dN = kCircErr * sqrt(Np[0] * Np[0] + Np[1] * Np[1] + Np[2] * Np[2]);
  const double dD = kCircErr * Dp;
  if (!(fabs(D) > 2.0 * dD)) {
    S.ok = false;
    S.c[0] = p.x; S.c[1] = p.y; S.c[2] = p.z;
    S.r = kInf;
    S.err = kInf;
    return S;
  }
  const double o[3] = {N[0] / D, N[1] / D, N[2] / D};
  S.r = sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
  S.c[0] = p.x + o[0];
  S.c[1] = p.y + o[1];
  S.c[2] = p.z + o[2];
  const double pm = fmax(fabs((double)p.x), fmax(fabs((double)p.y), fabs((double)p.z)));
  S.err = (2.0 * dN + S.r * dD) / (fabs(D) - dD) * (1.0 + 1e-6) + 8.0 * kEps * (S.r + pm);
  S.ok = true;
  return S;
}

// x strictly outside the true sphere (sufficient test).
__device__ __forceinline__ bool sph_outside(const Sphere& S, float3 x) {
  const double dx = (double)x.x - S.c[0], dy = (double)x.y - S.c[1], dz = (double)x.z - S.c[2];
  const double rr = S.r + 2.0 * S.err;
  return dx * dx + dy * dy + dz * dz > rr * rr * (1.0 + 1e-9);
}

// Bounded box of a grid cell: interior cells are [lo + i h, lo + (i+1) h];
// the first and last cells reach the set's bounding box (points beyond the
// last full cell are clamped into it); every side widened by the slack.
__device__ __forceinline__ void cell_box(const TSet& S, const double* hi, int i, int a, double& b0, double& b1) {
  b0 = i == 0 ? S.lo[a] : S.lo[a] + i * S.h;
  b1 = i == S.dims[a] - 1 ? hi[a] : S.lo[a] + (i + 1) * S.h;
  b0 -= S.slack;
  b1 += S.slack;
}

__device__ __forceinline__ int cell_coord(const TSet& S, double x, int a) {
  const double t = floor((x - S.lo[a]) * S.inv_h);
  if (!(t >= 0.0)) return 0;  // below the grid, or NaN
  return t > (double)(S.dims[a] - 1) ? S.dims[a] - 1 : (int)t;
}

__device__ __forceinline__ float3 f3(float4 v) { return make_float3(v.x, v.y, v.z); }

// Per-warp context of one star.
struct Ctx {
  const TSet* S;
  const float* xyz;            // all vertices, 3 floats each
  double hi[3];
  const int32_t* cell_start;   // global
  const float4* sorted;
  const float4* cand;          // this warp's candidates (shared)
  int ncand;
  int p;
  float3 P;
  double R;                    // every point within R of p is a candidate
  int lane;
  int bad;                     // flag bits (warp-uniform after reductions)
  unsigned long long* stats;   // per failure reason: stars that met it
};

__device__ __forceinline__ unsigned ballot(bool x) { return __ballot_sync(0xffffffffu, x); }

// Failure reasons counted in the statistics of dtfe_gpu_tess_stats.
enum {
  kWhyDuplicate = 0, kWhyCandidates, kWhyStar, kWhyNoStart, kWhyFlat, kWhyUndecided, kWhyTie, kWhyNotDelaunay,
  kWhyLink, kWhyOpen, kWhyOverflow, kWhyRun, kWhyCount
};
// stats[kWhyCount]: 1 + the first failing vertex, stats[kWhyCount + 1] its reason
constexpr int kStatsLen = kWhyCount + 2;

// Marks the star as failed (warp-uniform call).
__device__ __forceinline__ void fail(Ctx& C, int flag, int why) {
  C.bad |= flag;
  if (C.lane == 0) {
    atomicAdd(&C.stats[why], 1ull);
    if (atomicCAS(&C.stats[kWhyCount], 0ull, (unsigned long long)C.p + 1ull) == 0ull)
      C.stats[kWhyCount + 1] = (unsigned long long)why;
  }
}

__device__ __forceinline__ float3 point(const Ctx& C, int id) {
  const float* q = C.xyz + 3 * (int64_t)id;
  return make_float3(__ldg(q), __ldg(q + 1), __ldg(q + 2));
}

// A face (p, u, v) with its normal n = (u - p) x (v - p) in double and the
// magnitudes of n's two products per component: orient(p, u, v, x) is the
// sign of (x - p).n, filtered with the host's orientation bound (the same
// determinant expanded along x's row) and exact otherwise.
struct Face {
  float3 Pf, Uf, Vf;
  double P[3], n[3], na[3];
};

__device__ __forceinline__ Face make_face(float3 P, float3 U, float3 V) {
  Face F;
  F.Pf = P;
  F.Uf = U;
  F.Vf = V;
  F.P[0] = P.x; F.P[1] = P.y; F.P[2] = P.z;
  const double b[3] = {(double)U.x - P.x, (double)U.y - P.y, (double)U.z - P.z};
  const double c[3] = {(double)V.x - P.x, (double)V.y - P.y, (double)V.z - P.z};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int i = (k + 1) % 3, j = (k + 2) % 3;
    const double m1 = b[i] * c[j], m2 = b[j] * c[i];
    F.n[k] = m1 - m2;
    F.na[k] = fabs(m1) + fabs(m2);
  }
  return F;
}

__device__ __forceinline__ int orient_face(const Face& F, float3 X) {
  const double d0 = (double)X.x - F.P[0], d1 = (double)X.y - F.P[1], d2 = (double)X.z - F.P[2];
  const double det = d0 * F.n[0] + d1 * F.n[1] + d2 * F.n[2];
  const double perm = fabs(d0) * F.na[0] + fabs(d1) * F.na[1] + fabs(d2) * F.na[2];
  const double bound = kOrientErr * perm;
  if (det > bound) return 1;
  if (-det > bound) return -1;
  return orient_exact_f(F.Pf, F.Uf, F.Vf, X);
}

// In-sphere sign of x for the positively oriented (p, u, v, b) whose sphere
// is S: decided by the distance to the bounded centre when x is clearly in
// or out, else by the determinant.
__device__ __forceinline__ int insphere_face(const Face& F, float3 B, const Sphere& S, float3 X) {
  if (S.ok) {
    const double dx = (double)X.x - S.c[0], dy = (double)X.y - S.c[1], dz = (double)X.z - S.c[2];
    const double d2 = dx * dx + dy * dy + dz * dz;
    const double hi = S.r + 2.0 * S.err;
    if (d2 > hi * hi * (1.0 + 1e-9)) return -1;
    const double lo = S.r - 2.0 * S.err;
    if (lo > 0.0 && d2 < lo * lo * (1.0 - 1e-9)) return 1;
  }
  return insphere_f(F.Pf, F.Uf, F.Vf, B, X);
}

// Among the lanes' apex candidates for face F (best >= 0 on a lane, sphere
// sb), the one whose sphere holds none of the others: the apices are ordered
// by the position of their sphere centre along the face normal (smaller =
// better); overlapping error intervals are resolved with the exact in-sphere
// sign (an exact tie keeps the current winner: the verification of the
// winner's sphere reports it).  Returns the id (coordinates in W), -1 when no
// lane has one, -2 on failure (flag set).
__device__ __noinline__ int warp_select(Ctx& C, const Face& F, int best, float3 Bx, const Sphere& sb, float3& W) {
  double lo = kInf, hi = kInf;
  if (best >= 0) {
    if (sb.ok) {
      const double d[3] = {sb.c[0] - F.P[0], sb.c[1] - F.P[1], sb.c[2] - F.P[2]};
      const double lam = F.n[0] * d[0] + F.n[1] * d[1] + F.n[2] * d[2];
      const double nn = sqrt(F.n[0] * F.n[0] + F.n[1] * F.n[1] + F.n[2] * F.n[2]);
      const double e = (nn * sb.err + 4.0 * kEps * (fabs(F.n[0] * d[0]) + fabs(F.n[1] * d[1]) + fabs(F.n[2] * d[2]))) *
                       (1.0 + 1e-6);
      lo = lam - e;
      hi = lam + e;
    } else {
      lo = -kInf;
      hi = kInf * 0.5;  // below the empty lanes' kInf
    }
  }
  if (!ballot(best >= 0)) return -1;
  double mh = hi;
  int ml = C.lane;
  for (int off = 16; off; off >>= 1) {
    const double oh = __shfl_xor_sync(0xffffffffu, mh, off);
    const int ol = __shfl_xor_sync(0xffffffffu, ml, off);
    if (oh < mh || (oh == mh && ol < ml)) { mh = oh; ml = ol; }
  }
  int w = __shfl_sync(0xffffffffu, best, ml);
  W.x = __shfl_sync(0xffffffffu, Bx.x, ml);
  W.y = __shfl_sync(0xffffffffu, Bx.y, ml);
  W.z = __shfl_sync(0xffffffffu, Bx.z, ml);
  for (unsigned amb = ballot(best >= 0 && C.lane != ml && lo <= mh); amb; amb &= amb - 1) {
    const int l = __ffs(amb) - 1;
    const int id = __shfl_sync(0xffffffffu, best, l);
    float3 X;
    X.x = __shfl_sync(0xffffffffu, Bx.x, l);
    X.y = __shfl_sync(0xffffffffu, Bx.y, l);
    X.z = __shfl_sync(0xffffffffu, Bx.z, l);
    const int s = insphere_f(F.Pf, F.Uf, F.Vf, W, X);
    if (s == 2) {
      fail(C, kFlagUndecided, kWhyUndecided);
      return -2;
    }
    if (s > 0) { w = id; W = X; }
  }
  return w;
}

// Scan of the grid cells touched by the sphere Sp of the positively oriented
// (p, u, v, w).  Returns the best point beyond the face strictly inside the
// sphere (the apex over the whole set: every point beyond the face with a
// smaller sphere lies in this one; coordinates in Wb), -1 when the sphere
// holds no point (w is certified), -2 on failure: a point exactly on the
// sphere of a certified w (a tie), a point inside it not beyond the face, or
// an undecidable test (flag set).
__device__ __noinline__ int sphere_scan(Ctx& C, const Face& F, int u, int v, int w, float3 W, const Sphere& Sp,
                                        float3& Wb) {
  const TSet& S = *C.S;
  const double rad = Sp.r + 2.0 * Sp.err + S.slack;
  int c0[3], n[3];
  for (int a = 0; a < 3; ++a) {
    const int l = cell_coord(S, Sp.c[a] - rad, a), h = cell_coord(S, Sp.c[a] + rad, a);
    c0[a] = l;
    n[a] = h - l + 1;
  }
  const long long total = (long long)n[0] * n[1] * n[2];
  int best = -1, flag = 0, why = 0;
  bool on_w = false;
  float3 Bx = C.P;
  Sphere sb;
  sb.ok = false;
  for (long long t = C.lane; t < total; t += 32) {
    const int k = (int)(t % n[2]);
    const int j = (int)((t / n[2]) % n[1]);
    const int i = (int)(t / ((long long)n[1] * n[2]));
    const int ci[3] = {c0[0] + i, c0[1] + j, c0[2] + k};
    double d2 = 0.0;
    for (int a = 0; a < 3; ++a) {
      double b0, b1;
      cell_box(S, C.hi, ci[a], a, b0, b1);
      const double q = Sp.c[a] < b0 ? b0 - Sp.c[a] : (Sp.c[a] > b1 ? Sp.c[a] - b1 : 0.0);
      d2 += q * q;
    }
    if (d2 > rad * rad * (1.0 + 1e-9)) continue;
    const int64_t g = S.cell0 + ((int64_t)ci[0] * S.dims[1] + ci[1]) * S.dims[2] + ci[2];
    const int e0 = __ldg(&C.cell_start[g]), e1 = __ldg(&C.cell_start[g + 1]);
    for (int e = e0; e < e1 && !flag; ++e) {
      const float4 x4 = __ldg(&C.sorted[e]);
      const int id = __float_as_int(x4.w);
      if (id == C.p || id == u || id == v || id == w) continue;
      const float3 X = f3(x4);
      const int s0 = insphere_face(F, W, Sp, X);
      if (s0 == 2) { flag = kFlagUndecided; why = kWhyUndecided; break; }
      if (s0 == 0) { on_w = true; continue; }
      if (s0 < 0) continue;
      if (best >= 0 && insphere_face(F, Bx, sb, X) <= 0) continue;  // not better than this lane's best
      const int o = orient_face(F, X);
      if (o != 1) {
        flag = o == 2 ? kFlagUndecided : kFlagRepair;
        why = o == 2 ? kWhyUndecided : kWhyNotDelaunay;
        break;
      }
      best = id; Bx = X; sb = circum(C.P, F.Uf, F.Vf, X);
    }
    if (flag) break;
  }
  const unsigned fb = ballot(flag != 0);
  if (fb) {
    const int l = __ffs(fb) - 1;
    fail(C, __shfl_sync(0xffffffffu, flag, l), __shfl_sync(0xffffffffu, why, l));
    return -2;
  }
  const int r = warp_select(C, F, best, Bx, sb, Wb);
  if (r == -1 && ballot(on_w)) {  // w stays, and its sphere passes through another point
    fail(C, kFlagDegenerate, kWhyTie);
    return -2;
  }
  return r;
}

// Any point strictly beyond the plane of (p, u, v) (orient(p, u, v, x) > 0)
// over the whole grid: its id, -1 if none (a convex-hull face), -2 on a
// point of the plane on or inside the face's circumcircle, or an undecidable
// test (flag set).  (p, v, u, c) is the certified tetrahedron on the other
// side of the face (c < 0: none yet; every point of the plane then fails).
__device__ __noinline__ int halfspace_scan(Ctx& C, int u, float3 U, int v, float3 V, int c, float3 Cc) {
  const TSet& S = *C.S;
  const double A[3] = {(double)U.x - C.P.x, (double)U.y - C.P.y, (double)U.z - C.P.z};
  const double B[3] = {(double)V.x - C.P.x, (double)V.y - C.P.y, (double)V.z - C.P.z};
  const double nv[3] = {A[1] * B[2] - A[2] * B[1], A[2] * B[0] - A[0] * B[2], A[0] * B[1] - A[1] * B[0]};
  const double Pd[3] = {C.P.x, C.P.y, C.P.z};
  // slack on n.(x - p): rounding of n and of the products
  const double nn = fabs(nv[0]) + fabs(nv[1]) + fabs(nv[2]);
  const double ab = (fabs(A[0]) + fabs(A[1]) + fabs(A[2])) * (fabs(B[0]) + fabs(B[1]) + fabs(B[2]));
  const long long total = (long long)S.dims[0] * S.dims[1] * S.dims[2];
  int found = -1, flag = 0;
  for (long long t0 = 0; t0 < total; t0 += 32) {
    const long long t = t0 + C.lane;
    if (t < total) {
      const int k = (int)(t % S.dims[2]);
      const int j = (int)((t / S.dims[2]) % S.dims[1]);
      const int i = (int)(t / ((long long)S.dims[1] * S.dims[2]));
      const int ci[3] = {i, j, k};
      double m = 0.0, ext = 0.0;
      for (int a = 0; a < 3; ++a) {
        double b0, b1;
        cell_box(S, C.hi, ci[a], a, b0, b1);
        const double x = nv[a] > 0.0 ? b1 : b0;
        m += nv[a] * (x - Pd[a]);
        ext += fabs(x - Pd[a]);
      }
      if (m > -(1e-9 * (nn + ab) * ext + 1e-300)) {
        const int64_t g = S.cell0 + ((int64_t)i * S.dims[1] + j) * S.dims[2] + k;
        const int e0 = __ldg(&C.cell_start[g]), e1 = __ldg(&C.cell_start[g + 1]);
        for (int e = e0; e < e1 && found < 0 && !flag; ++e) {
          const float4 x4 = __ldg(&C.sorted[e]);
          const int id = __float_as_int(x4.w);
          if (id == C.p || id == u || id == v) continue;
          const float3 X = f3(x4);
          const int o = orient_f(C.P, U, V, X);
          if (o == 2) flag = kFlagUndecided;
          else if (o > 0) found = id;
          else if (o == 0) {
            // on the face's plane: harmless outside the face's circumcircle,
            // which is where the certified sphere across the face meets it
            const int s = c >= 0 ? insphere_f(C.P, V, U, Cc, X) : 0;
            if (s == 2) flag = kFlagUndecided;
            else if (s >= 0) flag = kFlagDegenerate;
          }
        }
      }
    }
    if (ballot(found >= 0 || flag != 0)) break;
  }
  const unsigned fb = ballot(flag != 0);
  if (fb) {
    const int f = __shfl_sync(0xffffffffu, flag, __ffs(fb) - 1);
    fail(C, f, f == kFlagUndecided ? kWhyUndecided : kWhyTie);
    return -2;
  }
  const unsigned hb = ballot(found >= 0);
  if (!hb) return -1;
  return __shfl_sync(0xffffffffu, found, __ffs(hb) - 1);
}

// Apex across the face (p, u, v): the point w with orient(p, u, v, w) > 0
// whose circumsphere with p, u, v holds no point of the set (face (p, u, v)
// being a Delaunay face).  Returns w >= 0 (coordinates in W), -1 when no
// point lies beyond the face (a hull face), -2 on failure (flag set).
// (p, v, u, c) is the certified tetrahedron on the other side (c < 0: none).
// full: certify against the grid even when the sphere fits the candidate ball.
__device__ __noinline__ int wrap(Ctx& C, int u, float3 U, int v, float3 V, int c, float3 Cc, bool full, float3& W) {
  const Face F = make_face(C.P, U, V);
  int best = -1, flag = 0;
  float3 Bx = C.P;
  Sphere sb;
  sb.ok = false;
  // gift wrapping over the candidates: each lane keeps the best of its share
  for (int j = C.lane; j < C.ncand; j += 32) {
    const float4 c4 = C.cand[j];
    const int id = __float_as_int(c4.w);
    if (id == C.p || id == u || id == v) continue;
    const float3 X = f3(c4);
    if (best >= 0) {
      const int si = insphere_face(F, Bx, sb, X);
      if (si == 2) { flag = kFlagUndecided; continue; }
      if (si <= 0) continue;
    }
    const int o = orient_face(F, X);
    if (o == 2) { flag = kFlagUndecided; continue; }
    if (o <= 0) continue;
    best = id; Bx = X; sb = circum(C.P, U, V, X);
  }
  if (ballot(flag != 0)) {
    fail(C, kFlagUndecided, kWhyUndecided);
    return -2;
  }
  int w = warp_select(C, F, best, Bx, sb, W);
  if (w == -2) return -2;
  bool from_cands = true;
  if (w < 0) {
    w = halfspace_scan(C, u, U, v, V, c, Cc);
    if (w < 0) return w;  // -1: hull face; -2: failure
    W = point(C, w);
    from_cands = false;
  }
  for (int it = 0; it < 4; ++it) {
    const Sphere Sp = circum(C.P, U, V, W);
    if (!Sp.ok) {
      fail(C, kFlagUndecided, kWhyUndecided);
      return -2;
    }
    if (!full && from_cands && 2.0 * (Sp.r + Sp.err) * (1.0 + 1e-9) < C.R) {
      // the sphere lies in the candidate ball: verify it against every
      // candidate (a point on it is a tie; one inside cannot occur)
      int bad = 0;
      for (int j = C.lane; j < C.ncand; j += 32) {
        const float4 c4 = C.cand[j];
        const int id = __float_as_int(c4.w);
        if (id == C.p || id == u || id == v || id == w) continue;
        const int si = insphere_face(F, W, Sp, f3(c4));
        if (si == 2) bad |= 1;
        else if (si == 0) bad |= 2;
        else if (si > 0) bad |= 4;
      }
      const unsigned b1 = ballot(bad & 1), b2 = ballot(bad & 2), b4 = ballot(bad & 4);
      if (b1 | b2 | b4) {
        if (b1) fail(C, kFlagUndecided, kWhyUndecided);
        else if (b4) fail(C, kFlagRepair, kWhyNotDelaunay);
        else fail(C, kFlagDegenerate, kWhyTie);
        return -2;
      }
      return w;
    }
    float3 Y;
    const int y = sphere_scan(C, F, u, v, w, W, Sp, Y);
    if (y == -2) return -2;
    if (y < 0) return w;
    w = y;
    W = Y;
    from_cands = false;
  }
  fail(C, kFlagRepair, kWhyNotDelaunay);
  return -2;
}

struct StarArgs {
  const float* xyz;
  const TSet* sets;
  const int64_t* vprefix;   // K+1
  const double* hi;         // 3 per set: bounding-box maxima
  int K;
  int64_t V;
  const int32_t* cell_start;
  const float4* sorted;
  const int32_t* pcell;     // per vertex: cell within its set's grid
  int4* out;
  unsigned long long* counts;
  int* flags;
  unsigned long long* next;
  unsigned long long* stats;
};

__device__ __forceinline__ int find_set(const int64_t* pre, int K, int64_t v) {
  int lo = 0, hi = K;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(&pre[mid]) <= v) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Edge k of link triangle (a, b, c): (a, b), (b, c), (c, a).
__device__ __forceinline__ void tri_edge(const int4& T, int k, int& x, int& y) {
  x = k == 0 ? T.x : (k == 1 ? T.y : T.z);
  y = k == 0 ? T.y : (k == 1 ? T.z : T.x);
}

// Points in the (2 rr + 1)^3 cells around ci (clipped to the grid).
__device__ int block_count(const TSet& S, const int32_t* cell_start, const int* ci, int rr, int lane, int* c0,
                           int* nc) {
  for (int a = 0; a < 3; ++a) {
    c0[a] = max(0, ci[a] - rr);
    nc[a] = min(S.dims[a] - 1, ci[a] + rr) - c0[a] + 1;
  }
  const int total = nc[0] * nc[1] * nc[2];
  int cnt = 0;
  for (int t = lane; t < total; t += 32) {
    const int k = t % nc[2], j = (t / nc[2]) % nc[1], i = t / (nc[1] * nc[2]);
    const int64_t g = S.cell0 + ((int64_t)(c0[0] + i) * S.dims[1] + (c0[1] + j)) * S.dims[2] + (c0[2] + k);
    cnt += __ldg(&cell_start[g + 1]) - __ldg(&cell_start[g]);
  }
  return __reduce_add_sync(0xffffffffu, cnt);
}

// Points of the block c0 + [0, nc) strictly closer to P than sqrt(d2max).
__device__ int block_count_within(const TSet& S, const int32_t* cell_start, const float4* sorted, const int* c0,
                                  const int* nc, int lane, float3 P, double d2max) {
  const int total = nc[0] * nc[1] * nc[2];
  int cnt = 0;
  for (int t = lane; t < total; t += 32) {
    const int k = t % nc[2], j = (t / nc[2]) % nc[1], i = t / (nc[1] * nc[2]);
    const int64_t g = S.cell0 + ((int64_t)(c0[0] + i) * S.dims[1] + (c0[1] + j)) * S.dims[2] + (c0[2] + k);
    const int e1 = __ldg(&cell_start[g + 1]);
    for (int e = __ldg(&cell_start[g]); e < e1; ++e) {
      const float4 x4 = __ldg(&sorted[e]);
      const double dx = (double)x4.x - P.x, dy = (double)x4.y - P.y, dz = (double)x4.z - P.z;
      cnt += dx * dx + dy * dy + dz * dz < d2max;
    }
  }
  return __reduce_add_sync(0xffffffffu, cnt);
}

// One warp per vertex p: p's Delaunay star, certified; emits the tetrahedra
// whose smallest vertex is p.  Work is fetched from a global counter so that
// slow stars (near the convex hull) do not hold up a fixed share of vertices.
__global__ void __launch_bounds__(kWarps * 32, 3) k_tess_stars(StarArgs A) {
  extern __shared__ float4 s_dyn[];
  __shared__ int s_fill[kWarps];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float4* cand = s_dyn + (size_t)wid * kCandCap;
  int4* tri = reinterpret_cast<int4*>(s_dyn + (size_t)kWarps * kCandCap) + (size_t)wid * kTriCap;
  for (;;) {
    unsigned long long pi = 0;
    if (lane == 0) pi = atomicAdd(A.next, 1ull);
    pi = __shfl_sync(0xffffffffu, pi, 0);
    if (pi >= (unsigned long long)A.V) break;
    const int p = (int)pi;
    const int s = find_set(A.vprefix, A.K, p);
    int fl = 0;
    if (lane == 0) fl = *(volatile int*)&A.flags[s];
    if (__shfl_sync(0xffffffffu, fl, 0) & (kFlagInput | kFlagOverflow)) continue;
    const TSet& S = A.sets[s];
    Ctx C;
    C.S = &S;
    C.xyz = A.xyz;
    C.cell_start = A.cell_start;
    C.sorted = A.sorted;
    C.cand = cand;
    C.p = p;
    C.lane = lane;
    C.bad = 0;
    C.stats = A.stats;
    for (int a = 0; a < 3; ++a) C.hi[a] = A.hi[3 * s + a];
    C.P = point(C, p);
    // ---- candidates: the 5^3 (else 3^3) cells around p's cell
    const int lid = __ldg(&A.pcell[p]);
    const int ci[3] = {lid / (S.dims[1] * S.dims[2]), (lid / S.dims[2]) % S.dims[1], lid % S.dims[2]};
    int rr = 2, c0[3], nc[3];
    int cnt = block_count(S, A.cell_start, ci, rr, lane, c0, nc);
    double rho2 = -1.0;  // >= 0: candidates limited to squared distance < rho2
    if (cnt > kCandCap) {
      rr = 1;
      cnt = block_count(S, A.cell_start, ci, rr, lane, c0, nc);
      if (cnt > kCandCap) {
        // dense cluster: the largest radius (bisection on its square) within
        // which the 3^3 block holds at most kCandCap points
        double lo2 = 0.0, hi2 = 0.0;
        const double Pd[3] = {C.P.x, C.P.y, C.P.z};
        for (int a = 0; a < 3; ++a) {
          double b0, b1, e0, e1;
          cell_box(S, C.hi, c0[a], a, b0, b1);
          cell_box(S, C.hi, c0[a] + nc[a] - 1, a, e0, e1);
          const double m = fmax(Pd[a] - b0, e1 - Pd[a]);
          hi2 += m * m;
        }
        for (int it = 0; it < 32; ++it) {
          const double mid = 0.5 * (lo2 + hi2);
          if (block_count_within(S, A.cell_start, A.sorted, c0, nc, lane, C.P, mid) <= kCandCap) lo2 = mid;
          else hi2 = mid;
        }
        rho2 = lo2;
      }
    }
    if (rho2 < 0.0) {
      const int total = nc[0] * nc[1] * nc[2];
      int base = 0;
      for (int t0 = 0; t0 < total; t0 += 32) {
        const int t = t0 + lane;
        int c = 0, e0 = 0;
        if (t < total) {
          const int k = t % nc[2], j = (t / nc[2]) % nc[1], i = t / (nc[1] * nc[2]);
          const int64_t g = S.cell0 + ((int64_t)(c0[0] + i) * S.dims[1] + (c0[1] + j)) * S.dims[2] + (c0[2] + k);
          e0 = __ldg(&A.cell_start[g]);
          c = __ldg(&A.cell_start[g + 1]) - e0;
        }
        int incl = c;
        for (int off = 1; off < 32; off <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, incl, off);
          if (lane >= off) incl += y;
        }
        for (int q = 0; q < c; ++q) cand[base + incl - c + q] = __ldg(&A.sorted[e0 + q]);
        base += __shfl_sync(0xffffffffu, incl, 31);
      }
      C.ncand = base;
    } else {
      if (lane == 0) s_fill[wid] = 0;
      __syncwarp();
      const int total = nc[0] * nc[1] * nc[2];
      for (int t = lane; t < total; t += 32) {
        const int k = t % nc[2], j = (t / nc[2]) % nc[1], i = t / (nc[1] * nc[2]);
        const int64_t g = S.cell0 + ((int64_t)(c0[0] + i) * S.dims[1] + (c0[1] + j)) * S.dims[2] + (c0[2] + k);
        const int e1 = __ldg(&A.cell_start[g + 1]);
        for (int e = __ldg(&A.cell_start[g]); e < e1; ++e) {
          const float4 x4 = __ldg(&A.sorted[e]);
          const double dx = (double)x4.x - C.P.x, dy = (double)x4.y - C.P.y, dz = (double)x4.z - C.P.z;
          if (dx * dx + dy * dy + dz * dz < rho2) {
            const int slot = atomicAdd(&s_fill[wid], 1);
            if (slot < kCandCap) cand[slot] = x4;
          }
        }
      }
      __syncwarp();
      C.ncand = min(s_fill[wid], kCandCap);
      __syncwarp();
    }
    __syncwarp();
    {
      double R = kInf;
      const double Pd[3] = {C.P.x, C.P.y, C.P.z};
      for (int a = 0; a < 3; ++a) {
        if (ci[a] - rr > 0) R = fmin(R, Pd[a] - (S.lo[a] + (ci[a] - rr) * S.h));
        if (ci[a] + rr < S.dims[a] - 1) R = fmin(R, S.lo[a] + (ci[a] + rr + 1) * S.h - Pd[a]);
      }
      if (rho2 >= 0.0) R = fmin(R, sqrt(rho2) * (1.0 - 1e-12));
      C.R = R - S.slack;
    }
    // ---- nearest neighbour q (a Delaunay edge); duplicates of p stop the set
    int q = -1;
    float3 Q = C.P;
    {
      double bd = kInf;
      int bi = 0x7fffffff;
      bool dup = false;
      for (int j = lane; j < C.ncand; j += 32) {
        const float4 c4 = cand[j];
        const int id = __float_as_int(c4.w);
        if (id == p) continue;
        if (c4.x == C.P.x && c4.y == C.P.y && c4.z == C.P.z) dup = true;
        const double dx = (double)c4.x - C.P.x, dy = (double)c4.y - C.P.y, dz = (double)c4.z - C.P.z;
        const double d2 = dx * dx + dy * dy + dz * dz;
        if (d2 < bd || (d2 == bd && id < bi)) { bd = d2; bi = id; }
      }
      for (int off = 16; off; off >>= 1) {
        const double od = __shfl_xor_sync(0xffffffffu, bd, off);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
        if (od < bd || (od == bd && oi < bi)) { bd = od; bi = oi; }
      }
      if (ballot(dup)) fail(C, kFlagDegenerate, kWhyDuplicate);
      if (bi != 0x7fffffff) { q = bi; Q = point(C, q); }
    }
    // ---- r: smallest circumradius of (p, q, r)
    int r = -1;
    float3 Rr = C.P;
    if (q >= 0 && !C.bad) {
      const double a[3] = {(double)Q.x - C.P.x, (double)Q.y - C.P.y, (double)Q.z - C.P.z};
      const double la = a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
      double br = kInf;
      int bi = 0x7fffffff;
      for (int j = lane; j < C.ncand; j += 32) {
        const float4 c4 = cand[j];
        const int id = __float_as_int(c4.w);
        if (id == p || id == q) continue;
        const double b[3] = {(double)c4.x - C.P.x, (double)c4.y - C.P.y, (double)c4.z - C.P.z};
        const double cx = a[1] * b[2] - a[2] * b[1], cy = a[2] * b[0] - a[0] * b[2], cz = a[0] * b[1] - a[1] * b[0];
        const double cr = cx * cx + cy * cy + cz * cz;
        if (!(cr > 0.0)) continue;
        const double lb = b[0] * b[0] + b[1] * b[1] + b[2] * b[2];
        const double d[3] = {a[0] - b[0], a[1] - b[1], a[2] - b[2]};
        const double rho = la * lb * (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) / cr;
        if (rho < br || (rho == br && id < bi)) { br = rho; bi = id; }
      }
      for (int off = 16; off; off >>= 1) {
        const double od = __shfl_xor_sync(0xffffffffu, br, off);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
        if (od < br || (od == br && oi < bi)) { br = od; bi = oi; }
      }
      if (bi != 0x7fffffff) { r = bi; Rr = point(C, r); }
    }
    if (!C.bad && (q < 0 || r < 0)) fail(C, q < 0 ? kFlagCapacity : kFlagDegenerate, kWhyNoStart);
    // ---- first tetrahedron: (p, q, r) closed on either side
    int nt = 0;
    if (!C.bad) {
      float3 W;
      int w = wrap(C, q, Q, r, Rr, -1, C.P, true, W);
      if (w >= 0) {
        if (lane == 0) tri[0] = make_int4(q, r, w, 7);
        nt = 1;
      } else if (w == -1) {
        w = wrap(C, r, Rr, q, Q, -1, C.P, true, W);
        if (w >= 0) {
          if (lane == 0) tri[0] = make_int4(r, q, w, 7);
          nt = 1;
        } else if (w == -1) {
          fail(C, kFlagDegenerate, kWhyFlat);  // every point on one plane
        }
      }
    }
    __syncwarp();
    // ---- grow the star across the open edges of its link
    for (int iter = 0; !C.bad && iter < 3 * kTriCap + 8; ++iter) {
      int ft = -1, fe = 0;
      for (int t0 = 0; t0 < nt; t0 += 32) {
        const int t = t0 + lane;
        const int m = t < nt ? (tri[t].w & 7) : 0;
        const unsigned b = ballot(m != 0);
        if (b) {
          const int src = __ffs(b) - 1;
          ft = t0 + src;
          fe = __ffs(__shfl_sync(0xffffffffu, m, src)) - 1;
          break;
        }
      }
      if (ft < 0) break;  // closed (or bounded by hull faces)
      const int4 T = tri[ft];
      int x, y;
      tri_edge(T, fe, x, y);
      const int c3 = fe == 0 ? T.z : (fe == 1 ? T.x : T.y);  // T's vertex off the crossed edge
      const float3 X = point(C, x), Y = point(C, y), Z = point(C, c3);
      float3 W;
      const int w = wrap(C, y, Y, x, X, c3, Z, false, W);
      __syncwarp();
      if (w == -2) break;
      if (lane == 0) tri[ft].w &= ~(1 << fe);
      __syncwarp();
      if (w == -1) continue;  // hull face
      // new triangle (y, x, w): edge 0 (y, x) is the twin just crossed;
      // edges 1 (x, w) and 2 (w, y) close against (w, x) and (y, w)
      bool g1 = false, g2 = false, inc = false;
      for (int t0 = 0; t0 < nt; t0 += 32) {
        const int t = t0 + lane;
        if (t < nt) {
          int4 Tt = tri[t];
          int m = Tt.w;
          for (int k = 0; k < 3; ++k) {
            int ea, eb;
            tri_edge(Tt, k, ea, eb);
            const bool open = (m >> k) & 1;
            if (ea == w && eb == x) {
              if (open && !g1) { m &= ~(1 << k); g1 = true; } else inc = true;
            } else if (ea == y && eb == w) {
              if (open && !g2) { m &= ~(1 << k); g2 = true; } else inc = true;
            } else if ((ea == x && eb == w) || (ea == w && eb == y) || (ea == y && eb == x)) {
              inc = true;
            }
          }
          if (m != Tt.w) tri[t].w = m;
        }
      }
      const unsigned b1 = ballot(g1), b2 = ballot(g2);
      if (ballot(inc) || __popc(b1) > 1 || __popc(b2) > 1) {
        fail(C, kFlagRepair, kWhyLink);
        break;
      }
      if (nt >= kTriCap) {
        fail(C, kFlagCapacity, kWhyStar);
        break;
      }
      if (lane == 0) tri[nt] = make_int4(y, x, w, (b1 ? 0 : 2) | (b2 ? 0 : 4));
      ++nt;
      __syncwarp();
    }
    // an unfinished star (iteration bound) is a failure
    if (!C.bad) {
      bool open = false;
      for (int t = lane; t < nt; t += 32) open |= (tri[t].w & 7) != 0;
      if (ballot(open) || nt == 0) fail(C, kFlagRepair, kWhyOpen);
    }
    if (C.bad) {
      if (lane == 0) atomicOr(&A.flags[s], C.bad);
      __syncwarp();
      continue;
    }
    // ---- emit the tetrahedra whose smallest vertex is p
    for (int t0 = 0; t0 < nt; t0 += 32) {
      const int t = t0 + lane;
      int4 T = make_int4(0, 0, 0, 0);
      bool e = false;
      if (t < nt) {
        T = tri[t];
        e = p < T.x && p < T.y && p < T.z;
      }
      const unsigned b = ballot(e);
      if (!b) continue;
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(&A.counts[s], (unsigned long long)__popc(b));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (e) {
        const unsigned long long idx = base + __popc(b & ((1u << lane) - 1u));
        if (idx < (unsigned long long)S.cap) A.out[S.out0 + idx] = make_int4(p, T.x, T.y, T.z);
        else {
          atomicOr(&A.flags[s], kFlagOverflow);
          atomicAdd(&A.stats[kWhyOverflow], 1ull);
        }
      }
    }
    __syncwarp();
  }
}

// ---- set-up: bounding boxes, grid frames, counting sort into cells -------

__device__ __forceinline__ int ford(float f) {
  const int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float funord(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

// grid: (chunks, sets); bb: per set min x, y, z then max x, y, z (ordered ints)
__global__ void k_tess_bbox(const float* __restrict__ xyz, const int64_t* __restrict__ vprefix, int* bb, int* flags) {
  const int s = blockIdx.y;
  const int64_t v0 = vprefix[s], v1 = vprefix[s + 1];
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  bool bad = false;
  for (int64_t v = v0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < v1; v += (int64_t)gridDim.x * blockDim.x) {
    for (int a = 0; a < 3; ++a) {
      const float x = __ldg(&xyz[3 * v + a]);
      if (!isfinite(x)) bad = true;
      else { mn[a] = fminf(mn[a], x); mx[a] = fmaxf(mx[a], x); }
    }
  }
  for (int a = 0; a < 3; ++a)
    for (int off = 16; off; off >>= 1) {
      mn[a] = fminf(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], off));
      mx[a] = fmaxf(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], off));
    }
  if (__ballot_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(&flags[s], kFlagInput);
  if ((threadIdx.x & 31) == 0 && mn[0] <= mx[0]) {
    for (int a = 0; a < 3; ++a) {
      atomicMin(&bb[6 * s + a], ford(mn[a]));
      atomicMax(&bb[6 * s + 3 + a], ford(mx[a]));
    }
  }
}

// One thread per set: grid of about two points per cell within the set's
// cell budget, the Morton frame of the host tessellator, output region.
__global__ void k_tess_frame(int K, const int64_t* __restrict__ vprefix, const int* __restrict__ bb,
                             const int64_t* __restrict__ cell_pre, const int64_t* __restrict__ out_pre, TSet* sets,
                             double* hi, int* flags) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= K) return;
  TSet S;
  S.v0 = vprefix[s];
  S.n = vprefix[s + 1] - S.v0;
  S.cell0 = cell_pre[s];
  S.out0 = out_pre[s];
  S.cap = out_pre[s + 1] - S.out0;
  const int64_t ncap = cell_pre[s + 1] - S.cell0;
  double ext[3], am = 0.0;
  bool flat = S.n < 4;
  for (int a = 0; a < 3; ++a) {
    const double l = funord(bb[6 * s + a]), h = funord(bb[6 * s + 3 + a]);
    S.lo[a] = l;
    hi[3 * s + a] = h;
    ext[a] = h - l;
    if (!(ext[a] > 0.0)) flat = true;
    am = fmax(am, fmax(fabs(l), fabs(h)));
    S.mlo[a] = l;
    S.mscale[a] = ext[a] > 0.0 ? (double)((1 << 21) - 1) / ext[a] : 0.0;
  }
  S.dims[0] = S.dims[1] = S.dims[2] = 1;
  S.h = 1.0;
  if (!flat) {
    const double target = (double)(S.n / 2 > 1 ? S.n / 2 : 1);
    double h = cbrt(ext[0] * ext[1] * ext[2] / target);
    bool fits = false;
    for (int it = 0; it < 400 && !fits; ++it) {
      int64_t prod = 1;
      for (int a = 0; a < 3; ++a) {
        double d = floor(ext[a] / h);
        d = d < 1.0 ? 1.0 : (d > 1048576.0 ? 1048576.0 : d);
        S.dims[a] = (int32_t)d;
        prod *= S.dims[a];
      }
      fits = prod <= ncap;
      if (!fits) h *= 1.05;
    }
    if (!fits) {
      S.dims[0] = S.dims[1] = S.dims[2] = 1;
      h = fmax(ext[0], fmax(ext[1], ext[2]));
    }
    S.h = h;
  } else {
    atomicOr(&flags[s], kFlagInput);
  }
  S.inv_h = 1.0 / S.h;
  S.slack = 1e-9 * (am + S.h);
  sets[s] = S;
}

__device__ __forceinline__ int cell_of(const TSet& S, const float* q) {
  const int i = cell_coord(S, q[0], 0), j = cell_coord(S, q[1], 1), k = cell_coord(S, q[2], 2);
  return (i * S.dims[1] + j) * S.dims[2] + k;
}

// grid: (chunks, sets)
__global__ void k_tess_count(const float* __restrict__ xyz, const TSet* __restrict__ sets, const int* flags,
                             int32_t* pcell, int* ccount) {
  const int s = blockIdx.y;
  if (flags[s] & kFlagInput) return;
  const TSet S = sets[s];
  for (int64_t v = S.v0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < S.v0 + S.n;
       v += (int64_t)gridDim.x * blockDim.x) {
    const int lid = cell_of(S, xyz + 3 * v);
    pcell[v] = lid;
    atomicAdd(&ccount[S.cell0 + lid], 1);
  }
}

__global__ void k_tess_place(const float* __restrict__ xyz, const TSet* __restrict__ sets, const int* flags,
                             const int32_t* __restrict__ pcell, const int32_t* __restrict__ cell_start, int* fill,
                             float4* sorted) {
  const int s = blockIdx.y;
  if (flags[s] & kFlagInput) return;
  const TSet S = sets[s];
  for (int64_t v = S.v0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < S.v0 + S.n;
       v += (int64_t)gridDim.x * blockDim.x) {
    const int64_t g = S.cell0 + pcell[v];
    const int pos = cell_start[g] + atomicAdd(&fill[g], 1);
    sorted[pos] = make_float4(xyz[3 * v], xyz[3 * v + 1], xyz[3 * v + 2], __int_as_float((int)v));
  }
}

// ---- canonical order (the host tessellator's) ----------------------------

__device__ __forceinline__ uint64_t spread21(uint64_t x) {
  x &= 0x1fffffULL;
  x = (x | (x << 32)) & 0x1f00000000ffffULL;
  x = (x | (x << 16)) & 0x1f0000ff0000ffULL;
  x = (x | (x << 8)) & 0x100f00f00f00f00fULL;
  x = (x | (x << 4)) & 0x10c30c30c30c30c3ULL;
  x = (x | (x << 2)) & 0x1249249249249249ULL;
  return x;
}

// The 12 orientation-preserving vertex orders of a tetrahedron.
__constant__ int8_t c_even[12][4] = {{0, 1, 2, 3}, {0, 2, 3, 1}, {0, 3, 1, 2}, {1, 0, 3, 2}, {1, 2, 0, 3},
                                     {1, 3, 2, 0}, {2, 0, 1, 3}, {2, 1, 3, 0}, {2, 3, 0, 1}, {3, 0, 2, 1},
                                     {3, 1, 0, 2}, {3, 2, 1, 0}};

__device__ __forceinline__ bool tuple_less(const int4& a, const int4& b) {
  if (a.x != b.x) return a.x < b.x;
  if (a.y != b.y) return a.y < b.y;
  if (a.z != b.z) return a.z < b.z;
  return a.w < b.w;
}

// grid: (chunks, sets).  Each emitted tetrahedron in its smallest even
// rotation, with the Morton key of its centroid (FP64, vertices in that
// rotation's order, as the host sums them).
__global__ void k_tess_canon(const float* __restrict__ xyz, const TSet* __restrict__ sets,
                             const unsigned long long* __restrict__ counts, const int4* __restrict__ out,
                             int4* canon, unsigned long long* keys, int32_t* vals) {
  const int s = blockIdx.y;
  const TSet S = sets[s];
  const int64_t n = (int64_t)min(counts[s], (unsigned long long)S.cap);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t slot = S.out0 + i;
    const int4 t = out[slot];
    const int v[4] = {t.x, t.y, t.z, t.w};
    int best = 0;
    for (int q = 1; q < 12; ++q)
      for (int k = 0; k < 4; ++k) {
        const int a = v[c_even[q][k]], b = v[c_even[best][k]];
        if (a != b) {
          if (a < b) best = q;
          break;
        }
      }
    int4 c;
    c.x = v[c_even[best][0]];
    c.y = v[c_even[best][1]];
    c.z = v[c_even[best][2]];
    c.w = v[c_even[best][3]];
    const int cv[4] = {c.x, c.y, c.z, c.w};
    double m[3] = {0.0, 0.0, 0.0};
    for (int a = 0; a < 4; ++a)
      for (int k = 0; k < 3; ++k) m[k] += 0.25 * (double)__ldg(&xyz[3 * (int64_t)cv[a] + k]);
    uint64_t key = 0;
    for (int k = 0; k < 3; ++k) {
      double tt = (m[k] - S.mlo[k]) * S.mscale[k];
      if (tt < 0) tt = 0;
      if (tt > (double)((1 << 21) - 1)) tt = (double)((1 << 21) - 1);
      key |= spread21((uint64_t)tt) << k;
    }
    canon[slot] = c;
    keys[slot] = key;
    vals[slot] = (int32_t)slot;
  }
}

__global__ void k_tess_segments(int K, const TSet* __restrict__ sets, const unsigned long long* __restrict__ counts,
                                int32_t* seg_begin, int32_t* seg_end) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= K) return;
  const TSet S = sets[s];
  seg_begin[s] = (int32_t)S.out0;
  seg_end[s] = (int32_t)(S.out0 + (int64_t)min(counts[s], (unsigned long long)S.cap));
}

// Equal Morton keys: order the run by vertex tuple (the host's tie rule).
__global__ void k_tess_ties(const TSet* __restrict__ sets, const unsigned long long* __restrict__ counts,
                            const unsigned long long* __restrict__ keys, const int4* __restrict__ canon,
                            int32_t* vals, int* flags, unsigned long long* stats) {
  const int s = blockIdx.y;
  const TSet S = sets[s];
  const int64_t n = (int64_t)min(counts[s], (unsigned long long)S.cap);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t pos = S.out0 + i;
    const unsigned long long k = keys[pos];
    if (i > 0 && keys[pos - 1] == k) continue;
    int64_t j = i + 1;
    while (j < n && j - i <= 64 && keys[S.out0 + j] == k) ++j;
    const int64_t L = j - i;
    if (L == 1) continue;
    if (L > 64) {
      atomicOr(&flags[s], kFlagRepair);
      atomicAdd(&stats[kWhyRun], 1ull);
      continue;
    }
    for (int64_t a = 1; a < L; ++a) {
      const int32_t x = vals[pos + a];
      const int4 cx = canon[x];
      int64_t b = a - 1;
      while (b >= 0 && tuple_less(cx, canon[vals[pos + b]])) {
        vals[pos + b + 1] = vals[pos + b];
        --b;
      }
      vals[pos + b + 1] = x;
    }
  }
}

__global__ void k_tess_gather(const TSet* __restrict__ sets, const int64_t* __restrict__ tpre,
                              const int32_t* __restrict__ vals, const int4* __restrict__ canon, int4* tets) {
  const int s = blockIdx.y;
  const TSet S = sets[s];
  const int64_t n = tpre[s + 1] - tpre[s];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    tets[tpre[s] + i] = canon[vals[S.out0 + i]];
}

}  // namespace

// ---- C ABI ----------------------------------------------------------------

namespace {

struct GpuTess {
  int K = 0;
  std::vector<int64_t> tprefix;
  std::vector<int32_t> status;
  int4* tets = nullptr;
  int64_t stats[kStatsLen] = {};
};

struct DevBufs {
  std::vector<void*> ptrs;
  bool failed = false;
  ~DevBufs() {
    for (void* p : ptrs) cudaFree(p);
  }
  template <class T>
  T* get(size_t n) {
    void* p = nullptr;
    if (cudaMalloc(&p, (n ? n : 1) * sizeof(T)) != cudaSuccess) {
      failed = true;
      return nullptr;
    }
    ptrs.push_back(p);
    return (T*)p;
  }
};

int cuda_fail(const char* where, cudaError_t e) {
  const std::string m = std::string(where) + ": " + cudaGetErrorString(e);
  return dtfe_internal_set_error(DTFE_ERR_CUDA, m.c_str());
}

#define TESS_CHECK(where)                         \
  do {                                            \
    cudaError_t e_ = cudaGetLastError();          \
    if (e_ != cudaSuccess) return cuda_fail(where, e_); \
  } while (0)

}  // namespace

extern "C" {

int dtfe_gpu_tessellate(void* stream, int32_t n_sets, const int64_t* vprefix, const float* xyz_dev, void** out) {
  if (!out) return dtfe_internal_set_error(DTFE_ERR_ARG, "dtfe_gpu_tessellate: out is NULL");
  *out = nullptr;
  if (n_sets < 1 || n_sets > 65535 || !vprefix || !xyz_dev)
    return dtfe_internal_set_error(DTFE_ERR_ARG, "dtfe_gpu_tessellate: need 1..65535 sets, vprefix and xyz");
  const int K = n_sets;
  if (vprefix[0] != 0) return dtfe_internal_set_error(DTFE_ERR_ARG, "dtfe_gpu_tessellate: vprefix[0] must be 0");
  int64_t maxn = 0;
  for (int s = 0; s < K; ++s) {
    if (vprefix[s + 1] < vprefix[s])
      return dtfe_internal_set_error(DTFE_ERR_ARG, "dtfe_gpu_tessellate: vprefix must not decrease");
    maxn = std::max<int64_t>(maxn, vprefix[s + 1] - vprefix[s]);
  }
  const int64_t V = vprefix[K];
  std::vector<int64_t> cpre(K + 1, 0), opre(K + 1, 0);
  for (int s = 0; s < K; ++s) {
    const int64_t n = vprefix[s + 1] - vprefix[s];
    cpre[s + 1] = cpre[s] + n / 2 + 8;
    opre[s + 1] = opre[s] + 8 * n + 4096;
  }
  const int64_t NC = cpre[K], NO = opre[K];
  if (V >= (int64_t)INT32_MAX || NO >= (int64_t)INT32_MAX || NC >= (int64_t)INT32_MAX)
    return dtfe_internal_set_error(DTFE_ERR_TOO_LARGE, "dtfe_gpu_tessellate: more than 2^31 vertices or slots");
  cudaStream_t st = (cudaStream_t)stream;
  DevBufs B;
  int64_t* d_vpre = B.get<int64_t>(K + 1);
  int64_t* d_cpre = B.get<int64_t>(K + 1);
  int64_t* d_opre = B.get<int64_t>(K + 1);
  int* d_bb = B.get<int>(6 * K);
  int* d_flags = B.get<int>(K);
  TSet* d_sets = B.get<TSet>(K);
  double* d_hi = B.get<double>(3 * K);
  int32_t* d_pcell = B.get<int32_t>(V);
  int* d_ccount = B.get<int>(NC + 1);
  int32_t* d_cstart = B.get<int32_t>(NC + 1);
  float4* d_sorted = B.get<float4>(V);
  int4* d_out = B.get<int4>(NO);
  unsigned long long* d_counts = B.get<unsigned long long>(K);
  unsigned long long* d_next = B.get<unsigned long long>(1);
  int4* d_canon = B.get<int4>(NO);
  unsigned long long* d_keys = B.get<unsigned long long>(NO);
  unsigned long long* d_keys2 = B.get<unsigned long long>(NO);
  int32_t* d_vals = B.get<int32_t>(NO);
  int32_t* d_vals2 = B.get<int32_t>(NO);
  int32_t* d_sb = B.get<int32_t>(K);
  int32_t* d_se = B.get<int32_t>(K);
  int64_t* d_tpre = B.get<int64_t>(K + 1);
  unsigned long long* d_stats = B.get<unsigned long long>(kStatsLen);
  if (B.failed) {
    cudaGetLastError();
    return dtfe_internal_set_error(DTFE_ERR_ALLOC, "dtfe_gpu_tessellate: device allocation failed");
  }
  std::vector<int> bb0(6 * (size_t)K);
  for (int s = 0; s < K; ++s)
    for (int a = 0; a < 3; ++a) {
      bb0[6 * s + a] = INT32_MAX;
      bb0[6 * s + 3 + a] = INT32_MIN;
    }
  cudaMemcpyAsync(d_vpre, vprefix, (K + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_cpre, cpre.data(), (K + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_opre, opre.data(), (K + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_bb, bb0.data(), bb0.size() * sizeof(int), cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(d_flags, 0, K * sizeof(int), st);
  cudaMemsetAsync(d_ccount, 0, (NC + 1) * sizeof(int), st);
  cudaMemsetAsync(d_counts, 0, K * sizeof(unsigned long long), st);
  cudaMemsetAsync(d_next, 0, sizeof(unsigned long long), st);
  cudaMemsetAsync(d_stats, 0, kStatsLen * sizeof(unsigned long long), st);
  TESS_CHECK("dtfe_gpu_tessellate: set-up copies");
  const unsigned bx = (unsigned)std::min<int64_t>(1024, std::max<int64_t>(1, (maxn + 1023) / 1024));
  k_tess_bbox<<<dim3(bx, K), 256, 0, st>>>(xyz_dev, d_vpre, d_bb, d_flags);
  k_tess_frame<<<(K + 127) / 128, 128, 0, st>>>(K, d_vpre, d_bb, d_cpre, d_opre, d_sets, d_hi, d_flags);
  k_tess_count<<<dim3(bx, K), 256, 0, st>>>(xyz_dev, d_sets, d_flags, d_pcell, d_ccount);
  TESS_CHECK("dtfe_gpu_tessellate: grid");
  {
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, d_ccount, d_cstart, (int)(NC + 1), st);
    void* tmp = B.get<char>(tb);
    if (!tmp) return dtfe_internal_set_error(DTFE_ERR_ALLOC, "dtfe_gpu_tessellate: scan scratch");
    cub::DeviceScan::ExclusiveSum(tmp, tb, d_ccount, d_cstart, (int)(NC + 1), st);
  }
  cudaMemsetAsync(d_ccount, 0, (NC + 1) * sizeof(int), st);
  k_tess_place<<<dim3(bx, K), 256, 0, st>>>(xyz_dev, d_sets, d_flags, d_pcell, d_cstart, d_ccount, d_sorted);
  TESS_CHECK("dtfe_gpu_tessellate: cells");
  {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaFuncSetAttribute(k_tess_stars, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kStarSmem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tess_stars, kWarps * 32, kStarSmem);
    const int64_t want = (V + kWarps - 1) / kWarps;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)std::max(1, sms) * std::max(1, per_sm)));
    StarArgs A;
    A.xyz = xyz_dev;
    A.sets = d_sets;
    A.vprefix = d_vpre;
    A.hi = d_hi;
    A.K = K;
    A.V = V;
    A.cell_start = d_cstart;
    A.sorted = d_sorted;
    A.pcell = d_pcell;
    A.out = d_out;
    A.counts = d_counts;
    A.flags = d_flags;
    A.next = d_next;
    A.stats = d_stats;
    if (V > 0) k_tess_stars<<<grid, kWarps * 32, kStarSmem, st>>>(A);
  }
  TESS_CHECK("dtfe_gpu_tessellate: stars");
  const unsigned bo = (unsigned)std::min<int64_t>(4096, std::max<int64_t>(1, (8 * maxn + 4096 + 1023) / 1024));
  k_tess_canon<<<dim3(bo, K), 256, 0, st>>>(xyz_dev, d_sets, d_counts, d_out, d_canon, d_keys, d_vals);
  k_tess_segments<<<(K + 127) / 128, 128, 0, st>>>(K, d_sets, d_counts, d_sb, d_se);
  TESS_CHECK("dtfe_gpu_tessellate: keys");
  {
    size_t tb = 0;
    cub::DeviceSegmentedRadixSort::SortPairs(nullptr, tb, d_keys, d_keys2, d_vals, d_vals2, (int)NO, K, d_sb, d_se, 0,
                                             63, st);
    void* tmp = B.get<char>(tb);
    if (!tmp) return dtfe_internal_set_error(DTFE_ERR_ALLOC, "dtfe_gpu_tessellate: sort scratch");
    cub::DeviceSegmentedRadixSort::SortPairs(tmp, tb, d_keys, d_keys2, d_vals, d_vals2, (int)NO, K, d_sb, d_se, 0,
                                             63, st);
  }
  k_tess_ties<<<dim3(bo, K), 256, 0, st>>>(d_sets, d_counts, d_keys2, d_canon, d_vals2, d_flags, d_stats);
  TESS_CHECK("dtfe_gpu_tessellate: sort");
  std::vector<unsigned long long> counts(K);
  std::vector<int> flags(K);
  cudaMemcpyAsync(counts.data(), d_counts, K * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(flags.data(), d_flags, K * sizeof(int), cudaMemcpyDeviceToHost, st);
  std::vector<unsigned long long> stats(kStatsLen);
  cudaMemcpyAsync(stats.data(), d_stats, kStatsLen * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail("dtfe_gpu_tessellate", e);
  GpuTess* G = new GpuTess();
  G->K = K;
  G->tprefix.assign(K + 1, 0);
  G->status.assign(K, 0);
  for (int i = 0; i < kWhyCount; ++i) G->stats[i] = (int64_t)stats[i];
  G->stats[kWhyCount] = (int64_t)stats[kWhyCount] - 1;
  G->stats[kWhyCount + 1] = stats[kWhyCount] ? (int64_t)stats[kWhyCount + 1] : -1;
  for (int s = 0; s < K; ++s) {
    int f = flags[s];
    if (counts[s] > (unsigned long long)(opre[s + 1] - opre[s])) f |= kFlagOverflow;
    G->status[s] = f;
    G->tprefix[s + 1] = G->tprefix[s] + (f ? 0 : (int64_t)counts[s]);
  }
  const int64_t T = G->tprefix[K];
  if (cudaMalloc(&G->tets, (T ? T : 1) * sizeof(int4)) != cudaSuccess) {
    cudaGetLastError();
    delete G;
    return dtfe_internal_set_error(DTFE_ERR_ALLOC, "dtfe_gpu_tessellate: output allocation failed");
  }
  cudaMemcpyAsync(d_tpre, G->tprefix.data(), (K + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st);
  k_tess_gather<<<dim3(bo, K), 256, 0, st>>>(d_sets, d_tpre, d_vals2, d_canon, G->tets);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    cudaFree(G->tets);
    delete G;
    return cuda_fail("dtfe_gpu_tessellate: gather", e);
  }
  *out = G;
  return DTFE_OK;
}

int dtfe_gpu_tess_sizes(void* tess, int64_t* tprefix, int32_t* status) {
  GpuTess* G = (GpuTess*)tess;
  if (!G) return dtfe_internal_set_error(DTFE_ERR_ARG, "dtfe_gpu_tess_sizes: NULL tessellation");
  if (tprefix) std::memcpy(tprefix, G->tprefix.data(), (G->K + 1) * sizeof(int64_t));
  if (status) std::memcpy(status, G->status.data(), G->K * sizeof(int32_t));
  return DTFE_OK;
}

int dtfe_gpu_tess_stats(void* tess, int64_t* counts, int32_t n) {
  GpuTess* G = (GpuTess*)tess;
  if (!G || !counts || n < 0) return dtfe_internal_set_error(DTFE_ERR_ARG, "dtfe_gpu_tess_stats: bad argument");
  for (int i = 0; i < n; ++i) counts[i] = i < kStatsLen ? G->stats[i] : 0;
  return DTFE_OK;
}

int dtfe_gpu_tess_export(void* tess, int32_t* tet_v, int32_t to_device) {
  GpuTess* G = (GpuTess*)tess;
  if (!G || !tet_v) return dtfe_internal_set_error(DTFE_ERR_ARG, "dtfe_gpu_tess_export: NULL argument");
  const int64_t T = G->tprefix[G->K];
  if (T == 0) return DTFE_OK;
  const cudaError_t e = cudaMemcpy(tet_v, G->tets, T * sizeof(int4),
                                   to_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail("dtfe_gpu_tess_export", e);
  return DTFE_OK;
}

int dtfe_gpu_tess_release(void* tess) {
  GpuTess* G = (GpuTess*)tess;
  if (!G) return DTFE_OK;
  cudaFree(G->tets);
  delete G;
  return DTFE_OK;
}

}  // extern "C"
