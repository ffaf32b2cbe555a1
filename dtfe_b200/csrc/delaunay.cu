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
//   1. gathers, from the 5^3 grid cells around p's cell (a uniform grid of
//      about two points per cell), the points closer to p than R, the
//      distance from p to the block's faces (a smaller radius holding at most
//      256 points in a dense cluster), into shared memory as double offsets
//      from p: every point within R of p is a candidate;
//   2. starts from p's nearest neighbour q, the candidate r whose triangle
//      pqr has the smallest circumradius (the smallest sphere through p, q, r
//      is then empty) and the apex s that closes pqr to a tetrahedron;
//   3. grows the star of p across the open edges of its link (the triangles
//      opposite p): across edge (u, v) the apex is the point on the far side
//      of plane (p, v, u) whose circumsphere with p, v, u contains no other
//      such point (gift wrapping; the spheres through p, v, u form a pencil
//      ordered by the position of their centre along the face normal);
//   4. certifies every tetrahedron it adds: its circumsphere is empty of all
//      points of the set.  A sphere inside the candidate ball is checked
//      against every candidate; a larger one against every point of the grid
//      columns it reaches (along the axis towards its centre), and the best
//      point found inside replaces the apex.  A link edge without any point
//      beyond it (certified by a column scan of the half-space) lies on the
//      convex hull; a point exactly on such a face's plane is harmless
//      outside the face's circumcircle;
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
constexpr int kCandCap = 256;        // candidates per warp
constexpr int kTriCap = 512;         // link triangles per warp
// dynamic shared memory per block: candidate offsets (3 doubles) and ids,
// link triangles (int4)
constexpr size_t kStarSmem = (size_t)kWarps * ((size_t)kCandCap * 28 + (size_t)kTriCap * 16);

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

// Circumsphere in the frame of the star's centre p: a, b, c are the offsets
// (rounded once to double) of three points from p.  The centre is
// N / D with N = |a|^2 (b x c) + |b|^2 (c x a) + |c|^2 (a x b) and
// D = 2 a.(b x c); both carry at most kCircErr times the sums of their
// terms' magnitudes (a first-order count of the roundings, the offsets'
// included, gives under 16 eps).  |c - true centre| <= err and
// |r - true radius| <= err; ok is false when D is not resolved.
struct Sphere {
  double c[3], r, err;  // c: offset of the centre from p
  bool ok;
};

__device__ __forceinline__ Sphere circum_rel(const double* A, const double* B, const double* C) {
  Sphere S;
  const double la = A[0] * A[0] + A[1] * A[1] + A[2] * A[2];
  const double lb = B[0] * B[0] + B[1] * B[1] + B[2] * B[2];
  const double lc = C[0] * C[0] + C[1] * C[1] + C[2] * C[2];
  double N[3], Np[3];
  double D = 0.0, Dp = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int i = (k + 1) % 3, j = (k + 2) % 3;
    const double x1 = B[i] * C[j], x2 = B[j] * C[i];
    const double y1 = C[i] * A[j], y2 = C[j] * A[i];
    const double z1 = A[i] * B[j], z2 = A[j] * B[i];
    const double bc = x1 - x2, bca = fabs(x1) + fabs(x2);
    N[k] = la * bc + lb * (y1 - y2) + lc * (z1 - z2);
    Np[k] = la * bca + lb * (fabs(y1) + fabs(y2)) + lc * (fabs(z1) + fabs(z2));
    D += A[k] * bc;
    Dp += fabs(A[k]) * bca;
  }
  D *= 2.0;
  Dp *= 2.0;
  const double dN = kCircErr * sqrt(Np[0] * Np[0] + Np[1] * Np[1] + Np[2] * Np[2]);
  const double dD = kCircErr * Dp;
  if (!(fabs(D) > 2.0 * dD)) {
    S.ok = false;
    S.c[0] = S.c[1] = S.c[2] = 0.0;
    S.r = kInf;
    S.err = kInf;
    return S;
  }
  const double inv = 1.0 / D;
  S.c[0] = N[0] * inv;
  S.c[1] = N[1] * inv;
  S.c[2] = N[2] * inv;
  S.r = sqrt(S.c[0] * S.c[0] + S.c[1] * S.c[1] + S.c[2] * S.c[2]);
  S.err = (2.0 * dN + S.r * dD) / (fabs(D) - dD) * (1.0 + 1e-6) + 8.0 * kEps * S.r;
  S.ok = true;
  return S;
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

// Per-warp context of one star.  Candidates are the points within R of p,
// stored as double offsets from p (structure of arrays in shared memory).
struct Ctx {
  const TSet* S;
  const float* xyz;            // all vertices, 3 floats each
  double hi[3];
  const int32_t* cell_start;   // global
  const float4* sorted;
  const double* cx;            // candidate offsets from p
  const double* cy;
  const double* cz;
  const int* cid;              // candidate vertex ids
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

__device__ __forceinline__ void rel(const Ctx& C, float3 X, double* d) {
  d[0] = (double)X.x - C.P.x;
  d[1] = (double)X.y - C.P.y;
  d[2] = (double)X.z - C.P.z;
}

// A face (p, u, v) in p's frame: the offsets a = u - p, b = v - p, the normal
// n = a x b and the magnitudes of n's two products per component.
// orient(p, u, v, x) is the sign of d.n (d = x - p), filtered with the host's
// orientation bound (the same determinant expanded along x's row) and exact
// otherwise (the float inputs fetched by id).
struct Face {
  int u, v;
  double a[3], b[3], n[3], na[3];
};

__device__ __forceinline__ Face make_face(const Ctx& C, int u, int v) {
  Face F;
  F.u = u;
  F.v = v;
  rel(C, point(C, u), F.a);
  rel(C, point(C, v), F.b);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int i = (k + 1) % 3, j = (k + 2) % 3;
    const double m1 = F.a[i] * F.b[j], m2 = F.a[j] * F.b[i];
    F.n[k] = m1 - m2;
    F.na[k] = fabs(m1) + fabs(m2);
  }
  return F;
}

__device__ __forceinline__ int orient_face(const Ctx& C, const Face& F, const double* d, int id) {
  const double det = d[0] * F.n[0] + d[1] * F.n[1] + d[2] * F.n[2];
  const double perm = fabs(d[0]) * F.na[0] + fabs(d[1]) * F.na[1] + fabs(d[2]) * F.na[2];
  const double bound = kOrientErr * perm;
  if (det > bound) return 1;
  if (-det > bound) return -1;
  return orient_exact_f(C.P, point(C, F.u), point(C, F.v), point(C, id));
}

// In-sphere sign of x (offset d, id) for the positively oriented (p, u, v, b)
// whose sphere is S: decided by the distance to the bounded centre when x is
// clearly in or out, else by the determinant over the float inputs.
__device__ __forceinline__ int insphere_face(const Ctx& C, const Face& F, int b, const Sphere& S, const double* d,
                                             int id) {
  if (S.ok) {
    const double dx = d[0] - S.c[0], dy = d[1] - S.c[1], dz = d[2] - S.c[2];
    const double d2 = dx * dx + dy * dy + dz * dz;
    const double hi = S.r + 2.0 * S.err;
    if (d2 > hi * hi * (1.0 + 1e-9)) return -1;
    const double lo = S.r - 2.0 * S.err;
    if (lo > 0.0 && d2 < lo * lo * (1.0 - 1e-9)) return 1;
  }
  return insphere_f(C.P, point(C, F.u), point(C, F.v), point(C, b), point(C, id));
}

// Among the lanes' apex candidates for face F (best >= 0 on a lane, offset
// bd, sphere sb), the one whose sphere holds none of the others: the apices
// are ordered by the position of their sphere centre along the face normal
// (smaller = better); overlapping error intervals are resolved with the exact
// in-sphere sign (an exact tie keeps the current winner: the verification of
// the winner's sphere reports it).  Returns the id (offset in Wd), -1 when no
// lane has one, -2 on failure (flag set).
__device__ __forceinline__ int warp_select(Ctx& C, const Face& F, int best, const double* bd, const Sphere& sb,
                                        double* Wd) {
  double lo = kInf, hi = kInf;
  if (best >= 0) {
    if (sb.ok) {
      const double lam = F.n[0] * sb.c[0] + F.n[1] * sb.c[1] + F.n[2] * sb.c[2];
      const double nn = sqrt(F.n[0] * F.n[0] + F.n[1] * F.n[1] + F.n[2] * F.n[2]);
      const double e = (nn * sb.err +
                        4.0 * kEps * (fabs(F.n[0] * sb.c[0]) + fabs(F.n[1] * sb.c[1]) + fabs(F.n[2] * sb.c[2]))) *
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
  for (int k = 0; k < 3; ++k) Wd[k] = __shfl_sync(0xffffffffu, bd[k], ml);
  for (unsigned amb = ballot(best >= 0 && C.lane != ml && lo <= mh); amb; amb &= amb - 1) {
    const int l = __ffs(amb) - 1;
    const int id = __shfl_sync(0xffffffffu, best, l);
    double X[3];
    for (int k = 0; k < 3; ++k) X[k] = __shfl_sync(0xffffffffu, bd[k], l);
    const int s = insphere_f(C.P, point(C, F.u), point(C, F.v), point(C, w), point(C, id));
    if (s == 2) {
      fail(C, kFlagUndecided, kWhyUndecided);
      return -2;
    }
    if (s > 0) {
      w = id;
      for (int k = 0; k < 3; ++k) Wd[k] = X[k];
    }
  }
  return w;
}

// Scan of the grid cells touched by the sphere Sp of the positively oriented
// (p, u, v, w).  Returns the best point beyond the face strictly inside the
// sphere (the apex over the whole set: every point beyond the face with a
// smaller sphere lies in this one; offset in Yd), -1 when the sphere holds
// no point (w is certified), -2 on failure: a point exactly on the sphere of
// a certified w (a tie), a point inside it not beyond the face, or an
// undecidable test (flag set).
__device__ __noinline__ int sphere_scan(Ctx& C, const Face& F, int w, const Sphere& Sp, double* Yd) {
  const TSet& S = *C.S;
  const double rad = Sp.r + 2.0 * Sp.err + S.slack;
  const double cen[3] = {C.P.x + Sp.c[0], C.P.y + Sp.c[1], C.P.z + Sp.c[2]};
  // columns of cells along a2, the axis of the centre's largest offset from p
  // (a large sphere then meets the grid in a thin cap across the columns);
  // in each column, the cells within the sphere's reach along a2
  int a2 = 0;
  for (int a = 1; a < 3; ++a)
    if (fabs(Sp.c[a]) > fabs(Sp.c[a2])) a2 = a;
  const int a0 = a2 == 0 ? 1 : 0, a1 = a2 == 2 ? 1 : 2;
  // a centre beyond the grid along a2 reaches it only within a disk
  const double gz = cen[a2] < S.lo[a2] ? S.lo[a2] - cen[a2] : (cen[a2] > C.hi[a2] ? cen[a2] - C.hi[a2] : 0.0);
  const double reach = sqrt(fmax(0.0, rad * rad * (1.0 + 1e-9) - gz * gz)) * (1.0 + 1e-9) + S.slack;
  const int i0 = cell_coord(S, cen[a0] - reach, a0), i1 = cell_coord(S, cen[a0] + reach, a0);
  const int j0 = cell_coord(S, cen[a1] - reach, a1), j1 = cell_coord(S, cen[a1] + reach, a1);
  const int nj = j1 - j0 + 1;
  const int ncol = (i1 - i0 + 1) * nj;
  int best = -1, flag = 0, why = 0;
  bool on_w = false;
  double bd[3] = {0.0, 0.0, 0.0};
  Sphere sb;
  sb.ok = false;
  for (int t = C.lane; t < ncol && !flag; t += 32) {
    int ci[3];
    ci[a0] = i0 + t / nj;
    ci[a1] = j0 + t % nj;
    double bx0, bx1, by0, by1;
    cell_box(S, C.hi, ci[a0], a0, bx0, bx1);
    cell_box(S, C.hi, ci[a1], a1, by0, by1);
    const double qx = cen[a0] < bx0 ? bx0 - cen[a0] : (cen[a0] > bx1 ? cen[a0] - bx1 : 0.0);
    const double qy = cen[a1] < by0 ? by0 - cen[a1] : (cen[a1] > by1 ? cen[a1] - by1 : 0.0);
    const double rest = rad * rad * (1.0 + 1e-9) - (qx * qx + qy * qy);
    if (rest < 0.0) continue;
    const double half = sqrt(rest) * (1.0 + 1e-9) + S.slack;
    const int k0 = cell_coord(S, cen[a2] - half, a2), k1 = cell_coord(S, cen[a2] + half, a2);
    for (int k = k0; k <= k1 && !flag; ++k) {
      ci[a2] = k;
      const int64_t g = S.cell0 + ((int64_t)ci[0] * S.dims[1] + ci[1]) * S.dims[2] + ci[2];
      const int e0 = __ldg(&C.cell_start[g]), e1 = __ldg(&C.cell_start[g + 1]);
      for (int e = e0; e < e1; ++e) {
        const float4 x4 = __ldg(&C.sorted[e]);
        const int id = __float_as_int(x4.w);
        if (id == C.p || id == F.u || id == F.v || id == w) continue;
        double d[3];
        rel(C, f3(x4), d);
        const int s0 = insphere_face(C, F, w, Sp, d, id);
        if (s0 == 2) { flag = kFlagUndecided; why = kWhyUndecided; break; }
        if (s0 == 0) { on_w = true; continue; }
        if (s0 < 0) continue;
        if (best >= 0 && insphere_face(C, F, best, sb, d, id) <= 0) continue;  // not better than this lane's best
        const int o = orient_face(C, F, d, id);
        if (o != 1) {
          flag = o == 2 ? kFlagUndecided : kFlagRepair;
          why = o == 2 ? kWhyUndecided : kWhyNotDelaunay;
          break;
        }
        best = id;
        bd[0] = d[0]; bd[1] = d[1]; bd[2] = d[2];
        sb = circum_rel(F.a, F.b, d);
      }
    }
  }
  const unsigned fb = ballot(flag != 0);
  if (fb) {
    const int l = __ffs(fb) - 1;
    fail(C, __shfl_sync(0xffffffffu, flag, l), __shfl_sync(0xffffffffu, why, l));
    return -2;
  }
  const int r = warp_select(C, F, best, bd, sb, Yd);
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
__device__ __noinline__ int halfspace_scan(Ctx& C, const Face& F, int c) {
  const TSet& S = *C.S;
  const double Pd[3] = {C.P.x, C.P.y, C.P.z};
  // columns of cells along the normal's dominant axis a2; in each, the cells
  // that reach beyond the plane (whose a2-coordinate over the column's
  // rectangle lies between the plane's values at its corners)
  int a2 = 0;
  for (int a = 1; a < 3; ++a)
    if (fabs(F.n[a]) > fabs(F.n[a2])) a2 = a;
  const int a0 = a2 == 0 ? 1 : 0, a1 = a2 == 2 ? 1 : 2;
  const long long ncol = (long long)S.dims[a0] * S.dims[a1];
  int found = -1, flag = 0;
  for (long long t0 = 0; t0 < ncol; t0 += 32) {
    const long long t = t0 + C.lane;
    if (t < ncol) {
      int ci[3];
      ci[a0] = (int)(t / S.dims[a1]);
      ci[a1] = (int)(t % S.dims[a1]);
      double x0, x1, y0, y1;
      cell_box(S, C.hi, ci[a0], a0, x0, x1);
      cell_box(S, C.hi, ci[a1], a1, y0, y1);
      const double xs[2] = {x0 - Pd[a0], x1 - Pd[a0]}, ys[2] = {y0 - Pd[a1], y1 - Pd[a1]};
      double tmin = kInf, tmax = -kInf;
      for (int u = 0; u < 2; ++u)
        for (int v = 0; v < 2; ++v) {
          const double tz = Pd[a2] - (F.n[a0] * xs[u] + F.n[a1] * ys[v]) / F.n[a2];
          tmin = fmin(tmin, tz);
          tmax = fmax(tmax, tz);
        }
      const double margin = 1e-6 * (fabs(Pd[a2]) + fabs(tmin) + fabs(tmax) + S.h) + S.slack;
      int k0, k1;
      if (F.n[a2] > 0.0) {
        k0 = cell_coord(S, tmin - margin, a2);
        k1 = S.dims[a2] - 1;
      } else {
        k0 = 0;
        k1 = cell_coord(S, tmax + margin, a2);
      }
      for (int k = k0; k <= k1 && found < 0 && !flag; ++k) {
        ci[a2] = k;
        const int64_t g = S.cell0 + ((int64_t)ci[0] * S.dims[1] + ci[1]) * S.dims[2] + ci[2];
        const int e0 = __ldg(&C.cell_start[g]), e1 = __ldg(&C.cell_start[g + 1]);
        for (int e = e0; e < e1 && found < 0 && !flag; ++e) {
          const float4 x4 = __ldg(&C.sorted[e]);
          const int id = __float_as_int(x4.w);
          if (id == C.p || id == F.u || id == F.v) continue;
          double d[3];
          rel(C, f3(x4), d);
          const int o = orient_face(C, F, d, id);
          if (o == 2) flag = kFlagUndecided;
          else if (o > 0) found = id;
          else if (o == 0) {
            // on the face's plane: harmless outside the face's circumcircle,
            // which is where the certified sphere across the face meets it
            const int s = c >= 0 ? insphere_f(C.P, point(C, F.v), point(C, F.u), point(C, c), f3(x4)) : 0;
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
// being a Delaunay face).  Returns w >= 0, -1 when no point lies beyond the
// face (a hull face), -2 on failure (flag set).  (p, v, u, c) is the
// certified tetrahedron on the other side (c < 0: none).
__device__ __noinline__ int orient_slow(const Ctx& C, const Face& F, int id) {
  return orient_exact_f(C.P, point(C, F.u), point(C, F.v), point(C, id));
}

__device__ __noinline__ int insphere_slow(const Ctx& C, const Face& F, int b, int id) {
  return insphere_f(C.P, point(C, F.u), point(C, F.v), point(C, b), point(C, id));
}

__device__ __noinline__ int wrap(Ctx& C, int u, int v, int c) {
  const Face F = make_face(C, u, v);
  // the loops below run on register copies (F and C live in memory: their
  // addresses go to the out-of-line scans)
  const double n0 = F.n[0], n1 = F.n[1], n2 = F.n[2], m0 = F.na[0], m1 = F.na[1], m2 = F.na[2];
  const double fa[3] = {F.a[0], F.a[1], F.a[2]}, fb[3] = {F.b[0], F.b[1], F.b[2]};
  const double* __restrict__ cx = C.cx;
  const double* __restrict__ cy = C.cy;
  const double* __restrict__ cz = C.cz;
  const int* __restrict__ cid = C.cid;
  const int ncand = C.ncand, lane = C.lane;
  int best = -1, flag = 0;
  double bd[3] = {0.0, 0.0, 0.0};
  Sphere sb;
  sb.ok = false;
  // gift wrapping over the candidates: each lane keeps the best of its share
  for (int j = lane; j < ncand; j += 32) {
    const int id = cid[j];
    if (id == u || id == v) continue;
    const double d[3] = {cx[j], cy[j], cz[j]};
    if (best >= 0) {
      int si = 0;
      if (sb.ok) {
        const double ex = d[0] - sb.c[0], ey = d[1] - sb.c[1], ez = d[2] - sb.c[2];
        const double e2 = ex * ex + ey * ey + ez * ez;
        const double hi = sb.r + 2.0 * sb.err, lo = sb.r - 2.0 * sb.err;
        if (e2 > hi * hi * (1.0 + 1e-9)) si = -1;
        else if (lo > 0.0 && e2 < lo * lo * (1.0 - 1e-9)) si = 1;
      }
      if (si == 0) si = insphere_slow(C, F, best, id);
      if (si == 2) { flag = 1; continue; }
      if (si <= 0) continue;
    }
    const double det = d[0] * n0 + d[1] * n1 + d[2] * n2;
    const double bound = kOrientErr * (fabs(d[0]) * m0 + fabs(d[1]) * m1 + fabs(d[2]) * m2);
    const int o = det > bound ? 1 : (-det > bound ? -1 : orient_slow(C, F, id));
    if (o == 2) { flag = 1; continue; }
    if (o <= 0) continue;
    best = id;
    bd[0] = d[0]; bd[1] = d[1]; bd[2] = d[2];
    sb = circum_rel(fa, fb, d);
  }
  if (ballot(flag != 0)) {
    fail(C, kFlagUndecided, kWhyUndecided);
    return -2;
  }
  double Wd[3];
  int w = warp_select(C, F, best, bd, sb, Wd);
  if (w == -2) return -2;
  bool from_cands = true;
  if (w < 0) {
    w = halfspace_scan(C, F, c);
    if (w < 0) return w;  // -1: hull face; -2: failure
    rel(C, point(C, w), Wd);
    from_cands = false;
  }
  for (int it = 0; it < 4; ++it) {
    const Sphere Sp = circum_rel(fa, fb, Wd);
    if (!Sp.ok) {
      fail(C, kFlagUndecided, kWhyUndecided);
      return -2;
    }
    if (from_cands && 2.0 * (Sp.r + Sp.err) * (1.0 + 1e-9) < C.R) {
      // the sphere lies in the candidate ball: verify it against every
      // candidate (a point on it is a tie; one inside cannot occur)
      const double hi = Sp.r + 2.0 * Sp.err, lo = Sp.r - 2.0 * Sp.err;
      const double hi2 = hi * hi * (1.0 + 1e-9), lo2 = lo > 0.0 ? lo * lo * (1.0 - 1e-9) : -1.0;
      int bad = 0;
      for (int j = lane; j < ncand; j += 32) {
        const int id = cid[j];
        if (id == u || id == v || id == w) continue;
        const double ex = cx[j] - Sp.c[0], ey = cy[j] - Sp.c[1], ez = cz[j] - Sp.c[2];
        const double e2 = ex * ex + ey * ey + ez * ez;
        if (e2 > hi2) continue;
        const int si = e2 < lo2 ? 1 : insphere_slow(C, F, w, id);
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
    double Yd[3];
    const int y = sphere_scan(C, F, w, Sp, Yd);
    if (y == -2) return -2;
    if (y < 0) return w;
    w = y;
    Wd[0] = Yd[0]; Wd[1] = Yd[1]; Wd[2] = Yd[2];
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

// Points of the block c0 + [0, nc) (other than p) strictly closer to P than
// sqrt(d2max).
__device__ int block_count_within(const Ctx& C, const int* c0, const int* nc, double d2max) {
  const TSet& S = *C.S;
  const int total = nc[0] * nc[1] * nc[2];
  int cnt = 0;
  for (int t = C.lane; t < total; t += 32) {
    const int k = t % nc[2], j = (t / nc[2]) % nc[1], i = t / (nc[1] * nc[2]);
    const int64_t g = S.cell0 + ((int64_t)(c0[0] + i) * S.dims[1] + (c0[1] + j)) * S.dims[2] + (c0[2] + k);
    const int e1 = __ldg(&C.cell_start[g + 1]);
    for (int e = __ldg(&C.cell_start[g]); e < e1; ++e) {
      const float4 x4 = __ldg(&C.sorted[e]);
      if (__float_as_int(x4.w) == C.p) continue;
      double d[3];
      rel(C, f3(x4), d);
      cnt += d[0] * d[0] + d[1] * d[1] + d[2] * d[2] < d2max;
    }
  }
  return __reduce_add_sync(0xffffffffu, cnt);
}

// One warp per vertex p: p's Delaunay star, certified; emits the tetrahedra
// whose smallest vertex is p.  Work is fetched from a global counter so that
// slow stars (near the convex hull) do not hold up a fixed share of vertices.
__global__ void __launch_bounds__(kWarps * 32, 3) k_tess_stars(StarArgs A) {
  extern __shared__ double s_dyn[];
  __shared__ int s_fill[kWarps];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* cx = s_dyn + (size_t)wid * 3 * kCandCap;
  double* cy = cx + kCandCap;
  double* cz = cy + kCandCap;
  int* cid = reinterpret_cast<int*>(s_dyn + (size_t)kWarps * 3 * kCandCap) + (size_t)wid * kCandCap;
  int4* tri = reinterpret_cast<int4*>(reinterpret_cast<int*>(s_dyn + (size_t)kWarps * 3 * kCandCap) +
                                      (size_t)kWarps * kCandCap) + (size_t)wid * kTriCap;
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
    C.cx = cx;
    C.cy = cy;
    C.cz = cz;
    C.cid = cid;
    C.p = p;
    C.lane = lane;
    C.bad = 0;
    C.stats = A.stats;
    for (int a = 0; a < 3; ++a) C.hi[a] = A.hi[3 * s + a];
    C.P = point(C, p);
    // ---- candidates: the points of the 5^3 cells around p's cell that lie
    // within R of p, R being the distance from p to the block's faces (or a
    // smaller radius holding at most kCandCap points, in dense clusters)
    const int lid = __ldg(&A.pcell[p]);
    const int ci[3] = {lid / (S.dims[1] * S.dims[2]), (lid / S.dims[2]) % S.dims[1], lid % S.dims[2]};
    const int rr = 2;
    int c0[3], nc[3];
    double R = kInf, corner2 = 0.0;
    {
      const double Pd[3] = {C.P.x, C.P.y, C.P.z};
      for (int a = 0; a < 3; ++a) {
        c0[a] = max(0, ci[a] - rr);
        nc[a] = min(S.dims[a] - 1, ci[a] + rr) - c0[a] + 1;
        if (ci[a] - rr > 0) R = fmin(R, Pd[a] - (S.lo[a] + (ci[a] - rr) * S.h));
        if (ci[a] + rr < S.dims[a] - 1) R = fmin(R, S.lo[a] + (ci[a] + rr + 1) * S.h - Pd[a]);
        double b0, b1, e0, e1;
        cell_box(S, C.hi, c0[a], a, b0, b1);
        cell_box(S, C.hi, c0[a] + nc[a] - 1, a, e0, e1);
        const double m = fmax(Pd[a] - b0, e1 - Pd[a]);
        corner2 += m * m;
      }
    }
    double thr2 = R < kInf ? R * R : corner2 * (1.0 + 1e-6);
    if (block_count_within(C, c0, nc, thr2) > kCandCap) {
      double lo2 = 0.0, hi2 = thr2;
      for (int it = 0; it < 32; ++it) {
        const double mid = 0.5 * (lo2 + hi2);
        if (block_count_within(C, c0, nc, mid) <= kCandCap) lo2 = mid;
        else hi2 = mid;
      }
      thr2 = lo2;
      R = fmin(R, sqrt(thr2) * (1.0 - 1e-12));
    }
    C.R = R - S.slack;
    if (lane == 0) s_fill[wid] = 0;
    __syncwarp();
    {
      const int total = nc[0] * nc[1] * nc[2];
      bool dup = false;
      for (int t = lane; t < total; t += 32) {
        const int k = t % nc[2], j = (t / nc[2]) % nc[1], i = t / (nc[1] * nc[2]);
        const int64_t g = S.cell0 + ((int64_t)(c0[0] + i) * S.dims[1] + (c0[1] + j)) * S.dims[2] + (c0[2] + k);
        const int e1 = __ldg(&A.cell_start[g + 1]);
        for (int e = __ldg(&A.cell_start[g]); e < e1; ++e) {
          const float4 x4 = __ldg(&A.sorted[e]);
          const int id = __float_as_int(x4.w);
          if (id == p) continue;
          double d[3];
          rel(C, f3(x4), d);
          const double d2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
          if (d2 == 0.0) dup = true;
          if (d2 < thr2) {
            const int slot = atomicAdd(&s_fill[wid], 1);
            if (slot < kCandCap) {
              cx[slot] = d[0];
              cy[slot] = d[1];
              cz[slot] = d[2];
              cid[slot] = id;
            }
          }
        }
      }
      __syncwarp();
      C.ncand = min(s_fill[wid], kCandCap);
      if (ballot(dup)) fail(C, kFlagDegenerate, kWhyDuplicate);  // duplicates of p stop the set
    }
    __syncwarp();
    // ---- nearest neighbour q (a Delaunay edge)
    int q = -1;
    if (!C.bad) {
      double bd = kInf;
      int bi = 0x7fffffff;
      for (int j = lane; j < C.ncand; j += 32) {
        const double d2 = cx[j] * cx[j] + cy[j] * cy[j] + cz[j] * cz[j];
        const int id = cid[j];
        if (d2 < bd || (d2 == bd && id < bi)) { bd = d2; bi = id; }
      }
      for (int off = 16; off; off >>= 1) {
        const double od = __shfl_xor_sync(0xffffffffu, bd, off);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
        if (od < bd || (od == bd && oi < bi)) { bd = od; bi = oi; }
      }
      if (bi != 0x7fffffff) q = bi;
    }
    // ---- r: smallest circumradius of (p, q, r)
    int r = -1;
    if (q >= 0) {
      double a[3];
      rel(C, point(C, q), a);
      const double la = a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
      double br = kInf;
      int bi = 0x7fffffff;
      for (int j = lane; j < C.ncand; j += 32) {
        const int id = cid[j];
        if (id == q) continue;
        const double b[3] = {cx[j], cy[j], cz[j]};
        const double ux = a[1] * b[2] - a[2] * b[1], uy = a[2] * b[0] - a[0] * b[2], uz = a[0] * b[1] - a[1] * b[0];
        const double cr = ux * ux + uy * uy + uz * uz;
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
      if (bi != 0x7fffffff) r = bi;
    }
    if (!C.bad && (q < 0 || r < 0)) fail(C, q < 0 ? kFlagCapacity : kFlagDegenerate, kWhyNoStart);
    // ---- first tetrahedron: (p, q, r) closed on either side
    int nt = 0;
    if (!C.bad) {
      int w = wrap(C, q, r, -1);
      if (w >= 0) {
        if (lane == 0) tri[0] = make_int4(q, r, w, 7);
        nt = 1;
      } else if (w == -1) {
        w = wrap(C, r, q, -1);
        if (w >= 0) {
          if (lane == 0) tri[0] = make_int4(r, q, w, 7);
          nt = 1;
        } else if (w == -1) {
          fail(C, kFlagDegenerate, kWhyFlat);  // every point on one plane
        }
      }
    }
    __syncwarp();
    // ---- grow the star across the open edges of its link; a triangle whose
    // edges are all closed stays closed, so the search starts at a cursor
    int cursor = 0;
    for (int iter = 0; !C.bad && iter < 3 * kTriCap + 8; ++iter) {
      int ft = -1, fe = 0;
      for (int t0 = cursor; t0 < nt; t0 += 32) {
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
      cursor = ft;
      const int4 T = tri[ft];
      int x, y;
      tri_edge(T, fe, x, y);
      const int c3 = fe == 0 ? T.z : (fe == 1 ? T.x : T.y);  // T's vertex off the crossed edge
      const int w = wrap(C, y, x, c3);
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
  if (n_sets < 1 || n_sets > 65535 || !vprefix)
    return dtfe_internal_set_error(DTFE_ERR_ARG, "dtfe_gpu_tessellate: need 1..65535 sets and vprefix");
  const int K = n_sets;
  if (vprefix[0] != 0) return dtfe_internal_set_error(DTFE_ERR_ARG, "dtfe_gpu_tessellate: vprefix[0] must be 0");
  int64_t maxn = 0;
  for (int s = 0; s < K; ++s) {
    if (vprefix[s + 1] < vprefix[s])
      return dtfe_internal_set_error(DTFE_ERR_ARG, "dtfe_gpu_tessellate: vprefix must not decrease");
    maxn = std::max<int64_t>(maxn, vprefix[s + 1] - vprefix[s]);
  }
  const int64_t V = vprefix[K];
  if (V > 0 && !xyz_dev) return dtfe_internal_set_error(DTFE_ERR_ARG, "dtfe_gpu_tessellate: xyz is NULL");
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
