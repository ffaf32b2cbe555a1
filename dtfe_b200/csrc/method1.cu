// Averaging method 1 on the GPU (sm_100a): quasi-random points inside every
// tetrahedron, each adding its interpolated fields, times its share of the
// tetrahedron's volume, to the grid cell it falls in; tetrahedra inside one
// cell add their vertex averages times their volume; every cell is divided
// by the cell volume (interpolateGrid_averaged_1,
// src/CGAL_triangulation/averaged_interpolation_1.cc:197-421).
//
// The reference scatters in tetrahedron order with float `+=`.  Here the
// scatter becomes a gather, so each cell sums its contributions in that same
// order, in the same float arithmetic, without atomics:
//   k_m1_cells<FILL>  one thread per tetrahedron: its points' cells (a
//                     64-bit mask over a 4x4x4 window around the first hit,
//                     else the range of all hits); FILL = 0 counts the
//                     (cell, tetrahedron) pairs per cell, FILL = 1 writes the
//                     tetrahedron into each cell's list
//   k_m1_sort         each cell's list into ascending tetrahedron order
//   k_m1_gather<S>    one thread per cell: for its tetrahedra in order, the
//                     single-cell contribution or the points that fall in
//                     the cell; then / cell volume, derived fields, stores
// Points come from a table of the first 100 NN Sobol points of the corner
// simplex (sobol.h), made on the host once per NN.
#include <cuda_runtime.h>
#include <cub/device/device_scan.cuh>

#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/dtfe_gpu.h"
#include "dtfe_device.cuh"
#include "sobol.h"
#include "tile_index.cuh"

extern "C" int dtfe_internal_set_error(int code, const char* msg);

namespace {

using namespace dtfe;

inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

struct M1Box {
  float lo[3], hi[3], dx[3];
  double inv_dx[3];  // 1 / dx in double (cell test fast path)
  int n[3];
  float gcv;  // dx0 dx1 dx2 in float
  int64_t tile;  // first flattened sample of the tile
  int64_t G;     // cells of the tile
};

struct M1Params {
  const int4* tet_v;
  const float4* posd;  // xyz, vertex density in .w
  const float4* vel4;
  const float* scal;
  const M1Box* boxes;
  const int64_t* tet_prefix;  // K + 1
  const dtfe_subbox* sub;
  const double* table;  // 3 per point: the float Sobol values, held as doubles
  int K, NN, fix;
  int64_t T, n_cells, G1, G2;
  uint32_t fields;
  float* out[DTFE_NUM_FIELDS];
};

__device__ __forceinline__ int m1_find_box(const int64_t* __restrict__ prefix, int K, int64_t s) {
  int lo = 0, hi = K;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(&prefix[mid]) <= s) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Per-tetrahedron setup of checkCellPosition, volume and point count
// (averaged_interpolation_1.cc:84-118, :276-282, :322-325).
struct M1Tet {
  double vM[3][3];
  float bp[3];
  float vol, factor;
  int np;      // points (0 for a single-cell tetrahedron)
  int one[3];  // its cell when single
};

// false: the tetrahedron's bounding box misses the region (cellOutsideRegion)
__device__ __forceinline__ bool m1_setup(const float X[4][3], const M1Box& B, int NN, M1Tet& m) {
  bool outside = false;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float mn = fminf(fminf(X[0][c], X[1][c]), fminf(X[2][c], X[3][c]));
    const float mx = fmaxf(fmaxf(X[0][c], X[1][c]), fmaxf(X[2][c], X[3][c]));
    outside = outside || mn > B.hi[c] || mx < B.lo[c];
  }
  if (outside) return false;
  int bc[3];
  bool one = true;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    m.bp[c] = (float)((double)X[0][c] - (double)B.lo[c]);
    bc[c] = (int)floorf(m.bp[c] / B.dx[c]);
    const float gl = (float)bc[c] * B.dx[c] + B.lo[c];
    const float gh = gl + B.dx[c];
#pragma unroll
    for (int a = 1; a < 4; ++a) one = one && X[a][c] >= gl && X[a][c] <= gh;
    one = one && bc[c] >= 0 && bc[c] < B.n[c];
  }
  double D[4][3];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) D[a][c] = (double)X[a][c];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) m.vM[r][c] = D[r + 1][c] - D[0][c];
  m.vol = (float)(orient_det(D[0], D[1], D[2], D[3]) / 6.0);
  if (one) {
    m.np = 0;
    m.one[0] = bc[0];
    m.one[1] = bc[1];
    m.one[2] = bc[2];
    m.factor = 0.f;
    return true;
  }
  const long long maxNN = 100LL * NN, minNN = NN / 6 + 1;
  const float ratio = m.vol / B.gcv;
  const long long tempInt = (long long)((float)NN * m.vol / B.gcv) + 1;
  m.np = (int)(ratio > (float)(1. / 6.) ? (tempInt > maxNN ? maxNN : tempInt) : minNN);
  m.factor = m.vol / (float)m.np;
  return true;
}

__device__ __forceinline__ void m1_point(const M1Tet& m, const double* __restrict__ table, int i, double p[3]) {
  const double q0 = __ldg(&table[3 * i]), q1 = __ldg(&table[3 * i + 1]), q2 = __ldg(&table[3 * i + 2]);
#pragma unroll
  for (int c = 0; c < 3; ++c) p[c] = q0 * m.vM[0][c] + q1 * m.vM[1][c] + q2 * m.vM[2][c];
}

// floor(x / d) with x / d rounded as IEEE division: from x * (1/d) unless
// that product lies within 1e-9 (relative) of an integer, where the rounded
// quotient could fall on the other side; then by the division itself.
__device__ __forceinline__ double floor_div(double x, double d, double inv) {
  const double q = x * inv;
  const double f = floor(q);
  const double frac = q - f;  // exact
  const double tol = 1e-9 * fmax(fabs(q), 1.0);
  if (frac <= tol || frac >= 1.0 - tol) return floor(x / d);
  return f;
}

// isGridCellIndex (:140-157): floor((basePosition + p) / dx) per axis
__device__ __forceinline__ bool m1_cell(const M1Tet& m, const M1Box& B, const double p[3], int cell[3]) {
  bool ok = true;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double f = floor_div((double)m.bp[c] + p[c], (double)B.dx[c], B.inv_dx[c]);
    ok = ok && f >= 0.0 && f < (double)B.n[c];
    cell[c] = ok ? (int)f : 0;
  }
  return ok;
}

__device__ __forceinline__ void load_tet_f(const M1Params& P, int64_t t, int v[4], float X[4][3]) {
  const int4 q = __ldg(&P.tet_v[t]);
  v[0] = q.x;
  v[1] = q.y;
  v[2] = q.z;
  v[3] = q.w;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const float4 r = __ldg(&P.posd[v[a]]);
    X[a][0] = r.x;
    X[a][1] = r.y;
    X[a][2] = r.z;
  }
}

// Cells receiving a tetrahedron's contributions: emit(flattened sample,
// point mask) once per cell.  The mask marks the points (of at most 64) that
// fall in the cell; 0 means "test every point" (single-cell tetrahedra, more
// than 64 points, or a tetrahedron wider than the 4x4x4 window, whose range
// of hit cells is emitted: a superset).
constexpr int kMaskPoints = 64;
template <class Emit>
__device__ __forceinline__ void m1_for_cells(const M1Params& P, int b, const M1Tet& m, Emit emit) {
  const M1Box& B = P.boxes[b];
  if (m.np == 0) {
    emit(B.tile + ((int64_t)m.one[0] * B.n[1] + m.one[1]) * B.n[2] + m.one[2], 0ull);
    return;
  }
  unsigned long long cells = 0ull;
  unsigned char win[kMaskPoints];
  int ref[3] = {0, 0, 0}, lo[3] = {0, 0, 0}, hi[3] = {-1, -1, -1};
  bool any = false, wide = false;
  const bool masks = m.np <= kMaskPoints;
  for (int i = 0; i < m.np; ++i) {
    double p[3];
    m1_point(m, P.table, i, p);
    int c[3];
    unsigned char w = 0xFF;
    if (m1_cell(m, B, p, c)) {
      if (!any) {
        any = true;
#pragma unroll
        for (int a = 0; a < 3; ++a) ref[a] = lo[a] = hi[a] = c[a];
      }
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        lo[a] = min(lo[a], c[a]);
        hi[a] = max(hi[a], c[a]);
      }
      const int ox = c[0] - ref[0] + 1, oy = c[1] - ref[1] + 1, oz = c[2] - ref[2] + 1;
      if (ox < 0 || ox > 3 || oy < 0 || oy > 3 || oz < 0 || oz > 3) {
        wide = true;
      } else {
        w = (unsigned char)(ox * 16 + oy * 4 + oz);
        cells |= 1ull << w;
      }
    }
    if (masks) win[i] = w;
  }
  if (!any) return;
  if (!wide) {
    while (cells) {
      const int bit = __ffsll((long long)cells) - 1;
      cells &= cells - 1;
      unsigned long long pm = 0ull;
      if (masks)
        for (int i = 0; i < m.np; ++i) pm |= (win[i] == bit ? 1ull : 0ull) << i;
      const int ci = ref[0] + (bit >> 4) - 1, cj = ref[1] + ((bit >> 2) & 3) - 1, ck = ref[2] + (bit & 3) - 1;
      emit(B.tile + ((int64_t)ci * B.n[1] + cj) * B.n[2] + ck, pm);
    }
    return;
  }
  for (int ci = lo[0]; ci <= hi[0]; ++ci)
    for (int cj = lo[1]; cj <= hi[1]; ++cj)
      for (int ck = lo[2]; ck <= hi[2]; ++ck) emit(B.tile + ((int64_t)ci * B.n[1] + cj) * B.n[2] + ck, 0ull);
}

// list entries: {tetrahedron, point mask}, sorted by tetrahedron
template <int FILL>
__global__ void __launch_bounds__(256) k_m1_cells(M1Params P, unsigned long long* __restrict__ cnt,
                                                  const int64_t* __restrict__ off, ulonglong2* __restrict__ list) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= P.T) return;
  if (t < __ldg(&P.tet_prefix[0]) || t >= __ldg(&P.tet_prefix[P.K])) return;
  const int b = m1_find_box(P.tet_prefix, P.K, t);
  int v[4];
  float X[4][3];
  load_tet_f(P, t, v, X);
  M1Tet m;
  if (!m1_setup(X, P.boxes[b], P.NN, m)) return;
  m1_for_cells(P, b, m, [&](int64_t s, unsigned long long pm) {
    if (FILL) {
      const unsigned long long k = atomicAdd(&cnt[s], 1ull);
      list[off[s] + (int64_t)k] = make_ulonglong2((unsigned long long)t, pm);
    } else {
      atomicAdd(&cnt[s], 1ull);
    }
  });
}

__global__ void k_m1_sort(int64_t n, const int64_t* __restrict__ off, ulonglong2* __restrict__ list) {
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int64_t a = off[s], e = off[s + 1];
  for (int64_t i = a + 1; i < e; ++i) {
    const ulonglong2 x = list[i];
    int64_t j = i - 1;
    while (j >= a && list[j].x > x.x) {
      list[j + 1] = list[j];
      --j;
    }
    list[j + 1] = x;
  }
}

template <int S>
__global__ void __launch_bounds__(128) k_m1_gather(M1Params P, const int64_t* __restrict__ off,
                                                   const ulonglong2* __restrict__ list) {
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= P.n_cells) return;
  // the cell of flattened sample s (tile order: sub-box, then x, y, z fastest)
  int b = 0;
  {
    int lo = 0, hi = P.K;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (P.boxes[mid].tile <= s) lo = mid;
      else hi = mid;
    }
    b = lo;
  }
  const M1Box& B = P.boxes[b];
  const int64_t local = s - B.tile;
  int ci, cj, ck;
  tile_ijk(local, B.n[1], B.n[2], ci, cj, ck);
  const bool fix = P.fix != 0;
  const bool has_vel = P.vel4 != nullptr;
  float aD = 0.f, aV[3] = {0.f, 0.f, 0.f}, aG[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  float aS[S > 0 ? S : 1], aSG[S > 0 ? 3 * S : 1];
#pragma unroll
  for (int q = 0; q < (S > 0 ? S : 1); ++q) aS[q] = 0.f;
#pragma unroll
  for (int q = 0; q < (S > 0 ? 3 * S : 1); ++q) aSG[q] = 0.f;
  for (int64_t e = off[s]; e < off[s + 1]; ++e) {
    const ulonglong2 pair = list[e];
    const int t = (int)pair.x;
    const unsigned long long pm = pair.y;
    int v[4];
    float X[4][3];
    load_tet_f(P, t, v, X);
    M1Tet m;
    if (!m1_setup(X, B, P.NN, m)) continue;
    // gradients (densityGrad, velocityGrad, scalarGrad; unaveraged_interpolation.cc:66-173)
    float M[3][3];
    matrix_inverse_f(m.vM, M);
    float dn[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) dn[a] = __ldg(&P.posd[v[a]]).w;
    float gr[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      float acc = 0.f;
#pragma unroll
      for (int j = 0; j < 3; ++j) acc += M[i][j] * (dn[j + 1] - dn[0]);
      gr[i] = acc;
    }
    float vv[4][3] = {};
    float VG[3][3] = {};
    if (has_vel) {
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        const float4 w = __ldg(&P.vel4[v[a]]);
        vv[a][0] = w.x;
        vv[a][1] = w.y;
        vv[a][2] = w.z;
      }
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          float acc = 0.f;
#pragma unroll
          for (int k = 0; k < 3; ++k) acc += M[i][k] * (vv[k + 1][j] - vv[0][j]);
          VG[i][j] = acc;
        }
    }
    float ss[4][S > 0 ? S : 1];
    float SG[S > 0 ? S : 1][3];
#pragma unroll
    for (int q = 0; q < S; ++q) {
#pragma unroll
      for (int a = 0; a < 4; ++a) ss[a][q] = __ldg(&P.scal[(int64_t)S * v[a] + q]);
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        float acc = 0.f;
#pragma unroll
        for (int k = 0; k < 3; ++k) acc += M[i][k] * (ss[k + 1][q] - ss[0][q]);
        SG[q][i] = acc;
      }
    }
    if (m.np == 0) {
      // the whole tetrahedron in this cell: vertex averages times the volume
      float a = 0.f;
#pragma unroll
      for (int k = 0; k < 4; ++k) a += dn[k];
      aD += (a / 4.f) * m.vol;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float av = 0.f;
#pragma unroll
        for (int k = 0; k < 4; ++k) av += vv[k][c];
        aV[c] += (av / 4.f) * m.vol;
      }
#pragma unroll
      for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int i = 0; i < 3; ++i) aG[j * 3 + i] += VG[i][j] * m.vol;
#pragma unroll
      for (int q = 0; q < S; ++q) {
        float as = 0.f;
#pragma unroll
        for (int k = 0; k < 4; ++k) as += ss[k][q];
        aS[q] += (as / 4.f) * m.vol;
#pragma unroll
        for (int i = 0; i < 3; ++i) aSG[3 * q + i] += SG[q][i] * m.vol;
      }
      continue;
    }
    // the gradients in double once per tetrahedron (the point products below
    // are double products of these float values)
    const double grd[3] = {(double)gr[0], (double)gr[1], (double)gr[2]};
    double VGd[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) VGd[i][j] = (double)VG[i][j];
    double SGd[S > 0 ? S : 1][3];
#pragma unroll
    for (int q = 0; q < S; ++q)
#pragma unroll
      for (int j = 0; j < 3; ++j) SGd[q][j] = (double)SG[q][j];
    // one point's contribution (densityValue, velocityValue, scalarValue and
    // the gradients, each times vol / n; :336-355)
    auto add_point = [&](const double p[3]) {
      const float f = m.factor;
      const float temp = (float)(p[0] * grd[0] + p[1] * grd[1] + p[2] * grd[2]);
      aD += (dn[0] + temp) * f;
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) {
        float tmp = 0.f;
        if (fix) {
#pragma unroll
          for (int j = 0; j < 3; ++j) tmp = (float)((double)tmp + VGd[j][cc] * p[j]);
        } else {
          tmp = (float)(VGd[2][cc] * p[2]);
        }
        aV[cc] += (tmp + vv[0][cc]) * f;
      }
#pragma unroll
      for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) aG[j * 3 + cc] += VG[cc][j] * f;
#pragma unroll
      for (int q = 0; q < S; ++q) {
        float tmp = 0.f;
        if (fix) {
#pragma unroll
          for (int j = 0; j < 3; ++j) tmp = (float)((double)tmp + SGd[q][j] * p[j]);
        } else {
          tmp = (float)(SGd[q][2] * p[2]);
        }
        aS[q] += (tmp + ss[0][q]) * f;
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) aSG[3 * q + cc] += SG[q][cc] * f;
      }
    };
    // the points in this cell, in ascending order: the mask's, else every
    // point that tests into the cell
    if (pm) {
      for (unsigned long long r = pm; r; r &= r - 1) {
        double p[3];
        m1_point(m, P.table, __ffsll((long long)r) - 1, p);
        add_point(p);
      }
    } else {
      for (int i = 0; i < m.np; ++i) {
        double p[3];
        m1_point(m, P.table, i, p);
        int c[3];
        if (m1_cell(m, B, p, c) && c[0] == ci && c[1] == cj && c[2] == ck) add_point(p);
      }
    }
  }
  // divide by the cell volume (:371-393) and store in the Quantities layout
  const float g = B.gcv;
  const dtfe_subbox& sb = P.sub[b];
  const int64_t cell = ((int64_t)(sb.tile_origin[0] + ci) * P.G1 + (sb.tile_origin[1] + cj)) * P.G2 +
                       (sb.tile_origin[2] + ck);
  const uint32_t F = P.fields;
  float gd[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) gd[q] = aG[q] / g;
  if (F & DTFE_FIELD_BIT(DTFE_DENSITY)) P.out[DTFE_DENSITY][cell] = aD / g;
  if (F & DTFE_FIELD_BIT(DTFE_VELOCITY))
#pragma unroll
    for (int c = 0; c < 3; ++c) P.out[DTFE_VELOCITY][3 * cell + c] = aV[c] / g;
  if (F & DTFE_FIELD_BIT(DTFE_VELOCITY_GRADIENT))
#pragma unroll
    for (int q = 0; q < 9; ++q) P.out[DTFE_VELOCITY_GRADIENT][9 * cell + q] = gd[q];
  if (F & (DTFE_FIELD_BIT(DTFE_VELOCITY_DIVERGENCE) | DTFE_FIELD_BIT(DTFE_VELOCITY_SHEAR) |
           DTFE_FIELD_BIT(DTFE_VELOCITY_VORTICITY))) {
    float dv, sh[5], vo[3];
    derived_fields(gd, dv, sh, vo);
    if (F & DTFE_FIELD_BIT(DTFE_VELOCITY_DIVERGENCE)) P.out[DTFE_VELOCITY_DIVERGENCE][cell] = dv;
    if (F & DTFE_FIELD_BIT(DTFE_VELOCITY_SHEAR))
#pragma unroll
      for (int q = 0; q < 5; ++q) P.out[DTFE_VELOCITY_SHEAR][5 * cell + q] = sh[q];
    if (F & DTFE_FIELD_BIT(DTFE_VELOCITY_VORTICITY))
#pragma unroll
      for (int q = 0; q < 3; ++q) P.out[DTFE_VELOCITY_VORTICITY][3 * cell + q] = vo[q];
  }
  if (S > 0 && (F & DTFE_FIELD_BIT(DTFE_SCALAR)))
#pragma unroll
    for (int q = 0; q < S; ++q) P.out[DTFE_SCALAR][(int64_t)S * cell + q] = aS[q] / g;
  if (S > 0 && (F & DTFE_FIELD_BIT(DTFE_SCALAR_GRADIENT)))
#pragma unroll
    for (int q = 0; q < 3 * S; ++q) P.out[DTFE_SCALAR_GRADIENT][(int64_t)3 * S * cell + q] = aSG[q] / g;
}

template <int S>
void launch_gather(const M1Params& P, const int64_t* off, const ulonglong2* list, cudaStream_t st) {
  const unsigned nb = (unsigned)((P.n_cells + 127) / 128);
  k_m1_gather<S><<<nb, 128, 0, st>>>(P, off, list);
}

}  // namespace

// Method 1 over every sub-box of the handle's tessellation into the device
// outputs out[] (main grid, Quantities layout).  regions: 6 floats per
// sub-box on the host.  *table / *table_nn cache the device point table;
// *scratch / *scratch_bytes the work buffers and *lists / *lists_bytes the
// per-cell tetrahedron lists (both grown as needed).  Waits once on the
// stream for the number of (cell, tetrahedron) pairs, so it cannot be
// captured into a graph.
extern "C" int dtfe_internal_method1(void* stream, int K, const dtfe_subbox* boxes_h, const dtfe_subbox* boxes_d,
                                     const float* regions_h, int64_t n_cells, int64_t G1, int64_t G2, int64_t T,
                                     const int4* tet_v, const float4* posd, const float4* vel4, const float* scal,
                                     int S, int NN, uint32_t fields, int fix, float* const out[DTFE_NUM_FIELDS],
                                     double** table, int* table_nn, void** scratch, size_t* scratch_bytes,
                                     void** lists, size_t* lists_bytes) {
  cudaStream_t st = (cudaStream_t)stream;
  if (NN < 1 || NN > (1 << 20)) return dtfe_internal_set_error(DTFE_ERR_ARG, "method 1 needs 1..2^20 points per cell");
  if (S < 0 || S > 8) return dtfe_internal_set_error(DTFE_ERR_ARG, "method 1 supports at most 8 scalars");
  // point table (first 100 NN simplex points)
  if (*table_nn != NN) {
    const size_t np = 100 * (size_t)NN;
    std::vector<float> hf(3 * np);
    sobol_simplex_table(np, hf.data());
    std::vector<double> h(hf.begin(), hf.end());  // exact: the reference multiplies these floats in double
    if (*table) cudaFree(*table);
    *table = nullptr;
    *table_nn = 0;
    if (cudaMalloc((void**)table, sizeof(double) * h.size()) != cudaSuccess)
      return dtfe_internal_set_error(DTFE_ERR_ALLOC, "cudaMalloc (method-1 points)");
    if (cudaMemcpyAsync(*table, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return dtfe_internal_set_error(DTFE_ERR_CUDA, "uploading the method-1 points");
    *table_nn = NN;
  }
  std::vector<M1Box> mb(K);
  std::vector<int64_t> tpre(K + 1);
  int64_t tile = 0;
  for (int b = 0; b < K; ++b) {
    const dtfe_subbox& s = boxes_h[b];
    M1Box& B = mb[b];
    for (int c = 0; c < 3; ++c) {
      B.lo[c] = regions_h[6 * b + 2 * c];
      B.hi[c] = regions_h[6 * b + 2 * c + 1];
      B.dx[c] = s.dx[c];
      B.n[c] = s.tile_dims[c];
    }
    B.gcv = B.dx[0] * B.dx[1] * B.dx[2];
    for (int c = 0; c < 3; ++c) B.inv_dx[c] = 1.0 / (double)B.dx[c];
    B.tile = tile;
    B.G = (int64_t)B.n[0] * B.n[1] * B.n[2];
    tile += B.G;
    tpre[b] = s.tet_offset;
  }
  tpre[K] = boxes_h[K - 1].tet_offset + boxes_h[K - 1].n_tets;
  if (tile != n_cells) return dtfe_internal_set_error(DTFE_ERR_STATE, "sub-box tiles do not cover the samples");
  // work buffers: boxes, tetrahedron prefix, counts, offsets, scan scratch;
  // the pair lists are sized after counting
  size_t cub_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, cub_bytes, (unsigned long long*)nullptr, (int64_t*)nullptr,
                                (int64_t)(n_cells + 1), st);
  const size_t fixed[] = {sizeof(M1Box) * K, sizeof(int64_t) * (K + 1), sizeof(unsigned long long) * (n_cells + 1),
                          sizeof(int64_t) * (n_cells + 1), cub_bytes};
  size_t need = 0;
  for (size_t q : fixed) need += align256(q);
  if (*scratch_bytes < need) {
    if (*scratch) cudaFree(*scratch);
    *scratch = nullptr;
    *scratch_bytes = 0;
    if (cudaMalloc(scratch, need) != cudaSuccess)
      return dtfe_internal_set_error(DTFE_ERR_ALLOC, "cudaMalloc (method-1 work buffers)");
    *scratch_bytes = need;
  }
  char* p = (char*)*scratch;
  M1Box* d_boxes = (M1Box*)p;
  p += align256(fixed[0]);
  int64_t* d_tpre = (int64_t*)p;
  p += align256(fixed[1]);
  unsigned long long* d_cnt = (unsigned long long*)p;
  p += align256(fixed[2]);
  int64_t* d_off = (int64_t*)p;
  p += align256(fixed[3]);
  void* d_cub = p;
  if (cudaMemcpyAsync(d_boxes, mb.data(), sizeof(M1Box) * K, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(d_tpre, tpre.data(), sizeof(int64_t) * (K + 1), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long) * (n_cells + 1), st) != cudaSuccess)
    return dtfe_internal_set_error(DTFE_ERR_CUDA, "method-1 setup copies");
  M1Params P;
  P.tet_v = tet_v;
  P.posd = posd;
  P.vel4 = vel4;
  P.scal = scal;
  P.boxes = d_boxes;
  P.tet_prefix = d_tpre;
  P.sub = boxes_d;
  P.table = *table;
  P.K = K;
  P.NN = NN;
  P.fix = fix;
  P.T = T;
  P.n_cells = n_cells;
  P.G1 = G1;
  P.G2 = G2;
  P.fields = fields;
  for (int q = 0; q < DTFE_NUM_FIELDS; ++q) P.out[q] = out[q];
  const unsigned tb = (unsigned)((T + 255) / 256);
  if (T > 0) k_m1_cells<0><<<tb, 256, 0, st>>>(P, d_cnt, nullptr, nullptr);
  if (cub::DeviceScan::ExclusiveSum(d_cub, cub_bytes, d_cnt, d_off, (int64_t)(n_cells + 1), st) != cudaSuccess)
    return dtfe_internal_set_error(DTFE_ERR_CUDA, "method-1 scan");
  int64_t pairs = 0;
  if (cudaMemcpyAsync(&pairs, d_off + n_cells, sizeof(int64_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return dtfe_internal_set_error(DTFE_ERR_CUDA, "method-1 pair count");
  // the (cell, tetrahedron) lists in their own buffer
  const size_t list_bytes = sizeof(ulonglong2) * (size_t)(pairs > 0 ? pairs : 1);
  if (*lists_bytes < list_bytes) {
    if (*lists) cudaFree(*lists);
    *lists = nullptr;
    *lists_bytes = 0;
    if (cudaMalloc(lists, list_bytes) != cudaSuccess)
      return dtfe_internal_set_error(DTFE_ERR_ALLOC, "cudaMalloc (method-1 lists)");
    *lists_bytes = list_bytes;
  }
  ulonglong2* d_list = (ulonglong2*)*lists;
  if (cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long) * (n_cells + 1), st) != cudaSuccess)
    return dtfe_internal_set_error(DTFE_ERR_CUDA, "method-1 fill reset");
  if (T > 0) k_m1_cells<1><<<tb, 256, 0, st>>>(P, d_cnt, d_off, d_list);
  const unsigned cb = (unsigned)((n_cells + 255) / 256);
  if (n_cells > 0) k_m1_sort<<<cb, 256, 0, st>>>(n_cells, d_off, d_list);
  switch (S) {
    case 0: launch_gather<0>(P, d_off, d_list, st); break;
    case 1: launch_gather<1>(P, d_off, d_list, st); break;
    case 2: launch_gather<2>(P, d_off, d_list, st); break;
    case 3: launch_gather<3>(P, d_off, d_list, st); break;
    case 4: launch_gather<4>(P, d_off, d_list, st); break;
    case 5: launch_gather<5>(P, d_off, d_list, st); break;
    case 6: launch_gather<6>(P, d_off, d_list, st); break;
    case 7: launch_gather<7>(P, d_off, d_list, st); break;
    default: launch_gather<8>(P, d_off, d_list, st); break;
  }
  if (cudaGetLastError() != cudaSuccess) return dtfe_internal_set_error(DTFE_ERR_CUDA, "method-1 launch");
  return DTFE_OK;
}
