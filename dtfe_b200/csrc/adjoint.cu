// Adjoint of the DTFE density / velocity-divergence grids and of the CIC /
// TSC density grids with respect to vertex (particle) positions, velocities
// and weights, at fixed tessellation topology and fixed sample->tetrahedron
// assignment.  The reference has no gradients; this is the backward half of
// the autograd function in dtfe_b200/autograd.py.
//
// Loss L = sum_c a_c rho(p_c) + c_c . vel(p_c) + b_c div(p_c), with a, c, b
// the gradients of L with respect to the density, velocity and divergence
// grids.  For a cell c in tetrahedron t (vertices 0..3, edge matrix A with
// rows x_k - x_0, offset r = p - x_0):
//   rho(p) = rho_0 + r . A^-1 drho,           drho_k = rho_k - rho_0,
//   VG = A^-1 DV,                              DV[k][i] = v_{k,i} - v_{0,i},
//   vel_i(p) = v_0i + sum_j u_j r_j VG[j][i]   (u = (1,1,1), or (0,0,1): the
//              reference's value evaluation, unaveraged_interpolation.cc:116),
//   div = tr VG.
// Reverse mode accumulates dL/dA^-1 and dL/dr per cell, then
// dL/dA = -A^-T (dL/dA^-1) A^-T and dL/dx_0 = -dL/dr - sum_k dL/dA[k].
// Vertex densities rho_v = 4 m_v / (rho_bar S_v), S_v = sum of incident
// volumes:  dL/dm_v = rhobar_v rho_v / m_v,  dL/dS_v = -rhobar_v rho_v / S_v,
// and each tetrahedron passes Vbar_t = sum_{v in t} dL/dS_v on to its
// vertices through dV_t/dx_j.
//
// Per-cell terms are evaluated in FP64 and scattered with FP64 atomics; S_v
// is the forward pass's exact volume sum (fixed_volume.cuh) and the volume
// term is gathered per vertex over the incidence lists (no atomics).
// Tetrahedra whose edge matrix the forward pass treats as singular
// (|det| / sum|M| <= 1e-6, triangulation_miscellaneous.cc:86-94) have zero
// gradient fields, so only the rho_0 term remains.

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/dtfe_gpu.h"
#include "fixed_volume.cuh"
#include "tile_index.cuh"
#include "predicates.h"

namespace {

struct AdjCellParams {
  const int4* tet_v;
  const float4* posd;   // x, y, z, vertex density
  const float4* vel4;
  const int* tet_c;     // located tetrahedron per flattened sample
  const dtfe_subbox* boxes;
  const int64_t* tile_prefix;
  const float* xs;
  const float* ys;
  const float* zs;
  int K;
  int64_t G1, G2, n_total;
  const float* a;       // dL/d density grid (main-grid layout) or null
  const float* b;       // dL/d divergence grid or null
  const float* c;       // dL/d velocity grid (3 per cell) or null
  float u[3];           // which offset terms the velocity value uses (1, 1, 1) or (0, 0, 1)
  double* g_rho;        // V: dL/d rho_v
  double* g_x;          // 3V
  double* g_v;          // 3V
};

__device__ __forceinline__ int find_box_a(const int64_t* __restrict__ prefix, int K, int64_t s) {
  int lo = 0, hi = K;
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (__ldg(&prefix[mid]) <= s) lo = mid;
    else hi = mid;
  }
  return lo;
}

// 3x3 inverse by the adjugate, or zero when the forward pass treats the
// matrix as singular.
__device__ __forceinline__ bool inverse3(const double A[3][3], double Mi[3][3]) {
  double c[3][3];
  c[0][0] = A[1][1] * A[2][2] - A[1][2] * A[2][1];
  c[0][1] = A[1][2] * A[2][0] - A[1][0] * A[2][2];
  c[0][2] = A[1][0] * A[2][1] - A[1][1] * A[2][0];
  c[1][0] = A[0][2] * A[2][1] - A[0][1] * A[2][2];
  c[1][1] = A[0][0] * A[2][2] - A[0][2] * A[2][0];
  c[1][2] = A[0][1] * A[2][0] - A[0][0] * A[2][1];
  c[2][0] = A[0][1] * A[1][2] - A[0][2] * A[1][1];
  c[2][1] = A[0][2] * A[1][0] - A[0][0] * A[1][2];
  c[2][2] = A[0][0] * A[1][1] - A[0][1] * A[1][0];
  const double det = A[0][0] * c[0][0] + A[0][1] * c[0][1] + A[0][2] * c[0][2];
  double s = 0;
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int q = 0; q < 3; ++q) s += fabs(A[r][q]);
  const bool ok = fabs(det / s) > 1.e-6;
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int q = 0; q < 3; ++q) Mi[r][q] = ok ? c[q][r] / det : 0.0;
  return ok;
}

__global__ void k_adjoint_cells(AdjCellParams P) {
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= P.n_total) return;
  const int t = P.tet_c[s];
  if (t < 0) return;  // outside the hull: the forward value is a constant 0
  const int b = find_box_a(P.tile_prefix, P.K, s);
  const dtfe_subbox& B = P.boxes[b];
  const int64_t local = s - P.tile_prefix[b];
  const int nz = B.tile_dims[2], ny = B.tile_dims[1];
  int i, j, k;
  tile_ijk(local, ny, nz, i, j, k);
  const int64_t cell = ((int64_t)(B.tile_origin[0] + i) * P.G1 + (B.tile_origin[1] + j)) * P.G2 + (B.tile_origin[2] + k);
  const double wa = P.a ? (double)P.a[cell] : 0.0;
  const double wb = P.b ? (double)P.b[cell] : 0.0;
  double wc[3] = {0.0, 0.0, 0.0};
  if (P.c)
#pragma unroll
    for (int q = 0; q < 3; ++q) wc[q] = (double)P.c[3 * cell + q];
  const bool has_v = wb != 0.0 || wc[0] != 0.0 || wc[1] != 0.0 || wc[2] != 0.0;
  if (wa == 0.0 && !has_v) return;
  const double p[3] = {(double)P.xs[B.coord_offset[0] + i], (double)P.ys[B.coord_offset[1] + j],
                       (double)P.zs[B.coord_offset[2] + k]};
  const int4 q4 = P.tet_v[t];
  const int v[4] = {q4.x, q4.y, q4.z, q4.w};
  double X[4][3], rho[4];
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const float4 r = P.posd[v[a]];
    X[a][0] = r.x; X[a][1] = r.y; X[a][2] = r.z;
    rho[a] = r.w;
  }
  double A[3][3], Mi[3][3];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) A[r][c] = X[r + 1][c] - X[0][c];
  inverse3(A, Mi);
  const double rel[3] = {p[0] - X[0][0], p[1] - X[0][1], p[2] - X[0][2]};
  double gAi[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};  // dL / d(A^-1)
  double grel[3] = {0, 0, 0};                            // dL / d(p - x_0)
  if (wa != 0.0) {
    // density = rho_0 + rel . g,  g = A^-1 drho
    double dr[3] = {rho[1] - rho[0], rho[2] - rho[0], rho[3] - rho[0]}, G[3], gd[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const double g = Mi[r][0] * dr[0] + Mi[r][1] * dr[1] + Mi[r][2] * dr[2];
      G[r] = wa * rel[r];
      grel[r] += wa * g;
    }
    double gsum = 0.0;
#pragma unroll
    for (int kk = 0; kk < 3; ++kk) {
      gd[kk] = Mi[0][kk] * G[0] + Mi[1][kk] * G[1] + Mi[2][kk] * G[2];
      gsum += gd[kk];
      atomicAdd(&P.g_rho[v[kk + 1]], gd[kk]);
    }
    atomicAdd(&P.g_rho[v[0]], wa - gsum);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int kk = 0; kk < 3; ++kk) gAi[r][kk] += G[r] * dr[kk];
  }
  if (has_v) {
    // velocity_i = v_0i + sum_j u_j rel_j VG[j][i],  divergence = tr VG,
    // VG = A^-1 DV
    double DV[3][3], VG[3][3], GV[3][3];
    const float4 u0 = P.vel4[v[0]];
#pragma unroll
    for (int kk = 0; kk < 3; ++kk) {
      const float4 u = P.vel4[v[kk + 1]];
      DV[kk][0] = (double)u.x - u0.x;
      DV[kk][1] = (double)u.y - u0.y;
      DV[kk][2] = (double)u.z - u0.z;
    }
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) VG[r][c] = Mi[r][0] * DV[0][c] + Mi[r][1] * DV[1][c] + Mi[r][2] * DV[2][c];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const double ur = (double)P.u[r] * rel[r];
      grel[r] += (double)P.u[r] * (wc[0] * VG[r][0] + wc[1] * VG[r][1] + wc[2] * VG[r][2]);
#pragma unroll
      for (int c = 0; c < 3; ++c) GV[r][c] = ur * wc[c] + (r == c ? wb : 0.0);
    }
    double g0[3] = {wc[0], wc[1], wc[2]};
#pragma unroll
    for (int kk = 0; kk < 3; ++kk)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double gdv = Mi[0][kk] * GV[0][c] + Mi[1][kk] * GV[1][c] + Mi[2][kk] * GV[2][c];
        atomicAdd(&P.g_v[3 * (int64_t)v[kk + 1] + c], gdv);
        g0[c] -= gdv;
      }
#pragma unroll
    for (int c = 0; c < 3; ++c) atomicAdd(&P.g_v[3 * (int64_t)v[0] + c], g0[c]);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int kk = 0; kk < 3; ++kk) gAi[r][kk] += GV[r][0] * DV[kk][0] + GV[r][1] * DV[kk][1] + GV[r][2] * DV[kk][2];
  }
  // dL/dA = -A^-T (dL/dA^-1) A^-T; A rows are x_{k+1} - x_0
  double T1[3][3];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) T1[r][c] = gAi[r][0] * Mi[c][0] + gAi[r][1] * Mi[c][1] + gAi[r][2] * Mi[c][2];
  double gx0[3] = {-grel[0], -grel[1], -grel[2]};
#pragma unroll
  for (int kk = 0; kk < 3; ++kk) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double gA = -(Mi[0][kk] * T1[0][c] + Mi[1][kk] * T1[1][c] + Mi[2][kk] * T1[2][c]);
      if (gA != 0.0) atomicAdd(&P.g_x[3 * (int64_t)v[kk + 1] + c], gA);
      gx0[c] -= gA;
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c)
    if (gx0[c] != 0.0) atomicAdd(&P.g_x[3 * (int64_t)v[0] + c], gx0[c]);
}

// dL/dm_v and dL/dS_v from dL/drho_v (hull vertices have a constant density).
__global__ void k_adjoint_vertices(int64_t V, const float4* __restrict__ posd, const float* __restrict__ w,
                                   const int* __restrict__ hull, const double* __restrict__ g_rho,
                                   const long long* __restrict__ vacc, const dtfe::VolScale* __restrict__ vscale,
                                   const int64_t* __restrict__ vprefix, int nsb, float factor,
                                   double* __restrict__ g_S, double* __restrict__ g_m) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= V) return;
  int b = 0;  // the vertex's sub-box: its unit
  for (int lo = 0, hi = nsb; hi - lo > 1;) {
    const int mid = (lo + hi) >> 1;
    if (vprefix[mid] <= i) lo = b = mid;
    else hi = mid;
  }
  const double S = (double)vacc[i] * vscale[b].unit;
  if (hull[i] || S == 0.0) {
    g_S[i] = 0.0;
    g_m[i] = 0.0;
    return;
  }
  // rho_v = (w * factor) / S
  const double gr = g_rho[i];
  g_m[i] = gr * (double)factor / S;
  g_S[i] = -gr * (double)w[i] * (double)factor / (S * S);
}

// Per tetrahedron: Vbar_t = sum over its vertices of dL/dS_v.
__global__ void k_adjoint_vbar(int64_t T, const int4* __restrict__ tet_v, const double* __restrict__ g_S,
                               double* __restrict__ vbar) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= T) return;
  const int4 q = tet_v[t];
  vbar[t] = g_S[q.x] + g_S[q.y] + g_S[q.z] + g_S[q.w];
}

// Per vertex: gather Vbar_t dV_t/dx_v over the incident tetrahedra, add the
// per-cell terms, and write FP32 gradients.  For a positively oriented
// (a, b, c, d): 6V = (b-a).((c-a)x(d-a)); dV/db = (c-a)x(d-a)/6 and
// cyclically, dV/da = -(dV/db + dV/dc + dV/dd).
__global__ void k_adjoint_gather(int64_t V, const int4* __restrict__ tet_v, const float4* __restrict__ posd,
                                 const double* __restrict__ vbar, const int64_t* __restrict__ off,
                                 const int* __restrict__ inc, const double* __restrict__ g_x,
                                 const double* __restrict__ g_v, const double* __restrict__ g_m,
                                 float* __restrict__ out_x, float* __restrict__ out_v, float* __restrict__ out_w) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= V) return;
  double gx[3] = {g_x[3 * i], g_x[3 * i + 1], g_x[3 * i + 2]};
  for (int64_t q = off[i], e = off[i + 1]; q < e; ++q) {
    const int t = inc[q];
    const double vb = vbar[t];
    if (vb == 0.0) continue;
    const int4 tv = tet_v[t];
    const int v[4] = {tv.x, tv.y, tv.z, tv.w};
    double X[4][3];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const float4 r = posd[v[a]];
      X[a][0] = r.x; X[a][1] = r.y; X[a][2] = r.z;
    }
    double d[4][3];
    // gradient of 6V wrt each vertex: for vertex j the cross product of the
    // other two edges from vertex 0 (j >= 1), and minus their sum for j = 0
    double e1[3], e2[3], e3[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) { e1[c] = X[1][c] - X[0][c]; e2[c] = X[2][c] - X[0][c]; e3[c] = X[3][c] - X[0][c]; }
    d[1][0] = e2[1] * e3[2] - e2[2] * e3[1]; d[1][1] = e2[2] * e3[0] - e2[0] * e3[2]; d[1][2] = e2[0] * e3[1] - e2[1] * e3[0];
    d[2][0] = e3[1] * e1[2] - e3[2] * e1[1]; d[2][1] = e3[2] * e1[0] - e3[0] * e1[2]; d[2][2] = e3[0] * e1[1] - e3[1] * e1[0];
    d[3][0] = e1[1] * e2[2] - e1[2] * e2[1]; d[3][1] = e1[2] * e2[0] - e1[0] * e2[2]; d[3][2] = e1[0] * e2[1] - e1[1] * e2[0];
#pragma unroll
    for (int c = 0; c < 3; ++c) d[0][c] = -(d[1][c] + d[2][c] + d[3][c]);
#pragma unroll
    for (int a = 0; a < 4; ++a)
      if (v[a] == (int)i)
#pragma unroll
        for (int c = 0; c < 3; ++c) gx[c] += vb * d[a][c] / 6.0;
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) out_x[3 * i + c] = (float)gx[c];
  if (out_v)
#pragma unroll
    for (int c = 0; c < 3; ++c) out_v[3 * i + c] = (float)g_v[3 * i + c];
  if (out_w) out_w[i] = (float)g_m[i];
}

}  // namespace

// Launch sequence used by dtfe_gpu_adjoint (dtfe_core.cu owns the buffers).
extern "C" int dtfe_internal_adjoint(void* stream, const void* cell_params, int64_t n_cells, int64_t V, int64_t T,
                                     const int4* tet_v, const float4* posd, const float* w, const int* hull,
                                     const long long* vacc, const dtfe::VolScale* vscale, const int64_t* vprefix,
                                     int nsb, const int64_t* off, const int* inc, float factor, double* g_rho,
                                     double* g_x, double* g_v, double* g_S, double* g_m, double* vbar, float* out_x,
                                     float* out_v, float* out_w) {
  cudaStream_t st = (cudaStream_t)stream;
  cudaMemsetAsync(g_rho, 0, sizeof(double) * V, st);
  cudaMemsetAsync(g_x, 0, sizeof(double) * 3 * V, st);
  cudaMemsetAsync(g_v, 0, sizeof(double) * 3 * V, st);
  AdjCellParams P = *(const AdjCellParams*)cell_params;
  P.g_rho = g_rho;
  P.g_x = g_x;
  P.g_v = g_v;
  if (n_cells > 0) k_adjoint_cells<<<(unsigned)((n_cells + 255) / 256), 256, 0, st>>>(P);
  if (V > 0)
    k_adjoint_vertices<<<(unsigned)((V + 255) / 256), 256, 0, st>>>(V, posd, w, hull, g_rho, vacc, vscale, vprefix,
                                                                    nsb, factor, g_S, g_m);
  if (T > 0) k_adjoint_vbar<<<(unsigned)((T + 255) / 256), 256, 0, st>>>(T, tet_v, g_S, vbar);
  if (V > 0)
    k_adjoint_gather<<<(unsigned)((V + 255) / 256), 256, 0, st>>>(V, tet_v, posd, vbar, off, inc, g_x, g_v, g_m,
                                                                  out_x, out_v, out_w);
  return cudaGetLastError() == cudaSuccess ? DTFE_OK : DTFE_ERR_CUDA;
}

extern "C" size_t dtfe_internal_adjoint_params_size() { return sizeof(AdjCellParams); }

extern "C" void dtfe_internal_adjoint_fill_params(void* out, const int4* tet_v, const float4* posd,
                                                  const float4* vel4, const int* tet_c, const dtfe_subbox* boxes,
                                                  const int64_t* tile_prefix, const float* xs, const float* ys,
                                                  const float* zs, int K, int64_t G1, int64_t G2, int64_t n_total,
                                                  const float* a, const float* b, const float* c, int full_value) {
  AdjCellParams* P = (AdjCellParams*)out;
  P->tet_v = tet_v;
  P->posd = posd;
  P->vel4 = vel4;
  P->tet_c = tet_c;
  P->boxes = boxes;
  P->tile_prefix = tile_prefix;
  P->xs = xs;
  P->ys = ys;
  P->zs = zs;
  P->K = K;
  P->G1 = G1;
  P->G2 = G2;
  P->n_total = n_total;
  P->a = a;
  P->b = b;
  P->c = c;
  P->u[0] = P->u[1] = full_value ? 1.f : 0.f;
  P->u[2] = 1.f;
  P->g_rho = P->g_x = P->g_v = nullptr;
}
