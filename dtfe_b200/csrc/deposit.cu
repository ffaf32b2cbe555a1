// NGP / CIC / TSC grid deposition on B200 (sm_100a) — the reference's
// comparison estimators NGP_interpolation_regular_grid
// (src/NGP_interpolation.cc:67-136), CIC_interpolation_regular_grid
// (src/CIC_interpolation.cc:67-273) and TSC_interpolation_regular_grid
// (src/TSC_interpolation.cc:67-254), per sub-box region.
//
// Each particle's stencil (cells and per-axis weights, clipped at the region
// edges exactly as the reference clips them) and each contribution
// result = w * wx * wy * wz are computed in the reference's float arithmetic.
// The contributions are accumulated in 64-bit fixed point: every sum is exact,
// so the grid is deterministic and independent of the order in which threads
// add.  The fixed-point scales are powers of two chosen from the total |mass|
// and |momentum| so that no cell can overflow.  A block of 512 particles
// (256 for TSC; Morton-ordered within its sub-box) whose stencils fit a tile
// of at most 2048 cells accumulates in shared memory first and flushes each
// touched cell with one global atomic per component; other blocks add to
// global memory directly.  The global sums of one cell (mass and the three momenta) share
// one 32-byte sector.

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/dtfe_gpu.h"

extern "C" int dtfe_internal_set_error(int code, const char* msg);

namespace {

constexpr int kDepBlock = 256;
// particles per thread: TSC's 3^3 stencils widen a block's tile, so its
// blocks take 256 particles, NGP's and CIC's 512
__host__ __device__ constexpr int dep_ppt(int kind) { return kind == 2 ? 1 : 2; }
constexpr int kTileCap = 2048;                      // cells of a block's shared tile

struct DepBox {
  int64_t off, n;         // particle range
  float lo[3], dx[3];     // region lower corner and cell size (float, as the reference)
  float inner[6], outer[6];
  int32_t origin[3], dims[3];
  int64_t tile_off;       // first flattened tile cell of this box
  float factor;           // density normalisation of this region
};

struct DepSaved {
  const float4* pw;
  const DepBox* boxes;
  const int64_t* prefix;
  int K;
  int64_t n;
  int kind;
  int64_t G1, G2, G;
  int valid;
};

struct DepParams {
  const float4* pw;       // x, y, z, weight
  const float4* vel;      // vx, vy, vz, 0 (may be null)
  const DepBox* boxes;
  const int64_t* prefix;  // K+1 particle offsets
  int K;
  int64_t n;
  int64_t G1, G2;
  const double* scales;   // device: fixed-point scales of mass and momentum, then their inverses
  unsigned long long* acc;    // per grid cell: mass, then (with velocity) px, py, pz
};

__device__ __forceinline__ int find_dep_box(const int64_t* __restrict__ prefix, int K, int64_t s) {
  int lo = 0, hi = K;
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (__ldg(&prefix[mid]) <= s) lo = mid;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ bool in_box(const float p[3], const float* b) {
  return p[0] >= b[0] && p[0] <= b[1] && p[1] >= b[2] && p[1] <= b[3] && p[2] >= b[4] && p[2] <= b[5];
}

__device__ __forceinline__ float tsc_a(float t) { return (float)(.5 * (0.5 - (double)t) * (0.5 - (double)t)); }
__device__ __forceinline__ float tsc_b(float t) { return (float)(.75 - (double)(t * t)); }
__device__ __forceinline__ float tsc_c(float t) { return (float)(.5 * (0.5 + (double)t) * (0.5 + (double)t)); }

// Stencil of one axis (cells local to the region, weights, count), as
// axis_weights of the reference's CIC/TSC loops.
template <int KIND>
__device__ __forceinline__ void axis_stencil(bool inner, float temp, int n, int cell[3], float w[3], int& count) {
  count = 0;
  if (inner) {
    cell[0] = (int)floorf(temp) - 1;
    cell[1] = cell[0] + 1;
    cell[2] = cell[1] + 1;
    temp = (float)((double)temp - ((double)cell[1] + 0.5));
    count = 3;
    if (KIND == 1) {
      if (temp < 0.f) { w[0] = -temp; w[1] = 1 + temp; w[2] = 0.f; }
      else { w[0] = 0.f; w[1] = 1 - temp; w[2] = temp; }
    } else {
      w[0] = tsc_a(temp); w[1] = tsc_b(temp); w[2] = tsc_c(temp);
    }
    return;
  }
  int ti = (int)floorf(temp);
  temp = (float)((double)temp - ((double)ti + 0.5));
  if (ti == -1) {
    cell[0] = 0; count = 1;
    w[0] = KIND == 1 ? temp : tsc_c(temp);
  } else if (ti == 0) {
    cell[0] = 0; cell[1] = 1; count = 2;
    if (KIND == 1) { w[0] = 1 - temp; w[1] = temp; }
    else { w[0] = tsc_b(temp); w[1] = tsc_c(temp); }
  } else if (ti == n - 1) {
    cell[0] = n - 2; cell[1] = n - 1; count = 2;
    if (KIND == 1) { w[0] = -temp; w[1] = 1 + temp; }
    else { w[0] = tsc_a(temp); w[1] = tsc_b(temp); }
  } else if (ti == n) {
    cell[0] = n - 1; count = 1;
    w[0] = KIND == 1 ? -temp : tsc_a(temp);
  } else if (!(ti < -1 || ti > n)) {
    cell[0] = ti - 1; cell[1] = ti; cell[2] = ti + 1; count = 3;
    if (KIND == 1) {
      if (temp < 0.f) { w[0] = -temp; w[1] = 1 + temp; w[2] = 0.f; }
      else { w[0] = 0.f; w[1] = 1 - temp; w[2] = temp; }
    } else {
      w[0] = tsc_a(temp); w[1] = tsc_b(temp); w[2] = tsc_c(temp);
    }
  }
}

__device__ __forceinline__ unsigned long long to_fixed(float v, double scale) {
  return (unsigned long long)llrint((double)v * scale);
}

// One particle's stencil: per axis up to three region-local cells and their
// weights.  CIC's interior stencil spans three cells of which one always has
// weight 0 (the reference loops over all three); that cell is dropped, which
// changes no sum and keeps the block's tile tight.
struct Stencil {
  int cell[3][3];
  float w[3][3];
  int count[3];
};

template <class T>
__device__ __forceinline__ T pick3(const T (&a)[3], int i) {
  return i == 0 ? a[0] : (i == 1 ? a[1] : a[2]);
}

template <int KIND>
__device__ __forceinline__ bool particle_stencil(const DepBox& B, const float p[3], Stencil& S) {
  S.count[0] = S.count[1] = S.count[2] = 0;
  if (KIND == 0) {
    bool ok = true;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      S.cell[j][0] = (int)floorf((p[j] - B.lo[j]) / B.dx[j]);
      S.w[j][0] = 1.f;
      ok = ok && S.cell[j][0] >= 0 && S.cell[j][0] < B.dims[j];
    }
    if (ok) S.count[0] = S.count[1] = S.count[2] = 1;
  } else {
    const bool inner = in_box(p, B.inner);
    if (inner || in_box(p, B.outer)) {
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        float temp = (p[j] - B.lo[j]) / B.dx[j];
        axis_stencil<KIND>(inner, temp, B.dims[j], S.cell[j], S.w[j], S.count[j]);
        if (KIND == 1 && S.count[j] == 3) {
          if (S.w[j][2] == 0.f) S.count[j] = 2;
          else if (S.w[j][0] == 0.f) {
            S.cell[j][0] = S.cell[j][1]; S.w[j][0] = S.w[j][1];
            S.cell[j][1] = S.cell[j][2]; S.w[j][1] = S.w[j][2];
            S.count[j] = 2;
          }
        }
      }
    }
  }
  return S.count[0] > 0 && S.count[1] > 0 && S.count[2] > 0;
}

// KIND: 0 NGP, 1 CIC, 2 TSC; VEL: momentum accumulated beside the mass.
// A block takes 256 dep_ppt(KIND) consecutive particles (Morton-ordered
// within their sub-box).  When they all belong to one sub-box and their
// stencils fit a tile of at most kTileCap cells, the block adds into that
// tile in shared memory and flushes each touched cell with one global atomic
// per component;
// otherwise every contribution goes to global memory directly.  Contributions
// that round to 0 in fixed point are not added at all.
template <int KIND, bool VEL>
__global__ void __launch_bounds__(kDepBlock, 3) k_deposit(DepParams P) {
  extern __shared__ unsigned long long s_acc[];  // [component][kTileCap]
  __shared__ int s_box, s_ok, s_lo[3], s_hi[3];
  constexpr int C = VEL ? 4 : 1;
  // stencil points per axis (CIC: two, once its zero-weight cell is dropped)
  constexpr int M = KIND == 0 ? 1 : (KIND == 1 ? 2 : 3);
  constexpr int M3 = M * M * M;
  const int rot = (threadIdx.x & 31) % M3;
  constexpr int kDepPPT = dep_ppt(KIND), kDepChunk = kDepBlock * kDepPPT;
  const int64_t base = (int64_t)blockIdx.x * kDepChunk;
  const int64_t end = min(base + (int64_t)kDepChunk, P.n);
  const double scale_m = __ldg(&P.scales[0]), scale_p = __ldg(&P.scales[1]);
  if (threadIdx.x == 0) {
    const int b = find_dep_box(P.prefix, P.K, base);
    s_box = b;
    s_ok = __ldg(&P.prefix[b + 1]) >= end;
    for (int c = 0; c < 3; ++c) { s_lo[c] = 0x7FFFFFFF; s_hi[c] = -0x7FFFFFFF; }
  }
  float4 q[kDepPPT], u[kDepPPT];
#pragma unroll
  for (int r = 0; r < kDepPPT; ++r) {
    const int64_t i = base + r * kDepBlock + threadIdx.x;
    q[r] = i < end ? __ldg(&P.pw[i]) : make_float4(0.f, 0.f, 0.f, 0.f);
    u[r] = (VEL && P.vel && i < end) ? __ldg(&P.vel[i]) : make_float4(0.f, 0.f, 0.f, 0.f);
  }
  __syncthreads();
  const bool one_box = s_ok;

  // the block's cell bounds (single-box blocks only)
  if (one_box) {
    const DepBox& B = P.boxes[s_box];
    int lo[3] = {0x7FFFFFFF, 0x7FFFFFFF, 0x7FFFFFFF}, hi[3] = {-0x7FFFFFFF, -0x7FFFFFFF, -0x7FFFFFFF};
#pragma unroll
    for (int r = 0; r < kDepPPT; ++r) {
      const int64_t i = base + r * kDepBlock + threadIdx.x;
      Stencil S;
      const float p[3] = {q[r].x, q[r].y, q[r].z};
      if (i < end && particle_stencil<KIND>(B, p, S)) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          lo[c] = min(lo[c], S.cell[c][0]);
          hi[c] = max(hi[c], S.count[c] == 1 ? S.cell[c][0] : S.count[c] == 2 ? S.cell[c][1] : S.cell[c][2]);
        }
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      lo[c] = __reduce_min_sync(0xffffffffu, lo[c]);
      hi[c] = __reduce_max_sync(0xffffffffu, hi[c]);
    }
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        atomicMin(&s_lo[c], lo[c]);
        atomicMax(&s_hi[c], hi[c]);
      }
    }
  }
  __syncthreads();
  const int tlo[3] = {s_lo[0], s_lo[1], s_lo[2]};
  bool staged = one_box && s_hi[0] >= tlo[0] && s_hi[1] >= tlo[1] && s_hi[2] >= tlo[2];
  int sy = 1, sz = 1;
  int64_t cells = 0;
  if (staged) {
    sy = s_hi[1] - tlo[1] + 1;
    sz = s_hi[2] - tlo[2] + 1;
    cells = (int64_t)(s_hi[0] - tlo[0] + 1) * sy * sz;
    staged = cells <= kTileCap;
  }
  if (staged) {
    for (int k = threadIdx.x; k < C * kTileCap; k += kDepBlock) s_acc[k] = 0ull;
    __syncthreads();
  }

#pragma unroll
  for (int r = 0; r < kDepPPT; ++r) {
    const int64_t i = base + r * kDepBlock + threadIdx.x;
    if (i >= end) continue;
    const int b = one_box ? s_box : find_dep_box(P.prefix, P.K, i);
    const DepBox& B = P.boxes[b];
    const float p[3] = {q[r].x, q[r].y, q[r].z};
    const float wt = q[r].w, v[3] = {u[r].x, u[r].y, u[r].z};
    Stencil S;
    if (!particle_stencil<KIND>(B, p, S)) continue;
    // The stencil's M^3 corners in an order rotated by the lane: neighbouring
    // particles of a warp share cells, and at one step of the loop the lanes
    // then mostly add to different cells instead of queueing on the same
    // shared word.  Fixed trip counts with guards and selects (not indexed
    // arrays) keep the stencil in registers.
#pragma unroll
    for (int s = 0; s < M3; ++s) {
      int qc = rot + s;
      if (qc >= M3) qc -= M3;
      const int a = qc / (M * M), bb = (qc / M) % M, c = qc % M;
      if (a >= S.count[0] || bb >= S.count[1] || c >= S.count[2]) continue;
      const float result = wt * pick3(S.w[0], a) * pick3(S.w[1], bb) * pick3(S.w[2], c);
      unsigned long long f[C];
      f[0] = to_fixed(result, scale_m);
      unsigned long long nz = f[0];
      if (VEL) {
#pragma unroll
        for (int k = 1; k < C; ++k) {
          f[k] = to_fixed(v[k - 1] * result, scale_p);
          nz |= f[k];
        }
      }
      if (nz == 0ull) continue;
      const int c0 = pick3(S.cell[0], a), c1 = pick3(S.cell[1], bb), c2 = pick3(S.cell[2], c);
      if (staged) {
        const int k = ((c0 - tlo[0]) * sy + (c1 - tlo[1])) * sz + (c2 - tlo[2]);
#pragma unroll
        for (int m = 0; m < C; ++m) atomicAdd(&s_acc[m * kTileCap + k], f[m]);
      } else {
        const int64_t idx = ((int64_t)(B.origin[0] + c0) * P.G1 + (B.origin[1] + c1)) * P.G2 + (B.origin[2] + c2);
#pragma unroll
        for (int m = 0; m < C; ++m) atomicAdd(&P.acc[C * idx + m], f[m]);
      }
    }
  }
  if (staged) {
    __syncthreads();
    const DepBox& B = P.boxes[s_box];
    const int syz = sy * sz;
    for (int k = threadIdx.x; k < (int)cells; k += kDepBlock) {
      const int ci = k / syz, cj = (k - ci * syz) / sz, ck = k - ci * syz - cj * sz;
      unsigned long long f[C], nz = 0ull;
#pragma unroll
      for (int m = 0; m < C; ++m) {
        f[m] = s_acc[m * kTileCap + k];
        nz |= f[m];
      }
      if (nz == 0ull) continue;
      const int64_t idx = ((int64_t)(B.origin[0] + tlo[0] + ci) * P.G1 + (B.origin[1] + tlo[1] + cj)) * P.G2 +
                          (B.origin[2] + tlo[2] + ck);
#pragma unroll
      for (int m = 0; m < C; ++m) atomicAdd(&P.acc[C * idx + m], f[m]);
    }
  }
}

// Fixed-point sums -> the reference's normalisation, per region: velocity =
// momentum / mass (float division), density = mass * (region cells /
// Box::volume() / rho_bar), Box::volume() being the hard-coded 35000^3.
__global__ void k_deposit_finalize(int64_t n_tile_cells, const DepBox* __restrict__ boxes,
                                   const int64_t* __restrict__ tile_prefix, int K, int64_t G1, int64_t G2,
                                   const unsigned long long* __restrict__ acc, int stride,
                                   const double* __restrict__ scales, float* __restrict__ density,
                                   float* __restrict__ velocity) {
  int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= n_tile_cells) return;
  const int b = find_dep_box(tile_prefix, K, s);
  const DepBox& B = boxes[b];
  const int64_t local = s - B.tile_off;
  const int k = (int)(local % B.dims[2]);
  const int j = (int)((local / B.dims[2]) % B.dims[1]);
  const int i = (int)(local / ((int64_t)B.dims[2] * B.dims[1]));
  const int64_t idx = ((int64_t)(B.origin[0] + i) * G1 + (B.origin[1] + j)) * G2 + (B.origin[2] + k);
  const double inv_m = __ldg(&scales[2]), inv_p = __ldg(&scales[3]);
  const float m = (float)((double)(long long)acc[stride * idx] * inv_m);
  if (velocity) {
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const float p = (float)((double)(long long)acc[stride * idx + 1 + q] * inv_p);
      velocity[3 * idx + q] = m != 0.f ? p / m : 0.f;
    }
  }
  if (density) density[idx] = m * B.factor;
}

// Adjoint of the deposited density for one particle: with loss weights
// a_c = dL/d(density_c) and density_c = factor_b * sum_p m_p W_pc,
//   dL/dm_p = factor_b sum_c a_c W_pc,  dL/dx_p = factor_b m_p sum_c a_c dW_pc/dx_p.
// W_pc is the product of the per-axis stencil weights of the forward pass;
// their derivatives follow the same clipped formulas (NGP: zero).
template <int KIND>
__device__ __forceinline__ void axis_stencil_grad(bool inner, float temp_in, int n, float dx, int cell[3],
                                                  float w[3], float dw[3], int& count) {
  axis_stencil<KIND>(inner, temp_in, n, cell, w, count);
  float t;
  if (inner) t = (float)((double)temp_in - ((double)((int)floorf(temp_in)) + 0.5));
  else {
    int ti = (int)floorf(temp_in);
    t = (float)((double)temp_in - ((double)ti + 0.5));
  }
  const float s = 1.f / dx;
  for (int q = 0; q < 3; ++q) dw[q] = 0.f;
  if (KIND == 1) {
    // every CIC branch is linear in t: recover the slope from the formulas
    if (inner) {
      if (t < 0.f) { dw[0] = -s; dw[1] = s; dw[2] = 0.f; }
      else { dw[0] = 0.f; dw[1] = -s; dw[2] = s; }
    } else {
      int ti = (int)floorf(temp_in);
      if (ti == -1) dw[0] = s;
      else if (ti == 0) { dw[0] = -s; dw[1] = s; }
      else if (ti == n - 1) { dw[0] = -s; dw[1] = s; }
      else if (ti == n) dw[0] = -s;
      else if (!(ti < -1 || ti > n)) {
        if (t < 0.f) { dw[0] = -s; dw[1] = s; dw[2] = 0.f; }
        else { dw[0] = 0.f; dw[1] = -s; dw[2] = s; }
      }
    }
  } else if (KIND == 2) {
    const float da = -(0.5f - t) * s, db = -2.f * t * s, dc = (0.5f + t) * s;
    if (inner) { dw[0] = da; dw[1] = db; dw[2] = dc; }
    else {
      int ti = (int)floorf(temp_in);
      if (ti == -1) dw[0] = dc;
      else if (ti == 0) { dw[0] = db; dw[1] = dc; }
      else if (ti == n - 1) { dw[0] = da; dw[1] = db; }
      else if (ti == n) dw[0] = da;
      else if (!(ti < -1 || ti > n)) { dw[0] = da; dw[1] = db; dw[2] = dc; }
    }
  }
}

template <int KIND>
__global__ void k_deposit_adjoint(const float4* __restrict__ pw, const DepBox* __restrict__ boxes,
                                  const int64_t* __restrict__ prefix, int K, int64_t n, int64_t G1, int64_t G2,
                                  const float* __restrict__ a, float* __restrict__ gx, float* __restrict__ gw) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int b = find_dep_box(prefix, K, i);
  const DepBox& B = boxes[b];
  const float4 q = pw[i];
  const float p[3] = {q.x, q.y, q.z};
  int cell[3][3], count[3] = {0, 0, 0};
  float w[3][3], dw[3][3];
  if (KIND == 0) {
    bool ok = true;
    for (int j = 0; j < 3; ++j) {
      cell[j][0] = (int)floorf((p[j] - B.lo[j]) / B.dx[j]);
      w[j][0] = 1.f;
      dw[j][0] = 0.f;
      ok = ok && cell[j][0] >= 0 && cell[j][0] < B.dims[j];
    }
    if (ok) count[0] = count[1] = count[2] = 1;
  } else {
    const bool inner = in_box(p, B.inner);
    if (inner || in_box(p, B.outer))
      for (int j = 0; j < 3; ++j)
        axis_stencil_grad<KIND>(inner, (p[j] - B.lo[j]) / B.dx[j], B.dims[j], B.dx[j], cell[j], w[j], dw[j],
                                count[j]);
  }
  double sm = 0.0, sx[3] = {0.0, 0.0, 0.0};
  for (int x0 = 0; x0 < count[0]; ++x0)
    for (int x1 = 0; x1 < count[1]; ++x1)
      for (int x2 = 0; x2 < count[2]; ++x2) {
        const int64_t idx = ((int64_t)(B.origin[0] + cell[0][x0]) * G1 + (B.origin[1] + cell[1][x1])) * G2 +
                            (B.origin[2] + cell[2][x2]);
        const double ac = (double)a[idx];
        if (ac == 0.0) continue;
        sm += ac * (double)w[0][x0] * w[1][x1] * w[2][x2];
        sx[0] += ac * (double)dw[0][x0] * w[1][x1] * w[2][x2];
        sx[1] += ac * (double)w[0][x0] * dw[1][x1] * w[2][x2];
        sx[2] += ac * (double)w[0][x0] * w[1][x1] * dw[2][x2];
      }
  if (gw) gw[i] = (float)(B.factor * sm);
  if (gx)
    for (int j = 0; j < 3; ++j) gx[3 * i + j] = (float)(B.factor * (double)q.w * sx[j]);
}

// Fixed-point scales from order-independent bounds: n x max|w| for the mass
// and n x max(|w| (|vx| + |vy| + |vz|)) for the momentum, times 8 (the
// clipped edge stencils' weights sum to at most 8 in magnitude), each scaled
// to stay below 2^61.  Maxima of non-negative floats by integer atomicMax on
// their bits.
__global__ void k_deposit_bounds(int64_t n, const float4* __restrict__ pw, const float4* __restrict__ vel,
                                 unsigned* __restrict__ maxbits) {
  float mw = 0.f, mp = 0.f;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float4 q = __ldg(&pw[i]);
    const float a = fabsf(q.w);
    mw = fmaxf(mw, a);
    if (vel) {
      const float4 u = __ldg(&vel[i]);
      mp = fmaxf(mp, a * (fabsf(u.x) + fabsf(u.y) + fabsf(u.z)));
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mw = fmaxf(mw, __shfl_xor_sync(0xffffffffu, mw, o));
    mp = fmaxf(mp, __shfl_xor_sync(0xffffffffu, mp, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&maxbits[0], __float_as_uint(mw));
    atomicMax(&maxbits[1], __float_as_uint(mp));
  }
}

__global__ void k_deposit_scales(int64_t n, const unsigned* __restrict__ maxbits, double* __restrict__ scales) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int q = 0; q < 2; ++q) {
    const double bound = 8.0 * (double)n * (double)__uint_as_float(maxbits[q]);
    const double s = ldexp(1.0, 61 - (int)ceil(log2(fmax(bound, 1e-30))));
    scales[q] = s;
    scales[2 + q] = 1.0 / s;
  }
}

__global__ void k_pack4(int64_t n, const float* __restrict__ a3, const float* __restrict__ b1, float4* __restrict__ out) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = make_float4(a3[3 * i], a3[3 * i + 1], a3[3 * i + 2], b1 ? b1[i] : 1.f);
}

extern "C" size_t dtfe_internal_deposit_saved_size() { return sizeof(DepSaved); }

template <int KIND>
void launch_deposit(bool with_vel, unsigned nb, cudaStream_t st, const DepParams& P) {
  if (with_vel) {
    const int smem = 4 * kTileCap * (int)sizeof(unsigned long long);
    cudaFuncSetAttribute(k_deposit<KIND, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    k_deposit<KIND, true><<<nb, kDepBlock, smem, st>>>(P);
  } else {
    k_deposit<KIND, false><<<nb, kDepBlock, kTileCap * sizeof(unsigned long long), st>>>(P);
  }
}

}  // namespace

// inputs_dev: xyz, w and vel are device pointers (else host pointers, copied
// on the stream).
extern "C" int dtfe_gpu_deposit_impl(void* stream, int32_t kind, const float* xyz, const float* w, const float* vel,
                                     int64_t n, int32_t n_boxes, const dtfe_deposit_box* boxes,
                                     const int32_t grid[3], double average_density, float* density_dev,
                                     float* velocity_dev, void** scratch, size_t* scratch_bytes, void* saved,
                                     int inputs_dev) {
  if (kind < 0 || kind > 2) return dtfe_internal_set_error(DTFE_ERR_ARG, "deposit kind must be 0 (NGP), 1 (CIC), 2 (TSC)");
  if (n < 0 || n_boxes <= 0 || !boxes || !grid) return dtfe_internal_set_error(DTFE_ERR_ARG, "bad deposit arguments");
  if (!(average_density > 0.0)) return dtfe_internal_set_error(DTFE_ERR_ARG, "averageDensity must be positive");
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t G = (int64_t)grid[0] * grid[1] * grid[2];
  // host-side box records: the reference's float region arithmetic
  std::vector<DepBox> hb(n_boxes);
  std::vector<int64_t> prefix(n_boxes + 1);
  for (int b = 0; b < n_boxes; ++b) {
    const dtfe_deposit_box& in = boxes[b];
    DepBox& B = hb[b];
    B.off = in.particle_offset;
    B.n = in.n_particles;
    if (B.off < 0 || B.off + B.n > n || (b > 0 && B.off != hb[b - 1].off + hb[b - 1].n))
      return dtfe_internal_set_error(DTFE_ERR_ARG, "deposit boxes must cover consecutive particle ranges");
    for (int c = 0; c < 3; ++c) {
      if (in.tile_dims[c] < (kind ? 3 : 1) || in.tile_origin[c] < 0 || in.tile_origin[c] + in.tile_dims[c] > grid[c])
        return dtfe_internal_set_error(DTFE_ERR_ARG, "deposit tile outside the grid (CIC/TSC need >= 3 cells per axis)");
      B.origin[c] = in.tile_origin[c];
      B.dims[c] = in.tile_dims[c];
      B.lo[c] = in.region[2 * c];
      B.dx[c] = (in.region[2 * c + 1] - in.region[2 * c]) / (float)in.tile_dims[c];
      const float pad = B.dx[c];
      const float ipad = (float)(-1.1 * (double)pad);
      B.outer[2 * c] = in.region[2 * c] - pad;
      B.outer[2 * c + 1] = in.region[2 * c + 1] + pad;
      B.inner[2 * c] = in.region[2 * c] - ipad;
      B.inner[2 * c + 1] = in.region[2 * c + 1] + ipad;
    }
    prefix[b] = B.off;
  }
  prefix[n_boxes] = hb[n_boxes - 1].off + hb[n_boxes - 1].n;
  std::vector<int64_t> tprefix(n_boxes + 1, 0);
  float vol = 1.f;
  for (int c = 0; c < 3; ++c) vol *= 35000;  // the reference's Box::volume()
  for (int b = 0; b < n_boxes; ++b) {
    DepBox& B = hb[b];
    const int64_t cells = (int64_t)B.dims[0] * B.dims[1] * B.dims[2];
    B.tile_off = tprefix[b];
    tprefix[b + 1] = tprefix[b] + cells;
    B.factor = (float)cells / vol / (float)average_density;
  }
  // scratch: particles (2 float4), boxes, prefix, accumulators (1 or 4 per cell)
  const int comps = velocity_dev ? 4 : 1;
  const size_t bytes_part = sizeof(float4) * 2 * (size_t)n;
  const size_t bytes_box = sizeof(DepBox) * n_boxes + 2 * sizeof(int64_t) * (n_boxes + 1);
  const size_t bytes_acc = sizeof(unsigned long long) * 4 * (size_t)G;
  const size_t bytes_tmp = sizeof(float) * 4 * (size_t)n;  // host inputs: 3-float records as they arrive
  const size_t need = bytes_part + bytes_box + bytes_acc + bytes_tmp + 4096;
  if (*scratch_bytes < need) {
    if (*scratch) cudaFree(*scratch);
    *scratch = nullptr;
    *scratch_bytes = 0;
    if (cudaMalloc(scratch, need) != cudaSuccess) return dtfe_internal_set_error(DTFE_ERR_ALLOC, "cudaMalloc (deposit)");
    *scratch_bytes = need;
  }
  char* base = (char*)*scratch;
  auto align = [](size_t x) { return (x + 255) & ~(size_t)255; };
  float4* d_pw = (float4*)base;
  float4* d_vel = d_pw + n;
  size_t o = align(bytes_part);
  unsigned long long* acc = (unsigned long long*)(base + o);
  o = align(o + bytes_acc);
  DepBox* d_boxes = (DepBox*)(base + o);
  int64_t* d_prefix = (int64_t*)(base + o + sizeof(DepBox) * n_boxes);
  int64_t* d_tprefix = d_prefix + (n_boxes + 1);
  float* tmp = (float*)(base + align(o + bytes_box));
  double* d_scales = (double*)(base + align(align(o + bytes_box) + bytes_tmp));
  unsigned* d_maxbits = (unsigned*)(d_scales + 4);
  cudaError_t e;
  if (n > 0 && inputs_dev) {
    k_pack4<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, xyz, w, d_pw);
    if (vel) k_pack4<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, vel, nullptr, d_vel);
  } else if (n > 0) {
    float* t3 = tmp;
    float* t1 = tmp + 3 * n;
    cudaMemcpyAsync(t3, xyz, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, st);
    if (w) cudaMemcpyAsync(t1, w, sizeof(float) * n, cudaMemcpyHostToDevice, st);
    k_pack4<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, t3, w ? t1 : nullptr, d_pw);
    if (vel) {
      cudaMemcpyAsync(t3, vel, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, st);
      k_pack4<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, t3, nullptr, d_vel);
    }
  }
  cudaMemcpyAsync(d_boxes, hb.data(), sizeof(DepBox) * n_boxes, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_prefix, prefix.data(), sizeof(int64_t) * (n_boxes + 1), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_tprefix, tprefix.data(), sizeof(int64_t) * (n_boxes + 1), cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * comps * (size_t)G, st);
  DepParams P;
  P.pw = d_pw;
  P.vel = vel ? d_vel : nullptr;
  P.boxes = d_boxes;
  P.prefix = d_prefix;
  P.K = n_boxes;
  P.n = n;
  P.G1 = grid[1];
  P.G2 = grid[2];
  cudaMemsetAsync(d_maxbits, 0, 2 * sizeof(unsigned), st);
  if (n > 0)
    k_deposit_bounds<<<(unsigned)std::min<int64_t>((n + 255) / 256, 4 * 148), 256, 0, st>>>(n, d_pw,
                                                                                          vel ? d_vel : nullptr,
                                                                                          d_maxbits);
  k_deposit_scales<<<1, 32, 0, st>>>(n, d_maxbits, d_scales);
  P.scales = d_scales;
  P.acc = acc;
  if (n > 0) {
    const int64_t chunk = (int64_t)kDepBlock * dep_ppt(kind);
    const unsigned nb = (unsigned)((n + chunk - 1) / chunk);
    if (kind == 0) launch_deposit<0>(velocity_dev != nullptr, nb, st, P);
    else if (kind == 1) launch_deposit<1>(velocity_dev != nullptr, nb, st, P);
    else launch_deposit<2>(velocity_dev != nullptr, nb, st, P);
  }
  const int64_t nt = tprefix[n_boxes];
  if (nt > 0)
    k_deposit_finalize<<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(nt, d_boxes, d_tprefix, n_boxes, grid[1], grid[2],
                                                                     acc, comps, d_scales,
                                                                     density_dev, velocity_dev);
  if ((e = cudaGetLastError()) != cudaSuccess) return dtfe_internal_set_error(DTFE_ERR_CUDA, cudaGetErrorString(e));
  // state for dtfe_gpu_deposit_adjoint (the scratch keeps particles and boxes)
  DepSaved& sv = *(DepSaved*)saved;
  sv.pw = d_pw;
  sv.boxes = d_boxes;
  sv.prefix = d_prefix;
  sv.K = n_boxes;
  sv.n = n;
  sv.kind = kind;
  sv.G1 = grid[1];
  sv.G2 = grid[2];
  sv.G = G;
  sv.valid = 1;
  return DTFE_OK;
}

extern "C" int dtfe_gpu_deposit_adjoint_impl(void* stream, const void* saved, const float* a_dev, float* gx_dev,
                                             float* gw_dev) {
  const DepSaved& sv = *(const DepSaved*)saved;
  if (!sv.valid) return dtfe_internal_set_error(DTFE_ERR_STATE, "no forward deposit on this handle");
  cudaStream_t st = (cudaStream_t)stream;
  if (sv.n == 0) return DTFE_OK;
  const unsigned nb = (unsigned)((sv.n + 255) / 256);
  if (sv.kind == 0)
    k_deposit_adjoint<0><<<nb, 256, 0, st>>>(sv.pw, sv.boxes, sv.prefix, sv.K, sv.n, sv.G1, sv.G2, a_dev, gx_dev, gw_dev);
  else if (sv.kind == 1)
    k_deposit_adjoint<1><<<nb, 256, 0, st>>>(sv.pw, sv.boxes, sv.prefix, sv.K, sv.n, sv.G1, sv.G2, a_dev, gx_dev, gw_dev);
  else
    k_deposit_adjoint<2><<<nb, 256, 0, st>>>(sv.pw, sv.boxes, sv.prefix, sv.K, sv.n, sv.G1, sv.G2, a_dev, gx_dev, gw_dev);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? DTFE_OK : dtfe_internal_set_error(DTFE_ERR_CUDA, cudaGetErrorString(e));
}
