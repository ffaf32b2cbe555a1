// SPH grid estimator on the GPU: the reference's SPH_interpolation
// (src/SPH_interpolation.cc:252-474) for every sub-box of the uploaded
// multi-tessellation (its padded particle set and its grid tile).
//
//   1. per sub-box a uniform cell grid over its particles' bounding box
//      (about two particles per cell), filled by a counting sort;
//   2. per particle: its N nearest particles of the sub-box (itself
//      included, as kdtree2 with correltime 0), h = sqrt(d_N)/2 and, when
//      scalar fields are asked for, the two-sided particle density d (:318-326);
//   3. per grid point: its N nearest particles, the gather half of the grid
//      sums with h = sqrt(d_N)/2 (:349-382);
//   4. per particle: every grid point of its tile within 2 h (squared float
//      distance <= 4 h^2, as kdtree2::r_nearest) receives the scatter half
//      (:399-432);
//   5. velocity and intensive scalars over the grid density, density times
//      1/averageDensity (:438-462).
// Every term is the reference's float expression (distances as float sums of
// float squares in axis order, kernel from the 1001-bin midpoint table,
// products in the reference's order; the translation unit is built with
// -fmad=false); sums run in FP64 and are rounded to float once.  Neighbour
// lists are exact: shells of cells are searched until no unvisited particle
// can be closer than the N-th, ties broken by particle index.  The search
// keeps each thread's sorted list in shared memory (columns per thread), so
// no list lives in local memory.

#include <cuda_runtime.h>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/dtfe_gpu.h"
#include "tile_index.cuh"

extern "C" int dtfe_internal_set_error(int code, const char* msg);

namespace {

constexpr int kTable = 1000;
constexpr int kSphBlock = 128;
constexpr int kMaxNeighbours = 128;

__constant__ float c_W[kTable + 1];

struct SphGrid {
  float lo[3];
  float inv[3];  // cells per unit length
  float smin;    // smallest cell edge
  int n[3];
  int64_t cell_off;
};

__device__ __forceinline__ int find_range(const int64_t* __restrict__ prefix, int K, int64_t s) {
  int lo = 0, hi = K;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(&prefix[mid]) <= s) lo = mid;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ int ordered(float f) {
  const int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
__device__ __forceinline__ float unordered(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7FFFFFFF); }

__device__ __forceinline__ float sqf(float a) { return a * a; }
// kdtree2's squared distance: float sum of float squares in axis order
__device__ __forceinline__ float dist2(float ax, float ay, float az, const float q[3]) {
  float d = 0.f;
  d += sqf(ax - q[0]);
  d += sqf(ay - q[1]);
  d += sqf(az - q[2]);
  return d;
}

// Per sub-box bounding box of its particles.  Vertices of a sub-box are
// contiguous, so a warp's lanes usually share one sub-box: they reduce in
// registers first and the first lane of each run of equal sub-boxes issues
// the six atomics.
__global__ void k_sph_bounds(int64_t v0, int64_t v1, const int64_t* __restrict__ vprefix, int K,
                             const float4* __restrict__ posd, int* __restrict__ bounds) {
  const int64_t i = v0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const bool valid = i < v1;
  int b = -1;
  int lo[3] = {0x7FFFFFFF, 0x7FFFFFFF, 0x7FFFFFFF}, hi[3] = {(int)0x80000000, (int)0x80000000, (int)0x80000000};
  if (valid) {
    b = find_range(vprefix, K, i);
    const float4 p = __ldg(&posd[i]);
    const float x[3] = {p.x, p.y, p.z};
#pragma unroll
    for (int c = 0; c < 3; ++c) lo[c] = hi[c] = ordered(x[c]);
  }
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int ob = __shfl_down_sync(0xffffffffu, b, o);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int ol = __shfl_down_sync(0xffffffffu, lo[c], o);
      const int oh = __shfl_down_sync(0xffffffffu, hi[c], o);
      if (lane + o < 32 && ob == b) {
        lo[c] = min(lo[c], ol);
        hi[c] = max(hi[c], oh);
      }
    }
  }
  const int prev = __shfl_up_sync(0xffffffffu, b, 1);
  if (b >= 0 && (lane == 0 || prev != b)) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      atomicMin(&bounds[6 * b + 2 * c], lo[c]);
      atomicMax(&bounds[6 * b + 2 * c + 1], hi[c]);
    }
  }
}

// One thread: cell grid of every sub-box (about two particles per cell).
__global__ void k_sph_params(int K, const int64_t* __restrict__ vprefix, const int* __restrict__ bounds,
                             SphGrid* __restrict__ grids, int64_t* __restrict__ total) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  int64_t off = 0;
  for (int b = 0; b < K; ++b) {
    SphGrid g;
    const int64_t np = vprefix[b + 1] - vprefix[b];
    float ext[3];
    double vol = 1.0;
    for (int c = 0; c < 3; ++c) {
      const float lo = np > 0 ? unordered(bounds[6 * b + 2 * c]) : 0.f;
      const float hi = np > 0 ? unordered(bounds[6 * b + 2 * c + 1]) : 0.f;
      g.lo[c] = lo;
      ext[c] = hi - lo;
      vol *= fmax((double)ext[c], 1e-6);
    }
    const double s = cbrt(vol * 2.0 / (double)(np > 0 ? np : 1));
    for (int c = 0; c < 3; ++c) {
      const int n = (int)floor((double)ext[c] / s);
      g.n[c] = n < 1 ? 1 : (n > 1024 ? 1024 : n);
    }
    // never more than np/2 cells (at least one): the cell arrays are sized so
    const int64_t cap = np / 2 > 1 ? np / 2 : 1;
    while ((int64_t)g.n[0] * g.n[1] * g.n[2] > cap) {
      const int c = (g.n[0] >= g.n[1] && g.n[0] >= g.n[2]) ? 0 : (g.n[1] >= g.n[2] ? 1 : 2);
      g.n[c] = g.n[c] / 2 > 1 ? g.n[c] / 2 : 1;
    }
    float smin = 3.4e38f;
    for (int c = 0; c < 3; ++c) {
      const int n = g.n[c];
      const float edge = ext[c] > 0.f ? ext[c] / (float)n : 1.f;
      g.inv[c] = 1.f / edge;
      smin = fminf(smin, edge);
    }
    // the cell edge the search bound may rely on: 1/inv rounds either way
    g.smin = smin * (1.f - 1e-6f);
    g.cell_off = off;
    off += (int64_t)g.n[0] * g.n[1] * g.n[2];
    grids[b] = g;
  }
  *total = off;
}

__device__ __forceinline__ int cell_axis(const SphGrid& g, float x, int c) {
  int k = (int)floorf((x - g.lo[c]) * g.inv[c]);
  return k < 0 ? 0 : (k >= g.n[c] ? g.n[c] - 1 : k);
}

__global__ void k_sph_count(int64_t v0, int64_t v1, const int64_t* __restrict__ vprefix, int K,
                            const SphGrid* __restrict__ grids, const float4* __restrict__ posd,
                            int* __restrict__ count, int* __restrict__ rank) {
  const int64_t i = v0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= v1) return;
  const SphGrid g = grids[find_range(vprefix, K, i)];
  const float4 p = __ldg(&posd[i]);
  const int64_t cell = g.cell_off + ((int64_t)cell_axis(g, p.x, 0) * g.n[1] + cell_axis(g, p.y, 1)) * g.n[2] +
                       cell_axis(g, p.z, 2);
  rank[i - v0] = atomicAdd(&count[cell], 1);
}

__global__ void k_sph_place(int64_t v0, int64_t v1, const int64_t* __restrict__ vprefix, int K,
                            const SphGrid* __restrict__ grids, const float4* __restrict__ posd,
                            const int* __restrict__ start, const int* __restrict__ rank, float4* __restrict__ sorted) {
  const int64_t i = v0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= v1) return;
  const SphGrid g = grids[find_range(vprefix, K, i)];
  const float4 p = __ldg(&posd[i]);
  const int64_t cell = g.cell_off + ((int64_t)cell_axis(g, p.x, 0) * g.n[1] + cell_axis(g, p.y, 1)) * g.n[2] +
                       cell_axis(g, p.z, 2);
  // position and particle index in one record, in cell order
  sorted[start[cell] + rank[i - v0]] = make_float4(p.x, p.y, p.z, __int_as_float((int)i));
}

__device__ __forceinline__ bool before(float d, int i, float e, int j) { return d < e || (d == e && i < j); }

// Distance from coordinate x to cell c's slab along axis a (0 inside).
// Boundary cells are open towards the outside (particles beyond the box
// are clamped into them), so their outer side counts as no gap.
__device__ __forceinline__ float cell_gap(const SphGrid& g, float x, int c, int a) {
  const float e = 1.f / g.inv[a];
  const float lo = g.lo[a] + (float)c * e, hi = lo + e;
  const float slack = 1e-3f * e;  // cell assignment rounds in float
  if (x < lo && c > 0) return fmaxf(lo - x - slack, 0.f);
  if (x > hi && c < g.n[a] - 1) return fmaxf(x - hi - slack, 0.f);
  return 0.f;
}

// The k nearest particles of q in one sub-box's cell grid, ascending by
// (squared distance, index), in this thread's shared-memory columns
// ld[slot * kSphBlock], li[slot * kSphBlock].  Returns the list length.
__device__ int knn(const SphGrid& g, const int* __restrict__ start, const float4* __restrict__ sorted,
                   const float q[3], int k, float* ld, int* li) {
  const int c0[3] = {cell_axis(g, q[0], 0), cell_axis(g, q[1], 1), cell_axis(g, q[2], 2)};
  const int rmax = max(g.n[0], max(g.n[1], g.n[2]));
  int m = 0;
  for (int r = 0; r <= rmax; ++r) {
    for (int dx = -r; dx <= r; ++dx) {
      const int x = c0[0] + dx;
      if (x < 0 || x >= g.n[0]) continue;
      for (int dy = -r; dy <= r; ++dy) {
        const int y = c0[1] + dy;
        if (y < 0 || y >= g.n[1]) continue;
        const bool face = (dx == -r || dx == r || dy == -r || dy == r);
        const int step = face ? 1 : (r > 0 ? 2 * r : 1);
        for (int dz = -r; dz <= r; dz += step) {
          const int z = c0[2] + dz;
          if (z < 0 || z >= g.n[2]) continue;
          if (m == k) {
            // skip cells wholly farther than the current k-th neighbour
            const float gap[3] = {cell_gap(g, q[0], x, 0), cell_gap(g, q[1], y, 1), cell_gap(g, q[2], z, 2)};
            const float md = gap[0] * gap[0] + gap[1] * gap[1] + gap[2] * gap[2];
            if (md > ld[(k - 1) * kSphBlock]) continue;
          }
          const int64_t cell = g.cell_off + ((int64_t)x * g.n[1] + y) * g.n[2] + z;
          const int a = __ldg(&start[cell]), e = __ldg(&start[cell + 1]);
          for (int u = a; u < e; ++u) {
            const float4 pp = __ldg(&sorted[u]);
            const int p = __float_as_int(pp.w);
            const float d = dist2(pp.x, pp.y, pp.z, q);
            if (m == k && !before(d, p, ld[(k - 1) * kSphBlock], li[(k - 1) * kSphBlock])) continue;
            int j = m < k ? m++ : k - 1;
            while (j > 0 && before(d, p, ld[(j - 1) * kSphBlock], li[(j - 1) * kSphBlock])) {
              ld[j * kSphBlock] = ld[(j - 1) * kSphBlock];
              li[j * kSphBlock] = li[(j - 1) * kSphBlock];
              --j;
            }
            ld[j * kSphBlock] = d;
            li[j * kSphBlock] = p;
          }
        }
      }
    }
    if (m == k) {
      // every particle outside rings 0..r is at least r * smin away
      const double b = (double)r * (double)g.smin;
      if ((double)ld[(k - 1) * kSphBlock] < b * b) break;
    }
  }
  return m;
}

struct SphParams {
  int K;
  const int64_t* vprefix;
  const SphGrid* grids;
  const int* start;
  const float4* sorted;  // x, y, z, particle index (as int bits) in cell order
  const float4* posd;
  const float* w;
  const float4* vel;
  const float* scal;
  int S;
  int k;
  int extensive;
  float dx;  // kernel table step 2/1000
  float* h;
  double* d;  // particle density (scalar fields only) or null
  // grid
  const dtfe_subbox* boxes;
  const int64_t* tile_prefix;
  int64_t n_cells;
  const float* xs;
  const float* ys;
  const float* zs;
  double* acc;  // per flattened tile sample: density, 3 velocity, S scalars
  int AC;       // doubles per sample
};

__global__ void __launch_bounds__(kSphBlock) k_sph_particles(SphParams P, int64_t v0, int64_t v1) {
  extern __shared__ unsigned char smem[];
  float* ld = reinterpret_cast<float*>(smem) + threadIdx.x;
  int* li = reinterpret_cast<int*>(smem + sizeof(float) * P.k * kSphBlock) + threadIdx.x;
  const int64_t i = v0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= v1) return;
  const int b = find_range(P.vprefix, P.K, i);
  const SphGrid g = P.grids[b];
  const float4 pi = __ldg(&P.posd[i]);
  const float q[3] = {pi.x, pi.y, pi.z};
  const int m = knn(g, P.start, P.sorted, q, P.k, ld, li);
  const float h = (float)((double)sqrtf(ld[(m - 1) * kSphBlock]) / 2.);
  P.h[i] = h;
  if (!P.d) return;
  const float c1 = 1.f / (h * h * h);
  const float wi = __ldg(&P.w[i]);
  double own = 0.0;
  for (int j = 0; j < m; ++j) {
    const int id = li[j * kSphBlock];
    const float r = sqrtf(ld[j * kSphBlock]);
    const int bin = (int)(r / (h * P.dx));
    own += (double)(0.5f * __ldg(&P.w[id]) * c1 * c_W[bin]);
    atomicAdd(&P.d[id], (double)(0.5f * wi * c1 * c_W[bin]));
  }
  atomicAdd(&P.d[i], own);
}

struct Sample {
  int b, i, j, k;
  int64_t local;
};

__device__ __forceinline__ Sample sample_of(const SphParams& P, int64_t s) {
  Sample c;
  c.b = find_range(P.tile_prefix, P.K, s);
  const dtfe_subbox& B = P.boxes[c.b];
  c.local = s - P.tile_prefix[c.b];
  const int nz = B.tile_dims[2], ny = B.tile_dims[1];
  tile_ijk(c.local, ny, nz, c.i, c.j, c.k);
  return c;
}

__global__ void __launch_bounds__(kSphBlock) k_sph_gather(SphParams P) {
  extern __shared__ unsigned char smem[];
  float* ld = reinterpret_cast<float*>(smem) + threadIdx.x;
  int* li = reinterpret_cast<int*>(smem + sizeof(float) * P.k * kSphBlock) + threadIdx.x;
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= P.n_cells) return;
  const Sample c = sample_of(P, s);
  const dtfe_subbox& B = P.boxes[c.b];
  const float q[3] = {__ldg(&P.xs[B.coord_offset[0] + c.i]), __ldg(&P.ys[B.coord_offset[1] + c.j]),
                      __ldg(&P.zs[B.coord_offset[2] + c.k])};
  const SphGrid g = P.grids[c.b];
  const int m = knn(g, P.start, P.sorted, q, P.k, ld, li);
  const float h = (float)((double)sqrtf(ld[(m - 1) * kSphBlock]) / 2.);
  const float c1 = 1.f / (h * h * h);
  double rd = 0.0, rv[3] = {0.0, 0.0, 0.0}, rs[DTFE_MAX_SCALARS];
  for (int q2 = 0; q2 < P.S; ++q2) rs[q2] = 0.0;
  for (int j = 0; j < m; ++j) {
    const int id = li[j * kSphBlock];
    const float r = sqrtf(ld[j * kSphBlock]);
    const int bin = (int)(r / (h * P.dx));
    const float t1 = 0.5f * __ldg(&P.w[id]) * c1 * c_W[bin];
    rd += (double)t1;
    if (P.vel) {
      const float4 v = __ldg(&P.vel[id]);
      rv[0] += (double)(v.x * t1);
      rv[1] += (double)(v.y * t1);
      rv[2] += (double)(v.z * t1);
    }
    for (int q2 = 0; q2 < P.S; ++q2) {
      const float sv = __ldg(&P.scal[(int64_t)P.S * id + q2]);
      rs[q2] += P.extensive ? (double)(sv * t1 / (float)P.d[id]) : (double)(sv * t1);
    }
  }
  double* a = P.acc + s * P.AC;
  a[0] = rd;
  a[1] = rv[0];
  a[2] = rv[1];
  a[3] = rv[2];
  for (int q2 = 0; q2 < P.S; ++q2) a[4 + q2] = rs[q2];
}

// First index of a sorted float table with value >= x (or > x when UPPER).
template <bool UPPER>
__device__ __forceinline__ int bound_in(const float* __restrict__ t, int n, float x) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    const float v = __ldg(&t[mid]);
    if (UPPER ? (v <= x) : (v < x)) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__global__ void __launch_bounds__(kSphBlock) k_sph_scatter(SphParams P, int64_t v0, int64_t v1) {
  const int64_t i = v0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= v1) return;
  const int b = find_range(P.vprefix, P.K, i);
  const dtfe_subbox& B = P.boxes[b];
  const float4 pp = __ldg(&P.posd[i]);
  const float p[3] = {pp.x, pp.y, pp.z};
  const float h = P.h[i];
  const float r2 = 4.f * h * h;
  const float rr = sqrtf(r2) * 1.0001f + 1e-6f;
  const float* tab[3] = {P.xs + B.coord_offset[0], P.ys + B.coord_offset[1], P.zs + B.coord_offset[2]};
  int lo[3], hi[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    lo[c] = bound_in<false>(tab[c], B.tile_dims[c], p[c] - rr);
    hi[c] = bound_in<true>(tab[c], B.tile_dims[c], p[c] + rr);
  }
  const float c1 = 0.5f * __ldg(&P.w[i]) * (1.f / (h * h * h));
  float v[3] = {0.f, 0.f, 0.f};
  if (P.vel) {
    const float4 u = __ldg(&P.vel[i]);
    v[0] = u.x; v[1] = u.y; v[2] = u.z;
  }
  const int64_t base = P.tile_prefix[b];
  for (int a = lo[0]; a < hi[0]; ++a)
    for (int bb = lo[1]; bb < hi[1]; ++bb)
      for (int cc = lo[2]; cc < hi[2]; ++cc) {
        const float y[3] = {__ldg(&tab[0][a]), __ldg(&tab[1][bb]), __ldg(&tab[2][cc])};
        const float dd = dist2(y[0], y[1], y[2], p);
        if (!(dd <= r2)) continue;
        const float r = sqrtf(dd);
        const int bin = (int)(r / (h * P.dx));
        const float t1 = c1 * c_W[bin];
        double* acc = P.acc + (base + ((int64_t)a * B.tile_dims[1] + bb) * B.tile_dims[2] + cc) * P.AC;
        atomicAdd(&acc[0], (double)t1);
        if (P.vel) {
          atomicAdd(&acc[1], (double)(v[0] * t1));
          atomicAdd(&acc[2], (double)(v[1] * t1));
          atomicAdd(&acc[3], (double)(v[2] * t1));
        }
        for (int q2 = 0; q2 < P.S; ++q2) {
          const float sv = __ldg(&P.scal[(int64_t)P.S * i + q2]);
          atomicAdd(&acc[4 + q2], P.extensive ? (double)(sv * t1) : (double)(sv * t1 / (float)P.d[i]));
        }
      }
}

__global__ void k_sph_finalize(SphParams P, int64_t G1, int64_t G2, float factor, float* __restrict__ dens,
                               float* __restrict__ vel, float* __restrict__ scal) {
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= P.n_cells) return;
  const Sample c = sample_of(P, s);
  const dtfe_subbox& B = P.boxes[c.b];
  const int64_t cell = ((int64_t)(B.tile_origin[0] + c.i) * G1 + (B.tile_origin[1] + c.j)) * G2 + (B.tile_origin[2] + c.k);
  const double* a = P.acc + s * P.AC;
  const float D = (float)a[0];
  if (vel)
#pragma unroll
    for (int q = 0; q < 3; ++q) vel[3 * cell + q] = (float)a[1 + q] / D;
  if (scal)
    for (int q = 0; q < P.S; ++q)
      scal[(int64_t)P.S * cell + q] = P.extensive ? (float)a[4 + q] : (float)a[4 + q] / D;
  if (dens) dens[cell] = D * factor;
}

float kernel_w(float x) {
  const float f = (float)(1. / 3.14159265);
  if (std::fabs(x) <= 1.) return f * (float)(1. - 1.5 * x * x + 0.75 * x * x * x);
  if (std::fabs(x) <= 2.) {
    const float t = (float)(2. - x);
    return f * (float)(0.25 * t * t * t);
  }
  return 0.f;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

// Sub-box geometry and vertex data of the handle; outputs in main-grid
// layout on the device.  fields: DTFE_FIELD_BIT of DTFE_DENSITY,
// DTFE_VELOCITY, DTFE_SCALAR.
extern "C" int dtfe_internal_sph(void* stream, int K, const dtfe_subbox* boxes_h, const dtfe_subbox* boxes_d,
                                 const int64_t* tile_prefix_d, int64_t n_cells, int64_t G1, int64_t G2,
                                 const float* xs, const float* ys, const float* zs, int64_t V, const float4* posd,
                                 const float* w, const float4* vel4, const float* scal, int S, int k,
                                 uint32_t fields, int extensive, double average_density, float* dens_out,
                                 float* vel_out, float* scal_out, void** scratch, size_t* scratch_bytes) {
  cudaStream_t st = (cudaStream_t)stream;
  if (k < 1 || k > kMaxNeighbours) return dtfe_internal_set_error(DTFE_ERR_ARG, "SPH neighbours must be in 1..128");
  const bool want_vel = (fields & DTFE_FIELD_BIT(DTFE_VELOCITY)) != 0;
  const bool want_sc = (fields & DTFE_FIELD_BIT(DTFE_SCALAR)) != 0;
  if ((want_vel && (!vel4 || !vel_out)) || (want_sc && (S <= 0 || !scal || !scal_out)))
    return dtfe_internal_set_error(DTFE_ERR_ARG, "SPH field requested without its input or output");
  if (!(average_density > 0.0)) return dtfe_internal_set_error(DTFE_ERR_ARG, "averageDensity must be positive");
  std::vector<int64_t> vprefix(K + 1);
  for (int b = 0; b < K; ++b) {
    vprefix[b] = boxes_h[b].vert_offset;
    if (boxes_h[b].n_verts < k)
      return dtfe_internal_set_error(DTFE_ERR_ARG, "a sub-box has fewer particles than SPH neighbours");
  }
  vprefix[K] = boxes_h[K - 1].vert_offset + boxes_h[K - 1].n_verts;
  const int64_t v0 = vprefix[0], v1 = vprefix[K], nv = v1 - v0;
  const int64_t cmax = nv / 2 + K + 1;  // k_sph_params makes at most np/2 cells (>= 1) per sub-box
  const int AC = 4 + (want_sc ? S : 0);
  size_t cub_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, cub_bytes, (int*)nullptr, (int*)nullptr, (int)(cmax + 1), st);
  const size_t sizes[] = {sizeof(int64_t) * (K + 1), sizeof(int) * 6 * K, sizeof(SphGrid) * K, sizeof(int64_t),
                          sizeof(int) * (cmax + 1), sizeof(int) * (cmax + 1), sizeof(int) * nv, sizeof(float4) * nv,
                          sizeof(float) * V, want_sc ? sizeof(double) * V : 0, sizeof(double) * AC * n_cells,
                          cub_bytes};
  constexpr int NB = sizeof(sizes) / sizeof(sizes[0]);
  size_t need = 0;
  for (int q = 0; q < NB; ++q) need += align256(sizes[q]);
  if (*scratch_bytes < need) {
    if (*scratch) cudaFree(*scratch);
    *scratch = nullptr;
    *scratch_bytes = 0;
    if (cudaMalloc(scratch, need) != cudaSuccess) return dtfe_internal_set_error(DTFE_ERR_ALLOC, "cudaMalloc (SPH)");
    *scratch_bytes = need;
  }
  char* base = (char*)*scratch;
  void* part[NB];
  for (int q = 0; q < NB; ++q) {
    part[q] = base;
    base += align256(sizes[q]);
  }
  int64_t* d_vprefix = (int64_t*)part[0];
  int* d_bounds = (int*)part[1];
  SphGrid* d_grids = (SphGrid*)part[2];
  int64_t* d_total = (int64_t*)part[3];
  int* d_count = (int*)part[4];
  int* d_start = (int*)part[5];
  int* d_rank = (int*)part[6];
  float4* d_sorted = (float4*)part[7];
  float* d_h = (float*)part[8];
  double* d_d = want_sc ? (double*)part[9] : nullptr;
  double* d_acc = (double*)part[10];
  void* d_cub = part[11];

  static bool table_ready[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  cudaError_t e;
  if (dev < 64 && !table_ready[dev]) {
    float W[kTable + 1];
    const float dx = (float)(2. / kTable);
    for (int q = 0; q <= kTable; ++q) W[q] = kernel_w((float)(dx * (q + 0.5)));
    if ((e = cudaMemcpyToSymbol(c_W, W, sizeof(W))) != cudaSuccess)
      return dtfe_internal_set_error(DTFE_ERR_CUDA, cudaGetErrorString(e));
    const int smem_max = (int)((sizeof(float) + sizeof(int)) * kMaxNeighbours * kSphBlock);
    cudaFuncSetAttribute(k_sph_particles, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    cudaFuncSetAttribute(k_sph_gather, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
    table_ready[dev] = true;
  }
  std::vector<int> init(6 * K);
  for (int b = 0; b < K; ++b)
    for (int c = 0; c < 3; ++c) {
      init[6 * b + 2 * c] = 0x7FFFFFFF;        // ordered(+max)
      init[6 * b + 2 * c + 1] = (int)0x80000000;  // ordered(-max)
    }
  cudaMemcpyAsync(d_vprefix, vprefix.data(), sizeof(int64_t) * (K + 1), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_bounds, init.data(), sizeof(int) * 6 * K, cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(d_count, 0, sizeof(int) * (cmax + 1), st);
  if (d_d) cudaMemsetAsync(d_d, 0, sizeof(double) * V, st);
  const unsigned nb_v = (unsigned)((nv + kSphBlock - 1) / kSphBlock);
  const unsigned nb_c = (unsigned)((n_cells + kSphBlock - 1) / kSphBlock);
  k_sph_bounds<<<nb_v, kSphBlock, 0, st>>>(v0, v1, d_vprefix, K, posd, d_bounds);
  k_sph_params<<<1, 1, 0, st>>>(K, d_vprefix, d_bounds, d_grids, d_total);
  k_sph_count<<<nb_v, kSphBlock, 0, st>>>(v0, v1, d_vprefix, K, d_grids, posd, d_count, d_rank);
  cub::DeviceScan::ExclusiveSum(d_cub, cub_bytes, d_count, d_start, (int)(cmax + 1), st);
  k_sph_place<<<nb_v, kSphBlock, 0, st>>>(v0, v1, d_vprefix, K, d_grids, posd, d_start, d_rank, d_sorted);
  SphParams P;
  P.K = K;
  P.vprefix = d_vprefix;
  P.grids = d_grids;
  P.start = d_start;
  P.sorted = d_sorted;
  P.posd = posd;
  P.w = w;
  P.vel = want_vel ? vel4 : nullptr;
  P.scal = want_sc ? scal : nullptr;
  P.S = want_sc ? S : 0;
  P.k = k;
  P.extensive = extensive ? 1 : 0;
  P.dx = (float)(2. / kTable);
  P.h = d_h;
  P.d = d_d;
  P.boxes = boxes_d;
  P.tile_prefix = tile_prefix_d;
  P.n_cells = n_cells;
  P.xs = xs;
  P.ys = ys;
  P.zs = zs;
  P.acc = d_acc;
  P.AC = AC;
  const size_t smem = (sizeof(float) + sizeof(int)) * (size_t)k * kSphBlock;
  k_sph_particles<<<nb_v, kSphBlock, smem, st>>>(P, v0, v1);
  k_sph_gather<<<nb_c, kSphBlock, smem, st>>>(P);
  k_sph_scatter<<<nb_v, kSphBlock, 0, st>>>(P, v0, v1);
  const float factor = (float)(1. / (double)(float)average_density);
  k_sph_finalize<<<nb_c, kSphBlock, 0, st>>>(P, G1, G2, factor, dens_out, want_vel ? vel_out : nullptr,
                                             want_sc ? scal_out : nullptr);
  if ((e = cudaGetLastError()) != cudaSuccess) return dtfe_internal_set_error(DTFE_ERR_CUDA, cudaGetErrorString(e));
  return DTFE_OK;
}
