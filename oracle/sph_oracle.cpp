// CPU oracle for the SPH grid estimator — TEST INFRASTRUCTURE ONLY.
//
// Restates SPH_interpolation (src/SPH_interpolation.cc:252-474) for the
// particles and grid of one region:
//   * kernel table: W[i] = SPH_smoothingKernel(dx (i + 0.5)), i = 0..1000,
//     dx = 2/1000 (:298-305, kernel :151-168);
//   * particle smoothing length h_i = sqrt(d_N)/2, d_N the squared distance
//     of the N-th nearest particle, the particle itself included (kdtree2
//     n_nearest_around_point with correltime 0);
//   * particle density d (needed for scalar fields only): for every particle
//     i and each of its N neighbours j (ascending distance),
//     d[i] += 0.5 w_j c_i W[bin], d[j] += 0.5 w_i c_i W[bin], c_i = 1/h_i^3,
//     bin = int(r / (h_i dx)) (:318-326);
//   * grid gather: per grid point its own N nearest particles, h = sqrt(d_N)/2
//     (:349-382);
//   * grid scatter: per particle i every grid point within 2 h_i (kdtree2
//     r_nearest, squared distance <= 4 h_i^2) receives 0.5 w_i c_i W[bin]
//     (:399-432);
//   * velocity and intensive scalars divided by the grid density, density
//     times 1/averageDensity (:438-462).
// Distances are float sums of float squares in axis order, as kdtree2.cpp
// computes them.  mode 0 reproduces the reference's float accumulation in
// its loop order; mode 1 evaluates the same float terms and sums them in
// double.  Neighbour search: a uniform cell grid with exact shell
// termination (the result is the set of the N smallest distances, ties
// broken by particle index).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

constexpr int kTable = 1000;

float kernel_w(float x) {
  const float factor = (float)(1. / 3.14159265);
  if (std::fabs(x) <= 1.) return factor * (float)(1. - 1.5 * x * x + 0.75 * x * x * x);
  if (std::fabs(x) <= 2.) {
    const float t = (float)(2. - x);
    return factor * (float)(0.25 * t * t * t);
  }
  return 0.f;
}

struct Table {
  float dx = (float)(2. / kTable);
  float W[kTable + 1];
  Table() {
    for (int i = 0; i <= kTable; ++i) W[i] = kernel_w((float)(dx * (i + 0.5)));
  }
};

inline float sq(float a) { return a * a; }

inline float dist2(const float* a, const float* b) {
  float d = 0.f;
  d += sq(a[0] - b[0]);
  d += sq(a[1] - b[1]);
  d += sq(a[2] - b[2]);
  return d;
}

struct CellGrid {
  float lo[3], s;
  int n[3];
  std::vector<int> start, idx;
  void build(const float* pos, int64_t np) {
    float mn[3] = {1e30f, 1e30f, 1e30f}, mx[3] = {-1e30f, -1e30f, -1e30f};
    for (int64_t i = 0; i < np; ++i)
      for (int c = 0; c < 3; ++c) {
        mn[c] = std::min(mn[c], pos[3 * i + c]);
        mx[c] = std::max(mx[c], pos[3 * i + c]);
      }
    double vol = 1.0;
    for (int c = 0; c < 3; ++c) vol *= std::max(1e-6, (double)(mx[c] - mn[c]));
    s = (float)std::cbrt(vol * 2.0 / std::max<int64_t>(np, 1));
    if (!(s > 0.f)) s = 1.f;
    for (int c = 0; c < 3; ++c) {
      lo[c] = mn[c];
      n[c] = std::max(1, std::min(1024, (int)((mx[c] - mn[c]) / s) + 1));
    }
    const int64_t nc = (int64_t)n[0] * n[1] * n[2];
    start.assign(nc + 1, 0);
    idx.resize(np);
    std::vector<int> cell(np);
    for (int64_t i = 0; i < np; ++i) {
      cell[i] = cell_of(pos + 3 * i);
      ++start[cell[i] + 1];
    }
    for (int64_t c = 0; c < nc; ++c) start[c + 1] += start[c];
    std::vector<int> fill(start.begin(), start.end() - 1);
    for (int64_t i = 0; i < np; ++i) idx[fill[cell[i]]++] = (int)i;
  }
  int axis(float x, int c) const {
    int k = (int)std::floor((x - lo[c]) / s);
    return std::min(std::max(k, 0), n[c] - 1);
  }
  int cell_of(const float* p) const { return (axis(p[0], 0) * n[1] + axis(p[1], 1)) * n[2] + axis(p[2], 2); }

  // The k nearest of q (squared distance, index), ascending; ties by index.
  void knn(const float* pos, const float* q, int k, std::vector<std::pair<float, int>>& out) const {
    out.clear();
    const int c0[3] = {axis(q[0], 0), axis(q[1], 1), axis(q[2], 2)};
    const int rmax = std::max(n[0], std::max(n[1], n[2]));
    for (int r = 0; r <= rmax; ++r) {
      for (int i = c0[0] - r; i <= c0[0] + r; ++i)
        for (int j = c0[1] - r; j <= c0[1] + r; ++j)
          for (int l = c0[2] - r; l <= c0[2] + r; ++l) {
            if (std::max(std::abs(i - c0[0]), std::max(std::abs(j - c0[1]), std::abs(l - c0[2]))) != r) continue;
            if (i < 0 || j < 0 || l < 0 || i >= n[0] || j >= n[1] || l >= n[2]) continue;
            const int c = (i * n[1] + j) * n[2] + l;
            for (int q2 = start[c]; q2 < start[c + 1]; ++q2) out.push_back({dist2(pos + 3 * idx[q2], q), idx[q2]});
          }
      if ((int)out.size() >= k) {
        std::sort(out.begin(), out.end());
        // every point outside the visited rings is at least r * s away
        const double bound = (double)r * s;
        if ((double)out[k - 1].first < bound * bound) break;
      }
    }
    std::sort(out.begin(), out.end());
    if ((int)out.size() > k) out.resize(k);
  }
};

template <class R>
void sph(const float* pos, const float* w, const float* vel, const float* scal, int S, int64_t np, const float* xs,
         const float* ys, const float* zs, const int32_t dims[3], double avg, int k, int extensive, double* dens_out,
         double* vel_out, double* scal_out) {
  static const Table tab;
  const int64_t G = (int64_t)dims[0] * dims[1] * dims[2];
  CellGrid cg;
  cg.build(pos, np);
  std::vector<float> h(np, 0.f);
  std::vector<R> d(np, (R)0);
  std::vector<std::pair<float, int>> nn;
  const int kk = (int)std::min<int64_t>(k, np);
  for (int64_t i = 0; i < np; ++i) {
    cg.knn(pos, pos + 3 * i, kk, nn);
    h[i] = (float)(std::sqrt(nn[kk - 1].first) / 2.);
    const float c1 = 1.f / (h[i] * h[i] * h[i]);
    for (const auto& e : nn) {
      const float r = std::sqrt(e.first);
      const int bin = (int)(r / (h[i] * tab.dx));
      d[i] += (R)(0.5f * w[e.second] * c1 * tab.W[bin]);
      d[e.second] += (R)(0.5f * w[i] * c1 * tab.W[bin]);
    }
  }
  std::vector<R> gd(G, (R)0), gv(3 * G, (R)0), gs((size_t)S * G, (R)0);
  for (int a = 0; a < dims[0]; ++a)
    for (int b = 0; b < dims[1]; ++b)
      for (int c = 0; c < dims[2]; ++c) {
        const int64_t g = ((int64_t)a * dims[1] + b) * dims[2] + c;
        const float y[3] = {xs[a], ys[b], zs[c]};
        cg.knn(pos, y, kk, nn);
        const float hh = (float)(std::sqrt(nn[kk - 1].first) / 2.);
        const float c1 = 1.f / (hh * hh * hh);
        R rd = 0, rv[3] = {0, 0, 0};
        std::vector<R> rs(S, (R)0);
        for (const auto& e : nn) {
          const float r = std::sqrt(e.first);
          const int bin = (int)(r / (hh * tab.dx));
          const float t1 = 0.5f * w[e.second] * c1 * tab.W[bin];
          rd += (R)t1;
          for (int q = 0; q < 3; ++q) rv[q] += (R)(vel ? vel[3 * e.second + q] * t1 : 0.f);
          for (int q = 0; q < S; ++q)
            rs[q] += extensive ? (R)(scal[(int64_t)S * e.second + q] * t1 / (float)d[e.second])
                               : (R)(scal[(int64_t)S * e.second + q] * t1);
        }
        gd[g] = rd;
        for (int q = 0; q < 3; ++q) gv[3 * g + q] = rv[q];
        for (int q = 0; q < S; ++q) gs[(size_t)S * g + q] = rs[q];
      }
  // scatter: grid points within 2 h of each particle, ascending distance
  std::vector<std::pair<float, int64_t>> pts;
  for (int64_t i = 0; i < np; ++i) {
    const float* p = pos + 3 * i;
    const float r2 = 4.f * h[i] * h[i];
    const float rr = std::sqrt(r2) * 1.0001f + 1e-6f;
    pts.clear();
    int lo_i[3], hi_i[3];
    const float* ax[3] = {xs, ys, zs};
    for (int c = 0; c < 3; ++c) {
      lo_i[c] = (int)(std::lower_bound(ax[c], ax[c] + dims[c], p[c] - rr) - ax[c]);
      hi_i[c] = (int)(std::upper_bound(ax[c], ax[c] + dims[c], p[c] + rr) - ax[c]);
    }
    for (int a = lo_i[0]; a < hi_i[0]; ++a)
      for (int b = lo_i[1]; b < hi_i[1]; ++b)
        for (int c = lo_i[2]; c < hi_i[2]; ++c) {
          const float y[3] = {xs[a], ys[b], zs[c]};
          const float dd = dist2(y, p);
          if (dd <= r2) pts.push_back({dd, ((int64_t)a * dims[1] + b) * dims[2] + c});
        }
    std::sort(pts.begin(), pts.end());
    const float c1 = 0.5f * w[i] * (1.f / (h[i] * h[i] * h[i]));
    for (const auto& e : pts) {
      const float r = std::sqrt(e.first);
      const int bin = (int)(r / (h[i] * tab.dx));
      const float t1 = c1 * tab.W[bin];
      const int64_t g = e.second;
      gd[g] += (R)t1;
      for (int q = 0; q < 3; ++q) gv[3 * g + q] += (R)(vel ? vel[3 * i + q] * t1 : 0.f);
      for (int q = 0; q < S; ++q)
        gs[(size_t)S * g + q] += extensive ? (R)(scal[(int64_t)S * i + q] * t1)
                                           : (R)(scal[(int64_t)S * i + q] * t1 / (float)d[i]);
    }
  }
  const float factor = (float)(1. / (double)(float)avg);
  for (int64_t g = 0; g < G; ++g) {
    const R D = gd[g];
    if (vel_out)
      for (int q = 0; q < 3; ++q) vel_out[3 * g + q] = (double)(gv[3 * g + q] / D);
    if (scal_out)
      for (int q = 0; q < S; ++q)
        scal_out[(size_t)S * g + q] = extensive ? (double)gs[(size_t)S * g + q] : (double)(gs[(size_t)S * g + q] / D);
    if (dens_out) dens_out[g] = (double)(D * (R)factor);
  }
}

}  // namespace

extern "C" {

// One region: np particles (pos 3np, w np, vel 3np or NULL, scal S*np or
// NULL), grid point coordinate tables xs/ys/zs (dims[0..2] entries, the
// reference's x += dx raster), k neighbours.  Outputs (doubles, G = product
// of dims): density, velocity (3G, may be NULL), scalars (S*G, may be NULL).
int oracle_sph(const float* pos, const float* w, const float* vel, const float* scal, int S, int64_t np,
               const float* xs, const float* ys, const float* zs, const int32_t dims[3], double avg, int k,
               int extensive, int mode, double* density, double* velocity, double* scalar) {
  if (np <= 0 || k <= 0) return 1;
  if (mode == 0)
    sph<float>(pos, w, vel, scal, S, np, xs, ys, zs, dims, avg, k, extensive, density, velocity, scalar);
  else
    sph<double>(pos, w, vel, scal, S, np, xs, ys, zs, dims, avg, k, extensive, density, velocity, scalar);
  return 0;
}

}  // extern "C"
