// CPU oracle for the NGP / CIC / TSC grid deposition — TEST INFRASTRUCTURE ONLY.
//
// Restates, for one region:
//   NGP_interpolation_regular_grid  src/NGP_interpolation.cc:67-136
//   CIC_interpolation_regular_grid  src/CIC_interpolation.cc:67-273
//   TSC_interpolation_regular_grid  src/TSC_interpolation.cc:67-254
// mode 0 ("ref"): the reference's float arithmetic and accumulation order
// (particles inside the region shrunk by 1.1 cells first, in input order,
// then the boundary particles with clipped stencils, in input order);
// mode 1 ("fp64"): the same weights and stencils evaluated and accumulated
// in double.  Outputs are doubles.

#include <cmath>
#include <cstdint>
#include <vector>

namespace {

// Box::volume() is hard-coded to 35000^3 (src/box.h:142-149).
template <class R>
R box_volume() {
  R t = 1;
  for (int i = 0; i < 3; ++i) t *= 35000;
  return t;
}

template <class R>
struct Stencil {
  int cell[3][3];
  R w[3][3];
  int count[3];
};

// Weights of one axis.  kind 1 CIC, 2 TSC.  inner: full 3-cell stencil.
template <class R>
void axis_weights(int kind, bool inner, R temp_in, int n, int cell[3], R w[3], int& count) {
  R temp = temp_in;
  count = 0;
  if (inner) {
    cell[0] = (int)std::floor(temp) - 1;
    cell[1] = cell[0] + 1;
    cell[2] = cell[1] + 1;
    temp = (R)((double)temp - ((double)cell[1] + 0.5));
    count = 3;
    if (kind == 1) {
      if (temp < 0.) { w[0] = -temp; w[1] = 1 + temp; w[2] = 0.; }
      else { w[0] = 0.; w[1] = 1 - temp; w[2] = temp; }
    } else {
      w[0] = (R)(.5 * (0.5 - (double)temp) * (0.5 - (double)temp));
      w[1] = (R)(.75 - (double)(temp * temp));
      w[2] = (R)(.5 * (0.5 + (double)temp) * (0.5 + (double)temp));
    }
    return;
  }
  int ti = (int)std::floor(temp);
  temp = (R)((double)temp - ((double)ti + 0.5));
  auto a = [&](R t) { return (R)(.5 * (0.5 - (double)t) * (0.5 - (double)t)); };
  auto b = [&](R t) { return (R)(.75 - (double)(t * t)); };
  auto c = [&](R t) { return (R)(.5 * (0.5 + (double)t) * (0.5 + (double)t)); };
  if (ti == -1) {
    cell[0] = 0; count = 1;
    w[0] = kind == 1 ? temp : c(temp);
  } else if (ti == 0) {
    cell[0] = 0; cell[1] = 1; count = 2;
    if (kind == 1) { w[0] = 1 - temp; w[1] = temp; }
    else { w[0] = b(temp); w[1] = c(temp); }
  } else if (ti == n - 1) {
    cell[0] = n - 2; cell[1] = n - 1; count = 2;
    if (kind == 1) { w[0] = -temp; w[1] = 1 + temp; }
    else { w[0] = a(temp); w[1] = b(temp); }
  } else if (ti == n) {
    cell[0] = n - 1; count = 1;
    w[0] = kind == 1 ? -temp : a(temp);
  } else if (!(ti < -1 || ti > n)) {
    cell[0] = ti - 1; cell[1] = ti; cell[2] = ti + 1; count = 3;
    if (kind == 1) {
      if (temp < 0.) { w[0] = -temp; w[1] = 1 + temp; w[2] = 0.; }
      else { w[0] = 0.; w[1] = 1 - temp; w[2] = temp; }
    } else {
      w[0] = a(temp); w[1] = b(temp); w[2] = c(temp);
    }
  }
}

template <class R>
void deposit(int kind, const float* pos, const float* wt, const float* vel, int64_t n, const float region[6],
             const int32_t grid[3], double avg, double* dens_out, double* vel_out) {
  const int64_t G = (int64_t)grid[0] * grid[1] * grid[2];
  std::vector<R> dens(G, 0), mom(3 * G, 0);
  float dx[3], inner[6], outer[6];
  for (int i = 0; i < 3; ++i) dx[i] = (region[2 * i + 1] - region[2 * i]) / (float)grid[i];
  for (int i = 0; i < 3; ++i) {
    float pad = dx[i];
    float ipad = (float)(-1.1 * (double)pad);
    outer[2 * i] = region[2 * i] - pad;
    outer[2 * i + 1] = region[2 * i + 1] + pad;
    inner[2 * i] = region[2 * i] - ipad;
    inner[2 * i + 1] = region[2 * i + 1] + ipad;
  }
  auto in_box = [](const float* p, const float* b) {
    return p[0] >= b[0] && p[0] <= b[1] && p[1] >= b[2] && p[1] <= b[3] && p[2] >= b[4] && p[2] <= b[5];
  };
  auto add = [&](int64_t i, int64_t idx, R result) {
    dens[idx] += result;
    for (int c = 0; c < 3; ++c) mom[3 * idx + c] += (R)(vel ? vel[3 * i + c] : 0.f) * result;
  };
  if (kind == 0) {
    for (int64_t i = 0; i < n; ++i) {
      int cell[3];
      bool ok = true;
      for (int j = 0; j < 3; ++j) {
        cell[j] = (int)std::floor((pos[3 * i + j] - region[2 * j]) / dx[j]);
        if (cell[j] < 0 || cell[j] >= grid[j]) ok = false;
      }
      if (!ok) continue;
      int64_t idx = ((int64_t)cell[0] * grid[1] + cell[1]) * grid[2] + cell[2];
      add(i, idx, (R)(wt ? wt[i] : 1.f));
    }
  } else {
    for (int pass = 0; pass < 2; ++pass)
      for (int64_t i = 0; i < n; ++i) {
        const float* p = &pos[3 * i];
        bool is_inner = in_box(p, inner);
        if (pass == 0 && !is_inner) continue;
        if (pass == 1 && (is_inner || !in_box(p, outer))) continue;
        Stencil<R> s;
        for (int j = 0; j < 3; ++j) {
          R temp = (R)((p[j] - region[2 * j]) / dx[j]);
          axis_weights<R>(kind, is_inner, temp, grid[j], s.cell[j], s.w[j], s.count[j]);
        }
        R w0 = (R)(wt ? wt[i] : 1.f);
        for (int a = 0; a < s.count[0]; ++a)
          for (int b = 0; b < s.count[1]; ++b)
            for (int c = 0; c < s.count[2]; ++c) {
              int64_t idx = ((int64_t)s.cell[0][a] * grid[1] + s.cell[1][b]) * grid[2] + s.cell[2][c];
              R result = w0 * s.w[0][a] * s.w[1][b] * s.w[2][c];
              add(i, idx, result);
            }
      }
  }
  R factor = (R)G / box_volume<R>() / (R)avg;
  for (int64_t i = 0; i < G; ++i) {
    if (vel_out)
      for (int c = 0; c < 3; ++c) vel_out[3 * i + c] = dens[i] != 0 ? (double)(mom[3 * i + c] / dens[i]) : 0.0;
    if (dens_out) dens_out[i] = (double)(dens[i] * factor);
  }
}

}  // namespace

extern "C" int oracle_deposit(int kind, int mode, const float* pos, const float* w, const float* vel, int64_t n,
                              const float region[6], const int32_t grid[3], double average_density,
                              double* density, double* velocity) {
  if (kind < 0 || kind > 2) return 1;
  if (kind > 0 && (grid[0] < 3 || grid[1] < 3 || grid[2] < 3)) return 1;
  if (mode == 0) deposit<float>(kind, pos, w, vel, n, region, grid, average_density, density, velocity);
  else deposit<double>(kind, pos, w, vel, n, region, grid, average_density, density, velocity);
  return 0;
}
