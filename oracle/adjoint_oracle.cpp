// CPU oracle for the adjoints — TEST INFRASTRUCTURE ONLY (tests/ use it as
// the checker of dtfe_gpu_adjoint_dev and dtfe_gpu_deposit_adjoint_dev; the
// product never calls it).
//
// The reference (lrwesterhoek/DTFE) has no gradients.  What is
// differentiated here is its forward arithmetic, restated in FP64:
//   * vertex density rho_v = factor * m_v / sum of incident tetrahedron
//     volumes (vertexDensity, src/triangulation_miscellaneous.cc:30-75), zero
//     on the convex hull;
//   * cell-centre density, velocity and velocity divergence from the tetrahedron that
//     holds the cell centre (interpolateGrid, src/unaveraged_interpolation.cc:
//     60-210: value at vertex 0 plus gradient . offset; gradient = inverse edge
//     matrix times value differences, src/triangulation_miscellaneous.cc:80-130
//     with its 1e-6 singular cutoff);
//   * NGP / CIC / TSC density (src/CIC_interpolation.cc, src/TSC_interpolation.cc:
//     per-axis stencils clipped at the region boundary, density = mass *
//     region cells / 35000^3 / average density).
// Loss L = sum_c a_c density_c (+ c_c . velocity_c + b_c divergence_c).  Each function comes
// as a loss (for central finite differences) and as its analytic gradient.
// Topology and the cell -> tetrahedron assignment are inputs (frozen).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

double orient6(const double* a, const double* b, const double* c, const double* d) {
  const double bx = b[0] - a[0], by = b[1] - a[1], bz = b[2] - a[2];
  const double cx = c[0] - a[0], cy = c[1] - a[1], cz = c[2] - a[2];
  const double dx = d[0] - a[0], dy = d[1] - a[1], dz = d[2] - a[2];
  return bx * (cy * dz - cz * dy) + by * (cz * dx - cx * dz) + bz * (cx * dy - cy * dx);
}

bool inverse3(const double A[3][3], double Mi[3][3]) {
  double c[3][3];
  for (int r = 0; r < 3; ++r)
    for (int q = 0; q < 3; ++q) {
      const int r1 = (r + 1) % 3, r2 = (r + 2) % 3, q1 = (q + 1) % 3, q2 = (q + 2) % 3;
      c[r][q] = A[r1][q1] * A[r2][q2] - A[r1][q2] * A[r2][q1];
    }
  const double det = A[0][0] * c[0][0] + A[0][1] * c[0][1] + A[0][2] * c[0][2];
  double s = 0;
  for (int r = 0; r < 3; ++r)
    for (int q = 0; q < 3; ++q) s += std::fabs(A[r][q]);
  const bool ok = std::fabs(det / s) > 1.e-6;
  for (int r = 0; r < 3; ++r)
    for (int q = 0; q < 3; ++q) Mi[r][q] = ok ? c[q][r] / det : 0.0;
  return ok;
}

struct Mesh {
  int64_t T, V;
  const int32_t* tv;
  const double* x;
  const double* w;
  const double* vel;
  const int32_t* hull;
  double factor;
  std::vector<double> vol, S, rho;
  void densities() {
    vol.assign(T, 0.0);
    S.assign(V, 0.0);
    rho.assign(V, 0.0);
    for (int64_t t = 0; t < T; ++t) {
      const int32_t* q = tv + 4 * t;
      vol[t] = orient6(x + 3 * q[0], x + 3 * q[1], x + 3 * q[2], x + 3 * q[3]) / 6.0;
      for (int a = 0; a < 4; ++a) S[q[a]] += vol[t];
    }
    for (int64_t v = 0; v < V; ++v) rho[v] = (hull[v] || S[v] == 0.0) ? 0.0 : factor * w[v] / S[v];
  }
};

}  // namespace

extern "C" {

// L = sum_c a_c rho(p_c) + c_c . vel(p_c) + b_c div(p_c) over G samples with
// loc[c] >= 0.  tv: 4T int32; x, vel: 3V; w, hull: V; pts: 3G; a, b: G and
// cw: 3G (each may be NULL).  full_value: velocity value from the full offset
// product (1) or from its z term only (0, unaveraged_interpolation.cc:116).
double oracle_dtfe_loss(int64_t T, const int32_t* tv, int64_t V, const double* x, const double* w,
                        const double* vel, const int32_t* hull, double factor, int64_t G, const int64_t* loc,
                        const double* pts, const double* a, const double* cw, const double* b, int full_value) {
  Mesh m{T, V, tv, x, w, vel, hull, factor, {}, {}, {}};
  m.densities();
  double L = 0.0;
  for (int64_t c = 0; c < G; ++c) {
    const int64_t t = loc[c];
    if (t < 0) continue;
    const double wa = a ? a[c] : 0.0, wb = b ? b[c] : 0.0;
    const double wc[3] = {cw ? cw[3 * c] : 0.0, cw ? cw[3 * c + 1] : 0.0, cw ? cw[3 * c + 2] : 0.0};
    const int32_t* q = tv + 4 * t;
    double A[3][3], Mi[3][3];
    for (int r = 0; r < 3; ++r)
      for (int k = 0; k < 3; ++k) A[r][k] = x[3 * q[r + 1] + k] - x[3 * q[0] + k];
    inverse3(A, Mi);
    if (cw) {
      for (int i = 0; i < 3; ++i) {
        double val = vel[3 * q[0] + i];
        for (int j = full_value ? 0 : 2; j < 3; ++j) {
          double g = 0;
          for (int k = 0; k < 3; ++k) g += Mi[j][k] * (vel[3 * q[k + 1] + i] - vel[3 * q[0] + i]);
          val += (pts[3 * c + j] - x[3 * q[0] + j]) * g;
        }
        L += wc[i] * val;
      }
    }
    if (wa != 0.0) {
      double val = m.rho[q[0]];
      for (int r = 0; r < 3; ++r) {
        double g = 0;
        for (int k = 0; k < 3; ++k) g += Mi[r][k] * (m.rho[q[k + 1]] - m.rho[q[0]]);
        val += (pts[3 * c + r] - x[3 * q[0] + r]) * g;
      }
      L += wa * val;
    }
    if (wb != 0.0) {
      double div = 0;
      for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 3; ++k) div += Mi[r][k] * (vel[3 * q[k + 1] + r] - vel[3 * q[0] + r]);
      L += wb * div;
    }
  }
  return L;
}

// Analytic gradient of oracle_dtfe_loss: gx, gv (3V) and gw (V), overwritten.
void oracle_dtfe_grad(int64_t T, const int32_t* tv, int64_t V, const double* x, const double* w, const double* vel,
                      const int32_t* hull, double factor, int64_t G, const int64_t* loc, const double* pts,
                      const double* a, const double* cw, const double* b, int full_value, double* gx, double* gv,
                      double* gw) {
  Mesh m{T, V, tv, x, w, vel, hull, factor, {}, {}, {}};
  m.densities();
  std::vector<double> grho(V, 0.0);
  std::memset(gx, 0, sizeof(double) * 3 * V);
  std::memset(gv, 0, sizeof(double) * 3 * V);
  for (int64_t c = 0; c < G; ++c) {
    const int64_t t = loc[c];
    if (t < 0) continue;
    const double wa = a ? a[c] : 0.0, wb = b ? b[c] : 0.0;
    const int32_t* q = tv + 4 * t;
    double A[3][3], Mi[3][3];
    for (int r = 0; r < 3; ++r)
      for (int k = 0; k < 3; ++k) A[r][k] = x[3 * q[r + 1] + k] - x[3 * q[0] + k];
    inverse3(A, Mi);
    // barycentric coordinates of the sample
    double lam[4], rr[3];
    for (int k = 0; k < 3; ++k) rr[k] = pts[3 * c + k] - x[3 * q[0] + k];
    for (int k = 0; k < 3; ++k) lam[k + 1] = Mi[0][k] * rr[0] + Mi[1][k] * rr[1] + Mi[2][k] * rr[2];
    lam[0] = 1.0 - lam[1] - lam[2] - lam[3];
    if (wa != 0.0) {
      double g[3];
      for (int r = 0; r < 3; ++r) {
        g[r] = 0;
        for (int k = 0; k < 3; ++k) g[r] += Mi[r][k] * (m.rho[q[k + 1]] - m.rho[q[0]]);
      }
      for (int j = 0; j < 4; ++j) {
        grho[q[j]] += wa * lam[j];
        for (int k = 0; k < 3; ++k) gx[3 * q[j] + k] -= wa * lam[j] * g[k];
      }
    }
    const double wc[3] = {cw ? cw[3 * c] : 0.0, cw ? cw[3 * c + 1] : 0.0, cw ? cw[3 * c + 2] : 0.0};
    if (wb != 0.0 || wc[0] != 0.0 || wc[1] != 0.0 || wc[2] != 0.0) {
      // velocity_i = v_0i + sum_j u_j r_j VG[j][i], divergence = tr VG,
      // VG = A^-1 DV; reverse mode through VG, r = p - x_0 and A^-1
      const double u[3] = {full_value ? 1.0 : 0.0, full_value ? 1.0 : 0.0, 1.0};
      double DV[3][3], VG[3][3], GV[3][3], GAi[3][3], grel[3];
      for (int k = 0; k < 3; ++k)
        for (int j = 0; j < 3; ++j) DV[k][j] = vel[3 * q[k + 1] + j] - vel[3 * q[0] + j];
      for (int r = 0; r < 3; ++r)
        for (int j = 0; j < 3; ++j) {
          VG[r][j] = 0;
          for (int k = 0; k < 3; ++k) VG[r][j] += Mi[r][k] * DV[k][j];
        }
      for (int r = 0; r < 3; ++r) {
        grel[r] = 0;
        for (int i = 0; i < 3; ++i) {
          GV[r][i] = u[r] * rr[r] * wc[i] + (r == i ? wb : 0.0);
          grel[r] += u[r] * wc[i] * VG[r][i];
        }
      }
      for (int i = 0; i < 3; ++i) gv[3 * q[0] + i] += wc[i];
      for (int k = 0; k < 3; ++k)
        for (int i = 0; i < 3; ++i) {
          double gdv = 0;
          for (int r = 0; r < 3; ++r) gdv += Mi[r][k] * GV[r][i];
          gv[3 * q[k + 1] + i] += gdv;
          gv[3 * q[0] + i] -= gdv;
        }
      for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 3; ++k) {
          GAi[r][k] = 0;
          for (int i = 0; i < 3; ++i) GAi[r][k] += GV[r][i] * DV[k][i];
        }
      // dL/dA[k][j] = -(A^-T GAi A^-T)[k][j]
      for (int k = 0; k < 3; ++k)
        for (int j = 0; j < 3; ++j) {
          double gA = 0;
          for (int r = 0; r < 3; ++r)
            for (int s2 = 0; s2 < 3; ++s2) gA -= Mi[r][k] * GAi[r][s2] * Mi[j][s2];
          gx[3 * q[k + 1] + j] += gA;
          gx[3 * q[0] + j] -= gA;
        }
      for (int j = 0; j < 3; ++j) gx[3 * q[0] + j] -= grel[j];
    }
  }
  // vertex densities: rho_v = factor w_v / S_v
  std::vector<double> gS(V, 0.0);
  for (int64_t v = 0; v < V; ++v) {
    if (m.hull[v] || m.S[v] == 0.0) {
      gw[v] = 0.0;
      continue;
    }
    gw[v] = grho[v] * factor / m.S[v];
    gS[v] = -grho[v] * factor * w[v] / (m.S[v] * m.S[v]);
  }
  for (int64_t t = 0; t < T; ++t) {
    const int32_t* q = tv + 4 * t;
    const double vb = gS[q[0]] + gS[q[1]] + gS[q[2]] + gS[q[3]];
    if (vb == 0.0) continue;
    const double* X[4] = {x + 3 * q[0], x + 3 * q[1], x + 3 * q[2], x + 3 * q[3]};
    // d(6V)/d x_j by perturbation-free formulas: for j >= 1 the cross product
    // of the other two edges from vertex 0 in cyclic order.
    double e[3][3];
    for (int r = 0; r < 3; ++r)
      for (int k = 0; k < 3; ++k) e[r][k] = X[r + 1][k] - X[0][k];
    double d[4][3];
    for (int j = 1; j <= 3; ++j) {
      const double* u = e[j % 3];
      const double* s = e[(j + 1) % 3];
      d[j][0] = u[1] * s[2] - u[2] * s[1];
      d[j][1] = u[2] * s[0] - u[0] * s[2];
      d[j][2] = u[0] * s[1] - u[1] * s[0];
    }
    for (int k = 0; k < 3; ++k) d[0][k] = -(d[1][k] + d[2][k] + d[3][k]);
    for (int j = 0; j < 4; ++j)
      for (int k = 0; k < 3; ++k) gx[3 * q[j] + k] += vb * d[j][k] / 6.0;
  }
}

// ---- NGP / CIC / TSC ------------------------------------------------------
// One axis of the stencil in FP64 (cells relative to the region, weights,
// their derivatives with respect to the normalised coordinate).  `inner`:
// the particle lies inside the region shrunk by the stencil half-width.
static int dep_axis(int kind, bool inner, double temp, int n, int cell[3], double w[3], double dw[3]) {
  auto tsc = [](double t, double* ww, double* dd) {
    ww[0] = 0.5 * (0.5 - t) * (0.5 - t);
    ww[1] = 0.75 - t * t;
    ww[2] = 0.5 * (0.5 + t) * (0.5 + t);
    dd[0] = -(0.5 - t);
    dd[1] = -2.0 * t;
    dd[2] = 0.5 + t;
  };
  auto cic = [](double t, double* ww, double* dd) {
    if (t < 0) { ww[0] = -t; ww[1] = 1 + t; ww[2] = 0; dd[0] = -1; dd[1] = 1; dd[2] = 0; }
    else { ww[0] = 0; ww[1] = 1 - t; ww[2] = t; dd[0] = 0; dd[1] = -1; dd[2] = 1; }
  };
  double W[3], D[3];
  if (inner) {
    const int c1 = (int)std::floor(temp);
    const double t = temp - (c1 + 0.5);
    kind == 1 ? cic(t, W, D) : tsc(t, W, D);
    for (int q = 0; q < 3; ++q) { cell[q] = c1 - 1 + q; w[q] = W[q]; dw[q] = D[q]; }
    return 3;
  }
  const int ti = (int)std::floor(temp);
  const double t = temp - (ti + 0.5);
  if (ti < -1 || ti > n) return 0;
  if (kind == 1) {
    // edge cells of the reference's CIC loop (linear in t, may be negative)
    if (ti == -1) { cell[0] = 0; w[0] = t; dw[0] = 1; return 1; }
    if (ti == 0) { cell[0] = 0; cell[1] = 1; w[0] = 1 - t; w[1] = t; dw[0] = -1; dw[1] = 1; return 2; }
    if (ti == n - 1) { cell[0] = n - 2; cell[1] = n - 1; w[0] = -t; w[1] = 1 + t; dw[0] = -1; dw[1] = 1; return 2; }
    if (ti == n) { cell[0] = n - 1; w[0] = -t; dw[0] = -1; return 1; }
    cic(t, W, D);
  } else {
    tsc(t, W, D);
    if (ti == -1) { cell[0] = 0; w[0] = W[2]; dw[0] = D[2]; return 1; }
    if (ti == 0) { cell[0] = 0; cell[1] = 1; w[0] = W[1]; w[1] = W[2]; dw[0] = D[1]; dw[1] = D[2]; return 2; }
    if (ti == n - 1) { cell[0] = n - 2; cell[1] = n - 1; w[0] = W[0]; w[1] = W[1]; dw[0] = D[0]; dw[1] = D[1]; return 2; }
    if (ti == n) { cell[0] = n - 1; w[0] = W[0]; dw[0] = D[0]; return 1; }
  }
  for (int q = 0; q < 3; ++q) { cell[q] = ti - 1 + q; w[q] = W[q]; dw[q] = D[q]; }
  return 3;
}

// L = sum_c a_c density_c of one region's deposition (kind 0 NGP, 1 CIC,
// 2 TSC); with gx / gw non-NULL also its gradient (3n, n).  Cell sizes and
// stencil extents follow the reference's float region arithmetic.
double oracle_deposit_loss_grad(int kind, const double* pos, const double* w, int64_t n, const float region[6],
                                const int32_t grid[3], double average_density, const double* a, double* gx,
                                double* gw) {
  float lo[3], dx[3];
  for (int k = 0; k < 3; ++k) {
    lo[k] = region[2 * k];
    dx[k] = (region[2 * k + 1] - region[2 * k]) / (float)grid[k];
  }
  const int64_t cells = (int64_t)grid[0] * grid[1] * grid[2];
  const float boxvol = 35000.f * 35000.f * 35000.f;
  const double factor = (double)((float)cells / boxvol / (float)average_density);
  // the reference's region tests: the full stencil inside the region shrunk
  // by 1.1 cells, the clipped one inside the region grown by one cell
  float inner_b[6], outer_b[6];
  for (int k = 0; k < 3; ++k) {
    const float ipad = (float)(-1.1 * (double)dx[k]);
    outer_b[2 * k] = region[2 * k] - dx[k];
    outer_b[2 * k + 1] = region[2 * k + 1] + dx[k];
    inner_b[2 * k] = region[2 * k] - ipad;
    inner_b[2 * k + 1] = region[2 * k + 1] + ipad;
  }
  double L = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    const double* p = pos + 3 * i;
    int cell[3][3], cnt[3] = {0, 0, 0};
    double ww[3][3], dw[3][3];
    if (kind == 0) {
      bool ok = true;
      for (int k = 0; k < 3; ++k) {
        cell[k][0] = (int)std::floor((p[k] - lo[k]) / dx[k]);
        ww[k][0] = 1;
        dw[k][0] = 0;
        ok = ok && cell[k][0] >= 0 && cell[k][0] < grid[k];
      }
      if (ok) cnt[0] = cnt[1] = cnt[2] = 1;
    } else {
      bool inner = true, outer = true;
      for (int k = 0; k < 3; ++k) {
        const float pk = (float)p[k];
        inner = inner && pk >= inner_b[2 * k] && pk <= inner_b[2 * k + 1];
        outer = outer && pk >= outer_b[2 * k] && pk <= outer_b[2 * k + 1];
      }
      if (inner || outer)
        for (int k = 0; k < 3; ++k)
          cnt[k] = dep_axis(kind, inner, (p[k] - lo[k]) / dx[k], grid[k], cell[k], ww[k], dw[k]);
    }
    double sm = 0, sx[3] = {0, 0, 0};
    for (int x0 = 0; x0 < cnt[0]; ++x0)
      for (int x1 = 0; x1 < cnt[1]; ++x1)
        for (int x2 = 0; x2 < cnt[2]; ++x2) {
          const int64_t idx = ((int64_t)cell[0][x0] * grid[1] + cell[1][x1]) * grid[2] + cell[2][x2];
          const double ac = a[idx];
          sm += ac * ww[0][x0] * ww[1][x1] * ww[2][x2];
          sx[0] += ac * dw[0][x0] / dx[0] * ww[1][x1] * ww[2][x2];
          sx[1] += ac * ww[0][x0] * dw[1][x1] / dx[1] * ww[2][x2];
          sx[2] += ac * ww[0][x0] * ww[1][x1] * dw[2][x2] / dx[2];
        }
    L += factor * w[i] * sm;
    if (gw) gw[i] = factor * sm;
    if (gx)
      for (int k = 0; k < 3; ++k) gx[3 * i + k] = factor * w[i] * sx[k];
  }
  return L;
}


// ---- local central finite differences --------------------------------------
// FP64 central differences of oracle_dtfe_loss with respect to the inputs of
// selected particles.  A particle is the set of vertices that are its
// periodic images (sel_verts[sel_off[i] .. sel_off[i+1])); a step moves all
// of them.  Only the terms a step changes are re-evaluated: the volumes of
// the tetrahedra around the images, the densities of those tetrahedra's
// vertices and the cells located in any tetrahedron of such a vertex, so the
// difference equals that of the full loss without its cost.
// out: 7 values per particle (d/dx, d/dy, d/dz, d/dvx, d/dvy, d/dvz, d/dw).
}  // extern "C"

namespace {

struct LocalFD {
  int64_t T, V, G;
  const int32_t* tv;
  const double* x;
  const double* w;
  const double* vel;
  const int32_t* hull;
  double factor;
  const int64_t* loc;
  const double* pts;
  const double *a, *cw, *b;
  int full;
  std::vector<int64_t> inc_off, tcell_off;
  std::vector<int32_t> inc, tcell;
  std::vector<double> vol, S;

  void build() {
    inc_off.assign(V + 1, 0);
    for (int64_t t = 0; t < T; ++t)
      for (int k = 0; k < 4; ++k) ++inc_off[tv[4 * t + k] + 1];
    for (int64_t v = 0; v < V; ++v) inc_off[v + 1] += inc_off[v];
    inc.resize(inc_off[V]);
    std::vector<int64_t> fill(inc_off.begin(), inc_off.end() - 1);
    for (int64_t t = 0; t < T; ++t)
      for (int k = 0; k < 4; ++k) inc[fill[tv[4 * t + k]]++] = (int32_t)t;
    tcell_off.assign(T + 1, 0);
    for (int64_t c = 0; c < G; ++c)
      if (loc[c] >= 0) ++tcell_off[loc[c] + 1];
    for (int64_t t = 0; t < T; ++t) tcell_off[t + 1] += tcell_off[t];
    tcell.resize(tcell_off[T]);
    fill.assign(tcell_off.begin(), tcell_off.end() - 1);
    for (int64_t c = 0; c < G; ++c)
      if (loc[c] >= 0) tcell[fill[loc[c]]++] = (int32_t)c;
    vol.assign(T, 0.0);
    S.assign(V, 0.0);
    for (int64_t t = 0; t < T; ++t) {
      const int32_t* q = tv + 4 * t;
      vol[t] = orient6(x + 3 * q[0], x + 3 * q[1], x + 3 * q[2], x + 3 * q[3]) / 6.0;
      for (int k = 0; k < 4; ++k) S[q[k]] += vol[t];
    }
  }
};

}  // namespace

extern "C" {

void oracle_dtfe_fd(int64_t T, const int32_t* tv, int64_t V, const double* x, const double* w, const double* vel,
                    const int32_t* hull, double factor, int64_t G, const int64_t* loc, const double* pts,
                    const double* a, const double* cw, const double* b, int full_value, int64_t n_sel,
                    const int64_t* sel_off, const int32_t* sel_verts, double h_pos, double h_vel, double h_w,
                    double* out) {
  LocalFD F{T, V, G, tv, x, w, vel, hull, factor, loc, pts, a, cw, b, full_value, {}, {}, {}, {}, {}, {}};
  F.build();
  for (int64_t i = 0; i < n_sel; ++i) {
    const int32_t* U = sel_verts + sel_off[i];
    const int nU = (int)(sel_off[i + 1] - sel_off[i]);
    std::vector<int32_t> T1, W, T2, cells;
    for (int u = 0; u < nU; ++u)
      for (int64_t q = F.inc_off[U[u]]; q < F.inc_off[U[u] + 1]; ++q) T1.push_back(F.inc[q]);
    std::sort(T1.begin(), T1.end());
    T1.erase(std::unique(T1.begin(), T1.end()), T1.end());
    for (int32_t t : T1)
      for (int k = 0; k < 4; ++k) W.push_back(tv[4 * t + k]);
    std::sort(W.begin(), W.end());
    W.erase(std::unique(W.begin(), W.end()), W.end());
    for (int32_t v : W)
      for (int64_t q = F.inc_off[v]; q < F.inc_off[v + 1]; ++q) T2.push_back(F.inc[q]);
    std::sort(T2.begin(), T2.end());
    T2.erase(std::unique(T2.begin(), T2.end()), T2.end());
    for (int32_t t : T2)
      for (int64_t q = F.tcell_off[t]; q < F.tcell_off[t + 1]; ++q) cells.push_back(F.tcell[q]);

    // local copies of the moved vertices' inputs
    auto in_U = [&](int32_t v) {
      for (int u = 0; u < nU; ++u)
        if (U[u] == v) return u;
      return -1;
    };
    std::vector<double> xu(3 * nU), vu(3 * nU), wu(nU);
    auto eval = [&]() {
      auto X = [&](int32_t v, int k) {
        const int u = in_U(v);
        return u >= 0 ? xu[3 * u + k] : x[3 * v + k];
      };
      auto Vl = [&](int32_t v, int k) {
        const int u = in_U(v);
        return u >= 0 ? vu[3 * u + k] : vel[3 * v + k];
      };
      auto Wt = [&](int32_t v) {
        const int u = in_U(v);
        return u >= 0 ? wu[u] : w[v];
      };
      // densities of W from updated incident volumes
      std::vector<double> rhoW(W.size());
      for (size_t k = 0; k < W.size(); ++k) {
        const int32_t v = W[k];
        double S = F.S[v];
        for (int64_t q = F.inc_off[v]; q < F.inc_off[v + 1]; ++q) {
          const int32_t t = F.inc[q];
          if (!std::binary_search(T1.begin(), T1.end(), t)) continue;
          double P[4][3];
          for (int j = 0; j < 4; ++j)
            for (int c = 0; c < 3; ++c) P[j][c] = X(tv[4 * t + j], c);
          S += orient6(P[0], P[1], P[2], P[3]) / 6.0 - F.vol[t];
        }
        rhoW[k] = (hull[v] || S == 0.0) ? 0.0 : factor * Wt(v) / S;
      }
      auto rho = [&](int32_t v) {
        auto it = std::lower_bound(W.begin(), W.end(), v);
        if (it != W.end() && *it == v) return rhoW[it - W.begin()];
        const double S = F.S[v];
        return (hull[v] || S == 0.0) ? 0.0 : factor * w[v] / S;
      };
      double L = 0.0;
      for (int32_t c : cells) {
        const int32_t* q = tv + 4 * loc[c];
        const double wa = a ? a[c] : 0.0, wb = b ? b[c] : 0.0;
        double A[3][3], Mi[3][3], rel[3];
        for (int r = 0; r < 3; ++r)
          for (int k = 0; k < 3; ++k) A[r][k] = X(q[r + 1], k) - X(q[0], k);
        inverse3(A, Mi);
        for (int k = 0; k < 3; ++k) rel[k] = pts[3 * c + k] - X(q[0], k);
        if (wa != 0.0) {
          double val = rho(q[0]);
          for (int r = 0; r < 3; ++r) {
            double g = 0;
            for (int k = 0; k < 3; ++k) g += Mi[r][k] * (rho(q[k + 1]) - rho(q[0]));
            val += rel[r] * g;
          }
          L += wa * val;
        }
        if (cw || wb != 0.0) {
          double VG[3][3];
          for (int r = 0; r < 3; ++r)
            for (int j = 0; j < 3; ++j) {
              VG[r][j] = 0;
              for (int k = 0; k < 3; ++k) VG[r][j] += Mi[r][k] * (Vl(q[k + 1], j) - Vl(q[0], j));
            }
          L += wb * (VG[0][0] + VG[1][1] + VG[2][2]);
          if (cw)
            for (int j = 0; j < 3; ++j) {
              double val = Vl(q[0], j);
              for (int r = full_value ? 0 : 2; r < 3; ++r) val += rel[r] * VG[r][j];
              L += cw[3 * c + j] * val;
            }
        }
      }
      return L;
    };
    auto reset = [&]() {
      for (int u = 0; u < nU; ++u) {
        for (int k = 0; k < 3; ++k) {
          xu[3 * u + k] = x[3 * U[u] + k];
          vu[3 * u + k] = vel[3 * U[u] + k];
        }
        wu[u] = w[U[u]];
      }
    };
    for (int p = 0; p < 7; ++p) {
      const double h = p < 3 ? h_pos : (p < 6 ? h_vel : h_w);
      double Lp, Lm;
      for (int sgn = 0; sgn < 2; ++sgn) {
        reset();
        const double d = sgn == 0 ? h : -h;
        for (int u = 0; u < nU; ++u) {
          if (p < 3) xu[3 * u + p] += d;
          else if (p < 6) vu[3 * u + p - 3] += d;
          else wu[u] += d;
        }
        (sgn == 0 ? Lp : Lm) = eval();
      }
      out[7 * i + p] = (Lp - Lm) / (2.0 * h);
    }
  }
}

}  // extern "C"
