// Host 3-D Delaunay tessellator.
//
// Replaces delaunayTriangulation() (src/CGAL_triangulation/triangulation.cpp:162-195),
// which inserts the spatially sorted particles one by one into a CGAL
// Delaunay_triangulation_3 (Epick kernel, Fast_location).  CGAL is not
// available to this project, so the same construction is written here:
//
//  * Bowyer-Watson incremental insertion with an "infinite vertex" closing the
//    convex hull (a tetrahedron that contains the infinite vertex is the
//    counterpart of CGAL's infinite cell, dt.is_infinite(cell));
//  * biased randomized insertion order (random rounds, each sorted along a
//    Morton curve) and a visibility walk from the last created tetrahedron,
//    the role CGAL::spatial_sort + insert(p, hint) play in the reference;
//  * exact predicates (predicates.h), so the result is the Delaunay
//    tessellation of the input doubles.  With strict in-sphere conflicts,
//    co-spherical ties keep the existing tetrahedra.
//
// Output is the flat format the GPU path consumes: finite tetrahedra only,
// positively oriented (CGAL's cell orientation), tet_v[4t+i] = vertex i,
// tet_n[4t+i] = the tetrahedron across the face opposite vertex i, or -1 when
// that face lies on the convex hull (the neighbour would be an infinite cell).
// Duplicate points are merged: like CGAL's insert() of an existing point they
// map onto the first inserted vertex at that position (vmap).

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

#include "predicates.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int32_t INF = -1;

inline uint64_t spread21(uint64_t x) {
  x &= 0x1fffffULL;
  x = (x | (x << 32)) & 0x1f00000000ffffULL;
  x = (x | (x << 16)) & 0x1f0000ff0000ffULL;
  x = (x | (x << 8)) & 0x100f00f00f00f00fULL;
  x = (x | (x << 4)) & 0x10c30c30c30c30c3ULL;
  x = (x | (x << 2)) & 0x1249249249249249ULL;
  return x;
}

struct MortonFrame {
  double lo[3], scale[3];
  MortonFrame(const double* P, int64_t n) {
    for (int k = 0; k < 3; ++k) { lo[k] = 1e300; scale[k] = -1e300; }
    for (int64_t i = 0; i < n; ++i)
      for (int k = 0; k < 3; ++k) {
        lo[k] = std::min(lo[k], P[3 * i + k]);
        scale[k] = std::max(scale[k], P[3 * i + k]);
      }
    for (int k = 0; k < 3; ++k) {
      double ext = scale[k] - lo[k];
      scale[k] = ext > 0 ? (double)((1 << 21) - 1) / ext : 0.0;
    }
  }
  uint64_t key(const double* p) const {
    uint64_t c[3];
    for (int k = 0; k < 3; ++k) {
      double t = (p[k] - lo[k]) * scale[k];
      if (t < 0) t = 0;
      if (t > (double)((1 << 21) - 1)) t = (double)((1 << 21) - 1);
      c[k] = (uint64_t)t;
    }
    return spread21(c[0]) | (spread21(c[1]) << 1) | (spread21(c[2]) << 2);
  }
};

struct Tessellator {
  const double* P;
  int64_t n;
  std::vector<int32_t> cells;  // per tetrahedron: 4 vertices, then 4 neighbours (one 32-byte record)
  std::vector<uint32_t> mark;
  std::vector<int32_t> freelist;
  std::vector<int32_t> vmap;
  uint32_t stamp = 0;
  int32_t hint = 0;
  int64_t n_dup = 0;
  int status = 0;

  // per-insertion scratch
  std::vector<int32_t> stack, cavity;
  std::vector<std::pair<int32_t, int>> boundary;
  std::vector<int32_t> created;
  std::vector<uint64_t> hkey;
  std::vector<int32_t> hval;
  std::vector<uint32_t> hstamp;
  uint32_t hround = 0;

  Tessellator(const double* pts, int64_t npts) : P(pts), n(npts) {}

  const double* pt(int32_t v) const { return P + 3 * (int64_t)v; }

  int32_t new_tet() {
    if (!freelist.empty()) {
      int32_t t = freelist.back();
      freelist.pop_back();
      return t;
    }
    int32_t t = (int32_t)(cells.size() / 8);
    cells.resize(cells.size() + 8);
    mark.push_back(0);
    return t;
  }

  int inf_index(int32_t t) const {
    for (int k = 0; k < 4; ++k)
      if (cells[8 * (int64_t)t + k] == INF) return k;
    return -1;
  }

  // orientation of tetrahedron t with vertex k replaced by point p
  int orient_with(int32_t t, int k, const double* p) const {
    const double* q[4];
    for (int i = 0; i < 4; ++i) q[i] = (i == k) ? p : pt(cells[8 * (int64_t)t + i]);
    return dtfe::orient(q[0], q[1], q[2], q[3]);
  }

  bool conflict(int32_t t, const double* p) const {
    int k = inf_index(t);
    if (k < 0) {
      const int32_t* v = &cells[8 * (int64_t)t];
      return dtfe::insphere(pt(v[0]), pt(v[1]), pt(v[2]), pt(v[3]), p) > 0;
    }
    int o = orient_with(t, k, p);
    if (o > 0) return true;
    if (o < 0) return false;
    // p on the plane of the hull face: in conflict iff it lies inside the
    // face's circumcircle, i.e. inside the circumsphere of the finite
    // neighbour across that face.
    int32_t f = cells[8 * (int64_t)t + 4 + k];
    const int32_t* v = &cells[8 * (int64_t)f];
    return dtfe::insphere(pt(v[0]), pt(v[1]), pt(v[2]), pt(v[3]), p) > 0;
  }

  // Walk to a tetrahedron in conflict with p.  Returns the tetrahedron, or
  // sets dup to the vertex that coincides with p.
  int32_t locate(const double* p, int32_t start, int32_t& dup) {
    dup = -1;
    int32_t t = start;
    int k = inf_index(t);
    if (k >= 0) {
      if (orient_with(t, k, p) > 0) return t;
      t = cells[8 * (int64_t)t + 4 + k];
    }
    int32_t prev = -1;
    uint32_t rot = 0;
    for (int64_t step = 0;; ++step) {
      bool moved = false;
      for (int j = 0; j < 4; ++j) {
        int i = (int)((j + rot) & 3);
        int32_t nb = cells[8 * (int64_t)t + 4 + i];
        if (nb == prev) continue;
        if (orient_with(t, i, p) < 0) {
          prev = t;
          t = nb;
          moved = true;
          break;
        }
      }
      if (!moved) break;
      if (inf_index(t) >= 0) return t;  // crossed a hull face
      rot = rot * 1103515245u + 12345u;
      rot >>= 16;
      if (step > 4 * (int64_t)(cells.size() / 8) + 1000) {
        status = 2;
        return t;
      }
    }
    for (int i = 0; i < 4; ++i) {
      const double* q = pt(cells[8 * (int64_t)t + i]);
      if (q[0] == p[0] && q[1] == p[1] && q[2] == p[2]) {
        dup = cells[8 * (int64_t)t + i];
        return t;
      }
    }
    return t;
  }

  void hash_reset(size_t need) {
    size_t sz = hkey.size();
    if (sz < 2 * need + 16) {
      sz = 64;
      while (sz < 2 * need + 16) sz <<= 1;
      hkey.assign(sz, 0);
      hval.assign(sz, 0);
      hstamp.assign(sz, 0);
      hround = 0;
    }
    ++hround;
  }

  // Registers the half-face (tet nt, local face m) keyed by edge (a,b); links
  // it with its twin when the twin is already registered.
  void hash_link(int32_t a, int32_t b, int32_t nt, int m) {
    if (a > b) std::swap(a, b);
    uint64_t key = ((uint64_t)(uint32_t)a << 32) | (uint32_t)b;
    size_t mask = hkey.size() - 1;
    size_t h = (size_t)((key * 0x9E3779B97F4A7C15ULL) >> 20) & mask;
    for (;;) {
      if (hstamp[h] != hround) {
        hstamp[h] = hround;
        hkey[h] = key;
        hval[h] = nt * 4 + m;
        return;
      }
      if (hkey[h] == key) {
        int32_t ot = hval[h] >> 2;
        int om = hval[h] & 3;
        cells[8 * (int64_t)nt + 4 + m] = ot;
        cells[8 * (int64_t)ot + 4 + om] = nt;
        hkey[h] = ~0ULL;  // consumed: each interior face has one twin
        return;
      }
      h = (h + 1) & mask;
    }
  }

  bool insert(int32_t pi) {
    const double* p = pt(pi);
    int32_t dup;
    int32_t t0 = locate(p, hint, dup);
    if (status) return false;
    if (dup >= 0) {
      vmap[pi] = dup;
      ++n_dup;
      return true;
    }
    const uint32_t s_in = ++stamp;
    const uint32_t s_out = ++stamp;
    stack.clear();
    cavity.clear();
    boundary.clear();
    stack.push_back(t0);
    mark[t0] = s_in;
    while (!stack.empty()) {
      int32_t t = stack.back();
      stack.pop_back();
      cavity.push_back(t);
      for (int k = 0; k < 4; ++k) {
        int32_t u = cells[8 * (int64_t)t + 4 + k];
        if (mark[u] == s_in) continue;
        if (mark[u] == s_out) {
          boundary.emplace_back(t, k);
          continue;
        }
        if (conflict(u, p)) {
          mark[u] = s_in;
          stack.push_back(u);
        } else {
          mark[u] = s_out;
          boundary.emplace_back(t, k);
        }
      }
    }
    created.clear();
    hash_reset(3 * boundary.size());
    for (auto& bf : boundary) {
      int32_t t = bf.first;
      int k = bf.second;
      int32_t u = cells[8 * (int64_t)t + 4 + k];
      int32_t nt = new_tet();
      mark[nt] = 0;
      for (int i = 0; i < 4; ++i) cells[8 * (int64_t)nt + i] = cells[8 * (int64_t)t + i];
      cells[8 * (int64_t)nt + k] = pi;
      cells[8 * (int64_t)nt + 4 + k] = u;
      for (int j = 0; j < 4; ++j)
        if (cells[8 * (int64_t)u + 4 + j] == t) {
          cells[8 * (int64_t)u + 4 + j] = nt;
          break;
        }
      created.push_back(nt);
    }
    for (size_t c = 0; c < created.size(); ++c) {
      int32_t nt = created[c];
      int k = boundary[c].second;
      for (int m = 0; m < 4; ++m) {
        if (m == k) continue;
        int32_t e[2];
        int ne = 0;
        for (int i = 0; i < 4; ++i)
          if (i != m && i != k) e[ne++] = cells[8 * (int64_t)nt + i];
        hash_link(e[0], e[1], nt, m);
      }
    }
    for (int32_t t : cavity) {
      cells[8 * (int64_t)t] = cells[8 * (int64_t)t + 1] = cells[8 * (int64_t)t + 2] = cells[8 * (int64_t)t + 3] = -2;
      freelist.push_back(t);
    }
    hint = created.back();
    return true;
  }

  // Builds the first tetrahedron and its four infinite neighbours.  Returns
  // the positions in `order` of the four points used, or false if all points
  // are coplanar.
  bool init(const std::vector<int32_t>& order, int used[4]) {
    int64_t m = (int64_t)order.size();
    int i0 = 0, i1 = -1, i2 = -1, i3 = -1;
    const double* p0 = pt(order[0]);
    for (int64_t i = 1; i < m && i1 < 0; ++i) {
      const double* q = pt(order[i]);
      if (q[0] != p0[0] || q[1] != p0[1] || q[2] != p0[2]) i1 = (int)i;
    }
    if (i1 < 0) return false;
    const double* p1 = pt(order[i1]);
    int tries = 0;
    for (int64_t cand = 1; cand < m && i3 < 0 && tries < 3; ++cand) {
      if (cand == i1) continue;
      const double* q = pt(order[cand]);
      double ux = p1[0] - p0[0], uy = p1[1] - p0[1], uz = p1[2] - p0[2];
      double vx = q[0] - p0[0], vy = q[1] - p0[1], vz = q[2] - p0[2];
      double cx = uy * vz - uz * vy, cy = uz * vx - ux * vz, cz = ux * vy - uy * vx;
      if (cx == 0 && cy == 0 && cz == 0) continue;
      ++tries;  // a rounded cross product can hide exact collinearity
      i2 = (int)cand;
      for (int64_t j = 1; j < m; ++j) {
        if (j == i1 || j == i2) continue;
        if (dtfe::orient(p0, p1, q, pt(order[j])) != 0) {
          i3 = (int)j;
          break;
        }
      }
    }
    if (i3 < 0) return false;  // all points coplanar
    used[0] = i0; used[1] = i1; used[2] = i2; used[3] = i3;
    int32_t v[4] = {order[i0], order[i1], order[i2], order[i3]};
    if (dtfe::orient(pt(v[0]), pt(v[1]), pt(v[2]), pt(v[3])) < 0) std::swap(v[2], v[3]);
    int32_t T[5];
    for (int i = 0; i < 5; ++i) T[i] = new_tet();
    for (int i = 0; i < 4; ++i) cells[8 * (int64_t)T[0] + i] = v[i];
    for (int k = 0; k < 4; ++k) {
      int32_t t = T[1 + k];
      for (int i = 0; i < 4; ++i) cells[8 * (int64_t)t + i] = v[i];
      cells[8 * (int64_t)t + k] = INF;
      // the infinite vertex lies on the far side of face k: flip orientation
      int a = (k + 1) & 3, b = (k + 2) & 3;
      std::swap(cells[8 * (int64_t)t + a], cells[8 * (int64_t)t + b]);
    }
    for (int x = 0; x < 5; ++x)
      for (int y = 0; y < 5; ++y) {
        if (x == y) continue;
        int32_t tx = T[x], ty = T[y];
        // face of tx opposite i is shared with ty when ty holds the other 3
        for (int i = 0; i < 4; ++i) {
          int shared = 0;
          for (int a = 0; a < 4; ++a) {
            if (a == i) continue;
            for (int b = 0; b < 4; ++b)
              if (cells[8 * (int64_t)ty + b] == cells[8 * (int64_t)tx + a]) { ++shared; break; }
          }
          if (shared == 3) cells[8 * (int64_t)tx + 4 + i] = ty;
        }
      }
    hint = T[0];
    return true;
  }

  int run(uint64_t seed) {
    vmap.resize(n);
    std::iota(vmap.begin(), vmap.end(), 0);
    if (n < 4) return 1;
    // biased randomized insertion order: shuffle, split into rounds of
    // doubling size, sort each round along a Morton curve
    std::vector<int32_t> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::mt19937_64 rng(seed);
    std::shuffle(order.begin(), order.end(), rng);
    MortonFrame frame(P, n);
    std::vector<int64_t> cuts;
    int64_t hi = n;
    cuts.push_back(hi);
    while (hi > 2048) {
      hi /= 2;
      cuts.push_back(hi);
    }
    cuts.push_back(0);
    std::reverse(cuts.begin(), cuts.end());
    {
      std::vector<std::pair<uint64_t, int32_t>> keyed;
      for (size_t r = 0; r + 1 < cuts.size(); ++r) {
        int64_t a = cuts[r], b = cuts[r + 1];
        keyed.resize(b - a);
        for (int64_t i = a; i < b; ++i) keyed[i - a] = {frame.key(pt(order[i])), order[i]};
        std::sort(keyed.begin(), keyed.end());
        for (int64_t i = a; i < b; ++i) order[i] = keyed[i - a].second;
      }
    }
    size_t reserve = (size_t)(n * 7.2) + 64;
    cells.reserve(8 * reserve);
    mark.reserve(reserve);
    int used[4];
    if (!init(order, used)) return 1;
    std::vector<char> skip(n, 0);
    for (int i = 0; i < 4; ++i) skip[used[i]] = 1;
    for (int64_t i = 0; i < n; ++i) {
      if (skip[i]) continue;
      if (!insert(order[i])) return status ? status : 3;
    }
    return 0;
  }
};

struct Result {
  std::vector<int32_t> tet_v, tet_n, vmap;
  int64_t n_dup = 0;
};

void compact(Tessellator& T, bool sort_tets, Result& R) {
  int64_t cap = (int64_t)T.cells.size() / 8;
  std::vector<int32_t> newid(cap, -1);
  std::vector<int32_t> finite;
  finite.reserve(cap);
  for (int64_t t = 0; t < cap; ++t) {
    const int32_t* v = &T.cells[8 * (int64_t)t];
    if (v[0] < 0 || v[1] < 0 || v[2] < 0 || v[3] < 0) continue;  // infinite or freed
    finite.push_back((int32_t)t);
  }
  // Canonical vertex order per tetrahedron: of the 12 orientation-preserving
  // (even) permutations the lexicographically smallest vertex tuple.  With
  // the sort below the output depends only on the point set (for a unique
  // Delaunay tessellation), not on the insertion order.
  static const int kEven[12][4] = {{0, 1, 2, 3}, {0, 2, 3, 1}, {0, 3, 1, 2}, {1, 0, 3, 2}, {1, 2, 0, 3},
                                   {1, 3, 2, 0}, {2, 0, 1, 3}, {2, 1, 3, 0}, {2, 3, 0, 1}, {3, 0, 2, 1},
                                   {3, 1, 0, 2}, {3, 2, 1, 0}};
  std::vector<int8_t> perm(cap, 0);
  for (int32_t t : finite) {
    const int32_t* v = &T.cells[8 * (int64_t)((int64_t)t)];
    int best = 0;
    for (int q = 1; q < 12; ++q)
      for (int k = 0; k < 4; ++k) {
        const int32_t a = v[kEven[q][k]], b = v[kEven[best][k]];
        if (a != b) {
          if (a < b) best = q;
          break;
        }
      }
    perm[t] = (int8_t)best;
  }
  auto vert = [&](int64_t t, int k) { return T.cells[8 * (int64_t)t + kEven[perm[t]][k]]; };
  if (sort_tets && !finite.empty()) {
    // order: Morton key of the centroid, then the vertex tuple (a total
    // order: no two tetrahedra share their vertices).  An LSD radix sort of
    // the keys (stable, 8 bits per pass) and a tuple sort inside each run of
    // equal keys give exactly that order.
    MortonFrame frame(T.P, T.n);
    const size_t nf = finite.size();
    std::vector<uint64_t> key(nf), key2(nf);
    std::vector<int32_t> ord(nf), ord2(nf);
    for (size_t i = 0; i < nf; ++i) {
      const int64_t t = finite[i];
      double c[3] = {0, 0, 0};
      for (int a = 0; a < 4; ++a)
        for (int k = 0; k < 3; ++k) c[k] += 0.25 * T.pt(vert(t, a))[k];
      key[i] = frame.key(c);
      ord[i] = (int32_t)i;
    }
    for (int shift = 0; shift < 64; shift += 8) {
      size_t count[257] = {0};
      for (size_t i = 0; i < nf; ++i) ++count[((key[i] >> shift) & 0xff) + 1];
      if (count[1 + ((key[0] >> shift) & 0xff)] == nf) continue;  // one digit value: nothing to move
      for (int d = 0; d < 256; ++d) count[d + 1] += count[d];
      for (size_t i = 0; i < nf; ++i) {
        const size_t dst = count[(key[i] >> shift) & 0xff]++;
        key2[dst] = key[i];
        ord2[dst] = ord[i];
      }
      key.swap(key2);
      ord.swap(ord2);
    }
    auto tuple_less = [&](int32_t x, int32_t y) {
      for (int a = 0; a < 4; ++a) {
        const int32_t vx = vert(finite[x], a), vy = vert(finite[y], a);
        if (vx != vy) return vx < vy;
      }
      return false;
    };
    for (size_t i = 0; i < nf;) {
      size_t j = i + 1;
      while (j < nf && key[j] == key[i]) ++j;
      if (j - i > 1) std::sort(ord.begin() + i, ord.begin() + j, tuple_less);
      i = j;
    }
    std::vector<int32_t> sorted(nf);
    for (size_t i = 0; i < nf; ++i) sorted[i] = finite[ord[i]];
    finite.swap(sorted);
  }
  for (size_t i = 0; i < finite.size(); ++i) newid[finite[i]] = (int32_t)i;
  R.tet_v.resize(4 * finite.size());
  R.tet_n.resize(4 * finite.size());
  for (size_t i = 0; i < finite.size(); ++i) {
    int64_t t = finite[i];
    for (int k = 0; k < 4; ++k) {
      const int src = kEven[perm[t]][k];
      R.tet_v[4 * i + k] = T.cells[8 * (int64_t)t + src];
      int32_t nb = T.cells[8 * (int64_t)t + 4 + src];
      R.tet_n[4 * i + k] = newid[nb];  // -1 for an infinite neighbour
    }
  }
  R.vmap.swap(T.vmap);
  R.n_dup = T.n_dup;
}

}  // namespace

extern "C" {

// Tessellates n points (xyz, 3 doubles each).  On success returns 0 and an
// opaque handle; query sizes with dtfe_tess_sizes, copy with dtfe_tess_export
// and release with dtfe_tess_release.  Return codes: 1 = fewer than four
// affinely independent points, 2 = point location did not terminate (input
// not finite), 3 = internal error.
int dtfe_tessellate(const double* xyz, int64_t n, uint64_t seed, int sort_tets,
                    void** handle) {
  *handle = nullptr;
  Tessellator T(xyz, n);
  int rc = T.run(seed);
  Result* R = new Result();
  if (rc == 0) compact(T, sort_tets != 0, *R);
  else {
    R->vmap.swap(T.vmap);
  }
  *handle = R;
  return rc;
}

// Tessellates k independent point sets in parallel (one host thread each),
// e.g. the padded sub-boxes of a decomposition.  rc[i] receives each status.
void dtfe_tessellate_batch(int k, const double* const* xyz, const int64_t* n,
                           uint64_t seed, int sort_tets, void** handles,
                           int* rc) {
#pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < k; ++i)
    rc[i] = dtfe_tessellate(xyz[i], n[i], seed, sort_tets, &handles[i]);
}

void dtfe_tess_sizes(void* handle, int64_t* n_tets, int64_t* n_points,
                     int64_t* n_dup) {
  Result* R = (Result*)handle;
  *n_tets = (int64_t)R->tet_v.size() / 4;
  *n_points = (int64_t)R->vmap.size();
  *n_dup = R->n_dup;
}

void dtfe_tess_export(void* handle, int32_t* tet_v, int32_t* tet_n, int32_t* vmap) {
  Result* R = (Result*)handle;
  if (tet_v) std::memcpy(tet_v, R->tet_v.data(), R->tet_v.size() * sizeof(int32_t));
  if (tet_n) std::memcpy(tet_n, R->tet_n.data(), R->tet_n.size() * sizeof(int32_t));
  if (vmap) std::memcpy(vmap, R->vmap.data(), R->vmap.size() * sizeof(int32_t));
}

void dtfe_tess_release(void* handle) { delete (Result*)handle; }

// Exposed for tests of the predicates against exact rational arithmetic.
int dtfe_orient(const double* a, const double* b, const double* c, const double* d) {
  return dtfe::orient(a, b, c, d);
}
int dtfe_orient_exact(const double* a, const double* b, const double* c, const double* d) {
  return dtfe::orient_exact(a, b, c, d);
}
int dtfe_insphere(const double* a, const double* b, const double* c, const double* d,
                  const double* e) {
  return dtfe::insphere(a, b, c, d, e);
}
int dtfe_insphere_exact(const double* a, const double* b, const double* c,
                        const double* d, const double* e) {
  return dtfe::insphere_exact(a, b, c, d, e);
}

}  // extern "C"
