// A minimal stand-in for the parts of CGAL's Delaunay_triangulation_3 API that
// the reference's interpolation sources use — TEST INFRASTRUCTURE ONLY.
//
// It lets the reference's own src/CGAL_triangulation/triangulation.cpp
// (vertexDensity, interpolateGrid, interpolateGrid_averaged_2/_3, ...) be
// compiled here, where CGAL is not installed, and run on the SAME flat
// tessellation the GPU path and the oracle use.  Nothing of CGAL's source is
// used; each name below is implemented from CGAL's documented behaviour:
//
//   insert(p, hint)       appends a vertex; the tessellation is built lazily on
//                         first query (the project's own exact tessellator), or
//                         loaded directly with load_flat()
//   locate(p,lt,li,lj,h)  visibility walk with exact predicates; points outside
//                         the hull return an infinite cell
//   incident_cells(v,out) finite and infinite cells around v, ascending id
//   is_infinite(c)        cell holds the infinite vertex
//   tetrahedron(c).volume()  signed volume, determinant / 6 in double
//   finite vertex / cell iteration, number_of_vertices()
//
// Cells keep the vertex order of the flat arrays, so vertex(0) — the
// reference's "base" vertex — is the same vertex as on the GPU.
#pragma once

#include <algorithm>
#include <chrono>
#include <cstddef>
#include <cstdint>
#include <iterator>
#include <map>
#include <utility>
#include <vector>

#include "../../dtfe_b200/csrc/morton.h"
#include "../../dtfe_b200/csrc/predicates.h"

extern "C" int dtfe_tessellate(const double* xyz, int64_t n, uint64_t seed, int sort_tets, void** handle);
extern "C" void dtfe_tess_sizes(void* handle, int64_t* n_tets, int64_t* n_points, int64_t* n_dup);
extern "C" void dtfe_tess_export(void* handle, int32_t* tet_v, int32_t* tet_n, int32_t* vmap);
extern "C" void dtfe_tess_release(void* handle);

namespace CGAL {

struct Exact_predicates_inexact_constructions_kernel {};
struct Fast_location {};

class Timer {
  std::chrono::steady_clock::time_point t0_;
  double acc_ = 0;
  bool running_ = false;

 public:
  void start() { t0_ = std::chrono::steady_clock::now(); running_ = true; }
  void stop() {
    if (running_) acc_ += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
    running_ = false;
  }
  double time() const { return acc_; }
  void reset() { acc_ = 0; }
};

struct Bbox_2 {
  double b[4];
  Bbox_2(double a = 0, double c = 0, double d = 0, double e = 0) : b{a, c, d, e} {}
};
struct Bbox_3 {
  double b[6];
  Bbox_3(double x0 = 0, double y0 = 0, double z0 = 0, double x1 = 0, double y1 = 0, double z1 = 0)
      : b{x0, y0, z0, x1, y1, z1} {}
  double xmin() const { return b[0]; }
  double ymin() const { return b[1]; }
  double zmin() const { return b[2]; }
  double xmax() const { return b[3]; }
  double ymax() const { return b[4]; }
  double zmax() const { return b[5]; }
};
inline bool do_overlap(const Bbox_3& a, const Bbox_3& c) {
  for (int k = 0; k < 3; ++k)
    if (a.b[k + 3] < c.b[k] || c.b[k + 3] < a.b[k]) return false;
  return true;
}

template <class FT>
struct Cartesian {
  struct Point_2 {
    FT c[2];
    Point_2(FT x = 0, FT y = 0) : c{x, y} {}
  };
};
template <class K>
struct Circle_2 {};

template <class Info, class K>
struct Triangulation_vertex_base_with_info_3 {
  typedef Info info_type;
};
template <class Vb>
struct Triangulation_data_structure_3 {
  typedef Vb vertex_base;
};

struct Point_3 {
  double c[3];
  Point_3() : c{0, 0, 0} {}
  Point_3(double x, double y, double z) : c{x, y, z} {}
  double operator[](int i) const { return c[i]; }
  double x() const { return c[0]; }
  double y() const { return c[1]; }
  double z() const { return c[2]; }
};

template <class Iter, class Traits>
void spatial_sort(Iter, Iter, const Traits&) {}  // insertion order does not change a Delaunay tessellation

template <class K, class Tds, class Loc>
class Delaunay_triangulation_3 {
 public:
  typedef Point_3 Point;
  typedef typename Tds::vertex_base::info_type Info;
  enum Locate_type { VERTEX = 0, EDGE, FACET, CELL, OUTSIDE_CONVEX_HULL, OUTSIDE_AFFINE_HULL };
  struct Cell;
  struct Vertex {
    Point p;
    Info inf;
    bool infinite = false;
    int64_t id = -1;
    Point& point() { return p; }
    const Point& point() const { return p; }
    Info& info() { return inf; }
  };
  struct Cell {
    Vertex* v[4] = {nullptr, nullptr, nullptr, nullptr};
    Cell* n[4] = {nullptr, nullptr, nullptr, nullptr};
    int64_t id = -1;
    bool infinite = false;
    Vertex* vertex(int i) const { return v[i]; }
    Cell* neighbor(int i) const { return n[i]; }
  };
  // CGAL handles default-construct to null (the reference relies on it:
  // `Cell_handle current;` is the first walk hint)
  template <class T>
  struct Handle {
    T* p = nullptr;
    Handle() = default;
    Handle(T* q) : p(q) {}
    T* operator->() const { return p; }
    T& operator*() const { return *p; }
    operator T*() const { return p; }
  };
  typedef Handle<Vertex> Vertex_handle;
  typedef Handle<Cell> Cell_handle;

  // iterators over handles (dereference yields the object, -> the handle)
  template <class T>
  struct HIter {
    typedef std::forward_iterator_tag iterator_category;
    typedef T value_type;
    typedef std::ptrdiff_t difference_type;
    typedef T* pointer;
    typedef T& reference;
    T* const* it;
    HIter(T* const* p = nullptr) : it(p) {}
    T* operator->() const { return *it; }
    T& operator*() const { return **it; }
    operator T*() const { return *it; }
    operator Handle<T>() const { return Handle<T>(*it); }
    HIter& operator++() { ++it; return *this; }
    bool operator!=(const HIter& o) const { return it != o.it; }
    bool operator==(const HIter& o) const { return it == o.it; }
  };
  typedef HIter<Vertex> Finite_vertices_iterator;
  typedef HIter<Cell> Finite_cells_iterator;
  typedef HIter<Cell> Cell_iterator;

  struct Tetrahedron {
    Point q[4];
    double volume() const { return dtfe::orient_det(q[0].c, q[1].c, q[2].c, q[3].c) / 6.0; }
    Bbox_3 bbox() const {
      double lo[3], hi[3];
      for (int k = 0; k < 3; ++k) {
        lo[k] = hi[k] = q[0].c[k];
        for (int a = 1; a < 4; ++a) {
          lo[k] = std::min(lo[k], q[a].c[k]);
          hi[k] = std::max(hi[k], q[a].c[k]);
        }
      }
      return Bbox_3(lo[0], lo[1], lo[2], hi[0], hi[1], hi[2]);
    }
  };

  Delaunay_triangulation_3() { inf_vertex_.infinite = true; }
  Delaunay_triangulation_3(const Delaunay_triangulation_3&) = delete;
  ~Delaunay_triangulation_3() { clear(); }

  void clear() {
    for (Vertex* v : verts_) delete v;
    for (Cell* c : cells_) delete c;
    verts_.clear();
    cells_.clear();
    finite_cells_.clear();
    finite_verts_.clear();
    incident_.clear();
    built_ = false;
  }

  // CGAL::insert: here the point is stored and the tessellation is (re)built
  // on the next query.
  Vertex_handle insert(const Point& p, Vertex_handle = Vertex_handle()) {
    Vertex* v = new Vertex();
    v->p = p;
    v->id = (int64_t)verts_.size();
    verts_.push_back(v);
    built_ = false;
    return v;
  }

  // Loads a flat tessellation (tet_v / tet_n as in include/dtfe_gpu.h, -1 on
  // the hull) over points xyz (3 per vertex).  Returns the vertex handles.
  const std::vector<Vertex*>& load_flat(int64_t nv, const float* xyz, int64_t nt, const int32_t* tv,
                                        const int32_t* tn) {
    clear();
    for (int64_t i = 0; i < nv; ++i) {
      Vertex* v = new Vertex();
      v->p = Point(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
      v->id = i;
      verts_.push_back(v);
    }
    link(nt, tv, tn);
    return verts_;
  }

  size_t number_of_vertices() { ensure(); return finite_verts_.size(); }
  size_t number_of_finite_cells() { ensure(); return finite_cells_.size(); }
  bool is_infinite(Cell_handle c) const { return c->infinite; }
  bool is_infinite(Vertex_handle v) const { return v->infinite; }

  Finite_vertices_iterator finite_vertices_begin() { ensure(); return Finite_vertices_iterator(finite_verts_.data()); }
  Finite_vertices_iterator finite_vertices_end() {
    ensure();
    return Finite_vertices_iterator(finite_verts_.data() + finite_verts_.size());
  }
  Finite_cells_iterator finite_cells_begin() { ensure(); return Finite_cells_iterator(finite_cells_.data()); }
  Finite_cells_iterator finite_cells_end() {
    ensure();
    return Finite_cells_iterator(finite_cells_.data() + finite_cells_.size());
  }

  template <class OutIt>
  OutIt incident_cells(Vertex_handle v, OutIt out) {
    ensure();
    for (Cell* c : incident_[v->id]) *out++ = c;
    return out;
  }

  Tetrahedron tetrahedron(Cell_handle c) const {
    Tetrahedron t;
    for (int a = 0; a < 4; ++a) t.q[a] = c->v[a]->p;
    return t;
  }

  Cell_handle locate(const Point& p, Locate_type& lt, int& li, int& lj, Cell_handle hint = Cell_handle()) {
    ensure();
    li = lj = 0;
    if (finite_cells_.empty()) {
      lt = OUTSIDE_AFFINE_HULL;
      return Cell_handle();
    }
    Cell* h = hint;
    Cell* t = (h && !h->infinite) ? h : (h && h->infinite ? h->n[0] : finite_cells_[0]);
    int zmask = 0;  // faces of the final cell through p
    for (size_t step = 0; step < 4 * finite_cells_.size() + 64; ++step) {
      int exit = -1;
      zmask = 0;
      for (int i = 0; i < 4 && exit < 0; ++i) {
        const int s = face_sign(t, i, p);
        if (s < 0) exit = i;
        else if (s == 0) zmask |= 1 << i;
      }
      if (exit < 0) break;
      Cell* nb = t->n[exit];
      if (nb->infinite) {
        lt = OUTSIDE_CONVEX_HULL;
        return nb;
      }
      t = nb;
    }
    lt = CELL;
    // p strictly inside: no other cell's closure holds it
    if (zmask == 0) return t;
    // canonical tie rule: lowest id among the finite cells whose closure
    // holds p (they share the face, edge or vertex through p), searched
    // across the faces through p
    Cell* best = t;
    constexpr int kSeen = 256;
    Cell* seen[kSeen];
    Cell* queue[kSeen];
    int n_seen = 1, n_queue = 1;
    seen[0] = queue[0] = t;
    while (n_queue > 0) {
      Cell* u = queue[--n_queue];
      for (int i = 0; i < 4; ++i) {
        if (face_sign(u, i, p) != 0) continue;
        Cell* nb = u->n[i];
        if (nb->infinite || std::find(seen, seen + n_seen, nb) != seen + n_seen) continue;
        if (n_seen == kSeen) return best;  // more cells around p than any vertex star holds here
        seen[n_seen++] = nb;
        bool inside = true;
        for (int k = 0; k < 4 && inside; ++k) inside = face_sign(nb, k, p) >= 0;
        if (!inside) continue;
        queue[n_queue++] = nb;
        if (nb->id < best->id) best = nb;
      }
    }
    return best;
  }
  Cell_handle locate(const Point& p, Locate_type& lt, int& li, Cell_handle hint = Cell_handle()) {
    int lj;
    return locate(p, lt, li, lj, hint);
  }

  int64_t cell_index(Cell_handle c) const { return c->infinite ? -1 : c->id; }

 private:
  std::vector<Vertex*> verts_, finite_verts_;
  std::vector<Cell*> cells_, finite_cells_;
  std::vector<std::vector<Cell*>> incident_;
  Vertex inf_vertex_;
  bool built_ = false;

  int face_sign(const Cell* t, int i, const Point& p) const {
    const double* q[4];
    for (int a = 0; a < 4; ++a) q[a] = (a == i) ? p.c : t->v[a]->p.c;
    return dtfe::orient(q[0], q[1], q[2], q[3]);
  }

  void ensure() {
    if (built_) return;
    // tessellate the inserted points with the project's exact tessellator,
    // numbered in the planner's Z-order (CGAL's own cell vertex order is
    // internal to it): the cells, their vertex order and ids are then those
    // of the planner's sub-box for the same points
    std::vector<double> pts(3 * verts_.size());
    for (size_t i = 0; i < verts_.size(); ++i)
      for (int k = 0; k < 3; ++k) pts[3 * i + k] = verts_[i]->p.c[k];
    const std::vector<int64_t> order = dtfe::morton_order(pts.data(), (int64_t)verts_.size());
    std::vector<double> xyz(3 * verts_.size());
    for (size_t r = 0; r < order.size(); ++r)
      for (int k = 0; k < 3; ++k) xyz[3 * r + k] = pts[3 * order[r] + k];
    void* h = nullptr;
    dtfe_tessellate(xyz.data(), (int64_t)verts_.size(), 12345, 1, &h);
    int64_t nt = 0, np = 0, nd = 0;
    dtfe_tess_sizes(h, &nt, &np, &nd);
    std::vector<int32_t> tv(4 * nt), tn(4 * nt), vm(np);
    dtfe_tess_export(h, tv.data(), tn.data(), vm.data());
    dtfe_tess_release(h);
    for (auto& q : tv) q = (int32_t)order[q];  // rank -> inserted vertex
    link(nt, tv.data(), tn.data());
  }

  void link(int64_t nt, const int32_t* tv, const int32_t* tn) {
    for (Cell* c : cells_) delete c;
    cells_.clear();
    finite_cells_.clear();
    for (int64_t t = 0; t < nt; ++t) {
      Cell* c = new Cell();
      c->id = t;
      for (int a = 0; a < 4; ++a) c->v[a] = verts_[tv[4 * t + a]];
      cells_.push_back(c);
      finite_cells_.push_back(c);
    }
    // one infinite cell per hull face, infinite vertex at index 0
    std::map<std::pair<int64_t, int64_t>, std::vector<std::pair<Cell*, int>>> hull_edges;
    for (int64_t t = 0; t < nt; ++t)
      for (int k = 0; k < 4; ++k) {
        int32_t nb = tn[4 * t + k];
        if (nb >= 0) {
          cells_[t]->n[k] = cells_[nb];
          continue;
        }
        Cell* ic = new Cell();
        ic->infinite = true;
        ic->id = (int64_t)cells_.size();
        ic->v[0] = &inf_vertex_;
        int m = 1;
        for (int a = 0; a < 4; ++a)
          if (a != k) ic->v[m++] = cells_[t]->v[a];
        ic->n[0] = cells_[t];
        cells_[t]->n[k] = ic;
        cells_.push_back(ic);
        for (int a = 1; a < 4; ++a) {
          int64_t e0 = ic->v[1 + (a % 3)]->id, e1 = ic->v[1 + ((a + 1) % 3)]->id;
          hull_edges[{std::min(e0, e1), std::max(e0, e1)}].push_back({ic, a});
        }
      }
    for (auto& kv : hull_edges)
      if (kv.second.size() == 2) {
        kv.second[0].first->n[kv.second[0].second] = kv.second[1].first;
        kv.second[1].first->n[kv.second[1].second] = kv.second[0].first;
      }
    incident_.assign(verts_.size(), {});
    for (Cell* c : cells_)
      for (int a = 0; a < 4; ++a)
        if (!c->v[a]->infinite) incident_[c->v[a]->id].push_back(c);
    finite_verts_.clear();
    for (Vertex* v : verts_)
      if (!incident_[v->id].empty()) finite_verts_.push_back(v);
    built_ = true;
  }
};

}  // namespace CGAL
