// Whole-run planning in C++ (include/dtfe_host.h, dtfe_plan_build): the
// steps the reference's DTFE() and DTFE_parallel() take before interpolating
// (src/DTFE.cpp:76-251, 287-385), for callers without Python — the DTFE()
// drop-in in particular.  Same arithmetic and ordering as dtfe_b200/plan.py
// (make_plan, make_deposit_plan), so both produce identical plans:
//   padding (updatePadding, given lengths included), average density,
//   --region and --partition / --partNo chunks, periodic images of the
//   padded box (findParticlesInBox), parallelGrid + optimalPartitionSplit into
//   sub-boxes, each sub-box's particles of its padded region, vertices in
//   Morton order, tessellation of every sub-box in parallel, concatenation
//   with global ids, per-sub-box coordinate tables (the x += dx raster).

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <memory>
#include <new>
#include <numeric>
#include <vector>

#include "../../include/dtfe_host.h"
#include "morton.h"

struct dtfe_plan_s {
  dtfe_plan_view view{};
  std::vector<int32_t> tet_v, tet_n, src;
  std::vector<float> xyz, weight, velocity, scalar, xs, ys, zs;
  std::vector<dtfe_subbox> boxes;
  std::vector<float> regions;  // 6 per sub-box: the tile region (xmin, xmax, ymin, ymax, zmin, zmax)
  std::vector<float> dep_pos, dep_weight, dep_velocity;
  std::vector<int64_t> dep_src;
  std::vector<dtfe_deposit_box> dep_boxes;
};

namespace {

struct PointSet {
  std::vector<int32_t> src;
  std::vector<float> pos;  // 3 per point
};

struct Tile {
  int64_t origin[3], dims[3];
  float region[6];
  int part_no;
};

PointSet select(const float* pos, int64_t n, const float box[6], const float padded[6], int periodic) {
  PointSet s;
  const int64_t m = dtfe_select_in_box(pos, n, box, padded, periodic, nullptr, nullptr);
  s.src.resize(m);
  s.pos.resize(3 * m);
  dtfe_select_in_box(pos, n, box, padded, periodic, s.src.data(), s.pos.data());
  return s;
}

// DTFE_parallel (src/DTFE.cpp:287-385) on one region's particles `all`:
// parallelGrid(n_parts) sub-boxes of the region's grid, balanced by
// optimalPartitionSplit, each with the particles of its padded sub-box
// (non-periodic, findParticlesInBox); the tiles are placed at `origin` in the
// output grid.  A single part interpolates the region directly with every
// particle (the one-thread branch, :300-305), under `single_part_no`.
int parallel_split(PointSet all, const int64_t grid[3], const float region[6], const int64_t origin[3],
                   int32_t n_parts, const float pad[6], int single_part_no, std::vector<PointSet>& sets,
                   std::vector<Tile>& tiles) {
  int64_t pg[3];
  dtfe_parallel_grid(n_parts, grid, pg);
  const int64_t np = pg[0] * pg[1] * pg[2];
  if (np == 1) {
    Tile t;
    for (int a = 0; a < 3; ++a) {
      t.origin[a] = origin[a];
      t.dims[a] = grid[a];
    }
    std::memcpy(t.region, region, sizeof(t.region));
    t.part_no = single_part_no;
    sets.push_back(std::move(all));
    tiles.push_back(t);
    return 0;
  }
  std::vector<int64_t> sub(6 * np);
  std::vector<float> coords(6 * np);
  const int64_t nall = (int64_t)all.src.size();
  if (dtfe_optimal_partition(all.pos.data(), nall, grid, region, pg, sub.data(), coords.data())) return 1;
  for (int64_t k = 0; k < np; ++k) {
    const float* r = &coords[6 * k];
    const float pb[6] = {r[0] - pad[0], r[1] + pad[1], r[2] - pad[2], r[3] + pad[3], r[4] - pad[4], r[5] + pad[5]};
    PointSet part = select(all.pos.data(), nall, r, pb, 0);
    for (auto& i : part.src) i = all.src[i];
    Tile t;
    for (int a = 0; a < 3; ++a) {
      t.origin[a] = origin[a] + sub[6 * k + 2 * a];
      t.dims[a] = sub[6 * k + 2 * a + 1] - sub[6 * k + 2 * a];
    }
    std::memcpy(t.region, r, sizeof(t.region));
    t.part_no = (int)k;  // DTFE_parallel's tempOptions.partNo = thread number
    sets.push_back(std::move(part));
    tiles.push_back(t);
  }
  return 0;
}

// findParticlesInBox of a subset: the particles of `from` in `padded`, with
// their input ids.
PointSet select_from(const PointSet& from, const float full_box[6], const float padded[6], int periodic) {
  PointSet s = select(from.pos.data(), (int64_t)from.src.size(), full_box, padded, periodic);
  for (auto& i : s.src) i = from.src[i];
  return s;
}

// The steps of DTFE() from its option checks to its DTFE_parallel calls
// (src/DTFE.cpp:76-251): --region selects the particles of the padded region
// (periodic images on the full box) and makes the region the full box,
// non-periodic; --partition splits the region with optimalPartitionSplit
// into chunks, each selecting the particles of its padded chunk, and runs
// DTFE_parallel on every chunk into its place in the main grid, or, with
// --partNo, on that one chunk into a grid of the chunk's size; otherwise the
// padded box (with periodic images) feeds one DTFE_parallel over the region.
// grid_out / region_out: the grid and region the results cover.
int flow(const float* pos, int64_t n, const float box[6], int periodic, const int32_t grid[3],
         const dtfe_plan_options& o, const float pad[6], std::vector<PointSet>& sets, std::vector<Tile>& tiles,
         int32_t grid_out[3], float region_out[6]) {
  const int64_t g64[3] = {grid[0], grid[1], grid[2]};
  const int64_t zero[3] = {0, 0, 0};
  float full[6];
  std::memcpy(full, box, sizeof(full));
  int per = periodic;
  PointSet cur;
  cur.src.resize(n);
  std::iota(cur.src.begin(), cur.src.end(), 0);
  cur.pos.assign(pos, pos + 3 * n);
  float region[6];
  std::memcpy(region, box, sizeof(region));
  if (o.region_on) {
    std::memcpy(region, o.region, sizeof(region));
    // Box::validSubBox (src/box.h:115-138)
    for (int a = 0; a < 3; ++a) {
      const float lo = box[2 * a], hi = box[2 * a + 1];
      const bool bad = per ? (region[2 * a] < 2 * lo - hi || region[2 * a + 1] > 2 * hi - lo)
                           : (region[2 * a] < lo || region[2 * a + 1] > hi);
      if (bad) return 4;
    }
    const float padded[6] = {region[0] - pad[0], region[1] + pad[1], region[2] - pad[2],
                             region[3] + pad[3], region[4] - pad[4], region[5] + pad[5]};
    cur = select_from(cur, full, padded, per);
    per = 0;
    std::memcpy(full, region, sizeof(full));
  }
  for (int a = 0; a < 3; ++a) grid_out[a] = grid[a];
  std::memcpy(region_out, region, sizeof(region));
  if (o.partition_on) {
    const int64_t parts[3] = {o.partition[0], o.partition[1], o.partition[2]};
    const int64_t np = parts[0] * parts[1] * parts[2];
    if (parts[0] < 1 || parts[1] < 1 || parts[2] < 1 || o.part_no >= np) return 1;
    std::vector<int64_t> sub(6 * np);
    std::vector<float> coords(6 * np);
    if (dtfe_optimal_partition(cur.pos.data(), (int64_t)cur.src.size(), g64, region, parts, sub.data(),
                               coords.data()))
      return 1;
    const int64_t first = o.part_no >= 0 ? o.part_no : 0, last = o.part_no >= 0 ? o.part_no + 1 : np;
    for (int64_t k = first; k < last; ++k) {
      const float* r = &coords[6 * k];
      const float padded[6] = {r[0] - pad[0], r[1] + pad[1], r[2] - pad[2], r[3] + pad[3], r[4] - pad[4],
                               r[5] + pad[5]};
      const int64_t dims[3] = {sub[6 * k + 1] - sub[6 * k], sub[6 * k + 3] - sub[6 * k + 2],
                               sub[6 * k + 5] - sub[6 * k + 4]};
      const int64_t at[3] = {sub[6 * k], sub[6 * k + 2], sub[6 * k + 4]};
      if (parallel_split(select_from(cur, full, padded, per), dims, r, o.part_no >= 0 ? zero : at, o.n_parts, pad,
                         (int)k, sets, tiles))
        return 1;
      if (o.part_no >= 0) {
        for (int a = 0; a < 3; ++a) grid_out[a] = (int32_t)dims[a];
        std::memcpy(region_out, r, sizeof(float) * 6);
      }
    }
    return 0;
  }
  if (!o.region_on && per) {
    const float padded[6] = {box[0] - pad[0], box[1] + pad[1], box[2] - pad[2],
                             box[3] + pad[3], box[4] - pad[4], box[5] + pad[5]};
    cur = select_from(cur, box, padded, 1);
  }
  return parallel_split(std::move(cur), g64, region, zero, o.n_parts, pad, -1, sets, tiles);
}

template <class T>
void gather(const T* in, int width, const std::vector<int32_t>& src, std::vector<T>& out) {
  out.resize(src.size() * width);
  for (size_t i = 0; i < src.size(); ++i)
    for (int c = 0; c < width; ++c) out[i * width + c] = in[(int64_t)src[i] * width + c];
}

int assemble(dtfe_plan_s& P, std::vector<PointSet>& sets, const std::vector<Tile>& tiles, const float* w,
             const float* vel, const float* scal, int32_t S) {
  const int k = (int)sets.size();
  for (auto& s : sets) {
    const std::vector<int64_t> o = dtfe::morton_order(s.pos.data(), (int64_t)s.pos.size() / 3);
    PointSet t;
    t.src.resize(o.size());
    t.pos.resize(3 * o.size());
    for (size_t i = 0; i < o.size(); ++i) {
      t.src[i] = s.src[o[i]];
      for (int c = 0; c < 3; ++c) t.pos[3 * i + c] = s.pos[3 * o[i] + c];
    }
    s = std::move(t);
  }
  std::vector<std::vector<double>> xyz64(k);
  std::vector<const double*> ptrs(k);
  std::vector<int64_t> ns(k);
  for (int i = 0; i < k; ++i) {
    xyz64[i].assign(sets[i].pos.begin(), sets[i].pos.end());
    ptrs[i] = xyz64[i].data();
    ns[i] = (int64_t)sets[i].src.size();
  }
  std::vector<void*> handles(k, nullptr);
  std::vector<int> rc(k, 0);
  dtfe_tessellate_batch(k, ptrs.data(), ns.data(), 12345, 1, handles.data(), rc.data());
  int64_t voff = 0, toff = 0, coff[3] = {0, 0, 0};
  int status = 0;
  P.boxes.resize(k);
  P.regions.resize(6 * k);
  for (int i = 0; i < k; ++i) {
    int64_t nt = 0, npt = 0, nd = 0;
    if (handles[i]) dtfe_tess_sizes(handles[i], &nt, &npt, &nd);
    std::vector<int32_t> tv(4 * nt), tn(4 * nt), vm(npt);
    if (handles[i]) {
      dtfe_tess_export(handles[i], tv.data(), tn.data(), vm.data());
      dtfe_tess_release(handles[i]);
    }
    if (rc[i] != 0 && rc[i] != 1) status = 2;
    const int64_t nv = ns[i];
    for (int64_t q = 0; q < 4 * nt; ++q) {
      P.tet_v.push_back((int32_t)(tv[q] + voff));
      P.tet_n.push_back(tn[q] >= 0 ? (int32_t)(tn[q] + toff) : -1);
    }
    P.xyz.insert(P.xyz.end(), sets[i].pos.begin(), sets[i].pos.end());
    P.src.insert(P.src.end(), sets[i].src.begin(), sets[i].src.end());
    const Tile& t = tiles[i];
    std::memcpy(&P.regions[6 * i], t.region, sizeof(t.region));
    dtfe_subbox& b = P.boxes[i];
    std::memset(&b, 0, sizeof(b));
    b.vert_offset = voff;
    b.n_verts = nv;
    b.tet_offset = toff;
    b.n_tets = nt;
    for (int a = 0; a < 3; ++a) {
      const float length = t.region[2 * a + 1] - t.region[2 * a];
      const float dx = length / (float)t.dims[a];
      b.tile_origin[a] = (int32_t)t.origin[a];
      b.tile_dims[a] = (int32_t)t.dims[a];
      b.coord_offset[a] = coff[a];
      b.dx[a] = dx;
      b.lo[a] = t.region[2 * a];
      std::vector<float>& table = a == 0 ? P.xs : (a == 1 ? P.ys : P.zs);
      const size_t at = table.size();
      table.resize(at + t.dims[a]);
      dtfe_axis_coords(t.region[2 * a], dx, t.dims[a], table.data() + at);
    }
    b.part_no = t.part_no;
    for (int a = 0; a < 3; ++a) coff[a] += t.dims[a];
    voff += nv;
    toff += nt;
  }
  std::vector<float> ones;
  if (!w) {
    int64_t mx = 0;
    for (int32_t s : P.src) mx = std::max<int64_t>(mx, s + 1);
    ones.assign(mx, 1.f);
    w = ones.data();
  }
  gather(w, 1, P.src, P.weight);
  if (vel) gather(vel, 3, P.src, P.velocity);
  if (scal && S > 0) gather(scal, S, P.src, P.scalar);
  return status;
}

void deposit_assemble(dtfe_plan_s& P, std::vector<PointSet>& sets, const std::vector<Tile>& tiles, const float* w,
                      const float* vel) {
  int64_t off = 0;
  P.dep_boxes.resize(sets.size());
  for (size_t k = 0; k < sets.size(); ++k) {
    const std::vector<int64_t> o = dtfe::morton_order(sets[k].pos.data(), (int64_t)sets[k].pos.size() / 3);
    for (int64_t i : o) {
      for (int c = 0; c < 3; ++c) P.dep_pos.push_back(sets[k].pos[3 * i + c]);
      P.dep_src.push_back(sets[k].src[i]);
    }
    dtfe_deposit_box& b = P.dep_boxes[k];
    std::memset(&b, 0, sizeof(b));
    b.particle_offset = off;
    b.n_particles = (int64_t)o.size();
    std::memcpy(b.region, tiles[k].region, sizeof(b.region));
    for (int a = 0; a < 3; ++a) {
      b.tile_origin[a] = (int32_t)tiles[k].origin[a];
      b.tile_dims[a] = (int32_t)tiles[k].dims[a];
    }
    off += (int64_t)o.size();
  }
  P.dep_weight.resize(P.dep_src.size());
  for (size_t i = 0; i < P.dep_src.size(); ++i) P.dep_weight[i] = w ? w[P.dep_src[i]] : 1.f;
  if (vel) {
    P.dep_velocity.resize(3 * P.dep_src.size());
    for (size_t i = 0; i < P.dep_src.size(); ++i)
      for (int c = 0; c < 3; ++c) P.dep_velocity[3 * i + c] = vel[3 * P.dep_src[i] + c];
  }
}

}  // namespace

extern "C" {

int dtfe_plan_build_ex(int kind, const float* pos, const float* w, const float* vel, const float* scal, int32_t S,
                       int64_t n, const float box[6], int periodic, const int32_t grid[3],
                       const dtfe_plan_options* opts, dtfe_plan* out) {
  if (!out || !box || !grid || !opts || (n > 0 && !pos) || opts->n_parts < 1 || kind < 0 || kind > 3) return 1;
  *out = nullptr;
  const dtfe_plan_options& o = *opts;
  if (o.padding_mode < DTFE_PAD_PARTICLES || o.padding_mode > DTFE_PAD_ABSOLUTE) return 1;
  std::unique_ptr<dtfe_plan_s> P(new (std::nothrow) dtfe_plan_s());
  if (!P) return 3;
  const int64_t g64[3] = {grid[0], grid[1], grid[2]};
  const float blen[3] = {box[1] - box[0], box[3] - box[2], box[5] - box[4]};
  // User_options::updatePadding (src/user_options.cc:1062-1089): six given
  // lengths unless all are zero (isNullBox), in box lengths or absolute;
  // else the particle count's padding for the estimator (DTFE/SPH 0,
  // TSC/NGP 1, CIC 2)
  float pad[6];
  bool given = false;
  for (int i = 0; i < 6; ++i) given = given || (o.padding_mode != DTFE_PAD_PARTICLES && o.padding[i] != 0.f);
  if (given) {
    for (int i = 0; i < 6; ++i)
      pad[i] = o.padding_mode == DTFE_PAD_RELATIVE ? o.padding[i] * blen[i % 2] : o.padding[i];
  } else {
    const int pad_kind = kind == DTFE_PLAN_DTFE ? 0 : (kind == DTFE_PLAN_CIC ? 2 : 1);
    dtfe_padding_length(pad_kind, o.padding_particles, n, blen, g64, pad);
  }
  const double rho_bar =
      o.average_density > 0.0 ? (double)(float)o.average_density : (double)dtfe_average_density(w, n);
  std::vector<PointSet> sets;
  std::vector<Tile> tiles;
  int32_t grid_out[3];
  float region_out[6];
  if (int frc = flow(pos, n, box, periodic, grid, o, pad, sets, tiles, grid_out, region_out)) return frc;
  int rc = 0;
  if (kind == DTFE_PLAN_DTFE) rc = assemble(*P, sets, tiles, w, vel, scal, S);
  else deposit_assemble(*P, sets, tiles, w, vel);
  if (rc) return rc;
  dtfe_plan_view& v = P->view;
  v.kind = kind;
  for (int a = 0; a < 3; ++a) v.grid[a] = grid_out[a];
  std::memcpy(v.region, region_out, sizeof(region_out));
  v.rho_bar = rho_bar;
  std::memcpy(v.padding, pad, sizeof(pad));
  v.n_verts = (int64_t)P->src.size();
  v.n_tets = (int64_t)P->tet_v.size() / 4;
  v.n_boxes = (int32_t)P->boxes.size();
  v.n_scalars = P->scalar.empty() ? 0 : S;
  v.tet_v = P->tet_v.data();
  v.tet_n = P->tet_n.data();
  v.xyz = P->xyz.data();
  v.src = P->src.data();
  v.weight = P->weight.data();
  v.velocity = P->velocity.empty() ? nullptr : P->velocity.data();
  v.scalar = P->scalar.empty() ? nullptr : P->scalar.data();
  v.boxes = P->boxes.data();
  v.regions = P->regions.empty() ? nullptr : P->regions.data();
  v.xs = P->xs.data();
  v.ys = P->ys.data();
  v.zs = P->zs.data();
  v.n_xs = (int64_t)P->xs.size();
  v.n_ys = (int64_t)P->ys.size();
  v.n_zs = (int64_t)P->zs.size();
  v.n_particles = (int64_t)P->dep_src.size();
  v.dep_pos = P->dep_pos.data();
  v.dep_weight = P->dep_weight.data();
  v.dep_velocity = P->dep_velocity.empty() ? nullptr : P->dep_velocity.data();
  v.dep_src = P->dep_src.data();
  v.n_dep_boxes = (int32_t)P->dep_boxes.size();
  v.dep_boxes = P->dep_boxes.data();
  *out = P.release();
  return 0;
}

int dtfe_plan_build(int kind, const float* pos, const float* w, const float* vel, const float* scal, int32_t S,
                    int64_t n, const float box[6], int periodic, const int32_t grid[3], int32_t n_parts,
                    float padding_particles, double average_density, dtfe_plan* out) {
  dtfe_plan_options o;
  std::memset(&o, 0, sizeof(o));
  o.n_parts = n_parts;
  o.padding_mode = DTFE_PAD_PARTICLES;
  o.padding_particles = padding_particles;
  o.part_no = -1;
  o.average_density = average_density;
  return dtfe_plan_build_ex(kind, pos, w, vel, scal, S, n, box, periodic, grid, &o, out);
}

int dtfe_plan_get(dtfe_plan p, dtfe_plan_view* view) {
  if (!p || !view) return 1;
  *view = p->view;
  return 0;
}

void dtfe_plan_release(dtfe_plan p) { delete p; }

}  // extern "C"
