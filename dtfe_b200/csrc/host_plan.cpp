// Host-side planning of a DTFE run: the control flow DTFE() executes before
// the tessellation is built.  Each function restates one reference routine
// with the same float arithmetic, so sub-box regions, padded particle sets and
// sample coordinates come out bit-identical.
//
//   dtfe_padding_length     User_options::updatePadding   src/user_options.cc:1062-1089
//   dtfe_average_density    averageDensity                src/subpartition.h:437-449
//                           (Box::volume() is hard-coded to 35000^3, src/box.h:142-149)
//   dtfe_select_in_box      findParticlesInBox / insertParticlesInBox
//                                                         src/subpartition.h:79-154
//   dtfe_parallel_grid      parallelGrid                  src/subpartition.h:454-555
//   dtfe_optimal_partition  optimalPartitionSplit + optimalSplit + NGP_particle_count
//                           src/subpartition.h:163-372, src/NGP_interpolation.cc:140-174
//   dtfe_axis_coords        the x += dx sample raster     unaveraged_interpolation.cc:252-358

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

// Padding length on each of the 6 box sides (xmin, xmax, ymin, ...).
// kind: 0 = DTFE or SPH, 1 = TSC or NGP, 2 = CIC.  The reference indexes the
// box lengths with i%2 rather than i/2 (so side 4 uses the x length); that is
// kept.  A non-null user padding (already in box units) is returned as is.
void dtfe_padding_length(int kind, float padding_particles, int64_t n_total,
                         const float full_box_length[3], const int64_t grid[3], float out[6]) {
  if (padding_particles <= 0.f) {
    for (int i = 0; i < 6; ++i) out[i] = 0.f;
    return;
  }
  for (int i = 0; i < 6; ++i) {
    if (kind == 0)
      out[i] = padding_particles / (float)(std::pow((double)n_total, 1. / 3)) * full_box_length[i % 2];
    else if (kind == 1)
      out[i] = full_box_length[i % 2] / (float)grid[i % 2];
    else
      out[i] = 0.f;
  }
}

// Sum of weights (double) over the hard-coded box volume, as a float.
float dtfe_average_density(const float* w, int64_t n) {
  double total = 0.;
  for (int64_t i = 0; i < n; ++i) total += w ? (double)w[i] : 1.0;
  float vol = 1.f;
  for (int i = 0; i < 3; ++i) vol *= 35000;
  return (float)(total / vol);
}

static inline bool in_box(const float* p, const float* b) {
  return p[0] >= b[0] && p[0] <= b[1] && p[1] >= b[2] && p[1] <= b[3] && p[2] >= b[4] && p[2] <= b[5];
}

// Particles inside the padded box.  Non-periodic: particles with
// padded[lo] <= pos <= padded[hi].  Periodic: for each of the 27 box
// translations (order i1,i2,i3 over {-1,0,1} times the full box length) the
// translated padded box selects particles, which are emitted shifted back by
// the translation — the reference's order and float arithmetic.  Returns the
// number selected; idx/pos_out (may be NULL for a count) receive the source
// index and the (shifted) position of each.
int64_t dtfe_select_in_box(const float* pos, int64_t n, const float full_box[6], const float padded[6],
                           int periodic, int32_t* idx_out, float* pos_out) {
  struct Off { float o[3]; float box[6]; };
  std::vector<Off> offs;
  if (!periodic) {
    Off o{{0.f, 0.f, 0.f}, {padded[0], padded[1], padded[2], padded[3], padded[4], padded[5]}};
    offs.push_back(o);
  } else {
    float len[3];
    for (int i = 0; i < 3; ++i) len[i] = full_box[2 * i + 1] - full_box[2 * i];
    for (int i1 = 0; i1 < 3; ++i1)
      for (int i2 = 0; i2 < 3; ++i2)
        for (int i3 = 0; i3 < 3; ++i3) {
          Off o;
          o.o[0] = (float)(i1 - 1) * len[0];
          o.o[1] = (float)(i2 - 1) * len[1];
          o.o[2] = (float)(i3 - 1) * len[2];
          for (int k = 0; k < 3; ++k) {
            o.box[2 * k] = padded[2 * k] + o.o[k];
            o.box[2 * k + 1] = padded[2 * k + 1] + o.o[k];
          }
          offs.push_back(o);
        }
  }
  // parallel two-pass selection preserving the serial order
  const int64_t chunk = 1 << 16;
  const int64_t nchunks = (n + chunk - 1) / chunk;
  const int64_t nblk = (int64_t)offs.size() * nchunks;
  std::vector<int64_t> count(nblk + 1, 0);
#pragma omp parallel for schedule(static)
  for (int64_t b = 0; b < nblk; ++b) {
    const Off& o = offs[b / nchunks];
    int64_t lo = (b % nchunks) * chunk, hi = std::min<int64_t>(n, lo + chunk);
    int64_t c = 0;
    for (int64_t i = lo; i < hi; ++i) c += in_box(&pos[3 * i], o.box);
    count[b + 1] = c;
  }
  for (int64_t b = 0; b < nblk; ++b) count[b + 1] += count[b];
  if (idx_out || pos_out) {
#pragma omp parallel for schedule(static)
    for (int64_t b = 0; b < nblk; ++b) {
      const Off& o = offs[b / nchunks];
      int64_t lo = (b % nchunks) * chunk, hi = std::min<int64_t>(n, lo + chunk);
      int64_t k = count[b];
      for (int64_t i = lo; i < hi; ++i) {
        const float* p = &pos[3 * i];
        if (!in_box(p, o.box)) continue;
        if (idx_out) idx_out[k] = (int32_t)i;
        if (pos_out) {
          pos_out[3 * k] = p[0] - o.o[0];
          pos_out[3 * k + 1] = p[1] - o.o[1];
          pos_out[3 * k + 2] = p[2] - o.o[2];
        }
        ++k;
      }
    }
  }
  return count[nblk];
}

// parallelGrid: a 2^a 3^b processor grid close to n_threads, balanced over
// the axes and no finer than the main grid.
void dtfe_parallel_grid(int64_t n_threads, const int64_t main_grid[3], int64_t grid[3]) {
  const int D = 3;
  int64_t n = n_threads;
  int x2 = 0, x3 = 0;
  while (n / 2 != 0) { n /= 2; ++x2; }
  n = n_threads;
  while (n / 3 != 0) { n /= 3; ++x3; }
  n = n_threads;
  int64_t diff = n;
  int j2 = 0, j3 = 0;
  int64_t napprox = 1;
  for (int i2 = 0; i2 <= x2; ++i2) {
    int64_t temp = napprox;
    for (int i3 = 0; i3 <= x3; ++i3) {
      // (n-temp) is unsigned in the reference: only temp <= n qualifies
      if (temp <= n && (n - temp) < diff) {
        diff = n - temp;
        j2 = i2;
        j3 = i3;
      }
      temp *= 3;
    }
    napprox *= 2;
  }
  x2 = j2;
  x3 = j3;
  for (int i = 0; i < D; ++i) grid[i] = 1;
  while (x3 - D >= 0) {
    for (int i = 0; i < D; ++i) grid[i] *= 3;
    x3 -= D;
  }
  for (int i = D - 1; i >= (D - x3); --i) grid[i] *= 3;
  int i1 = x2 > (D - x3) ? (D - x3) : x2;
  for (int i = 0; i < i1; ++i) grid[i % (D - x3)] *= 2;
  for (int i = 0; i < x2 - i1; ++i) grid[i % D] *= 2;
  for (int i = 0; i < D; ++i) {
    if (main_grid[i] >= grid[i]) continue;
    int next1 = (i + 1) % D, next2 = (i + 2) % D;
    while (grid[i] > main_grid[i] && grid[i] % 3 == 0) {
      grid[i] /= 3;
      if (3 * grid[next1] <= main_grid[next1]) grid[next1] *= 3;
      else if (3 * grid[next2] <= main_grid[next2]) grid[next2] *= 3;
    }
    while (grid[i] > main_grid[i] && grid[i] % 2 == 0) {
      grid[i] /= 2;
      if (2 * grid[next1] <= main_grid[next1]) grid[next1] *= 2;
      else if (2 * grid[next2] <= main_grid[next2]) grid[next2] *= 2;
    }
  }
}

// optimalSplit: indices splitting `counts` into `parts` runs of similar sums.
static void optimal_split(const std::vector<size_t>& counts, size_t parts, size_t* idx) {
  if (parts <= 1 || counts.size() == 1) return;
  size_t total = 0;
  for (size_t c : counts) total += c;
  size_t load = total / parts;
  size_t remaining = total, temp = 0, pic = 1;
  idx[0] = 0;
  idx[parts] = counts.size();
  for (size_t i = 0; i < counts.size(); ++i) {
    temp += counts[i];
    if (temp >= load) {
      size_t t1 = ((remaining + counts[i]) - temp) / (parts - pic);
      size_t t2 = (remaining - temp) / (parts - pic);
      if (i == 0) {
      } else if (i == counts.size() - 1) {
        temp -= counts[i];
        --i;
      } else if (pic > 1 && (i - idx[pic - 1]) == 1) {
      } else if (std::abs((int)temp - (int)t1) < std::abs((int)temp - (int)t2)) {
        temp -= counts[i];
        --i;
      }
      idx[pic] = i;
      remaining -= temp;
      load = remaining / (parts - pic);
      temp = 0;
      ++pic;
      if (pic == parts) break;
    }
  }
}

// optimalPartitionSplit over the main grid of `region` (6 floats): splits
// along x, then y inside each x slab, then z, balancing NGP particle counts.
// subgrid (6 per partition): [x0,x1,y0,y1,z0,z1) cell ranges; coords (6 per
// partition): region bounds region[lo] + dx * index (float).  Partition p has
// index (px*part[1] + py)*part[2] + pz.  Returns 0, or 1 when a partition
// count exceeds the grid.
int dtfe_optimal_partition(const float* pos, int64_t n, const int64_t grid_in[3], const float region[6],
                           const int64_t part_in[3], int64_t* subgrid, float* coords) {
  const size_t grid[3] = {(size_t)grid_in[0], (size_t)grid_in[1], (size_t)grid_in[2]};
  const size_t part[3] = {(size_t)part_in[0], (size_t)part_in[1], (size_t)part_in[2]};
  for (int i = 0; i < 3; ++i)
    if (part[i] == 0 || part[i] > grid[i]) return 1;
  float dx[3];
  for (int i = 0; i < 3; ++i) dx[i] = (region[2 * i + 1] - region[2 * i]) / grid[i];
  // NGP_particle_count
  std::vector<int> counts(grid[0] * grid[1] * grid[2], 0);
  for (int64_t p = 0; p < n; ++p) {
    int cell[3];
    bool ok = true;
    for (int j = 0; j < 3; ++j) {
      cell[j] = (int)std::floor((pos[3 * p + j] - region[2 * j]) / dx[j]);
      if (cell[j] < 0 || (size_t)cell[j] >= grid[j]) ok = false;
    }
    if (!ok) continue;
    counts[cell[0] * grid[1] * grid[2] + cell[1] * grid[2] + cell[2]] += 1;
  }
  const size_t np = part[0] * part[1] * part[2];
  std::vector<size_t> xs(part[0] + 1, 0), ys(part[1] + 1, 0), zs(part[2] + 1, 0);
  if (part[0] > 1) {
    std::vector<size_t> tc(grid[0], 0);
    for (size_t i1 = 0; i1 < grid[0]; ++i1)
      for (size_t i2 = 0; i2 < grid[1]; ++i2)
        for (size_t i3 = 0; i3 < grid[2]; ++i3) tc[i1] += counts[i1 * grid[1] * grid[2] + i2 * grid[2] + i3];
    optimal_split(tc, part[0], xs.data());
  } else {
    xs[0] = 0;
    xs[1] = grid[0];
  }
  for (size_t i1 = 0; i1 < part[0]; ++i1)
    for (size_t i2 = 0; i2 < part[1]; ++i2)
      for (size_t i3 = 0; i3 < part[2]; ++i3) {
        size_t p = i1 * part[1] * part[2] + i2 * part[2] + i3;
        subgrid[6 * p + 0] = (int64_t)xs[i1];
        subgrid[6 * p + 1] = (int64_t)xs[i1 + 1];
        coords[6 * p + 0] = region[0] + dx[0] * xs[i1];
        coords[6 * p + 1] = region[0] + dx[0] * xs[i1 + 1];
      }
  for (size_t i = 0; i < part[0]; ++i) {
    if (part[1] > 1) {
      std::vector<size_t> tc(grid[1], 0);
      for (size_t i1 = xs[i]; i1 < xs[i + 1]; ++i1)
        for (size_t i2 = 0; i2 < grid[1]; ++i2)
          for (size_t i3 = 0; i3 < grid[2]; ++i3) tc[i2] += counts[i1 * grid[1] * grid[2] + i2 * grid[2] + i3];
      optimal_split(tc, part[1], ys.data());
    } else {
      ys[0] = 0;
      ys[1] = grid[1];
    }
    for (size_t i2 = 0; i2 < part[1]; ++i2)
      for (size_t i3 = 0; i3 < part[2]; ++i3) {
        size_t p = i * part[1] * part[2] + i2 * part[2] + i3;
        subgrid[6 * p + 2] = (int64_t)ys[i2];
        subgrid[6 * p + 3] = (int64_t)ys[i2 + 1];
        coords[6 * p + 2] = region[2] + dx[1] * ys[i2];
        coords[6 * p + 3] = region[2] + dx[1] * ys[i2 + 1];
      }
  }
  for (size_t i = 0; i < part[0]; ++i)
    for (size_t j = 0; j < part[1]; ++j) {
      // The z balance counts particles over the y range ys[j..j+1] left by the
      // y loop, i.e. the split of the LAST x slab, for every slab (the
      // reference reuses ySplitIndices, src/subpartition.h:334-339).
      size_t y0 = ys[j], y1 = ys[j + 1];
      if (part[2] > 1) {
        std::vector<size_t> tc(grid[2], 0);
        for (size_t i1 = xs[i]; i1 < xs[i + 1]; ++i1)
          for (size_t i2 = y0; i2 < y1; ++i2)
            for (size_t i3 = 0; i3 < grid[2]; ++i3) tc[i3] += counts[i1 * grid[1] * grid[2] + i2 * grid[2] + i3];
        optimal_split(tc, part[2], zs.data());
      } else {
        zs[0] = 0;
        zs[1] = grid[2];
      }
      for (size_t i3 = 0; i3 < part[2]; ++i3) {
        size_t p = i * part[1] * part[2] + j * part[2] + i3;
        subgrid[6 * p + 4] = (int64_t)zs[i3];
        subgrid[6 * p + 5] = (int64_t)zs[i3 + 1];
        coords[6 * p + 4] = region[4] + dx[2] * zs[i3];
        coords[6 * p + 5] = region[4] + dx[2] * zs[i3 + 1];
      }
    }
  (void)np;
  return 0;
}

// Sample coordinates along one axis: x = lo + dx/2 (double, rounded to
// float), then x += dx in float.
void dtfe_axis_coords(float lo, float dx, int64_t n, float* out) {
  float x = (float)((double)lo + (double)dx / 2.);
  for (int64_t i = 0; i < n; ++i) {
    out[i] = x;
    x += dx;
  }
}

}  // extern "C"

// ---- packed tessellation (dtfe_tets_pack / dtfe_tets_unpack) ----------------
// The flat arrays are mostly small differences: with Morton-ordered
// vertices and tetrahedra (and the smallest vertex first in every
// tetrahedron) a tetrahedron's vertices lie close to its first one, its first
// vertex close to the smallest first vertex of its block of 256, and its
// neighbours close to itself.  Every one of a tetrahedron's 8 fields (first
// vertex - block base, three vertex offsets, four neighbour deltas) takes 1
// or 2 bytes, a flag bit per field says which; values that fit neither are
// escaped to a 32-bit list.  About 10-11 bytes per tetrahedron instead of 32.
// Layout:
//   header       10 x int64: magic, T, n_blocks, n_escapes, and the byte
//                offsets of block_base, block_esc, block_off, flags, data, escapes
//   block_base   int32 per block: smallest first vertex of its tetrahedra
//   block_esc    int32 per block + 1: escapes before the block
//   block_off    int64 per block + 1: byte offset of the block in data
//   flags        uint8 per tetrahedron: bit f set = field f takes 2 bytes
//   data         the fields, tetrahedron after tetrahedron, little endian:
//                vertex fields unsigned (all ones: escaped), neighbour
//                fields signed (minimum: no neighbour, maximum: escaped)
//   escapes      int32 values of the escaped fields, in (tetrahedron, field)
//                order
namespace {
constexpr int64_t kPackBlock = 256;
constexpr int64_t kPackMagic = 0x32505444;  // "DTP2"

struct PackHeader {
  int64_t magic, T, n_blocks, n_esc, off_base, off_esc, off_boff, off_flags, off_data, off_escapes;
};

inline size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }

struct TetCode {
  uint8_t flag;
  int nbytes, nesc;
  uint16_t val[8];   // field codes (1 or 2 bytes each)
  int32_t esc[8];
};

// Field codes of one tetrahedron against block base `base`.
inline void encode_tet(int64_t t, const int32_t* v, const int32_t* n, int32_t base, TetCode& c) {
  c.flag = 0;
  c.nbytes = 0;
  c.nesc = 0;
  auto unsigned_field = [&](int f, int64_t o, int32_t full) {
    if (o >= 0 && o < 0xFF) { c.val[f] = (uint16_t)o; c.nbytes += 1; }
    else if (o >= 0 && o < 0xFFFF) { c.val[f] = (uint16_t)o; c.flag |= (uint8_t)(1u << f); c.nbytes += 2; }
    else { c.val[f] = 0xFF; c.nbytes += 1; c.esc[c.nesc++] = full; }
  };
  unsigned_field(0, (int64_t)v[0] - base, v[0]);
  for (int k = 1; k < 4; ++k) unsigned_field(k, (int64_t)v[k] - v[0], v[k]);
  for (int k = 0; k < 4; ++k) {
    const int f = 4 + k;
    if (n[k] < 0) { c.val[f] = (uint16_t)(uint8_t)(int8_t)-128; c.nbytes += 1; continue; }
    const int64_t d = (int64_t)n[k] - t;
    if (d >= -127 && d <= 126) { c.val[f] = (uint16_t)(uint8_t)(int8_t)d; c.nbytes += 1; }
    else if (d >= -32767 && d <= 32766) { c.val[f] = (uint16_t)(int16_t)d; c.flag |= (uint8_t)(1u << f); c.nbytes += 2; }
    else { c.val[f] = 127; c.nbytes += 1; c.esc[c.nesc++] = n[k]; }
  }
}
}  // namespace

extern "C" {

// Packs T tetrahedra (tet_v, tet_n: 4 int32 each).  out == NULL: returns the
// packed size in bytes; otherwise writes it (out must hold that many bytes)
// and returns the same size.  Negative on bad arguments.
int64_t dtfe_tets_pack(const int32_t* tet_v, const int32_t* tet_n, int64_t T, void* out) {
  if (T < 0 || (T > 0 && (!tet_v || !tet_n))) return -1;
  const int64_t nb = (T + kPackBlock - 1) / kPackBlock;
  std::vector<int32_t> base(nb), cnt(nb + 1, 0);
  std::vector<int64_t> boff(nb + 1, 0);
#pragma omp parallel for schedule(static)
  for (int64_t b = 0; b < nb; ++b) {
    const int64_t t0 = b * kPackBlock, t1 = std::min(T, t0 + kPackBlock);
    int32_t m = tet_v[4 * t0];
    for (int64_t t = t0; t < t1; ++t) m = std::min(m, tet_v[4 * t]);
    base[b] = m;
    int ne = 0;
    int64_t bytes = 0;
    TetCode c;
    for (int64_t t = t0; t < t1; ++t) {
      encode_tet(t, tet_v + 4 * t, tet_n + 4 * t, m, c);
      ne += c.nesc;
      bytes += c.nbytes;
    }
    cnt[b + 1] = ne;
    boff[b + 1] = bytes;
  }
  for (int64_t b = 0; b < nb; ++b) {
    cnt[b + 1] += cnt[b];
    boff[b + 1] += boff[b];
  }
  PackHeader hd;
  hd.magic = kPackMagic;
  hd.T = T;
  hd.n_blocks = nb;
  hd.n_esc = cnt[nb];
  hd.off_base = (int64_t)align16(sizeof(PackHeader));
  hd.off_esc = hd.off_base + (int64_t)align16(sizeof(int32_t) * nb);
  hd.off_boff = hd.off_esc + (int64_t)align16(sizeof(int32_t) * (nb + 1));
  hd.off_flags = hd.off_boff + (int64_t)align16(sizeof(int64_t) * (nb + 1));
  hd.off_data = hd.off_flags + (int64_t)align16((size_t)T);
  hd.off_escapes = hd.off_data + (int64_t)align16((size_t)boff[nb] + 16);
  const int64_t total = hd.off_escapes + (int64_t)align16(sizeof(int32_t) * hd.n_esc);
  if (!out) return total;
  char* o = (char*)out;
  std::memset(o, 0, (size_t)total);
  std::memcpy(o, &hd, sizeof(hd));
  std::memcpy(o + hd.off_base, base.data(), sizeof(int32_t) * nb);
  std::memcpy(o + hd.off_esc, cnt.data(), sizeof(int32_t) * (nb + 1));
  std::memcpy(o + hd.off_boff, boff.data(), sizeof(int64_t) * (nb + 1));
  uint8_t* flags = (uint8_t*)(o + hd.off_flags);
  uint8_t* data = (uint8_t*)(o + hd.off_data);
  int32_t* esc = (int32_t*)(o + hd.off_escapes);
#pragma omp parallel for schedule(static)
  for (int64_t b = 0; b < nb; ++b) {
    const int64_t t0 = b * kPackBlock, t1 = std::min(T, t0 + kPackBlock);
    uint8_t* d = data + boff[b];
    int32_t* e = esc + cnt[b];
    TetCode c;
    for (int64_t t = t0; t < t1; ++t) {
      encode_tet(t, tet_v + 4 * t, tet_n + 4 * t, base[b], c);
      flags[t] = c.flag;
      for (int f = 0; f < 8; ++f) {
        *d++ = (uint8_t)(c.val[f] & 0xFF);
        if (c.flag >> f & 1) *d++ = (uint8_t)(c.val[f] >> 8);
      }
      for (int q = 0; q < c.nesc; ++q) *e++ = c.esc[q];
    }
  }
  return total;
}

// Host decoder of dtfe_tets_pack's format (the device decodes in
// dtfe_gpu_upload_packed).  Returns 0, or 1 for a malformed buffer.
int dtfe_tets_unpack(const void* packed, int64_t bytes, int32_t* tet_v, int32_t* tet_n) {
  if (!packed || bytes < (int64_t)sizeof(PackHeader)) return 1;
  PackHeader hd;
  std::memcpy(&hd, packed, sizeof(hd));
  if (hd.magic != kPackMagic || hd.off_escapes + 4 * hd.n_esc > bytes) return 1;
  const char* p = (const char*)packed;
  const int32_t* base = (const int32_t*)(p + hd.off_base);
  const int32_t* cnt = (const int32_t*)(p + hd.off_esc);
  const int64_t* boff = (const int64_t*)(p + hd.off_boff);
  const uint8_t* flags = (const uint8_t*)(p + hd.off_flags);
  const uint8_t* data = (const uint8_t*)(p + hd.off_data);
  const int32_t* esc = (const int32_t*)(p + hd.off_escapes);
  for (int64_t b = 0; b < hd.n_blocks; ++b) {
    const uint8_t* d = data + boff[b];
    const int32_t* e = esc + cnt[b];
    for (int64_t t = b * kPackBlock; t < std::min(hd.T, (b + 1) * kPackBlock); ++t) {
      uint32_t raw[8];
      bool wide[8];
      for (int f = 0; f < 8; ++f) {
        wide[f] = flags[t] >> f & 1;
        raw[f] = *d++;
        if (wide[f]) raw[f] |= (uint32_t)(*d++) << 8;
      }
      int32_t* v = tet_v + 4 * t;
      auto uval = [&](int f, int32_t ref) -> int32_t {
        const bool escaped = wide[f] ? raw[f] == 0xFFFF : raw[f] == 0xFF;
        return escaped ? *e++ : ref + (int32_t)raw[f];
      };
      v[0] = uval(0, base[b]);
      for (int k = 1; k < 4; ++k) v[k] = uval(k, v[0]);
      for (int k = 0; k < 4; ++k) {
        const int f = 4 + k;
        const int32_t sv = wide[f] ? (int32_t)(int16_t)raw[f] : (int32_t)(int8_t)raw[f];
        const int32_t lo = wide[f] ? -32768 : -128, hi = wide[f] ? 32767 : 127;
        tet_n[4 * t + k] = sv == lo ? -1 : (sv == hi ? *e++ : (int32_t)(t + sv));
      }
    }
  }
  return 0;
}

}  // extern "C"

// ---- vertex-only packed tessellation (dtfe_tets_pack_vertices) ------------
// The neighbour array follows from the vertex array (two tetrahedra are
// neighbours across the face whose three vertices both hold), so it need
// not cross PCIe at all: the device derives it (dtfe_gpu_upload_packed).
// The vertices are coded as differences: the first vertex against the
// previous tetrahedron's first vertex (signed), the second against the first,
// the smaller of the last two against the second and the larger against the
// smaller (all positive: the first vertex is the smallest and the second the
// smallest of the rest in the canonical order), with one bit saying whether
// the third vertex is the larger.  Every field takes 1 or 2 bytes, a 4-bit
// width flag per tetrahedron says which, and values that fit neither are
// escaped to a 32-bit list (as the difference itself).  About 5 bytes per
// tetrahedron instead of 32.
// Layout:
//   header       10 x int64: magic "DTP3", T, n_blocks, n_escapes, and the byte
//                offsets of block_base, block_esc, block_off, flags, orient, data
//                (the escapes follow the data at its 16-byte aligned end)
//   block_base   int32 per block: the first vertex of the block's first
//                tetrahedron (its own first field is 0)
//   block_esc    int32 per block + 1: escapes before the block
//   block_off    int64 per block + 1: byte offset of the block in data
//   flags        4 bits per tetrahedron (even t: low nibble): bit f set = field f takes 2 bytes
//   orient       1 bit per tetrahedron (bit t % 8 of byte t / 8): the third vertex is the larger
//   data         the fields, tetrahedron after tetrahedron, little endian:
//                field 0 signed (maximum: escaped), fields 1-3 unsigned (all ones: escaped)
//   escapes      int32 values of the escaped fields, in (tetrahedron, field) order
namespace {
constexpr int64_t kPack3Magic = 0x33505444;  // "DTP3"

struct Tet3Code {
  uint8_t flag;
  bool orient;
  int nbytes, nesc;
  uint16_t val[4];
  int32_t esc[4];
};

inline bool encode_tet3(const int32_t* v, int32_t prev0, Tet3Code& c) {
  c.flag = 0;
  c.nbytes = 0;
  c.nesc = 0;
  const int32_t lo = std::min(v[2], v[3]), hi = std::max(v[2], v[3]);
  c.orient = v[2] > v[3];
  if (!(v[1] > v[0] && lo > v[1] && hi > lo)) return false;  // not in canonical order
  const int64_t d0 = (int64_t)v[0] - prev0;
  if (d0 >= -127 && d0 <= 126) { c.val[0] = (uint16_t)(uint8_t)(int8_t)d0; c.nbytes += 1; }
  else if (d0 >= -32767 && d0 <= 32766) { c.val[0] = (uint16_t)(int16_t)d0; c.flag |= 1; c.nbytes += 2; }
  else { c.val[0] = 127; c.nbytes += 1; c.esc[c.nesc++] = (int32_t)d0; }
  const int64_t d[3] = {(int64_t)v[1] - v[0], (int64_t)lo - v[1], (int64_t)hi - lo};
  for (int f = 1; f < 4; ++f) {
    const int64_t o = d[f - 1];
    if (o < 0xFF) { c.val[f] = (uint16_t)o; c.nbytes += 1; }
    else if (o < 0xFFFF) { c.val[f] = (uint16_t)o; c.flag |= (uint8_t)(1u << f); c.nbytes += 2; }
    else { c.val[f] = 0xFF; c.nbytes += 1; c.esc[c.nesc++] = (int32_t)o; }
  }
  return true;
}
}  // namespace

extern "C" {

// Packs T tetrahedra given by their vertices alone (tet_v: 4 int32 each, in
// the canonical order of the planner's tessellations: the smallest vertex
// first, the second the smallest of the rest).  out == NULL: returns the size
// in bytes; otherwise writes it and returns the same size.  Negative on bad
// arguments or a tetrahedron not in canonical order.
int64_t dtfe_tets_pack_vertices(const int32_t* tet_v, int64_t T, void* out) {
  if (T < 0 || (T > 0 && !tet_v)) return -1;
  const int64_t nb = (T + kPackBlock - 1) / kPackBlock;
  std::vector<int32_t> base(nb), cnt(nb + 1, 0);
  std::vector<int64_t> boff(nb + 1, 0);
  int bad = 0;
#pragma omp parallel for schedule(static) reduction(+ : bad)
  for (int64_t b = 0; b < nb; ++b) {
    const int64_t t0 = b * kPackBlock, t1 = std::min(T, t0 + kPackBlock);
    base[b] = tet_v[4 * t0];
    int ne = 0;
    int64_t bytes = 0;
    Tet3Code c;
    for (int64_t t = t0; t < t1; ++t) {
      if (!encode_tet3(tet_v + 4 * t, t == t0 ? base[b] : tet_v[4 * (t - 1)], c)) ++bad;
      ne += c.nesc;
      bytes += c.nbytes;
    }
    cnt[b + 1] = ne;
    boff[b + 1] = bytes;
  }
  if (bad) return -2;
  for (int64_t b = 0; b < nb; ++b) {
    cnt[b + 1] += cnt[b];
    boff[b + 1] += boff[b];
  }
  PackHeader hd;
  hd.magic = kPack3Magic;
  hd.T = T;
  hd.n_blocks = nb;
  hd.n_esc = cnt[nb];
  hd.off_base = (int64_t)align16(sizeof(PackHeader));
  hd.off_esc = hd.off_base + (int64_t)align16(sizeof(int32_t) * nb);
  hd.off_boff = hd.off_esc + (int64_t)align16(sizeof(int32_t) * (nb + 1));
  hd.off_flags = hd.off_boff + (int64_t)align16(sizeof(int64_t) * (nb + 1));
  // off_data holds the orientation bits' offset; the data follows them
  hd.off_data = hd.off_flags + (int64_t)align16((size_t)(T + 1) / 2);
  hd.off_escapes = hd.off_data + (int64_t)align16((size_t)(T + 7) / 8);
  const int64_t data_end = hd.off_escapes + (int64_t)align16((size_t)boff[nb] + 16);
  const int64_t total = data_end + (int64_t)align16(sizeof(int32_t) * hd.n_esc);
  if (!out) return total;
  char* o = (char*)out;
  std::memset(o, 0, (size_t)total);
  std::memcpy(o, &hd, sizeof(hd));
  std::memcpy(o + hd.off_base, base.data(), sizeof(int32_t) * nb);
  std::memcpy(o + hd.off_esc, cnt.data(), sizeof(int32_t) * (nb + 1));
  std::memcpy(o + hd.off_boff, boff.data(), sizeof(int64_t) * (nb + 1));
  uint8_t* flags = (uint8_t*)(o + hd.off_flags);
  uint8_t* orient = (uint8_t*)(o + hd.off_data);
  uint8_t* data = (uint8_t*)(o + hd.off_escapes);
  int32_t* esc = (int32_t*)(o + data_end);
  // blocks of 256 tetrahedra start on whole flag and orientation bytes
#pragma omp parallel for schedule(static)
  for (int64_t b = 0; b < nb; ++b) {
    const int64_t t0 = b * kPackBlock, t1 = std::min(T, t0 + kPackBlock);
    uint8_t* d = data + boff[b];
    int32_t* e = esc + cnt[b];
    Tet3Code c;
    for (int64_t t = t0; t < t1; ++t) {
      encode_tet3(tet_v + 4 * t, t == t0 ? base[b] : tet_v[4 * (t - 1)], c);
      flags[t >> 1] |= (uint8_t)(c.flag << ((t & 1) * 4));
      if (c.orient) orient[t >> 3] |= (uint8_t)(1u << (t & 7));
      for (int f = 0; f < 4; ++f) {
        *d++ = (uint8_t)(c.val[f] & 0xFF);
        if (c.flag >> f & 1) *d++ = (uint8_t)(c.val[f] >> 8);
      }
      for (int q = 0; q < c.nesc; ++q) *e++ = c.esc[q];
    }
  }
  return total;
}

// Host decoder of dtfe_tets_pack_vertices' format: restores tet_v.  Returns
// 0, or 1 for a malformed buffer.
int dtfe_tets_unpack_vertices(const void* packed, int64_t bytes, int32_t* tet_v) {
  if (!packed || bytes < (int64_t)sizeof(PackHeader)) return 1;
  PackHeader hd;
  std::memcpy(&hd, packed, sizeof(hd));
  if (hd.magic != kPack3Magic || hd.T < 0 || hd.n_blocks != (hd.T + kPackBlock - 1) / kPackBlock) return 1;
  const char* p = (const char*)packed;
  const int64_t* boff = (const int64_t*)(p + hd.off_boff);
  const int64_t data_end = hd.off_escapes + (int64_t)align16((size_t)boff[hd.n_blocks] + 16);
  if (data_end + 4 * hd.n_esc > bytes) return 1;
  const int32_t* base = (const int32_t*)(p + hd.off_base);
  const int32_t* cnt = (const int32_t*)(p + hd.off_esc);
  const uint8_t* flags = (const uint8_t*)(p + hd.off_flags);
  const uint8_t* orient = (const uint8_t*)(p + hd.off_data);
  const uint8_t* data = (const uint8_t*)(p + hd.off_escapes);
  const int32_t* esc = (const int32_t*)(p + data_end);
  for (int64_t b = 0; b < hd.n_blocks; ++b) {
    const uint8_t* d = data + boff[b];
    const int32_t* e = esc + cnt[b];
    int32_t prev = base[b];
    for (int64_t t = b * kPackBlock; t < std::min(hd.T, (b + 1) * kPackBlock); ++t) {
      const int flag = (flags[t >> 1] >> ((t & 1) * 4)) & 15;
      uint32_t raw[4];
      for (int f = 0; f < 4; ++f) {
        raw[f] = *d++;
        if (flag >> f & 1) raw[f] |= (uint32_t)(*d++) << 8;
      }
      const bool w0 = flag & 1;
      const int32_t s0 = w0 ? (int32_t)(int16_t)raw[0] : (int32_t)(int8_t)raw[0];
      const int32_t d0 = s0 == (w0 ? 32767 : 127) ? *e++ : s0;
      int32_t dd[3];
      for (int f = 1; f < 4; ++f) {
        const bool wide = flag >> f & 1;
        dd[f - 1] = raw[f] == (wide ? 0xFFFFu : 0xFFu) ? *e++ : (int32_t)raw[f];
      }
      int32_t* v = tet_v + 4 * t;
      v[0] = prev + d0;
      v[1] = v[0] + dd[0];
      const int32_t lo = v[1] + dd[1], hi = lo + dd[2];
      const bool third_larger = orient[t >> 3] >> (t & 7) & 1;
      v[2] = third_larger ? hi : lo;
      v[3] = third_larger ? lo : hi;
      prev = v[0];
    }
  }
  return 0;
}

}  // extern "C"
