// Exact, order-independent sums of tetrahedron volumes per vertex.
//
// Every FP64 volume is rounded once to a 64-bit integer multiple of
// q = (bounding-box volume of the vertices) * 2^-62 and the multiples are
// added as integers, so a vertex's sum does not depend on the order in which
// threads add (integer addition is associative) and never overflows: the
// cells around a vertex are disjoint and lie inside the convex hull, so
// their volumes add up to at most the bounding box's, 2^62 q.  Each term's
// rounding error is at most q/2, i.e. 2^-63 of the bounding-box volume.
// The bounding box is that of the tessellation's own vertices (one sub-box),
// so a sub-box gives the same sums whichever other sub-boxes share its
// upload.  Shared by the GPU kernels and the CPU oracle.
#pragma once

#include <cstdint>
#include <cstring>

#if defined(__CUDACC__)
#define DTFE_FV __host__ __device__ __forceinline__
#else
#define DTFE_FV inline
#endif

namespace dtfe {

// Order-preserving map of a float to an int (for atomicMin / atomicMax on
// bounding boxes): a < b exactly when key(a) < key(b).
DTFE_FV int float_order_key(float f) {
  int i;
  memcpy(&i, &f, sizeof(i));
  return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
DTFE_FV float float_from_order_key(int k) {
  const int i = k >= 0 ? k : k ^ 0x7FFFFFFF;
  float f;
  memcpy(&f, &i, sizeof(f));
  return f;
}

// Volume of the bounding box (xmin, xmax, ymin, ymax, zmin, zmax given as
// float order keys), in double: the float differences are exact in double,
// their product rounds twice.
DTFE_FV double bbox_volume(const int k[6]) {
  const double dx = (double)float_from_order_key(k[1]) - (double)float_from_order_key(k[0]);
  const double dy = (double)float_from_order_key(k[3]) - (double)float_from_order_key(k[2]);
  const double dz = (double)float_from_order_key(k[5]) - (double)float_from_order_key(k[4]);
  return (dx * dy) * dz;
}

// Scale of one tessellation: inv_q = 2^62 / box volume turns a volume into
// integer units (0 for an empty or flat box: every volume is then 0), unit =
// box volume * 2^-62 turns a sum of units back (exact: a power-of-two
// scaling).
struct VolScale {
  double inv_q, unit;
};
DTFE_FV VolScale vol_scale(double box_volume) {
  VolScale s;
  s.inv_q = box_volume > 0.0 ? 0x1p62 / box_volume : 0.0;
  s.unit = box_volume * 0x1p-62;
  return s;
}
DTFE_FV double fixed_scale(double box_volume) { return vol_scale(box_volume).inv_q; }
DTFE_FV double fixed_unit(double box_volume) { return vol_scale(box_volume).unit; }

// The sum back in volume units, then the vertex density as in vertexDensity
// (triangulation.cpp:266-269): (w * factor) / volume, 0 on the hull or
// without volume.
DTFE_FV float density_from_fixed(long long sum, double unit, float w, float factor, bool hull) {
  const double vol = (double)sum * unit;
  return (hull || !(vol > 0.0)) ? 0.f : (float)((double)(w * factor) / vol);
}

}  // namespace dtfe

#undef DTFE_FV
