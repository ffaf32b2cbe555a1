/* Host half of the drop-in boundary: the control flow the reference's DTFE()
 * runs before interpolating (padding, periodic images, sub-box split,
 * tessellation), producing the flat arrays that include/dtfe_gpu.h consumes.
 * Built into libdtfe_host.so (no CUDA).  Every function returns 0 on
 * success; plans are owned by the library until dtfe_plan_release.
 *
 * Reference routines restated (src/ of lrwesterhoek/DTFE):
 *   dtfe_padding_length      User_options::updatePadding   src/user_options.cc:1062-1089
 *   dtfe_average_density     averageDensity                src/subpartition.h:437-449
 *   dtfe_select_in_box       findParticlesInBox            src/subpartition.h:79-154
 *   dtfe_parallel_grid       parallelGrid                  src/subpartition.h:454-555
 *   dtfe_optimal_partition   optimalPartitionSplit         src/subpartition.h:163-372
 *   dtfe_axis_coords         the x += dx sample raster     src/unaveraged_interpolation.cc:252-358
 *   dtfe_tessellate(_batch)  delaunayTriangulation         src/CGAL_triangulation/triangulation.cpp:162-195
 *   dtfe_plan_build(_ex)     DTFE() + DTFE_parallel() up to the interpolation
 *                            src/DTFE.cpp:76-251, 287-385
 *   dtfe_write_binary        writeBinaryFile               src/io/binary_io.cc:185-216
 *   dtfe_field_suffix        writeOutputData's file names  src/input_output.cc:216-275
 */
#ifndef DTFE_HOST_H
#define DTFE_HOST_H

#include <stdint.h>

#include "dtfe_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

void dtfe_padding_length(int kind, float padding_particles, int64_t n_total, const float full_box_length[3],
                         const int64_t grid[3], float out[6]);
float dtfe_average_density(const float* w, int64_t n);
int64_t dtfe_select_in_box(const float* pos, int64_t n, const float full_box[6], const float padded[6],
                           int periodic, int32_t* out_idx, float* out_pos);
void dtfe_parallel_grid(int64_t n_threads, const int64_t main_grid[3], int64_t grid[3]);
int dtfe_optimal_partition(const float* pos, int64_t n, const int64_t grid[3], const float region[6],
                           const int64_t parts[3], int64_t* subgrid, float* coords);
void dtfe_axis_coords(float lo, float dx, int64_t n, float* out);

int dtfe_tessellate(const double* xyz, int64_t n, uint64_t seed, int sort_tets, void** handle);
void dtfe_tessellate_batch(int k, const double* const* xyz, const int64_t* n, uint64_t seed, int sort_tets,
                           void** handles, int* rc);
void dtfe_tess_sizes(void* handle, int64_t* n_tets, int64_t* n_points, int64_t* n_duplicates);
void dtfe_tess_export(void* handle, int32_t* tet_v, int32_t* tet_n, int32_t* vmap);
void dtfe_tess_release(void* handle);

/* Packed tessellation for the PCIe transfer (dtfe_gpu_upload_packed), about
 * 11 bytes per tetrahedron instead of 32: per tetrahedron a flag byte and
 * eight 1- or 2-byte fields (first vertex from the smallest first vertex of
 * its block of 256, the other vertices from the first, neighbours from the
 * tetrahedron's own id), values that fit neither escaped to 32 bits.
 * out == NULL returns the size in bytes; otherwise writes the buffer and
 * returns its size (negative: bad arguments).  dtfe_tets_unpack restores
 * the arrays (0 on success, 1 for a malformed buffer). */
int64_t dtfe_tets_pack(const int32_t* tet_v, const int32_t* tet_n, int64_t T, void* out);
int dtfe_tets_unpack(const void* packed, int64_t bytes, int32_t* tet_v, int32_t* tet_n);
/* Vertex-only packed form (format "DTP3"), about 5 bytes per tetrahedron:
 * the neighbours are not sent, the device derives them.  Per tetrahedron
 * four 1- or 2-byte differences (first vertex against the previous
 * tetrahedron's, second against the first, the smaller of the last two
 * against the second, the larger against the smaller), a 4-bit width flag
 * and a bit saying whether the third vertex is the larger; escapes to 32
 * bits.  The tetrahedra must be in the planner's canonical vertex order
 * (the first vertex the smallest, the second the smallest of the rest;
 * returns -2 otherwise).  Sizes and return values as dtfe_tets_pack;
 * dtfe_tets_unpack_vertices restores tet_v. */
int64_t dtfe_tets_pack_vertices(const int32_t* tet_v, int64_t T, void* out);
int dtfe_tets_unpack_vertices(const void* packed, int64_t bytes, int32_t* tet_v);

/* ---- whole-run planning --------------------------------------------------- */
enum {
  DTFE_PLAN_DTFE = 0, /* tessellated sub-boxes (DTFE and SPH) */
  DTFE_PLAN_NGP = 1,  /* particle regions only, the estimators' own padding */
  DTFE_PLAN_CIC = 2,
  DTFE_PLAN_TSC = 3
};

typedef struct dtfe_plan_s* dtfe_plan;

/* Read-only view of a plan (pointers owned by the plan). */
typedef struct {
  int32_t kind;
  int32_t grid[3];
  double rho_bar;      /* averageDensity used (given, or Sum(w)/35000^3) */
  float padding[6];
  /* DTFE_PLAN_DTFE: the flat multi-tessellation for dtfe_gpu_upload /
   * dtfe_gpu_set_subboxes */
  int64_t n_verts, n_tets;
  int32_t n_boxes, n_scalars;
  const int32_t* tet_v;   /* 4 T */
  const int32_t* tet_n;   /* 4 T */
  const float* xyz;       /* 3 V */
  const int32_t* src;     /* V: input particle of each vertex */
  const float* weight;    /* V */
  const float* velocity;  /* 3 V or NULL */
  const float* scalar;    /* S V or NULL */
  const dtfe_subbox* boxes;
  const float* regions;   /* 6 per sub-box: its tile region (dtfe_gpu_set_regions) */
  const float *xs, *ys, *zs;
  int64_t n_xs, n_ys, n_zs;
  /* DTFE_PLAN_NGP/CIC/TSC: particle copies per region for dtfe_gpu_deposit */
  int64_t n_particles;
  const float* dep_pos;       /* 3 n */
  const float* dep_weight;    /* n */
  const float* dep_velocity;  /* 3 n or NULL */
  const int64_t* dep_src;     /* n */
  int32_t n_dep_boxes;
  const dtfe_deposit_box* dep_boxes;
  /* the region the grid covers: the box, the --region, or with --partNo the
   * chunk (the reference sets userOptions.region to it, src/DTFE.cpp:151) */
  float region[6];
} dtfe_plan_view;

/* Options of DTFE() that change the planning (User_options members,
 * src/user_options.h:100-190). */
enum {
  DTFE_PAD_PARTICLES = 0, /* --padding n: n particle spacings (paddingParticles) */
  DTFE_PAD_RELATIVE = 1,  /* --padding l1..l6: lengths in box lengths */
  DTFE_PAD_ABSOLUTE = 2   /* --paddingMpc l1..l6: lengths in the particles' units */
};
typedef struct {
  int32_t n_parts;          /* parallelGrid split (the OpenMP thread count) */
  int32_t padding_mode;     /* DTFE_PAD_*; six zero lengths fall back to the particle count, as
                               User_options::updatePadding (isNullBox) */
  float padding_particles;  /* paddingParticles (5 by default) */
  float padding[6];         /* paddingLength: left/right per axis, x first */
  int32_t region_on;        /* --region: interpolate only region[6] */
  float region[6];          /* absolute coordinates (User_options::updateEntries converts box
                               fractions, src/user_options.cc:952-958) */
  int32_t partition_on;     /* --partition: split into partition[0..2] chunks */
  int32_t partition[3];
  int32_t part_no;          /* --partNo: only that chunk (its own grid); -1 all chunks */
  double average_density;   /* <= 0: the reference's automatic value */
} dtfe_plan_options;

/* Plans one box of n particles (pos 3n, w n or NULL = unit, vel 3n or
 * NULL, scal S*n or NULL) in [box] on a grid of grid[0..2] cells, split
 * into parallelGrid(n_parts) sub-boxes (the reference's OpenMP thread
 * count), with the reference's padding for `kind` (padding_particles = its
 * --padding, 5 by default) and periodic images when `periodic`.
 * average_density <= 0 takes the reference's automatic value.  The same
 * arithmetic as dtfe_b200/plan.py (make_plan / make_deposit_plan). */
int dtfe_plan_build(int kind, const float* pos, const float* w, const float* vel, const float* scal, int32_t S,
                    int64_t n, const float box[6], int periodic, const int32_t grid[3], int32_t n_parts,
                    float padding_particles, double average_density, dtfe_plan* out);
/* Same with DTFE()'s region, partition and padding options
 * (src/DTFE.cpp:76-251): --region selects the particles of the padded region
 * and interpolates only there; --partition plans every chunk of
 * optimalPartitionSplit with its own padded particles, each split further
 * into n_parts sub-boxes, all placed in the main grid (the GPU runs them in
 * one batched step instead of one chunk after another); --partNo plans one
 * chunk onto a grid of its own size (view.grid, view.region).  Returns 0, 1
 * for bad arguments, 4 for a region that is not a valid sub-box of the box
 * (Box::validSubBox, src/box.h:115-138). */
int dtfe_plan_build_ex(int kind, const float* pos, const float* w, const float* vel, const float* scal, int32_t S,
                       int64_t n, const float box[6], int periodic, const int32_t grid[3],
                       const dtfe_plan_options* opts, dtfe_plan* out);
int dtfe_plan_get(dtfe_plan p, dtfe_plan_view* view);
void dtfe_plan_release(dtfe_plan p);

/* Output files in the reference's binary format (outputFileType 101).
 * dtfe_write_binary writes `bytes` raw bytes of `data` (a field's cells x
 * components floats) to `path`, created or truncated, without a header: the
 * file writeBinaryFile (src/io/binary_io.cc:185-216) makes from the
 * corresponding Quantities vector.  DTFE_ERR_IO when the file cannot be
 * opened or fully written.  dtfe_field_suffix gives writeOutputData's file
 * suffix (src/input_output.cc:216-275) of field `slot` for uQuantities
 * (averaged = 0: ".den", ".vel", ".velGrad", ...) or aQuantities
 * (".a_den", ...); NULL for a slot without a file (the unaveraged velocity
 * standard deviation) or out of range. */
int dtfe_write_binary(const char* path, const void* data, int64_t bytes);
const char* dtfe_field_suffix(int32_t slot, int32_t averaged);

#ifdef __cplusplus
}
#endif
#endif /* DTFE_HOST_H */
