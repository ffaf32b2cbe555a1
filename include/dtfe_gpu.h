/*
 * dtfe_gpu.h — C ABI of the B200 DTFE interpolation path.
 *
 * The reference exposes one C++ entry point,
 *     void DTFE(std::vector<Particle_data>*, std::vector<Sample_point>&,
 *               User_options&, Quantities* u, Quantities* a)
 * (src/DTFE.h:36-40, body src/DTFE.cpp:76-251), whose hot section is
 * DTFE_interpolation() after the Delaunay tessellation is built
 * (src/CGAL_triangulation/triangulation.cpp:98-144) and DTFE_parallel()
 * for the sub-box split (src/DTFE.cpp:287-385).  This header is the seam at
 * that point: the host builds the tessellation, flattens it, and drives the
 * device through these functions.  A C++ shim with the reference's exact
 * DTFE(...) signature (include/dtfe/DTFE.h) sits on top of it.
 *
 * Conventions
 *  - Every function returns an int status (DTFE_OK = 0); nothing calls exit().
 *  - Plain pointers and sizes only.  Pointers are HOST memory unless the
 *    argument name ends in _dev.
 *  - A handle owns its device buffers and one CUDA stream; use one handle
 *    from one host thread at a time.  Calls are ordered on that stream.
 *  - Tetrahedra are positively oriented (CGAL's cell orientation);
 *    tet_v[4t+i] is vertex i of tetrahedron t and tet_n[4t+i] is the
 *    tetrahedron across the face opposite vertex i, or -1 on the convex hull
 *    (the reference's infinite cells).  Indices are global over all sub-boxes.
 *  - Grids are x-slowest, z-fastest (gridCellIndex,
 *    src/CGAL_triangulation/triangulation_miscellaneous.cc:219-237); each
 *    output field is an array of cells, each cell holding the field's
 *    components contiguously, i.e. the layout of the vectors in struct
 *    Quantities (src/quantities.h:56-76).
 */
#ifndef DTFE_GPU_H
#define DTFE_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
enum {
  DTFE_OK = 0,
  DTFE_ERR_ARG = 1,          /* invalid argument or size */
  DTFE_ERR_CUDA = 2,         /* CUDA runtime error (message: dtfe_last_error) */
  DTFE_ERR_ALLOC = 3,        /* device allocation failed */
  DTFE_ERR_STATE = 4,        /* call out of order (e.g. interpolate before upload) */
  DTFE_ERR_WALK = 5,         /* a point-location walk hit its step limit */
  DTFE_ERR_DEGENERATE = 6,   /* fewer than 4 vertices: no tetrahedra */
  DTFE_ERR_NO_DEVICE = 7,    /* no usable CUDA device / extension */
  DTFE_ERR_TOO_LARGE = 8,    /* request exceeds a documented maximum */
  DTFE_ERR_IO = 9            /* an output file could not be opened or written */
};

/* ---- output field slots (bit i of a field mask = slot i) --------------- */
enum {
  DTFE_DENSITY = 0,              /* 1 component            */
  DTFE_VELOCITY = 1,             /* 3 components           */
  DTFE_VELOCITY_GRADIENT = 2,    /* 9: [j*3+i] = d v_j / d x_i */
  DTFE_VELOCITY_DIVERGENCE = 3,  /* 1                      */
  DTFE_VELOCITY_SHEAR = 4,       /* 5: xx,xy,xz,yy,yz traceless */
  DTFE_VELOCITY_VORTICITY = 5,   /* 3: xy,xz,yz            */
  DTFE_VELOCITY_STD = 6,         /* 1 (Monte-Carlo method only) */
  DTFE_SCALAR = 7,               /* S components           */
  DTFE_SCALAR_GRADIENT = 8,      /* 3*S: [s*3+i]           */
  DTFE_NUM_FIELDS = 9
};
#define DTFE_FIELD_BIT(slot) (1u << (slot))

/* ---- interpolation methods (User_options::method, plus plain sampling) -- */
enum {
  DTFE_METHOD_CENTRE = 0,       /* field at the cell centre (uQuantities) */
  DTFE_METHOD_TETRAHEDRA = 1,   /* n points per cell on average, placed in
                                   the tetrahedra (Sobol) and scattered to
                                   the cells (interpolateGrid_averaged_1,
                                   averaged_interpolation_1.cc:197-421)   */
  DTFE_METHOD_MONTE_CARLO = 2,  /* mean of n random points per cell       */
  DTFE_METHOD_EQUIDISTANT = 3   /* mean of n = m^3 equidistant points     */
};

/* ---- behaviour flags ---------------------------------------------------- */
/* Reference velocityValue()/scalarValue() keep only the z term of the
 * gradient product (unaveraged_interpolation.cc:116,159).  Default: keep that
 * behaviour for parity; this flag evaluates the full dot product instead. */
#define DTFE_FLAG_FIX_VALUE_INTERP 1u
/* Reference interpolateGrid() skips its `z += dx` after a sample outside the
 * hull (the `continue` at unaveraged_interpolation.cc:304 jumps over :353),
 * so every later sample of that z pencil re-locates the same outside point
 * and gets zeros; interpolateRedshiftCone() does the same with `psi += dx`
 * (:466 jumps over :527).  Default (cell centres and cone bins): the same
 * zeros, for parity; this flag evaluates those samples at their own centres
 * instead. */
#define DTFE_FLAG_FIX_OUTSIDE_RASTER 2u

/* ---- limits -------------------------------------------------------------- */
#define DTFE_MAX_SCALARS 8
#define DTFE_MAX_STD_SAMPLES 64   /* velocity_std keeps every sample velocity */

typedef struct dtfe_gpu_s* dtfe_handle;

typedef struct {
  int32_t device;        /* CUDA device ordinal */
  int32_t n_scalars;     /* S, 0..DTFE_MAX_SCALARS */
  int32_t max_walk_steps;/* 0 = default (65536) */
  int32_t reserved;
} dtfe_config;

/* One sub-box: a padded tessellation of its own and the grid tile it owns.
 * (DTFE_parallel / --partition chunks, src/DTFE.cpp:169-218,287-385;
 * copySubgridInformation, src/subpartition.h:376-383.)  A single-box run is
 * one sub-box covering the whole grid. */
typedef struct {
  int64_t vert_offset, n_verts;   /* vertex range of this tessellation */
  int64_t tet_offset, n_tets;     /* tetrahedron range */
  int32_t tile_origin[3];         /* first main-grid cell of the tile */
  int32_t tile_dims[3];           /* tile size in cells */
  int64_t coord_offset[3];        /* into the per-axis coordinate tables */
  float   dx[3];                  /* cell size of the tile (float, as the reference) */
  float   lo[3];                  /* lower corner of the tile region */
  int32_t part_no;                /* partition number (Monte-Carlo seed offset) */
  int32_t reserved;
} dtfe_subbox;

typedef struct {
  int32_t method;       /* DTFE_METHOD_* */
  int32_t n_samples;    /* points per cell for methods 2 and 3 */
  uint64_t seed;        /* Monte-Carlo key (randomSeed) */
  uint32_t fields;      /* mask of DTFE_FIELD_BIT(slot) */
  uint32_t flags;       /* DTFE_FLAG_* */
} dtfe_interp_opts;

typedef struct {
  int64_t n_samples_located;  /* point locations performed */
  int64_t n_outside;          /* samples outside the hull (zeros, as infinite cells) */
  int64_t n_walk_failures;    /* walks that hit the step limit */
  int64_t n_walk_steps;       /* total walk steps */
  int64_t n_exact_tests;      /* orientation tests resolved by exact arithmetic */
  int64_t n_ties;             /* samples on a shared face/edge/vertex */
} dtfe_status;

/* ---- lifecycle ---------------------------------------------------------- */
int dtfe_gpu_create(const dtfe_config* cfg, dtfe_handle* out);
int dtfe_gpu_destroy(dtfe_handle h);
/* Last error message of this thread (static storage). */
const char* dtfe_last_error(void);

/* Upload a (multi-)tessellation and its vertex data (host arrays).
 * xyz: 3V floats (vertex positions, Particle_data::pos), w: V weights,
 * vel: 3V velocities or NULL, scal: V*S scalars or NULL.  tet_n may be NULL:
 * the device then derives the neighbours from tet_v (the other tetrahedron
 * holding a face's three vertices, -1 on the hull), so only half the arrays
 * cross PCIe.
 * Every tet_v entry must lie in [0, n_verts) and every tet_n entry in
 * [-1, n_tets): a device kernel checks them before anything indexes with
 * them and the call returns DTFE_ERR_ARG (the handle then holds nothing)
 * otherwise.
 * Replaces the CGAL vertex storage filled by vertexData::setData
 * (src/CGAL_triangulation/vertexData.h:45-56). */
int dtfe_gpu_upload(dtfe_handle h, const int32_t* tet_v, const int32_t* tet_n,
                    int64_t n_tets, const float* xyz, const float* w,
                    const float* vel, const float* scal, int64_t n_verts);
/* Same, with the tetrahedra in a packed form (include/dtfe_host.h):
 * dtfe_tets_pack (about 11.5 bytes per tetrahedron instead of 32; a kernel
 * restores tet_v and tet_n) or dtfe_tets_pack_vertices (about 5 bytes; a
 * kernel restores tet_v and the neighbours are derived on the device from
 * the vertices: across each face the other tetrahedron holding its three
 * vertices, -1 on the hull).  A malformed buffer is refused when its header
 * is wrong, else reported by the next status read (DTFE_ERR_ARG) with every
 * bad tetrahedron stored as vertex 0 four times.  No counterpart in the
 * reference (its tessellation never leaves the host). */
int dtfe_gpu_upload_packed(dtfe_handle h, const void* packed, int64_t packed_bytes, const float* xyz,
                           const float* w, const float* vel, const float* scal, int64_t n_verts);
/* Same, with the input particles crossing once instead of one record per
 * padded vertex (a periodic box's padding repeats about a third of its
 * particles): xyz (3 n), w (n), vel (3 n or NULL), scal (S n or NULL) are
 * the n_particles input particles, and vertex_codes holds per vertex its
 * source particle in bits 0-26 and its periodic image in bits 27-31
 * (i1 * 9 + i2 * 3 + i3, i in {0, 1, 2}; 13 = unshifted).  A kernel places
 * vertex v at its particle's position minus (i - 1) * box_length per axis in
 * float, the arithmetic of the padded-box selection (findParticlesInBox,
 * src/subpartition.h:79-154), so the vertices equal the padded set the host
 * tessellated.  At most 2^27 particles (DTFE_ERR_TOO_LARGE); a code out of
 * range is reported by the next status read (DTFE_ERR_ARG).  No counterpart
 * in the reference. */
int dtfe_gpu_upload_packed_particles(dtfe_handle h, const void* packed, int64_t packed_bytes, const float* xyz,
                                     const float* w, const float* vel, const float* scal, int64_t n_particles,
                                     const uint32_t* vertex_codes, int64_t n_verts, const float box_length[3]);
/* Orders uploads between two handles used alternately (double buffering
 * across snapshots): every later upload on h waits until the host->device
 * copies of after's most recent upload have crossed, so the two handles'
 * inputs use the copy engine one after the other instead of sharing it
 * (their kernels and downloads still overlap).  after = NULL removes the
 * link; remove it before destroying `after`.  No counterpart in the
 * reference. */
int dtfe_gpu_chain_uploads(dtfe_handle h, dtfe_handle after);

/* Describe the sub-boxes and the main grid.  xs/ys/zs hold the sample
 * coordinates of every tile along each axis (the reference's running
 * float sums x += dx, unaveraged_interpolation.cc:270-358).  The tile
 * regions default to lo + dx * tile_dims; dtfe_gpu_set_regions gives the
 * exact ones. */
int dtfe_gpu_set_subboxes(dtfe_handle h, int32_t n_boxes, const dtfe_subbox* boxes,
                          const float* xs, int64_t n_xs, const float* ys, int64_t n_ys,
                          const float* zs, int64_t n_zs, const int32_t grid[3]);
/* The region of every sub-box's tile (6 floats per sub-box: xmin, xmax,
 * ymin, ymax, zmin, zmax; the reference's per-thread userOptions.region,
 * src/DTFE.cpp:331-356), after dtfe_gpu_set_subboxes.  Averaging method 1
 * skips tetrahedra whose bounding box misses it
 * (averaged_interpolation_1.cc:67-77).  Each xmin/ymin/zmin must equal the
 * sub-box's lo. */
int dtfe_gpu_set_regions(dtfe_handle h, int32_t n_boxes, const float* regions);

/* Vertex densities rho_v = w_v (D+1) / (rho_bar * sum of incident volumes),
 * 0 on the hull (vertexDensity, triangulation.cpp:200-279).  Each FP64
 * volume is added as an exact integer in units of 2^-62 of its sub-box's
 * vertex bounding-box volume, so the sums do not depend on the order the
 * GPU adds in (the reference adds floats in its incident-cell order). */
int dtfe_gpu_vertex_density(dtfe_handle h, double rho_bar);

/* Interpolate to the grid.  out[slot] receives field `slot` when its bit is
 * set in opts->fields (host pointers, sized grid cells x components).
 * (interpolateGrid, unaveraged_interpolation.cc:209-369;
 *  interpolateGrid_averaged_2/_3, averaged_interpolation_2.cc:35-233,664-866;
 *  computeDivergenceShearVorticity, src/DTFE.cpp:394-475.) */
int dtfe_gpu_interpolate(dtfe_handle h, const dtfe_interp_opts* opts,
                         float* const out[DTFE_NUM_FIELDS], dtfe_status* st);
/* Same, writing into device buffers. */
int dtfe_gpu_interpolate_dev(dtfe_handle h, const dtfe_interp_opts* opts,
                             float* const out_dev[DTFE_NUM_FIELDS], dtfe_status* st);
/* Same as dtfe_gpu_interpolate, but returns once the work and the copies
 * into the host buffers are queued on the handle's stream: the buffers (best
 * pinned) are valid after dtfe_gpu_synchronize; the walk counters come from
 * dtfe_gpu_read_status.  Lets a caller overlap one handle's transfers with
 * another's (double buffering across snapshots). */
int dtfe_gpu_interpolate_async(dtfe_handle h, const dtfe_interp_opts* opts, float* const out[DTFE_NUM_FIELDS]);
/* Fields at user sampling points (interpolateUserSampling,
 * unaveraged_interpolation.cc:560-691; DTFE() runs user samples without the
 * sub-box split, src/DTFE.cpp:301): n points (xyz, 3 floats each, host);
 * those outside region[6] (closed box) are dropped, the rest are located and
 * evaluated as cell centres are (zeros outside the hull), in order.  The
 * handle must hold one sub-box and its vertex densities; opts->method must be
 * DTFE_METHOD_CENTRE.  out[slot] (host) receives *n_out rows of the field's
 * components (size them for n). */
int dtfe_gpu_interpolate_points(dtfe_handle h, int64_t n, const float* xyz, const float region[6],
                                const dtfe_interp_opts* opts, float* const out[DTFE_NUM_FIELDS], int64_t* n_out);
/* Volume averages at user sampling points (interpolateUserSampling_averaged_2,
 * averaged_interpolation_2.cc:470-647; the reference switches any averaged
 * field at user points to this method, src/user_options.cc:962-972): for
 * every point inside region[6], opts->n_samples points
 * float(position + u delta) per axis, u in (-0.5, 0.5) (delta: 3 floats per
 * point, Sample_point::delta), each located and evaluated as a cell centre;
 * the mean over the samples, those outside the hull counted as zeros.
 * opts->method must be DTFE_METHOD_MONTE_CARLO; u comes from Philox4x32-10
 * keyed by opts->seed and counted by (point index, sample), so it is
 * reproducible but not the reference's mt19937 stream.  No velocity
 * standard deviation (the reference computes none here). */
int dtfe_gpu_average_points(dtfe_handle h, int64_t n, const float* xyz, const float* delta, const float region[6],
                            const dtfe_interp_opts* opts, float* const out[DTFE_NUM_FIELDS], int64_t* n_out);
/* Fields on a redshift-cone grid (interpolateRedshiftCone,
 * unaveraged_interpolation.cc:381-547; DTFE() runs cones without the sub-box
 * split, src/DTFE.cpp:301).  cone = (r_min, r_max, theta_min, theta_max,
 * psi_min, psi_max), distances in the particles' units and angles in degrees
 * (User_options::redshiftCone); origin = the cone's apex
 * (User_options::originPosition); dims = bins in r, theta, psi
 * (User_options::gridSize).  Sample (i, j, k) is the centre of its bin,
 * (o0 + r sin(theta) cos(psi), o1 + r sin(theta) sin(psi), o2 + r cos(theta))
 * in the reference's float arithmetic, written to row (i dims[1] + j) dims[2]
 * + k of out[slot] (host, dims[0] dims[1] dims[2] rows); outside the hull
 * zeros.  As in the reference, a sample outside the hull leaves psi where it
 * was, so the rest of its psi row repeats that sample (zeros);
 * DTFE_FLAG_FIX_OUTSIDE_RASTER advances psi regardless.  Theta limits outside
 * [0, 180] or a psi range of 360 degrees or more are refused (DTFE_ERR_ARG,
 * src/user_options.cc:1000-1009).  The handle must hold one sub-box and its
 * vertex densities.  opts->method DTFE_METHOD_CENTRE gives the bin centres;
 * DTFE_METHOD_MONTE_CARLO the bin averages of interpolateRedshiftCone_averaged_2
 * (averaged_interpolation_2.cc:245-466): opts->n_samples points per bin with
 * r, theta, psi each float(centre + u size), u in (-0.5, 0.5) from Philox
 * keyed by opts->seed and counted by (bin, sample), sin and cos of the random
 * angles in double rounded to float; outside points count as zeros; no stuck
 * psi there (the reference's averaged loop has none). */
int dtfe_gpu_interpolate_cone(dtfe_handle h, const float cone[6], const float origin[3], const int32_t dims[3],
                              const dtfe_interp_opts* opts, float* const out[DTFE_NUM_FIELDS]);
/* Same, writing into device buffers (dims[0] dims[1] dims[2] rows each). */
int dtfe_gpu_interpolate_cone_dev(dtfe_handle h, const float cone[6], const float origin[3], const int32_t dims[3],
                                  const dtfe_interp_opts* opts, float* const out_dev[DTFE_NUM_FIELDS]);
/* Particles of a padded box on the device (findParticlesInBox /
 * insertParticlesInBox, src/subpartition.h:79-154; the same selection as
 * dtfe_select_in_box in include/dtfe_host.h, bit for bit): pos_dev holds n
 * positions (3 floats each).  Non-periodic: particles with
 * padded[lo] <= pos <= padded[hi].  Periodic: for each of the 27 translations
 * (i1, i2, i3 over {-1, 0, 1}, offset (i - 1) x box length of full_box) the
 * translated padded box selects particles, emitted shifted back by the
 * offset, translation after translation, in input order within one.
 * *count = the number selected; idx_dev (int32 source indices) and
 * pos_out_dev (shifted positions), when not NULL, receive them if count <=
 * capacity (else DTFE_ERR_TOO_LARGE with *count set, nothing written).
 * n must be below 2^31. */
int dtfe_gpu_select_in_box_dev(dtfe_handle h, const float* pos_dev, int64_t n, const float full_box[6],
                               const float padded[6], int periodic, int32_t* idx_dev, float* pos_out_dev,
                               int64_t capacity, int64_t* count);

/* Writes n_floats floats of device memory (a field in the Quantities layout)
 * to `path` in the reference's binary output format: the raw floats, no
 * header, the file writeBinaryFile (src/io/binary_io.cc:185-216) writes for
 * the same field; name it with dtfe_field_suffix (include/dtfe_host.h) as
 * writeOutputData does.  The copy is ordered after earlier work on the
 * handle's stream and streamed through two pinned buffers (the copy of one
 * chunk overlaps the file write of the previous), so a device-resident field
 * needs no host copy of its own.  DTFE_ERR_IO when the file cannot be opened
 * or fully written. */
int dtfe_gpu_write_binary_dev(dtfe_handle h, const char* path, const float* data_dev, int64_t n_floats);
/* Same as dtfe_gpu_interpolate_dev, but only queues the work on the handle's
 * stream and returns without waiting: consecutive steps (vertex densities,
 * interpolation, ...) then run back to back on the device; the walk counters
 * and a walk failure are reported by dtfe_gpu_read_status. */
int dtfe_gpu_interpolate_dev_async(dtfe_handle h, const dtfe_interp_opts* opts,
                                   float* const out_dev[DTFE_NUM_FIELDS]);

/* ---- NGP / CIC / TSC comparison estimators ------------------------------
 * One record per region (the reference deposits per sub-box region, with
 * stencils clipped at the region's edges): the region's particles are
 * [particle_offset, particle_offset + n_particles) of the particle arrays and
 * its cells are the tile at tile_origin of the main grid. */
typedef struct {
  int64_t particle_offset, n_particles;
  float region[6];          /* xmin, xmax, ymin, ymax, zmin, zmax */
  int32_t tile_origin[3];
  int32_t tile_dims[3];
} dtfe_deposit_box;
enum { DTFE_DEPOSIT_NGP = 0, DTFE_DEPOSIT_CIC = 1, DTFE_DEPOSIT_TSC = 2 };

/* Deposits particle mass and momentum onto the grid and returns density
 * (normalised as the reference: cells / Box::volume() / average_density, with
 * the reference's fixed Box::volume() of 35000^3) and velocity = momentum /
 * mass.  Host arrays: xyz 3n, w n (NULL: unit weights), vel 3n (NULL: no
 * velocity); density (G floats) and velocity (3G floats, may be NULL) are host
 * outputs; cells outside every tile are 0.  Sums are exact (64-bit fixed
 * point) and so independent of thread order.
 * (NGP_interpolation_regular_grid src/NGP_interpolation.cc:67-136,
 *  CIC_interpolation_regular_grid src/CIC_interpolation.cc:67-273,
 *  TSC_interpolation_regular_grid src/TSC_interpolation.cc:67-254.) */
int dtfe_gpu_deposit(dtfe_handle h, int32_t kind, const float* xyz, const float* w, const float* vel,
                     int64_t n, int32_t n_boxes, const dtfe_deposit_box* boxes, const int32_t grid[3],
                     double average_density, float* density, float* velocity);
/* Same with device outputs (density_dev: G floats, velocity_dev: 3G or NULL). */
int dtfe_gpu_deposit_dev(dtfe_handle h, int32_t kind, const float* xyz, const float* w, const float* vel,
                         int64_t n, int32_t n_boxes, const dtfe_deposit_box* boxes, const int32_t grid[3],
                         double average_density, float* density_dev, float* velocity_dev);
/* Same with the particles already on the device as well (xyz_dev 3n floats,
 * w_dev n or NULL, vel_dev 3n or NULL): no host copy at all.  Not in the
 * reference, whose particles live in host memory; for callers that keep
 * their particles resident between steps. */
int dtfe_gpu_deposit_resident(dtfe_handle h, int32_t kind, const float* xyz_dev, const float* w_dev,
                              const float* vel_dev, int64_t n, int32_t n_boxes, const dtfe_deposit_box* boxes,
                              const int32_t grid[3], double average_density, float* density_dev,
                              float* velocity_dev);

/* ---- batched step as one CUDA graph --------------------------------------
 * The reference loops over its sub-boxes (DTFE_parallel, src/DTFE.cpp:
 * 287-385), one thread each.  Here every sub-box of the handle is one range
 * of one launch per kernel; dtfe_gpu_graph_build runs one plain step
 * (vertex densities with rho_bar, seeds, interpolation with *opts into the
 * device buffers out_dev) and then captures the same launches into a CUDA
 * graph; dtfe_gpu_graph_launch replays it on the handle's stream without
 * waiting.  The graph holds the handle's buffers, the launch variants chosen
 * at build time and the out_dev pointers: any later upload or set_subboxes
 * drops it (DTFE_ERR_STATE on launch until rebuilt).  dtfe_gpu_read_status
 * waits for the stream and returns the counters of the last step. */
int dtfe_gpu_graph_build(dtfe_handle h, double rho_bar, const dtfe_interp_opts* opts,
                         float* const out_dev[DTFE_NUM_FIELDS]);
int dtfe_gpu_graph_launch(dtfe_handle h);
int dtfe_gpu_read_status(dtfe_handle h, dtfe_status* status);

/* SPH estimator (SPH_interpolation, src/SPH_interpolation.cc:252-474) on the
 * uploaded vertices and sub-boxes: each sub-box's particles (its vertices,
 * padding included) and grid tile, n_neighbors nearest neighbours (1..128,
 * the particle itself counted), density normalised by average_density.
 * fields: DTFE_FIELD_BIT(DTFE_DENSITY) | DTFE_FIELD_BIT(DTFE_VELOCITY) |
 * DTFE_FIELD_BIT(DTFE_SCALAR); extensive selects the reference's extensive
 * scalar convention.  Host outputs (G, 3G, S*G floats; NULL for fields not
 * asked for).  The reference's float terms, FP64 sums, one rounding. */
int dtfe_gpu_sph(dtfe_handle h, int32_t n_neighbors, uint32_t fields, int32_t extensive, double average_density,
                 float* density, float* velocity, float* scalar);
/* Same with device outputs. */
int dtfe_gpu_sph_dev(dtfe_handle h, int32_t n_neighbors, uint32_t fields, int32_t extensive,
                     double average_density, float* density_dev, float* velocity_dev, float* scalar_dev);

/* ---- adjoints (no counterpart in the reference, which has no gradients) --
 * Gradients of L = sum_c a_c density_c + c_c . velocity_c + b_c divergence_c
 * (the grids of the preceding dtfe_gpu_interpolate* call on the same handle,
 * which must have used DTFE_METHOD_CENTRE) with respect to the vertex
 * positions (3V floats), velocities (3V, may be NULL) and weights (V, may be
 * NULL), at fixed tessellation topology and fixed cell -> tetrahedron
 * assignment.  a = grad_density_dev (G floats), c = grad_velocity_dev (3G),
 * b = grad_divergence_dev (G); each may be NULL (zero).  The velocity value
 * is differentiated as the forward call evaluated it (with or without
 * DTFE_FLAG_FIX_VALUE_INTERP).  All pointers are device pointers.  Vertices
 * that are periodic images of one particle each receive their own share; the
 * particle's gradient is their sum.  DTFE_ERR_STATE without a preceding
 * vertex density and centre interpolation. */
int dtfe_gpu_adjoint_dev(dtfe_handle h, const float* grad_density_dev, const float* grad_velocity_dev,
                         const float* grad_divergence_dev, float* grad_xyz_dev, float* grad_vel_dev,
                         float* grad_w_dev);
/* Gradient of L = sum_c a_c density_c for the density of the last
 * dtfe_gpu_deposit* call on this handle, with respect to that call's particle
 * positions (3n) and weights (n, may be NULL); device pointers. */
int dtfe_gpu_deposit_adjoint_dev(dtfe_handle h, const float* grad_density_dev, float* grad_xyz_dev,
                                 float* grad_w_dev);

/* Autotuner: times each way of locating the cell centres — variants 0..2:
 * every tetrahedron tests the centres inside its bounding box while its
 * volume is computed (the default, 0); variants 3..8: a walk per centre from
 * a seed tetrahedron — with its register budgets, and each register budget
 * of the evaluation kernel, on the loaded data for the cell-centre method
 * and the given field mask (whole steps: volumes, location, evaluation), and
 * keeps the fastest.  All variants locate the same canonical tetrahedra.
 * chosen[0..1] (may be NULL) receive the selected variant indices.  No
 * counterpart in the reference (its loops have no launch parameters). */
int dtfe_gpu_autotune(dtfe_handle h, uint32_t fields, int32_t* chosen);
/* Number of launch variants of the location (counts[0]) and evaluation
 * (counts[1]) kernels that dtfe_gpu_autotune chooses among. */
int dtfe_gpu_variant_counts(int32_t counts[2]);
/* Selects launch variants explicitly (indices as reported by autotune). */
int dtfe_gpu_set_variants(dtfe_handle h, int32_t locate_variant, int32_t eval_variant);

/* Copy the vertex densities (V floats) to the host. */
int dtfe_gpu_download_vertex_density(dtfe_handle h, float* dens);

/* Locate np points (host doubles, 3 per point) with the device walk from
 * tetrahedron `start`; out[i] = canonical tetrahedron id, -1 outside the
 * hull, -2 walk failure.  (dt.locate, unaveraged_interpolation.cc:289.) */
int dtfe_gpu_locate_points(dtfe_handle h, int64_t np, const double* pts, int32_t start,
                           int32_t* out);
/* The tetrahedron each cell centre was located in by the handle's last
 * cell-centre interpolation: loc (host, grid cells) receives per main-grid
 * cell the canonical tetrahedron id (the Cell_handle that dt.locate returns
 * at unaveraged_interpolation.cc:289, as an index into tet_v), -1 for a
 * centre outside the hull (the reference's infinite cell) and for cells
 * outside every tile.  DTFE_ERR_STATE before a cell-centre interpolation. */
int dtfe_gpu_download_located(dtfe_handle h, int32_t* loc);
/* Tile exchange between ranks that split one box (the multi-GPU form of
 * copySubgridResultsToMain, src/subpartition.h:399-432): tiles holds
 * n_tiles records of 6 int32 (origin x, y, z, dims x, y, z) of a grid of
 * grid[0..2] cells; a field has ncomp floats per cell in the Quantities
 * layout.  gather copies the tiles' values out of field_dev into packed_dev,
 * tile after tile (x, y, z order inside a tile); scatter writes a packed
 * buffer back into the tiles of field_dev.  Device pointers, ordered on the
 * handle's stream; the call returns once the copy is done. */
int dtfe_gpu_tiles_gather_dev(dtfe_handle h, int32_t n_tiles, const int32_t* tiles, const int32_t grid[3],
                              int32_t ncomp, const float* field_dev, float* packed_dev);
int dtfe_gpu_tiles_scatter_dev(dtfe_handle h, int32_t n_tiles, const int32_t* tiles, const int32_t grid[3],
                               int32_t ncomp, const float* packed_dev, float* field_dev);
/* Copies the device's tessellation arrays (4 T int32 each, either may be
 * NULL) to the host: after a packed or neighbour-less upload, the restored
 * tet_v and the derived tet_n. */
int dtfe_gpu_download_tets(dtfe_handle h, int32_t* tet_v, int32_t* tet_n);
/* Step limit of every point-location walk (dtfe_config::max_walk_steps;
 * 0 = the default 65536).  A walk that reaches it counts as a failure: its
 * sample gets zeros and the call reports DTFE_ERR_WALK with
 * dtfe_status::n_walk_failures > 0; the handle stays usable.  The reference
 * has no such limit (CGAL's walk has none; its errors exit the process,
 * src/message.h:57-64). */
int dtfe_gpu_set_max_walk_steps(dtfe_handle h, int32_t max_walk_steps);

/* Delaunay tessellation on the device, the counterpart of
 * delaunayTriangulation() (src/CGAL_triangulation/triangulation.cpp:162-195)
 * and of the host tessellator dtfe_tessellate / dtfe_tess_sizes /
 * dtfe_tess_export / dtfe_tess_release (include/dtfe_host.h), whose output
 * it reproduces: n_sets independent float32 point sets, set s being the
 * vertices vprefix[s] .. vprefix[s+1]-1 (host array, vprefix[0] = 0) of the
 * DEVICE array xyz (3 floats per vertex).  Each set gives its finite
 * Delaunay tetrahedra, positively oriented, each in its smallest even vertex
 * rotation, sorted by the Morton key of the FP64 centroid and then by the
 * vertex tuple; vertex ids are global (index into xyz).  stream: a
 * cudaStream_t (NULL = the default stream); the call returns when the
 * tessellation is complete.  Every tetrahedron is certified (empty
 * circumsphere over the whole set, exact predicates).  A set whose certificate
 * meets an exact tie (five co-spherical or four coplanar deciding points,
 * duplicates), a non-finite coordinate or a capacity limit is not
 * tessellated: its status is non-zero (flag bits: 1 tie, 2 capacity,
 * 4 output overflow, 8 certificate repair failed, 16 exact arithmetic out of
 * range, 32 non-finite or flat input) and it has no tetrahedra; the host
 * tessellator, whose insertion order breaks such ties as CGAL's does, is then
 * the one to use for it. */
int dtfe_gpu_tessellate(void* stream, int32_t n_sets, const int64_t* vprefix, const float* xyz, void** tess);
/* tprefix (n_sets+1, may be NULL): tetrahedron offsets of the sets in the
 * exported array; status (n_sets, may be NULL): 0 or the flag bits above. */
int dtfe_gpu_tess_sizes(void* tess, int64_t* tprefix, int32_t* status);
/* Copies the tprefix[n_sets] tetrahedra (4 int32 each) to tet_v: a host
 * pointer, or a device pointer when to_device is non-zero. */
int dtfe_gpu_tess_export(void* tess, int32_t* tet_v, int32_t to_device);
/* Why stars failed, summed over all sets: counts[i] (i < n, up to 12) is
 * the number of vertex stars that met reason i: 0 duplicate point,
 * 1 candidate capacity, 2 star capacity, 3 no start triangle, 4 all points
 * on one plane, 5 exact arithmetic out of range, 6 exact tie, 7 face not
 * Delaunay, 8 inconsistent link, 9 unclosed link, 10 output overflow,
 * 11 more than 64 equal Morton keys; counts[12] is the first vertex whose
 * star failed (global id, -1 if none) and counts[13] its reason. */
int dtfe_gpu_tess_stats(void* tess, int64_t* counts, int32_t n);
int dtfe_gpu_tess_release(void* tess);

/* Vertex densities without any device allocation, for callers that cannot
 * let a library allocate: host applications that hand out all device memory
 * from their own fixed-budget pool, or latency-critical loops where an
 * allocation and the synchronisation it may imply are unacceptable.  No
 * counterpart in the reference (it has no GPU path).
 * Inputs and output are DEVICE pointers on the current device: tet_v/tet_n
 * (4 int32 per tetrahedron, 16-byte aligned), xyz (3 floats per vertex), w
 * (V floats); dens receives V floats: rho_v = w (D+1) / (rho_bar * sum of
 * incident volumes), 0 on the hull (vertexDensity,
 * triangulation.cpp:200-279), with the volumes summed exactly as integers
 * in units of 2^-62 of the vertices' bounding-box volume, so every call
 * gives the same bits, those of dtfe_gpu_vertex_density for the same
 * vertices uploaded as one sub-box.  Scratch
 * is a static device array for at most DTFE_NOALLOC_MAX_VERTS vertices
 * (12 MiB, resident on every device that loads the library until exit);
 * larger inputs return DTFE_ERR_TOO_LARGE.  All calls share that scratch:
 * calls that overlap on the GPU race.  The first call on a device looks up
 * the scratch address; make it before any stream capture.  stream: a
 * cudaStream_t (NULL = default stream); every call returns only after that
 * stream has finished the work (it reads back its range check).  A tet_v
 * entry outside [0, n_verts) returns DTFE_ERR_ARG and leaves dens as it was. */
#define DTFE_NOALLOC_MAX_VERTS (1 << 20)
int dtfe_vertex_density_noalloc(const int32_t* tet_v_dev, const int32_t* tet_n_dev, int64_t n_tets,
                                const float* xyz_dev, const float* w_dev, int64_t n_verts,
                                double rho_bar, float* dens_dev, void* stream);

/* Stream the handle's work is ordered on (a cudaStream_t). */
void* dtfe_gpu_stream(dtfe_handle h);
/* Block until the handle's stream is idle. */
int dtfe_gpu_synchronize(dtfe_handle h);

#ifdef __cplusplus
}
#endif
#endif /* DTFE_GPU_H */
