// DTFE interpolation path on B200 (sm_100a): kernels and the C ABI of
// include/dtfe_gpu.h.
//
// Pipeline (all on the handle's stream):
//   upload              tessellation (plain, packed, or its vertices alone)
//                       and vertex data; k_unpack_tets / k_unpack_tet_vertices
//                       decode packed forms; without neighbours the device
//                       derives them (incidence lists, k_neighbours_star);
//                       k_hull_marks flags the vertices of hull faces (the
//                       reference's infinite cells)
//   k_tet_volume_bins   per step, one thread per tetrahedron: signed FP64
//                       volume added into its vertices' exact sums
//                       (fixed_volume.cuh), and per grid cell the walk seed:
//                       the tetrahedron whose centroid is nearest the cell's
//                       sample point among those whose centroid lies in it
//   k_vertex_density    rho_v = w (D+1)/(rho_bar sum V), 0 on the hull
//                       (vertexDensity, triangulation.cpp:200-279)
//   k_locate_eval       one thread per cell: walk from the seed to the cell
//                       centre (canonical tetrahedron, bit-exact location),
//                       then the reference's per-sample arithmetic and the
//                       divergence/shear/vorticity epilogue, every requested
//                       field written once (k_locate_cells + k_eval_centre:
//                       the same in two kernels)
//   k_average           methods 2/3: n points per cell, each walked from the
//                       centre's tetrahedron (averaged_interpolation_2.cc:123,145)

#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <map>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/dtfe_gpu.h"
#include "dtfe_device.cuh"
#include "fixed_volume.cuh"
#include "philox.h"
#include "tile_index.cuh"

using namespace dtfe;

namespace {

thread_local std::string g_last_error;

int set_error(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

#define DTFE_CUDA_TRY(expr)                                                          \
  do {                                                                               \
    cudaError_t _e = (expr);                                                         \
    if (_e != cudaSuccess)                                                           \
      return set_error(DTFE_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
  } while (0)

constexpr int64_t kMaxCells = 0x7FFFFFFF;  // cell keys are int32
enum { CNT_LOCATED, CNT_OUTSIDE, CNT_FAIL, CNT_STEPS, CNT_EXACT, CNT_TIES, CNT_N };
// after the per-step counters, kept across steps: tetrahedra a packed upload
// could not decode (cleared by every upload); exact orientation tests and
// boundary hits of the centre raster (cleared by every raster)
constexpr int CNT_DECODE = CNT_N;
constexpr int CNT_RASTER_EXACT = CNT_N + 1;
constexpr int CNT_RASTER_TIES = CNT_N + 2;
constexpr int CNT_ALL = CNT_N + 3;

// ---------------------------------------------------------------------------
__global__ void k_pack_xyz(int64_t n, const float* __restrict__ xyz, float4* __restrict__ out, float wval) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = make_float4(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], wval);
}

// Vertices from the input particles: code = source particle (bits 0-26) |
// periodic image (bits 27-31, i1 * 9 + i2 * 3 + i3 with i in {0, 1, 2}); the
// vertex sits at the particle's position minus (i - 1) * box length per
// axis, the float arithmetic of the padded-box selection
// (findParticlesInBox, src/subpartition.h:79-154).  A code outside
// [0, n_src) x [0, 27) counts into *bad and yields particle 0 unshifted.
constexpr uint32_t kSrcBits = 27;
__global__ void k_gather_particles(int64_t V, int S, const uint32_t* __restrict__ codes,
                                   const float* __restrict__ pxyz, const float* __restrict__ pvel,
                                   const float* __restrict__ pw, const float* __restrict__ pscal, int64_t n_src,
                                   float L0, float L1, float L2, float4* __restrict__ posd,
                                   float4* __restrict__ vel4, float* __restrict__ w, float* __restrict__ scal,
                                   unsigned long long* __restrict__ bad) {
  const int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (v >= V) return;
  const uint32_t c = __ldg(&codes[v]);
  int64_t s = c & ((1u << kSrcBits) - 1u);
  int img = (int)(c >> kSrcBits);
  if (s >= n_src || img > 26) {
    atomicAdd(bad, 1ull);
    s = 0;
    img = 13;
  }
  const float o0 = (float)(img / 9 - 1) * L0, o1 = (float)((img / 3) % 3 - 1) * L1, o2 = (float)(img % 3 - 1) * L2;
  posd[v] = make_float4(__ldg(&pxyz[3 * s]) - o0, __ldg(&pxyz[3 * s + 1]) - o1, __ldg(&pxyz[3 * s + 2]) - o2, 0.f);
  vel4[v] = pvel ? make_float4(__ldg(&pvel[3 * s]), __ldg(&pvel[3 * s + 1]), __ldg(&pvel[3 * s + 2]), 0.f)
                 : make_float4(0.f, 0.f, 0.f, 0.f);
  w[v] = __ldg(&pw[s]);
  for (int k = 0; k < S; ++k) scal[v * S + k] = pscal ? __ldg(&pscal[s * S + k]) : 0.f;
}

// Range check of a plain upload before any kernel indexes with it: vertex
// ids in [0, V), neighbour ids (when given) in [-1, T).  Reads only the
// uploaded arrays;
// every tetrahedron out of range counts into *bad.
__global__ void k_check_tets(int64_t T, int64_t V, const int4* __restrict__ tet_v, const int4* __restrict__ tet_n,
                             unsigned long long* __restrict__ bad) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  bool ok = true;
  if (t < T) {
    const int4 v = __ldg(&tet_v[t]);
    const int4 n = tet_n ? __ldg(&tet_n[t]) : make_int4(-1, -1, -1, -1);
    ok = v.x >= 0 && v.x < V && v.y >= 0 && v.y < V && v.z >= 0 && v.z < V && v.w >= 0 && v.w < V &&
         n.x >= -1 && n.x < T && n.y >= -1 && n.y < T && n.z >= -1 && n.z < T && n.w >= -1 && n.w < T;
  }
  const unsigned nbad = __popc(__ballot_sync(0xffffffffu, !ok));
  if ((threadIdx.x & 31) == 0 && nbad) atomicAdd(bad, (unsigned long long)nbad);
}

// Interleaved tetrahedron records for the record walk: rec[2t] = vertices,
// rec[2t+1] = neighbours.
__global__ void k_build_records(int64_t T, const int4* __restrict__ tet_v, const int4* __restrict__ tet_n,
                                int4* __restrict__ rec) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= T) return;
  rec[2 * t] = __ldg(&tet_v[t]);
  rec[2 * t + 1] = __ldg(&tet_n[t]);
}

__global__ void k_hull_marks(int64_t T, const int4* __restrict__ tet_v, const int4* __restrict__ tet_n,
                             int* __restrict__ hull) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= T) return;
  int4 n = __ldg(&tet_n[t]);
  if (n.x >= 0 && n.y >= 0 && n.z >= 0 && n.w >= 0) return;
  int4 v = __ldg(&tet_v[t]);
  if (n.x < 0) { hull[v.y] = 1; hull[v.z] = 1; hull[v.w] = 1; }
  if (n.y < 0) { hull[v.x] = 1; hull[v.z] = 1; hull[v.w] = 1; }
  if (n.z < 0) { hull[v.x] = 1; hull[v.y] = 1; hull[v.w] = 1; }
  if (n.w < 0) { hull[v.x] = 1; hull[v.y] = 1; hull[v.z] = 1; }
}

__device__ __forceinline__ int find_box(const int64_t* __restrict__ prefix, int K, int64_t s) {
  int lo = 0, hi = K;  // prefix[lo] <= s < prefix[hi]
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (__ldg(&prefix[mid]) <= s) lo = mid;
    else hi = mid;
  }
  return lo;
}

// ---- vertex -> tetrahedron incidence (built once per upload) ------------
// Decoder of the packed tessellation (dtfe_tets_pack, host_plan.cpp): one
// thread per tetrahedron, one block per packing block of 256.  The block's
// bytes are staged in shared memory with coalesced 4-byte loads; a block scan
// of the tetrahedra's sizes (8 bytes + one per bit of the flag byte) places
// each thread's fields, a second scan of the escaped fields its first escaped
// value.  Every read is checked against the buffer and every decoded index
// against the vertex and tetrahedron counts: a violation counts into *err
// (reported by the next status read) and stores vertex 0 / no neighbour, so
// that a malformed buffer cannot send later kernels out of range.
constexpr int kPackBlock = 256;
constexpr int kPackMaxBlockBytes = kPackBlock * 16;

// Exclusive block-wide prefix sum of x over kPackBlock threads (all must call).
__device__ __forceinline__ int pack_block_scan(int x, int* s_warp, int* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int inc = x;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= d) inc += y;
  }
  if (lane == 31) s_warp[wid] = inc;
  __syncthreads();
  int before = 0, all = 0;
#pragma unroll
  for (int q = 0; q < kPackBlock / 32; ++q) {
    const int v = s_warp[q];
    before += q < wid ? v : 0;
    all += v;
  }
  if (total) *total = all;
  return before + inc - x;
}

__global__ void __launch_bounds__(kPackBlock)
    k_unpack_tets(int64_t T, int64_t V, const int32_t* __restrict__ base, const int32_t* __restrict__ esc_off,
                  const int64_t* __restrict__ boff, const uint8_t* __restrict__ flags,
                  const uint32_t* __restrict__ data, int64_t data_bytes, const int32_t* __restrict__ esc,
                  int64_t n_esc, int4* __restrict__ tet_v, int4* __restrict__ tet_n, unsigned long long* err) {
  __shared__ uint32_t s_data[kPackMaxBlockBytes / 4 + 2];
  __shared__ int s_scan[2][kPackBlock / 32];
  const int64_t b = blockIdx.x;
  const int64_t t = b * kPackBlock + threadIdx.x;
  const bool valid = t < T;
  const int flag = valid ? (int)__ldg(&flags[t]) : 0;
  const int size = valid ? 8 + __popc(flag) : 0;
  int block_bytes;
  const int off = pack_block_scan(size, s_scan[0], &block_bytes);
  const int64_t b0 = __ldg(&boff[b]), b1 = __ldg(&boff[b + 1]);
  const bool block_ok = b0 >= 0 && b1 - b0 == block_bytes && b1 <= data_bytes;
  // stage the block from the 4-byte word holding its first byte; data_bytes
  // is a multiple of 16, so rounding b1 up to a word stays inside the data
  const int64_t w0 = block_ok ? b0 >> 2 : 0;
  const int nw = block_ok ? (int)(((b1 + 3) >> 2) - w0) : 0;
  for (int i = threadIdx.x; i < nw; i += kPackBlock) s_data[i] = __ldg(&data[w0 + i]);
  __syncthreads();
  // off + size <= block_bytes <= kPackMaxBlockBytes: in s_data even when the
  // block is rejected (its bytes are then unused)
  const uint8_t* sb = (const uint8_t*)s_data + (block_ok ? (b0 & 3) : 0);
  uint32_t raw[8];
  int p = off, ne = 0;
#pragma unroll
  for (int f = 0; f < 8; ++f) {
    const bool wide = (flag >> f) & 1;
    raw[f] = sb[p++];
    if (wide) raw[f] |= (uint32_t)sb[p++] << 8;
    if (f < 4) ne += raw[f] == (wide ? 0xFFFFu : 0xFFu);
    else ne += (wide ? (int)(int16_t)raw[f] : (int)(int8_t)raw[f]) == (wide ? 32767 : 127);
  }
  if (!valid) ne = 0;
  const int e_in = pack_block_scan(ne, s_scan[1], nullptr);
  if (!valid) return;
  const int64_t e0 = (int64_t)__ldg(&esc_off[b]) + e_in;
  bool ok = block_ok && e0 >= 0 && e0 + ne <= n_esc;
  int v[4] = {0, 0, 0, 0}, n[4] = {-1, -1, -1, -1};
  if (ok) {
    const int32_t* e = esc + e0;
    const int32_t b_base = __ldg(&base[b]);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const bool wide = (flag >> k) & 1;
      const bool escaped = raw[k] == (wide ? 0xFFFFu : 0xFFu);
      v[k] = escaped ? __ldg(e++) : (k ? v[0] : b_base) + (int)raw[k];
      ok = ok && v[k] >= 0 && v[k] < V;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const bool wide = (flag >> (4 + k)) & 1;
      const int sv = wide ? (int)(int16_t)raw[4 + k] : (int)(int8_t)raw[4 + k];
      const int lo = wide ? -32768 : -128, hi = wide ? 32767 : 127;
      const int64_t m = sv == lo ? -1 : (sv == hi ? (int64_t)__ldg(e++) : t + sv);
      ok = ok && m >= -1 && m < T;
      n[k] = (int)m;
    }
  }
  if (!ok) {
    atomicAdd(err, 1ull);
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = 0, n[k] = -1;
  }
  tet_v[t] = make_int4(v[0], v[1], v[2], v[3]);
  tet_n[t] = make_int4(n[0], n[1], n[2], n[3]);
}

// Decoder of the vertex-only packed tessellation (dtfe_tets_pack_vertices,
// host_plan.cpp), laid out as k_unpack_tets: one thread per tetrahedron, one
// block per packing block of 256, the block's bytes staged in shared memory.
// Block scans place each thread's fields (4 bytes + one per bit of its width
// nibble) and its first escape, and a third scan adds up the first-vertex
// differences from the block's base.  Every read is checked against the
// buffer and every vertex against [0, V) and the canonical order (first
// vertex smallest, second smallest of the rest); a violation counts into
// *err and stores vertex 0 four times, so later kernels stay in range.
__global__ void __launch_bounds__(kPackBlock)
    k_unpack_tet_vertices(int64_t T, int64_t V, const int32_t* __restrict__ base, const int32_t* __restrict__ esc_off,
                          const int64_t* __restrict__ boff, const uint8_t* __restrict__ flags,
                          const uint8_t* __restrict__ orient, const uint32_t* __restrict__ data, int64_t data_bytes,
                          const int32_t* __restrict__ esc, int64_t n_esc, int4* __restrict__ tet_v,
                          unsigned long long* err) {
  __shared__ uint32_t s_data[kPackMaxBlockBytes / 4 + 2];
  __shared__ int s_scan[3][kPackBlock / 32];
  const int64_t b = blockIdx.x;
  const int64_t t = b * kPackBlock + threadIdx.x;
  const bool valid = t < T;
  const int flag = valid ? ((int)__ldg(&flags[t >> 1]) >> ((t & 1) * 4)) & 15 : 0;
  const int size = valid ? 4 + __popc(flag) : 0;
  int block_bytes;
  const int off = pack_block_scan(size, s_scan[0], &block_bytes);
  const int64_t b0 = __ldg(&boff[b]), b1 = __ldg(&boff[b + 1]);
  const bool block_ok = b0 >= 0 && b1 - b0 == block_bytes && b1 <= data_bytes;
  const int64_t w0 = block_ok ? b0 >> 2 : 0;
  const int nw = block_ok ? (int)(((b1 + 3) >> 2) - w0) : 0;
  for (int i = threadIdx.x; i < nw; i += kPackBlock) s_data[i] = __ldg(&data[w0 + i]);
  __syncthreads();
  const uint8_t* sb = (const uint8_t*)s_data + (block_ok ? (b0 & 3) : 0);
  uint32_t raw[4];
  int p = off, ne = 0;
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    const bool wide = (flag >> f) & 1;
    raw[f] = sb[p++];
    if (wide) raw[f] |= (uint32_t)sb[p++] << 8;
    if (f == 0) ne += (wide ? (int)(int16_t)raw[0] : (int)(int8_t)raw[0]) == (wide ? 32767 : 127);
    else ne += raw[f] == (wide ? 0xFFFFu : 0xFFu);
  }
  if (!valid) ne = 0;
  const int e_in = pack_block_scan(ne, s_scan[1], nullptr);
  const int64_t e0 = (int64_t)__ldg(&esc_off[b]) + e_in;
  bool ok = block_ok && e0 >= 0 && e0 + ne <= n_esc;
  const int32_t* e = esc + (ok ? e0 : 0);
  int d[4] = {0, 0, 0, 0};
  if (valid && ok) {
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      const bool wide = (flag >> f) & 1;
      if (f == 0) {
        const int sv = wide ? (int)(int16_t)raw[0] : (int)(int8_t)raw[0];
        d[0] = sv == (wide ? 32767 : 127) ? __ldg(e++) : sv;
      } else {
        d[f] = raw[f] == (wide ? 0xFFFFu : 0xFFu) ? __ldg(e++) : (int)raw[f];
      }
    }
  }
  // first vertex: the block's base plus the differences up to this tetrahedron
  const int before = pack_block_scan(d[0], s_scan[2], nullptr);
  if (!valid) return;
  const int64_t v0 = (int64_t)__ldg(&base[b]) + before + d[0];
  const int64_t v1 = v0 + d[1], lo = v1 + d[2], hi = lo + d[3];
  ok = ok && v0 >= 0 && d[1] > 0 && d[2] > 0 && d[3] > 0 && hi < V;
  if (!ok) {
    atomicAdd(err, 1ull);
    tet_v[t] = make_int4(0, 0, 0, 0);
    return;
  }
  const bool third_larger = (__ldg(&orient[t >> 3]) >> (t & 7)) & 1;
  tet_v[t] = make_int4((int)v0, (int)v1, (int)(third_larger ? hi : lo), (int)(third_larger ? lo : hi));
}

__device__ __forceinline__ bool holds(const int4& u, int v) { return u.x == v || u.y == v || u.z == v || u.w == v; }

// Fallback for the faces k_neighbours_star left unset (kUnsetNeighbour):
// across face (a, b, c) of t lies the other tetrahedron of the list of the
// face's smallest vertex that holds all three (-1 if none: the convex hull,
// CGAL's infinite cell).  Any list order will do.  A tetrahedron holding the
// face has its smallest vertex as its own smallest or second smallest, so
// the star lists (k_fill_star) hold it.
constexpr int kUnsetNeighbour = (int)0x80808080;  // the byte pattern 0x80 of a memset
__device__ __forceinline__ int face_neighbour(int t, int a, int b, int c, const int64_t* __restrict__ off,
                                              const int* __restrict__ inc, const int4* __restrict__ tet_v) {
  const int m = min(a, min(b, c));
  for (int64_t i = __ldg(&off[m]), e = __ldg(&off[m + 1]); i < e; ++i) {
    const int u = __ldg(&inc[i]);
    if (u == t) continue;
    const int4 q = __ldg(&tet_v[u]);
    if (holds(q, a) && holds(q, b) && holds(q, c)) return u;
  }
  return -1;
}

__global__ void k_derive_neighbours(int64_t T, const int4* __restrict__ tet_v, const int64_t* __restrict__ off,
                                    const int* __restrict__ inc, int4* __restrict__ tet_n) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= T) return;
  int4 cur = tet_n[t];
  if (cur.x != kUnsetNeighbour && cur.y != kUnsetNeighbour && cur.z != kUnsetNeighbour &&
      cur.w != kUnsetNeighbour)
    return;
  const int4 q = __ldg(&tet_v[t]);
  if (cur.x == kUnsetNeighbour) cur.x = face_neighbour((int)t, q.y, q.z, q.w, off, inc, tet_v);
  if (cur.y == kUnsetNeighbour) cur.y = face_neighbour((int)t, q.x, q.z, q.w, off, inc, tet_v);
  if (cur.z == kUnsetNeighbour) cur.z = face_neighbour((int)t, q.x, q.y, q.w, off, inc, tet_v);
  if (cur.w == kUnsetNeighbour) cur.w = face_neighbour((int)t, q.x, q.y, q.z, off, inc, tet_v);
  tet_n[t] = cur;
}

// Neighbours from the stars of the vertices: every face is settled at its
// smallest vertex v, by the one warp that reads v's star list (the
// tetrahedra whose smallest or second smallest vertex is v, k_fill_star:
// only these have a face whose smallest vertex is v).  Each listed
// tetrahedron contributes its faces through v whose other two vertices are
// larger than v, keyed by those two vertices; the two entries with the same
// key are the tetrahedra on either side (one entry alone: a hull face, -1).
// The entries of one vertex sit in its group's shared table.  A first pass
// gives each vertex a group of 8 lanes (four vertices' dependent loads --
// list offsets, list, tetrahedra -- in flight per warp) and a table of 96
// entries; the few vertices with more (about 0.1% of a Zel'dovich
// tessellation) are listed and settled by a second pass with a warp and 768
// entries each; faces of larger stars stay unset for k_derive_neighbours.
// Each tetrahedron's vertices are read twice.
//   FROM_LIST = false: every vertex v < V; stars above CAP are appended to
//                      list (count in *n_list, at most list_cap kept).
//   FROM_LIST = true:  the listed vertices.
//   HASH: the two entries of a face are paired through a shared hash table
//         of 2 CAP slots (one atomicCAS per entry) instead of every entry
//         scanning the table (n^2 compares per vertex).
template <int THREADS, int LANES, int CAP, bool FROM_LIST, bool HASH>
__global__ void __launch_bounds__(THREADS) k_neighbours_star(int64_t V, const int4* __restrict__ tet_v,
                                                            const int64_t* __restrict__ off,
                                                            const int* __restrict__ inc, int* __restrict__ tet_n,
                                                            int* __restrict__ list, unsigned* __restrict__ n_list,
                                                            unsigned list_cap) {
  constexpr int kGroups = THREADS / LANES;
  constexpr int H = HASH ? 2 * CAP : 1;  // hash slots, a power of two
  static_assert(!HASH || (CAP & (CAP - 1)) == 0, "hash table size must be a power of two");
  __shared__ unsigned long long s_key[kGroups][CAP];
  __shared__ int s_tet[kGroups][CAP];
  __shared__ unsigned char s_face[kGroups][CAP];
  __shared__ unsigned long long s_hkey[kGroups][H];  // 0: empty (a key is never 0: hi > lo >= 0)
  __shared__ unsigned char s_hidx[kGroups][H];       // the first entry of the slot's key
  __shared__ unsigned char s_state[kGroups][CAP];    // 0 first and unpaired, 1 first and paired,
                                                     // 2 + slot: second entry
  const int g = threadIdx.x / LANES, gl = threadIdx.x % LANES;
  if (HASH) {
    for (int k = gl; k < H; k += LANES) s_hkey[g][k] = 0ull;
  }
  const unsigned gmask = LANES == 32 ? 0xffffffffu
                                     : ((1u << (LANES & 31)) - 1u) << ((threadIdx.x & 31) & ~(LANES - 1));
  unsigned long long* key = s_key[g];
  int* tet = s_tet[g];
  unsigned char* face = s_face[g];
  const int64_t n_items = FROM_LIST ? (int64_t)min(*n_list, list_cap) : V;
  for (int64_t it = (int64_t)blockIdx.x * kGroups + g; it < n_items; it += (int64_t)gridDim.x * kGroups) {
    const int64_t v = FROM_LIST ? (int64_t)__ldg(&list[it]) : it;
    const int64_t a = __ldg(&off[v]), e = __ldg(&off[v + 1]);
    int n = 0;  // entries so far (uniform in the group)
    for (int64_t base = a; base < e; base += LANES) {
      const int64_t q = base + gl;
      int cnt = 0, u = -1;
      unsigned long long k3[3];
      int f3[3];
      if (q < e) {
        u = __ldg(&inc[q]);
        const int4 tv = __ldg(&tet_v[u]);
        const int vv[4] = {tv.x, tv.y, tv.z, tv.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          if (vv[k] == (int)v) continue;  // the face opposite v does not hold v
          int x = -1, y = -1;
#pragma unroll
          for (int m = 0; m < 4; ++m)
            if (m != k && vv[m] != (int)v) {
              if (x < 0) x = vv[m];
              else y = vv[m];
            }
          if (x > (int)v && y > (int)v) {
            const unsigned lo = (unsigned)min(x, y), hi = (unsigned)max(x, y);
            const unsigned long long kk = ((unsigned long long)lo << 32) | hi;
            // constant indices keep k3 / f3 in registers
            if (cnt == 0) { k3[0] = kk; f3[0] = k; }
            else if (cnt == 1) { k3[1] = kk; f3[1] = k; }
            else { k3[2] = kk; f3[2] = k; }
            ++cnt;
          }
        }
      }
      int incl = cnt;
#pragma unroll
      for (int d = 1; d < LANES; d <<= 1) {
        const int y = __shfl_up_sync(gmask, incl, d, LANES);
        if (gl >= d) incl += y;
      }
      const int pos = n + incl - cnt;
#pragma unroll
      for (int c = 0; c < 3; ++c)
        if (c < cnt && pos + c < CAP) {
          key[pos + c] = k3[c];
          tet[pos + c] = u;
          face[pos + c] = (unsigned char)f3[c];
        }
      n += __shfl_sync(gmask, incl, LANES - 1, LANES);
    }
    __syncwarp(gmask);
    if (n > CAP) {
      if (!FROM_LIST && gl == 0) {
        const unsigned slot = atomicAdd(n_list, 1u);
        if (slot < list_cap) list[slot] = (int)v;
      }
    } else if (HASH) {
      unsigned long long* hk = s_hkey[g];
      unsigned char* hi = s_hidx[g];
      unsigned char* st = s_state[g];
      // insert: the first entry of a key claims a slot, the second finds it
      for (int j = gl; j < n; j += LANES) {
        const unsigned long long kj = key[j];
        unsigned h = ((unsigned)kj * 0x9E3779B1u ^ (unsigned)(kj >> 32) * 0x85EBCA77u) & (H - 1);
        unsigned char state = 0;
        for (int probe = 0; probe < H; ++probe) {
          const unsigned long long old = atomicCAS(&hk[h], 0ull, kj);
          if (old == 0ull) {
            hi[h] = (unsigned char)j;
            break;
          }
          if (old == kj) {
            state = (unsigned char)(2 + h);
            break;
          }
          h = (h + 1) & (H - 1);
        }
        st[j] = state;
      }
      __syncwarp(gmask);
      // pair: each second entry links itself and the first one
      for (int j = gl; j < n; j += LANES) {
        if (st[j] < 2) continue;
        const int f = hi[st[j] - 2];
        tet_n[4 * (int64_t)tet[j] + face[j]] = tet[f];
        tet_n[4 * (int64_t)tet[f] + face[f]] = tet[j];
        st[f] = 1;
      }
      __syncwarp(gmask);
      // unpaired first entries lie on the hull; then empty the table
      for (int j = gl; j < n; j += LANES)
        if (st[j] == 0) tet_n[4 * (int64_t)tet[j] + face[j]] = -1;
      for (int k = gl; k < H; k += LANES) hk[k] = 0ull;
    } else {
      for (int j = gl; j < n; j += LANES) {
        const unsigned long long kj = key[j];
        int partner = -1;
        for (int i = 0; i < n; ++i)
          if (i != j && key[i] == kj) {
            partner = tet[i];
            break;
          }
        tet_n[4 * (int64_t)tet[j] + face[j]] = partner;
      }
    }
    __syncwarp(gmask);
  }
}

// The two smallest of a tetrahedron's four vertex ids (a < b).
__device__ __forceinline__ void two_smallest(const int4& q, int& a, int& b) {
  const int lo1 = min(q.x, q.y), hi1 = max(q.x, q.y), lo2 = min(q.z, q.w), hi2 = max(q.z, q.w);
  a = min(lo1, lo2);
  b = min(max(lo1, lo2), min(hi1, hi2));
}

// Star lists: each tetrahedron at its smallest and second smallest vertex.
__global__ void k_degree_star(int64_t T, const int4* __restrict__ tet_v, int* __restrict__ deg) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= T) return;
  int a, b;
  two_smallest(__ldg(&tet_v[t]), a, b);
  atomicAdd(&deg[a], 1);
  atomicAdd(&deg[b], 1);
}

__global__ void k_fill_star(int64_t T, const int4* __restrict__ tet_v, const int64_t* __restrict__ off,
                            int* __restrict__ cursor, int* __restrict__ inc) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= T) return;
  int a, b;
  two_smallest(__ldg(&tet_v[t]), a, b);
  inc[__ldg(&off[a]) + atomicAdd(&cursor[a], 1)] = (int)t;
  inc[__ldg(&off[b]) + atomicAdd(&cursor[b], 1)] = (int)t;
}

__global__ void k_degree(int64_t T, const int4* __restrict__ tet_v, int* __restrict__ deg) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= T) return;
  int4 v = __ldg(&tet_v[t]);
  atomicAdd(&deg[v.x], 1);
  atomicAdd(&deg[v.y], 1);
  atomicAdd(&deg[v.z], 1);
  atomicAdd(&deg[v.w], 1);
}

// Exclusive scan of n ints into int64 offsets (out has n+1 entries):
// per-block scans of kScanBlock items, a single-block scan of the block
// totals, then the block offsets are added.
constexpr int kScanBlock = 1024;
__global__ void k_scan_blocks(int64_t n, const int* __restrict__ in, int64_t* __restrict__ out,
                              int64_t* __restrict__ block_sums) {
  __shared__ int64_t sh[kScanBlock];
  int64_t i = blockIdx.x * (int64_t)kScanBlock + threadIdx.x;
  int64_t x = i < n ? (int64_t)in[i] : 0;
  sh[threadIdx.x] = x;
  __syncthreads();
  for (int off = 1; off < kScanBlock; off <<= 1) {
    int64_t y = threadIdx.x >= off ? sh[threadIdx.x - off] : 0;
    __syncthreads();
    sh[threadIdx.x] += y;
    __syncthreads();
  }
  if (i < n) out[i] = sh[threadIdx.x] - x;  // exclusive
  if (threadIdx.x == kScanBlock - 1) block_sums[blockIdx.x] = sh[threadIdx.x];
}

__global__ void k_scan_totals(int64_t nb, int64_t* __restrict__ block_sums, int64_t* __restrict__ total) {
  // one block: sequential chunks, each scanned in shared memory
  __shared__ int64_t sh[kScanBlock];
  int64_t carry = 0;
  for (int64_t base = 0; base < nb; base += kScanBlock) {
    int64_t i = base + threadIdx.x;
    int64_t x = i < nb ? block_sums[i] : 0;
    sh[threadIdx.x] = x;
    __syncthreads();
    for (int off = 1; off < kScanBlock; off <<= 1) {
      int64_t y = threadIdx.x >= off ? sh[threadIdx.x - off] : 0;
      __syncthreads();
      sh[threadIdx.x] += y;
      __syncthreads();
    }
    if (i < nb) block_sums[i] = carry + sh[threadIdx.x] - x;
    int64_t tot = sh[kScanBlock - 1];
    __syncthreads();
    carry += tot;
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void k_scan_add(int64_t n, int64_t* __restrict__ out, const int64_t* __restrict__ block_sums) {
  int64_t i = blockIdx.x * (int64_t)kScanBlock + threadIdx.x;
  if (i < n) out[i] += block_sums[blockIdx.x];
}

__global__ void k_fill_incidence(int64_t T, const int4* __restrict__ tet_v, const int64_t* __restrict__ off,
                                 int* __restrict__ cursor, int* __restrict__ inc) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= T) return;
  int4 q = __ldg(&tet_v[t]);
  int v[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    int pos = atomicAdd(&cursor[v[a]], 1);
    inc[off[v[a]] + pos] = (int)t;
  }
}

// ---- per step ------------------------------------------------------------
constexpr int kVolBlock = 64;  // 64: 5.67 ms per 256^3 step; 128: 5.70; 256: 5.77; 512: 6.21

// Signed volume of every tetrahedron (FP64, streamed out once) and, when
// DO_BINS, the walk seeds: per grid cell, among the tetrahedra whose
// centroid lies in the cell, the one whose centroid is nearest the cell's
// sample point (squared distance in float, ties to the lower id), kept as
// (distance bits << 32 | id) by a 64-bit atomicMin.  Tetrahedra are
// Morton-sorted, so neighbouring lanes often bin to the same cell: a
// segmented minimum over each run of equal cells in the warp leaves one
// atomic per run.  The seed only starts the walk (the located tetrahedron
// does not depend on it), so the centroid's cell uses a fast approximate
// division (the range checks keep the index in the tile).
// Per-vertex volume sums in exact integer units (fixed_volume.cuh): the
// scale of each tetrahedron's sub-box (tprefix: nsb + 1 tetrahedron range
// starts), one reduction per vertex.
struct VolSums {
  long long* acc;
  const VolScale* scale;
  const int64_t* tprefix;
  int nsb;
};
__device__ __forceinline__ void add_volume(const VolSums& S, int64_t t, const int v[4], double vol) {
  const int b = S.nsb > 1 ? find_box(S.tprefix, S.nsb, t) : 0;
  const unsigned long long q = (unsigned long long)__double2ll_rn(vol * S.scale[b].inv_q);
#pragma unroll
  for (int a = 0; a < 4; ++a) atomicAdd((unsigned long long*)&S.acc[v[a]], q);
}

constexpr unsigned long long kEmptySeed = ~0ull;
constexpr int kVolTPT = 2;  // tetrahedra per thread of the step's volume kernel (4: slower)
template <bool DO_BINS>
__global__ void __launch_bounds__(kVolBlock) k_tet_volume_bins(
    int64_t T, const int4* __restrict__ tet_v, const float4* __restrict__ posd, VolSums VS,
    const dtfe_subbox* __restrict__ boxes, const int64_t* __restrict__ tprefix,
    const int64_t* __restrict__ bin_offset, int K, const float* __restrict__ xs, const float* __restrict__ ys,
    const float* __restrict__ zs, unsigned long long* __restrict__ bins) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int key = -1;
  unsigned long long val = kEmptySeed;
  if (t < T) {
    int4 q = __ldg(&tet_v[t]);
    int v[4] = {q.x, q.y, q.z, q.w};
    float X[4][3];
#pragma unroll
    for (int a = 0; a < 4; ++a) load_posf(posd, v[a], X[a]);
    double D[4][3];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int c = 0; c < 3; ++c) D[a][c] = (double)X[a][c];
    add_volume(VS, t, v, orient_det(D[0], D[1], D[2], D[3]) / 6.0);
    if (DO_BINS) {
      const int b = find_box(tprefix, K, t);
      const dtfe_subbox& B = boxes[b];
      int idx[3];
      float cen[3];
      bool inside = true;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        cen[c] = 0.25f * ((X[0][c] + X[1][c]) + (X[2][c] + X[3][c]));
        const float f = floorf(__fdividef(cen[c] - __ldg(&B.lo[c]), __ldg(&B.dx[c])));
        const int n = __ldg(&B.tile_dims[c]);
        inside = inside && (f >= 0.f && f < (float)n);
        idx[c] = inside ? (int)f : 0;
      }
      if (inside) {
        key = (int)(__ldg(&bin_offset[b]) +
                    ((int64_t)idx[0] * __ldg(&B.tile_dims[1]) + idx[1]) * __ldg(&B.tile_dims[2]) + idx[2]);
        const float dxs = cen[0] - __ldg(&xs[B.coord_offset[0] + idx[0]]);
        const float dys = cen[1] - __ldg(&ys[B.coord_offset[1] + idx[1]]);
        const float dzs = cen[2] - __ldg(&zs[B.coord_offset[2] + idx[2]]);
        const float d2 = dxs * dxs + dys * dys + dzs * dzs;
        val = ((unsigned long long)__float_as_uint(d2) << 32) | (unsigned)t;
      }
    }
  }
  if (DO_BINS) {
    // segmented minimum over runs of equal keys; the run's first lane issues
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long ov = __shfl_down_sync(0xffffffffu, val, o);
      const int ok = __shfl_down_sync(0xffffffffu, key, o);
      if (lane + o < 32 && ok == key && ov < val) val = ov;
    }
    const int prev = __shfl_up_sync(0xffffffffu, key, 1);
    if (key >= 0 && (lane == 0 || prev != key)) atomicMin(&bins[key], val);
  }
}

// k_tet_volume_bins<true> with TPT tetrahedra per thread: a warp takes
// 32 TPT consecutive tetrahedra, lane l the l-th, (32 + l)-th, ..., and issues
// all their records' loads, then all their position gathers, before any
// arithmetic, so TPT times the gathers are in flight per thread.
template <int TPT>
__global__ void __launch_bounds__(kVolBlock) k_tet_volume_bins2(
    int64_t T, const int4* __restrict__ tet_v, const float4* __restrict__ posd, VolSums VS,
    const dtfe_subbox* __restrict__ boxes, const int64_t* __restrict__ tprefix,
    const int64_t* __restrict__ bin_offset, int K, const float* __restrict__ xs, const float* __restrict__ ys,
    const float* __restrict__ zs, unsigned long long* __restrict__ bins) {
  const int lane = threadIdx.x & 31;
  const int64_t base = ((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5) * (32 * TPT);
  int4 q[TPT];
#pragma unroll
  for (int r = 0; r < TPT; ++r) {
    const int64_t t = base + 32 * r + lane;
    q[r] = t < T ? __ldg(&tet_v[t]) : make_int4(0, 0, 0, 0);
  }
  float X[TPT][4][3];
#pragma unroll
  for (int r = 0; r < TPT; ++r) {
    const int v[4] = {q[r].x, q[r].y, q[r].z, q[r].w};
#pragma unroll
    for (int a = 0; a < 4; ++a) load_posf(posd, v[a], X[r][a]);
  }
#pragma unroll
  for (int r = 0; r < TPT; ++r) {
    const int64_t t = base + 32 * r + lane;
    int key = -1;
    unsigned long long val = kEmptySeed;
    if (t < T) {
      const int v[4] = {q[r].x, q[r].y, q[r].z, q[r].w};
      double D[4][3];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) D[a][c] = (double)X[r][a][c];
      add_volume(VS, t, v, orient_det(D[0], D[1], D[2], D[3]) / 6.0);
      const int b = find_box(tprefix, K, t);
      const dtfe_subbox& B = boxes[b];
      int idx[3];
      float cen[3];
      bool inside = true;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        cen[c] = 0.25f * ((X[r][0][c] + X[r][1][c]) + (X[r][2][c] + X[r][3][c]));
        const float f = floorf(__fdividef(cen[c] - __ldg(&B.lo[c]), __ldg(&B.dx[c])));
        const int n = __ldg(&B.tile_dims[c]);
        inside = inside && (f >= 0.f && f < (float)n);
        idx[c] = inside ? (int)f : 0;
      }
      if (inside) {
        key = (int)(__ldg(&bin_offset[b]) +
                    ((int64_t)idx[0] * __ldg(&B.tile_dims[1]) + idx[1]) * __ldg(&B.tile_dims[2]) + idx[2]);
        const float dxs = cen[0] - __ldg(&xs[B.coord_offset[0] + idx[0]]);
        const float dys = cen[1] - __ldg(&ys[B.coord_offset[1] + idx[1]]);
        const float dzs = cen[2] - __ldg(&zs[B.coord_offset[2] + idx[2]]);
        const float d2 = dxs * dxs + dys * dys + dzs * dzs;
        val = ((unsigned long long)__float_as_uint(d2) << 32) | (unsigned)t;
      }
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long ov = __shfl_down_sync(0xffffffffu, val, o);
      const int ok = __shfl_down_sync(0xffffffffu, key, o);
      if (lane + o < 32 && ok == key && ov < val) val = ov;
    }
    const int prev = __shfl_up_sync(0xffffffffu, key, 1);
    if (key >= 0 && (lane == 0 || prev != key)) atomicMin(&bins[key], val);
  }
}

// Signed FP64 volume of every tetrahedron (as k_tet_volume_bins) and the
// location of every cell centre, without a walk: a centre lies in the closure
// of a tetrahedron only inside its bounding box, so each thread finds the
// centres of its sub-box's tile in its box (index ranges from the tile's
// raster formula x_i = lo + (i + 1/2) dx, widened by the largest deviation of
// the coordinate tables from it, measured on the host: conservative), the
// block scans its threads' counts and its 256 threads test the block's
// candidates in turn (owner by binary search over the scan) with the exact
// orientation predicates.  Every tetrahedron whose closure holds the centre
// takes part in an atomicMin on its slot (preset to 0xFFFFFFFF = outside),
// which leaves the lowest such id: the canonical tie rule.
constexpr int kRasterBlock = 256;
struct RasterAxis {
  double lo, inv_dx, margin;
};
template <int MINB>
__global__ void __launch_bounds__(kRasterBlock, MINB) k_tet_volume_raster(
    int64_t T, const int4* __restrict__ tet_v, const float4* __restrict__ posd, VolSums VS,
    const dtfe_subbox* __restrict__ boxes, const int64_t* __restrict__ tprefix,
    const int64_t* __restrict__ tile_prefix, const RasterAxis* __restrict__ axes, int K,
    const float* __restrict__ xs, const float* __restrict__ ys, const float* __restrict__ zs,
    unsigned* __restrict__ tet_c, unsigned long long* __restrict__ counters) {
  __shared__ float s_X[kRasterBlock][13];
  __shared__ int s_meta[kRasterBlock][7];  // i0, j0, k0, nj, nk, box, tetrahedron
  __shared__ long long s_scan[kRasterBlock];
  __shared__ long long s_warp[kRasterBlock / 32];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int64_t t = blockIdx.x * (int64_t)kRasterBlock + tid;
  long long cnt = 0;
  if (t < T) {
    int4 q = __ldg(&tet_v[t]);
    int v[4] = {q.x, q.y, q.z, q.w};
    float X[4][3];
#pragma unroll
    for (int a = 0; a < 4; ++a) load_posf(posd, v[a], X[a]);
    double D[4][3];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int c = 0; c < 3; ++c) D[a][c] = (double)X[a][c];
    add_volume(VS, t, v, orient_det(D[0], D[1], D[2], D[3]) / 6.0);
    if (t >= __ldg(&tprefix[0]) && t < __ldg(&tprefix[K])) {
      const int b = find_box(tprefix, K, t);
      int r0[3], nr[3];
      cnt = 1;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float lo = fminf(fminf(X[0][c], X[1][c]), fminf(X[2][c], X[3][c]));
        const float hi = fmaxf(fmaxf(X[0][c], X[1][c]), fmaxf(X[2][c], X[3][c]));
        const RasterAxis A = axes[3 * b + c];
        const double n = (double)__ldg(&boxes[b].tile_dims[c]);
        const double f0 = fmax(ceil(((double)lo - A.lo) * A.inv_dx - 0.5 - A.margin), 0.0);
        const double f1 = fmin(floor(((double)hi - A.lo) * A.inv_dx - 0.5 + A.margin), n - 1.0);
        r0[c] = f1 >= f0 ? (int)f0 : 0;
        nr[c] = f1 >= f0 ? (int)(f1 - f0) + 1 : 0;
        cnt *= nr[c];
      }
      if (cnt) {
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int c = 0; c < 3; ++c) s_X[tid][3 * a + c] = X[a][c];
        s_meta[tid][0] = r0[0];
        s_meta[tid][1] = r0[1];
        s_meta[tid][2] = r0[2];
        s_meta[tid][3] = nr[1];
        s_meta[tid][4] = nr[2];
        s_meta[tid][5] = b;
        s_meta[tid][6] = (int)t;
      }
    }
  }
  // inclusive block scan of the candidate counts
  long long inc = cnt;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const long long y = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= d) inc += y;
  }
  if (lane == 31) s_warp[wid] = inc;
  __syncthreads();
  long long before = 0;
#pragma unroll
  for (int w = 0; w < kRasterBlock / 32; ++w) before += w < wid ? s_warp[w] : 0;
  s_scan[tid] = before + inc;
  __syncthreads();
  const long long total = s_scan[kRasterBlock - 1];
  int nexact = 0, nties = 0;
  for (long long qi = tid; qi < total; qi += kRasterBlock) {
    int lo = 0, hi = kRasterBlock - 1;  // first owner with s_scan > qi
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (s_scan[mid] > qi) hi = mid;
      else lo = mid + 1;
    }
    const int o = lo;
    const int local = (int)(qi - (o ? s_scan[o - 1] : 0));
    const int nj = s_meta[o][3], nk = s_meta[o][4], b = s_meta[o][5];
    const int k = s_meta[o][2] + local % nk;
    const int j = s_meta[o][1] + (local / nk) % nj;
    const int i = s_meta[o][0] + local / (nk * nj);
    const dtfe_subbox& B = boxes[b];
    const float pf[3] = {__ldg(&xs[B.coord_offset[0] + i]), __ldg(&ys[B.coord_offset[1] + j]),
                         __ldg(&zs[B.coord_offset[2] + k])};
    float X[4][3];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int c = 0; c < 3; ++c) X[a][c] = s_X[o][3 * a + c];
    int zmask;
    if (first_exit_face_f32(X, pf, 15, zmask, nexact) < 0) {
      const int64_t slot =
          __ldg(&tile_prefix[b]) + ((int64_t)i * __ldg(&B.tile_dims[1]) + j) * __ldg(&B.tile_dims[2]) + k;
      atomicMin(&tet_c[slot], (unsigned)s_meta[o][6]);
      nties += zmask != 0;
    }
  }
  const unsigned re = __reduce_add_sync(0xffffffffu, (unsigned)nexact);
  const unsigned rt = __reduce_add_sync(0xffffffffu, (unsigned)nties);
  if (lane == 0 && re) atomicAdd(&counters[0], (unsigned long long)re);
  if (lane == 0 && rt) atomicAdd(&counters[1], (unsigned long long)rt);
}

// rho_v = (w * factor) / (its exact volume sum * its sub-box's unit), 0 on
// the hull or without incident tetrahedra (vertexDensity,
// triangulation.cpp:200-279).  vprefix: nsb + 1 vertex range starts.
constexpr int kDensBlock = 256;
__global__ void __launch_bounds__(kDensBlock) k_vertex_density(
    int64_t V, const float* __restrict__ w, const long long* __restrict__ acc, const int* __restrict__ hull,
    const VolScale* __restrict__ scale, const int64_t* __restrict__ vprefix, int nsb, float factor,
    float4* __restrict__ posd) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= V) return;
  const int b = nsb > 1 ? find_box(vprefix, nsb, i) : 0;
  posd[i].w = density_from_fixed(__ldg(&acc[i]), __ldg(&scale[b].unit), __ldg(&w[i]), factor, __ldg(&hull[i]) != 0);
}

// Bounding box of every sub-box's vertices (float order keys).  Grid-stride
// over 32-vertex chunks: a warp keeps running per-lane extremes while its
// chunks stay in one sub-box and reduces them into that box's six atomics
// when the box changes and at its end (chunks that straddle two sub-boxes
// add per vertex), so the six words of a box see a few atomics per warp
// instead of one per 32 vertices.
__device__ __forceinline__ void bbox_flush(int b, const int lo[3], const int hi[3], int* __restrict__ bbox) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const int l = __reduce_min_sync(0xffffffffu, lo[c]);
    const int u = __reduce_max_sync(0xffffffffu, hi[c]);
    if ((threadIdx.x & 31) == 0 && l <= u) {
      atomicMin(&bbox[6 * b + 2 * c], l);
      atomicMax(&bbox[6 * b + 2 * c + 1], u);
    }
  }
}

__global__ void __launch_bounds__(256) k_box_bbox(int64_t V, const float4* __restrict__ posd,
                                                  const int64_t* __restrict__ vprefix, int nsb,
                                                  int* __restrict__ bbox) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  int cur = -1;  // the warp's current sub-box (warp-uniform)
  int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
  for (int64_t base = warp * 32; base < V; base += n_warps * 32) {
    const int64_t i = base + lane;
    const bool valid = i < V;
    const int b = valid ? (nsb > 1 ? find_box(vprefix, nsb, i) : 0) : -1;
    int k[3] = {INT_MAX, INT_MAX, INT_MAX};
    if (valid) {
      const float4 r = __ldg(&posd[i]);
      k[0] = float_order_key(r.x);
      k[1] = float_order_key(r.y);
      k[2] = float_order_key(r.z);
    }
    const int b0 = __shfl_sync(0xffffffffu, b, 0);
    const bool uniform = __all_sync(0xffffffffu, b == b0 || b < 0);
    if (uniform && b0 == cur) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        lo[c] = min(lo[c], k[c]);
        if (valid) hi[c] = max(hi[c], k[c]);
      }
      continue;
    }
    if (cur >= 0) bbox_flush(cur, lo, hi, bbox);
#pragma unroll
    for (int c = 0; c < 3; ++c) { lo[c] = INT_MAX; hi[c] = INT_MIN; }
    if (uniform) {
      cur = b0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        lo[c] = k[c];
        if (valid) hi[c] = k[c];
      }
    } else {
      cur = -1;
      if (valid) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          atomicMin(&bbox[6 * b + 2 * c], k[c]);
          atomicMax(&bbox[6 * b + 2 * c + 1], k[c]);
        }
      }
    }
  }
  if (cur >= 0) bbox_flush(cur, lo, hi, bbox);
}

__global__ void k_box_bbox_init(int nsb, int* __restrict__ bbox) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 6 * nsb) bbox[i] = (i & 1) ? INT_MIN : INT_MAX;
}

__global__ void k_box_scales(int nsb, const int* __restrict__ bbox, const int64_t* __restrict__ vprefix,
                             VolScale* __restrict__ scale) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nsb) return;
  scale[b] = vprefix[b + 1] > vprefix[b] ? vol_scale(bbox_volume(bbox + 6 * b)) : VolScale{0.0, 0.0};
}

// Offsets of the 26 neighbouring cells, nearest first (faces, edges, corners).
__constant__ signed char c_nbr[26][3] = {
    {0, 0, -1}, {0, 0, 1}, {0, -1, 0}, {0, 1, 0}, {-1, 0, 0}, {1, 0, 0},
    {0, -1, -1}, {0, -1, 1}, {0, 1, -1}, {0, 1, 1}, {-1, 0, -1}, {-1, 0, 1},
    {1, 0, -1}, {1, 0, 1}, {-1, -1, 0}, {-1, 1, 0}, {1, -1, 0}, {1, 1, 0},
    {-1, -1, -1}, {-1, -1, 1}, {-1, 1, -1}, {-1, 1, 1}, {1, -1, -1}, {1, -1, 1},
    {1, 1, -1}, {1, 1, 1}};

struct InterpParams {
  const int4* tet_v;
  const int4* tet_n;
  const int4* tet_rec = nullptr;  // interleaved records (vertices, neighbours) per tetrahedron
  const float4* posd;
  const float4* vel4;
  const float* scal;
  const unsigned long long* bins;  // walk seeds (distance bits << 32 | tetrahedron)
  const dtfe_subbox* boxes;
  const int64_t* tile_prefix;
  const int64_t* bin_offset;
  const float* eq_off;  // K * NN * 3 equidistant offsets (method 3)
  const float* xs;
  const float* ys;
  const float* zs;
  int K;
  int64_t G1, G2;
  int64_t n_total;
  int NN;
  uint64_t seed;
  uint32_t fields;
  int fix;
  int max_steps;
  int count_centres;  // the centres were placed by the raster: the evaluation counts them
  const int64_t* pencil_prefix;  // K + 1: z pencils (tile x by y) before each sub-box
  int S;                         // scalars per vertex
  float* out[DTFE_NUM_FIELDS];
  unsigned long long* counters;
};

__device__ __forceinline__ bool has_field(uint32_t f, int slot) { return (f >> slot) & 1u; }

// Writes one C-component field of a warp's 32 cells.  When the cells are
// consecutive in the grid (the usual case: k is the fastest index) the values
// go through shared memory and leave as contiguous 16-byte stores; otherwise
// each lane stores its own.
template <int C>
__device__ __forceinline__ void store_field(float* __restrict__ out, int64_t cell, bool valid,
                                            const float* val, bool contig, int64_t c0, float* stage) {
  const int lane = threadIdx.x & 31;
  if (contig) {
#pragma unroll
    for (int c = 0; c < C; ++c) stage[lane * C + c] = val[c];
    __syncwarp();
    float4* dst = reinterpret_cast<float4*>(out + c0 * C);
    const float4* src = reinterpret_cast<const float4*>(stage);
#pragma unroll
    for (int q = lane; q < 8 * C; q += 32) dst[q] = src[q];
    __syncwarp();
  } else if (valid) {
#pragma unroll
    for (int c = 0; c < C; ++c) out[cell * C + c] = val[c];
  }
}

constexpr int kInterpBlock = 256;

// Geometry of flattened sample s (tile order: sub-box, then x, y, z fastest).
struct SampleCell {
  int b, i, j, k;
  int64_t local, cell;
  float x, y, z;
};

__device__ __forceinline__ SampleCell sample_cell(const InterpParams& P, int64_t s) {
  SampleCell c;
  c.b = find_box(P.tile_prefix, P.K, s);
  const dtfe_subbox& B = P.boxes[c.b];
  c.local = s - __ldg(&P.tile_prefix[c.b]);
  const int nz = B.tile_dims[2], ny = B.tile_dims[1];
  tile_ijk(c.local, ny, nz, c.i, c.j, c.k);
  c.x = __ldg(&P.xs[B.coord_offset[0] + c.i]);
  c.y = __ldg(&P.ys[B.coord_offset[1] + c.j]);
  c.z = __ldg(&P.zs[B.coord_offset[2] + c.k]);
  c.cell = ((int64_t)(B.tile_origin[0] + c.i) * P.G1 + (B.tile_origin[1] + c.j)) * P.G2 + (B.tile_origin[2] + c.k);
  return c;
}

__device__ __forceinline__ void fold_counters(const InterpParams& P, unsigned n_loc, unsigned n_out, unsigned n_fail,
                                              const WalkStats& st) {
  unsigned vals[CNT_N] = {n_loc, n_out, n_fail, (unsigned)st.steps, (unsigned)st.exact, (unsigned)st.tie};
#pragma unroll
  for (int c = 0; c < CNT_N; ++c) {
    unsigned r = __reduce_add_sync(0xffffffffu, vals[c]);
    if ((threadIdx.x & 31) == 0 && r) atomicAdd(&P.counters[c], (unsigned long long)r);
  }
}

// Seed tetrahedron of one sample: its cell's bin, else the nearest of the 26
// neighbouring cells with one, else the sub-box's first tetrahedron.
// -1 when the sub-box has no tetrahedra (fewer than four non-coplanar
// particles): its samples are outside, as the reference's zeros for such a
// triangulation (triangulation_miscellaneous.cc:121-138).
__device__ __forceinline__ int seed_of(const InterpParams& P, const SampleCell& c) {
  const dtfe_subbox& B = P.boxes[c.b];
  if (B.n_tets == 0) return -1;
  const unsigned long long* bins = P.bins + __ldg(&P.bin_offset[c.b]);
  unsigned long long s0 = __ldg(&bins[c.local]);
  if (s0 == kEmptySeed) {
    const int nx = B.tile_dims[0], ny = B.tile_dims[1], nz = B.tile_dims[2];
    for (int q = 0; q < 26 && s0 == kEmptySeed; ++q) {
      const int ii = c.i + c_nbr[q][0], jj = c.j + c_nbr[q][1], kk = c.k + c_nbr[q][2];
      if (ii < 0 || jj < 0 || kk < 0 || ii >= nx || jj >= ny || kk >= nz) continue;
      s0 = __ldg(&bins[((int64_t)ii * ny + jj) * nz + kk]);
    }
  }
  int t0 = s0 == kEmptySeed ? -1 : (int)(unsigned)(s0 & 0xFFFFFFFFull);
  if (t0 < B.tet_offset || t0 >= B.tet_offset + B.n_tets) t0 = (int)B.tet_offset;
  return t0;
}

// Point location of every cell centre: seed from the cell's bin (the lowest
// tetrahedron whose centroid lies in the cell, else in the nearest of the 26
// neighbouring cells that has one), then the walk.  Writes the canonical
// tetrahedron (or kOutside) per sample.  Each thread locates R consecutive
// samples; within one z pencil the next sample starts from the previous hit
// (the reference's raster hint) instead of its bin.
template <int R>
__device__ __forceinline__ void locate_cells_body(const InterpParams& P, int* __restrict__ tet_c) {
  WalkStats st{0, 0, 0};
  unsigned n_loc = 0, n_out = 0, n_fail = 0;
  const int64_t nthreads = (int64_t)gridDim.x * blockDim.x;
  const int64_t n_groups = (P.n_total + R - 1) / R;
  const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  for (int64_t g0 = tid - (threadIdx.x & 31); g0 < n_groups; g0 += nthreads) {
    const int64_t g = g0 + (threadIdx.x & 31);
    int prev_hit = -1, prev_b = -1, prev_j = -1, prev_i = -1;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int64_t s = g * R + r;
      if (g >= n_groups || s >= P.n_total) break;
      const SampleCell c = sample_cell(P, s);
      const int t0 = (r > 0 && prev_hit >= 0 && prev_b == c.b && prev_j == c.j && prev_i == c.i) ? prev_hit
                                                                                             : seed_of(P, c);
      const double pc[3] = {(double)c.x, (double)c.y, (double)c.z};
      int v[4];
      float X[4][3];
      int tc = t0 < 0 ? kOutside : walk_locate<true>(P.tet_v, P.tet_n, P.posd, pc, t0, P.max_steps, v, X, st);
      ++n_loc;
      if (tc == kWalkFail) { ++n_fail; tc = kOutside; }
      if (tc < 0) ++n_out;
      tet_c[s] = tc;
      prev_hit = tc;
      prev_b = c.b;
      prev_j = c.j;
      prev_i = c.i;
    }
  }
  fold_counters(P, n_loc, n_out, n_fail, st);
}

template <int BS, int MINB, int R>
__global__ void __launch_bounds__(BS, MINB) k_locate_cells(InterpParams P, int* __restrict__ tet_c) {
  locate_cells_body<R>(P, tet_c);
}

// Field evaluation at the located cell centres (method 0): every lane does
// the same work, so the warp stays converged.
template <int S, int MINB>
__global__ void __launch_bounds__(kInterpBlock, MINB) k_eval_centre(InterpParams P, const int* __restrict__ tet_c) {
  constexpr int CMAX = (3 * S > 9) ? 3 * S : 9;
  __shared__ __align__(16) float s_stage[kInterpBlock / 32][32 * CMAX];
  float* stage = s_stage[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const uint32_t F = P.fields;
  const bool want_grad = has_field(F, DTFE_VELOCITY_GRADIENT) || has_field(F, DTFE_VELOCITY_DIVERGENCE) ||
                         has_field(F, DTFE_VELOCITY_SHEAR) || has_field(F, DTFE_VELOCITY_VORTICITY);
  const bool want_vel = has_field(F, DTFE_VELOCITY) || want_grad;
  const bool want_dens = has_field(F, DTFE_DENSITY);
  const bool want_sc = S > 0 && (has_field(F, DTFE_SCALAR) || has_field(F, DTFE_SCALAR_GRADIENT));
  const bool fix = P.fix != 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t base0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) - lane;
  unsigned n_loc = 0, n_out = 0;  // centres placed by the raster
  for (int64_t base = base0; base < P.n_total; base += stride) {
    const int64_t s = base + lane;
    const bool valid = s < P.n_total;
    int64_t cell = -1;
    CellOut e;
    e.dens = 0.f;
#pragma unroll
    for (int c = 0; c < 3; ++c) e.vel[c] = 0.f;
#pragma unroll
    for (int c = 0; c < 9; ++c) e.grad[c] = 0.f;
#pragma unroll
    for (int q = 0; q < S; ++q) {
      e.sc[q] = 0.f;
#pragma unroll
      for (int c = 0; c < 3; ++c) e.scg[3 * q + c] = 0.f;
    }
    if (valid) {
      const SampleCell c = sample_cell(P, s);
      cell = c.cell;
      const int t = __ldg(&tet_c[s]);
      n_loc += 1;
      n_out += t < 0;
      if (t >= 0) {
        int v[4];
        float X[4][3];
        load_tet(P.tet_v, P.posd, t, v, X);
        const double pc[3] = {(double)c.x, (double)c.y, (double)c.z};
        cell_eval<S>(v, X, pc, P.posd, P.vel4, P.scal, want_dens, want_vel, want_sc, fix, e);
      }
    }
    const int64_t c0 = __shfl_sync(0xffffffffu, cell, 0);
    const bool contig = __all_sync(0xffffffffu, valid && cell == c0 + lane) && (c0 % 4 == 0);
    if (has_field(F, DTFE_DENSITY)) store_field<1>(P.out[DTFE_DENSITY], cell, valid, &e.dens, contig, c0, stage);
    if (has_field(F, DTFE_VELOCITY)) store_field<3>(P.out[DTFE_VELOCITY], cell, valid, e.vel, contig, c0, stage);
    if (has_field(F, DTFE_VELOCITY_GRADIENT))
      store_field<9>(P.out[DTFE_VELOCITY_GRADIENT], cell, valid, e.grad, contig, c0, stage);
    if (has_field(F, DTFE_VELOCITY_DIVERGENCE) || has_field(F, DTFE_VELOCITY_SHEAR) ||
        has_field(F, DTFE_VELOCITY_VORTICITY)) {
      float dv, sh[5], vo[3];
      derived_fields(e.grad, dv, sh, vo);
      if (has_field(F, DTFE_VELOCITY_DIVERGENCE))
        store_field<1>(P.out[DTFE_VELOCITY_DIVERGENCE], cell, valid, &dv, contig, c0, stage);
      if (has_field(F, DTFE_VELOCITY_SHEAR))
        store_field<5>(P.out[DTFE_VELOCITY_SHEAR], cell, valid, sh, contig, c0, stage);
      if (has_field(F, DTFE_VELOCITY_VORTICITY))
        store_field<3>(P.out[DTFE_VELOCITY_VORTICITY], cell, valid, vo, contig, c0, stage);
    }
    if (S > 0 && has_field(F, DTFE_SCALAR))
      store_field<(S > 0 ? S : 1)>(P.out[DTFE_SCALAR], cell, valid, e.sc, contig, c0, stage);
    if (S > 0 && has_field(F, DTFE_SCALAR_GRADIENT))
      store_field<(S > 0 ? 3 * S : 1)>(P.out[DTFE_SCALAR_GRADIENT], cell, valid, e.scg, contig, c0, stage);
  }
  if (P.count_centres) fold_counters(P, n_loc, n_out, 0, WalkStats{0, 0, 0});
}

// Cell centres located and evaluated in one pass (locate variants 9..11):
// each lane walks from its seed as k_locate_cells does, then evaluates with
// the tetrahedron the walk ends in, whose vertices and positions are still
// in registers; the warp is converged again after the walk, so the
// evaluation and the staged stores run as in k_eval_centre.
template <int S, int MINB, bool REC = false>
__global__ void __launch_bounds__(kInterpBlock, MINB) k_locate_eval(InterpParams P, int* __restrict__ tet_c) {
  constexpr int CMAX = (3 * S > 9) ? 3 * S : 9;
  __shared__ __align__(16) float s_stage[kInterpBlock / 32][32 * CMAX];
  float* stage = s_stage[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const uint32_t F = P.fields;
  const bool want_grad = has_field(F, DTFE_VELOCITY_GRADIENT) || has_field(F, DTFE_VELOCITY_DIVERGENCE) ||
                         has_field(F, DTFE_VELOCITY_SHEAR) || has_field(F, DTFE_VELOCITY_VORTICITY);
  const bool want_vel = has_field(F, DTFE_VELOCITY) || want_grad;
  const bool want_dens = has_field(F, DTFE_DENSITY);
  const bool want_sc = S > 0 && (has_field(F, DTFE_SCALAR) || has_field(F, DTFE_SCALAR_GRADIENT));
  const bool fix = P.fix != 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t base0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) - lane;
  WalkStats wst{0, 0, 0};
  unsigned n_loc = 0, n_out = 0, n_fail = 0;
  for (int64_t base = base0; base < P.n_total; base += stride) {
    const int64_t s = base + lane;
    const bool valid = s < P.n_total;
    int64_t cell = -1;
    CellOut e;
    e.dens = 0.f;
#pragma unroll
    for (int c = 0; c < 3; ++c) e.vel[c] = 0.f;
#pragma unroll
    for (int c = 0; c < 9; ++c) e.grad[c] = 0.f;
#pragma unroll
    for (int q = 0; q < S; ++q) {
      e.sc[q] = 0.f;
#pragma unroll
      for (int c = 0; c < 3; ++c) e.scg[3 * q + c] = 0.f;
    }
    if (valid) {
      const SampleCell c = sample_cell(P, s);
      cell = c.cell;
      // the walk ends with the located tetrahedron's vertices and positions
      // in registers: the evaluation uses them directly
      const double pc[3] = {(double)c.x, (double)c.y, (double)c.z};
      int v[4];
      float X[4][3], D[4];
      const int t0 = seed_of(P, c);
      int t = t0 < 0 ? kOutside
                     : (REC ? walk_locate_rec<true>(P.tet_rec, P.tet_v, P.tet_n, P.posd, pc, t0, P.max_steps, v, X,
                                                    D, wst)
                            : walk_locate<true>(P.tet_v, P.tet_n, P.posd, pc, t0, P.max_steps, v, X, wst));
      ++n_loc;
      if (t == kWalkFail) {
        ++n_fail;
        t = kOutside;
      }
      n_out += t < 0;
      tet_c[s] = t;
      if (t >= 0)
        cell_eval<S>(v, X, pc, P.posd, P.vel4, P.scal, want_dens, want_vel, want_sc, fix, e, REC ? D : nullptr);
    }
    const int64_t c0 = __shfl_sync(0xffffffffu, cell, 0);
    const bool contig = __all_sync(0xffffffffu, valid && cell == c0 + lane) && (c0 % 4 == 0);
    if (has_field(F, DTFE_DENSITY)) store_field<1>(P.out[DTFE_DENSITY], cell, valid, &e.dens, contig, c0, stage);
    if (has_field(F, DTFE_VELOCITY)) store_field<3>(P.out[DTFE_VELOCITY], cell, valid, e.vel, contig, c0, stage);
    if (has_field(F, DTFE_VELOCITY_GRADIENT))
      store_field<9>(P.out[DTFE_VELOCITY_GRADIENT], cell, valid, e.grad, contig, c0, stage);
    if (has_field(F, DTFE_VELOCITY_DIVERGENCE) || has_field(F, DTFE_VELOCITY_SHEAR) ||
        has_field(F, DTFE_VELOCITY_VORTICITY)) {
      float dv, sh[5], vo[3];
      derived_fields(e.grad, dv, sh, vo);
      if (has_field(F, DTFE_VELOCITY_DIVERGENCE))
        store_field<1>(P.out[DTFE_VELOCITY_DIVERGENCE], cell, valid, &dv, contig, c0, stage);
      if (has_field(F, DTFE_VELOCITY_SHEAR))
        store_field<5>(P.out[DTFE_VELOCITY_SHEAR], cell, valid, sh, contig, c0, stage);
      if (has_field(F, DTFE_VELOCITY_VORTICITY))
        store_field<3>(P.out[DTFE_VELOCITY_VORTICITY], cell, valid, vo, contig, c0, stage);
    }
    if (S > 0 && has_field(F, DTFE_SCALAR))
      store_field<(S > 0 ? S : 1)>(P.out[DTFE_SCALAR], cell, valid, e.sc, contig, c0, stage);
    if (S > 0 && has_field(F, DTFE_SCALAR_GRADIENT))
      store_field<(S > 0 ? 3 * S : 1)>(P.out[DTFE_SCALAR_GRADIENT], cell, valid, e.scg, contig, c0, stage);
  }
  fold_counters(P, n_loc, n_out, n_fail, wst);
}

// Zeroes every sample of a pencil of nz samples after its first outside one
// (tet_c[s0 + k] < 0): the pencil's samples are tet_c[s0 .. s0 + nz), its
// cells P.out rows c0 .. c0 + nz.  One warp reads the located tetrahedra 32 at
// a time; later inside samples are marked outside and their fields zeroed.
__device__ __forceinline__ void zero_after_outside(const InterpParams& P, int* __restrict__ tet_c, int64_t s0,
                                                   int64_t c0, int nz, int lane) {
  bool seen = false;
  for (int k0 = 0; k0 < nz; k0 += 32) {
    const int k = k0 + lane;
    const bool valid = k < nz;
    const int t = valid ? tet_c[s0 + k] : 0;
    const unsigned outside = __ballot_sync(0xffffffffu, valid && t < 0);
    const bool poison = seen || (outside & ((1u << lane) - 1u)) != 0;
    if (valid && poison && t >= 0) {
      tet_c[s0 + k] = kOutside;
      const int64_t cell = c0 + k;
      for (int slot = 0; slot < DTFE_NUM_FIELDS; ++slot) {
        if (!has_field(P.fields, slot) || !P.out[slot]) continue;
        const int nc = slot == DTFE_VELOCITY || slot == DTFE_VELOCITY_VORTICITY ? 3
                     : slot == DTFE_VELOCITY_GRADIENT ? 9
                     : slot == DTFE_VELOCITY_SHEAR ? 5
                     : slot == DTFE_SCALAR ? P.S
                     : slot == DTFE_SCALAR_GRADIENT ? 3 * P.S : 1;
        for (int c = 0; c < nc; ++c) P.out[slot][cell * nc + c] = 0.f;
      }
    }
    seen = seen || outside != 0u;
  }
}

// The reference's cell-centre raster after an outside sample: it skips
// `z += dx` (unaveraged_interpolation.cc:304 jumps over :353), so the rest of
// the z pencil re-locates that outside point and gets zeros.  One warp per
// pencil of the sub-box tiles.
__global__ void __launch_bounds__(256) k_outside_pencils(InterpParams P, int* __restrict__ tet_c, int64_t n_pencils) {
  // the locate kernels of this call have counted the outside samples: none,
  // nothing to zero (every thread reads the same count, so all return)
  if (*(volatile const unsigned long long*)&P.counters[CNT_OUTSIDE] == 0ull) return;
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t q = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; q < n_pencils; q += nw) {
    const int b = find_box(P.pencil_prefix, P.K, q);
    const dtfe_subbox& B = P.boxes[b];
    const int ny = B.tile_dims[1], nz = B.tile_dims[2];
    const uint32_t local = (uint32_t)(q - __ldg(&P.pencil_prefix[b]));
    const int i = (int)(local / (uint32_t)ny), j = (int)(local - (uint32_t)i * (uint32_t)ny);
    const int64_t s0 = __ldg(&P.tile_prefix[b]) + (int64_t)local * nz;
    const int64_t c0 = ((int64_t)(B.tile_origin[0] + i) * P.G1 + (B.tile_origin[1] + j)) * P.G2 + B.tile_origin[2];
    zero_after_outside(P, tet_c, s0, c0, nz, lane);
  }
}

// The same on a redshift-cone grid: an outside sample skips `psi += dx`
// (unaveraged_interpolation.cc:466 jumps over :527), so the rest of its psi
// row repeats it.  Rows of nz samples, sample index = output row.
__global__ void __launch_bounds__(256) k_cone_rows(InterpParams P, int* __restrict__ tet_c, int64_t n_rows, int nz) {
  if (*(volatile const unsigned long long*)&P.counters[CNT_OUTSIDE] == 0ull) return;  // no bin outside
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t q = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; q < n_rows; q += nw)
    zero_after_outside(P, tet_c, q * nz, q * nz, nz, lane);
}

// Particles of the padded box (findParticlesInBox / insertParticlesInBox,
// src/subpartition.h:79-154): for each of up to 27 box translations (order
// i1, i2, i3 over {-1, 0, 1}, offset (i - 1) * box length in float) the
// translated padded box selects particles (closed, isParticleInBox), which
// are emitted shifted back by the offset (float subtraction), translation
// after translation, particles in input order within one.  Block b covers
// chunk b % nchunks of translation b / nchunks, so the exclusive prefix of
// the per-block counts is every block's first output row.
constexpr int kSelChunk = 1024;
struct SelBoxes {
  float box[27][6];
  float off[27][3];
};
__device__ __forceinline__ bool sel_in(const float* __restrict__ pos, int64_t i, const float* b) {
  const float x = __ldg(&pos[3 * i]), y = __ldg(&pos[3 * i + 1]), z = __ldg(&pos[3 * i + 2]);
  return x >= b[0] && x <= b[1] && y >= b[2] && y <= b[3] && z >= b[4] && z <= b[5];
}
__global__ void __launch_bounds__(kSelChunk) k_select_count(const float* __restrict__ pos, int64_t n,
                                                            int64_t nchunks, SelBoxes S, int* __restrict__ counts) {
  const int64_t b = blockIdx.x;
  const int o = (int)(b / nchunks);
  const int64_t i = (b - (int64_t)o * nchunks) * kSelChunk + threadIdx.x;
  const int c = __syncthreads_count(i < n && sel_in(pos, i, S.box[o]));
  if (threadIdx.x == 0) counts[b] = c;
}
__global__ void __launch_bounds__(kSelChunk) k_select_write(const float* __restrict__ pos, int64_t n,
                                                            int64_t nchunks, SelBoxes S,
                                                            const int64_t* __restrict__ first,
                                                            int32_t* __restrict__ idx_out,
                                                            float* __restrict__ pos_out) {
  __shared__ int warp_first[kSelChunk / 32];
  const int64_t b = blockIdx.x;
  const int o = (int)(b / nchunks);
  const int64_t i = (b - (int64_t)o * nchunks) * kSelChunk + threadIdx.x;
  const bool in = i < n && sel_in(pos, i, S.box[o]);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned m = __ballot_sync(0xffffffffu, in);
  if (lane == 0) warp_first[warp] = __popc(m);
  __syncthreads();
  if (warp == 0) {
    const int v = warp_first[lane];  // kSelChunk / 32 == 32 warps
    int incl = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += y;
    }
    warp_first[lane] = incl - v;
  }
  __syncthreads();
  if (in) {
    const int64_t at = __ldg(&first[b]) + warp_first[warp] + __popc(m & ((1u << lane) - 1u));
    if (idx_out) idx_out[at] = (int32_t)i;
    if (pos_out) {
#pragma unroll
      for (int k = 0; k < 3; ++k) pos_out[3 * at + k] = __fsub_rn(__ldg(&pos[3 * i + k]), S.off[o][k]);
    }
  }
}

// Fields at user sampling points (interpolateUserSampling,
// unaveraged_interpolation.cc:560-691), one thread per point of a single
// sub-box's tessellation.  keep[i]: the point lies in the region (closed);
// idx: exclusive prefix of keep, the point's output row.  Seed: the bin of the
// tile cell nearest the point (when the seeds are built), else the sub-box's
// first tetrahedron; then the walk and the cell-centre arithmetic at the
// point.
struct Region6 {
  float r[6];
};
__global__ void k_points_keep(int64_t n, const float* __restrict__ pts, Region6 R, int* __restrict__ keep) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  bool in = true;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float q = pts[3 * i + c];
    in = in && q >= R.r[2 * c] && q <= R.r[2 * c + 1];
  }
  keep[i] = in ? 1 : 0;
}

// Where k_points_eval takes its points.  User sampling points: those kept,
// each written to its prefix row.
struct PointList {
  const float* pts;
  const int* keep;
  const int64_t* idx;
  __device__ __forceinline__ bool get(int64_t i, float pf[3], int64_t& row) const {
    if (!keep[i]) return false;
#pragma unroll
    for (int c = 0; c < 3; ++c) pf[c] = pts[3 * i + c];
    row = idx[i];
    return true;
  }
};
// Redshift-cone bins (unaveraged_interpolation.cc:441-447): sample
// (i, j, k) = row (i n1 + j) n2 + k at o + (r st cp, r st sp, r ct), each
// product and sum rounded in float left to right as the reference's
// expression is (no contraction).  Tables: r[n0], st/ct[n1], cp/sp[n2].
struct ConeGrid {
  const float* r;
  const float* st;
  const float* ct;
  const float* cp;
  const float* sp;
  float o[3];
  uint32_t n1, n2;
  __device__ __forceinline__ bool get(int64_t s, float pf[3], int64_t& row) const {
    const uint64_t ij = (uint64_t)s / n2;
    const uint32_t k = (uint32_t)((uint64_t)s - ij * n2);
    const uint32_t i = (uint32_t)(ij / n1), j = (uint32_t)(ij - (uint64_t)i * n1);
    const float ri = __ldg(&r[i]);
    const float rs = __fmul_rn(ri, __ldg(&st[j]));
    pf[0] = __fadd_rn(o[0], __fmul_rn(rs, __ldg(&cp[k])));
    pf[1] = __fadd_rn(o[1], __fmul_rn(rs, __ldg(&sp[k])));
    pf[2] = __fadd_rn(o[2], __fmul_rn(ri, __ldg(&ct[j])));
    row = s;
    return true;
  }
};

// Walk seed of a point in the handle's single sub-box: the bin of the tile
// cell nearest the point (when the seeds are built), so points beyond the
// tile (padding zone, outside the hull) start at the tile's edge; else the
// sub-box's first tetrahedron.  -1 for a sub-box without tetrahedra.  The
// located tetrahedron does not depend on the start.
__device__ __forceinline__ int point_seed(const InterpParams& P, const float pf[3], int use_bins) {
  const dtfe_subbox& B = P.boxes[0];
  int t0 = B.n_tets > 0 ? (int)B.tet_offset : -1;
  if (use_bins && t0 >= 0 && B.tile_dims[0] > 0 && B.tile_dims[1] > 0 && B.tile_dims[2] > 0) {
    SampleCell c;
    int ijk[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float f = floorf((pf[a] - B.lo[a]) / B.dx[a]);
      ijk[a] = (int)fminf(fmaxf(f, 0.f), (float)(B.tile_dims[a] - 1));
    }
    c.b = 0;
    c.i = ijk[0];
    c.j = ijk[1];
    c.k = ijk[2];
    c.local = ((int64_t)ijk[0] * B.tile_dims[1] + ijk[1]) * B.tile_dims[2] + ijk[2];
    t0 = seed_of(P, c);
  }
  return t0;
}

template <int S>
__device__ __forceinline__ void zero_out(CellOut& e) {
  e.dens = 0.f;
#pragma unroll
  for (int c = 0; c < 3; ++c) e.vel[c] = 0.f;
#pragma unroll
  for (int c = 0; c < 9; ++c) e.grad[c] = 0.f;
#pragma unroll
  for (int q = 0; q < S; ++q) {
    e.sc[q] = 0.f;
#pragma unroll
    for (int c = 0; c < 3; ++c) e.scg[3 * q + c] = 0.f;
  }
}

// One output row of every requested field (derived fields from the gradient).
template <int S>
__device__ __forceinline__ void store_row(const InterpParams& P, int64_t o, const CellOut& e) {
  const uint32_t F = P.fields;
  if (has_field(F, DTFE_DENSITY)) P.out[DTFE_DENSITY][o] = e.dens;
  if (has_field(F, DTFE_VELOCITY))
#pragma unroll
    for (int c = 0; c < 3; ++c) P.out[DTFE_VELOCITY][3 * o + c] = e.vel[c];
  if (has_field(F, DTFE_VELOCITY_GRADIENT))
#pragma unroll
    for (int c = 0; c < 9; ++c) P.out[DTFE_VELOCITY_GRADIENT][9 * o + c] = e.grad[c];
  if (has_field(F, DTFE_VELOCITY_DIVERGENCE) || has_field(F, DTFE_VELOCITY_SHEAR) ||
      has_field(F, DTFE_VELOCITY_VORTICITY)) {
    float dv, sh[5], vo[3];
    derived_fields(e.grad, dv, sh, vo);
    if (has_field(F, DTFE_VELOCITY_DIVERGENCE)) P.out[DTFE_VELOCITY_DIVERGENCE][o] = dv;
    if (has_field(F, DTFE_VELOCITY_SHEAR))
#pragma unroll
      for (int c = 0; c < 5; ++c) P.out[DTFE_VELOCITY_SHEAR][5 * o + c] = sh[c];
    if (has_field(F, DTFE_VELOCITY_VORTICITY))
#pragma unroll
      for (int c = 0; c < 3; ++c) P.out[DTFE_VELOCITY_VORTICITY][3 * o + c] = vo[c];
  }
  if (S > 0 && has_field(F, DTFE_SCALAR))
#pragma unroll
    for (int q = 0; q < S; ++q) P.out[DTFE_SCALAR][(int64_t)S * o + q] = e.sc[q];
  if (S > 0 && has_field(F, DTFE_SCALAR_GRADIENT))
#pragma unroll
    for (int q = 0; q < 3 * S; ++q) P.out[DTFE_SCALAR_GRADIENT][(int64_t)3 * S * o + q] = e.scg[q];
}

// tet_out (may be null): the located tetrahedron of each row, kOutside when
// outside the hull.  Four blocks per SM (64 registers), as the fused
// cell-centre kernel's default: the walks are latency-bound.
template <int S, class Src>
__global__ void __launch_bounds__(256, 4) k_points_eval(InterpParams P, int64_t n, Src src, int use_bins,
                                                     int* __restrict__ tet_out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  float pf[3];
  int64_t o = 0;
  const bool active = i < n && src.get(i, pf, o);
  WalkStats st{0, 0, 0};
  unsigned n_loc = 0, n_out = 0, n_fail = 0;
  if (active) {
    const double p[3] = {(double)pf[0], (double)pf[1], (double)pf[2]};
    const int t0 = point_seed(P, pf, use_bins);
    int v[4];
    float X[4][3];
    int t = t0 < 0 ? kOutside : walk_locate<true>(P.tet_v, P.tet_n, P.posd, p, t0, P.max_steps, v, X, st);
    ++n_loc;
    if (t == kWalkFail) {
      ++n_fail;
      t = kOutside;
    }
    n_out += t < 0;
    CellOut e;
    zero_out<S>(e);
    const uint32_t F = P.fields;
    const bool want_grad = has_field(F, DTFE_VELOCITY_GRADIENT) || has_field(F, DTFE_VELOCITY_DIVERGENCE) ||
                           has_field(F, DTFE_VELOCITY_SHEAR) || has_field(F, DTFE_VELOCITY_VORTICITY);
    const bool want_vel = has_field(F, DTFE_VELOCITY) || want_grad;
    const bool want_sc = S > 0 && (has_field(F, DTFE_SCALAR) || has_field(F, DTFE_SCALAR_GRADIENT));
    if (t >= 0) cell_eval<S>(v, X, p, P.posd, P.vel4, P.scal, has_field(F, DTFE_DENSITY), want_vel, want_sc, P.fix != 0, e);
    if (tet_out) tet_out[o] = t;
    store_row<S>(P, o, e);
  }
  fold_counters(P, n_loc, n_out, n_fail, st);
}

// Volume averages at point samples (averaged_interpolation_2.cc:245-662):
// NN points per sample, offsets u in (-0.5, 0.5) from Philox keyed by
// (seed, sample index, w) instead of the reference's mt19937 stream (the
// comparison with the reference is statistical); each point walked from the
// tetrahedron of the sample's centre (the reference's `previous` hint), the
// fields summed in float in sample order, points outside the hull skipped
// but counted, divided by NN (:154-155, 195).
// Sources: user points (interpolateUserSampling_averaged_2, :470-647): point
// = float(position + u delta) per axis; redshift-cone bins
// (interpolateRedshiftCone_averaged_2, :245-466): r, theta, psi each
// float(centre + u d), then o + (r sin theta) cos psi ... in float, with
// sin/cos evaluated in double and rounded to float.
struct PointAvgList {
  PointList pl;
  const float* delta;
  __device__ __forceinline__ bool get(int64_t i, float pf[3], int64_t& row) const { return pl.get(i, pf, row); }
  __device__ __forceinline__ void sample(int64_t i, const double u[3], float pf[3]) const {
#pragma unroll
    for (int c = 0; c < 3; ++c)
      pf[c] = (float)__dadd_rn((double)pl.pts[3 * i + c], __dmul_rn(u[c], (double)delta[3 * i + c]));
  }
};
struct ConeAvgGrid {
  ConeGrid g;
  const float* th;  // theta bin centres [n1]
  const float* ps;  // psi bin centres [n2]
  float d[3];       // bin sizes in r, theta, psi (radians)
  __device__ __forceinline__ bool get(int64_t s, float pf[3], int64_t& row) const { return g.get(s, pf, row); }
  __device__ __forceinline__ void sample(int64_t s, const double u[3], float pf[3]) const {
    const uint64_t ij = (uint64_t)s / g.n2;
    const uint32_t k = (uint32_t)((uint64_t)s - ij * g.n2);
    const uint32_t i = (uint32_t)(ij / g.n1), j = (uint32_t)(ij - (uint64_t)i * g.n1);
    const float R = (float)__dadd_rn((double)__ldg(&g.r[i]), __dmul_rn(u[0], (double)d[0]));
    const float T = (float)__dadd_rn((double)__ldg(&th[j]), __dmul_rn(u[1], (double)d[1]));
    const float Q = (float)__dadd_rn((double)__ldg(&ps[k]), __dmul_rn(u[2], (double)d[2]));
    const float st = (float)sin((double)T), ct = (float)cos((double)T);
    const float cq = (float)cos((double)Q), sq = (float)sin((double)Q);
    const float rs = __fmul_rn(R, st);
    pf[0] = __fadd_rn(g.o[0], __fmul_rn(rs, cq));
    pf[1] = __fadd_rn(g.o[1], __fmul_rn(rs, sq));
    pf[2] = __fadd_rn(g.o[2], __fmul_rn(R, ct));
  }
};

template <int S, class Src>
__global__ void __launch_bounds__(256, 4) k_points_average(InterpParams P, int64_t n, Src src, int use_bins,
                                                        uint64_t key) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  float pc[3];
  int64_t o = 0;
  const bool active = i < n && src.get(i, pc, o);
  WalkStats st{0, 0, 0};
  unsigned n_loc = 0, n_out = 0, n_fail = 0;
  if (active) {
    const uint32_t F = P.fields;
    const bool want_grad = has_field(F, DTFE_VELOCITY_GRADIENT) || has_field(F, DTFE_VELOCITY_DIVERGENCE) ||
                           has_field(F, DTFE_VELOCITY_SHEAR) || has_field(F, DTFE_VELOCITY_VORTICITY);
    const bool want_vel = has_field(F, DTFE_VELOCITY) || want_grad;
    const bool want_dens = has_field(F, DTFE_DENSITY);
    const bool want_sc = S > 0 && (has_field(F, DTFE_SCALAR) || has_field(F, DTFE_SCALAR_GRADIENT));
    int t0 = point_seed(P, pc, use_bins);
    if (t0 >= 0) {
      // the centre's tetrahedron seeds the sample walks
      const double p[3] = {(double)pc[0], (double)pc[1], (double)pc[2]};
      int v[4];
      float X[4][3];
      const int tc = walk_locate<true>(P.tet_v, P.tet_n, P.posd, p, t0, P.max_steps, v, X, st);
      ++n_loc;
      if (tc == kWalkFail) ++n_fail;
      if (tc >= 0) t0 = tc;
    }
    CellOut acc;
    zero_out<S>(acc);
    const int NN = P.NN;
    for (int w = 0; w < NN && t0 >= 0; ++w) {
      double u[3];
      mc_offsets(key, (uint64_t)i, (uint32_t)w, u);
      float pf[3];
      src.sample(i, u, pf);
      const double p[3] = {(double)pf[0], (double)pf[1], (double)pf[2]};
      int v[4];
      float X[4][3];
      int t = walk_locate<true>(P.tet_v, P.tet_n, P.posd, p, t0, P.max_steps, v, X, st);
      ++n_loc;
      if (t == kWalkFail) {
        ++n_fail;
        t = kOutside;
      }
      n_out += t < 0;
      if (t < 0) continue;
      CellOut e;
      zero_out<S>(e);  // fields not requested stay 0 in the sums
      cell_eval<S>(v, X, p, P.posd, P.vel4, P.scal, want_dens, want_vel, want_sc, P.fix != 0, e);
      acc.dens += e.dens;
#pragma unroll
      for (int q = 0; q < 3; ++q) acc.vel[q] += e.vel[q];
#pragma unroll
      for (int q = 0; q < 9; ++q) acc.grad[q] += e.grad[q];
#pragma unroll
      for (int q = 0; q < S; ++q) {
        acc.sc[q] += e.sc[q];
#pragma unroll
        for (int r = 0; r < 3; ++r) acc.scg[3 * q + r] += e.scg[3 * q + r];
      }
    }
    const float fn = (float)NN;
    acc.dens = acc.dens / fn;
#pragma unroll
    for (int q = 0; q < 3; ++q) acc.vel[q] = acc.vel[q] / fn;
#pragma unroll
    for (int q = 0; q < 9; ++q) acc.grad[q] = acc.grad[q] / fn;
#pragma unroll
    for (int q = 0; q < S; ++q) {
      acc.sc[q] = acc.sc[q] / fn;
#pragma unroll
      for (int r = 0; r < 3; ++r) acc.scg[3 * q + r] = acc.scg[3 * q + r] / fn;
    }
    store_row<S>(P, o, acc);
  }
  fold_counters(P, n_loc, n_out, n_fail, st);
}

// Cell averages (methods 2 and 3): n points per cell, each walked from the
// cell centre's tetrahedron (averaged_interpolation_2.cc:123,145), summed in
// sample order as the reference does, divided by n; infinite-cell points are
// skipped but counted.
template <int METHOD, int S>
__global__ void __launch_bounds__(kInterpBlock) k_average(InterpParams P, const int* __restrict__ tet_c) {
  constexpr int CMAX = (3 * S > 9) ? 3 * S : 9;
  __shared__ __align__(16) float s_stage[kInterpBlock / 32][32 * CMAX];
  float* stage = s_stage[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const uint32_t F = P.fields;
  const bool want_grad = has_field(F, DTFE_VELOCITY_GRADIENT) || has_field(F, DTFE_VELOCITY_DIVERGENCE) ||
                         has_field(F, DTFE_VELOCITY_SHEAR) || has_field(F, DTFE_VELOCITY_VORTICITY);
  const bool want_vel = has_field(F, DTFE_VELOCITY) || want_grad || has_field(F, DTFE_VELOCITY_STD);
  const bool want_dens = has_field(F, DTFE_DENSITY);
  const bool want_sc = S > 0 && (has_field(F, DTFE_SCALAR) || has_field(F, DTFE_SCALAR_GRADIENT));
  const bool want_std = METHOD == DTFE_METHOD_MONTE_CARLO && has_field(F, DTFE_VELOCITY_STD);
  const bool fix = P.fix != 0;
  WalkStats st{0, 0, 0};
  unsigned n_loc = 0, n_fail = 0, n_out_c = 0;

  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t base0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) - lane;
  for (int64_t base = base0; base < P.n_total; base += stride) {
    const int64_t s = base + lane;
    const bool valid = s < P.n_total;
    int64_t cell = -1;
    float aD = 0.f, aV[3] = {0.f, 0.f, 0.f}, aG[9], aS[S > 0 ? S : 1], aSG[S > 0 ? 3 * S : 1];
    float sdev = 0.f;
#pragma unroll
    for (int c = 0; c < 9; ++c) aG[c] = 0.f;
#pragma unroll
    for (int q = 0; q < (S > 0 ? S : 1); ++q) aS[q] = 0.f;
#pragma unroll
    for (int q = 0; q < (S > 0 ? 3 * S : 1); ++q) aSG[q] = 0.f;

    if (valid) {
      const SampleCell c = sample_cell(P, s);
      const dtfe_subbox& B = P.boxes[c.b];
      cell = c.cell;
      const double pc[3] = {(double)c.x, (double)c.y, (double)c.z};
      const int tc = __ldg(&tet_c[s]);
      if (P.count_centres) {
        ++n_loc;
        n_out_c += tc < 0;
      }
      const int tstart = tc >= 0 ? tc : (int)B.tet_offset;
      const int NN = P.NN;
      const uint64_t key = mc_key(P.seed, B.part_no);
      float stdacc[3] = {0.f, 0.f, 0.f};
      for (int w = 0; w < NN; ++w) {
        double p[3];
        if (METHOD == DTFE_METHOD_MONTE_CARLO) {
          double u[3];
          mc_offsets(key, (uint64_t)cell, (uint32_t)w, u);
          p[0] = u[0] * (double)B.dx[0] + pc[0];
          p[1] = u[1] * (double)B.dx[1] + pc[1];
          p[2] = u[2] * (double)B.dx[2] + pc[2];
        } else {
          const float* eo = P.eq_off + ((int64_t)c.b * NN + w) * 3;
          p[0] = (double)(c.x + __ldg(&eo[0]));
          p[1] = (double)(c.y + __ldg(&eo[1]));
          p[2] = (double)(c.z + __ldg(&eo[2]));
        }
        int vv[4];
        float XX[4][3];
        // a sub-box without tetrahedra: every point outside
        int t = B.n_tets > 0 ? walk_locate(P.tet_v, P.tet_n, P.posd, p, tstart, P.max_steps, vv, XX, st) : kOutside;
        ++n_loc;
        if (t == kWalkFail) { ++n_fail; t = kOutside; }
        if (t < 0) continue;
        CellOut e;
        cell_eval<S>(vv, XX, p, P.posd, P.vel4, P.scal, want_dens, want_vel, want_sc, fix, e);
        aD += e.dens;
#pragma unroll
        for (int q = 0; q < 3; ++q) aV[q] += e.vel[q];
#pragma unroll
        for (int q = 0; q < 9; ++q) aG[q] += e.grad[q];
#pragma unroll
        for (int q = 0; q < S; ++q) {
          aS[q] += e.sc[q];
#pragma unroll
          for (int r = 0; r < 3; ++r) aSG[3 * q + r] += e.scg[3 * q + r];
        }
        if (want_std) {
#pragma unroll
          for (int q = 0; q < 3; ++q) stdacc[q] += e.vel[q];
        }
      }
      const float fn = (float)NN;
      aD = aD / fn;
#pragma unroll
      for (int q = 0; q < 3; ++q) aV[q] = aV[q] / fn;
#pragma unroll
      for (int q = 0; q < 9; ++q) aG[q] = aG[q] / fn;
#pragma unroll
      for (int q = 0; q < S; ++q) {
        aS[q] = aS[q] / fn;
#pragma unroll
        for (int r = 0; r < 3; ++r) aSG[3 * q + r] = aSG[3 * q + r] / fn;
      }
      if (want_std) {
        // standardDeviation (triangulation_miscellaneous.cc:256-271); the
        // second pass re-walks the samples (their velocities are not kept)
        float mean[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) mean[q] = stdacc[q] / fn;
        float r = 0.f;
        for (int w = 0; w < NN; ++w) {
          float vel[3] = {0.f, 0.f, 0.f};
          double u[3], p[3];
          mc_offsets(key, (uint64_t)cell, (uint32_t)w, u);
          p[0] = u[0] * (double)B.dx[0] + pc[0];
          p[1] = u[1] * (double)B.dx[1] + pc[1];
          p[2] = u[2] * (double)B.dx[2] + pc[2];
          int vv[4];
          float XX[4][3];
          WalkStats st2{0, 0, 0};
          int t = B.n_tets > 0 ? walk_locate(P.tet_v, P.tet_n, P.posd, p, tstart, P.max_steps, vv, XX, st2)
                               : kOutside;
          if (t >= 0) {
            CellOut e;
            cell_eval<0>(vv, XX, p, P.posd, P.vel4, P.scal, false, true, false, fix, e);
#pragma unroll
            for (int q = 0; q < 3; ++q) vel[q] = e.vel[q];
          }
#pragma unroll
          for (int q = 0; q < 3; ++q) {
            float d = vel[q] - mean[q];
            r += d * d;
          }
        }
        sdev = sqrtf(r / fn);
      }
    }

    const int64_t c0 = __shfl_sync(0xffffffffu, cell, 0);
    const bool contig = __all_sync(0xffffffffu, valid && cell == c0 + lane) && (c0 % 4 == 0);
    if (has_field(F, DTFE_DENSITY)) store_field<1>(P.out[DTFE_DENSITY], cell, valid, &aD, contig, c0, stage);
    if (has_field(F, DTFE_VELOCITY)) store_field<3>(P.out[DTFE_VELOCITY], cell, valid, aV, contig, c0, stage);
    if (has_field(F, DTFE_VELOCITY_GRADIENT))
      store_field<9>(P.out[DTFE_VELOCITY_GRADIENT], cell, valid, aG, contig, c0, stage);
    if (has_field(F, DTFE_VELOCITY_DIVERGENCE) || has_field(F, DTFE_VELOCITY_SHEAR) ||
        has_field(F, DTFE_VELOCITY_VORTICITY)) {
      float dv, sh[5], vo[3];
      derived_fields(aG, dv, sh, vo);
      if (has_field(F, DTFE_VELOCITY_DIVERGENCE))
        store_field<1>(P.out[DTFE_VELOCITY_DIVERGENCE], cell, valid, &dv, contig, c0, stage);
      if (has_field(F, DTFE_VELOCITY_SHEAR))
        store_field<5>(P.out[DTFE_VELOCITY_SHEAR], cell, valid, sh, contig, c0, stage);
      if (has_field(F, DTFE_VELOCITY_VORTICITY))
        store_field<3>(P.out[DTFE_VELOCITY_VORTICITY], cell, valid, vo, contig, c0, stage);
    }
    if (want_std) store_field<1>(P.out[DTFE_VELOCITY_STD], cell, valid, &sdev, contig, c0, stage);
    if (S > 0 && has_field(F, DTFE_SCALAR))
      store_field<(S > 0 ? S : 1)>(P.out[DTFE_SCALAR], cell, valid, aS, contig, c0, stage);
    if (S > 0 && has_field(F, DTFE_SCALAR_GRADIENT))
      store_field<(S > 0 ? 3 * S : 1)>(P.out[DTFE_SCALAR_GRADIENT], cell, valid, aSG, contig, c0, stage);
  }
  fold_counters(P, n_loc, n_out_c, n_fail, st);
}

// Locate arbitrary points (tests): canonical tetrahedron or -1 / -2.
__global__ void k_locate_points(int64_t np, const double* __restrict__ pts, const int4* __restrict__ tet_v,
                                const int4* __restrict__ tet_n, const float4* __restrict__ posd,
                                int start, int max_steps, int* __restrict__ out) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= np) return;
  double p[3] = {pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]};
  int v[4];
  float X[4][3];
  WalkStats st{0, 0, 0};
  out[i] = walk_locate(tet_v, tet_n, posd, p, start, max_steps, v, X, st);
}

}  // namespace

// Tiles of a main grid <-> their values packed tile after tile (x, y, z
// order inside a tile), the layout the tile exchange between ranks sends
// (copySubgridResultsToMain, src/subpartition.h:399-432).  One thread per
// packed float: its tile by binary search over the tiles' packed offsets;
// consecutive threads walk z, so both sides are read and written in runs.
struct TileRec {
  int32_t o[3], d[3];
};
__global__ void k_tiles_copy(int n_tiles, const TileRec* __restrict__ tiles, const int64_t* __restrict__ start,
                             int64_t G1, int64_t G2, int ncomp, int to_packed, const float* __restrict__ src,
                             float* __restrict__ dst) {
  const int64_t total = __ldg(&start[n_tiles]) * ncomp;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = e / ncomp;
    const int c = (int)(e - s * ncomp);
    int lo = 0, hi = n_tiles;  // start[lo] <= s < start[hi]
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (__ldg(&start[mid]) <= s) lo = mid;
      else hi = mid;
    }
    const TileRec T = tiles[lo];
    const int64_t local = s - __ldg(&start[lo]);
    const int64_t plane = (int64_t)T.d[1] * T.d[2];
    const int64_t i = local / plane, r = local - i * plane;
    const int64_t j = r / T.d[2], k = r - j * T.d[2];
    const int64_t cell = ((T.o[0] + i) * G1 + (T.o[1] + j)) * G2 + (T.o[2] + k);
    if (to_packed) dst[e] = src[cell * ncomp + c];
    else dst[cell * ncomp + c] = src[e];
  }
}

// ---------------------------------------------------------------------------
// Handle
struct dtfe_gpu_s {
  int device = 0;
  cudaStream_t stream = nullptr;
  int S = 0;
  int max_steps = 65536;
  int64_t T = 0, V = 0;
  int4* tet_v = nullptr;
  int4* tet_n = nullptr;
  float4* posd = nullptr;
  float4* vel4 = nullptr;
  float* scal = nullptr;
  float* w = nullptr;
  long long* vacc = nullptr;      // per-vertex volume sums in exact units (fixed_volume.cuh)
  VolScale* vscale = nullptr;     // per sub-box: its units (from its vertices' bounding box)
  int* vbbox = nullptr;           // per sub-box bounding box (float order keys)
  int64_t* sb_vprefix = nullptr;  // nsb + 1 vertex range starts of the scale boxes
  int64_t* sb_tprefix = nullptr;  // nsb + 1 tetrahedron range starts
  int nsb = 0;                    // scale boxes: the sub-boxes, or the whole upload before set_subboxes
  bool scale_ready = false;
  std::vector<int64_t> sb_vprefix_h, sb_tprefix_h;  // host copies of sb_vprefix / sb_tprefix
  int64_t* inc_off = nullptr;     // V+1 offsets into inc
  int* inc = nullptr;             // incident tetrahedra per vertex (built when needed)
  bool inc_ready = false;
  int* scratch_i = nullptr;       // V ints (degrees / fill cursors)
  int64_t* scan_blocks = nullptr; // block totals of the offset scan
  int* hull = nullptr;
  bool has_vel = false, has_scal = false;
  bool density_ready = false;
  // sub-boxes
  int K = 0;
  std::vector<dtfe_subbox> boxes_h;
  dtfe_subbox* boxes = nullptr;
  int64_t* tile_prefix = nullptr;
  int64_t* pencil_prefix = nullptr;  // K + 1: z pencils before each sub-box
  int64_t n_pencils = 0;
  int64_t* tet_prefix = nullptr;  // K+1 tetrahedron range starts
  int64_t* bin_offset = nullptr;
  unsigned long long* bins = nullptr;
  int* tet_c = nullptr;   // located tetrahedron of every cell centre
  // launch variants (dtfe_gpu_autotune); the defaults are the fastest on
  // the 256^3 Zel'dovich workload: seeded walk and evaluation in one kernel
  // at 4 blocks per SM (evaluation variant 2 for the averaging methods)
  int loc_variant = 11;
  int eval_variant = 2;
  int64_t n_cells = 0;
  float *xs = nullptr, *ys = nullptr, *zs = nullptr;
  int32_t grid[3] = {0, 0, 0};
  bool prep_ready = false;        // volumes and centre locations (raster) or walk seeds are current
  bool prep_raster = false;       // ... prepared by the raster
  int prep_variant = 0;           // ... with this locate variant
  RasterAxis* raster_axes = nullptr;  // per sub-box and axis: raster formula and its margin
  float* eq_off = nullptr;
  int eq_nn = 0;
  unsigned long long* counters = nullptr;
  float* out_buf[DTFE_NUM_FIELDS] = {};
  size_t out_cap[DTFE_NUM_FIELDS] = {};
  std::map<void*, size_t> caps;  // bytes held by each device buffer
  void* dep_scratch = nullptr;    // grid deposition scratch
  size_t dep_bytes = 0;
  float* dep_out = nullptr;       // host-output deposition staging (4 per cell)
  alignas(16) char dep_saved[128] = {};  // particle/box state of the last deposit (adjoint)
  // adjoint state
  bool tet_c_valid = false;       // tet_c holds the centres of the last centre interpolation
  bool tet_c_fix = false;         // that interpolation used DTFE_FLAG_FIX_VALUE_INTERP
  float factor = 0.f;             // (D+1)/rho_bar of the last vertex-density call
  double *g_rho = nullptr, *g_x = nullptr, *g_v = nullptr, *g_S = nullptr, *g_m = nullptr, *vbar = nullptr;
  float* adj_a = nullptr;         // device copies of host loss weights
  cudaGraphExec_t step_graph = nullptr;  // captured step (dtfe_gpu_graph_build)
  char* upload_buf = nullptr;     // staging of packed tetrahedra and 3-float vertex records
  cudaEvent_t ev_h2d = nullptr;   // recorded when an upload's copies have crossed
  dtfe_gpu_s* upload_after = nullptr;  // uploads wait for this handle's latest copies
  void* sph_scratch = nullptr;    // SPH cell grids, neighbour bookkeeping, FP64 sums
  size_t sph_bytes = 0;
  std::vector<float> regions_h;   // 6 per sub-box: tile regions (averaging method 1)
  float* pts_buf = nullptr;       // user sampling points: positions, then the output rows
  int* pts_keep = nullptr;
  int64_t* pts_idx = nullptr;
  int64_t* pts_blocks = nullptr;
  float* pts_out = nullptr;
  int* sel_counts = nullptr;      // dtfe_gpu_select_in_box_dev: per-block counts and first rows
  int64_t* sel_first = nullptr;
  int64_t* sel_blocks = nullptr;
  char* io_stage[2] = {nullptr, nullptr};  // pinned staging of dtfe_gpu_write_binary_dev
  cudaEvent_t io_ev[2] = {nullptr, nullptr};
  double* m1_table = nullptr;     // method-1 Sobol points (100 NN x 3)
  int m1_table_nn = 0;
  void* m1_scratch = nullptr;     // method-1 counts, offsets, scan scratch
  size_t m1_bytes = 0;
  void* m1_lists = nullptr;       // method-1 tetrahedra of every cell
  size_t m1_lists_bytes = 0;
  float* sph_out = nullptr;       // host-output SPH staging
  int4* tet_rec = nullptr;        // interleaved (vertices, neighbours) per tetrahedron, built on first use
  bool rec_ready = false;
  TileRec* tile_recs = nullptr;   // dtfe_gpu_tiles_*: the tiles of one call
  int64_t* tile_start = nullptr;  // ... and their packed offsets
};

namespace {

// Device allocation that keeps a buffer when it is already large enough, so
// repeated uploads of same-sized inputs do not reallocate.
template <typename Tp>
int dev_alloc(dtfe_handle h, Tp** p, size_t count) {
  size_t bytes = count * sizeof(Tp);
  size_t& cap = h->caps[(void*)p];
  if (*p && cap >= bytes) return DTFE_OK;
  if (*p) {
    cudaFree(*p);
    *p = nullptr;
    cap = 0;
  }
  if (count == 0) return DTFE_OK;
  cudaError_t e = cudaMalloc((void**)p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    return set_error(DTFE_ERR_ALLOC, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  cap = bytes;
  return DTFE_OK;
}

inline unsigned blocks_for(int64_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

int field_components(int slot, int S) {
  switch (slot) {
    case DTFE_DENSITY: return 1;
    case DTFE_VELOCITY: return 3;
    case DTFE_VELOCITY_GRADIENT: return 9;
    case DTFE_VELOCITY_DIVERGENCE: return 1;
    case DTFE_VELOCITY_SHEAR: return 5;
    case DTFE_VELOCITY_VORTICITY: return 3;
    case DTFE_VELOCITY_STD: return 1;
    case DTFE_SCALAR: return S;
    case DTFE_SCALAR_GRADIENT: return 3 * S;
  }
  return 0;
}

// A captured step refers to the handle's buffers as they were at capture.
void drop_graph(dtfe_handle h) {
  if (h->step_graph) {
    cudaStreamSynchronize(h->stream);
    cudaGraphExecDestroy(h->step_graph);
    h->step_graph = nullptr;
  }
}

// Launch variants chosen by dtfe_gpu_autotune.  Locate variants 0..2 place
// the cell centres with the raster fused into the volume kernel (3, 2 or 4
// blocks per SM); variants 3..8 walk from seeds (blocks per SM, samples per
// thread); variants 9..11 walk and evaluate in one kernel (3, 2 or 4 blocks
// per SM; for the averaging methods they walk as variant 3); variants 12..13
// do the same over the interleaved 32-byte tetrahedron records (4 or 3
// blocks per SM).  Evaluation variants: register budget of the evaluation
// kernel.
constexpr int kNumRasterVariants = 3;
struct LocVariant { int block, minb, r; };
constexpr LocVariant kWalkVariants[] = {{256, 3, 1}, {256, 2, 1}, {256, 4, 1}, {256, 3, 2}, {256, 4, 2}, {256, 3, 4}};
constexpr int kNumWalkVariants = sizeof(kWalkVariants) / sizeof(kWalkVariants[0]);
struct FusedVariant { int minb; bool rec; };
constexpr FusedVariant kFused[] = {{3, false}, {2, false}, {4, false}, {4, true}, {3, true}};
constexpr int kFirstFused = kNumRasterVariants + kNumWalkVariants;
constexpr int kNumLocVariants = kFirstFused + sizeof(kFused) / sizeof(kFused[0]);
inline bool uses_records(int loc_variant) {
  return loc_variant >= kFirstFused && kFused[loc_variant - kFirstFused].rec;
}
inline bool is_raster(int loc_variant) { return loc_variant < kNumRasterVariants; }
inline bool is_fused(int loc_variant) { return loc_variant >= kFirstFused; }
constexpr int kNumEvalVariants = 3;

// Vertex -> tetrahedron incidence lists (in no particular order within a
// vertex): degrees, their scan into offsets, the fill.  star: each
// tetrahedron listed at its two smallest vertices only (deriving the
// neighbours of a neighbour-less upload); else at all four (the adjoint).
int build_incidence(dtfe_handle h, bool star = false) {
  const int64_t V = h->V, T = h->T;
  int rc;
  if ((rc = dev_alloc(h, &h->inc_off, V + 1)) || (rc = dev_alloc(h, &h->inc, 4 * T)) ||
      (rc = dev_alloc(h, &h->scratch_i, V + 1)) ||
      (rc = dev_alloc(h, &h->scan_blocks, (V + kScanBlock - 1) / kScanBlock + 1)))
    return rc;
  cudaStream_t st = h->stream;
  if (V) {
    DTFE_CUDA_TRY(cudaMemsetAsync(h->scratch_i, 0, sizeof(int) * V, st));
    if (T && star) k_degree_star<<<blocks_for(T, 256), 256, 0, st>>>(T, h->tet_v, h->scratch_i);
    else if (T) k_degree<<<blocks_for(T, 256), 256, 0, st>>>(T, h->tet_v, h->scratch_i);
    const int64_t nb = (V + kScanBlock - 1) / kScanBlock;
    k_scan_blocks<<<(unsigned)nb, kScanBlock, 0, st>>>(V, h->scratch_i, h->inc_off, h->scan_blocks);
    k_scan_totals<<<1, kScanBlock, 0, st>>>(nb, h->scan_blocks, h->inc_off + V);
    k_scan_add<<<(unsigned)nb, kScanBlock, 0, st>>>(V, h->inc_off, h->scan_blocks);
    DTFE_CUDA_TRY(cudaMemsetAsync(h->scratch_i, 0, sizeof(int) * V, st));
    if (T && star)
      k_fill_star<<<blocks_for(T, 256), 256, 0, st>>>(T, h->tet_v, h->inc_off, h->scratch_i, h->inc);
    else if (T)
      k_fill_incidence<<<blocks_for(T, 256), 256, 0, st>>>(T, h->tet_v, h->inc_off, h->scratch_i, h->inc);
  }
  DTFE_CUDA_TRY(cudaGetLastError());
  h->inc_ready = !star;
  return DTFE_OK;
}

// The units of the exact volume sums (fixed_volume.cuh), one per sub-box
// (the whole upload before dtfe_gpu_set_subboxes): the bounding box of its
// vertices, then its scale.  Once per upload and sub-box layout.
int ensure_scales(dtfe_handle h) {
  if (h->scale_ready) return DTFE_OK;
  const int nsb = h->K > 0 ? h->K : 1;
  std::vector<int64_t> vp(nsb + 1), tp(nsb + 1);
  if (h->K > 0) {
    for (int b = 0; b < nsb; ++b) {
      vp[b] = h->boxes_h[b].vert_offset;
      tp[b] = h->boxes_h[b].tet_offset;
    }
    vp[nsb] = h->boxes_h[nsb - 1].vert_offset + h->boxes_h[nsb - 1].n_verts;
    tp[nsb] = h->boxes_h[nsb - 1].tet_offset + h->boxes_h[nsb - 1].n_tets;
  } else {
    vp[0] = tp[0] = 0;
    vp[1] = h->V;
    tp[1] = h->T;
  }
  int rc;
  if ((rc = dev_alloc(h, &h->sb_vprefix, nsb + 1)) || (rc = dev_alloc(h, &h->sb_tprefix, nsb + 1)) ||
      (rc = dev_alloc(h, &h->vbbox, 6 * (size_t)nsb)) || (rc = dev_alloc(h, &h->vscale, (size_t)nsb)))
    return rc;
  cudaStream_t st = h->stream;
  // the prefix tables cross only when they change (a new sub-box layout or
  // counts), from handle-owned copies: a step whose upload keeps the layout
  // queues kernels only, so its host thread never waits for the device here
  if (vp != h->sb_vprefix_h || tp != h->sb_tprefix_h) {
    h->sb_vprefix_h = std::move(vp);
    h->sb_tprefix_h = std::move(tp);
    DTFE_CUDA_TRY(cudaMemcpyAsync(h->sb_vprefix, h->sb_vprefix_h.data(), sizeof(int64_t) * (nsb + 1),
                                  cudaMemcpyHostToDevice, st));
    DTFE_CUDA_TRY(cudaMemcpyAsync(h->sb_tprefix, h->sb_tprefix_h.data(), sizeof(int64_t) * (nsb + 1),
                                  cudaMemcpyHostToDevice, st));
  }
  k_box_bbox_init<<<blocks_for(6 * nsb, 256), 256, 0, st>>>(nsb, h->vbbox);
  if (h->V)
    k_box_bbox<<<(unsigned)std::min<int64_t>(blocks_for(h->V, 256), 148 * 4), 256, 0, st>>>(h->V, h->posd,
                                                                                           h->sb_vprefix, nsb,
                                                                                           h->vbbox);
  k_box_scales<<<blocks_for(nsb, 64), 64, 0, st>>>(nsb, h->vbbox, h->sb_vprefix, h->vscale);
  DTFE_CUDA_TRY(cudaGetLastError());
  h->nsb = nsb;
  h->scale_ready = true;
  return DTFE_OK;
}

// Per step, before the interpolation: the tetrahedron volumes, added into
// their vertices' exact sums, and either the cell centres' tetrahedra
// (raster) or the walk seeds.  Without sub-boxes, volumes only.
int launch_prep(dtfe_handle h) {
  cudaStream_t st = h->stream;
  const bool raster = is_raster(h->loc_variant);
  int src = ensure_scales(h);
  if (src) return src;
  DTFE_CUDA_TRY(cudaMemsetAsync(h->counters + CNT_RASTER_EXACT, 0, 2 * sizeof(unsigned long long), st));
  if (h->V) DTFE_CUDA_TRY(cudaMemsetAsync(h->vacc, 0, sizeof(long long) * h->V, st));
  const VolSums VS{h->vacc, h->vscale, h->sb_tprefix, h->nsb};
  if (h->K > 0 && raster) {
    int rc = dev_alloc(h, &h->tet_c, h->n_cells);
    if (rc) return rc;
    DTFE_CUDA_TRY(cudaMemsetAsync(h->tet_c, 0xFF, sizeof(int) * h->n_cells, st));
    if (h->T > 0) {
      const unsigned nb = blocks_for(h->T, kRasterBlock);
      auto* k = h->loc_variant == 1 ? k_tet_volume_raster<2>
                                    : (h->loc_variant == 2 ? k_tet_volume_raster<4> : k_tet_volume_raster<3>);
      k<<<nb, kRasterBlock, 0, st>>>(h->T, h->tet_v, h->posd, VS, h->boxes, h->tet_prefix, h->tile_prefix,
                                     h->raster_axes, h->K, h->xs, h->ys, h->zs, (unsigned*)h->tet_c,
                                     h->counters + CNT_RASTER_EXACT);
    }
  } else if (h->K > 0) {
    DTFE_CUDA_TRY(cudaMemsetAsync(h->bins, 0xFF, sizeof(unsigned long long) * h->n_cells, st));
    if (h->T > 0)
      k_tet_volume_bins2<kVolTPT><<<blocks_for((h->T + kVolTPT - 1) / kVolTPT, kVolBlock), kVolBlock, 0, st>>>(
          h->T, h->tet_v, h->posd, VS, h->boxes, h->tet_prefix, h->bin_offset, h->K, h->xs, h->ys, h->zs,
          h->bins);
  } else if (h->T > 0) {
    k_tet_volume_bins<false><<<blocks_for(h->T, kVolBlock), kVolBlock, 0, st>>>(
        h->T, h->tet_v, h->posd, VS, h->boxes, h->tet_prefix, h->bin_offset, h->K, h->xs, h->ys, h->zs,
        h->bins);
  }
  DTFE_CUDA_TRY(cudaGetLastError());
  h->prep_ready = h->K > 0;
  h->prep_raster = raster;
  h->prep_variant = h->loc_variant;
  return DTFE_OK;
}

int prepare_centres(dtfe_handle h) {
  if (h->prep_ready && h->prep_raster == is_raster(h->loc_variant) &&
      (!h->prep_raster || h->prep_variant == h->loc_variant))
    return DTFE_OK;
  return launch_prep(h);
}

void launch_locate(int variant, const InterpParams& P, int* tet_c, cudaStream_t st) {
  if (is_raster(variant)) return;
  const LocVariant& L = kWalkVariants[variant - kNumRasterVariants];
  const int64_t groups = (P.n_total + L.r - 1) / L.r;
  const unsigned grid = (unsigned)((groups + L.block - 1) / L.block);
  switch (variant) {
    case 3: k_locate_cells<256, 3, 1><<<grid, 256, 0, st>>>(P, tet_c); break;
    case 4: k_locate_cells<256, 2, 1><<<grid, 256, 0, st>>>(P, tet_c); break;
    case 5: k_locate_cells<256, 4, 1><<<grid, 256, 0, st>>>(P, tet_c); break;
    case 6: k_locate_cells<256, 3, 2><<<grid, 256, 0, st>>>(P, tet_c); break;
    case 7: k_locate_cells<256, 4, 2><<<grid, 256, 0, st>>>(P, tet_c); break;
    default: k_locate_cells<256, 3, 4><<<grid, 256, 0, st>>>(P, tet_c); break;
  }
}

template <int S>
void launch_eval(int method, int evariant, const InterpParams& P, const int* tet_c, cudaStream_t st, unsigned grid,
                 unsigned block) {
  if (method == DTFE_METHOD_CENTRE) {
    if (evariant == 1) k_eval_centre<S, 2><<<grid, block, 0, st>>>(P, tet_c);
    else if (evariant == 2) k_eval_centre<S, 4><<<grid, block, 0, st>>>(P, tet_c);
    else k_eval_centre<S, 3><<<grid, block, 0, st>>>(P, tet_c);
  } else if (method == DTFE_METHOD_MONTE_CARLO) {
    k_average<DTFE_METHOD_MONTE_CARLO, S><<<grid, block, 0, st>>>(P, tet_c);
  } else {
    k_average<DTFE_METHOD_EQUIDISTANT, S><<<grid, block, 0, st>>>(P, tet_c);
  }
}

template <int S>
void launch_fused(int fv, const InterpParams& P, int* tet_c, cudaStream_t st, unsigned grid, unsigned block) {
  const FusedVariant& F = kFused[fv];
  // record walks are built for the scalar counts a handle accepts (0-4, 8)
  constexpr bool kRecOk = S <= 4 || S == 8;
  if (F.rec && kRecOk) {
    if (F.minb == 4) k_locate_eval<S, 4, kRecOk><<<grid, block, 0, st>>>(P, tet_c);
    else k_locate_eval<S, 3, kRecOk><<<grid, block, 0, st>>>(P, tet_c);
  } else if (F.minb == 2) {
    k_locate_eval<S, 2><<<grid, block, 0, st>>>(P, tet_c);
  } else if (F.minb == 4) {
    k_locate_eval<S, 4><<<grid, block, 0, st>>>(P, tet_c);
  } else {
    k_locate_eval<S, 3><<<grid, block, 0, st>>>(P, tet_c);
  }
}

void launch_fused_s(int S, int fv, const InterpParams& P, int* tet_c, cudaStream_t st, unsigned grid,
                    unsigned block) {
  switch (S) {
    case 0: launch_fused<0>(fv, P, tet_c, st, grid, block); break;
    case 1: launch_fused<1>(fv, P, tet_c, st, grid, block); break;
    case 2: launch_fused<2>(fv, P, tet_c, st, grid, block); break;
    case 3: launch_fused<3>(fv, P, tet_c, st, grid, block); break;
    case 4: launch_fused<4>(fv, P, tet_c, st, grid, block); break;
    case 5: launch_fused<5>(fv, P, tet_c, st, grid, block); break;
    case 6: launch_fused<6>(fv, P, tet_c, st, grid, block); break;
    case 7: launch_fused<7>(fv, P, tet_c, st, grid, block); break;
    default: launch_fused<8>(fv, P, tet_c, st, grid, block); break;
  }
}

void launch_eval_s(int method, int S, int evariant, const InterpParams& P, const int* tet_c, cudaStream_t st,
                   unsigned grid, unsigned block) {
  switch (S) {
    case 0: launch_eval<0>(method, evariant, P, tet_c, st, grid, block); break;
    case 1: launch_eval<1>(method, evariant, P, tet_c, st, grid, block); break;
    case 2: launch_eval<2>(method, evariant, P, tet_c, st, grid, block); break;
    case 3: launch_eval<3>(method, evariant, P, tet_c, st, grid, block); break;
    case 4: launch_eval<4>(method, evariant, P, tet_c, st, grid, block); break;
    case 5: launch_eval<5>(method, evariant, P, tet_c, st, grid, block); break;
    case 6: launch_eval<6>(method, evariant, P, tet_c, st, grid, block); break;
    case 7: launch_eval<7>(method, evariant, P, tet_c, st, grid, block); break;
    default: launch_eval<8>(method, evariant, P, tet_c, st, grid, block); break;
  }
}

}  // namespace

extern "C" {

const char* dtfe_last_error(void) { return g_last_error.c_str(); }

// Records an error message for dtfe_last_error() from other translation units.
int dtfe_internal_set_error(int code, const char* msg) { return set_error(code, msg ? msg : ""); }

int dtfe_gpu_create(const dtfe_config* cfg, dtfe_handle* out) {
  if (!out) return set_error(DTFE_ERR_ARG, "null output handle");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return set_error(DTFE_ERR_NO_DEVICE, "no CUDA device");
  dtfe_config c = cfg ? *cfg : dtfe_config{0, 0, 0, 0};
  if (c.device < 0 || c.device >= ndev) return set_error(DTFE_ERR_ARG, "bad device ordinal");
  if (c.n_scalars < 0 || c.n_scalars > DTFE_MAX_SCALARS || c.n_scalars == 5 || c.n_scalars == 6 ||
      c.n_scalars == 7)
    return set_error(DTFE_ERR_ARG, "n_scalars must be 0-4 or 8");
  DTFE_CUDA_TRY(cudaSetDevice(c.device));
  dtfe_handle h = new dtfe_gpu_s();
  h->device = c.device;
  h->S = c.n_scalars;
  h->max_steps = c.max_walk_steps > 0 ? c.max_walk_steps : 65536;
  cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_h2d, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return set_error(DTFE_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
  }
  int rc = dev_alloc(h, &h->counters, CNT_ALL);
  if (!rc && cudaMemsetAsync(h->counters, 0, sizeof(unsigned long long) * CNT_ALL, h->stream) != cudaSuccess)
    rc = set_error(DTFE_ERR_CUDA, "clearing the status counters");
  if (rc) {
    cudaEventDestroy(h->ev_h2d);
    cudaStreamDestroy(h->stream);
    delete h;
    return rc;
  }
  *out = h;
  return DTFE_OK;
}

int dtfe_gpu_destroy(dtfe_handle h) {
  if (!h) return DTFE_OK;
  cudaSetDevice(h->device);
  cudaStreamSynchronize(h->stream);
  if (h->step_graph) cudaGraphExecDestroy(h->step_graph);
  void* ptrs[] = {h->tet_v, h->tet_n, h->posd, h->vel4, h->scal, h->w, h->vacc, h->vscale, h->vbbox,
                  h->sb_vprefix, h->sb_tprefix, h->inc_off, h->inc,
                  h->scratch_i, h->scan_blocks, h->hull, h->pts_buf, h->pts_keep, h->pts_idx, h->pts_blocks,
                  h->pts_out,
                  h->boxes, h->tile_prefix, h->pencil_prefix, h->tet_prefix, h->bin_offset, h->bins,
                  h->xs, h->ys, h->zs, h->eq_off, h->counters, h->tet_c, h->raster_axes};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (int i = 0; i < DTFE_NUM_FIELDS; ++i)
    if (h->out_buf[i]) cudaFree(h->out_buf[i]);
  if (h->dep_scratch) cudaFree(h->dep_scratch);
  for (void* p : {(void*)h->g_rho, (void*)h->g_x, (void*)h->g_v, (void*)h->g_S, (void*)h->g_m, (void*)h->vbar,
                  (void*)h->adj_a, h->sph_scratch, (void*)h->sph_out, (void*)h->upload_buf, (void*)h->m1_table,
                  h->m1_scratch, h->m1_lists, (void*)h->sel_counts, (void*)h->sel_first, (void*)h->sel_blocks,
                  (void*)h->tile_recs, (void*)h->tile_start, (void*)h->tet_rec})
    if (p) cudaFree(p);
  if (h->dep_out) cudaFree(h->dep_out);
  for (int i = 0; i < 2; ++i) {
    if (h->io_stage[i]) cudaFreeHost(h->io_stage[i]);
    if (h->io_ev[i]) cudaEventDestroy(h->io_ev[i]);
  }
  cudaEventDestroy(h->ev_h2d);
  cudaStreamDestroy(h->stream);
  delete h;
  return DTFE_OK;
}

void* dtfe_gpu_stream(dtfe_handle h) { return h ? (void*)h->stream : nullptr; }

int dtfe_gpu_synchronize(dtfe_handle h) {
  if (!h) return set_error(DTFE_ERR_ARG, "null handle");
  DTFE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return DTFE_OK;
}

// Common body of the two uploads: tets(h) copies or decodes the
// tetrahedron arrays into h->tet_v / h->tet_n on h->stream.
extern "C++" {
// tets_bytes: staging the tetrahedra need on the device (0: they are copied
// straight into tet_v / tet_n); tets_h2d(h, stage) queues their host->device
// copies, tets_finish(h, stage) the kernels that complete them.  All copies
// of an upload are queued before any of its kernels, so that a chained
// handle's upload (dtfe_gpu_chain_uploads) can start on the copy engine as
// soon as these have crossed.
// Vertices given as codes into the input particle arrays (k_gather_particles)
// instead of one record each.
struct ParticleSource {
  const uint32_t* codes;  // n_verts host codes
  int64_t n;              // particles
  float len[3];           // box lengths of the periodic images
};

template <class TetH2D, class TetFinish>
static int upload_impl(dtfe_handle h, int64_t n_tets, const float* xyz, const float* w, const float* vel,
                       const float* scal, int64_t n_verts, size_t tets_bytes, TetH2D tets_h2d,
                       TetFinish tets_finish, bool derive_neighbours = false,
                       const ParticleSource* ps = nullptr) {
  if (!h || !xyz || !w || (ps && n_verts > 0 && !ps->codes)) return set_error(DTFE_ERR_ARG, "null argument");
  if (n_tets < 0 || n_verts < 0 || n_tets > 0x7FFFFFFF || n_verts >= 0x7F7F7F7F)
    return set_error(DTFE_ERR_TOO_LARGE, "tetrahedron or vertex count beyond int32 indexing");
  if (ps && (ps->n < 0 || ps->n > ((int64_t)1 << kSrcBits)))
    return set_error(DTFE_ERR_TOO_LARGE, "more than 2^27 particles for vertex codes");
  if (ps && n_verts > 0 && ps->n == 0) return set_error(DTFE_ERR_ARG, "vertex codes without particles");
  DTFE_CUDA_TRY(cudaSetDevice(h->device));
  int rc;
  h->T = n_tets;
  h->V = n_verts;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t tets_stage = al(tets_bytes);
  const size_t vert_stage = sizeof(float) * 3 * (size_t)n_verts;
  // particle mode: xyz, vel (3n each), w (n), scalars (S n), codes (V)
  const int64_t np = ps ? ps->n : 0;
  const size_t p3 = al(sizeof(float) * 3 * (size_t)np), p1 = al(sizeof(float) * (size_t)np);
  const size_t ps_stage = ps ? 2 * p3 + p1 + al(sizeof(float) * h->S * (size_t)np) +
                                   al(sizeof(uint32_t) * (size_t)n_verts)
                             : 0;
  if ((rc = dev_alloc(h, &h->tet_v, n_tets)) || (rc = dev_alloc(h, &h->tet_n, n_tets)) ||
      (rc = dev_alloc(h, &h->posd, n_verts)) || (rc = dev_alloc(h, &h->vel4, n_verts)) ||
      (rc = dev_alloc(h, &h->w, n_verts)) || (rc = dev_alloc(h, &h->vacc, n_verts)) ||
      (rc = dev_alloc(h, &h->hull, n_verts)) ||
      (rc = dev_alloc(h, &h->scal, (size_t)n_verts * h->S)) ||
      // staging kept in the handle (an allocation per upload would map and
      // unmap device memory every time): tetrahedra, positions, velocities
      (rc = dev_alloc(h, &h->upload_buf, tets_stage + (ps ? ps_stage : 2 * vert_stage))))
    return rc;
  cudaStream_t st = h->stream;
  char* stage = h->upload_buf;
  float* sx = (float*)(stage + tets_stage);
  float* sv = (float*)(stage + tets_stage + vert_stage);
  // copies first: wait for the chained handle's transfers, queue ours, mark them
  if (h->upload_after) DTFE_CUDA_TRY(cudaStreamWaitEvent(st, h->upload_after->ev_h2d, 0));
  if (n_tets && (rc = tets_h2d(h, stage))) return rc;
  if (ps) {
    char* q = stage + tets_stage;
    float* pxyz = (float*)q;
    float* pvel = (float*)(q + p3);
    float* pw = (float*)(q + 2 * p3);
    float* pscal = (float*)(q + 2 * p3 + p1);
    uint32_t* pcode = (uint32_t*)(q + 2 * p3 + p1 + al(sizeof(float) * h->S * (size_t)np));
    if (np) {
      DTFE_CUDA_TRY(cudaMemcpyAsync(pxyz, xyz, sizeof(float) * 3 * np, cudaMemcpyHostToDevice, st));
      if (vel) DTFE_CUDA_TRY(cudaMemcpyAsync(pvel, vel, sizeof(float) * 3 * np, cudaMemcpyHostToDevice, st));
      DTFE_CUDA_TRY(cudaMemcpyAsync(pw, w, sizeof(float) * np, cudaMemcpyHostToDevice, st));
      if (h->S > 0 && scal)
        DTFE_CUDA_TRY(cudaMemcpyAsync(pscal, scal, sizeof(float) * h->S * np, cudaMemcpyHostToDevice, st));
    }
    if (n_verts)
      DTFE_CUDA_TRY(cudaMemcpyAsync(pcode, ps->codes, sizeof(uint32_t) * n_verts, cudaMemcpyHostToDevice, st));
  } else if (n_verts) {
    DTFE_CUDA_TRY(cudaMemcpyAsync(sx, xyz, vert_stage, cudaMemcpyHostToDevice, st));
    if (vel) DTFE_CUDA_TRY(cudaMemcpyAsync(sv, vel, vert_stage, cudaMemcpyHostToDevice, st));
    DTFE_CUDA_TRY(cudaMemcpyAsync(h->w, w, sizeof(float) * n_verts, cudaMemcpyHostToDevice, st));
    if (h->S > 0 && scal)
      DTFE_CUDA_TRY(cudaMemcpyAsync(h->scal, scal, sizeof(float) * h->S * n_verts, cudaMemcpyHostToDevice, st));
  }
  DTFE_CUDA_TRY(cudaEventRecord(h->ev_h2d, st));
  // then the kernels: decode the tetrahedra, pack positions and velocities
  // into 16-byte records
  DTFE_CUDA_TRY(cudaMemsetAsync(h->counters + CNT_DECODE, 0, sizeof(unsigned long long), st));
  if (n_tets && (rc = tets_finish(h, stage))) {
    // nothing usable was uploaded: later calls see an empty handle
    h->T = h->V = 0;
    h->density_ready = h->prep_ready = h->tet_c_valid = false;
    drop_graph(h);
    return rc;
  }
  if (ps && n_verts) {
    const char* q = stage + tets_stage;
    k_gather_particles<<<blocks_for(n_verts, 256), 256, 0, st>>>(
        n_verts, h->S, (const uint32_t*)(q + 2 * p3 + p1 + al(sizeof(float) * h->S * (size_t)np)),
        (const float*)q, vel ? (const float*)(q + p3) : nullptr, (const float*)(q + 2 * p3),
        (h->S > 0 && scal) ? (const float*)(q + 2 * p3 + p1) : nullptr, np, ps->len[0], ps->len[1], ps->len[2],
        h->posd, h->vel4, h->w, h->scal, h->counters + CNT_DECODE);
  } else if (n_verts) {
    k_pack_xyz<<<blocks_for(n_verts, 256), 256, 0, st>>>(n_verts, sx, h->posd, 0.f);
    if (vel) k_pack_xyz<<<blocks_for(n_verts, 256), 256, 0, st>>>(n_verts, sv, h->vel4, 0.f);
    else DTFE_CUDA_TRY(cudaMemsetAsync(h->vel4, 0, sizeof(float4) * n_verts, st));
    if (h->S > 0 && !scal) DTFE_CUDA_TRY(cudaMemsetAsync(h->scal, 0, sizeof(float) * h->S * n_verts, st));
  }
  // star lists, for deriving the neighbours
  h->inc_ready = false;
  if (derive_neighbours && (rc = build_incidence(h, true))) return rc;
  // neighbours from the vertices, when they did not cross: every face at its
  // smallest vertex's star, then the few faces of very large stars
  if (n_tets && derive_neighbours) {
    DTFE_CUDA_TRY(cudaMemsetAsync(h->tet_n, 0x80, sizeof(int4) * n_tets, st));
    // after the star fill, scratch_i holds the list of large stars and
    // scratch_i[V] its count
    int* big = h->scratch_i;
    unsigned* n_big = (unsigned*)(h->scratch_i + n_verts);
    DTFE_CUDA_TRY(cudaMemsetAsync(n_big, 0, sizeof(unsigned), st));
    const int64_t want = (n_verts + 15) / 16;
    k_neighbours_star<128, 8, 64, false, true><<<(unsigned)std::min<int64_t>(want, 148 * 64), 128, 0, st>>>(
        n_verts, h->tet_v, h->inc_off, h->inc, (int*)h->tet_n, big, n_big, (unsigned)n_verts);
    k_neighbours_star<128, 32, 768, true, false><<<148 * 4, 128, 0, st>>>(
        n_verts, h->tet_v, h->inc_off, h->inc, (int*)h->tet_n, big, n_big, (unsigned)n_verts);
    k_derive_neighbours<<<blocks_for(n_tets, 256), 256, 0, st>>>(n_tets, h->tet_v, h->inc_off, h->inc, h->tet_n);
  }
  // hull vertices (a property of the tessellation's topology)
  if (n_verts) DTFE_CUDA_TRY(cudaMemsetAsync(h->hull, 0, sizeof(int) * n_verts, st));
  if (n_tets) k_hull_marks<<<blocks_for(n_tets, 256), 256, 0, st>>>(n_tets, h->tet_v, h->tet_n, h->hull);
  DTFE_CUDA_TRY(cudaGetLastError());
  h->has_vel = vel != nullptr;
  h->has_scal = scal != nullptr;
  h->rec_ready = false;
  h->scale_ready = false;
  h->density_ready = false;
  h->prep_ready = false;
  h->tet_c_valid = false;
  drop_graph(h);
  return DTFE_OK;
}
}  // extern "C++"

int dtfe_gpu_upload(dtfe_handle h, const int32_t* tet_v, const int32_t* tet_n, int64_t n_tets,
                    const float* xyz, const float* w, const float* vel, const float* scal,
                    int64_t n_verts) {
  if (n_tets > 0 && !tet_v) return set_error(DTFE_ERR_ARG, "null argument");
  return upload_impl(
      h, n_tets, xyz, w, vel, scal, n_verts, 0,
      [&](dtfe_handle hh, char*) -> int {
        DTFE_CUDA_TRY(cudaMemcpyAsync(hh->tet_v, tet_v, 16 * n_tets, cudaMemcpyHostToDevice, hh->stream));
        if (tet_n)
          DTFE_CUDA_TRY(cudaMemcpyAsync(hh->tet_n, tet_n, 16 * n_tets, cudaMemcpyHostToDevice, hh->stream));
        return DTFE_OK;
      },
      [&](dtfe_handle hh, char*) -> int {
        // every id in range before the hull, incidence and walk kernels use
        // them: the check waits for its count (the packed path's decoder
        // sanitises instead and reports at the next status read)
        unsigned long long bad = 0;
        k_check_tets<<<blocks_for(n_tets, 256), 256, 0, hh->stream>>>(n_tets, n_verts, hh->tet_v,
                                                                       tet_n ? hh->tet_n : nullptr,
                                                                       hh->counters + CNT_DECODE);
        DTFE_CUDA_TRY(cudaGetLastError());
        DTFE_CUDA_TRY(cudaMemcpyAsync(&bad, hh->counters + CNT_DECODE, sizeof(bad), cudaMemcpyDeviceToHost,
                                      hh->stream));
        DTFE_CUDA_TRY(cudaStreamSynchronize(hh->stream));
        if (bad) {
          DTFE_CUDA_TRY(cudaMemsetAsync(hh->counters + CNT_DECODE, 0, sizeof(unsigned long long), hh->stream));
          return set_error(DTFE_ERR_ARG, std::to_string(bad) + " tetrahedra with a vertex id outside [0, n_verts)"
                                         " or a neighbour id outside [-1, n_tets)");
        }
        return DTFE_OK;
      },
      tet_n == nullptr);
}

// The vertex-only packed form ("DTP3", dtfe_tets_pack_vertices): header
// magic, T, n_blocks, n_escapes, then the byte offsets of block bases, escape
// prefix, block byte offsets, width flags, orientation bits and data; the
// escapes follow the data's 16-byte aligned end.  The neighbours are derived
// on the device from the vertices.
static int upload_packed_vertices(dtfe_handle h, const int64_t hd[10], const void* packed, int64_t packed_bytes,
                                  const float* xyz, const float* w, const float* vel, const float* scal,
                                  int64_t n_verts, const ParticleSource* ps) {
  const int64_t T = hd[1], nb = hd[2], n_esc = hd[3];
  bool ok = T >= 0 && nb == (T + kPackBlock - 1) / kPackBlock && n_esc >= 0 && hd[4] >= 80 &&
            hd[5] >= hd[4] + 4 * nb && hd[6] >= hd[5] + 4 * (nb + 1) && hd[7] >= hd[6] + 8 * (nb + 1) &&
            hd[8] >= hd[7] + (T + 1) / 2 && hd[9] >= hd[8] + (T + 7) / 8 && hd[9] <= packed_bytes;
  for (int k = 4; k < 10; ++k) ok = ok && hd[k] % 16 == 0;
  int64_t data_end = 0;
  if (ok) {
    int64_t last = 0;  // byte size of the data: the last block offset
    std::memcpy(&last, (const char*)packed + hd[6] + 8 * nb, sizeof(last));
    ok = last >= 0 && last <= packed_bytes;
    data_end = hd[9] + ((last + 16 + 15) & ~(int64_t)15);
    ok = ok && data_end + 4 * n_esc <= packed_bytes;
  }
  if (!ok) return set_error(DTFE_ERR_ARG, "not a packed tessellation (dtfe_tets_pack_vertices)");
  return upload_impl(
      h, T, xyz, w, vel, scal, n_verts, (size_t)packed_bytes,
      [&](dtfe_handle hh, char* dev) -> int {
        DTFE_CUDA_TRY(cudaMemcpyAsync(dev, packed, (size_t)packed_bytes, cudaMemcpyHostToDevice, hh->stream));
        return DTFE_OK;
      },
      [&](dtfe_handle hh, char* dev) -> int {
        k_unpack_tet_vertices<<<(unsigned)nb, kPackBlock, 0, hh->stream>>>(
            T, n_verts, (const int32_t*)(dev + hd[4]), (const int32_t*)(dev + hd[5]), (const int64_t*)(dev + hd[6]),
            (const uint8_t*)(dev + hd[7]), (const uint8_t*)(dev + hd[8]), (const uint32_t*)(dev + hd[9]),
            data_end - hd[9], (const int32_t*)(dev + data_end), n_esc, hh->tet_v, hh->counters + CNT_DECODE);
        DTFE_CUDA_TRY(cudaGetLastError());
        return DTFE_OK;
      },
      true, ps);
}

static int upload_packed_any(dtfe_handle h, const void* packed, int64_t packed_bytes, const float* xyz,
                             const float* w, const float* vel, const float* scal, int64_t n_verts,
                             const ParticleSource* ps) {
  // header: magic "DTP2", T, n_blocks, n_escapes, then the byte offsets of
  // block bases, escape prefix, block byte offsets, flags, data, escapes
  int64_t hd[10];
  if (!packed || packed_bytes < (int64_t)sizeof(hd)) return set_error(DTFE_ERR_ARG, "null or short packed buffer");
  std::memcpy(hd, packed, sizeof(hd));
  if (hd[0] == 0x33505444)
    return upload_packed_vertices(h, hd, packed, packed_bytes, xyz, w, vel, scal, n_verts, ps);
  const int64_t T = hd[1], nb = hd[2], n_esc = hd[3];
  bool ok = hd[0] == 0x32505444 && T >= 0 && nb == (T + kPackBlock - 1) / kPackBlock && n_esc >= 0 &&
            hd[4] >= (int64_t)sizeof(hd) && hd[5] >= hd[4] + 4 * nb && hd[6] >= hd[5] + 4 * (nb + 1) &&
            hd[7] >= hd[6] + 8 * (nb + 1) && hd[8] >= hd[7] + T && hd[9] >= hd[8] &&
            hd[9] + 4 * n_esc <= packed_bytes;
  for (int k = 4; k < 10; ++k) ok = ok && hd[k] % 16 == 0;
  if (!ok) return set_error(DTFE_ERR_ARG, "not a packed tessellation (dtfe_tets_pack)");
  return upload_impl(
      h, T, xyz, w, vel, scal, n_verts, (size_t)packed_bytes,
      [&](dtfe_handle hh, char* dev) -> int {
        DTFE_CUDA_TRY(cudaMemcpyAsync(dev, packed, (size_t)packed_bytes, cudaMemcpyHostToDevice, hh->stream));
        return DTFE_OK;
      },
      [&](dtfe_handle hh, char* dev) -> int {
        k_unpack_tets<<<(unsigned)nb, kPackBlock, 0, hh->stream>>>(
            T, n_verts, (const int32_t*)(dev + hd[4]), (const int32_t*)(dev + hd[5]),
            (const int64_t*)(dev + hd[6]), (const uint8_t*)(dev + hd[7]), (const uint32_t*)(dev + hd[8]),
            hd[9] - hd[8], (const int32_t*)(dev + hd[9]), n_esc, hh->tet_v, hh->tet_n, hh->counters + CNT_DECODE);
        DTFE_CUDA_TRY(cudaGetLastError());
        return DTFE_OK;
      },
      false, ps);
}

int dtfe_gpu_upload_packed(dtfe_handle h, const void* packed, int64_t packed_bytes, const float* xyz,
                           const float* w, const float* vel, const float* scal, int64_t n_verts) {
  return upload_packed_any(h, packed, packed_bytes, xyz, w, vel, scal, n_verts, nullptr);
}

int dtfe_gpu_upload_packed_particles(dtfe_handle h, const void* packed, int64_t packed_bytes, const float* xyz,
                                     const float* w, const float* vel, const float* scal, int64_t n_particles,
                                     const uint32_t* vertex_codes, int64_t n_verts, const float box_length[3]) {
  if (!box_length) return set_error(DTFE_ERR_ARG, "null argument");
  ParticleSource ps{vertex_codes, n_particles, {box_length[0], box_length[1], box_length[2]}};
  return upload_packed_any(h, packed, packed_bytes, xyz, w, vel, scal, n_verts, &ps);
}

int dtfe_gpu_chain_uploads(dtfe_handle h, dtfe_handle after) {
  if (!h || after == h) return set_error(DTFE_ERR_ARG, "bad handles");
  if (after && after->device != h->device) return set_error(DTFE_ERR_ARG, "handles on different devices");
  h->upload_after = after;
  return DTFE_OK;
}

int dtfe_gpu_set_subboxes(dtfe_handle h, int32_t n_boxes, const dtfe_subbox* boxes, const float* xs,
                          int64_t n_xs, const float* ys, int64_t n_ys, const float* zs, int64_t n_zs,
                          const int32_t grid[3]) {
  if (!h || n_boxes <= 0 || !boxes || !xs || !ys || !zs || !grid)
    return set_error(DTFE_ERR_ARG, "null or empty sub-box description");
  DTFE_CUDA_TRY(cudaSetDevice(h->device));
  std::vector<int64_t> tprefix(n_boxes + 1), tetpre(n_boxes + 1), boff(n_boxes), ppre(n_boxes + 1);
  int64_t cells = 0;
  for (int b = 0; b < n_boxes; ++b) {
    const dtfe_subbox& B = boxes[b];
    for (int a = 0; a < 3; ++a) {
      int64_t nt = a == 0 ? n_xs : (a == 1 ? n_ys : n_zs);
      if (B.tile_dims[a] <= 0 || B.tile_origin[a] < 0 || B.tile_origin[a] + B.tile_dims[a] > grid[a] ||
          B.coord_offset[a] < 0 || B.coord_offset[a] + B.tile_dims[a] > nt || !(B.dx[a] > 0.f))
        return set_error(DTFE_ERR_ARG, "sub-box tile outside the grid or coordinate tables");
    }
    if (B.vert_offset < 0 || B.vert_offset + B.n_verts > h->V || B.tet_offset < 0 ||
        B.tet_offset + B.n_tets > h->T)
      return set_error(DTFE_ERR_ARG, "sub-box vertex/tetrahedron range outside the upload");
    if (b > 0 && (B.vert_offset != boxes[b - 1].vert_offset + boxes[b - 1].n_verts ||
                  B.tet_offset != boxes[b - 1].tet_offset + boxes[b - 1].n_tets))
      return set_error(DTFE_ERR_ARG, "sub-box vertex and tetrahedron ranges must be consecutive");
    tprefix[b] = cells;
    boff[b] = cells;
    ppre[b + 1] = ppre[b] + (int64_t)B.tile_dims[0] * B.tile_dims[1];
    tetpre[b] = B.tet_offset;
    cells += (int64_t)B.tile_dims[0] * B.tile_dims[1] * B.tile_dims[2];
  }
  tprefix[n_boxes] = cells;
  tetpre[n_boxes] = boxes[n_boxes - 1].tet_offset + boxes[n_boxes - 1].n_tets;
  if (cells >= kMaxCells) return set_error(DTFE_ERR_TOO_LARGE, "more than 2^31 grid cells");
  // raster formula of every tile axis, x_i ~ lo + (i + 1/2) dx, and the
  // largest deviation of its coordinate table from it (in cells): the
  // raster's index ranges widened by it cannot miss a centre
  std::vector<RasterAxis> axes((size_t)3 * n_boxes);
  for (int b = 0; b < n_boxes; ++b)
    for (int a = 0; a < 3; ++a) {
      const dtfe_subbox& B = boxes[b];
      const float* tab = (a == 0 ? xs : (a == 1 ? ys : zs)) + B.coord_offset[a];
      RasterAxis& A = axes[3 * b + a];
      A.lo = (double)B.lo[a];
      A.inv_dx = 1.0 / (double)B.dx[a];
      double dev = 0.0;
      for (int i = 0; i < B.tile_dims[a]; ++i)
        dev = std::max(dev, std::fabs(((double)tab[i] - A.lo) * A.inv_dx - 0.5 - (double)i));
      if (!(dev < 1e6)) return set_error(DTFE_ERR_ARG, "coordinate table far from the tile's raster");
      A.margin = dev + 1e-6;
    }
  int rc;
  if ((rc = dev_alloc(h, &h->raster_axes, (size_t)3 * n_boxes)) ||
      (rc = dev_alloc(h, &h->boxes, n_boxes)) || (rc = dev_alloc(h, &h->tile_prefix, n_boxes + 1)) ||
      (rc = dev_alloc(h, &h->pencil_prefix, n_boxes + 1)) ||
      (rc = dev_alloc(h, &h->tet_prefix, n_boxes + 1)) || (rc = dev_alloc(h, &h->bin_offset, n_boxes)) ||
      (rc = dev_alloc(h, &h->bins, cells)) || (rc = dev_alloc(h, &h->xs, n_xs)) ||
      (rc = dev_alloc(h, &h->ys, n_ys)) || (rc = dev_alloc(h, &h->zs, n_zs)))
    return rc;
  cudaStream_t st = h->stream;
  DTFE_CUDA_TRY(cudaMemcpyAsync(h->boxes, boxes, sizeof(dtfe_subbox) * n_boxes, cudaMemcpyHostToDevice, st));
  DTFE_CUDA_TRY(cudaMemcpyAsync(h->tile_prefix, tprefix.data(), sizeof(int64_t) * (n_boxes + 1),
                                cudaMemcpyHostToDevice, st));
  DTFE_CUDA_TRY(cudaMemcpyAsync(h->pencil_prefix, ppre.data(), sizeof(int64_t) * (n_boxes + 1),
                                cudaMemcpyHostToDevice, st));
  DTFE_CUDA_TRY(cudaMemcpyAsync(h->tet_prefix, tetpre.data(), sizeof(int64_t) * (n_boxes + 1),
                                cudaMemcpyHostToDevice, st));
  DTFE_CUDA_TRY(cudaMemcpyAsync(h->bin_offset, boff.data(), sizeof(int64_t) * n_boxes, cudaMemcpyHostToDevice, st));
  DTFE_CUDA_TRY(cudaMemcpyAsync(h->xs, xs, sizeof(float) * n_xs, cudaMemcpyHostToDevice, st));
  DTFE_CUDA_TRY(cudaMemcpyAsync(h->ys, ys, sizeof(float) * n_ys, cudaMemcpyHostToDevice, st));
  DTFE_CUDA_TRY(cudaMemcpyAsync(h->zs, zs, sizeof(float) * n_zs, cudaMemcpyHostToDevice, st));
  DTFE_CUDA_TRY(cudaMemcpyAsync(h->raster_axes, axes.data(), sizeof(RasterAxis) * axes.size(),
                                cudaMemcpyHostToDevice, st));
  DTFE_CUDA_TRY(cudaStreamSynchronize(st));  // host vectors go out of scope
  h->K = n_boxes;
  h->boxes_h.assign(boxes, boxes + n_boxes);
  h->regions_h.resize((size_t)6 * n_boxes);
  for (int b = 0; b < n_boxes; ++b)
    for (int a = 0; a < 3; ++a) {
      h->regions_h[6 * b + 2 * a] = boxes[b].lo[a];
      h->regions_h[6 * b + 2 * a + 1] = boxes[b].lo[a] + boxes[b].dx[a] * (float)boxes[b].tile_dims[a];
    }
  h->n_cells = cells;
  h->n_pencils = ppre[n_boxes];
  h->scale_ready = false;  // the exact sums' units are per sub-box
  h->grid[0] = grid[0]; h->grid[1] = grid[1]; h->grid[2] = grid[2];
  h->prep_ready = false;
  h->eq_nn = 0;
  drop_graph(h);
  return DTFE_OK;
}

int dtfe_gpu_set_regions(dtfe_handle h, int32_t n_boxes, const float* regions) {
  if (!h || !regions) return set_error(DTFE_ERR_ARG, "null argument");
  if (n_boxes != h->K) return set_error(DTFE_ERR_STATE, "regions must follow dtfe_gpu_set_subboxes, one per sub-box");
  for (int b = 0; b < n_boxes; ++b)
    for (int a = 0; a < 3; ++a) {
      const float lo = regions[6 * b + 2 * a], hi = regions[6 * b + 2 * a + 1];
      if (lo != h->boxes_h[b].lo[a] || !(hi >= lo))
        return set_error(DTFE_ERR_ARG, "region lower corner differs from the sub-box's lo, or hi < lo");
    }
  h->regions_h.assign(regions, regions + (size_t)6 * n_boxes);
  return DTFE_OK;
}

int dtfe_gpu_vertex_density(dtfe_handle h, double rho_bar) {
  if (!h) return set_error(DTFE_ERR_ARG, "null handle");
  if (!(rho_bar > 0.0)) return set_error(DTFE_ERR_ARG, "averageDensity must be positive");
  if (h->V == 0) return set_error(DTFE_ERR_STATE, "nothing uploaded");
  DTFE_CUDA_TRY(cudaSetDevice(h->device));
  cudaStream_t st = h->stream;
  int rc = launch_prep(h);
  if (rc) return rc;
  // the reference's factor: (NO_DIM+1.)/averageDensity stored as Real
  float rb = (float)rho_bar;
  float factor = (float)(4.0 / (double)rb);
  h->factor = factor;
  k_vertex_density<<<blocks_for(h->V, kDensBlock), kDensBlock, 0, st>>>(h->V, h->w, h->vacc, h->hull, h->vscale,
                                                                       h->sb_vprefix, h->nsb, factor, h->posd);
  DTFE_CUDA_TRY(cudaGetLastError());
  h->density_ready = true;
  return DTFE_OK;
}

int dtfe_gpu_download_vertex_density(dtfe_handle h, float* dens) {
  if (!h || !dens) return set_error(DTFE_ERR_ARG, "null argument");
  if (!h->density_ready) return set_error(DTFE_ERR_STATE, "vertex density not computed");
  DTFE_CUDA_TRY(cudaSetDevice(h->device));
  // .w of each float4: strided copy
  DTFE_CUDA_TRY(cudaMemcpy2DAsync(dens, sizeof(float), (const char*)h->posd + 12, sizeof(float4),
                                  sizeof(float), h->V, cudaMemcpyDeviceToHost, h->stream));
  DTFE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return DTFE_OK;
}

// Validation, one-time set-up and every launch of one interpolation on the
// handle's stream; nothing waits for the GPU after the set-up, so the
// launches can be captured into a graph once the set-up has run.
int dtfe_internal_method1(void* stream, int K, const dtfe_subbox* boxes_h, const dtfe_subbox* boxes_d,
                          const float* regions_h, int64_t n_cells, int64_t G1, int64_t G2, int64_t T,
                          const int4* tet_v, const float4* posd, const float4* vel4, const float* scal, int S, int NN,
                          uint32_t fields, int fix, float* const out[DTFE_NUM_FIELDS], double** table, int* table_nn,
                          void** scratch, size_t* scratch_bytes, void** lists, size_t* lists_bytes);

static int interp_enqueue(dtfe_handle h, const dtfe_interp_opts* o, float* const out_dev[DTFE_NUM_FIELDS]) {
  if (!h || !o) return set_error(DTFE_ERR_ARG, "null argument");
  if (h->K == 0) return set_error(DTFE_ERR_STATE, "sub-boxes not set");
  if (h->T == 0) return set_error(DTFE_ERR_DEGENERATE, "no tetrahedra");
  if (!h->density_ready) return set_error(DTFE_ERR_STATE, "vertex density not computed");
  int method = o->method;
  if (method != DTFE_METHOD_CENTRE && method != DTFE_METHOD_TETRAHEDRA && method != DTFE_METHOD_MONTE_CARLO &&
      method != DTFE_METHOD_EQUIDISTANT)
    return set_error(DTFE_ERR_ARG, "unknown method");
  int NN = method == DTFE_METHOD_CENTRE ? 1 : o->n_samples;
  if (NN < 1) return set_error(DTFE_ERR_ARG, "n_samples must be >= 1");
  uint32_t F = o->fields;
  if (F >> DTFE_NUM_FIELDS) return set_error(DTFE_ERR_ARG, "unknown field bits");
  if ((F & DTFE_FIELD_BIT(DTFE_VELOCITY_STD)) && method != DTFE_METHOD_MONTE_CARLO)
    return set_error(DTFE_ERR_ARG, "velocity_std needs the Monte-Carlo method");
  if (h->S == 0 && (F & (DTFE_FIELD_BIT(DTFE_SCALAR) | DTFE_FIELD_BIT(DTFE_SCALAR_GRADIENT))))
    return set_error(DTFE_ERR_ARG, "scalar fields requested but n_scalars == 0");
  for (int s = 0; s < DTFE_NUM_FIELDS; ++s)
    if ((F >> s & 1u) && !out_dev[s]) return set_error(DTFE_ERR_ARG, "missing output buffer");
  if (method == DTFE_METHOD_TETRAHEDRA) {
    // points inside the tetrahedra, gathered per cell (method1.cu)
    DTFE_CUDA_TRY(cudaMemsetAsync(h->counters, 0, sizeof(unsigned long long) * CNT_N, h->stream));
    float* outs[DTFE_NUM_FIELDS];
    for (int s = 0; s < DTFE_NUM_FIELDS; ++s) outs[s] = (F >> s & 1u) ? out_dev[s] : nullptr;
    const int rc1 = dtfe_internal_method1(h->stream, h->K, h->boxes_h.data(), h->boxes, h->regions_h.data(),
                                          h->n_cells, h->grid[1], h->grid[2], h->T, h->tet_v, h->posd,
                                          h->has_vel ? h->vel4 : nullptr, h->S > 0 ? h->scal : nullptr, h->S, NN,
                                          F, (o->flags & DTFE_FLAG_FIX_VALUE_INTERP) ? 1 : 0, outs, &h->m1_table,
                                          &h->m1_table_nn, &h->m1_scratch, &h->m1_bytes, &h->m1_lists,
                                          &h->m1_lists_bytes);
    h->tet_c_valid = false;
    return rc1;
  }
  int rc = prepare_centres(h);
  if (rc) return rc;
  cudaStream_t st = h->stream;
  if (method == DTFE_METHOD_EQUIDISTANT) {
    int n = (int)std::lround(std::cbrt((double)NN));
    if (n * n * n != NN) return set_error(DTFE_ERR_ARG, "equidistant sampling needs a perfect cube");
    if (h->eq_nn != NN) {
      // equidistant offsets (averaged_interpolation_2.cc:726-740), per sub-box
      std::vector<float> eq((size_t)h->K * NN * 3);
      for (int b = 0; b < h->K; ++b) {
        const float* dx = h->boxes_h[b].dx;
        for (int i1 = 0; i1 < n; ++i1)
          for (int i2 = 0; i2 < n; ++i2)
            for (int i3 = 0; i3 < n; ++i3) {
              int idx = i1 * n * n + i2 * n + i3;
              float* e = &eq[((size_t)b * NN + idx) * 3];
              e[2] = (float)((i3 + 0.5) * (double)dx[2] / n - (double)dx[2] / 2.);
              e[0] = (float)((i1 + 0.5) * (double)dx[0] / n - (double)dx[0] / 2.);
              e[1] = (float)((i2 + 0.5) * (double)dx[1] / n - (double)dx[1] / 2.);
            }
      }
      if ((rc = dev_alloc(h, &h->eq_off, eq.size()))) return rc;
      DTFE_CUDA_TRY(cudaMemcpyAsync(h->eq_off, eq.data(), sizeof(float) * eq.size(), cudaMemcpyHostToDevice, st));
      DTFE_CUDA_TRY(cudaStreamSynchronize(st));
      h->eq_nn = NN;
    }
  }
  DTFE_CUDA_TRY(cudaMemsetAsync(h->counters, 0, sizeof(unsigned long long) * CNT_N, st));
  InterpParams P;
  if (uses_records(h->loc_variant) && method == DTFE_METHOD_CENTRE && !h->rec_ready) {
    if ((rc = dev_alloc(h, &h->tet_rec, 2 * (size_t)h->T))) return rc;
    k_build_records<<<blocks_for(h->T, 256), 256, 0, st>>>(h->T, h->tet_v, h->tet_n, h->tet_rec);
    DTFE_CUDA_TRY(cudaGetLastError());
    h->rec_ready = true;
  }
  P.tet_v = h->tet_v;
  P.tet_n = h->tet_n;
  P.tet_rec = h->tet_rec;
  P.posd = h->posd;
  P.vel4 = h->vel4;
  P.scal = h->scal;
  P.bins = h->bins;
  P.boxes = h->boxes;
  P.tile_prefix = h->tile_prefix;
  P.bin_offset = h->bin_offset;
  P.eq_off = h->eq_off;
  P.xs = h->xs;
  P.ys = h->ys;
  P.zs = h->zs;
  P.K = h->K;
  P.pencil_prefix = h->pencil_prefix;
  P.S = h->S;
  P.G1 = h->grid[1];
  P.G2 = h->grid[2];
  P.n_total = h->n_cells;
  P.NN = NN;
  P.seed = o->seed;
  P.fields = F;
  P.fix = (o->flags & DTFE_FLAG_FIX_VALUE_INTERP) ? 1 : 0;
  P.max_steps = h->max_steps;
  P.count_centres = is_raster(h->loc_variant) ? 1 : 0;
  for (int s = 0; s < DTFE_NUM_FIELDS; ++s) P.out[s] = (F >> s & 1u) ? out_dev[s] : nullptr;
  P.counters = h->counters;
  const unsigned block = kInterpBlock;
  unsigned grid = blocks_for(h->n_cells, block);
  // every output must be 16-byte aligned for the staged stores
  for (int q = 0; q < DTFE_NUM_FIELDS; ++q)
    if (P.out[q] && ((uintptr_t)P.out[q] & 15))
      return set_error(DTFE_ERR_ARG, "output buffers must be 16-byte aligned");
  if ((rc = dev_alloc(h, &h->tet_c, h->n_cells))) return rc;
  const bool fused = is_fused(h->loc_variant) && method == DTFE_METHOD_CENTRE;
  if (fused) {
    launch_fused_s(h->S, h->loc_variant - kFirstFused, P, h->tet_c, st, grid, block);
  } else {
    launch_locate(is_fused(h->loc_variant) ? kNumRasterVariants : h->loc_variant, P, h->tet_c, st);
    launch_eval_s(method, h->S, h->eval_variant, P, h->tet_c, st, grid, block);
  }
  // the reference's raster after an outside sample (DTFE_FLAG_FIX_OUTSIDE_RASTER: off)
  if (method == DTFE_METHOD_CENTRE && !(o->flags & DTFE_FLAG_FIX_OUTSIDE_RASTER) && h->n_pencils > 0) {
    const int64_t want = (h->n_pencils * 32 + 255) / 256;
    k_outside_pencils<<<(unsigned)std::min<int64_t>(want, 148 * 16), 256, 0, st>>>(P, h->tet_c, h->n_pencils);
  }
  h->tet_c_valid = method == DTFE_METHOD_CENTRE;  // the adjoint differentiates centre values only
  h->tet_c_fix = (o->flags & DTFE_FLAG_FIX_VALUE_INTERP) != 0;
  DTFE_CUDA_TRY(cudaGetLastError());
  return DTFE_OK;
}

static int read_status(dtfe_handle h, dtfe_status* status) {
  cudaStream_t st = h->stream;
  unsigned long long cnt[CNT_ALL];
  DTFE_CUDA_TRY(cudaMemcpyAsync(cnt, h->counters, sizeof(cnt), cudaMemcpyDeviceToHost, st));
  DTFE_CUDA_TRY(cudaStreamSynchronize(st));
  if (status) {
    status->n_samples_located = (int64_t)cnt[CNT_LOCATED];
    status->n_outside = (int64_t)cnt[CNT_OUTSIDE];
    status->n_walk_failures = (int64_t)cnt[CNT_FAIL];
    status->n_walk_steps = (int64_t)cnt[CNT_STEPS];
    status->n_exact_tests = (int64_t)(cnt[CNT_EXACT] + cnt[CNT_RASTER_EXACT]);
    status->n_ties = (int64_t)(cnt[CNT_TIES] + cnt[CNT_RASTER_TIES]);
  }
  if (cnt[CNT_DECODE]) return set_error(DTFE_ERR_ARG, "packed tessellation did not decode (malformed buffer)");
  if (cnt[CNT_FAIL]) return set_error(DTFE_ERR_WALK, "point-location walk hit its step limit");
  return DTFE_OK;
}

static int interpolate_impl(dtfe_handle h, const dtfe_interp_opts* o, float* const out_dev[DTFE_NUM_FIELDS],
                            dtfe_status* status) {
  int rc = interp_enqueue(h, o, out_dev);
  if (rc) return rc;
  return read_status(h, status);
}

// Times every launch variant of the locate and evaluation kernels on the
// loaded data (cell-centre method, the given fields, into scratch outputs) and
// keeps the fastest of each.  chosen (may be NULL) receives the two indices.
static int autotune_impl(dtfe_handle h, uint32_t fields, int32_t* chosen) {
  if (!h->density_ready) return set_error(DTFE_ERR_STATE, "vertex density not computed");
  if (h->K == 0) return set_error(DTFE_ERR_STATE, "sub-boxes not set");
  const int64_t G = (int64_t)h->grid[0] * h->grid[1] * h->grid[2];
  float* dev[DTFE_NUM_FIELDS] = {};
  for (int s = 0; s < DTFE_NUM_FIELDS; ++s) {
    if (!(fields >> s & 1u)) continue;
    size_t need = (size_t)G * field_components(s, h->S);
    int rc = dev_alloc(h, &h->out_buf[s], need);
    if (rc) return rc;
    h->out_cap[s] = std::max(h->out_cap[s], need);
    dev[s] = h->out_buf[s];
  }
  dtfe_interp_opts o = {DTFE_METHOD_CENTRE, 1, 0, fields, 0};
  cudaEvent_t e0, e1;
  DTFE_CUDA_TRY(cudaEventCreate(&e0));
  DTFE_CUDA_TRY(cudaEventCreate(&e1));
  // every timed call redoes the per-step preparation (volumes and centre
  // raster or walk seeds), so that the locate variants compare whole steps
  auto time_call = [&](float* ms) -> int {
    h->prep_ready = false;
    int rc = interpolate_impl(h, &o, dev, nullptr);  // warm
    if (rc) return rc;
    float best = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
      h->prep_ready = false;
      cudaEventRecord(e0, h->stream);
      rc = interpolate_impl(h, &o, dev, nullptr);
      if (rc) return rc;
      cudaEventRecord(e1, h->stream);
      cudaEventSynchronize(e1);
      float t = 0.f;
      cudaEventElapsedTime(&t, e0, e1);
      best = std::min(best, t);
    }
    *ms = best;
    return DTFE_OK;
  };
  int rc = DTFE_OK;
  float best = 1e30f;
  int best_loc = 0, best_eval = 0;
  h->eval_variant = 0;
  for (int v = 0; v < kNumLocVariants && !rc; ++v) {
    h->loc_variant = v;
    float t;
    rc = time_call(&t);
    if (!rc && t < best) { best = t; best_loc = v; }
  }
  h->loc_variant = best_loc;
  best = 1e30f;
  for (int v = 0; v < kNumEvalVariants && !rc; ++v) {
    h->eval_variant = v;
    float t;
    rc = time_call(&t);
    if (!rc && t < best) { best = t; best_eval = v; }
  }
  h->eval_variant = best_eval;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (chosen) {
    chosen[0] = best_loc;
    chosen[1] = best_eval;
  }
  return rc;
}

int dtfe_gpu_autotune(dtfe_handle h, uint32_t fields, int32_t* chosen) {
  if (!h) return set_error(DTFE_ERR_ARG, "null handle");
  DTFE_CUDA_TRY(cudaSetDevice(h->device));
  return autotune_impl(h, fields, chosen);
}

int dtfe_gpu_variant_counts(int32_t counts[2]) {
  if (!counts) return set_error(DTFE_ERR_ARG, "null argument");
  counts[0] = kNumLocVariants;
  counts[1] = kNumEvalVariants;
  return DTFE_OK;
}

int dtfe_gpu_set_variants(dtfe_handle h, int32_t locate_variant, int32_t eval_variant) {
  if (!h) return set_error(DTFE_ERR_ARG, "null handle");
  if (locate_variant < 0 || locate_variant >= kNumLocVariants || eval_variant < 0 ||
      eval_variant >= kNumEvalVariants)
    return set_error(DTFE_ERR_ARG, "unknown launch variant");
  h->loc_variant = locate_variant;
  h->eval_variant = eval_variant;
  return DTFE_OK;
}

int dtfe_gpu_deposit_impl(void* stream, int32_t kind, const float* xyz, const float* w, const float* vel, int64_t n,
                          int32_t n_boxes, const dtfe_deposit_box* boxes, const int32_t grid[3],
                          double average_density, float* density_dev, float* velocity_dev, void** scratch,
                          size_t* scratch_bytes, void* saved, int inputs_dev);
int dtfe_gpu_deposit_adjoint_impl(void* stream, const void* saved, const float* a_dev, float* gx_dev, float* gw_dev);
int dtfe_internal_adjoint(void* stream, const void* cell_params, int64_t n_cells, int64_t V, int64_t T,
                          const int4* tet_v, const float4* posd, const float* w, const int* hull,
                          const long long* vacc, const VolScale* vscale, const int64_t* vprefix, int nsb,
                          const int64_t* off, const int* inc, float factor, double* g_rho, double* g_x, double* g_v,
                          double* g_S, double* g_m, double* vbar, float* out_x, float* out_v, float* out_w);
size_t dtfe_internal_adjoint_params_size();
int dtfe_internal_sph(void* stream, int K, const dtfe_subbox* boxes_h, const dtfe_subbox* boxes_d,
                      const int64_t* tile_prefix_d, int64_t n_cells, int64_t G1, int64_t G2, const float* xs,
                      const float* ys, const float* zs, int64_t V, const float4* posd, const float* w,
                      const float4* vel4, const float* scal, int S, int k, uint32_t fields, int extensive,
                      double average_density, float* dens_out, float* vel_out, float* scal_out, void** scratch,
                      size_t* scratch_bytes);
void dtfe_internal_adjoint_fill_params(void* out, const int4* tet_v, const float4* posd, const float4* vel4,
                                       const int* tet_c, const dtfe_subbox* boxes, const int64_t* tile_prefix,
                                       const float* xs, const float* ys, const float* zs, int K, int64_t G1,
                                       int64_t G2, int64_t n_total, const float* a, const float* b,
                                       const float* c, int full_value);

static int deposit_common(dtfe_handle h, int32_t kind, const float* xyz, const float* w, const float* vel,
                          int64_t n, int32_t n_boxes, const dtfe_deposit_box* boxes, const int32_t grid[3],
                          double average_density, float* density_dev, float* velocity_dev, int inputs_dev) {
  if (!h || !grid || (n > 0 && !xyz)) return set_error(DTFE_ERR_ARG, "null argument");
  DTFE_CUDA_TRY(cudaSetDevice(h->device));
  int64_t G = (int64_t)grid[0] * grid[1] * grid[2];
  if (density_dev) DTFE_CUDA_TRY(cudaMemsetAsync(density_dev, 0, sizeof(float) * G, h->stream));
  if (velocity_dev) DTFE_CUDA_TRY(cudaMemsetAsync(velocity_dev, 0, sizeof(float) * 3 * G, h->stream));
  int rc = dtfe_gpu_deposit_impl(h->stream, kind, xyz, w, vel, n, n_boxes, boxes, grid, average_density,
                                 density_dev, velocity_dev, &h->dep_scratch, &h->dep_bytes, h->dep_saved,
                                 inputs_dev);
  if (rc) return rc;
  DTFE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return DTFE_OK;
}

int dtfe_gpu_deposit_dev(dtfe_handle h, int32_t kind, const float* xyz, const float* w, const float* vel, int64_t n,
                         int32_t n_boxes, const dtfe_deposit_box* boxes, const int32_t grid[3],
                         double average_density, float* density_dev, float* velocity_dev) {
  return deposit_common(h, kind, xyz, w, vel, n, n_boxes, boxes, grid, average_density, density_dev, velocity_dev,
                        0);
}

int dtfe_gpu_deposit_resident(dtfe_handle h, int32_t kind, const float* xyz_dev, const float* w_dev,
                              const float* vel_dev, int64_t n, int32_t n_boxes, const dtfe_deposit_box* boxes,
                              const int32_t grid[3], double average_density, float* density_dev,
                              float* velocity_dev) {
  return deposit_common(h, kind, xyz_dev, w_dev, vel_dev, n, n_boxes, boxes, grid, average_density, density_dev,
                        velocity_dev, 1);
}

int dtfe_gpu_deposit(dtfe_handle h, int32_t kind, const float* xyz, const float* w, const float* vel, int64_t n,
                     int32_t n_boxes, const dtfe_deposit_box* boxes, const int32_t grid[3], double average_density,
                     float* density, float* velocity) {
  if (!h || !grid) return set_error(DTFE_ERR_ARG, "null argument");
  DTFE_CUDA_TRY(cudaSetDevice(h->device));
  int64_t G = (int64_t)grid[0] * grid[1] * grid[2];
  int rc = dev_alloc(h, &h->dep_out, 4 * (size_t)G);
  if (rc) return rc;
  float* dd = density ? h->dep_out : nullptr;
  float* dv = velocity ? h->dep_out + G : nullptr;
  rc = dtfe_gpu_deposit_dev(h, kind, xyz, w, vel, n, n_boxes, boxes, grid, average_density, dd, dv);
  if (rc) return rc;
  if (density) DTFE_CUDA_TRY(cudaMemcpyAsync(density, dd, sizeof(float) * G, cudaMemcpyDeviceToHost, h->stream));
  if (velocity) DTFE_CUDA_TRY(cudaMemcpyAsync(velocity, dv, sizeof(float) * 3 * G, cudaMemcpyDeviceToHost, h->stream));
  DTFE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return DTFE_OK;
}

int dtfe_gpu_adjoint_dev(dtfe_handle h, const float* grad_density_dev, const float* grad_velocity_dev,
                         const float* grad_divergence_dev, float* grad_xyz_dev, float* grad_vel_dev,
                         float* grad_w_dev) {
  if (!h || !grad_xyz_dev) return set_error(DTFE_ERR_ARG, "null argument");
  if (!h->density_ready || !h->tet_c_valid)
    return set_error(DTFE_ERR_STATE, "adjoint needs a preceding vertex density and cell-centre interpolation");
  DTFE_CUDA_TRY(cudaSetDevice(h->device));
  int rc;
  if ((rc = dev_alloc(h, &h->g_rho, h->V)) || (rc = dev_alloc(h, &h->g_x, 3 * h->V)) ||
      (rc = dev_alloc(h, &h->g_v, 3 * h->V)) || (rc = dev_alloc(h, &h->g_S, h->V)) ||
      (rc = dev_alloc(h, &h->g_m, h->V)) || (rc = dev_alloc(h, &h->vbar, h->T)))
    return rc;
  alignas(16) char params[512];
  if (dtfe_internal_adjoint_params_size() > sizeof(params)) return set_error(DTFE_ERR_STATE, "params size");
  dtfe_internal_adjoint_fill_params(params, h->tet_v, h->posd, h->vel4, h->tet_c, h->boxes, h->tile_prefix, h->xs,
                                    h->ys, h->zs, h->K, h->grid[1], h->grid[2], h->n_cells, grad_density_dev,
                                    grad_divergence_dev, grad_velocity_dev, h->tet_c_fix ? 1 : 0);
  // the volume-gradient gather runs over the incidence lists (built once per upload)
  if (!h->inc_ready && (rc = build_incidence(h))) return rc;
  rc = dtfe_internal_adjoint(h->stream, params, h->n_cells, h->V, h->T, h->tet_v, h->posd, h->w, h->hull, h->vacc,
                             h->vscale, h->sb_vprefix, h->nsb, h->inc_off, h->inc, h->factor, h->g_rho, h->g_x,
                             h->g_v, h->g_S, h->g_m, h->vbar, grad_xyz_dev, grad_vel_dev, grad_w_dev);
  if (rc) return set_error(rc, "adjoint kernels failed");
  DTFE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return DTFE_OK;
}

int dtfe_gpu_sph_dev(dtfe_handle h, int32_t n_neighbors, uint32_t fields, int32_t extensive,
                     double average_density, float* density_dev, float* velocity_dev, float* scalar_dev) {
  if (!h) return set_error(DTFE_ERR_ARG, "null handle");
  if (h->K == 0 || h->V == 0) return set_error(DTFE_ERR_STATE, "upload and sub-boxes needed");
  if (fields & ~(DTFE_FIELD_BIT(DTFE_DENSITY) | DTFE_FIELD_BIT(DTFE_VELOCITY) | DTFE_FIELD_BIT(DTFE_SCALAR)))
    return set_error(DTFE_ERR_ARG, "SPH computes density, velocity and scalar fields only");
  DTFE_CUDA_TRY(cudaSetDevice(h->device));
  const int64_t G = (int64_t)h->grid[0] * h->grid[1] * h->grid[2];
  if (density_dev) DTFE_CUDA_TRY(cudaMemsetAsync(density_dev, 0, sizeof(float) * G, h->stream));
  if (velocity_dev) DTFE_CUDA_TRY(cudaMemsetAsync(velocity_dev, 0, sizeof(float) * 3 * G, h->stream));
  if (scalar_dev && h->S) DTFE_CUDA_TRY(cudaMemsetAsync(scalar_dev, 0, sizeof(float) * h->S * G, h->stream));
  int rc = dtfe_internal_sph(h->stream, h->K, h->boxes_h.data(), h->boxes, h->tile_prefix, h->n_cells, h->grid[1],
                             h->grid[2], h->xs, h->ys, h->zs, h->V, h->posd, h->w, h->vel4, h->scal, h->S,
                             n_neighbors, fields, extensive, average_density,
                             (fields & DTFE_FIELD_BIT(DTFE_DENSITY)) ? density_dev : nullptr, velocity_dev,
                             scalar_dev, &h->sph_scratch, &h->sph_bytes);
  if (rc) return rc;
  DTFE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return DTFE_OK;
}

int dtfe_gpu_sph(dtfe_handle h, int32_t n_neighbors, uint32_t fields, int32_t extensive, double average_density,
                 float* density, float* velocity, float* scalar) {
  if (!h) return set_error(DTFE_ERR_ARG, "null handle");
  DTFE_CUDA_TRY(cudaSetDevice(h->device));
  const int64_t G = (int64_t)h->grid[0] * h->grid[1] * h->grid[2];
  const bool wv = (fields & DTFE_FIELD_BIT(DTFE_VELOCITY)) != 0, ws = (fields & DTFE_FIELD_BIT(DTFE_SCALAR)) != 0;
  if ((wv && !velocity) || (ws && !scalar) || ((fields & DTFE_FIELD_BIT(DTFE_DENSITY)) && !density))
    return set_error(DTFE_ERR_ARG, "missing output buffer");
  int rc = dev_alloc(h, &h->sph_out, (size_t)(1 + 3 + h->S) * G);
  if (rc) return rc;
  float* dd = h->sph_out;
  float* dv = wv ? h->sph_out + G : nullptr;
  float* ds = ws ? h->sph_out + 4 * G : nullptr;
  rc = dtfe_gpu_sph_dev(h, n_neighbors, fields, extensive, average_density, dd, dv, ds);
  if (rc) return rc;
  if (density && (fields & DTFE_FIELD_BIT(DTFE_DENSITY)))
    DTFE_CUDA_TRY(cudaMemcpyAsync(density, dd, sizeof(float) * G, cudaMemcpyDeviceToHost, h->stream));
  if (dv) DTFE_CUDA_TRY(cudaMemcpyAsync(velocity, dv, sizeof(float) * 3 * G, cudaMemcpyDeviceToHost, h->stream));
  if (ds) DTFE_CUDA_TRY(cudaMemcpyAsync(scalar, ds, sizeof(float) * h->S * G, cudaMemcpyDeviceToHost, h->stream));
  DTFE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return DTFE_OK;
}

int dtfe_gpu_deposit_adjoint_dev(dtfe_handle h, const float* grad_density_dev, float* grad_xyz_dev,
                                 float* grad_w_dev) {
  if (!h || !grad_density_dev) return set_error(DTFE_ERR_ARG, "null argument");
  DTFE_CUDA_TRY(cudaSetDevice(h->device));
  int rc = dtfe_gpu_deposit_adjoint_impl(h->stream, h->dep_saved, grad_density_dev, grad_xyz_dev, grad_w_dev);
  if (rc) return rc;
  DTFE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return DTFE_OK;
}

int dtfe_gpu_interpolate_dev(dtfe_handle h, const dtfe_interp_opts* opts,
                             float* const out_dev[DTFE_NUM_FIELDS], dtfe_status* st) {
  if (!h) return set_error(DTFE_ERR_ARG, "null handle");
  DTFE_CUDA_TRY(cudaSetDevice(h->device));
  return interpolate_impl(h, opts, out_dev, st);
}

}  // extern "C"

namespace {

// Argument checks shared by the point-sample entry points (user points,
// redshift cones): one sub-box with its vertex densities, the centre method,
// known fields with their output buffers.
int check_point_call(dtfe_handle h, const dtfe_interp_opts* o, float* const out[DTFE_NUM_FIELDS], const char* what,
                     bool centre_ok = true, bool average_ok = false) {
  const bool centre = o->method == DTFE_METHOD_CENTRE, average = o->method == DTFE_METHOD_MONTE_CARLO;
  if (!((centre && centre_ok) || (average && average_ok)))
    return set_error(DTFE_ERR_ARG, std::string(what) + (average_ok ? (centre_ok ? " take the centre or the Monte-Carlo method"
                                                                                : " take the Monte-Carlo method")
                                                                   : " take the centre method"));
  if (average && o->n_samples < 1) return set_error(DTFE_ERR_ARG, "Monte-Carlo averages need n_samples >= 1");
  if (h->K != 1)
    return set_error(DTFE_ERR_STATE,
                     std::string(what) + " need one sub-box (the reference runs them without the split)");
  if (!h->density_ready) return set_error(DTFE_ERR_STATE, "vertex density not computed");
  const uint32_t F = o->fields;
  if ((F >> DTFE_NUM_FIELDS) || (F & DTFE_FIELD_BIT(DTFE_VELOCITY_STD)))
    return set_error(DTFE_ERR_ARG, std::string("unknown field bits or velocity_std at ") + what);
  if (h->S == 0 && (F & (DTFE_FIELD_BIT(DTFE_SCALAR) | DTFE_FIELD_BIT(DTFE_SCALAR_GRADIENT))))
    return set_error(DTFE_ERR_ARG, "scalar fields requested but n_scalars == 0");
  for (int q = 0; q < DTFE_NUM_FIELDS; ++q)
    if ((F >> q & 1u) && !out[q]) return set_error(DTFE_ERR_ARG, "missing output buffer");
  return DTFE_OK;
}

size_t point_components(dtfe_handle h, uint32_t F) {
  size_t comps = 0;
  for (int q = 0; q < DTFE_NUM_FIELDS; ++q)
    if (F >> q & 1u) comps += (size_t)field_components(q, h->S);
  return comps;
}

// Interpolation parameters of a point-sample launch: the handle's single
// sub-box, outputs staged field after field in h->pts_out (`rows` rows each).
InterpParams point_params(dtfe_handle h, const dtfe_interp_opts* o, int64_t rows) {
  InterpParams P;
  std::memset(&P, 0, sizeof(P));
  P.tet_v = h->tet_v;
  P.tet_n = h->tet_n;
  P.posd = h->posd;
  P.vel4 = h->vel4;
  P.scal = h->scal;
  P.bins = h->bins;
  P.boxes = h->boxes;
  P.tile_prefix = h->tile_prefix;
  P.bin_offset = h->bin_offset;
  P.K = h->K;
  P.G1 = h->grid[1];
  P.G2 = h->grid[2];
  P.fields = o->fields;
  P.fix = (o->flags & DTFE_FLAG_FIX_VALUE_INTERP) ? 1 : 0;
  P.max_steps = h->max_steps;
  P.counters = h->counters;
  P.S = h->S;
  size_t at = 0;
  for (int q = 0; q < DTFE_NUM_FIELDS; ++q) {
    if (!(o->fields >> q & 1u)) continue;
    P.out[q] = h->pts_out + at * (size_t)rows;
    at += (size_t)field_components(q, h->S);
  }
  return P;
}

template <class Src>
void launch_points_eval(dtfe_handle h, const InterpParams& P, int64_t n, const Src& src, int use_bins,
                        int* tet_out) {
  const unsigned g = blocks_for(n, 256);
  cudaStream_t st = h->stream;
  switch (h->S) {
    case 0: k_points_eval<0, Src><<<g, 256, 0, st>>>(P, n, src, use_bins, tet_out); break;
    case 1: k_points_eval<1, Src><<<g, 256, 0, st>>>(P, n, src, use_bins, tet_out); break;
    case 2: k_points_eval<2, Src><<<g, 256, 0, st>>>(P, n, src, use_bins, tet_out); break;
    case 3: k_points_eval<3, Src><<<g, 256, 0, st>>>(P, n, src, use_bins, tet_out); break;
    case 4: k_points_eval<4, Src><<<g, 256, 0, st>>>(P, n, src, use_bins, tet_out); break;
    case 5: k_points_eval<5, Src><<<g, 256, 0, st>>>(P, n, src, use_bins, tet_out); break;
    case 6: k_points_eval<6, Src><<<g, 256, 0, st>>>(P, n, src, use_bins, tet_out); break;
    case 7: k_points_eval<7, Src><<<g, 256, 0, st>>>(P, n, src, use_bins, tet_out); break;
    default: k_points_eval<8, Src><<<g, 256, 0, st>>>(P, n, src, use_bins, tet_out); break;
  }
}

template <class Src>
void launch_points_average(dtfe_handle h, const InterpParams& P, int64_t n, const Src& src, int use_bins,
                           uint64_t key) {
  const unsigned g = blocks_for(n, 256);
  cudaStream_t st = h->stream;
  switch (h->S) {
    case 0: k_points_average<0, Src><<<g, 256, 0, st>>>(P, n, src, use_bins, key); break;
    case 1: k_points_average<1, Src><<<g, 256, 0, st>>>(P, n, src, use_bins, key); break;
    case 2: k_points_average<2, Src><<<g, 256, 0, st>>>(P, n, src, use_bins, key); break;
    case 3: k_points_average<3, Src><<<g, 256, 0, st>>>(P, n, src, use_bins, key); break;
    case 4: k_points_average<4, Src><<<g, 256, 0, st>>>(P, n, src, use_bins, key); break;
    case 5: k_points_average<5, Src><<<g, 256, 0, st>>>(P, n, src, use_bins, key); break;
    case 6: k_points_average<6, Src><<<g, 256, 0, st>>>(P, n, src, use_bins, key); break;
    case 7: k_points_average<7, Src><<<g, 256, 0, st>>>(P, n, src, use_bins, key); break;
    default: k_points_average<8, Src><<<g, 256, 0, st>>>(P, n, src, use_bins, key); break;
  }
}

// Per-axis tables of a redshift-cone grid in the reference's float arithmetic
// (checkAngles, triangulation_miscellaneous.cc:162-197; the bin loops of
// interpolateRedshiftCone, unaveraged_interpolation.cc:387-447; the checks of
// src/user_options.cc:1000-1009).  tab: r[n0], st[n1], ct[n1], cp[n2], sp[n2],
// theta[n1], psi[n2]; d: the bin sizes (r, theta and psi in radians).
int cone_tables(const float cone[6], const int32_t dims[3], std::vector<float>& tab, float d[3]) {
  float b[6];
  for (int i = 0; i < 6; ++i) b[i] = cone[i];
  for (int a = 0; a < 3; ++a)
    if (dims[a] <= 0) return set_error(DTFE_ERR_ARG, "redshift-cone bins must be positive");
  if (!(b[2] >= 0.f && b[2] <= 180.f && b[3] >= 0.f && b[3] <= 180.f))
    return set_error(DTFE_ERR_ARG, "redshift-cone theta limits must lie in [0, 180] degrees");
  if (!(b[5] - b[4] < 360.f)) return set_error(DTFE_ERR_ARG, "the psi range of a redshift cone spans 360 degrees or more");
  for (int i = 4; i < 6; ++i) b[i] -= std::floor(b[i] / 360.f) * 360.f;  // psi into [0, 360)
  if (b[4] > b[5]) b[5] += 360.f;
  const float rad = (float)(3.14159265 / 180.);  // the reference's PI (define.h:47)
  for (int i = 2; i < 6; ++i) b[i] *= rad;
  float dx[3];
  for (int a = 0; a < 3; ++a) dx[a] = (b[2 * a + 1] - b[2 * a]) / (float)dims[a];
  const size_t n0 = (size_t)dims[0], n1 = (size_t)dims[1], n2 = (size_t)dims[2];
  tab.assign(n0 + 3 * n1 + 3 * n2, 0.f);
  float* r = tab.data();
  float* st = r + n0;
  float* ct = st + n1;
  float* cp = ct + n1;
  float* sp = cp + n2;
  float* th = sp + n2;
  float* ps = th + n1;
  float x = (float)((double)b[0] + (double)dx[0] / 2.);
  for (size_t i = 0; i < n0; ++i, x += dx[0]) r[i] = x;
  x = (float)((double)b[2] + (double)dx[1] / 2.);
  for (size_t j = 0; j < n1; ++j, x += dx[1]) {
    th[j] = x;
    st[j] = std::sin(x);
    ct[j] = std::cos(x);
  }
  x = (float)((double)b[4] + (double)dx[2] / 2.);
  for (size_t k = 0; k < n2; ++k, x += dx[2]) {
    ps[k] = x;
    cp[k] = std::cos(x);
    sp[k] = std::sin(x);
  }
  for (int a = 0; a < 3; ++a) d[a] = dx[a];
  return DTFE_OK;
}

// Copies the staged rows of every requested field into the caller's host
// buffers and waits for them.
int copy_point_rows(dtfe_handle h, const InterpParams& P, uint32_t F, int64_t m, float* const out[DTFE_NUM_FIELDS]) {
  for (int q = 0; q < DTFE_NUM_FIELDS; ++q)
    if ((F >> q & 1u) && m > 0)
      DTFE_CUDA_TRY(cudaMemcpyAsync(out[q], P.out[q], sizeof(float) * (size_t)field_components(q, h->S) * m,
                                    cudaMemcpyDeviceToHost, h->stream));
  DTFE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return DTFE_OK;
}

}  // namespace

extern "C" {

int dtfe_gpu_interpolate_points(dtfe_handle h, int64_t n, const float* xyz, const float region[6],
                                const dtfe_interp_opts* o, float* const out[DTFE_NUM_FIELDS], int64_t* n_out) {
  if (!h || !o || !region || !out || !n_out || (n > 0 && !xyz) || n < 0) return set_error(DTFE_ERR_ARG, "null argument");
  int rc = check_point_call(h, o, out, "user sampling points");
  if (rc) return rc;
  *n_out = 0;
  if (n == 0) return DTFE_OK;
  DTFE_CUDA_TRY(cudaSetDevice(h->device));
  if ((rc = prepare_centres(h))) return rc;
  cudaStream_t st = h->stream;
  const uint32_t F = o->fields;
  const size_t comps = point_components(h, F);
  const int64_t nb = (n + kScanBlock - 1) / kScanBlock;
  if ((rc = dev_alloc(h, &h->pts_buf, (size_t)3 * n)) || (rc = dev_alloc(h, &h->pts_keep, (size_t)n)) ||
      (rc = dev_alloc(h, &h->pts_idx, (size_t)n + 1)) || (rc = dev_alloc(h, &h->pts_blocks, (size_t)nb + 1)) ||
      (rc = dev_alloc(h, &h->pts_out, std::max<size_t>(comps, 1) * (size_t)n)))
    return rc;
  DTFE_CUDA_TRY(cudaMemcpyAsync(h->pts_buf, xyz, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, st));
  Region6 R;
  for (int c = 0; c < 6; ++c) R.r[c] = region[c];
  k_points_keep<<<blocks_for(n, 256), 256, 0, st>>>(n, h->pts_buf, R, h->pts_keep);
  k_scan_blocks<<<(unsigned)nb, kScanBlock, 0, st>>>(n, h->pts_keep, h->pts_idx, h->pts_blocks);
  k_scan_totals<<<1, kScanBlock, 0, st>>>(nb, h->pts_blocks, h->pts_idx + n);
  k_scan_add<<<(unsigned)nb, kScanBlock, 0, st>>>(n, h->pts_idx, h->pts_blocks);
  DTFE_CUDA_TRY(cudaMemsetAsync(h->counters, 0, sizeof(unsigned long long) * CNT_N, st));
  const InterpParams P = point_params(h, o, n);
  const int use_bins = h->prep_ready && !h->prep_raster ? 1 : 0;
  launch_points_eval(h, P, n, PointList{h->pts_buf, h->pts_keep, h->pts_idx}, use_bins, nullptr);
  DTFE_CUDA_TRY(cudaGetLastError());
  int64_t m = 0;
  DTFE_CUDA_TRY(cudaMemcpyAsync(&m, h->pts_idx + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  DTFE_CUDA_TRY(cudaStreamSynchronize(st));
  if ((rc = copy_point_rows(h, P, F, m, out))) return rc;
  *n_out = m;
  h->tet_c_valid = false;
  return read_status(h, nullptr);
}

int dtfe_gpu_average_points(dtfe_handle h, int64_t n, const float* xyz, const float* delta, const float region[6],
                            const dtfe_interp_opts* o, float* const out[DTFE_NUM_FIELDS], int64_t* n_out) {
  if (!h || !o || !region || !out || !n_out || (n > 0 && (!xyz || !delta)) || n < 0)
    return set_error(DTFE_ERR_ARG, "null argument");
  int rc = check_point_call(h, o, out, "volume averages at user sampling points", false, true);
  if (rc) return rc;
  *n_out = 0;
  if (n == 0) return DTFE_OK;
  DTFE_CUDA_TRY(cudaSetDevice(h->device));
  if ((rc = prepare_centres(h))) return rc;
  cudaStream_t st = h->stream;
  const uint32_t F = o->fields;
  const size_t comps = point_components(h, F);
  const int64_t nb = (n + kScanBlock - 1) / kScanBlock;
  // pts_buf: positions, then the cell sizes
  if ((rc = dev_alloc(h, &h->pts_buf, (size_t)6 * n)) || (rc = dev_alloc(h, &h->pts_keep, (size_t)n)) ||
      (rc = dev_alloc(h, &h->pts_idx, (size_t)n + 1)) || (rc = dev_alloc(h, &h->pts_blocks, (size_t)nb + 1)) ||
      (rc = dev_alloc(h, &h->pts_out, std::max<size_t>(comps, 1) * (size_t)n)))
    return rc;
  DTFE_CUDA_TRY(cudaMemcpyAsync(h->pts_buf, xyz, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, st));
  DTFE_CUDA_TRY(cudaMemcpyAsync(h->pts_buf + 3 * n, delta, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, st));
  Region6 R;
  for (int c = 0; c < 6; ++c) R.r[c] = region[c];
  k_points_keep<<<blocks_for(n, 256), 256, 0, st>>>(n, h->pts_buf, R, h->pts_keep);
  k_scan_blocks<<<(unsigned)nb, kScanBlock, 0, st>>>(n, h->pts_keep, h->pts_idx, h->pts_blocks);
  k_scan_totals<<<1, kScanBlock, 0, st>>>(nb, h->pts_blocks, h->pts_idx + n);
  k_scan_add<<<(unsigned)nb, kScanBlock, 0, st>>>(n, h->pts_idx, h->pts_blocks);
  DTFE_CUDA_TRY(cudaMemsetAsync(h->counters, 0, sizeof(unsigned long long) * CNT_N, st));
  InterpParams P = point_params(h, o, n);
  P.NN = o->n_samples;
  const int use_bins = h->prep_ready && !h->prep_raster ? 1 : 0;
  PointAvgList src{PointList{h->pts_buf, h->pts_keep, h->pts_idx}, h->pts_buf + 3 * n};
  // interpolateUserSampling_averaged_2: no partition, so the seed itself
  launch_points_average(h, P, n, src, use_bins, mc_key(o->seed, -1));
  DTFE_CUDA_TRY(cudaGetLastError());
  int64_t m = 0;
  DTFE_CUDA_TRY(cudaMemcpyAsync(&m, h->pts_idx + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  DTFE_CUDA_TRY(cudaStreamSynchronize(st));
  if ((rc = copy_point_rows(h, P, F, m, out))) return rc;
  *n_out = m;
  h->tet_c_valid = false;
  return read_status(h, nullptr);
}

}  // extern "C"

namespace {

// Queues a redshift-cone interpolation into the device rows outp[slot]
// (dims[0] dims[1] dims[2] rows each); P receives the launch parameters.
int cone_enqueue(dtfe_handle h, const float cone[6], const float origin[3], const int32_t dims[3],
                 const dtfe_interp_opts* o, float* const outp[DTFE_NUM_FIELDS], InterpParams& P) {
  std::vector<float> tab;
  float d[3];
  int rc = cone_tables(cone, dims, tab, d);
  if (rc) return rc;
  const int64_t n = (int64_t)dims[0] * dims[1] * dims[2];
  if ((rc = prepare_centres(h))) return rc;
  cudaStream_t st = h->stream;
  // pts_buf holds the cone's tables, pts_keep the located tetrahedra
  if ((rc = dev_alloc(h, &h->pts_buf, tab.size())) || (rc = dev_alloc(h, &h->pts_keep, (size_t)n))) return rc;
  DTFE_CUDA_TRY(cudaMemcpyAsync(h->pts_buf, tab.data(), sizeof(float) * tab.size(), cudaMemcpyHostToDevice, st));
  DTFE_CUDA_TRY(cudaMemsetAsync(h->counters, 0, sizeof(unsigned long long) * CNT_N, st));
  P = point_params(h, o, n);
  for (int q = 0; q < DTFE_NUM_FIELDS; ++q) P.out[q] = (o->fields >> q & 1u) ? outp[q] : nullptr;
  ConeGrid src;
  src.r = h->pts_buf;
  src.st = src.r + dims[0];
  src.ct = src.st + dims[1];
  src.cp = src.ct + dims[1];
  src.sp = src.cp + dims[2];
  for (int c = 0; c < 3; ++c) src.o[c] = origin[c];
  src.n1 = (uint32_t)dims[1];
  src.n2 = (uint32_t)dims[2];
  const int use_bins = h->prep_ready && !h->prep_raster ? 1 : 0;
  if (o->method == DTFE_METHOD_MONTE_CARLO) {
    // interpolateRedshiftCone_averaged_2: no partition, so the seed itself
    P.NN = o->n_samples;
    ConeAvgGrid avg;
    avg.g = src;
    avg.th = src.sp + dims[2];
    avg.ps = avg.th + dims[1];
    for (int a = 0; a < 3; ++a) avg.d[a] = d[a];
    launch_points_average(h, P, n, avg, use_bins, mc_key(o->seed, -1));
    DTFE_CUDA_TRY(cudaGetLastError());
    h->tet_c_valid = false;
    return DTFE_OK;
  }
  launch_points_eval(h, P, n, src, use_bins, h->pts_keep);
  DTFE_CUDA_TRY(cudaGetLastError());
  if (!(o->flags & DTFE_FLAG_FIX_OUTSIDE_RASTER)) {
    const int64_t rows = (int64_t)dims[0] * dims[1];
    const int64_t want = (rows + 7) / 8;  // 8 warps per block
    k_cone_rows<<<(unsigned)std::min<int64_t>(want, 148 * 16), 256, 0, st>>>(P, h->pts_keep, rows, dims[2]);
    DTFE_CUDA_TRY(cudaGetLastError());
  }
  h->tet_c_valid = false;
  return DTFE_OK;
}

}  // namespace

extern "C" {

int dtfe_gpu_interpolate_cone(dtfe_handle h, const float cone[6], const float origin[3], const int32_t dims[3],
                              const dtfe_interp_opts* o, float* const out[DTFE_NUM_FIELDS]) {
  if (!h || !o || !cone || !origin || !dims || !out) return set_error(DTFE_ERR_ARG, "null argument");
  int rc = check_point_call(h, o, out, "redshift-cone grids", true, true);
  if (rc) return rc;
  for (int a = 0; a < 3; ++a)
    if (dims[a] <= 0) return set_error(DTFE_ERR_ARG, "redshift-cone bins must be positive");
  const int64_t n = (int64_t)dims[0] * dims[1] * dims[2];
  DTFE_CUDA_TRY(cudaSetDevice(h->device));
  const size_t comps = point_components(h, o->fields);
  if ((rc = dev_alloc(h, &h->pts_out, std::max<size_t>(comps, 1) * (size_t)n))) return rc;
  float* stage[DTFE_NUM_FIELDS] = {};
  size_t at = 0;
  for (int q = 0; q < DTFE_NUM_FIELDS; ++q) {
    if (!(o->fields >> q & 1u)) continue;
    stage[q] = h->pts_out + at * (size_t)n;
    at += (size_t)field_components(q, h->S);
  }
  InterpParams P;
  if ((rc = cone_enqueue(h, cone, origin, dims, o, stage, P))) return rc;
  if ((rc = copy_point_rows(h, P, o->fields, n, out))) return rc;
  return read_status(h, nullptr);
}

int dtfe_gpu_interpolate_cone_dev(dtfe_handle h, const float cone[6], const float origin[3], const int32_t dims[3],
                                  const dtfe_interp_opts* o, float* const out_dev[DTFE_NUM_FIELDS]) {
  if (!h || !o || !cone || !origin || !dims || !out_dev) return set_error(DTFE_ERR_ARG, "null argument");
  int rc = check_point_call(h, o, out_dev, "redshift-cone grids", true, true);
  if (rc) return rc;
  DTFE_CUDA_TRY(cudaSetDevice(h->device));
  InterpParams P;
  if ((rc = cone_enqueue(h, cone, origin, dims, o, out_dev, P))) return rc;
  return read_status(h, nullptr);
}

int dtfe_gpu_select_in_box_dev(dtfe_handle h, const float* pos_dev, int64_t n, const float full_box[6],
                               const float padded[6], int periodic, int32_t* idx_dev, float* pos_out_dev,
                               int64_t capacity, int64_t* count) {
  if (!h || !full_box || !padded || !count || n < 0 || (n > 0 && !pos_dev) || capacity < 0)
    return set_error(DTFE_ERR_ARG, "null argument");
  if (n >= (int64_t(1) << 31)) return set_error(DTFE_ERR_TOO_LARGE, "particle indices are 32-bit");
  *count = 0;
  if (n == 0) return DTFE_OK;
  DTFE_CUDA_TRY(cudaSetDevice(h->device));
  SelBoxes S;
  int n_off = 1;
  if (!periodic) {
    for (int k = 0; k < 6; ++k) S.box[0][k] = padded[k];
    for (int k = 0; k < 3; ++k) S.off[0][k] = 0.f;
  } else {
    float len[3];
    for (int k = 0; k < 3; ++k) len[k] = full_box[2 * k + 1] - full_box[2 * k];
    n_off = 27;
    for (int i1 = 0; i1 < 3; ++i1)
      for (int i2 = 0; i2 < 3; ++i2)
        for (int i3 = 0; i3 < 3; ++i3) {
          const int o = i1 * 9 + i2 * 3 + i3;
          const int ii[3] = {i1, i2, i3};
          for (int k = 0; k < 3; ++k) {
            S.off[o][k] = (float)(ii[k] - 1) * len[k];
            S.box[o][2 * k] = padded[2 * k] + S.off[o][k];
            S.box[o][2 * k + 1] = padded[2 * k + 1] + S.off[o][k];
          }
        }
  }
  const int64_t nchunks = (n + kSelChunk - 1) / kSelChunk;
  const int64_t nblk = nchunks * n_off;
  const int64_t nb = (nblk + kScanBlock - 1) / kScanBlock;
  int rc;
  if ((rc = dev_alloc(h, &h->sel_counts, (size_t)nblk)) || (rc = dev_alloc(h, &h->sel_first, (size_t)nblk + 1)) ||
      (rc = dev_alloc(h, &h->sel_blocks, (size_t)nb + 1)))
    return rc;
  cudaStream_t st = h->stream;
  k_select_count<<<(unsigned)nblk, kSelChunk, 0, st>>>(pos_dev, n, nchunks, S, h->sel_counts);
  k_scan_blocks<<<(unsigned)nb, kScanBlock, 0, st>>>(nblk, h->sel_counts, h->sel_first, h->sel_blocks);
  k_scan_totals<<<1, kScanBlock, 0, st>>>(nb, h->sel_blocks, h->sel_first + nblk);
  k_scan_add<<<(unsigned)nb, kScanBlock, 0, st>>>(nblk, h->sel_first, h->sel_blocks);
  DTFE_CUDA_TRY(cudaGetLastError());
  int64_t total = 0;
  DTFE_CUDA_TRY(cudaMemcpyAsync(&total, h->sel_first + nblk, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  DTFE_CUDA_TRY(cudaStreamSynchronize(st));
  *count = total;
  if (!idx_dev && !pos_out_dev) return DTFE_OK;
  if (total > capacity)
    return set_error(DTFE_ERR_TOO_LARGE, "selection larger than the output capacity (count returned)");
  k_select_write<<<(unsigned)nblk, kSelChunk, 0, st>>>(pos_dev, n, nchunks, S, h->sel_first, idx_dev, pos_out_dev);
  DTFE_CUDA_TRY(cudaGetLastError());
  DTFE_CUDA_TRY(cudaStreamSynchronize(st));
  return DTFE_OK;
}

// File chunk of dtfe_gpu_write_binary_dev: two pinned buffers of this size.
static const int64_t kIoChunk = int64_t(1) << 25;

int dtfe_gpu_write_binary_dev(dtfe_handle h, const char* path, const float* data_dev, int64_t n_floats) {
  if (!h || !path || n_floats < 0 || (n_floats > 0 && !data_dev)) return set_error(DTFE_ERR_ARG, "null argument");
  DTFE_CUDA_TRY(cudaSetDevice(h->device));
  for (int i = 0; i < 2; ++i) {
    if (!h->io_stage[i]) DTFE_CUDA_TRY(cudaHostAlloc((void**)&h->io_stage[i], (size_t)kIoChunk, cudaHostAllocDefault));
    if (!h->io_ev[i]) DTFE_CUDA_TRY(cudaEventCreateWithFlags(&h->io_ev[i], cudaEventDisableTiming));
  }
  std::FILE* f = std::fopen(path, "wb");
  if (!f) return set_error(DTFE_ERR_IO, std::string("cannot open ") + path + " for writing");
  const int64_t bytes = n_floats * (int64_t)sizeof(float);
  const int64_t n_chunks = (bytes + kIoChunk - 1) / kIoChunk;
  const char* src = reinterpret_cast<const char*>(data_dev);
  auto chunk_size = [&](int64_t c) { return (size_t)std::min(kIoChunk, bytes - c * kIoChunk); };
  auto enqueue = [&](int64_t c) -> cudaError_t {
    cudaError_t e = cudaMemcpyAsync(h->io_stage[c & 1], src + c * kIoChunk, chunk_size(c), cudaMemcpyDeviceToHost,
                                    h->stream);
    return e == cudaSuccess ? cudaEventRecord(h->io_ev[c & 1], h->stream) : e;
  };
  // the copy of chunk c + 1 runs while chunk c is written to the file; a
  // buffer is refilled only after its previous chunk has been written
  int rc = DTFE_OK;
  cudaError_t e = n_chunks > 0 ? enqueue(0) : cudaSuccess;
  for (int64_t c = 0; c < n_chunks && e == cudaSuccess && rc == DTFE_OK; ++c) {
    if (c + 1 < n_chunks) e = enqueue(c + 1);
    if (e == cudaSuccess) e = cudaEventSynchronize(h->io_ev[c & 1]);
    if (e == cudaSuccess && std::fwrite(h->io_stage[c & 1], 1, chunk_size(c), f) != chunk_size(c))
      rc = set_error(DTFE_ERR_IO, std::string("short write to ") + path);
  }
  if (e != cudaSuccess) {
    cudaStreamSynchronize(h->stream);  // no copy into a staging buffer outlives the call
    std::fclose(f);
    return set_error(DTFE_ERR_CUDA, std::string("writing ") + path + ": " + cudaGetErrorString(e));
  }
  if (rc != DTFE_OK) cudaStreamSynchronize(h->stream);
  if (std::fclose(f) != 0 && rc == DTFE_OK) rc = set_error(DTFE_ERR_IO, std::string("cannot close ") + path);
  return rc;
}

int dtfe_gpu_interpolate_dev_async(dtfe_handle h, const dtfe_interp_opts* opts,
                                   float* const out_dev[DTFE_NUM_FIELDS]) {
  if (!h) return set_error(DTFE_ERR_ARG, "null handle");
  DTFE_CUDA_TRY(cudaSetDevice(h->device));
  return interp_enqueue(h, opts, out_dev);
}

int dtfe_gpu_graph_build(dtfe_handle h, double rho_bar, const dtfe_interp_opts* opts,
                         float* const out_dev[DTFE_NUM_FIELDS]) {
  if (!h || !opts) return set_error(DTFE_ERR_ARG, "null argument");
  if (opts->method == DTFE_METHOD_TETRAHEDRA)
    return set_error(DTFE_ERR_ARG, "averaging method 1 sizes its lists on the host: not capturable");
  DTFE_CUDA_TRY(cudaSetDevice(h->device));
  drop_graph(h);
  // one plain step first: allocations, equidistant offsets and the walk
  // check happen here, so the captured launches need none of them
  int rc = dtfe_gpu_vertex_density(h, rho_bar);
  if (rc) return rc;
  if ((rc = interpolate_impl(h, opts, out_dev, nullptr))) return rc;
  cudaGraph_t g = nullptr;
  DTFE_CUDA_TRY(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  rc = dtfe_gpu_vertex_density(h, rho_bar);
  if (!rc) rc = interp_enqueue(h, opts, out_dev);
  cudaError_t e = cudaStreamEndCapture(h->stream, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return set_error(DTFE_ERR_CUDA, cudaGetErrorString(e));
  e = cudaGraphInstantiate(&h->step_graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    h->step_graph = nullptr;
    return set_error(DTFE_ERR_CUDA, cudaGetErrorString(e));
  }
  return DTFE_OK;
}

int dtfe_gpu_graph_launch(dtfe_handle h) {
  if (!h) return set_error(DTFE_ERR_ARG, "null handle");
  if (!h->step_graph) return set_error(DTFE_ERR_STATE, "no step graph built (or the handle changed since)");
  DTFE_CUDA_TRY(cudaSetDevice(h->device));
  DTFE_CUDA_TRY(cudaGraphLaunch(h->step_graph, h->stream));
  return DTFE_OK;
}

int dtfe_gpu_read_status(dtfe_handle h, dtfe_status* status) {
  if (!h) return set_error(DTFE_ERR_ARG, "null handle");
  DTFE_CUDA_TRY(cudaSetDevice(h->device));
  return read_status(h, status);
}

// Device buffers for host-output calls: one per requested field, zeroed
// (cells outside every tile keep zeros, as the reference's reserved vectors).
static int host_out_buffers(dtfe_handle h, const dtfe_interp_opts* opts, float* const out[DTFE_NUM_FIELDS],
                            float* dev[DTFE_NUM_FIELDS]) {
  int64_t G = (int64_t)h->grid[0] * h->grid[1] * h->grid[2];
  for (int s = 0; s < DTFE_NUM_FIELDS; ++s) {
    dev[s] = nullptr;
    if (!(opts->fields >> s & 1u)) continue;
    if (!out[s]) return set_error(DTFE_ERR_ARG, "missing output buffer");
    size_t need = (size_t)G * field_components(s, h->S);
    if (h->out_cap[s] < need) {
      int rc = dev_alloc(h, &h->out_buf[s], need);
      if (rc) return rc;
      h->out_cap[s] = need;
    }
    dev[s] = h->out_buf[s];
    DTFE_CUDA_TRY(cudaMemsetAsync(dev[s], 0, need * sizeof(float), h->stream));
  }
  return DTFE_OK;
}

static int copy_out(dtfe_handle h, float* const out[DTFE_NUM_FIELDS], float* const dev[DTFE_NUM_FIELDS]) {
  int64_t G = (int64_t)h->grid[0] * h->grid[1] * h->grid[2];
  for (int s = 0; s < DTFE_NUM_FIELDS; ++s) {
    if (!dev[s]) continue;
    size_t need = (size_t)G * field_components(s, h->S);
    DTFE_CUDA_TRY(cudaMemcpyAsync(out[s], dev[s], need * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  }
  return DTFE_OK;
}

int dtfe_gpu_interpolate(dtfe_handle h, const dtfe_interp_opts* opts, float* const out[DTFE_NUM_FIELDS],
                         dtfe_status* st) {
  if (!h || !opts || !out) return set_error(DTFE_ERR_ARG, "null argument");
  DTFE_CUDA_TRY(cudaSetDevice(h->device));
  float* dev[DTFE_NUM_FIELDS];
  int rc = host_out_buffers(h, opts, out, dev);
  if (rc || (rc = interpolate_impl(h, opts, dev, st)) || (rc = copy_out(h, out, dev))) return rc;
  DTFE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return DTFE_OK;
}

int dtfe_gpu_interpolate_async(dtfe_handle h, const dtfe_interp_opts* opts, float* const out[DTFE_NUM_FIELDS]) {
  if (!h || !opts || !out) return set_error(DTFE_ERR_ARG, "null argument");
  DTFE_CUDA_TRY(cudaSetDevice(h->device));
  float* dev[DTFE_NUM_FIELDS];
  int rc = host_out_buffers(h, opts, out, dev);
  if (rc || (rc = interp_enqueue(h, opts, dev)) || (rc = copy_out(h, out, dev))) return rc;
  return DTFE_OK;
}

// Canonical location of np points (host doubles) starting from tetrahedron
// `start`; out receives tetrahedron ids, -1 (outside the hull) or -2 (walk
// failure).  Test and diagnostic entry point.
int dtfe_gpu_locate_points(dtfe_handle h, int64_t np, const double* pts, int32_t start, int32_t* out) {
  if (!h || (np > 0 && (!pts || !out))) return set_error(DTFE_ERR_ARG, "null argument");
  if (h->T == 0) return set_error(DTFE_ERR_DEGENERATE, "no tetrahedra");
  if (start < 0 || start >= h->T) return set_error(DTFE_ERR_ARG, "start tetrahedron out of range");
  if (np == 0) return DTFE_OK;
  DTFE_CUDA_TRY(cudaSetDevice(h->device));
  cudaStream_t st = h->stream;
  double* dp = nullptr;
  int* dout = nullptr;
  DTFE_CUDA_TRY(cudaMallocAsync((void**)&dp, sizeof(double) * 3 * np, st));
  DTFE_CUDA_TRY(cudaMallocAsync((void**)&dout, sizeof(int) * np, st));
  DTFE_CUDA_TRY(cudaMemcpyAsync(dp, pts, sizeof(double) * 3 * np, cudaMemcpyHostToDevice, st));
  k_locate_points<<<blocks_for(np, 128), 128, 0, st>>>(np, dp, h->tet_v, h->tet_n, h->posd, start,
                                                       h->max_steps, dout);
  DTFE_CUDA_TRY(cudaGetLastError());
  DTFE_CUDA_TRY(cudaMemcpyAsync(out, dout, sizeof(int) * np, cudaMemcpyDeviceToHost, st));
  DTFE_CUDA_TRY(cudaFreeAsync(dp, st));
  DTFE_CUDA_TRY(cudaFreeAsync(dout, st));
  DTFE_CUDA_TRY(cudaStreamSynchronize(st));
  return DTFE_OK;
}

int dtfe_gpu_download_tets(dtfe_handle h, int32_t* tet_v, int32_t* tet_n) {
  if (!h) return set_error(DTFE_ERR_ARG, "null handle");
  if (h->T > 0 && (!tet_v && !tet_n)) return set_error(DTFE_ERR_ARG, "null argument");
  DTFE_CUDA_TRY(cudaSetDevice(h->device));
  if (tet_v && h->T)
    DTFE_CUDA_TRY(cudaMemcpyAsync(tet_v, h->tet_v, 16 * h->T, cudaMemcpyDeviceToHost, h->stream));
  if (tet_n && h->T)
    DTFE_CUDA_TRY(cudaMemcpyAsync(tet_n, h->tet_n, 16 * h->T, cudaMemcpyDeviceToHost, h->stream));
  DTFE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return DTFE_OK;
}

// dtfe_gpu_tiles_gather_dev / dtfe_gpu_tiles_scatter_dev
static int tiles_copy(dtfe_handle h, int32_t n_tiles, const int32_t* tiles, const int32_t grid[3], int32_t ncomp,
                      const float* src_dev, float* dst_dev, int to_packed) {
  if (!h || n_tiles < 0 || (n_tiles > 0 && (!tiles || !src_dev || !dst_dev)) || !grid || ncomp < 1)
    return set_error(DTFE_ERR_ARG, "null argument or bad size");
  if (n_tiles == 0) return DTFE_OK;
  std::vector<TileRec> recs((size_t)n_tiles);
  std::vector<int64_t> start((size_t)n_tiles + 1, 0);
  for (int t = 0; t < n_tiles; ++t) {
    for (int a = 0; a < 3; ++a) {
      recs[t].o[a] = tiles[6 * t + a];
      recs[t].d[a] = tiles[6 * t + 3 + a];
      if (recs[t].o[a] < 0 || recs[t].d[a] < 0 || (int64_t)recs[t].o[a] + recs[t].d[a] > grid[a])
        return set_error(DTFE_ERR_ARG, "tile outside the grid");
    }
    start[t + 1] = start[t] + (int64_t)recs[t].d[0] * recs[t].d[1] * recs[t].d[2];
  }
  DTFE_CUDA_TRY(cudaSetDevice(h->device));
  int rc;
  if ((rc = dev_alloc(h, &h->tile_recs, (size_t)n_tiles)) || (rc = dev_alloc(h, &h->tile_start, (size_t)n_tiles + 1)))
    return rc;
  cudaStream_t st = h->stream;
  DTFE_CUDA_TRY(cudaMemcpyAsync(h->tile_recs, recs.data(), sizeof(TileRec) * n_tiles, cudaMemcpyHostToDevice, st));
  DTFE_CUDA_TRY(cudaMemcpyAsync(h->tile_start, start.data(), sizeof(int64_t) * (n_tiles + 1),
                                cudaMemcpyHostToDevice, st));
  const int64_t total = start[n_tiles] * ncomp;
  if (total > 0) {
    const unsigned nb = (unsigned)std::min<int64_t>((total + 255) / 256, 148 * 64);
    k_tiles_copy<<<nb, 256, 0, st>>>(n_tiles, h->tile_recs, h->tile_start, grid[1], grid[2], ncomp, to_packed,
                                     src_dev, dst_dev);
    DTFE_CUDA_TRY(cudaGetLastError());
  }
  DTFE_CUDA_TRY(cudaStreamSynchronize(st));  // the host tables go out of scope
  return DTFE_OK;
}

int dtfe_gpu_tiles_gather_dev(dtfe_handle h, int32_t n_tiles, const int32_t* tiles, const int32_t grid[3],
                              int32_t ncomp, const float* field_dev, float* packed_dev) {
  return tiles_copy(h, n_tiles, tiles, grid, ncomp, field_dev, packed_dev, 1);
}

int dtfe_gpu_tiles_scatter_dev(dtfe_handle h, int32_t n_tiles, const int32_t* tiles, const int32_t grid[3],
                               int32_t ncomp, const float* packed_dev, float* field_dev) {
  return tiles_copy(h, n_tiles, tiles, grid, ncomp, packed_dev, field_dev, 0);
}

int dtfe_gpu_set_max_walk_steps(dtfe_handle h, int32_t max_walk_steps) {
  if (!h) return set_error(DTFE_ERR_ARG, "null handle");
  if (max_walk_steps < 0) return set_error(DTFE_ERR_ARG, "max_walk_steps must be >= 0");
  h->max_steps = max_walk_steps > 0 ? max_walk_steps : 65536;
  drop_graph(h);  // a captured step holds the old limit
  return DTFE_OK;
}

// Per grid cell the tetrahedron its centre was located in by the last
// cell-centre interpolation (tet_c is kept per sample, in tile order: each
// sample goes back to its main-grid cell); -1 outside the hull and for cells
// outside every tile.
int dtfe_gpu_download_located(dtfe_handle h, int32_t* loc) {
  if (!h || !loc) return set_error(DTFE_ERR_ARG, "null argument");
  if (!h->tet_c_valid) return set_error(DTFE_ERR_STATE, "no cell-centre interpolation to report");
  DTFE_CUDA_TRY(cudaSetDevice(h->device));
  std::vector<int32_t> per_sample((size_t)h->n_cells);
  DTFE_CUDA_TRY(cudaMemcpyAsync(per_sample.data(), h->tet_c, sizeof(int32_t) * h->n_cells, cudaMemcpyDeviceToHost,
                                h->stream));
  DTFE_CUDA_TRY(cudaStreamSynchronize(h->stream));
  const int64_t G = (int64_t)h->grid[0] * h->grid[1] * h->grid[2];
  std::fill(loc, loc + G, -1);
  int64_t s = 0;
  for (const dtfe_subbox& B : h->boxes_h)
    for (int i = 0; i < B.tile_dims[0]; ++i)
      for (int j = 0; j < B.tile_dims[1]; ++j) {
        const int64_t row = ((int64_t)(B.tile_origin[0] + i) * h->grid[1] + (B.tile_origin[1] + j)) * h->grid[2] +
                            B.tile_origin[2];
        for (int k = 0; k < B.tile_dims[2]; ++k, ++s) loc[row + k] = per_sample[s] < 0 ? -1 : per_sample[s];
      }
  return DTFE_OK;
}

}  // extern "C"
