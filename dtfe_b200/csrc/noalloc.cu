// Vertex densities for callers that cannot allocate device memory.
//
// Some host applications own every byte of device memory (a fixed budget
// handed out by their own pool) and do not let libraries they call use
// cudaMalloc; others call from latency-critical loops where an allocation
// and the device synchronisation it can imply are not acceptable.  For them
// this entry point computes vertex densities without allocating anything:
// the caller passes the inputs and the output in device memory, and the only
// scratch (the per-vertex volume sums, hull flags, the vertices' bounding box
// and an error counter) lives in file-scope device arrays sized for at most
// DTFE_NOALLOC_MAX_VERTS vertices.
//
// The volume sums are exact integer sums of the FP64 tetrahedron volumes in
// units of 2^-62 of the vertices' bounding-box volume (fixed_volume.cuh), so
// the result does not depend on the order the GPU adds in: every call on the
// same input gives the same densities, bit for bit.
//
// Those arrays exist once per device that loads this library and stay
// resident until the process exits.  Every call shares them, so calls that
// overlap on the GPU (different streams, different host threads) race and
// must be serialised by the caller.  Each call clears the parts it uses.
//
// The device address of the arrays is looked up (cudaGetSymbolAddress) by the
// first call made on each device, with that device current; make that first
// call before any stream capture.  Every call returns only after its stream
// has finished its work: it reads back the range check's count.

#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/dtfe_gpu.h"
#include "fixed_volume.cuh"
#include "predicates.h"

extern "C" int dtfe_internal_set_error(int code, const char* msg);

namespace {

static __device__ __align__(256) long long g_noalloc_volsum[DTFE_NOALLOC_MAX_VERTS];
static __device__ __align__(256) int g_noalloc_hull[DTFE_NOALLOC_MAX_VERTS];
static __device__ __align__(256) unsigned long long g_noalloc_bad[1];
static __device__ __align__(256) int g_noalloc_bbox[6];

struct Scratch {
  long long* volsum = nullptr;
  int* hull = nullptr;
  unsigned long long* bad = nullptr;
  int* bbox = nullptr;
};

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
Scratch g_scratch[kMaxDevices];
bool g_ready[kMaxDevices] = {};

// Device addresses of the scratch arrays on device `dev` (current).
int scratch_for(int dev, Scratch* out) {
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_ready[dev]) {
    Scratch s;
    cudaError_t e[4] = {cudaGetSymbolAddress((void**)&s.volsum, g_noalloc_volsum),
                        cudaGetSymbolAddress((void**)&s.hull, g_noalloc_hull),
                        cudaGetSymbolAddress((void**)&s.bad, g_noalloc_bad),
                        cudaGetSymbolAddress((void**)&s.bbox, g_noalloc_bbox)};
    for (cudaError_t x : e)
      if (x != cudaSuccess)
        return dtfe_internal_set_error(DTFE_ERR_CUDA, (std::string("cudaGetSymbolAddress: ") +
                                                       cudaGetErrorString(x)).c_str());
    g_scratch[dev] = s;
    g_ready[dev] = true;
  }
  *out = g_scratch[dev];
  return DTFE_OK;
}

__global__ void k_noalloc_bbox_init(int* __restrict__ bbox) {
  if (threadIdx.x < 6) bbox[threadIdx.x] = (threadIdx.x & 1) ? INT_MIN : INT_MAX;
}

// Bounding box of the vertices (float order keys, min/max per axis).
__global__ void __launch_bounds__(256) k_noalloc_bbox(int64_t V, const float* __restrict__ xyz,
                                                      int* __restrict__ bbox) {
  int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < V; i += (int64_t)gridDim.x * blockDim.x)
    for (int c = 0; c < 3; ++c) {
      const int k = dtfe::float_order_key(xyz[3 * i + c]);
      lo[c] = min(lo[c], k);
      hi[c] = max(hi[c], k);
    }
  for (int c = 0; c < 3; ++c) {
    const int a = __reduce_min_sync(0xffffffffu, lo[c]), b = __reduce_max_sync(0xffffffffu, hi[c]);
    if ((threadIdx.x & 31) == 0) {
      atomicMin(&bbox[2 * c], a);
      atomicMax(&bbox[2 * c + 1], b);
    }
  }
}

__global__ void k_noalloc_volume(int64_t T, int64_t V, const int4* __restrict__ tet_v,
                                 const int4* __restrict__ tet_n, const float* __restrict__ xyz,
                                 const int* __restrict__ bbox, long long* __restrict__ volsum,
                                 int* __restrict__ hull, unsigned long long* __restrict__ bad) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= T) return;
  int4 v = tet_v[t];
  int4 n = tet_n[t];
  int id[4] = {v.x, v.y, v.z, v.w};
  for (int a = 0; a < 4; ++a)
    if (id[a] < 0 || id[a] >= V) {
      atomicAdd(bad, 1ull);
      return;
    }
  const double inv_q = dtfe::fixed_scale(dtfe::bbox_volume(bbox));
  double X[4][3];
  for (int a = 0; a < 4; ++a)
    for (int k = 0; k < 3; ++k) X[a][k] = (double)xyz[3 * (int64_t)id[a] + k];
  const double vt = dtfe::orient_det(X[0], X[1], X[2], X[3]) / 6.0;
  const unsigned long long q = (unsigned long long)__double2ll_rn(vt * inv_q);
  for (int a = 0; a < 4; ++a) atomicAdd((unsigned long long*)&volsum[id[a]], q);
  int nb[4] = {n.x, n.y, n.z, n.w};
  for (int i = 0; i < 4; ++i)
    if (nb[i] < 0)
      for (int a = 0; a < 4; ++a)
        if (a != i) hull[id[a]] = 1;
}

// Writes the densities only when every vertex id was in range: with a bad id
// the caller's buffer is left as it was.
__global__ void k_noalloc_density(int64_t V, const float* __restrict__ w, const long long* __restrict__ volsum,
                                  const int* __restrict__ hull, const int* __restrict__ bbox,
                                  const unsigned long long* __restrict__ bad, float factor,
                                  float* __restrict__ dens) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= V || *bad != 0ull) return;
  dens[i] = dtfe::density_from_fixed(volsum[i], dtfe::fixed_unit(dtfe::bbox_volume(bbox)), w[i], factor,
                                     hull[i] != 0);
}

}  // namespace

extern "C" int dtfe_vertex_density_noalloc(const int32_t* tet_v_dev, const int32_t* tet_n_dev,
                                           int64_t n_tets, const float* xyz_dev, const float* w_dev,
                                           int64_t n_verts, double rho_bar, float* dens_dev, void* stream) {
  if (n_verts < 0 || n_tets < 0) return dtfe_internal_set_error(DTFE_ERR_ARG, "negative size");
  if (n_verts > DTFE_NOALLOC_MAX_VERTS)
    return dtfe_internal_set_error(
        DTFE_ERR_TOO_LARGE, ("dtfe_vertex_density_noalloc: " + std::to_string(n_verts) +
                             " vertices exceed the static scratch of DTFE_NOALLOC_MAX_VERTS = " +
                             std::to_string(DTFE_NOALLOC_MAX_VERTS) + "; use dtfe_gpu_vertex_density")
                                .c_str());
  if (n_tets > 0x7FFFFFFF) return dtfe_internal_set_error(DTFE_ERR_TOO_LARGE, "too many tetrahedra");
  if (!(rho_bar > 0.0)) return dtfe_internal_set_error(DTFE_ERR_ARG, "averageDensity must be positive");
  if (n_verts == 0) return DTFE_OK;
  if (!xyz_dev || !w_dev || !dens_dev || (n_tets > 0 && (!tet_v_dev || !tet_n_dev)))
    return dtfe_internal_set_error(DTFE_ERR_ARG, "null device pointer");
  if (((uintptr_t)tet_v_dev | (uintptr_t)tet_n_dev) & 15)
    return dtfe_internal_set_error(DTFE_ERR_ARG, "tet_v/tet_n must be 16-byte aligned");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return dtfe_internal_set_error(DTFE_ERR_NO_DEVICE, "no current CUDA device");
  Scratch s;
  int rc = scratch_for(dev, &s);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  if ((e = cudaMemsetAsync(s.volsum, 0, sizeof(long long) * n_verts, st)) != cudaSuccess ||
      (e = cudaMemsetAsync(s.hull, 0, sizeof(int) * n_verts, st)) != cudaSuccess ||
      (e = cudaMemsetAsync(s.bad, 0, sizeof(unsigned long long), st)) != cudaSuccess)
    return dtfe_internal_set_error(DTFE_ERR_CUDA, cudaGetErrorString(e));
  k_noalloc_bbox_init<<<1, 32, 0, st>>>(s.bbox);
  k_noalloc_bbox<<<(unsigned)std::min<int64_t>((n_verts + 255) / 256, 1024), 256, 0, st>>>(n_verts, xyz_dev,
                                                                                         s.bbox);
  if (n_tets > 0)
    k_noalloc_volume<<<(unsigned)((n_tets + 255) / 256), 256, 0, st>>>(n_tets, n_verts, (const int4*)tet_v_dev,
                                                                       (const int4*)tet_n_dev, xyz_dev, s.bbox,
                                                                       s.volsum, s.hull, s.bad);
  float rb = (float)rho_bar;
  float factor = (float)(4.0 / (double)rb);
  k_noalloc_density<<<(unsigned)((n_verts + 255) / 256), 256, 0, st>>>(n_verts, w_dev, s.volsum, s.hull, s.bbox,
                                                                       s.bad, factor, dens_dev);
  if ((e = cudaGetLastError()) != cudaSuccess) return dtfe_internal_set_error(DTFE_ERR_CUDA, cudaGetErrorString(e));
  unsigned long long bad = 0;
  if ((e = cudaMemcpyAsync(&bad, s.bad, sizeof(bad), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess)
    return dtfe_internal_set_error(DTFE_ERR_CUDA, cudaGetErrorString(e));
  if (bad)
    return dtfe_internal_set_error(DTFE_ERR_ARG, "tet_v holds vertex ids outside [0, n_verts); dens left unchanged");
  return DTFE_OK;
}
