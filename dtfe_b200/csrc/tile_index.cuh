// Tile-local sample index -> (i, j, k), k fastest (the reference's raster
// order, x slowest).  Tile indices are below 2^31 (dtfe_gpu_set_subboxes
// refuses 2^31 cells or more), so 32-bit division suffices; 64-bit division
// takes many more instructions on the GPU.
#pragma once

#include <cstdint>

__device__ __forceinline__ void tile_ijk(int64_t local, int ny, int nz, int& i, int& j, int& k) {
  const uint32_t l = (uint32_t)local, uz = (uint32_t)nz, uy = (uint32_t)ny;
  const uint32_t q = l / uz;
  k = (int)(l - q * uz);
  const uint32_t r = q / uy;
  j = (int)(q - r * uy);
  i = (int)r;
}
