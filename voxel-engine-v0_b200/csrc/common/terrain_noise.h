// Seeded terrain noise of the synthetic worlds (world/hash.rs:2-32 hashing,
// lattice value noise with smoothstep interpolation, 4-octave height field),
// shared by the host producer and the device clipmap generator so both
// evaluate the same binary64 operation sequence (no contraction on either
// side: g++ -ffp-contract=off, nvcc -fmad=false).
#pragma once

#include <math.h>
#include <stdint.h>

#include "vxe/vxe.h"

#ifdef __CUDACC__
#define VXE_HD __host__ __device__ __forceinline__
#else
#define VXE_HD inline
#endif

namespace vxe {
namespace terrain {

VXE_HD uint32_t mix32(uint32_t v) {
  v ^= v >> 16;
  v *= 0x7feb352du;
  v ^= v >> 15;
  v *= 0x846ca68bu;
  v ^= v >> 16;
  return v;
}
VXE_HD uint32_t hash2(uint32_t seed, int32_t x, int32_t z) {
  return mix32(seed ^ ((uint32_t)x * 0x9e3779b1u) ^ ((uint32_t)z * 0x85ebca6bu));
}
VXE_HD uint32_t hash3(uint32_t seed, int32_t x, int32_t y, int32_t z) {
  return mix32(seed ^ ((uint32_t)x * 0x9e3779b1u) ^ ((uint32_t)y * 0x85ebca6bu) ^ ((uint32_t)z * 0xc2b2ae35u));
}
VXE_HD double u01(uint32_t v) { return (double)v * (1.0 / 4294967296.0); }
VXE_HD double fade(double t) { return t * t * (3.0 - 2.0 * t); }

VXE_HD double value_noise2(uint32_t seed, double x, double z) {
  const double gx = floor(x), gz = floor(z);
  const int32_t ix = (int32_t)gx, iz = (int32_t)gz;
  const double fx = fade(x - gx), fz = fade(z - gz);
  const double a = u01(hash2(seed, ix, iz)), b = u01(hash2(seed, ix + 1, iz));
  const double c = u01(hash2(seed, ix, iz + 1)), d = u01(hash2(seed, ix + 1, iz + 1));
  const double x0 = a + (b - a) * fx, x1 = c + (d - c) * fx;
  return x0 + (x1 - x0) * fz;
}

VXE_HD double value_noise3(uint32_t seed, double x, double y, double z) {
  const double gx = floor(x), gy = floor(y), gz = floor(z);
  const int32_t ix = (int32_t)gx, iy = (int32_t)gy, iz = (int32_t)gz;
  const double fx = fade(x - gx), fy = fade(y - gy), fz = fade(z - gz);
  double c[2][2][2];
  for (int k = 0; k < 2; ++k)
    for (int j = 0; j < 2; ++j)
      for (int i = 0; i < 2; ++i) c[k][j][i] = u01(hash3(seed, ix + i, iy + j, iz + k));
  double yz[2][2];
  for (int k = 0; k < 2; ++k)
    for (int j = 0; j < 2; ++j) yz[k][j] = c[k][j][0] + (c[k][j][1] - c[k][j][0]) * fx;
  const double z0 = yz[0][0] + (yz[0][1] - yz[0][0]) * fy;
  const double z1 = yz[1][0] + (yz[1][1] - yz[1][0]) * fy;
  return z0 + (z1 - z0) * fz;
}

// Surface height in voxels: 4 octaves, persistence 0.5, lacunarity 2, mapped
// linearly onto [height_min, height_max].
VXE_HD int32_t ground(const vxe_world_params& p, int32_t wx, int32_t wz) {
  double spacing = p.height_scale_vox > 0.f ? (double)p.height_scale_vox : 64.0;
  double amp = 1.0, sum = 0.0, norm = 0.0;
  for (int o = 0; o < 4; ++o) {
    sum += amp * value_noise2(p.seed + 0x9E37u * (uint32_t)(o + 1), wx / spacing, wz / spacing);
    norm += amp;
    amp *= 0.5;
    spacing *= 0.5;
  }
  const double n = sum / norm;  // [0, 1)
  const int32_t span = p.height_max - p.height_min + 1;
  const int32_t h = p.height_min + (int32_t)floor(n * (double)span);
  return h < p.height_min ? p.height_min : (h > p.height_max ? p.height_max : h);
}

// Clipmap texel at world (x, z) metres: the surface height in metres
// (clipmap.rs sample with voxel 0.1 m).
VXE_HD float clip_sample(const vxe_world_params& p, float wx_m, float wz_m) {
  const float vs = 0.1f;
  const int32_t wx = (int32_t)floorf(wx_m / vs), wz = (int32_t)floorf(wz_m / vs);
  return (float)ground(p, wx, wz) * vs;
}

}  // namespace terrain
}  // namespace vxe
