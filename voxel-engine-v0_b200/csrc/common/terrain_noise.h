// Seeded terrain noise of the synthetic worlds (world/hash.rs:2-32 hashing,
// lattice value noise with smoothstep interpolation, 4-octave height field,
// caves, carving, trees and light voxels), shared by the host producer and
// the device clipmap generator and chunk builder so all of them
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

// Cave carving: two octaves of 3D value noise above the threshold.
VXE_HD bool cave(const vxe_world_params& p, int32_t wx, int32_t wy, int32_t wz) {
  if (!(p.cave_threshold < 1.0f)) return false;
  const uint32_t s = p.seed ^ 0xCA7E5EEDu;
  const double v = (value_noise3(s, wx / 16.0, wy / 16.0, wz / 16.0) +
                    0.5 * value_noise3(s + 7u, wx / 8.0, wy / 8.0, wz / 8.0)) /
                   1.5;
  return v > (double)p.cave_threshold;
}

// Trees: one candidate per 1 m cell (10 voxels); trunk of WOOD, crown LEAF.
struct Tree {
  int32_t x, z, base, trunk, r;
};
VXE_HD bool tree_at_cell(const vxe_world_params& p, int32_t mx, int32_t mz, Tree* t) {
  const uint32_t h = hash2(p.seed ^ 0x7EEu, mx, mz);
  if (h % 61u != 0u) return false;
  t->x = mx * 10 + 5;
  t->z = mz * 10 + 5;
  t->base = ground(p, t->x, t->z) + 1;
  t->trunk = 14 + (int32_t)((h >> 8) % 10u);
  t->r = 5 + (int32_t)((h >> 16) % 4u);
  return true;
}

// Decoration above the surface (g = column ground): light voxels, trees.
VXE_HD uint8_t decor(const vxe_world_params& p, int32_t wx, int32_t wy, int32_t wz, int32_t g) {
  if (p.features & 2u) {
    if (wy == g + 1 && hash2(p.seed ^ 0x119u, wx, wz) % 331u == 0u) return VXE_MAT_LIGHT;
  }
  if (p.features & 1u) {
    const int32_t mx0 = (int32_t)floor((wx - 14) / 10.0), mx1 = (int32_t)floor((wx + 14) / 10.0);
    const int32_t mz0 = (int32_t)floor((wz - 14) / 10.0), mz1 = (int32_t)floor((wz + 14) / 10.0);
    uint8_t best = VXE_MAT_AIR;
    for (int32_t mz = mz0; mz <= mz1; ++mz)
      for (int32_t mx = mx0; mx <= mx1; ++mx) {
        Tree t;
        if (!tree_at_cell(p, mx, mz, &t)) continue;
        if (wx == t.x && wz == t.z && wy >= t.base && wy < t.base + t.trunk) return VXE_MAT_WOOD;
        const int32_t cy = t.base + t.trunk;
        const int32_t dx = wx - t.x, dy = wy - cy, dz = wz - t.z;
        if (dx * dx + dy * dy + dz * dz <= t.r * t.r) best = VXE_MAT_LEAF;
      }
    return best;
  }
  return VXE_MAT_AIR;
}

// Material of world voxel (wx, wy, wz) over a column of ground height g.
VXE_HD uint8_t material(const vxe_world_params& p, int32_t wx, int32_t wy, int32_t wz, int32_t g) {
  uint8_t m;
  if (wy < g) {
    m = (wy >= g - p.dirt_depth) ? VXE_MAT_DIRT : VXE_MAT_STONE;
  } else if (wy == g) {
    m = VXE_MAT_GRASS;
  } else {
    m = VXE_MAT_AIR;
  }
  if (m != VXE_MAT_AIR) {
    if (cave(p, wx, wy, wz)) m = VXE_MAT_AIR;
    else if (p.carve_mod != 0u && hash3(p.seed ^ 0x5EEDu, wx, wy, wz) % p.carve_mod == 0u) m = VXE_MAT_AIR;
  }
  if (m == VXE_MAT_AIR && wy > g && p.features != 0u) m = decor(p, wx, wy, wz, g);
  return m;
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
