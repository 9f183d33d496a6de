// build_kernels.cuh -- the chunk builder on the device.
//
// The reference builds chunks on CPU worker threads (svo/builder.rs:846-986):
// material fill, column tops and colinfo (builder.rs:742-805), macro
// occupancy (builder.rs:809-841), ground min-mip (mips.rs:4-90), the
// bottom-up octree with stone and uniform collapse (builder_svo.rs:337-534)
// and ropes (builder_ropes.rs:76-195).  These kernels produce the same
// records byte for byte for a batch of chunks:
//
//   k_build_columns  one thread per voxel column, 16 blocks per chunk: the
//                    surface height, the 64 materials of the column, its
//                    colinfo entry, and -- with the 2x2 neighbour columns
//                    read by warp shuffles -- the level-1 ground minimum and
//                    the state words of the level-5 cells (2^3 voxels) it
//                    heads, plus a per-block solid voxel count (a warp
//                    whose columns all lie above the surface of a world
//                    without decorations stores zero rows instead);
//   k_build_svo      one CTA per chunk: ground min-mip, the cell states of
//                    levels 4..0 and their scans, the level-5 child offsets
//                    (16 rounds of one exclusive scan, voxel records written
//                    as they go), node emission, ropes top-down (one thread
//                    per node, its parent found from its key), macro bits; a chunk with no solid voxel
//                    writes its lone air root and returns.
//
// Octree cells.  A cell of level l (0 = the chunk, 6 = a voxel) holds
// 2^(6-l) voxels per side; its cells are numbered px + pz*S + py*S*S with
// S = 2^l, the order in which the host builder scans them.  A cell is
// present when any voxel inside is solid.  A present cell of level < 6 is
//   - a stone leaf when every voxel inside is solid and its top voxel lies
//     below (lowest ground of its columns - dirt depth),
//   - else a uniform leaf when all 8 children are present leaves of one
//     material,
//   - else internal: its present children are packed, in child order
//     ci = x | y<<1 | z<<2, into level l+1's node list, whose entries are
//     ordered by parent cell number.
// The node list is root, then the children lists of levels 1..6.  The state
// word of a cell keeps what its parent and the emission need: the mask of
// present children (bits 0..7), the leaf material (8..15), leaf (16), full
// (17).  Cells that are not internal contribute no children, so a cell's
// child offset is the exclusive prefix sum of popcount(mask) over internal
// cells of its level.
#pragma once

#include "../common/terrain_noise.h"

namespace vxe {
namespace build {

constexpr int kSide = 64;
constexpr uint32_t kVoxels = 64u * 64u * 64u;
constexpr uint32_t kColumns = 64u * 64u;
constexpr uint32_t kCells5 = 32u * 32u * 32u;
constexpr uint32_t kInvalid = 0xFFFFFFFFu;
constexpr uint32_t ST_MASK = 0xFFu;
constexpr uint32_t ST_LEAF = 1u << 16;
constexpr uint32_t ST_FULL = 1u << 17;
constexpr int SVO_THREADS = 512;
constexpr int SVO_WARPS = SVO_THREADS / 32;
// Voxel records of one level-5 round staged in (dynamic) shared memory so
// they leave as contiguous stores; a round with more writes them directly.
constexpr uint32_t kStageNodes = 2048u;
constexpr size_t kStageBytes = kStageNodes * 16u;
// Shared state words of levels 4..0 (4096 + 512 + 64 + 8 + 1 cells).
constexpr uint32_t kLowCells = 4681u;
__host__ __device__ constexpr uint32_t low_off(int l) {
  return l == 4 ? 0u : l == 3 ? 4096u : l == 2 ? 4608u : l == 1 ? 4672u : 4680u;
}
// Ground min-mip levels 1..6 (32^2 + 16^2 + 8^2 + 4^2 + 2^2 + 1).
constexpr uint32_t kMipWords = 1365u;
__host__ __device__ constexpr uint32_t mip_off(int lv) {
  return lv == 1 ? 0u : lv == 2 ? 1024u : lv == 3 ? 1280u : lv == 4 ? 1344u : lv == 5 ? 1360u : 1364u;
}

struct BuildArgs {
  vxe_world_params wp;
  double cave_smin;      // least s = n1 + 0.5 n2 with s / 1.5 > cave threshold
  const int32_t* coords;  // n chunk coordinates (x, y, z)
  uint32_t n;
  uint8_t* mat;           // n * 64^3 materials
  int32_t* mip1;          // n * 32^2 level-1 ground minima (2x2 columns)
  uint32_t* solid_part;   // n * 16 solid voxel counts, one per column block
  uint32_t* st5;          // n * 32^3 level-5 state words
  uint32_t* kb5;          // n * 32^3 level-5 child offsets
  uint32_t node_cap;
  vxe_node* nodes;        // n * node_cap
  vxe_node_ropes* ropes;  // n * node_cap
  uint32_t* macro;        // n * 16
  uint32_t* colinfo;      // n * 2048
  uint32_t* counts;       // n * 2: node_count, solid_voxels (may be null)
  // Resident builds: chunk i goes to its place -- nodes and ropes at
  // node_base (at most node_count of them), macro and colinfo words and the
  // meta record at its slot -- instead of the i-indexed layout above.
  const vxe_build_place* place;
  vxe_chunk_meta* metas;
  uint32_t* error_word;
};

// Error word bit of a resident build whose chunk needs more nodes than its
// place reserves (its meta then marks it empty).
constexpr uint32_t ERR_BUILD = 1u << 7;

__device__ __forceinline__ int32_t chunk_coord(const BuildArgs& B, uint32_t chunk, int axis) {
  if (B.place) return axis == 0 ? B.place[chunk].cx : axis == 1 ? B.place[chunk].cy : B.place[chunk].cz;
  return B.coords[3 * chunk + axis];
}
__device__ __forceinline__ uint32_t chunk_slot(const BuildArgs& B, uint32_t chunk) {
  return B.place ? B.place[chunk].slot : chunk;
}

// Exclusive scan of one value per thread over the CTA; *total gets the sum.
// Ends with a barrier, so `ws` may be reused at once.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* ws, uint32_t* total) {
  const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (uint32_t o = 1; o < 32u; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31u) ws[w] = x;
  __syncthreads();
  if (w == 0) {
    uint32_t s = lane < (uint32_t)SVO_WARPS ? ws[lane] : 0u;
#pragma unroll
    for (uint32_t o = 1; o < (uint32_t)SVO_WARPS; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < (uint32_t)SVO_WARPS) ws[lane] = s;
  }
  __syncthreads();
  const uint32_t base = w ? ws[w - 1] : 0u;
  *total = ws[SVO_WARPS - 1];
  __syncthreads();
  return base + x - v;
}

__device__ __forceinline__ uint32_t cell_key(uint32_t x, uint32_t y, uint32_t z, uint32_t level) {
  return x | (y << 6) | (z << 12) | (level << 18);
}

// State word of a level-l cell (l < 6) from its 8 children's present / leaf /
// full bits and materials (builder_svo.rs:337-534 collapse rules).
__device__ __forceinline__ uint32_t cell_state(const uint32_t (&cs)[8], int32_t top_y, int32_t gmin,
                                               int32_t dirt_depth) {
  uint32_t mask = 0, full = ST_FULL, uniform = 1u;
  const uint32_t m0 = (cs[0] >> 8) & 0xFFu;
#pragma unroll
  for (int ci = 0; ci < 8; ++ci) {
    if (cs[ci] & ST_MASK) mask |= 1u << ci;
    full &= cs[ci];
    uniform &= (cs[ci] & ST_LEAF) && (cs[ci] & ST_MASK) && ((cs[ci] >> 8) & 0xFFu) == m0 ? 1u : 0u;
  }
  if (!mask) return 0u;
  if (full && top_y < gmin - dirt_depth) return mask | ((uint32_t)VXE_MAT_STONE << 8) | ST_LEAF | ST_FULL;
  if (mask == 0xFFu && uniform) return mask | (m0 << 8) | ST_LEAF | full;
  return mask | full;
}

// Level-6 (voxel) pseudo state: present leaf, full, of its material.
__device__ __forceinline__ uint32_t voxel_state(uint32_t m) {
  return m ? (0x1u | (m << 8) | ST_LEAF | ST_FULL) : 0u;
}

// Materials of one voxel column, bottom-up.  terrain::material evaluated
// with its per-column work done once, every value still going through the
// same operations on the same operands, so the materials are the same:
//   - cave noise: per octave (lattice 16 and 8 voxels) the x-interpolated
//     lattice values of the current y cell are kept; moving up one cell
//     reuses the upper row as the new lower one.  The y fraction of a lattice
//     cell depends only on wy mod 16 (or 8), so its fade comes from a table
//     filled with terrain::fade.  The cave test s / 1.5 > threshold is
//     monotone in s = n1 + 0.5 n2, so it is s >= cave_smin, the least binary64
//     s that passes, found on the host;
//   - the light voxel test and the trees whose trunk or crown reaches the
//     column are found once.
struct ColumnMaterial {
  int32_t wx, wz, g;
  bool caves, light;
  int32_t ix[2], iz[2], iy[2];
  double fx[2], fz[2], yz[2][4];
  uint32_t ntrees;
  // trees reaching the column (at most the 4 x 4 candidate cells); kept apart
  // from the scalars above so those stay in registers
  struct T {
    int32_t dxx, dzz, cy, r2, base, top;  // base = INT32_MAX unless the trunk is this column
  };

  __device__ void init(const vxe_world_params& p, int32_t x, int32_t z, int32_t ground, T (&trees)[16]) {
    wx = x;
    wz = z;
    g = ground;
    caves = p.cave_threshold < 1.0f;
#pragma unroll
    for (int o = 0; o < 2; ++o) {
      const double div = o == 0 ? 16.0 : 8.0;
      const double xx = wx / div, zz = wz / div;
      const double gx = floor(xx), gz = floor(zz);
      ix[o] = (int32_t)gx;
      iz[o] = (int32_t)gz;
      fx[o] = terrain::fade(xx - gx);
      fz[o] = terrain::fade(zz - gz);
      iy[o] = INT32_MIN;
    }
    light = (p.features & 2u) && terrain::hash2(p.seed ^ 0x119u, wx, wz) % 331u == 0u;
    ntrees = 0;
    if (p.features & 1u) {
      const int32_t mx0 = (int32_t)floor((wx - 14) / 10.0), mx1 = (int32_t)floor((wx + 14) / 10.0);
      const int32_t mz0 = (int32_t)floor((wz - 14) / 10.0), mz1 = (int32_t)floor((wz + 14) / 10.0);
      for (int32_t mz = mz0; mz <= mz1; ++mz)
        for (int32_t mx = mx0; mx <= mx1; ++mx) {
          terrain::Tree t;
          if (!terrain::tree_at_cell(p, mx, mz, &t)) continue;
          const int32_t dx = wx - t.x, dz = wz - t.z;
          const bool trunk = wx == t.x && wz == t.z;
          if (!trunk && dx * dx + dz * dz > t.r * t.r) continue;  // neither trunk nor crown reaches the column
          T& e = trees[ntrees++];
          e.dxx = dx * dx;
          e.dzz = dz * dz;
          e.cy = t.base + t.trunk;
          e.r2 = t.r * t.r;
          e.base = trunk ? t.base : INT32_MAX;
          e.top = t.base + t.trunk;
        }
    }
  }

  // x-interpolated lattice row (iy + j, iz + k) of octave o
  __device__ __forceinline__ double row(uint32_t seed, int o, int32_t cy, int k) const {
    const double a = terrain::u01(terrain::hash3(seed, ix[o], cy, iz[o] + k));
    const double b = terrain::u01(terrain::hash3(seed, ix[o] + 1, cy, iz[o] + k));
    return a + (b - a) * fx[o];
  }

  // value_noise3 at (wx, wy, wz) / (16 or 8) for octave o; fy = fade of the
  // y fraction (table)
  __device__ __forceinline__ double noise(uint32_t seed, int o, int32_t cy, double fy) {
    if (cy != iy[o]) {
      if (cy == iy[o] + 1) {
        yz[o][0] = yz[o][1];
        yz[o][2] = yz[o][3];
      } else {
        yz[o][0] = row(seed, o, cy, 0);
        yz[o][2] = row(seed, o, cy, 1);
      }
      yz[o][1] = row(seed, o, cy + 1, 0);
      yz[o][3] = row(seed, o, cy + 1, 1);
      iy[o] = cy;
    }
    const double z0 = yz[o][0] + (yz[o][1] - yz[o][0]) * fy;
    const double z1 = yz[o][2] + (yz[o][3] - yz[o][2]) * fy;
    return z0 + (z1 - z0) * fz[o];
  }

  __device__ uint32_t at(const vxe_world_params& p, double cave_smin, const double* fade16, const double* fade8,
                         int32_t wy, const T (&trees)[16]) {
    uint32_t m;
    if (wy < g) {
      m = (wy >= g - p.dirt_depth) ? VXE_MAT_DIRT : VXE_MAT_STONE;
    } else if (wy == g) {
      m = VXE_MAT_GRASS;
    } else {
      m = VXE_MAT_AIR;
    }
    if (m != VXE_MAT_AIR) {
      bool cave = false;
      if (caves) {
        const uint32_t s = p.seed ^ 0xCA7E5EEDu;
        const double n1 = noise(s, 0, wy >> 4, fade16[wy & 15]);
        const double n2 = noise(s + 7u, 1, wy >> 3, fade8[wy & 7]);
        cave = n1 + 0.5 * n2 >= cave_smin;
      }
      if (cave) m = VXE_MAT_AIR;
      else if (p.carve_mod != 0u && terrain::hash3(p.seed ^ 0x5EEDu, wx, wy, wz) % p.carve_mod == 0u) m = VXE_MAT_AIR;
    }
    if (m == VXE_MAT_AIR && wy > g && p.features != 0u) {
      if (light && wy == g + 1) return VXE_MAT_LIGHT;
      uint32_t best = VXE_MAT_AIR;
      for (uint32_t i = 0; i < ntrees; ++i) {
        const T& e = trees[i];
        if (wy >= e.base && wy < e.top) return VXE_MAT_WOOD;
        const int32_t dy = wy - e.cy;
        if (e.dxx + dy * dy + e.dzz <= e.r2) best = VXE_MAT_LEAF;
      }
      m = best;
    }
    return m;
  }
};

// Lane layout of a column block: 16 x 16 columns, warp w covering rows
// z = 2w, 2w+1 with lane = x | (z & 1) << 4, so a 2x2 column group is lanes
// {l, l^1, l^16, l^17}.  Every 8 layers the group holds 4 level-5 cells; the
// lane of role r = (x & 1) | (z & 1) << 1 builds the state of cell r.
__global__ void __launch_bounds__(256) k_build_columns(const __grid_constant__ BuildArgs B) {
  __shared__ uint32_t red[8];
  __shared__ double fade16[16], fade8[8];
  if (threadIdx.x < 16) fade16[threadIdx.x] = terrain::fade((double)threadIdx.x / 16.0);
  else if (threadIdx.x < 24) fade8[threadIdx.x - 16] = terrain::fade((double)(threadIdx.x - 16) / 8.0);
  __syncthreads();
  const uint32_t chunk = blockIdx.x >> 4, tile = blockIdx.x & 15u;
  if (chunk >= B.n) return;
  const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  const uint32_t x = ((tile & 3u) << 4) | (lane & 15u), z = ((tile >> 2) << 4) | (w << 1) | (lane >> 4);
  const uint32_t role = (x & 1u) | ((z & 1u) << 1);
  const int32_t ox = chunk_coord(B, chunk, 0) * kSide, oy = chunk_coord(B, chunk, 1) * kSide,
                oz = chunk_coord(B, chunk, 2) * kSide;
  const int32_t wx = ox + (int32_t)x, wz = oz + (int32_t)z;
  const int32_t g = terrain::ground(B.wp, wx, wz);
  ColumnMaterial col;
  ColumnMaterial::T trees[16];
  col.init(B.wp, wx, wz, g, trees);
  const int32_t gx = min(g, __shfl_xor_sync(0xFFFFFFFFu, g, 1));
  const int32_t gmin = min(gx, __shfl_xor_sync(0xFFFFFFFFu, gx, 16));
  if (role == 0u) B.mip1[(size_t)chunk * 1024u + (z >> 1) * 32u + (x >> 1)] = gmin;
  uint8_t* mat = B.mat + (size_t)chunk * kVoxels + z * 64u + x;
  uint32_t* st5 = B.st5 + (size_t)chunk * kCells5 + (z >> 1) * 32u + (x >> 1);
  uint32_t top = 255u, top_m = 0u, solid = 0u;
  if (__all_sync(0xFFFFFFFFu, B.wp.features == 0u && oy > g)) {
    // Every voxel of the warp's 32 columns lies above its surface and the
    // world has no decorations: all air.  Materials and level-5 states are
    // zero; stored as 16-byte rows (16 x of one z row / 4 cells of one row).
    const uint32_t z0 = ((tile >> 2) << 4) | (w << 1), x0 = (tile & 3u) << 4;
    uint8_t* m0 = B.mat + (size_t)chunk * kVoxels + z0 * 64u + x0;
    for (uint32_t j = lane; j < 128u; j += 32u)  // 64 layers x 2 rows
      *reinterpret_cast<uint4*>(m0 + (j >> 1) * 4096u + (j & 1u) * 64u) = make_uint4(0u, 0u, 0u, 0u);
    uint32_t* s0 = B.st5 + (size_t)chunk * kCells5 + (z0 >> 1) * 32u + (x0 >> 1);
    for (uint32_t j = lane; j < 64u; j += 32u)  // 32 cell layers x 8 cells
      *reinterpret_cast<uint4*>(s0 + (j >> 1) * 1024u + (j & 1u) * 4u) = make_uint4(0u, 0u, 0u, 0u);
  } else {
#pragma unroll 1
  for (uint32_t kb = 0; kb < 8u; ++kb) {
    uint64_t acc = 0;  // 16 bits per layer pair: materials of y = 2k, 2k+1
#pragma unroll 1
    for (uint32_t y = 8u * kb; y < 8u * kb + 8u; ++y) {
      const uint32_t m = col.at(B.wp, B.cave_smin, fade16, fade8, oy + (int32_t)y, trees);
      mat[y * 4096u] = (uint8_t)m;
      if (m) {
        top = y;
        top_m = m;
        ++solid;
      }
      acc |= (uint64_t)m << (8u * (y - 8u * kb));
    }
    // lane l sends the pair its partner needs: partner role = role ^ d
    const uint32_t own = (uint32_t)(acc >> (16u * role)) & 0xFFFFu;
    const uint32_t fx1 = __shfl_xor_sync(0xFFFFFFFFu, (uint32_t)(acc >> (16u * (role ^ 1u))) & 0xFFFFu, 1);
    const uint32_t fz1 = __shfl_xor_sync(0xFFFFFFFFu, (uint32_t)(acc >> (16u * (role ^ 2u))) & 0xFFFFu, 16);
    const uint32_t fxz = __shfl_xor_sync(0xFFFFFFFFu, (uint32_t)(acc >> (16u * (role ^ 3u))) & 0xFFFFu, 17);
    uint32_t cs[8];
#pragma unroll
    for (int ci = 0; ci < 8; ++ci) {
      // the column at offset d = (dx, dz) from the group's x-even / z-even
      // column is the lane of role d, i.e. this lane ^ (d ^ role)
      const uint32_t f = ((uint32_t)(ci & 1) | (uint32_t)((ci >> 1) & 2)) ^ role;
      const uint32_t pair = f == 0u ? own : f == 1u ? fx1 : f == 2u ? fz1 : fxz;
      cs[ci] = voxel_state((pair >> (8 * ((ci >> 1) & 1))) & 0xFFu);
    }
    const uint32_t k = 4u * kb + role;
    st5[k * 1024u] = cell_state(cs, oy + (int32_t)(2u * k + 1u), gmin, B.wp.dirt_depth);
  }
  }
  // colinfo (builder.rs:742-771): column pairs (x even, x odd) share a word
  const uint32_t e = top | (top_m << 8), eo = __shfl_xor_sync(0xFFFFFFFFu, e, 1);
  if ((lane & 1u) == 0u)
    B.colinfo[(size_t)chunk_slot(B, chunk) * VXE_COLINFO_WORDS_PER_CHUNK + ((z * 64u + x) >> 1)] = e | (eo << 16);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) solid += __shfl_xor_sync(0xFFFFFFFFu, solid, o);
  if (lane == 0) red[w] = solid;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t sum = 0;
    for (int i = 0; i < 8; ++i) sum += red[i];
    B.solid_part[(size_t)chunk * 16u + tile] = sum;
  }
}

__device__ __forceinline__ vxe_node node_of(uint32_t st, uint32_t kid_base, uint32_t key) {
  vxe_node n;
  if (st & ST_LEAF) {
    n.child_base = kInvalid;
    n.child_mask = 0u;
    n.material = (st >> 8) & 0xFFu;
  } else {
    n.child_base = kid_base;
    n.child_mask = st & ST_MASK;
    n.material = 0u;
  }
  n.key = key;
  return n;
}

// builder_ropes.rs "down": the neighbour itself when it is a leaf (or
// absent), else its child on the near side (`ci`), absent when not present.
__device__ __forceinline__ uint32_t rope_down(uint32_t nei, const vxe_node& n, uint32_t ci) {
  if (nei == kInvalid) return kInvalid;
  if (n.child_base == kInvalid) return nei;
  if (!(n.child_mask & (1u << ci))) return kInvalid;
  return n.child_base + (uint32_t)__popc(n.child_mask & ((1u << ci) - 1u));
}

// Node index of the present level-l cell (x, y, z), l = 1..5, whose parent
// is internal: its parent's child offset plus its rank among the parent's
// present children (state words and offsets of levels 4..0 in shared memory).
__device__ __forceinline__ uint32_t level_node(const uint32_t* st, const uint32_t* kb, const uint32_t* bases, int l,
                                               uint32_t x, uint32_t y, uint32_t z) {
  const int pl = l - 1;
  const uint32_t ps = 1u << pl;
  const uint32_t pi = (x >> 1) + ((z >> 1) + (y >> 1) * ps) * ps;
  const uint32_t ci = (x & 1u) | ((y & 1u) << 1) | ((z & 1u) << 2);
  const uint32_t mask = st[low_off(pl) + pi] & ST_MASK;
  return bases[l] + kb[low_off(pl) + pi] + (uint32_t)__popc(mask & ((1u << ci) - 1u));
}

// Counts and, for a resident build, the slot's ChunkMetaGpu (macro_empty <=>
// no solid voxel); a resident chunk needing more nodes than its place
// reserves gets an empty meta and the error bit.
__device__ void write_counts_meta(const BuildArgs& B, uint32_t chunk, uint32_t node_count, uint32_t solid) {
  if (B.counts) {
    B.counts[2u * chunk] = node_count;
    B.counts[2u * chunk + 1u] = solid;
  }
  if (B.place) {
    const vxe_build_place& pl = B.place[chunk];
    const bool fits = node_count <= pl.node_count;
    vxe_chunk_meta m;
    m.origin[0] = pl.cx * kSide;
    m.origin[1] = pl.cy * kSide;
    m.origin[2] = pl.cz * kSide;
    m.origin[3] = 0;
    m.node_base = pl.node_base;
    m.node_count = fits ? node_count : 0u;
    m.macro_base = pl.slot * VXE_MACRO_WORDS_PER_CHUNK;
    m.colinfo_base = pl.slot * VXE_COLINFO_WORDS_PER_CHUNK;
    m.macro_empty = fits ? (solid == 0u ? 1u : 0u) : 1u;
    m._pad0 = m._pad1 = m._pad2 = 0u;
    B.metas[pl.slot] = m;
    if (!fits) atomicOr(B.error_word, ERR_BUILD);
  }
}

__global__ void __launch_bounds__(SVO_THREADS, 2) k_build_svo(const __grid_constant__ BuildArgs B) {
  __shared__ uint32_t st[kLowCells];
  __shared__ uint32_t kb[kLowCells];
  __shared__ int32_t mip[kMipWords];
  __shared__ uint32_t ws[SVO_WARPS];
  __shared__ uint32_t K[8];  // K[l]: entries of level l's node list (l = 1..6)
  __shared__ uint32_t bases[8];
  extern __shared__ uint4 stage[];  // kStageNodes voxel records of one level-5 round

  const uint32_t chunk = blockIdx.x, t = threadIdx.x;
  if (chunk >= B.n) return;
  const uint8_t* mat = B.mat + (size_t)chunk * kVoxels;
  uint32_t* st5 = B.st5 + (size_t)chunk * kCells5;
  uint32_t* kb5 = B.kb5 + (size_t)chunk * kCells5;
  const int32_t chunk_oy = chunk_coord(B, chunk, 1) * kSide;
  const int32_t dirt = B.wp.dirt_depth;
  uint32_t solid = 0;
#pragma unroll
  for (int i = 0; i < 16; ++i) solid += B.solid_part[(size_t)chunk * 16u + i];
  if (solid == 0u) {
    // No solid voxel: the list is the root alone, an air leaf with no
    // neighbours; every macro bit is clear (what the general path gives).
    const uint32_t cap = B.place ? B.place[chunk].node_count : B.node_cap;
    if (t < VXE_MACRO_WORDS_PER_CHUNK) B.macro[(size_t)chunk_slot(B, chunk) * VXE_MACRO_WORDS_PER_CHUNK + t] = 0u;
    if (t == 0) {
      write_counts_meta(B, chunk, 1u, 0u);
      if (cap >= 1u) {
        const size_t node0 = B.place ? (size_t)B.place[chunk].node_base : (size_t)chunk * cap;
        B.nodes[node0] = node_of(ST_LEAF, 0u, 0u);
        vxe_node_ropes r;
        r.px = r.nx = r.py = r.ny = r.pz = r.nz = kInvalid;
        r._pad0 = r._pad1 = 0u;
        B.ropes[node0] = r;
      }
    }
    return;
  }

  // -- ground min-mip levels 1..6 (mips.rs:4-90) ------------------------------
  for (uint32_t i = t; i < 1024u; i += SVO_THREADS) mip[i] = B.mip1[(size_t)chunk * 1024u + i];
  __syncthreads();
  for (int lv = 2; lv <= 6; ++lv) {
    const uint32_t side = 64u >> lv, cside = side * 2u;
    const int32_t* c = mip + mip_off(lv - 1);
    for (uint32_t i = t; i < side * side; i += SVO_THREADS) {
      const uint32_t x = i % side, z = i / side;
      const uint32_t i00 = (2u * z) * cside + 2u * x;
      mip[mip_off(lv) + i] = min(min(c[i00], c[i00 + 1]), min(c[i00 + cside], c[i00 + cside + 1]));
    }
    __syncthreads();
  }

  // -- levels 4..0 states (level 5 comes from the column kernel) -------------
  for (uint32_t j = 0; j < 8u; j += 2u) {  // level 4: two cells per step, 8 st5 loads each
    uint2 q[2][4];
#pragma unroll
    for (uint32_t u = 0; u < 2u; ++u) {
      const uint32_t i = t + SVO_THREADS * (j + u), px = i & 15u, pz = (i >> 4) & 15u, py = i >> 8;
#pragma unroll
      for (uint32_t d = 0; d < 4u; ++d)  // d = dy * 2 + dz
        q[u][d] = *reinterpret_cast<const uint2*>(st5 + ((2u * py + (d >> 1)) * 32u + 2u * pz + (d & 1u)) * 32u + 2u * px);
    }
#pragma unroll
    for (uint32_t u = 0; u < 2u; ++u) {
      const uint32_t i = t + SVO_THREADS * (j + u), px = i & 15u, pz = (i >> 4) & 15u, py = i >> 8;
      uint32_t cs[8];
#pragma unroll
      for (int ci = 0; ci < 8; ++ci) {
        const uint2 v = q[u][((ci >> 1) & 1) * 2 + ((ci >> 2) & 1)];
        cs[ci] = (ci & 1) ? v.y : v.x;
      }
      st[low_off(4) + i] = cell_state(cs, chunk_oy + (int32_t)(py * 4u + 3u), mip[mip_off(2) + pz * 16u + px], dirt);
    }
  }
  __syncthreads();
  for (int l = 3; l >= 0; --l) {
    const uint32_t side = 1u << l, cells = side * side * side, cside = side * 2u;
    const uint32_t* cst = st + low_off(l + 1);
    const uint32_t psize = 64u >> l;
    for (uint32_t i = t; i < cells; i += SVO_THREADS) {
      const uint32_t px = i & (side - 1u), pz = (i >> l) & (side - 1u), py = i >> (2 * l);
      uint32_t cs[8];
#pragma unroll
      for (int ci = 0; ci < 8; ++ci)
        cs[ci] = cst[((2u * py + ((ci >> 1) & 1)) * cside + 2u * pz + ((ci >> 2) & 1)) * cside + 2u * px + (ci & 1)];
      const int32_t top_y = chunk_oy + (int32_t)(py * psize + psize - 1u);
      const int32_t gmin = mip[mip_off(6 - l) + pz * side + px];
      st[low_off(l) + i] = cell_state(cs, top_y, gmin, dirt);
    }
    __syncthreads();
  }

  // -- child offsets of levels 4..0 -------------------------------------------
  {
    // level 4: 8 consecutive cells per thread
    uint32_t cnt[8], sum = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const uint32_t s = st[low_off(4) + 8u * t + k];
      cnt[k] = (s & ST_MASK) && !(s & ST_LEAF) ? (uint32_t)__popc(s & ST_MASK) : 0u;
      sum += cnt[k];
    }
    uint32_t total;
    uint32_t off = block_excl_scan(sum, ws, &total);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      kb[low_off(4) + 8u * t + k] = off;
      off += cnt[k];
    }
    if (t == 0) K[5] = total;
    for (int l = 3; l >= 0; --l) {
      const uint32_t cells = 1u << (3 * l);
      const uint32_t s = t < cells ? st[low_off(l) + t] : 0u;
      const uint32_t c = (s & ST_MASK) && !(s & ST_LEAF) ? (uint32_t)__popc(s & ST_MASK) : 0u;
      const uint32_t o = block_excl_scan(c, ws, &total);
      if (t < cells) kb[low_off(l) + t] = o;
      if (t == 0) K[l + 1] = total;
    }
  }
  __syncthreads();
  // bases[l] = first node of level l's list (l = 1..6)
  if (t == 0) {
    bases[0] = 0u;
    bases[1] = 1u;
    for (int l = 2; l <= 6; ++l) bases[l] = bases[l - 1] + K[l - 1];
  }
  __syncthreads();

  // -- level-5 child offsets and the voxel list: 16 rounds of 2048 cells, 4
  // consecutive cells (one row of 8 voxels in x) per thread; each round's
  // loads are issued before the previous round's scan.  Voxel records go out
  // as their offsets become known, each one only below node_cap.
  const uint32_t cap = B.place ? B.place[chunk].node_count : B.node_cap;
  const size_t first = B.place ? (size_t)B.place[chunk].node_base : (size_t)chunk * cap;
  vxe_node* nodes = B.nodes + first;
  vxe_node_ropes* ropes = B.ropes + first;
  uint32_t carry = 0;
  uint4 s4;
  uint64_t rows[4];  // d = dy * 2 + dz: the 8 voxels (x = 8 * (t & 7) ...) of each row
  auto load_round = [&](uint32_t r, uint4& sv, uint64_t (&rw)[4]) {
    const uint32_t c0 = r * 2048u + 4u * t, px0 = c0 & 31u, pz = (c0 >> 5) & 31u, py = c0 >> 10;
    sv = *reinterpret_cast<const uint4*>(st5 + c0);
#pragma unroll
    for (uint32_t d = 0; d < 4u; ++d)
      rw[d] = *reinterpret_cast<const uint64_t*>(mat + (2u * py + (d >> 1)) * 4096u + (2u * pz + (d & 1u)) * 64u + 2u * px0);
  };
  load_round(0, s4, rows);
#pragma unroll 1
  for (uint32_t r = 0; r < 16u; ++r) {
    const uint32_t c0 = r * 2048u + 4u * t, px0 = c0 & 31u, pz = (c0 >> 5) & 31u, py = c0 >> 10;
    const uint32_t sv[4] = {s4.x, s4.y, s4.z, s4.w};
    const uint64_t rw[4] = {rows[0], rows[1], rows[2], rows[3]};
    if (r + 1u < 16u) load_round(r + 1u, s4, rows);
    uint32_t cnt[4], sum = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      cnt[k] = (sv[k] & ST_MASK) && !(sv[k] & ST_LEAF) ? (uint32_t)__popc(sv[k] & ST_MASK) : 0u;
      sum += cnt[k];
    }
    uint32_t total;
    const uint32_t round0 = carry;
    const uint32_t off0 = carry + block_excl_scan(sum, ws, &total);
    carry += total;
    const bool staged = total <= kStageNodes;  // block-uniform
    uint32_t off = off0;
    uint4 kv;
    kv.x = off; off += cnt[0];
    kv.y = off; off += cnt[1];
    kv.z = off; off += cnt[2];
    kv.w = off;
    *reinterpret_cast<uint4*>(kb5 + c0) = kv;
    uint32_t o = bases[6] + off0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (!cnt[k]) continue;
#pragma unroll
      for (int ci = 0; ci < 8; ++ci) {
        if (!((sv[k] >> ci) & 1u)) continue;
        const uint32_t cx = 2u * (px0 + k) + (ci & 1), cy = 2u * py + ((ci >> 1) & 1), cz = 2u * pz + ((ci >> 2) & 1);
        const uint32_t mat_ci =
            (uint32_t)(rw[((ci >> 1) & 1) * 2 + ((ci >> 2) & 1)] >> (8 * (2 * k + (ci & 1)))) & 0xFFu;
        const uint4 rec = make_uint4(kInvalid, 0u, mat_ci, cell_key(cx, cy, cz, 6u));
        if (staged) stage[o - bases[6] - round0] = rec;
        else if (o < cap) *reinterpret_cast<uint4*>(nodes + o) = rec;
        ++o;
      }
    }
    if (staged) {  // the round's records leave shared memory as one contiguous run
      __syncthreads();
      const uint32_t first = bases[6] + round0;
      for (uint32_t i = t; i < total; i += SVO_THREADS)
        if (first + i < cap) *reinterpret_cast<uint4*>(nodes + first + i) = stage[i];
      // the next round's scan barriers order these reads before its stores
    }
  }
  if (t == 0) {
    K[6] = carry;
    bases[7] = bases[6] + carry;
  }
  __syncthreads();  // kb5 and the voxel records visible to the CTA
  const uint32_t node_count = bases[7];

  if (t == 0) write_counts_meta(B, chunk, node_count, solid);
  // macro bits: bit mx + 8*(my + 8*mz) <=> level-3 cell present (builder.rs:809-841)
  if (t < VXE_MACRO_WORDS_PER_CHUNK) {
    uint32_t word = 0;
    for (uint32_t b = 0; b < 32u; ++b) {
      const uint32_t bit = 32u * t + b, mx = bit & 7u, my = (bit >> 3) & 7u, mz = bit >> 6;
      if (st[low_off(3) + mx + (mz << 3) + (my << 6)] & ST_MASK) word |= 1u << b;
    }
    B.macro[(size_t)chunk_slot(B, chunk) * VXE_MACRO_WORDS_PER_CHUNK + t] = word;
  }
  if (node_count > cap) return;  // the caller rebuilds with a larger cap

  // -- emission: the root, then each internal cell's children ---------------
  if (t == 0) {
    const uint32_t s = st[low_off(0)];
    nodes[0] = s & ST_MASK ? node_of(s, kb[low_off(0)] + bases[1], 0u) : node_of(ST_LEAF, 0u, 0u);
  }
  for (int l = 0; l <= 4; ++l) {  // parents of levels 0..4, children of levels 1..5
    const uint32_t side = 1u << l, cells = side * side * side, cside = side * 2u;
    for (uint32_t i = t; i < cells; i += SVO_THREADS) {
      const uint32_t s = st[low_off(l) + i];
      if (!(s & ST_MASK) || (s & ST_LEAF)) continue;
      const uint32_t px = i & (side - 1u), pz = (i >> l) & (side - 1u), py = i >> (2 * l);
      uint32_t cs[8], ckb[8];
#pragma unroll
      for (int ci = 0; ci < 8; ++ci) {  // all child loads first
        const uint32_t c = ((2u * py + ((ci >> 1) & 1)) * cside + 2u * pz + ((ci >> 2) & 1)) * cside + 2u * px + (ci & 1);
        const bool has = (s >> ci) & 1u;
        cs[ci] = !has ? 0u : l == 4 ? st5[c] : st[low_off(l + 1) + c];
        ckb[ci] = !has ? 0u : l == 4 ? kb5[c] : kb[low_off(l + 1) + c];
      }
      uint32_t o = bases[l + 1] + kb[low_off(l) + i];
#pragma unroll
      for (int ci = 0; ci < 8; ++ci) {
        if (!((s >> ci) & 1u)) continue;
        const uint32_t cx = 2u * px + (ci & 1), cy = 2u * py + ((ci >> 1) & 1), cz = 2u * pz + ((ci >> 2) & 1);
        nodes[o++] = node_of(cs[ci], ckb[ci] + bases[l + 2], cell_key(cx, cy, cz, (uint32_t)l + 1u));
      }
    }
  }
  __syncthreads();  // node records visible to the CTA

  // -- ropes, top-down (builder_ropes.rs:76-195) -------------------------------
  if (t == 0) {
    vxe_node_ropes r;
    r.px = r.nx = r.py = r.ny = r.pz = r.nz = kInvalid;
    r._pad0 = r._pad1 = 0u;
    ropes[0] = r;
  }
  __syncthreads();
  // One thread per node of level l's list (consecutive lanes, consecutive
  // records): its parent -- the node of the cell above it, found from its key
  // and the shared level states -- and the parent's ropes and children give
  // its 6 ropes; siblings read the same parent and neighbour records, so those
  // loads hit L1.
  for (int l = 1; l <= 6; ++l) {
    const uint32_t lo = bases[l], hi = bases[l] + K[l];
    for (uint32_t k = lo + t; k < hi; k += SVO_THREADS) {
      const uint32_t key = nodes[k].key;
      const uint32_t hx = key & 1u, hy = (key >> 6) & 1u, hz = (key >> 12) & 1u;
      const uint32_t p = l == 1 ? 0u
                                : level_node(st, kb, bases, l - 1, (key & 63u) >> 1, ((key >> 6) & 63u) >> 1,
                                             ((key >> 12) & 63u) >> 1);
      const uint32_t ci = hx | (hy << 1) | (hz << 2);
      const vxe_node pn = nodes[p];
      const vxe_node_ropes pr = ropes[p];
      auto kid = [&](uint32_t c) -> uint32_t {
        return (pn.child_mask & (1u << c)) ? pn.child_base + (uint32_t)__popc(pn.child_mask & ((1u << c) - 1u))
                                           : kInvalid;
      };
      auto down = [&](uint32_t nei, uint32_t c) -> uint32_t {
        return nei == kInvalid ? kInvalid : rope_down(nei, nodes[nei], c);
      };
      const uint32_t sx = kid(ci ^ 1u), sy = kid(ci ^ 2u), sz = kid(ci ^ 4u);
      vxe_node_ropes r;
      r.px = (hx == 0 && sx != kInvalid) ? sx : down(pr.px, 0u | (hy << 1) | (hz << 2));
      r.nx = (hx == 1 && sx != kInvalid) ? sx : down(pr.nx, 1u | (hy << 1) | (hz << 2));
      r.py = (hy == 0 && sy != kInvalid) ? sy : down(pr.py, hx | (0u << 1) | (hz << 2));
      r.ny = (hy == 1 && sy != kInvalid) ? sy : down(pr.ny, hx | (1u << 1) | (hz << 2));
      r.pz = (hz == 0 && sz != kInvalid) ? sz : down(pr.pz, hx | (hy << 1) | (0u << 2));
      r.nz = (hz == 1 && sz != kInvalid) ? sz : down(pr.nz, hx | (hy << 1) | (1u << 2));
      r._pad0 = r._pad1 = 0u;
      ropes[k] = r;
    }
    __syncthreads();
  }
}

}  // namespace build
}  // namespace vxe
