// build_kernels.cuh -- the chunk builder on the device.
//
// The reference builds chunks on CPU worker threads (svo/builder.rs:846-986):
// material fill, column tops and colinfo (builder.rs:742-805), macro
// occupancy (builder.rs:809-841), ground min-mip (mips.rs:4-90), the
// bottom-up octree with stone and uniform collapse (builder_svo.rs:337-534)
// and ropes (builder_ropes.rs:76-195).  These kernels produce the same
// records byte for byte for a batch of chunks:
//
//   k_build_ground  one thread per column: surface height (z*64 + x)
//   k_build_fill    one thread per voxel: material (y*64*64 + z*64 + x)
//   k_build_svo     one CTA per chunk: colinfo, macro bits, the octree cell
//                   states bottom-up, one exclusive scan per level for the
//                   packed child offsets, node emission, ropes top-down.
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
  const int32_t* coords;  // n chunk coordinates (x, y, z)
  uint32_t n;
  uint8_t* mat;           // n * 64^3 materials
  int32_t* ground;        // n * 64^2 surface heights
  uint32_t* st5;          // n * 32^3 level-5 state words
  uint32_t* kb5;          // n * 32^3 level-5 child offsets
  uint32_t node_cap;
  vxe_node* nodes;        // n * node_cap
  vxe_node_ropes* ropes;  // n * node_cap
  uint32_t* macro;        // n * 16
  uint32_t* colinfo;      // n * 2048
  uint32_t* counts;       // n * 2: node_count, solid_voxels
};

__global__ void __launch_bounds__(256) k_build_ground(const __grid_constant__ BuildArgs B) {
  const uint32_t chunk = blockIdx.x >> 4, col = ((blockIdx.x & 15u) << 8) | threadIdx.x;
  if (chunk >= B.n) return;
  const int32_t ox = B.coords[3 * chunk] * kSide, oz = B.coords[3 * chunk + 2] * kSide;
  B.ground[(size_t)chunk * kColumns + col] = terrain::ground(B.wp, ox + (int32_t)(col & 63u), oz + (int32_t)(col >> 6));
}

__global__ void __launch_bounds__(256) k_build_fill(const __grid_constant__ BuildArgs B) {
  const uint32_t chunk = blockIdx.x >> 10, i = ((blockIdx.x & 1023u) << 8) | threadIdx.x;
  if (chunk >= B.n) return;
  const int32_t ox = B.coords[3 * chunk] * kSide, oy = B.coords[3 * chunk + 1] * kSide,
                oz = B.coords[3 * chunk + 2] * kSide;
  const int32_t g = B.ground[(size_t)chunk * kColumns + (i & 4095u)];
  B.mat[(size_t)chunk * kVoxels + i] =
      terrain::material(B.wp, ox + (int32_t)(i & 63u), oy + (int32_t)(i >> 12), oz + (int32_t)((i >> 6) & 63u), g);
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

__device__ __forceinline__ uint32_t child_of(const vxe_node* nodes, uint32_t p, uint32_t ci) {
  const vxe_node n = nodes[p];
  if (!(n.child_mask & (1u << ci))) return kInvalid;
  return n.child_base + (uint32_t)__popc(n.child_mask & ((1u << ci) - 1u));
}

__device__ __forceinline__ uint32_t rope_down(const vxe_node* nodes, uint32_t nei, uint32_t ci) {
  if (nei == kInvalid) return kInvalid;
  if (nodes[nei].child_base == kInvalid) return nei;
  return child_of(nodes, nei, ci);
}

__global__ void __launch_bounds__(SVO_THREADS, 2) k_build_svo(const __grid_constant__ BuildArgs B) {
  __shared__ uint32_t st[kLowCells];
  __shared__ uint32_t kb[kLowCells];
  __shared__ int32_t mip[kMipWords];
  __shared__ uint32_t ws[SVO_WARPS];
  __shared__ uint32_t red[SVO_WARPS];
  __shared__ uint32_t K[8];  // K[l]: entries of level l's node list (l = 1..6)

  const uint32_t chunk = blockIdx.x, t = threadIdx.x;
  if (chunk >= B.n) return;
  const uint8_t* mat = B.mat + (size_t)chunk * kVoxels;
  const int32_t* ground = B.ground + (size_t)chunk * kColumns;
  uint32_t* st5 = B.st5 + (size_t)chunk * kCells5;
  uint32_t* kb5 = B.kb5 + (size_t)chunk * kCells5;
  const int32_t chunk_oy = B.coords[3 * chunk + 1] * kSide;
  const int32_t dirt = B.wp.dirt_depth;

  // -- column tops -> colinfo (builder.rs:742-805), solid voxel count --------
  {
    uint32_t solid = 0;
    const uint32_t* mw = reinterpret_cast<const uint32_t*>(mat);
    for (uint32_t w = t; w < kColumns / 4u; w += SVO_THREADS) {  // 4 columns per word
      uint32_t top[4] = {255u, 255u, 255u, 255u}, tm[4] = {0u, 0u, 0u, 0u};
      for (uint32_t y = 0; y < 64u; ++y) {
        const uint32_t v = mw[y * (kColumns / 4u) + w];
        if (!v) continue;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const uint32_t m = (v >> (8 * k)) & 0xFFu;
          if (m) { top[k] = y; tm[k] = m; ++solid; }
        }
      }
      uint32_t* ci = B.colinfo + (size_t)chunk * VXE_COLINFO_WORDS_PER_CHUNK + 2u * w;
      ci[0] = (top[0] | (tm[0] << 8)) | ((top[1] | (tm[1] << 8)) << 16);
      ci[1] = (top[2] | (tm[2] << 8)) | ((top[3] | (tm[3] << 8)) << 16);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) solid += __shfl_xor_sync(0xFFFFFFFFu, solid, o);
    if ((t & 31u) == 0) red[t >> 5] = solid;
  }

  // -- ground min-mip levels 1..6 (mips.rs:4-90) ------------------------------
  for (uint32_t i = t; i < 1024u; i += SVO_THREADS) {
    const uint32_t x = i & 31u, z = i >> 5;
    const int32_t* g = ground + (2u * z) * 64u + 2u * x;
    mip[i] = min(min(g[0], g[1]), min(g[64], g[65]));
  }
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

  // -- level 5 states + child offsets: 16 rounds of 2048 cells, 4 per thread --
  uint32_t carry = 0;
  for (uint32_t r = 0; r < 16u; ++r) {
    const uint32_t c0 = r * 2048u + 4u * t;  // 4 consecutive px of one (py, pz) row
    const uint32_t px0 = c0 & 31u, pz = (c0 >> 5) & 31u, py = c0 >> 10;
    uint32_t s4[4], cnt[4], sum = 0;
    uint64_t rows[2][2];
#pragma unroll
    for (int dy = 0; dy < 2; ++dy)
#pragma unroll
      for (int dz = 0; dz < 2; ++dz)
        rows[dy][dz] = *reinterpret_cast<const uint64_t*>(mat + (2u * py + dy) * 4096u + (2u * pz + dz) * 64u + 2u * px0);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      uint32_t cs[8];
#pragma unroll
      for (int ci = 0; ci < 8; ++ci)
        cs[ci] = voxel_state((uint32_t)(rows[(ci >> 1) & 1][(ci >> 2) & 1] >> (8 * (2 * k + (ci & 1)))) & 0xFFu);
      const int32_t top_y = chunk_oy + (int32_t)(py * 2u) + 1;
      const int32_t gmin = mip[mip_off(1) + pz * 32u + px0 + k];
      s4[k] = cell_state(cs, top_y, gmin, dirt);
      cnt[k] = (s4[k] & ST_MASK) && !(s4[k] & ST_LEAF) ? (uint32_t)__popc(s4[k] & ST_MASK) : 0u;
      sum += cnt[k];
    }
    uint32_t total;
    uint32_t off = carry + block_excl_scan(sum, ws, &total);
    carry += total;
    uint4 kv;
    kv.x = off; off += cnt[0];
    kv.y = off; off += cnt[1];
    kv.z = off; off += cnt[2];
    kv.w = off;
    *reinterpret_cast<uint4*>(st5 + c0) = make_uint4(s4[0], s4[1], s4[2], s4[3]);
    *reinterpret_cast<uint4*>(kb5 + c0) = kv;
  }
  if (t == 0) K[6] = carry;
  __syncthreads();  // st5 visible to the CTA

  // -- levels 4..0 states ---------------------------------------------------
  for (int l = 4; l >= 0; --l) {
    const uint32_t side = 1u << l, cells = side * side * side, cside = side * 2u;
    const uint32_t* cst = l == 4 ? st5 : st + low_off(l + 1);
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

  // bases[l] = first node of level l's list
  uint32_t bases[8];
  bases[0] = 0u;
  bases[1] = 1u;
#pragma unroll
  for (int l = 2; l <= 7; ++l) bases[l] = bases[l - 1] + K[l - 1];
  const uint32_t node_count = bases[6] + K[6];

  if (t == 0) {
    uint32_t solid = 0;
    for (int w = 0; w < SVO_WARPS; ++w) solid += red[w];
    B.counts[2u * chunk] = node_count;
    B.counts[2u * chunk + 1u] = solid;
  }
  // macro bits: bit mx + 8*(my + 8*mz) <=> level-3 cell present (builder.rs:809-841)
  if (t < VXE_MACRO_WORDS_PER_CHUNK) {
    uint32_t word = 0;
    for (uint32_t b = 0; b < 32u; ++b) {
      const uint32_t bit = 32u * t + b, mx = bit & 7u, my = (bit >> 3) & 7u, mz = bit >> 6;
      if (st[low_off(3) + mx + (mz << 3) + (my << 6)] & ST_MASK) word |= 1u << b;
    }
    B.macro[(size_t)chunk * VXE_MACRO_WORDS_PER_CHUNK + t] = word;
  }
  if (node_count > B.node_cap) return;  // the caller rebuilds with a larger cap

  vxe_node* nodes = B.nodes + (size_t)chunk * B.node_cap;
  vxe_node_ropes* ropes = B.ropes + (size_t)chunk * B.node_cap;

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
      uint32_t o = bases[l + 1] + kb[low_off(l) + i];
#pragma unroll 1
      for (int ci = 0; ci < 8; ++ci) {
        if (!(s & (1u << ci))) continue;
        const uint32_t cx = 2u * px + (ci & 1), cy = 2u * py + ((ci >> 1) & 1), cz = 2u * pz + ((ci >> 2) & 1);
        const uint32_t c = (cy * cside + cz) * cside + cx;
        const uint32_t cs = l == 4 ? st5[c] : st[low_off(l + 1) + c];
        const uint32_t ckb = l == 4 ? kb5[c] : kb[low_off(l + 1) + c];
        nodes[o++] = node_of(cs, ckb + bases[l + 2], cell_key(cx, cy, cz, (uint32_t)l + 1u));
      }
    }
  }
  for (uint32_t i = t; i < kCells5; i += SVO_THREADS) {  // level-5 parents, voxel children
    const uint32_t s = st5[i];
    if (!(s & ST_MASK) || (s & ST_LEAF)) continue;
    const uint32_t px = i & 31u, pz = (i >> 5) & 31u, py = i >> 10;
    uint32_t o = bases[6] + kb5[i];
#pragma unroll 1
    for (int ci = 0; ci < 8; ++ci) {
      if (!(s & (1u << ci))) continue;
      const uint32_t cx = 2u * px + (ci & 1), cy = 2u * py + ((ci >> 1) & 1), cz = 2u * pz + ((ci >> 2) & 1);
      vxe_node n;
      n.child_base = kInvalid;
      n.child_mask = 0u;
      n.material = mat[cy * 4096u + cz * 64u + cx];
      n.key = cell_key(cx, cy, cz, 6u);
      nodes[o++] = n;
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
  for (int l = 0; l <= 5; ++l) {  // parents in level l's list
    const uint32_t lo = bases[l], hi = l == 0 ? 1u : bases[l] + K[l];
    for (uint32_t p = lo + t; p < hi; p += SVO_THREADS) {
      const vxe_node pn = nodes[p];
      if (pn.child_base == kInvalid) continue;
      const vxe_node_ropes pr = ropes[p];
      uint32_t kid[8];
#pragma unroll
      for (uint32_t ci = 0; ci < 8; ++ci)
        kid[ci] = (pn.child_mask & (1u << ci)) ? pn.child_base + (uint32_t)__popc(pn.child_mask & ((1u << ci) - 1u))
                                                : kInvalid;
#pragma unroll 1
      for (uint32_t ci = 0; ci < 8; ++ci) {
        if (kid[ci] == kInvalid) continue;
        const uint32_t hx = ci & 1u, hy = (ci >> 1) & 1u, hz = (ci >> 2) & 1u;
        const uint32_t sx = kid[ci ^ 1u], sy = kid[ci ^ 2u], sz = kid[ci ^ 4u];
        vxe_node_ropes r;
        r.px = (hx == 0 && sx != kInvalid) ? sx : rope_down(nodes, pr.px, 0u | (hy << 1) | (hz << 2));
        r.nx = (hx == 1 && sx != kInvalid) ? sx : rope_down(nodes, pr.nx, 1u | (hy << 1) | (hz << 2));
        r.py = (hy == 0 && sy != kInvalid) ? sy : rope_down(nodes, pr.py, hx | (0u << 1) | (hz << 2));
        r.ny = (hy == 1 && sy != kInvalid) ? sy : rope_down(nodes, pr.ny, hx | (1u << 1) | (hz << 2));
        r.pz = (hz == 0 && sz != kInvalid) ? sz : rope_down(nodes, pr.pz, hx | (hy << 1) | (0u << 2));
        r.nz = (hz == 1 && sz != kInvalid) ? sz : rope_down(nodes, pr.nz, hx | (hy << 1) | (1u << 2));
        r._pad0 = r._pad1 = 0u;
        ropes[kid[ci]] = r;
      }
    }
    __syncthreads();
  }
}

}  // namespace build
}  // namespace vxe
