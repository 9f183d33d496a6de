// producer.cpp -- host-side data producers for the vxe passes.
//
// C++ port of the reference producers that feed the primary / godray /
// composite bindings:
//   * seeded synthetic world (replaces world/generator.rs Perlin terrain; the
//     hash is world/hash.rs:2-32),
//   * the chunk pipeline of svo/builder.rs:846-986: material fill, column tops
//     (builder.rs:742-805), summed-volume table (builder_prefix.rs:53-134),
//     macro occupancy (builder.rs:809-841), ground min-mip (mips.rs:4-90),
//     bottom-up SVO with stone / uniform collapse (builder_svo.rs:69-534) and
//     ropes (builder_ropes.rs:76-195),
//   * camera packing (app/app.rs:411-511, app/camera.rs:95-111),
//   * the toroidal clipmap update (clipmap.rs:182-577).
// Node order is part of the hit-record contract, so the SVO packing order
// below (parents in linear (y,z,x) scan, children ci = 0..7, levels root-first)
// is kept exactly as the reference emits it.
#include "vxe/vxe.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "../common/terrain_noise.h"

namespace {

constexpr uint32_t kInvalid = 0xFFFFFFFFu;
constexpr int kSide = 64;
constexpr int kSide2 = kSide * kSide;
constexpr int kSide3 = kSide2 * kSide;

// Hashing, value noise and the material rules: terrain_noise.h (shared with
// the device).

struct World {
  vxe_world_params p;

  int32_t ground(int32_t wx, int32_t wz) const { return vxe::terrain::ground(p, wx, wz); }
  uint8_t material(int32_t wx, int32_t wy, int32_t wz, int32_t g) const {
    return vxe::terrain::material(p, wx, wy, wz, g);
  }
};

// Fill material (y*64*64 + z*64 + x) and ground (z*64 + x) for a chunk.
void fill_chunk(const World& w, int32_t cx, int32_t cy, int32_t cz, uint8_t* mat, int32_t* ground) {
  const int32_t ox = cx * kSide, oy = cy * kSide, oz = cz * kSide;
  for (int lz = 0; lz < kSide; ++lz)
    for (int lx = 0; lx < kSide; ++lx) ground[lz * kSide + lx] = w.ground(ox + lx, oz + lz);
  for (int ly = 0; ly < kSide; ++ly)
    for (int lz = 0; lz < kSide; ++lz)
      for (int lx = 0; lx < kSide; ++lx)
        mat[ly * kSide2 + lz * kSide + lx] =
            w.material(ox + lx, oy + ly, oz + lz, ground[lz * kSide + lx]);
}

// ----------------------------------------------------------------------------
// Summed-volume table, 65^3, index z*65*65 + y*65 + x (builder_prefix.rs).
// ----------------------------------------------------------------------------
struct Sat {
  static constexpr int D = kSide + 1;
  std::vector<uint32_t> v;
  explicit Sat(const uint8_t* mat) : v((size_t)D * D * D, 0u) {
    for (int z = 1; z <= kSide; ++z)
      for (int y = 1; y <= kSide; ++y) {
        uint32_t run = 0;
        const uint8_t* row = mat + (size_t)(y - 1) * kSide2 + (size_t)(z - 1) * kSide;
        for (int x = 1; x <= kSide; ++x) {
          run += row[x - 1] != 0 ? 1u : 0u;
          at(x, y, z) = run;
        }
      }
    for (int z = 1; z <= kSide; ++z)
      for (int x = 1; x <= kSide; ++x) {
        uint32_t run = 0;
        for (int y = 1; y <= kSide; ++y) { run += at(x, y, z); at(x, y, z) = run; }
      }
    for (int y = 1; y <= kSide; ++y)
      for (int x = 1; x <= kSide; ++x) {
        uint32_t run = 0;
        for (int z = 1; z <= kSide; ++z) { run += at(x, y, z); at(x, y, z) = run; }
      }
  }
  uint32_t& at(int x, int y, int z) { return v[((size_t)z * D + y) * D + x]; }
  uint32_t get(int x, int y, int z) const { return v[((size_t)z * D + y) * D + x]; }
  uint32_t cube(int x0, int y0, int z0, int s) const {
    const int x1 = x0 + s, y1 = y0 + s, z1 = z0 + s;
    const int64_t r = (int64_t)get(x1, y1, z1) - get(x0, y1, z1) - get(x1, y0, z1) - get(x1, y1, z0) +
                      get(x0, y0, z1) + get(x0, y1, z0) + get(x1, y0, z0) - get(x0, y0, z0);
    return (uint32_t)r;
  }
};

// Min pyramid of the 64x64 ground heights (mips.rs).
struct GroundMin {
  std::vector<std::vector<int32_t>> lv;
  explicit GroundMin(const int32_t* g) {
    lv.emplace_back(g, g + kSide2);
    int side = kSide;
    while (side > 1) {
      const int ns = side / 2;
      std::vector<int32_t> n((size_t)ns * ns);
      const auto& c = lv.back();
      for (int z = 0; z < ns; ++z)
        for (int x = 0; x < ns; ++x) {
          const int i00 = (2 * z) * side + 2 * x;
          n[(size_t)z * ns + x] =
              std::min(std::min(c[i00], c[i00 + 1]), std::min(c[i00 + side], c[i00 + side + 1]));
        }
      lv.push_back(std::move(n));
      side = ns;
    }
  }
  int32_t query_min(int x0, int z0, int size) const {
    int level = 0;
    while ((1 << level) < size) ++level;
    const int side = kSide >> level;
    return lv[level][(size_t)(z0 / size) * side + (x0 / size)];
  }
};

inline uint32_t pack_key(int ox, int oy, int oz, int size) {
  int sh = 0;
  while ((1 << sh) < size) ++sh;
  const uint32_t lvl = 6u - (uint32_t)sh;
  return (((uint32_t)ox >> sh) & 63u) | ((((uint32_t)oy >> sh) & 63u) << 6) |
         ((((uint32_t)oz >> sh) & 63u) << 12) | ((lvl & 7u) << 18);
}
inline vxe_node leaf(int ox, int oy, int oz, int size, uint32_t mat) {
  return vxe_node{kInvalid, 0u, mat, pack_key(ox, oy, oz, size)};
}

// Bottom-up octree (builder_svo.rs:337-534).  Returns root-first flattened nodes.
std::vector<vxe_node> build_svo(const uint8_t* mat, int32_t chunk_oy, const Sat& sat, const GroundMin& gm,
                                int32_t dirt_depth) {
  // Level 6: compact solid voxels in linear (y,z,x) order.
  std::vector<vxe_node> child_nodes;
  std::vector<uint32_t> child_grid(kSide3, kInvalid);
  for (int i = 0; i < kSide3; ++i) {
    if (mat[i] == 0) continue;
    const int x = i & 63, z = (i >> 6) & 63, y = i >> 12;
    child_grid[i] = (uint32_t)child_nodes.size();
    child_nodes.push_back(leaf(x, y, z, 1, mat[i]));
  }
  std::vector<std::vector<vxe_node>> packed(7);
  int child_side = kSide, child_size = 1;
  for (int lvl = 5; lvl >= 0; --lvl) {
    const int psize = child_size * 2, pside = child_side / 2;
    const int pcells = pside * pside * pside;
    int pbits = 0;
    while ((1 << pbits) < pside) ++pbits;
    std::vector<uint8_t> mask(pcells, 0);
    auto child_at = [&](int cx, int cy, int cz) {
      return child_grid[((size_t)cy * child_side + cz) * child_side + cx];
    };
    auto coords = [&](int pi, int* px, int* py, int* pz) {
      *px = pi & (pside - 1);
      *pz = (pi >> pbits) & (pside - 1);
      *py = pi >> (2 * pbits);
    };
    for (int pi = 0; pi < pcells; ++pi) {
      int px, py, pz;
      coords(pi, &px, &py, &pz);
      uint8_t m = 0;
      for (int ci = 0; ci < 8; ++ci)
        if (child_at(px * 2 + (ci & 1), py * 2 + ((ci >> 1) & 1), pz * 2 + ((ci >> 2) & 1)) != kInvalid)
          m |= (uint8_t)(1u << ci);
      mask[pi] = m;
    }
    std::vector<uint32_t> parent_grid(pcells, kInvalid);
    uint32_t pcount = 0;
    for (int pi = 0; pi < pcells; ++pi)
      if (mask[pi]) parent_grid[pi] = pcount++;
    std::vector<vxe_node> parents(pcount, leaf(0, 0, 0, psize, 0));
    std::vector<vxe_node> kids;
    for (int pi = 0; pi < pcells; ++pi) {
      const uint8_t m = mask[pi];
      if (!m) continue;
      int px, py, pz;
      coords(pi, &px, &py, &pz);
      const int ox = px * psize, oy = py * psize, oz = pz * psize;
      vxe_node& out = parents[parent_grid[pi]];
      // Stone collapse: fully solid and entirely below (ground min - dirt).
      const int32_t gmin = gm.query_min(ox, oz, psize);
      const int32_t y1 = chunk_oy + oy + psize - 1;
      if (y1 < gmin - dirt_depth && sat.cube(ox, oy, oz, psize) == (uint32_t)(psize * psize * psize)) {
        out = leaf(ox, oy, oz, psize, VXE_MAT_STONE);
        continue;
      }
      // Uniform collapse: 8 leaf children of one material.
      if (m == 0xFF) {
        const vxe_node& c0 = child_nodes[child_at(px * 2, py * 2, pz * 2)];
        if (c0.child_base == kInvalid) {
          bool ok = true;
          for (int ci = 1; ci < 8 && ok; ++ci) {
            const uint32_t ic = child_at(px * 2 + (ci & 1), py * 2 + ((ci >> 1) & 1), pz * 2 + ((ci >> 2) & 1));
            const vxe_node& c = child_nodes[ic];
            ok = c.child_base == kInvalid && c.material == c0.material;
          }
          if (ok) {
            out = leaf(ox, oy, oz, psize, c0.material);
            continue;
          }
        }
      }
      const uint32_t base = (uint32_t)kids.size();
      uint32_t cm = 0;
      for (int ci = 0; ci < 8; ++ci) {
        if (!(m & (1u << ci))) continue;
        kids.push_back(child_nodes[child_at(px * 2 + (ci & 1), py * 2 + ((ci >> 1) & 1), pz * 2 + ((ci >> 2) & 1))]);
        cm |= 1u << ci;
      }
      out = vxe_node{base, cm, 0u, pack_key(ox, oy, oz, psize)};
    }
    packed[lvl + 1] = std::move(kids);
    child_nodes = std::move(parents);
    child_grid = std::move(parent_grid);
    child_side = pside;
    child_size = psize;
  }
  vxe_node root = child_nodes.empty() ? leaf(0, 0, 0, kSide, VXE_MAT_AIR) : child_nodes[0];
  uint32_t bases[7] = {0, 0, 0, 0, 0, 0, 0};
  uint32_t cur = 1;
  for (int l = 1; l <= 6; ++l) { bases[l] = cur; cur += (uint32_t)packed[l].size(); }
  if (root.child_base != kInvalid) root.child_base += bases[1];
  for (int l = 1; l < 6; ++l)
    for (auto& n : packed[l])
      if (n.child_base != kInvalid) n.child_base += bases[l + 1];
  std::vector<vxe_node> out;
  out.reserve(cur);
  out.push_back(root);
  for (int l = 1; l <= 6; ++l) out.insert(out.end(), packed[l].begin(), packed[l].end());
  return out;
}

// Ropes (builder_ropes.rs:76-195): neighbour of each child across each face,
// a sibling when present, else the parent's rope target descended one level.
void build_ropes(const std::vector<vxe_node>& nodes, std::vector<vxe_node_ropes>& ropes) {
  ropes.assign(nodes.size(), vxe_node_ropes{kInvalid, kInvalid, kInvalid, kInvalid, kInvalid, kInvalid, 0u, 0u});
  auto child_of = [&](uint32_t p, uint32_t ci) -> uint32_t {
    const vxe_node& n = nodes[p];
    if (!(n.child_mask & (1u << ci))) return kInvalid;
    return n.child_base + (uint32_t)__builtin_popcount(n.child_mask & ((1u << ci) - 1u));
  };
  auto down = [&](uint32_t nei, uint32_t hx, uint32_t hy, uint32_t hz) -> uint32_t {
    if (nei == kInvalid) return kInvalid;
    if (nodes[nei].child_base == kInvalid) return nei;
    return child_of(nei, hx | (hy << 1) | (hz << 2));
  };
  // Iterative DFS in the same visiting order as the recursive reference.
  std::vector<uint32_t> stack;
  stack.push_back(0);
  while (!stack.empty()) {
    const uint32_t idx = stack.back();
    stack.pop_back();
    const vxe_node p = nodes[idx];
    if (p.child_base == kInvalid) continue;
    const vxe_node_ropes pr = ropes[idx];
    uint32_t kid[8];
    for (uint32_t ci = 0; ci < 8; ++ci) kid[ci] = child_of(idx, ci);
    for (uint32_t ci = 0; ci < 8; ++ci) {
      if (kid[ci] == kInvalid) continue;
      const uint32_t hx = ci & 1u, hy = (ci >> 1) & 1u, hz = (ci >> 2) & 1u;
      vxe_node_ropes r{};
      const uint32_t sx = kid[ci ^ 1u], sy = kid[ci ^ 2u], sz = kid[ci ^ 4u];
      r.px = (hx == 0 && sx != kInvalid) ? sx : down(pr.px, 0, hy, hz);
      r.nx = (hx == 1 && sx != kInvalid) ? sx : down(pr.nx, 1, hy, hz);
      r.py = (hy == 0 && sy != kInvalid) ? sy : down(pr.py, hx, 0, hz);
      r.ny = (hy == 1 && sy != kInvalid) ? sy : down(pr.ny, hx, 1, hz);
      r.pz = (hz == 0 && sz != kInvalid) ? sz : down(pr.pz, hx, hy, 0);
      r.nz = (hz == 1 && sz != kInvalid) ? sz : down(pr.nz, hx, hy, 1);
      ropes[kid[ci]] = r;
    }
    // Children only read their parent's ropes, so any visiting order that
    // handles a parent before its children gives the same result.
    for (int ci = 7; ci >= 0; --ci)
      if (kid[ci] != kInvalid) stack.push_back(kid[ci]);
  }
}

vxe_status build_all(const uint8_t* mat, int32_t chunk_oy, const int32_t* ground, int32_t dirt_depth,
                     vxe_built_chunk* out) {
  std::memset(out, 0, sizeof(*out));
  // Column tops (builder.rs:775-805) and colinfo packing (builder.rs:742-771).
  uint8_t top_y[kSide2], top_m[kSide2];
  std::memset(top_y, 255, sizeof(top_y));
  std::memset(top_m, 0, sizeof(top_m));
  uint32_t solid = 0;
  for (int ly = 0; ly < kSide; ++ly)
    for (int col = 0; col < kSide2; ++col) {
      const uint8_t m = mat[(size_t)ly * kSide2 + col];
      if (m) { top_y[col] = (uint8_t)ly; top_m[col] = m; ++solid; }
    }
  for (int idx = 0; idx < kSide2; ++idx) {
    const uint32_t e = (uint32_t)top_y[idx] | ((uint32_t)top_m[idx] << 8);
    uint32_t& w = out->colinfo_words[idx >> 1];
    w = (idx & 1) ? ((w & 0x0000FFFFu) | (e << 16)) : ((w & 0xFFFF0000u) | e);
  }
  out->solid_voxels = solid;
  const Sat sat(mat);
  // Macro bits: 8^3 cells of 8^3 voxels, bit = mx + 8*(my + 8*mz).
  for (int mz = 0; mz < 8; ++mz)
    for (int my = 0; my < 8; ++my)
      for (int mx = 0; mx < 8; ++mx)
        if (sat.cube(mx * 8, my * 8, mz * 8, 8) > 0) {
          const uint32_t bit = (uint32_t)(mx + 8 * (my + 8 * mz));
          out->macro_words[bit >> 5] |= 1u << (bit & 31u);
        }
  const GroundMin gm(ground);
  std::vector<vxe_node> nodes = build_svo(mat, chunk_oy, sat, gm, dirt_depth);
  std::vector<vxe_node_ropes> ropes;
  build_ropes(nodes, ropes);
  out->node_count = (uint32_t)nodes.size();
  out->nodes = (vxe_node*)std::malloc(sizeof(vxe_node) * nodes.size());
  out->ropes = (vxe_node_ropes*)std::malloc(sizeof(vxe_node_ropes) * ropes.size());
  if (!out->nodes || !out->ropes) {
    std::free(out->nodes);
    std::free(out->ropes);
    out->nodes = nullptr;
    out->ropes = nullptr;
    return VXE_ERR_OOM;
  }
  std::memcpy(out->nodes, nodes.data(), sizeof(vxe_node) * nodes.size());
  std::memcpy(out->ropes, ropes.data(), sizeof(vxe_node_ropes) * ropes.size());
  return VXE_OK;
}

// ----------------------------------------------------------------------------
// Camera (double precision, rounded to f32 at the end)
// ----------------------------------------------------------------------------
struct M4 { double m[4][4]; };  // m[col][row]

M4 mul(const M4& a, const M4& b) {
  M4 r{};
  for (int c = 0; c < 4; ++c)
    for (int rr = 0; rr < 4; ++rr) {
      double s = 0;
      for (int k = 0; k < 4; ++k) s += a.m[k][rr] * b.m[c][k];
      r.m[c][rr] = s;
    }
  return r;
}

bool inverse(const M4& a, M4* out) {
  double m[4][8];
  for (int r = 0; r < 4; ++r) {
    for (int c = 0; c < 4; ++c) m[r][c] = a.m[c][r];
    for (int c = 0; c < 4; ++c) m[r][4 + c] = r == c ? 1.0 : 0.0;
  }
  for (int c = 0; c < 4; ++c) {
    int piv = c;
    for (int r = c + 1; r < 4; ++r)
      if (std::fabs(m[r][c]) > std::fabs(m[piv][c])) piv = r;
    if (std::fabs(m[piv][c]) < 1e-300) return false;
    if (piv != c)
      for (int k = 0; k < 8; ++k) std::swap(m[c][k], m[piv][k]);
    const double inv = 1.0 / m[c][c];
    for (int k = 0; k < 8; ++k) m[c][k] *= inv;
    for (int r = 0; r < 4; ++r) {
      if (r == c) continue;
      const double f = m[r][c];
      for (int k = 0; k < 8; ++k) m[r][k] -= f * m[c][k];
    }
  }
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) out->m[c][r] = m[r][4 + c];
  return true;
}

void mulv(const M4& a, const double v[4], double o[4]) {
  for (int r = 0; r < 4; ++r) o[r] = a.m[0][r] * v[0] + a.m[1][r] * v[1] + a.m[2][r] * v[2] + a.m[3][r] * v[3];
}

double halton(uint32_t index, uint32_t base) {
  double f = 1.0, r = 0.0;
  while (index > 0) {
    f /= (double)base;
    r += f * (double)(index % base);
    index /= base;
  }
  return r;
}

void store(float dst[4][4], const M4& m) {
  for (int c = 0; c < 4; ++c)
    for (int r = 0; r < 4; ++r) dst[c][r] = (float)m.m[c][r];
}

// ----------------------------------------------------------------------------
// Clipmap (clipmap.rs:182-577)
// ----------------------------------------------------------------------------
}  // namespace

struct vxe_clipmap_state {
  World world;
  uint32_t levels, res;
  float base_cell;
  int32_t last_ox[VXE_CLIP_LEVELS_MAX], last_oz[VXE_CLIP_LEVELS_MAX];
  bool valid[VXE_CLIP_LEVELS_MAX];
  uint32_t off_x[VXE_CLIP_LEVELS_MAX], off_z[VXE_CLIP_LEVELS_MAX];
  std::vector<std::vector<float>> data;
  std::vector<vxe_clip_patch> patches;
  std::vector<vxe_clip_patch_geom> geoms;
  bool with_data = true;  // false: record the geometry only (vxe_clipmap_plan)

  float sample(float wx_m, float wz_m) const {
    const float vs = 0.1f;
    const int32_t wx = (int32_t)std::floor(wx_m / vs), wz = (int32_t)std::floor(wz_m / vs);
    return (float)world.ground(wx, wz) * vs;
  }
  // Patch of logical texels [lx0, lx0+w) x [lz0, lz0+h) placed at storage (sx, sz).
  void emit(uint32_t lvl, float ox_m, float oz_m, float cell, uint32_t lx0, uint32_t lz0, uint32_t w,
            uint32_t h, uint32_t sx, uint32_t sz) {
    geoms.push_back(vxe_clip_patch_geom{lvl, sx, sz, w, h, lx0, lz0, ox_m, oz_m, cell});
    if (!with_data) {
      data.emplace_back();
      patches.push_back(vxe_clip_patch{lvl, sx, sz, w, h, nullptr});
      return;
    }
    std::vector<float> d((size_t)w * h);
    for (uint32_t z = 0; z < h; ++z) {
      const float wz = oz_m + ((float)(lz0 + z) + 0.5f) * cell;
      for (uint32_t x = 0; x < w; ++x) {
        const float wx = ox_m + ((float)(lx0 + x) + 0.5f) * cell;
        d[(size_t)z * w + x] = sample(wx, wz);
      }
    }
    data.push_back(std::move(d));
    patches.push_back(vxe_clip_patch{lvl, sx, sz, w, h, nullptr});
  }
};

extern "C" {

int32_t vxe_ground_height(const vxe_world_params* wp, int32_t wx, int32_t wz) {
  if (!wp) return 0;
  World w{*wp};
  return w.ground(wx, wz);
}

vxe_status vxe_chunk_materials(const vxe_world_params* wp, int32_t cx, int32_t cy, int32_t cz, uint8_t* out) {
  if (!wp || !out) return VXE_ERR_INVALID_ARG;
  World w{*wp};
  std::vector<int32_t> g(kSide2);
  fill_chunk(w, cx, cy, cz, out, g.data());
  return VXE_OK;
}

vxe_status vxe_build_from_materials(const uint8_t* mat, int32_t chunk_oy, const int32_t* ground,
                                    int32_t dirt_depth, vxe_built_chunk* out) {
  if (!mat || !ground || !out) return VXE_ERR_INVALID_ARG;
  try {
    return build_all(mat, chunk_oy, ground, dirt_depth, out);
  } catch (const std::bad_alloc&) {
    return VXE_ERR_OOM;
  }
}

vxe_status vxe_build_chunk(const vxe_world_params* wp, int32_t cx, int32_t cy, int32_t cz, vxe_built_chunk* out) {
  if (!wp || !out) return VXE_ERR_INVALID_ARG;
  try {
    World w{*wp};
    std::vector<uint8_t> mat(kSide3);
    std::vector<int32_t> g(kSide2);
    fill_chunk(w, cx, cy, cz, mat.data(), g.data());
    return build_all(mat.data(), cy * kSide, g.data(), wp->dirt_depth, out);
  } catch (const std::bad_alloc&) {
    return VXE_ERR_OOM;
  }
}

void vxe_free_chunk(vxe_built_chunk* c) {
  if (!c) return;
  std::free(c->nodes);
  std::free(c->ropes);
  c->nodes = nullptr;
  c->ropes = nullptr;
  c->node_count = 0;
}

vxe_status vxe_build_camera(const vxe_camera_params* p, vxe_camera_gpu* out) {
  if (!p || !out || p->present_h == 0 || p->internal_w == 0 || p->internal_h == 0) return VXE_ERR_INVALID_ARG;
  std::memset(out, 0, sizeof(*out));
  const double yaw = p->yaw, pitch = p->pitch;
  double f[3] = {std::sin(yaw) * std::cos(pitch), std::sin(pitch), std::cos(yaw) * std::cos(pitch)};
  double fl = std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
  for (double& v : f) v /= fl;
  const double eye[3] = {p->pos[0], p->pos[1], p->pos[2]};
  // look_to_rh: s = normalize(cross(f, up)), u = cross(s, f).
  double s[3] = {f[1] * 0.0 - f[2] * 1.0, f[2] * 0.0 - f[0] * 0.0, f[0] * 1.0 - f[1] * 0.0};
  const double sl = std::sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
  for (double& v : s) v /= sl;
  const double u[3] = {s[1] * f[2] - s[2] * f[1], s[2] * f[0] - s[0] * f[2], s[0] * f[1] - s[1] * f[0]};
  M4 view{};
  for (int i = 0; i < 3; ++i) {
    view.m[i][0] = s[i];
    view.m[i][1] = u[i];
    view.m[i][2] = -f[i];
    view.m[i][3] = 0.0;
  }
  view.m[3][0] = -(eye[0] * s[0] + eye[1] * s[1] + eye[2] * s[2]);
  view.m[3][1] = -(eye[0] * u[0] + eye[1] * u[1] + eye[2] * u[2]);
  view.m[3][2] = (eye[0] * f[0] + eye[1] * f[1] + eye[2] * f[2]);
  view.m[3][3] = 1.0;
  const double aspect = (double)p->present_w / (double)p->present_h;
  const double h = 1.0 / std::tan(0.5 * (double)p->fovy_rad);
  const double w = h / aspect;
  const double r = (double)p->z_far / ((double)p->z_near - (double)p->z_far);
  M4 proj{};
  proj.m[0][0] = w;
  proj.m[1][1] = h;
  proj.m[2][2] = r;
  proj.m[2][3] = -1.0;
  proj.m[3][2] = r * (double)p->z_near;
  M4 view_inv, proj_inv;
  if (!inverse(view, &view_inv) || !inverse(proj, &proj_inv)) return VXE_ERR_INVALID_ARG;
  const M4 view_proj = mul(proj, view);
  store(out->view_inv, view_inv);
  store(out->proj_inv, proj_inv);
  store(out->view_proj, view_proj);
  if (p->has_prev) std::memcpy(out->prev_view_proj, p->prev_view_proj, sizeof(out->prev_view_proj));
  else store(out->prev_view_proj, view_proj);
  double jx = 0.0, jy = 0.0;
  if (p->jitter) {
    jx = halton(p->frame_index + 1u, 2) - 0.5;
    jy = halton(p->frame_index + 1u, 3) - 0.5;
  }
  const double rw = (double)p->internal_w, rh = (double)p->internal_h;
  auto ray_at = [&](double px, double py, double o[3]) {
    const double ndc[4] = {2.0 * px / rw - 1.0, 1.0 - 2.0 * py / rh, 1.0, 1.0};
    double vp[4];
    mulv(proj_inv, ndc, vp);
    const double vd[4] = {vp[0] / vp[3], vp[1] / vp[3], vp[2] / vp[3], 0.0};
    double wd[4];
    mulv(view_inv, vd, wd);
    o[0] = wd[0];
    o[1] = wd[1];
    o[2] = wd[2];
  };
  double r00[3], r10[3], r01[3];
  ray_at(0.5 + jx, 0.5 + jy, r00);
  ray_at(1.5 + jx, 0.5 + jy, r10);
  ray_at(0.5 + jx, 1.5 + jy, r01);
  for (int i = 0; i < 3; ++i) {
    out->cam_pos[i] = p->pos[i];
    out->ray00[i] = (float)r00[i];
    out->ray_dx[i] = (float)(r10[i] - r00[i]);
    out->ray_dy[i] = (float)(r01[i] - r00[i]);
  }
  out->cam_pos[3] = 1.0f;
  out->chunk_size = VXE_CHUNK_SIZE;
  out->chunk_count = p->chunk_count;
  out->max_steps = 128u;
  out->frame_index = p->frame_index;
  out->voxel_params[0] = 0.1f;
  out->voxel_params[1] = p->time_s;
  out->voxel_params[2] = 2.0f;
  out->voxel_params[3] = 0.002f;
  for (int i = 0; i < 3; ++i) {
    out->grid_origin_chunk[i] = p->grid_origin_chunk[i];
    out->grid_dims[i] = p->grid_dims[i];
  }
  out->render_present_px[0] = p->internal_w;
  out->render_present_px[1] = p->internal_h;
  out->render_present_px[2] = p->present_w;
  out->render_present_px[3] = p->present_h;
  return VXE_OK;
}

vxe_clipmap_state* vxe_clipmap_new(const vxe_world_params* wp, uint32_t levels, uint32_t res, float base_cell_m) {
  if (!wp || levels == 0 || levels > VXE_CLIP_LEVELS_MAX || res == 0 || res > 65535u) return nullptr;
  auto* s = new (std::nothrow) vxe_clipmap_state();
  if (!s) return nullptr;
  s->world = World{*wp};
  s->levels = levels;
  s->res = res;
  s->base_cell = base_cell_m;
  for (uint32_t i = 0; i < VXE_CLIP_LEVELS_MAX; ++i) {
    s->valid[i] = false;
    s->last_ox[i] = s->last_oz[i] = 0;
    s->off_x[i] = s->off_z[i] = 0;
  }
  return s;
}

void vxe_clipmap_free(vxe_clipmap_state* s) { delete s; }

vxe_status vxe_clipmap_update(vxe_clipmap_state* s, float cam_x, float cam_z, vxe_clipmap_gpu* params,
                              const vxe_clip_patch** patches, uint32_t* n_patches) {
  if (!s || !params || !patches || !n_patches) return VXE_ERR_INVALID_ARG;
  s->data.clear();
  s->patches.clear();
  s->geoms.clear();
  std::memset(params, 0, sizeof(*params));
  params->levels = s->levels;
  params->res = s->res;
  params->base_cell_m = s->base_cell;
  const int32_t res_i = (int32_t)s->res;
  const int32_t guard = 16;
  // Pass 1: decide whether this frame updates (any first / forced / moved).
  bool any = false;
  for (uint32_t i = 0; i < s->levels; ++i) {
    const float cell = s->base_cell * (float)(1u << i);
    const float half = (float)s->res * 0.5f;
    const int32_t nox = (int32_t)std::floor((cam_x - half * cell) / cell);
    const int32_t noz = (int32_t)std::floor((cam_z - half * cell) / cell);
    if (!s->valid[i] || nox != s->last_ox[i] || noz != s->last_oz[i]) any = true;
    if (s->valid[i]) {
      const int32_t lx = (int32_t)std::floor((cam_x - (float)s->last_ox[i] * cell) / cell);
      const int32_t lz = (int32_t)std::floor((cam_z - (float)s->last_oz[i] * cell) / cell);
      if (lx < guard || lz < guard || lx >= res_i - guard || lz >= res_i - guard) any = true;
    }
  }
  for (uint32_t i = 0; i < s->levels; ++i) {
    const float cell = s->base_cell * (float)(1u << i);
    const float half = (float)s->res * 0.5f;
    const int32_t nox = (int32_t)std::floor((cam_x - half * cell) / cell);
    const int32_t noz = (int32_t)std::floor((cam_z - half * cell) / cell);
    const float ox_m = (float)nox * cell, oz_m = (float)noz * cell;
    const bool first = !s->valid[i];
    const int32_t dx = first ? 0 : nox - s->last_ox[i];
    const int32_t dz = first ? 0 : noz - s->last_oz[i];
    const bool moved = first || dx != 0 || dz != 0;
    if (any && moved) {
      const uint32_t adx = (uint32_t)std::abs(dx), adz = (uint32_t)std::abs(dz);
      if (first || adx >= s->res || adz >= s->res) {
        s->valid[i] = true;
        s->last_ox[i] = nox;
        s->last_oz[i] = noz;
        s->off_x[i] = s->off_z[i] = 0;
        s->emit(i, ox_m, oz_m, cell, 0, 0, s->res, s->res, 0, 0);
      } else {
        s->off_x[i] = (uint32_t)((((int32_t)s->off_x[i] + dx) % res_i + res_i) % res_i);
        s->off_z[i] = (uint32_t)((((int32_t)s->off_z[i] + dz) % res_i + res_i) % res_i);
        s->last_ox[i] = nox;
        s->last_oz[i] = noz;
        const uint32_t res = s->res;
        if (dx != 0) {
          const uint32_t cols = adx;
          const uint32_t lx0 = dx > 0 ? res - cols : 0u;
          const uint32_t sx0 = (lx0 + s->off_x[i]) % res;
          if (sx0 + cols <= res) {
            s->emit(i, ox_m, oz_m, cell, lx0, 0, cols, res, sx0, 0);
          } else {
            const uint32_t a = res - sx0, b = sx0 + cols - res;
            s->emit(i, ox_m, oz_m, cell, lx0, 0, a, res, sx0, 0);
            s->emit(i, ox_m, oz_m, cell, lx0 + a, 0, b, res, 0, 0);
          }
        }
        if (dz != 0) {
          const uint32_t rows = adz;
          const uint32_t lz0 = dz > 0 ? res - rows : 0u;
          const uint32_t sz0 = (lz0 + s->off_z[i]) % res;
          if (sz0 + rows <= res) {
            s->emit(i, ox_m, oz_m, cell, 0, lz0, res, rows, 0, sz0);
          } else {
            const uint32_t a = res - sz0, b = sz0 + rows - res;
            s->emit(i, ox_m, oz_m, cell, 0, lz0, res, a, 0, sz0);
            s->emit(i, ox_m, oz_m, cell, 0, lz0 + a, res, b, 0, 0);
          }
        }
      }
    }
    const float cox = s->valid[i] ? (float)s->last_ox[i] * cell : ox_m;
    const float coz = s->valid[i] ? (float)s->last_oz[i] * cell : oz_m;
    params->level[i][0] = cox;
    params->level[i][1] = coz;
    params->level[i][2] = cell;
    params->level[i][3] = 0.0f;
    params->offset[i][0] = s->off_x[i];
    params->offset[i][1] = s->off_z[i];
  }
  // Levels beyond `levels` keep cell 1.0 like the reference's default fill.
  for (uint32_t i = s->levels; i < VXE_CLIP_LEVELS_MAX; ++i) params->level[i][2] = 1.0f;
  for (size_t k = 0; k < s->patches.size(); ++k) s->patches[k].data = s->with_data ? s->data[k].data() : nullptr;
  *patches = s->patches.empty() ? nullptr : s->patches.data();
  *n_patches = (uint32_t)s->patches.size();
  return VXE_OK;
}

vxe_status vxe_clipmap_plan(vxe_clipmap_state* s, float cam_x, float cam_z, vxe_clipmap_gpu* params,
                            const vxe_clip_patch_geom** geoms, uint32_t* n_geoms, vxe_world_params* world) {
  if (!s || !params || !geoms || !n_geoms || !world) return VXE_ERR_INVALID_ARG;
  const vxe_clip_patch* patches = nullptr;
  uint32_t n = 0;
  s->with_data = false;
  const vxe_status st = vxe_clipmap_update(s, cam_x, cam_z, params, &patches, &n);
  s->with_data = true;
  if (st != VXE_OK) return st;
  *geoms = s->geoms.empty() ? nullptr : s->geoms.data();
  *n_geoms = (uint32_t)s->geoms.size();
  *world = s->world.p;
  return VXE_OK;
}

}  // extern "C"
