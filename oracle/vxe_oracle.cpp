// vxe_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Scalar CPU restatement of voxel-engine-v0's compute frame (WGSL), used as
// the parity checker for the CUDA passes and as the timed CPU baseline.
// Nothing in the product links or calls this file; only tests/,
// __graft_entry__.smoke() and bench.py (cpu_baseline / --impl reference) load
// the library built from it.
//
// Structure follows the reference shaders function by function; each block
// cites the WGSL it restates (paths relative to the reference project root,
// under src/shaders/).  WGSL builtins are spelled out explicitly:
//   mix(a,b,t) = a*(1-t) + b*t, smoothstep per the WGSL spec, clamp = min(max),
//   normalize(v) = v * (1/sqrt(dot(v,v))), inverseSqrt(x) = 1/sqrt(x),
//   f32->i32/u32 conversions saturate (NaN -> 0), nearest+clamp sampling
//   (render/state/mod.rs:216-225) = clamp(floor(uv*size), 0, size-1),
//   exp/pow/sin/cos from include/vxe/detmath.h.
// Compile with -ffp-contract=off (no FMA contraction) so every float op is a
// single IEEE binary32 operation, exactly as the device code evaluates it.
//
// Parity status: the reference is Rust + WGSL and cannot run here as it is
// (no Rust toolchain, no graphics stack).  Its shaders are translated to C++
// instead (oracle/wgsl_to_cpp.py) and run beside this restatement: whole
// frames of the five compute passes, every image, and the traces and helpers
// function by function (oracle_shading_eval, ora_scene_eval, ora_trace_chunk
// and ora_primary_tile below; tests/test_oracle_wgsl_pin.py), bit for bit.
// The scene traversal is also checked against an independent FP64 voxel DDA
// (tests/test_oracle_kat.py).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../include/vxe/detmath.h"
#include "../include/vxe/vxe.h"

namespace {

// ---------------------------------------------------------------------------
// Constants (common.wgsl:16-332, app/config.rs)
// ---------------------------------------------------------------------------
constexpr uint32_t INVALID = 0xFFFFFFFFu;
constexpr uint32_t LEAF = 0xFFFFFFFFu;
constexpr float BIG = 1e30f;
constexpr float EPS_INV = 1e-8f;
constexpr uint32_t MAT_AIR = 0, MAT_GRASS = 1, MAT_DIRT = 2, MAT_STONE = 3, MAT_WOOD = 4, MAT_LEAF = 5,
                   MAT_LIGHT = 6;
constexpr float SUN_DIR_X = 0.61237244f, SUN_DIR_Y = 0.5f, SUN_DIR_Z = 0.61237244f;
constexpr float SUN_INTENSITY = 5.0f;
constexpr float SHADOW_BIAS = 2e-4f;
constexpr uint32_t VSM_STEPS = 16;
constexpr float LEAF_LIGHT_TRANSMIT = 0.50f, GRASS_LIGHT_TRANSMIT = 0.70f, MIN_TRANS = 0.03f;
constexpr float GODRAY_ENERGY_BOOST = 8.0f, GODRAY_KNEE_INTEGRATE = 0.35f, GODRAY_COMPOSITE_SCALE = 6.5f;
constexpr float GODRAY_FADE_NEAR = 40.0f, GODRAY_FADE_FAR = 80.0f, GODRAY_KNEE_COMPOSITE = 0.25f;
constexpr float FOG_HEIGHT_FALLOFF = 0.18f, FOG_MAX_DIST = 120.0f, FOG_PRIMARY_SCALE = 0.02f,
                FOG_GODRAY_SCALE = 1.0f, FOG_COLOR_SKY_BLEND = 0.10f;
constexpr float GODRAY_MAX_DIST = 100.0f, GODRAY_SCATTER_HEIGHT_FALLOFF = 0.04f, GODRAY_SCATTER_MIN_FRAC = 0.35f;
constexpr float GODRAY_BLACK_LEVEL = 0.004f, GODRAY_EDGE0 = 0.004f, GODRAY_EDGE1 = 0.035f;
constexpr float GODRAY_BASE_HAZE = 0.02f, GODRAY_HAZE_NEAR_FADE = 18.0f, GODRAY_TV_CUTOFF = 0.02f;
constexpr uint32_t GODRAY_STEPS_FAST = 24, GODRAY_MIN_STEPS = 8, GODRAY_STEP_Q = 4;
constexpr float GODRAY_STEPS_PER_METER = 1.25f, GODRAY_EDGE_ENERGY_BOOST = 2.5f;
constexpr float INV_4PI = 0.0795774715f, PHASE_G = 0.15f, PHASE_MIE_W = 0.20f;
constexpr float CLOUD_BASE_H = 170.0f, CLOUD_TOP_H = 250.0f, CLOUD_UV_SCALE = 0.0016f;
constexpr float CLOUD_WIND_X = 0.020f, CLOUD_WIND_Y = 0.012f, CLOUD_COVERAGE = 0.40f, CLOUD_SOFTNESS = 0.08f;
constexpr float CLOUD_DENSITY = 0.058f, CLOUD_PUFF_POW = 1.8f, CLOUD_DETAIL_W = 0.35f;
constexpr uint32_t CLOUD_STEPS_VIEW = 8, CLOUD_STEPS_LIGHT = 4;
constexpr float CLOUD_HORIZON_Y0 = 0.02f, CLOUD_HORIZON_Y1 = 0.25f, CLOUD_SILVER_POW = 8.0f, CLOUD_SILVER_STR = 0.6f;
constexpr float CLOUD_SHADOW_ABSORB = 6.0f, CLOUD_SHADOW_STRENGTH = 0.45f, CLOUD_SUN_DISC_DIM_POW = 8.0f,
                CLOUD_SUN_DISC_DIM_FLOOR = 0.0f, CLOUD_GODRAY_W = 0.50f, SKY_EXPOSURE = 0.40f;
constexpr float WIND_CELL_FREQ = 2.5f, WIND_RAMP_Y0 = 2.0f, WIND_RAMP_Y1 = 14.0f;
constexpr float WIND_GUST_TIME_FREQ = 0.9f, WIND_FLUTTER_TIME_FREQ = 4.2f, WIND_GUST_WEIGHT = 0.75f,
                WIND_FLUTTER_WEIGHT = 0.25f, WIND_VERTICAL_SCALE = 0.25f, LEAF_VERTICAL_REDUCE = 0.15f;
constexpr float LEAF_OFFSET_AMP = 0.75f, LEAF_OFFSET_MAX_FRAC = 0.75f, LEAF_LOD_DISP_START = 25.0f,
                LEAF_LOD_DISP_END = 70.0f, TAU = 6.28318530718f;
constexpr float PRIMARY_NUDGE_VOXEL_FRAC = 1e-3f, PRIMARY_HIT_MARGIN = 0.08f, PRIMARY_HIT_WINDOW = 0.60f,
                PRIMARY_HIT_DEPTH_REL0 = 0.04f, PRIMARY_HIT_DEPTH_REL1 = 0.12f;
constexpr float SHADOW_TAA_ALPHA = 0.20f;
constexpr uint32_t SHADOW_SUBSAMPLE_MASK = 7;
constexpr float PRIMARY_HIT_MOTION_PX0 = 0.50f, PRIMARY_HIT_MOTION_PX1 = 1.75f;
constexpr float J0_SCALE = 1.31f, COMPOSITE_SHARPEN = 0.1f, POST_EXPOSURE = 0.15f;
constexpr uint32_t CLIP_LEVELS_MAX = 16, HF_MAX_STEPS = 48, HF_BISECT = 3;
constexpr float HF_DT_MAX = 48.0f;
constexpr uint32_t LIGHT_MAX_DIST_VOX = 16, LIGHT_RAYS = 8, LIGHT_EARLY_HITS = 4;
constexpr float LIGHT_SOFT_RADIUS_VOX = 3.0f, LIGHT_NEAR_CLAMP_VOX = 1.25f, LIGHT_RANGE_VOX = 80.0f,
                LIGHT_WRAP = 0.15f, LIGHT_DIRECT_GAIN = 1.00f, LIGHT_INDIRECT_GAIN = 0.65f;
constexpr float VOXEL_AO_MAX_DIST = 40.0f, LOCAL_LIGHT_MAX_DIST = 50.0f, FAR_SHADING_DIST = 64.0f;
constexpr float LOCAL_TAA_ALPHA = 0.80f, COMPOSITE_TAA_ALPHA = 0.45f;
constexpr float GRASS_LAYER_HEIGHT_VOX = 1.55f, GRASS_HIT_EPS_VOX = 0.008f, GRASS_STEP_MIN_VOX = 0.02f;
constexpr float GRASS_VOXEL_SEGS = 6.0f, GRASS_VOXEL_THICKNESS_VOX = 0.15f, GRASS_VOXEL_TAPER = 0.25f,
                GRASS_OVERHANG_VOX = 0.6f, GRASS_LOD_MID_START = 18.0f, GRASS_LOD_FAR_START = 45.0f;
constexpr uint32_t GRASS_BLADE_COUNT = 3, GRASS_TRACE_STEPS = 7, GRASS_BLADE_COUNT_MID = 2,
                   GRASS_BLADE_COUNT_FAR = 1, GRASS_SEGS_MID = 4, GRASS_SEGS_FAR = 2, GRASS_TRACE_STEPS_MID = 5,
                   GRASS_TRACE_STEPS_FAR = 3;
constexpr float ALBEDO_VAR_GAIN = 3.5f;
constexpr uint32_t MACRO_DIM = 8, MAX_TILE_CHUNKS = 192, PRIMARY_MAX_TILE_CHUNKS = 24, TILE_SIZE = 8;

// ---------------------------------------------------------------------------
// Scalar helpers with WGSL semantics
// ---------------------------------------------------------------------------
inline float fmin_(float a, float b) {
  if (a != a) return b;
  if (b != b) return a;
  if (a < b) return a;
  if (b < a) return b;
  return std::signbit(a) ? a : b;
}
inline float fmax_(float a, float b) {
  if (a != a) return b;
  if (b != b) return a;
  if (a > b) return a;
  if (b > a) return b;
  return std::signbit(a) ? b : a;
}
inline float clampf(float x, float lo, float hi) { return fmin_(fmax_(x, lo), hi); }
inline float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
inline float smooth(float e0, float e1, float x) {
  const float t = clampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}
inline float fract(float x) { return x - std::floor(x); }
inline float signf(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }
inline int32_t to_i32(float f) {
  if (f != f) return 0;
  if (f >= 2147483648.0f) return INT32_MAX;
  if (f <= -2147483648.0f) return INT32_MIN;
  return (int32_t)f;
}
inline uint32_t to_u32(float f) {
  if (f != f || f <= 0.0f) return 0u;
  if (f >= 4294967296.0f) return 0xFFFFFFFFu;
  return (uint32_t)f;
}
inline int32_t clampi(int32_t x, int32_t lo, int32_t hi) { return std::min(std::max(x, lo), hi); }
inline uint32_t clampu(uint32_t x, uint32_t lo, uint32_t hi) { return std::min(std::max(x, lo), hi); }
inline float sinf_(float x) { return vxe_sinf(x); }
inline float cosf_(float x) { return vxe_cosf(x); }
inline float expf_(float x) { return vxe_expf(x); }
inline float powf_(float x, float y) { return vxe_powf(x, y); }
inline float bits_f(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }
inline uint32_t f_bits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }

struct v2 { float x, y; };
struct v3 { float x, y, z; };
struct v4 { float x, y, z, w; };
struct i3 { int32_t x, y, z; };

inline v2 V2(float x, float y) { return v2{x, y}; }
inline v3 V3(float x, float y, float z) { return v3{x, y, z}; }
inline v3 V3s(float s) { return v3{s, s, s}; }
inline v2 operator+(v2 a, v2 b) { return {a.x + b.x, a.y + b.y}; }
inline v2 operator-(v2 a, v2 b) { return {a.x - b.x, a.y - b.y}; }
inline v2 operator*(v2 a, v2 b) { return {a.x * b.x, a.y * b.y}; }
inline v2 operator*(v2 a, float s) { return {a.x * s, a.y * s}; }
inline v2 operator*(float s, v2 a) { return {s * a.x, s * a.y}; }
inline v2 operator/(v2 a, v2 b) { return {a.x / b.x, a.y / b.y}; }
inline v3 operator+(v3 a, v3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline v3 operator-(v3 a, v3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline v3 operator-(v3 a) { return {-a.x, -a.y, -a.z}; }
inline v3 operator*(v3 a, v3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline v3 operator*(v3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline v3 operator*(float s, v3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline v3 operator/(v3 a, v3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
inline v3 operator/(v3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline float dot(v2 a, v2 b) { return a.x * b.x + a.y * b.y; }
inline float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float length(v2 a) { return std::sqrt(dot(a, a)); }
inline float length(v3 a) { return std::sqrt(dot(a, a)); }
inline v2 normalize(v2 a) { const float inv = 1.0f / std::sqrt(dot(a, a)); return a * inv; }
inline v3 normalize(v3 a) { const float inv = 1.0f / std::sqrt(dot(a, a)); return a * inv; }
inline v3 cross(v3 a, v3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline v3 vmin(v3 a, v3 b) { return {fmin_(a.x, b.x), fmin_(a.y, b.y), fmin_(a.z, b.z)}; }
inline v3 vmax(v3 a, v3 b) { return {fmax_(a.x, b.x), fmax_(a.y, b.y), fmax_(a.z, b.z)}; }
inline v3 vabs(v3 a) { return {std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }
inline v3 vfloor(v3 a) { return {std::floor(a.x), std::floor(a.y), std::floor(a.z)}; }
inline v2 vfloor(v2 a) { return {std::floor(a.x), std::floor(a.y)}; }
inline v2 vfract(v2 a) { return {fract(a.x), fract(a.y)}; }
inline v3 vclamp(v3 x, v3 lo, v3 hi) { return vmin(vmax(x, lo), hi); }
inline v3 vmix(v3 a, v3 b, float t) { return {mixf(a.x, b.x, t), mixf(a.y, b.y, t), mixf(a.z, b.z, t)}; }
inline v3 vmix3(v3 a, v3 b, v3 t) { return {mixf(a.x, b.x, t.x), mixf(a.y, b.y, t.y), mixf(a.z, b.z, t.z)}; }
inline float max3(v3 v) { return fmax_(v.x, fmax_(v.y, v.z)); }
inline float min3(v3 v) { return fmin_(v.x, fmin_(v.y, v.z)); }
inline bool in_unit_square(v2 uv) { return uv.x >= 0.0f && uv.y >= 0.0f && uv.x <= 1.0f && uv.y <= 1.0f; }

const v3 SUN_DIR = {SUN_DIR_X, SUN_DIR_Y, SUN_DIR_Z};
const v3 SUN_COLOR = {1.0f, 0.94f, 0.72f};
const v3 FOG_COLOR_GROUND = {0.40f, 0.42f, 0.45f};

// ---------------------------------------------------------------------------
// Bindings
// ---------------------------------------------------------------------------
struct Counters {
  uint64_t node_loads = 0, rope_loads = 0, meta_loads = 0, grid_loads = 0, macro_loads = 0, colinfo_loads = 0,
           clip_loads = 0, oob = 0;
};

struct Scene {
  const vxe_camera_gpu* cam;
  const vxe_chunk_meta* chunks;
  uint64_t chunks_n;
  const vxe_node* nodes;
  uint64_t nodes_n;
  const uint32_t* grid;
  uint64_t grid_n;
  const uint32_t* macro;  // macro_occ words as bound for this pass
  uint64_t macro_n;
  const vxe_node_ropes* ropes;
  uint64_t ropes_n;
  const uint32_t* colinfo;
  uint64_t colinfo_n;
  const vxe_clipmap_gpu* clip;
  const float* clip_tex;  // layers * res * res
  uint32_t clip_layers, clip_res;
  Counters* ctr;
  Counters* trace_ctr = nullptr;  // primary pass: loads of the voxel trace phase only
};

struct Node { uint32_t child_base, child_mask, material, key; };

inline Node node_global(const Scene& s, uint32_t gi) {
  s.ctr->node_loads++;
  if (gi >= s.nodes_n) { s.ctr->oob++; return Node{0, 0, 0, 0}; }
  const vxe_node& n = s.nodes[gi];
  return Node{n.child_base, n.child_mask, n.material, n.key};
}
inline Node node_at(const Scene& s, uint32_t base, uint32_t local) { return node_global(s, base + local); }
inline vxe_chunk_meta chunk_at(const Scene& s, uint32_t slot) {
  s.ctr->meta_loads++;
  if (slot >= s.chunks_n) { s.ctr->oob++; vxe_chunk_meta z; std::memset(&z, 0, sizeof z); return z; }
  return s.chunks[slot];
}
inline uint32_t grid_at(const Scene& s, uint32_t idx) {
  s.ctr->grid_loads++;
  if (idx >= s.grid_n) { s.ctr->oob++; return 0u; }
  return s.grid[idx];
}
inline uint32_t macro_word(const Scene& s, uint32_t idx) {
  s.ctr->macro_loads++;
  if (idx >= s.macro_n) { s.ctr->oob++; return 0u; }
  return s.macro[idx];
}
inline uint32_t colinfo_word(const Scene& s, uint32_t idx) {
  s.ctr->colinfo_loads++;
  if (idx >= s.colinfo_n) { s.ctr->oob++; return 0u; }
  return s.colinfo[idx];
}
inline uint32_t rope_face(const Scene& s, uint32_t gi, uint32_t face) {
  s.ctr->rope_loads++;
  if (gi >= s.ropes_n) { s.ctr->oob++; return 0u; }
  const vxe_node_ropes& r = s.ropes[gi];
  switch (face) {
    case 0: return r.px;
    case 1: return r.nx;
    case 2: return r.py;
    case 3: return r.ny;
    case 4: return r.pz;
    default: return r.nz;
  }
}
inline float clip_texel(const Scene& s, int32_t sx, int32_t sz, uint32_t level) {
  s.ctr->clip_loads++;
  if (level >= s.clip_layers || sx < 0 || sz < 0 || (uint32_t)sx >= s.clip_res || (uint32_t)sz >= s.clip_res) {
    s.ctr->oob++;
    return 0.0f;
  }
  return s.clip_tex[((size_t)level * s.clip_res + (uint32_t)sz) * s.clip_res + (uint32_t)sx];
}

inline v3 cam_pos(const Scene& s) { return V3(s.cam->cam_pos[0], s.cam->cam_pos[1], s.cam->cam_pos[2]); }
inline float vs_(const Scene& s) { return s.cam->voxel_params[0]; }

// ---------------------------------------------------------------------------
// common.wgsl helpers
// ---------------------------------------------------------------------------
inline float macro_cell_size(float root_size) { return root_size / (float)MACRO_DIM; }  // common.wgsl:426
inline uint32_t macro_bit_index(uint32_t mx, uint32_t my, uint32_t mz) {                 // common.wgsl:431
  return mx + MACRO_DIM * (my + MACRO_DIM * mz);
}
inline bool macro_test(const Scene& s, uint32_t macro_base, uint32_t bit) {  // common.wgsl:435-440
  const uint32_t w = bit >> 5, b = bit & 31u;
  return (macro_word(s, macro_base + w) & (1u << b)) != 0u;
}
inline float safe_inv(float x) { return std::fabs(x) < EPS_INV ? BIG : 1.0f / x; }  // common.wgsl:442
inline v3 safe_inv3(v3 r) { return V3(safe_inv(r.x), safe_inv(r.y), safe_inv(r.z)); }

inline v3 ray_dir_from_pixel(const Scene& s, v2 px) {  // common.wgsl:456-459
  const vxe_camera_gpu* c = s.cam;
  const v3 d = V3(c->ray00[0] + px.x * c->ray_dx[0] + px.y * c->ray_dy[0],
                  c->ray00[1] + px.x * c->ray_dx[1] + px.y * c->ray_dy[1],
                  c->ray00[2] + px.x * c->ray_dx[2] + px.y * c->ray_dy[2]);
  return normalize(d);
}

inline v2 prev_uv_from_world(const Scene& s, v3 p) {  // common.wgsl:461-467
  const float(*m)[4] = s.cam->prev_view_proj;
  // column-major: clip = c0*x + c1*y + c2*z + c3*1
  const float cx = m[0][0] * p.x + m[1][0] * p.y + m[2][0] * p.z + m[3][0] * 1.0f;
  const float cy = m[0][1] * p.x + m[1][1] * p.y + m[2][1] * p.z + m[3][1] * 1.0f;
  const float cw = m[0][3] * p.x + m[1][3] * p.y + m[2][3] * p.z + m[3][3] * 1.0f;
  const float invw = 1.0f / fmax_(cw, 1e-6f);
  const float nx = cx * invw, ny = cy * invw;
  const float ux = nx * 0.5f + 0.5f, uy = ny * 0.5f + 0.5f;
  return V2(ux, 1.0f - uy);
}

v2 intersect_aabb(v3 ro, v3 rd, v3 bmin, v3 bmax) {  // common.wgsl:473-510
  const float eps = 1e-8f;
  float t_enter = -1e30f, t_exit = 1e30f;
  const float r[3] = {ro.x, ro.y, ro.z}, d[3] = {rd.x, rd.y, rd.z};
  const float lo[3] = {bmin.x, bmin.y, bmin.z}, hi[3] = {bmax.x, bmax.y, bmax.z};
  for (int a = 0; a < 3; ++a) {
    if (std::fabs(d[a]) < eps) {
      if (r[a] < lo[a] || r[a] > hi[a]) return V2(1.0f, 0.0f);
    } else {
      const float inv = 1.0f / d[a];
      const float t0 = (lo[a] - r[a]) * inv, t1 = (hi[a] - r[a]) * inv;
      t_enter = fmax_(t_enter, fmin_(t0, t1));
      t_exit = fmin_(t_exit, fmax_(t0, t1));
    }
  }
  return V2(t_enter, t_exit);
}

inline uint32_t child_rank(uint32_t mask, uint32_t ci) {  // common.wgsl:512-516
  return (uint32_t)__builtin_popcount(mask & ((1u << ci) - 1u));
}

uint32_t grid_lookup_slot(const Scene& s, int32_t cx, int32_t cy, int32_t cz) {  // common.wgsl:518-541
  const int32_t ix = cx - s.cam->grid_origin_chunk[0], iy = cy - s.cam->grid_origin_chunk[1],
                iz = cz - s.cam->grid_origin_chunk[2];
  if (ix < 0 || iy < 0 || iz < 0) return INVALID;
  const uint32_t nx = s.cam->grid_dims[0], ny = s.cam->grid_dims[1], nz = s.cam->grid_dims[2];
  if ((uint32_t)ix >= nx || (uint32_t)iy >= ny || (uint32_t)iz >= nz) return INVALID;
  return grid_at(s, (uint32_t)iz * ny * nx + (uint32_t)iy * nx + (uint32_t)ix);
}

inline i3 chunk_coord_from_pos(v3 p, float cs) {  // common.wgsl:543-554
  const float eps = 1e-6f * cs;
  const float px = p.x - signf(p.x) * eps, py = p.y - signf(p.y) * eps, pz = p.z - signf(p.z) * eps;
  return i3{to_i32(std::floor(px / cs)), to_i32(std::floor(py / cs)), to_i32(std::floor(pz / cs))};
}

inline uint32_t chunk_max_depth(const Scene& s) {  // common.wgsl:569-572
  return 31u - (uint32_t)__builtin_clz(s.cam->chunk_size);
}

// Hashes / noise (common.wgsl:595-662)
inline uint32_t hash_u32(uint32_t v) {
  v ^= v >> 16;
  v *= 0x7feb352du;
  v ^= v >> 15;
  v *= 0x846ca68bu;
  v ^= v >> 16;
  return v;
}
inline uint32_t hash2_u32(uint32_t x, uint32_t y) { return hash_u32(x * 0x8da6b343u ^ y * 0xd8163841u); }
inline uint32_t hash3_u32(uint32_t x, uint32_t y, uint32_t z) {
  return hash_u32(x * 0x8da6b343u ^ y * 0xd8163841u ^ z * 0xcb1ab31fu);
}
constexpr float U32_TO_F01 = 1.0f / 4294967296.0f;
inline float hash12(v2 p) {
  const uint32_t ix = (uint32_t)to_i32(std::floor(p.x)), iy = (uint32_t)to_i32(std::floor(p.y));
  return (float)hash2_u32(ix, iy) * U32_TO_F01;
}
inline float hash31(v3 p) {
  const uint32_t ix = (uint32_t)to_i32(std::floor(p.x)), iy = (uint32_t)to_i32(std::floor(p.y)),
                 iz = (uint32_t)to_i32(std::floor(p.z));
  return (float)hash3_u32(ix, iy, iz) * U32_TO_F01;
}
float value_noise(v2 p) {
  const v2 i = vfloor(p), f = vfract(p);
  const float a = hash12(i), b = hash12(i + V2(1.0f, 0.0f)), c = hash12(i + V2(0.0f, 1.0f)),
              d = hash12(i + V2(1.0f, 1.0f));
  const v2 u = V2(f.x * f.x * (3.0f - 2.0f * f.x), f.y * f.y * (3.0f - 2.0f * f.y));
  const float x1 = mixf(a, b, u.x), x2 = mixf(c, d, u.x);
  return mixf(x1, x2, u.y);
}
float fbm(v2 p) {
  v2 x = p;
  float sum = 0.0f, amp = 0.5f;
  for (uint32_t i = 0; i < 5; ++i) {
    sum += amp * value_noise(x);
    // rot = mat2x2(0.8,-0.6, 0.6,0.8) column-major: rot*x = (0.8x+0.6y, -0.6x+0.8y)
    const v2 r = V2(0.8f * x.x + 0.6f * x.y, -0.6f * x.x + 0.8f * x.y);
    x = r * 2.0f + V2(17.0f, 9.0f);
    amp *= 0.5f;
  }
  return sum;
}

inline bool is_bad(v3 v) {  // common.wgsl:692-706
  auto bad = [](float x) { return x != x || std::fabs(x) > 1.0e30f; };
  return bad(v.x) || bad(v.y) || bad(v.z);
}
inline v3 ray_eps_vec(v3 rd, float e) {  // common.wgsl:708-715
  return V3(rd.x >= 0.0f ? e : -e, rd.y >= 0.0f ? e : -e, rd.z >= 0.0f ? e : -e);
}

// ---------------------------------------------------------------------------
// aabb.wgsl
// ---------------------------------------------------------------------------
struct CubeSlab { v3 tminv, tmaxv; float t_enter, t_exit; };

CubeSlab cube_slab_inv(v3 ro, v3 inv, v3 bmin, float size) {  // aabb.wgsl:16-84
  const v3 bmax = bmin + V3s(size);
  v3 t0 = (bmin - ro) * inv, t1 = (bmax - ro) * inv;
  const float INV_PARALLEL = 1e20f;
  const CubeSlab miss{V3s(BIG), V3s(-BIG), BIG, -BIG};
  if (std::fabs(inv.x) > INV_PARALLEL) {
    if (ro.x < bmin.x || ro.x >= bmax.x) return miss;
    t0.x = -BIG; t1.x = BIG;
  }
  if (std::fabs(inv.y) > INV_PARALLEL) {
    if (ro.y < bmin.y || ro.y >= bmax.y) return miss;
    t0.y = -BIG; t1.y = BIG;
  }
  if (std::fabs(inv.z) > INV_PARALLEL) {
    if (ro.z < bmin.z || ro.z >= bmax.z) return miss;
    t0.z = -BIG; t1.z = BIG;
  }
  const v3 tminv = vmin(t0, t1), tmaxv = vmax(t0, t1);
  return CubeSlab{tminv, tmaxv, max3(tminv), min3(tmaxv)};
}

struct BoxHit { bool hit; float t, t_exit; v3 n; };

BoxHit cube_hit_normal_from_slab(v3 rd, const CubeSlab& slab, float t_min, float t_max) {  // aabb.wgsl:95-141
  const float t0 = fmax_(slab.t_enter, t_min);
  if (slab.t_exit < t0 || t0 > t_max) return BoxHit{false, BIG, slab.t_exit, V3s(0.0f)};
  const float te = slab.t_enter;
  const float eps = 1e-5f * fmax_(1.0f, std::fabs(te));
  const bool mx = std::fabs(slab.tminv.x - te) <= eps, my = std::fabs(slab.tminv.y - te) <= eps,
             mz = std::fabs(slab.tminv.z - te) <= eps;
  uint32_t axis = 0;
  if (mx || my || mz) {
    float best = -1.0f;
    if (mx) { best = std::fabs(rd.x); axis = 0; }
    if (my && std::fabs(rd.y) > best) { best = std::fabs(rd.y); axis = 1; }
    if (mz && std::fabs(rd.z) > best) { best = std::fabs(rd.z); axis = 2; }
  } else {
    float bestv = slab.tminv.x;
    axis = 0;
    if (slab.tminv.y > bestv) { bestv = slab.tminv.y; axis = 1; }
    if (slab.tminv.z > bestv) { bestv = slab.tminv.z; axis = 2; }
  }
  v3 n = V3s(0.0f);
  if (axis == 0) n = V3(rd.x > 0.0f ? -1.0f : 1.0f, 0.0f, 0.0f);
  if (axis == 1) n = V3(0.0f, rd.y > 0.0f ? -1.0f : 1.0f, 0.0f);
  if (axis == 2) n = V3(0.0f, 0.0f, rd.z > 0.0f ? -1.0f : 1.0f);
  return BoxHit{true, t0, slab.t_exit, n};
}

inline BoxHit aabb_hit_normal_inv(v3 ro, v3 rd, v3 inv, v3 bmin, float size, float tmin, float tmax) {
  return cube_hit_normal_from_slab(rd, cube_slab_inv(ro, inv, bmin, size), tmin, tmax);
}

// ---------------------------------------------------------------------------
// svo_query.wgsl
// ---------------------------------------------------------------------------
struct LeafQuery { v3 bmin; float size; uint32_t mat; };

LeafQuery query_leaf_at(const Scene& s, v3 p, v3 root_bmin, float root_size, uint32_t node_base,
                        uint32_t macro_base) {  // svo_query.wgsl:11-108
  uint32_t idx = node_base;
  v3 bmin = root_bmin;
  float size = root_size;
  if (macro_base != INVALID) {
    const float cell = macro_cell_size(root_size);
    const v3 lp = p - root_bmin;
    if (lp.x < 0.0f || lp.y < 0.0f || lp.z < 0.0f || lp.x >= root_size || lp.y >= root_size || lp.z >= root_size)
      return LeafQuery{root_bmin, root_size, MAT_AIR};
    const int32_t mx = to_i32(std::floor(lp.x / cell)), my = to_i32(std::floor(lp.y / cell)),
                  mz = to_i32(std::floor(lp.z / cell));
    if (mx < 0 || my < 0 || mz < 0 || mx >= (int32_t)MACRO_DIM || my >= (int32_t)MACRO_DIM || mz >= (int32_t)MACRO_DIM)
      return LeafQuery{root_bmin, root_size, MAT_AIR};
    if (!macro_test(s, macro_base, macro_bit_index((uint32_t)mx, (uint32_t)my, (uint32_t)mz)))
      return LeafQuery{root_bmin, root_size, MAT_AIR};
  }
  for (uint32_t d = 0; d < 32; ++d) {
    const Node n = node_global(s, idx);
    if (n.child_base == LEAF) return LeafQuery{bmin, size, n.material};
    if (d >= chunk_max_depth(s)) return LeafQuery{bmin, size, MAT_AIR};
    const float half = size * 0.5f;
    const v3 mid = bmin + V3s(half);
    const float e = 1e-6f * size;
    const uint32_t hx = p.x > mid.x + e ? 1u : 0u, hy = p.y > mid.y + e ? 1u : 0u, hz = p.z > mid.z + e ? 1u : 0u;
    const uint32_t ci = hx | (hy << 1) | (hz << 2);
    const v3 cb = bmin + V3(hx ? half : 0.0f, hy ? half : 0.0f, hz ? half : 0.0f);
    if ((n.child_mask & (1u << ci)) == 0u) return LeafQuery{cb, half, MAT_AIR};
    idx = node_base + (n.child_base + child_rank(n.child_mask, ci));
    bmin = cb;
    size = half;
  }
  return LeafQuery{bmin, size, MAT_AIR};
}

LeafQuery query_leaf_world(const Scene& s, v3 p) {  // svo_query.wgsl:115-136
  const float vs = vs_(s);
  const float cs = (float)s.cam->chunk_size * vs;
  const i3 c = chunk_coord_from_pos(p, cs);
  const uint32_t slot = grid_lookup_slot(s, c.x, c.y, c.z);
  if (slot == INVALID || slot >= s.cam->chunk_count) return LeafQuery{p, vs, MAT_AIR};
  const vxe_chunk_meta ch = chunk_at(s, slot);
  const v3 rb = V3((float)ch.origin[0], (float)ch.origin[1], (float)ch.origin[2]) * vs;
  return query_leaf_at(s, p, rb, (float)s.cam->chunk_size * vs, ch.node_base, ch.macro_base);
}

// ---------------------------------------------------------------------------
// wind.wgsl / leaves.wgsl
// ---------------------------------------------------------------------------
inline float hash1(v3 p) { return fract(sinf_(dot(p, V3(127.1f, 311.7f, 74.7f))) * 43758.5453f); }

v3 wind_field(v3 pos, float t) {  // wind.wgsl:10-36
  const v3 cell = vfloor(pos * WIND_CELL_FREQ);
  const float ph0 = hash1(cell), ph1 = hash1(cell + V3(19.0f, 7.0f, 11.0f));
  const v2 dir = normalize(V2(0.9f, 0.4f));
  const float h = clampf((pos.y - WIND_RAMP_Y0) / fmax_(WIND_RAMP_Y1 - WIND_RAMP_Y0, 1e-3f), 0.0f, 1.0f);
  const float gust = sinf_(t * WIND_GUST_TIME_FREQ + dot(V2(pos.x, pos.z), V2(0.35f, 0.22f)) + ph0 * TAU);
  const float flutter = sinf_(t * WIND_FLUTTER_TIME_FREQ + dot(V2(pos.x, pos.z), V2(1.7f, 1.1f)) + ph1 * TAU);
  const v2 xz = dir * (WIND_GUST_WEIGHT * gust + WIND_FLUTTER_WEIGHT * flutter) * h;
  const float y = WIND_VERTICAL_SCALE * flutter * h;
  return V3(xz.x, y, xz.y);
}

inline v3 clamp_len(v3 v, float max_len) {  // wind.wgsl:38-42
  const float l2 = dot(v, v);
  if (l2 <= max_len * max_len) return v;
  return v * (max_len / std::sqrt(l2));
}

v3 leaf_cube_offset(const Scene& s, v3 bmin, float size, float time_s, float strength) {  // leaves.wgsl:5-18
  const v3 center = bmin + V3s(0.5f * size);
  const float d = length(center - cam_pos(s));
  const float fade = smooth(LEAF_LOD_DISP_START, LEAF_LOD_DISP_END, d);
  const float se = strength * (1.0f - fade);
  v3 w = wind_field(center, time_s) * se;
  w = V3(w.x, LEAF_VERTICAL_REDUCE * w.y, w.z);
  const float amp = LEAF_OFFSET_AMP * size;
  return clamp_len(w * amp, LEAF_OFFSET_MAX_FRAC * size);
}

BoxHit leaf_displaced_cube_hit(const Scene& s, v3 ro, v3 rd, v3 bmin, float size, float time_s, float strength,
                               float tmin, float tmax) {  // leaves.wgsl:26-43
  const v3 off = leaf_cube_offset(s, bmin, size, time_s, strength);
  const v3 b2 = bmin + off;
  return aabb_hit_normal_inv(ro, rd, safe_inv3(rd), b2, size, tmin, tmax);
}

// ---------------------------------------------------------------------------
// grass.wgsl
// ---------------------------------------------------------------------------
struct GrassCell { v3 bmin_m, id_vox; };
struct GrassHit { bool hit; float t; v3 n; };

GrassCell pick_grass_cell_in_chunk_with_bias(v3 hp, v3 bias_dir, v3 root_bmin, i3 origin_vox, float vs,
                                            int32_t csv) {  // grass.wgsl:10-44
  const float root_size_m = (float)csv * vs;
  const float bias = 0.05f * vs;
  v3 lxz = (hp - root_bmin) - bias_dir * bias;
  lxz.x = clampf(lxz.x, 0.0f, root_size_m - 1e-6f);
  lxz.z = clampf(lxz.z, 0.0f, root_size_m - 1e-6f);
  const float y_in = (hp - bias_dir * bias).y - 1e-4f * vs;
  const float ly = clampf(y_in - root_bmin.y, 0.0f, root_size_m - 1e-6f);
  int32_t ix = to_i32(std::floor(lxz.x / vs)), iy = to_i32(std::floor(ly / vs)), iz = to_i32(std::floor(lxz.z / vs));
  ix = clampi(ix, 0, csv - 1);
  iy = clampi(iy, 0, csv - 1);
  iz = clampi(iz, 0, csv - 1);
  const v3 bmin = root_bmin + V3((float)ix, (float)iy, (float)iz) * vs;
  const v3 id = V3((float)(origin_vox.x + ix), (float)(origin_vox.y + iy), (float)(origin_vox.z + iz));
  return GrassCell{bmin, id};
}

GrassCell grass_cell_from_world(v3 hp, v3 rd, v3 root_bmin, float vs, int32_t csv) {  // grass.wgsl:64-84
  const i3 o{to_i32(std::floor(root_bmin.x / vs)), to_i32(std::floor(root_bmin.y / vs)),
             to_i32(std::floor(root_bmin.z / vs))};
  return pick_grass_cell_in_chunk_with_bias(hp, rd, root_bmin, o, vs, csv);
}

GrassCell grass_cell_from_world_global(v3 hp, v3 rd, float vs) {  // grass.wgsl:86-104
  const float bias = 0.05f * vs;
  const v3 p = hp - rd * bias;
  const float py = p.y - 1e-4f * vs;
  const int32_t ix = to_i32(std::floor(p.x / vs)), iy = to_i32(std::floor(py / vs)), iz = to_i32(std::floor(p.z / vs));
  const v3 id = V3((float)ix, (float)iy, (float)iz);
  return GrassCell{id * vs, id};
}

inline float sdf_box(v3 p, v3 c, v3 b) {  // grass.wgsl:106-111
  const v3 q = vabs(p - c) - b;
  const float outside = length(vmax(q, V3s(0.0f)));
  const float inside = fmin_(fmax_(q.x, fmax_(q.y, q.z)), 0.0f);
  return outside + inside;
}

inline v3 ortho_basis_x(v3 n) {  // grass.wgsl:120-126 (column 0)
  const v3 up = std::fabs(n.y) > 0.999f ? V3(1.0f, 0.0f, 0.0f) : V3(0.0f, 1.0f, 0.0f);
  return normalize(cross(up, n));
}

inline v4 grass_blade_params(v3 id, uint32_t i) {  // grass.wgsl:353-368
  const float fi = (float)i;
  const float h0 = hash31(id + V3(fi * 7.3f, 1.1f, 2.9f));
  const float h1 = hash31(id + V3(fi * 3.7f, 8.4f, 0.6f));
  return v4{fract(h0 * 1.61803398875f), fract(h0 * 2.41421356237f), fract(h0 * 3.14159265359f),
            0.35f + 0.65f * (h1 * h1)};
}

inline v2 grass_wind_xz(v3 root, float t, float strength) {  // grass.wgsl:185-189
  const v3 w = wind_field(root, t) * strength;
  return V2(w.x, w.z);
}

float grass_sdf_lod(const Scene& s, v3 p, v3 cb, v3 id, float time_s, float strength, uint32_t lod) {
  // grass.wgsl:192-350
  const float vs = vs_(s);
  const float top_y = cb.y + vs;
  const float layer_h = GRASS_LAYER_HEIGHT_VOX * vs;
  const float y01 = (p.y - top_y) / fmax_(layer_h, 1e-6f);
  if (y01 < 0.0f || y01 > 1.0f) return BIG;
  const float over = GRASS_OVERHANG_VOX * vs;
  if (p.x < cb.x - over || p.x > cb.x + vs + over || p.z < cb.z - over || p.z > cb.z + vs + over) return BIG;
  const float blade_len = layer_h * (0.65f + 0.35f * hash31(id + V3(9.1f, 3.7f, 5.2f)));
  uint32_t blade_count = GRASS_BLADE_COUNT;
  uint32_t segs = to_u32(fmax_(3.0f, std::floor(GRASS_VOXEL_SEGS)));
  if (lod == 1u) {
    blade_count = std::min(blade_count, GRASS_BLADE_COUNT_MID);
    segs = std::min(segs, GRASS_SEGS_MID);
  } else if (lod == 2u) {
    blade_count = std::min(blade_count, GRASS_BLADE_COUNT_FAR);
    segs = std::min(segs, GRASS_SEGS_FAR);
  }
  const float inv_segs = 1.0f / fmax_((float)segs, 1.0f);
  float dmin = BIG;
  const float clump_r = 0.18f * vs;
  const float base_r = (GRASS_VOXEL_THICKNESS_VOX * vs) * 0.85f;
  for (uint32_t i = 0; i < blade_count; ++i) {
    const v4 uvpw = grass_blade_params(id, i);
    const float u0 = uvpw.x, v0 = uvpw.y, ph = uvpw.z, wR = uvpw.w;
    const float cfi = (float)(i % 5u);
    const float cu = hash31(id + V3(13.7f + cfi, 2.1f, 9.9f));
    const float cv = hash31(id + V3(4.2f + cfi, 7.3f, 1.4f));
    const float inset = 0.10f;
    const float cux = mixf(inset, 1.0f - inset, cu), cvz = mixf(inset, 1.0f - inset, cv);
    const v2 clump_center = V2(cb.x + cux * vs, cb.z + cvz * vs);
    const float ang = TAU * u0;
    const float rr = clump_r * (0.15f + 0.85f * v0);
    const v2 root_xz = clump_center + V2(cosf_(ang), sinf_(ang)) * rr;
    const v3 root = V3(root_xz.x, top_y, root_xz.y);
    const v2 w_xz = 0.35f * grass_wind_xz(root + V3(0.0f, ph, 0.0f), time_s, strength);
    const float lean_ang = TAU * fract(u0 * 1.73f + v0 * 2.11f);
    const v2 lean_dir = V2(cosf_(lean_ang), sinf_(lean_ang));
    const float lean_amt = 0.10f + 0.25f * (v0 * v0);
    const float r0 = base_r * mixf(0.85f, 1.35f, wR);
    const float roll = TAU * (0.15f * ph + 0.10f * wR);
    const v2 roll_dir = V2(cosf_(roll), sinf_(roll));
    const v3 side_hint = normalize(V3(lean_dir.x * roll_dir.x - lean_dir.y * roll_dir.y, 0.12f,
                                      lean_dir.x * roll_dir.y + lean_dir.y * roll_dir.x));
    for (uint32_t sg = 0; sg < segs; ++sg) {
      const float t01a = (float)sg * inv_segs;
      const float t01b = ((float)sg + 1.0f) * inv_segs;
      const float ya = t01a * blade_len, yb = t01b * blade_len;
      const float seg_h = yb - ya;
      const float bend_a = (blade_len * t01a) * (0.55f + 0.45f * t01a);
      const float bend_b = (blade_len * t01b) * (0.55f + 0.45f * t01b);
      const v2 bva = w_xz * t01a + lean_dir * lean_amt;
      const v2 bvb = w_xz * t01b + lean_dir * lean_amt;
      const v2 offa = bva * bend_a, offb = bvb * bend_b;
      const v3 pa = root + V3(offa.x, ya, offa.y);
      const v3 pb = root + V3(offb.x, yb, offb.y);
      const v3 T = normalize(pb - pa);
      v3 S = side_hint - T * dot(side_hint, T);
      const float s2 = dot(S, S);
      if (s2 < 1e-6f) S = ortho_basis_x(T);
      else S = S * (1.0f / std::sqrt(s2));
      const v3 N = cross(T, S);
      const v3 mid = 0.5f * (pa + pb);
      const v3 d = p - mid;
      const v3 local = V3(dot(d, S), dot(d, T), dot(d, N));
      const float tmid = 0.5f * (t01a + t01b);
      const float taper_shape = powf_(clampf(1.0f - tmid, 0.0f, 1.0f), 3.0f);
      const float taper = mixf(GRASS_VOXEL_TAPER, 1.0f, taper_shape);
      const float half_w = r0 * taper * 0.7f;
      const float dbox = sdf_box(local, V3s(0.0f), V3(half_w, 0.5f * seg_h, half_w));
      dmin = fmin_(dmin, dbox);
    }
  }
  return dmin;
}

v3 grass_sdf_normal_lod(const Scene& s, v3 p, v3 cb, v3 id, float time_s, float strength, uint32_t lod) {
  // grass.wgsl:370-408
  if (lod != 0u) {
    const float vs = vs_(s);
    const float top_y = cb.y + vs;
    const v3 root = V3(cb.x + 0.5f * vs, top_y, cb.z + 0.5f * vs);
    const v2 w = grass_wind_xz(root, time_s, strength);
    const float tilt = 0.35f;
    return normalize(V3(-w.x * tilt, 1.0f, -w.y * tilt));
  }
  const float e = 0.01f * vs_(s);
  const float dx = grass_sdf_lod(s, p + V3(e, 0.0f, 0.0f), cb, id, time_s, strength, lod) -
                   grass_sdf_lod(s, p - V3(e, 0.0f, 0.0f), cb, id, time_s, strength, lod);
  const float dy = grass_sdf_lod(s, p + V3(0.0f, e, 0.0f), cb, id, time_s, strength, lod) -
                   grass_sdf_lod(s, p - V3(0.0f, e, 0.0f), cb, id, time_s, strength, lod);
  const float dz = grass_sdf_lod(s, p + V3(0.0f, 0.0f, e), cb, id, time_s, strength, lod) -
                   grass_sdf_lod(s, p - V3(0.0f, 0.0f, e), cb, id, time_s, strength, lod);
  return normalize(V3(dx, dy, dz));
}

float grass_self_shadow(const Scene& s, v3 hp, v3 cb, v3 id, float time_s, float strength, uint32_t lod) {
  // grass.wgsl:410-447
  const float vs = vs_(s);
  v3 p = hp + SUN_DIR * (0.02f * vs);
  const float max_dist = (0.55f + 0.35f * (float)lod) * vs;
  const uint32_t steps = lod != 0u ? 4u : 6u;
  const float dt = max_dist / (float)steps;
  float occ = 0.0f;
  for (uint32_t i = 0; i < steps; ++i) {
    const float d = grass_sdf_lod(s, p, cb, id, time_s, strength, lod);
    occ += clampf(1.0f - d / (0.05f * vs), 0.0f, 1.0f);
    p = p + SUN_DIR * dt;
  }
  return expf_(-0.35f * occ);
}

inline uint32_t grass_lod_from_t(float t) {  // grass.wgsl:540-545
  if (t >= GRASS_LOD_FAR_START) return 2u;
  if (t >= GRASS_LOD_MID_START) return 1u;
  return 0u;
}

GrassHit grass_layer_trace_lod(const Scene& s, v3 ro, v3 rd, float t_start, float t_end, v3 cb, v3 id, float time_s,
                               float strength, uint32_t lod) {  // grass.wgsl:456-491
  const float vs = vs_(s);
  float t = t_start;
  uint32_t steps = GRASS_TRACE_STEPS;
  if (lod == 1u) steps = GRASS_TRACE_STEPS_MID;
  if (lod == 2u) steps = GRASS_TRACE_STEPS_FAR;
  for (uint32_t i = 0; i < steps; ++i) {
    if (t > t_end) break;
    const v3 p = ro + rd * t;
    const float d = grass_sdf_lod(s, p, cb, id, time_s, strength, lod);
    if (d < GRASS_HIT_EPS_VOX * vs) {
      return GrassHit{true, t, grass_sdf_normal_lod(s, p, cb, id, time_s, strength, lod)};
    }
    t += fmax_(d, GRASS_STEP_MIN_VOX * vs);
  }
  return GrassHit{false, BIG, V3s(0.0f)};
}

GrassHit try_grass_slab_hit(const Scene& s, v3 ro, v3 rd, float t_min, float t_max, v3 cb, v3 id, float vs,
                            float time_s, float strength) {  // grass.wgsl:494-538
  const float layer_h = GRASS_LAYER_HEIGHT_VOX * vs;
  const float over = GRASS_OVERHANG_VOX * vs;
  const v3 sb0 = V3(cb.x - over, cb.y + vs, cb.z - over);
  const v3 sb1 = V3(cb.x + vs + over, cb.y + vs + layer_h, cb.z + vs + over);
  const v2 rs = intersect_aabb(ro, rd, sb0, sb1);
  const float t0 = fmax_(rs.x, t_min);
  float t1 = fmin_(rs.y, t_max);
  const v2 rv = intersect_aabb(ro, rd, cb, cb + V3s(vs));
  const float clip_eps = 0.01f * vs;
  if (rv.y > rv.x) {
    if (rv.x > t0) t1 = fmin_(t1, rv.x - clip_eps);
  }
  if (t1 <= t0) return GrassHit{false, BIG, V3s(0.0f)};
  return grass_layer_trace_lod(s, ro, rd, t0, t1, cb, id, time_s, strength, grass_lod_from_t(t0));
}

// ---------------------------------------------------------------------------
// chunk_trace.wgsl
// ---------------------------------------------------------------------------
struct HitGeom {
  uint32_t hit, mat;
  float t;
  v3 n, root_bmin;
  float root_size;
  uint32_t node_base, macro_base;
  // hit-record extras (not in the reference): leaf node + leaf cube
  uint32_t node;
  v3 leaf_bmin;
  float leaf_size;
};

inline HitGeom miss_hitgeom() {  // chunk_trace.wgsl:40-51
  HitGeom h;
  h.hit = 0; h.mat = MAT_AIR; h.t = BIG; h.n = V3s(0.0f); h.root_bmin = V3s(0.0f); h.root_size = 0.0f;
  h.node_base = 0; h.macro_base = INVALID; h.node = INVALID; h.leaf_bmin = V3s(0.0f); h.leaf_size = 0.0f;
  return h;
}

struct ChunkTraceResult { HitGeom hit; bool anchor_valid; uint32_t anchor_key; };

inline bool point_in_cube(v3 p, v3 bmin, float size) {  // chunk_trace.wgsl:54-59
  const v3 bmax = bmin + V3s(size);
  return p.x >= bmin.x && p.x < bmax.x && p.y >= bmin.y && p.y < bmax.y && p.z >= bmin.z && p.z < bmax.z;
}

inline uint32_t node_level(uint32_t k) { return (k >> 18) & 7u; }
inline uint32_t node_x(uint32_t k) { return k & 63u; }
inline uint32_t node_y(uint32_t k) { return (k >> 6) & 63u; }
inline uint32_t node_z(uint32_t k) { return (k >> 12) & 63u; }

inline v4 node_cube_from_key(v3 rb, float rs, uint32_t key) {  // chunk_trace.wgsl:123-128
  const float sz = rs / (float)(1u << node_level(key));
  const v3 b = rb + V3((float)node_x(key), (float)node_y(key), (float)node_z(key)) * sz;
  return v4{b.x, b.y, b.z, sz};
}

struct AnchorNode { bool valid; uint32_t idx; v3 bmin; float size; uint32_t key; };

AnchorNode anchor_from_key(const Scene& s, uint32_t node_base, v3 rb, float rs, uint32_t key) {
  // chunk_trace.wgsl:138-191
  if (key == INVALID) return AnchorNode{false, 0, V3s(0.0f), 0.0f, INVALID};
  const uint32_t lvl = std::min(node_level(key), chunk_max_depth(s));
  const uint32_t tx = node_x(key), ty = node_y(key), tz = node_z(key);
  uint32_t idx = 0;
  v3 bmin = rb;
  float size = rs;
  for (uint32_t d = 0; d < 32; ++d) {
    if (d >= lvl) return AnchorNode{true, idx, bmin, size, node_at(s, node_base, idx).key};
    const Node n = node_at(s, node_base, idx);
    if (n.child_base == LEAF) return AnchorNode{true, idx, bmin, size, n.key};
    const uint32_t sh = (lvl - 1u) - d;
    const uint32_t hx = (tx >> sh) & 1u, hy = (ty >> sh) & 1u, hz = (tz >> sh) & 1u;
    const uint32_t ci = hx | (hy << 1) | (hz << 2);
    if ((n.child_mask & (1u << ci)) == 0u) return AnchorNode{true, idx, bmin, size, n.key};
    const float half = size * 0.5f;
    bmin = bmin + V3(hx ? half : 0.0f, hy ? half : 0.0f, hz ? half : 0.0f);
    size = half;
    idx = n.child_base + child_rank(n.child_mask, ci);
  }
  return AnchorNode{true, idx, bmin, size, node_at(s, node_base, idx).key};
}

struct LeafState {
  bool has_node;
  uint32_t idx_local;
  v3 bmin;
  float size;
  uint32_t mat;
  bool has_anchor;
  uint32_t anchor_idx;
  v3 anchor_bmin;
  float anchor_size;
};

AnchorNode anchor_from_leaf(const Scene& s, const LeafState& l, uint32_t node_base) {  // chunk_trace.wgsl:193-203
  if (l.has_node) return AnchorNode{true, l.idx_local, l.bmin, l.size, node_at(s, node_base, l.idx_local).key};
  if (l.has_anchor)
    return AnchorNode{true, l.anchor_idx, l.anchor_bmin, l.anchor_size, node_at(s, node_base, l.anchor_idx).key};
  return AnchorNode{false, 0, V3s(0.0f), 0.0f, INVALID};
}

struct ExitFaceRes { uint32_t face, amb; };

ExitFaceRes exit_face_from_slab_safe(v3 rd, const CubeSlab& slab) {  // chunk_trace.wgsl:233-272
  const float te = slab.t_exit;
  const float eps = 1e-5f * fmax_(1.0f, std::fabs(te));
  const bool mx = std::fabs(rd.x) >= EPS_INV && std::fabs(slab.tmaxv.x - te) <= eps;
  const bool my = std::fabs(rd.y) >= EPS_INV && std::fabs(slab.tmaxv.y - te) <= eps;
  const bool mz = std::fabs(rd.z) >= EPS_INV && std::fabs(slab.tmaxv.z - te) <= eps;
  const uint32_t c = (mx ? 1u : 0u) + (my ? 1u : 0u) + (mz ? 1u : 0u);
  if (c >= 2u) return ExitFaceRes{0, 1};
  uint32_t axis = 0;
  if (c == 1u) {
    if (mx) axis = 0;
    if (my) axis = 1;
    if (mz) axis = 2;
  } else {
    float bestv = slab.tmaxv.x;
    axis = 0;
    if (slab.tmaxv.y < bestv) { bestv = slab.tmaxv.y; axis = 1; }
    if (slab.tmaxv.z < bestv) { bestv = slab.tmaxv.z; axis = 2; }
  }
  if (axis == 0) return ExitFaceRes{rd.x > 0.0f ? 0u : 1u, 0};
  if (axis == 1) return ExitFaceRes{rd.y > 0.0f ? 2u : 3u, 0};
  return ExitFaceRes{rd.z > 0.0f ? 4u : 5u, 0};
}

LeafState descend_leaf_sparse(const Scene& s, v3 p, uint32_t node_base, uint32_t start_idx, v3 start_bmin,
                              float start_size) {  // chunk_trace.wgsl:296-358
  uint32_t idx = start_idx;
  v3 bmin = start_bmin;
  float size = start_size;
  const uint32_t max_d = chunk_max_depth(s);
  for (uint32_t d = 0; d < 32; ++d) {
    const Node n = node_at(s, node_base, idx);
    if (n.child_base == LEAF) return LeafState{true, idx, bmin, size, n.material, false, 0, V3s(0.0f), 0.0f};
    if (d >= max_d) return LeafState{true, idx, bmin, size, MAT_AIR, false, 0, V3s(0.0f), 0.0f};
    const float half = size * 0.5f;
    const v3 mid = bmin + V3s(half);
    const float e = 1e-6f * size;
    const uint32_t hx = p.x > mid.x + e ? 1u : 0u, hy = p.y > mid.y + e ? 1u : 0u, hz = p.z > mid.z + e ? 1u : 0u;
    const uint32_t ci = hx | (hy << 1) | (hz << 2);
    const v3 cb = bmin + V3(hx ? half : 0.0f, hy ? half : 0.0f, hz ? half : 0.0f);
    if ((n.child_mask & (1u << ci)) == 0u) return LeafState{false, INVALID, cb, half, MAT_AIR, true, idx, bmin, size};
    idx = n.child_base + child_rank(n.child_mask, ci);
    bmin = cb;
    size = half;
  }
  return LeafState{false, INVALID, start_bmin, start_size, MAT_AIR, false, INVALID, V3s(0.0f), 0.0f};
}

struct MacroDDAState {
  bool enabled;
  int32_t mx, my, mz, step_x, step_y, step_z;
  float tMaxX, tMaxY, tMaxZ, tDeltaX, tDeltaY, tDeltaZ, cell;
};

MacroDDAState macro_dda_init(v3 ro, v3 rd, v3 inv, float tcur, v3 rb, float rs, uint32_t macro_base) {
  // chunk_trace.wgsl:397-475
  MacroDDAState st;
  st.enabled = false;
  st.mx = st.my = st.mz = 0;
  st.step_x = st.step_y = st.step_z = 0;
  st.tMaxX = st.tMaxY = st.tMaxZ = BIG;
  st.tDeltaX = st.tDeltaY = st.tDeltaZ = BIG;
  st.cell = 0.0f;
  if (macro_base == INVALID) return st;
  const float cell = macro_cell_size(rs);
  const v3 p = ro + rd * tcur;
  const v3 lp = p - rb;
  if (lp.x < 0.0f || lp.y < 0.0f || lp.z < 0.0f || lp.x >= rs || lp.y >= rs || lp.z >= rs) return st;
  const int32_t mx = to_i32(std::floor(lp.x / cell)), my = to_i32(std::floor(lp.y / cell)),
                mz = to_i32(std::floor(lp.z / cell));
  if (mx < 0 || my < 0 || mz < 0 || mx >= 8 || my >= 8 || mz >= 8) return st;
  st.enabled = true;
  st.mx = mx; st.my = my; st.mz = mz;
  st.step_x = rd.x > 0.0f ? 1 : -1;
  st.step_y = rd.y > 0.0f ? 1 : -1;
  st.step_z = rd.z > 0.0f ? 1 : -1;
  st.tDeltaX = std::fabs(cell * inv.x);
  st.tDeltaY = std::fabs(cell * inv.y);
  st.tDeltaZ = std::fabs(cell * inv.z);
  st.cell = cell;
  if (std::fabs(rd.x) >= EPS_INV) {
    const float bx = rb.x + (float)(mx + (rd.x > 0.0f ? 1 : 0)) * cell;
    st.tMaxX = tcur + (bx - p.x) * inv.x;
  }
  if (std::fabs(rd.y) >= EPS_INV) {
    const float by = rb.y + (float)(my + (rd.y > 0.0f ? 1 : 0)) * cell;
    st.tMaxY = tcur + (by - p.y) * inv.y;
  }
  if (std::fabs(rd.z) >= EPS_INV) {
    const float bz = rb.z + (float)(mz + (rd.z > 0.0f ? 1 : 0)) * cell;
    st.tMaxZ = tcur + (bz - p.z) * inv.z;
  }
  return st;
}

inline float macro_dda_t_exit(const MacroDDAState& st) { return fmin_(st.tMaxX, fmin_(st.tMaxY, st.tMaxZ)); }

void macro_dda_step(MacroDDAState& st) {  // chunk_trace.wgsl:536-559
  const float tn = macro_dda_t_exit(st);
  const float e = 1e-6f * fmax_(1.0f, std::fabs(tn));
  if (std::fabs(st.tMaxX - tn) <= e) { st.mx += st.step_x; st.tMaxX += st.tDeltaX; }
  if (std::fabs(st.tMaxY - tn) <= e) { st.my += st.step_y; st.tMaxY += st.tDeltaY; }
  if (std::fabs(st.tMaxZ - tn) <= e) { st.mz += st.step_z; st.tMaxZ += st.tDeltaZ; }
  if (st.mx < 0 || st.my < 0 || st.mz < 0 || st.mx >= 8 || st.my >= 8 || st.mz >= 8) st.enabled = false;
}

void macro_dda_sync(MacroDDAState& st, float tcur) {  // chunk_trace.wgsl:561-568
  for (uint32_t i = 0; i < 32; ++i) {
    if (!st.enabled) break;
    if (tcur < macro_dda_t_exit(st)) break;
    macro_dda_step(st);
  }
}

struct MacroStep { bool valid, empty; float t_exit; };

MacroStep macro_dda_current(const Scene& s, const MacroDDAState& st, uint32_t macro_base) {  // chunk_trace.wgsl:570-587
  MacroStep o{st.enabled, false, macro_dda_t_exit(st)};
  if (!st.enabled || macro_base == INVALID) { o.valid = false; return o; }
  o.empty = !macro_test(s, macro_base, macro_bit_index((uint32_t)st.mx, (uint32_t)st.my, (uint32_t)st.mz));
  return o;
}

// colinfo (chunk_trace.wgsl:1284-1308)
inline uint32_t colinfo_entry_u16(const Scene& s, uint32_t base, uint32_t lx, uint32_t lz) {
  const uint32_t idx = lz * 64u + lx;
  const uint32_t word = colinfo_word(s, base + (idx >> 1));
  return (idx & 1u) == 0u ? (word & 0xFFFFu) : ((word >> 16) & 0xFFFFu);
}
struct ColInfo { bool valid; uint32_t y_vox, mat; };
inline ColInfo colinfo_decode(uint32_t e) {
  const uint32_t y8 = e & 0xFFu, m8 = (e >> 8) & 0xFFu;
  if (y8 == 255u) return ColInfo{false, 0, 0};
  return ColInfo{true, y8, m8};
}

GrassHit probe_grass_columns_xz_dda(const Scene& s, v3 ro, v3 rd, v3 inv, float t0_in, float t1_in, v3 rb,
                                    i3 origin_vox, float vs, uint32_t colinfo_base, float time_s,
                                    float strength) {  // chunk_trace.wgsl:1358-1504
  const float t0 = t0_in, t1 = t1_in;
  if (t1 <= t0) return GrassHit{false, BIG, V3s(0.0f)};
  const float eps = 1e-4f * vs;
  float t = t0 + eps;
  if (t > t1) t = t0;
  v3 p = ro + rd * t;
  int32_t lx = to_i32(std::floor((p.x - rb.x) / vs)), lz = to_i32(std::floor((p.z - rb.z) / vs));
  lx = clampi(lx, 0, 63);
  lz = clampi(lz, 0, 63);
  const int32_t stepX = rd.x > 0.0f ? 1 : -1, stepZ = rd.z > 0.0f ? 1 : -1;
  float tMaxX = BIG, tDeltaX = BIG, tMaxZ = BIG, tDeltaZ = BIG;
  if (std::fabs(rd.x) >= EPS_INV) {
    const float nextX = rb.x + (float)(stepX > 0 ? lx + 1 : lx) * vs;
    tMaxX = t + (nextX - p.x) * inv.x;
    tDeltaX = vs * std::fabs(inv.x);
  }
  if (std::fabs(rd.z) >= EPS_INV) {
    const float nextZ = rb.z + (float)(stepZ > 0 ? lz + 1 : lz) * vs;
    tMaxZ = t + (nextZ - p.z) * inv.z;
    tDeltaZ = vs * std::fabs(inv.z);
  }
  for (uint32_t it = 0; it < 64u; ++it) {
    if (t > t1) break;
    const float tNext = fmin_(fmin_(tMaxX, tMaxZ), t1);
    const ColInfo ci = colinfo_decode(colinfo_entry_u16(s, colinfo_base, (uint32_t)lx, (uint32_t)lz));
    if (ci.valid && ci.mat == MAT_GRASS) {
      const int32_t wx = origin_vox.x + lx, wy = origin_vox.y + (int32_t)ci.y_vox, wz = origin_vox.z + lz;
      const v3 id = V3((float)wx, (float)wy, (float)wz);
      const v3 cb = id * vs;
      const float sy0 = cb.y + vs;
      const float sy1 = sy0 + GRASS_LAYER_HEIGHT_VOX * vs;
      const float yA = ro.y + rd.y * t, yB = ro.y + rd.y * tNext;
      const float seg0 = fmin_(yA, yB), seg1 = fmax_(yA, yB);
      if (!(seg1 < sy0 || seg0 > sy1)) {
        const GrassHit gh = try_grass_slab_hit(s, ro, rd, t, tNext, cb, id, vs, time_s, strength);
        if (gh.hit) return gh;
      }
    }
    if (tNext >= t1) break;
    const float tStep = fmin_(tMaxX, tMaxZ);
    const float epsTie = 1e-6f * fmax_(1.0f, std::fabs(tStep));
    if (std::fabs(tMaxX - tStep) <= epsTie) { lx += stepX; tMaxX += tDeltaX; }
    if (std::fabs(tMaxZ - tStep) <= epsTie) { lz += stepZ; tMaxZ += tDeltaZ; }
    t = tStep + eps;
    if (lx < 0 || lx > 63 || lz < 0 || lz > 63) break;
    p = ro + rd * t;
  }
  return GrassHit{false, BIG, V3s(0.0f)};
}

struct TraceOpts { bool geom_only; };

inline HitGeom make_hit(uint32_t mat, float t, v3 n, v3 rb, float rs, const vxe_chunk_meta& ch, uint32_t node,
                        v3 lb, float ls) {
  HitGeom o = miss_hitgeom();
  o.hit = 1; o.t = t; o.mat = mat; o.n = n; o.root_bmin = rb; o.root_size = rs; o.node_base = ch.node_base;
  o.macro_base = ch.macro_base; o.node = node; o.leaf_bmin = lb; o.leaf_size = ls;
  return o;
}

ChunkTraceResult trace_chunk_rope_interval_nomacro(const Scene& s, v3 ro, v3 rd, v3 inv, const vxe_chunk_meta& ch,
                                                   float t_enter, float t_exit, bool use_anchor,
                                                   uint32_t anchor_key, const TraceOpts& opt) {
  // chunk_trace.wgsl:669-961
  const float vs = vs_(s);
  const v3 rb = V3((float)ch.origin[0], (float)ch.origin[1], (float)ch.origin[2]) * vs;
  const float rs = (float)s.cam->chunk_size * vs;
  const float eps_step = 1e-4f * vs;
  float tcur = fmax_(t_enter, 0.0f) + eps_step;
  AnchorNode an{false, 0, V3s(0.0f), 0.0f, INVALID};
  if (use_anchor) an = anchor_from_key(s, ch.node_base, rb, rs, anchor_key);
  const float grass_probe_max_leaf = 8.0f * vs;
  const i3 ov{ch.origin[0], ch.origin[1], ch.origin[2]};
  const float time_s = s.cam->voxel_params[1], strength = s.cam->voxel_params[2];
  bool have_leaf = false;
  LeafState leaf{};
  const uint32_t MAX_ITERS = 128u + s.cam->chunk_size * 2u;
  for (uint32_t it = 0; it < MAX_ITERS; ++it) {
    if (tcur > t_exit) break;
    const v3 p = ro + rd * tcur;
    const v3 pq = p + ray_eps_vec(rd, 1e-4f * vs);
    if (!have_leaf || !point_in_cube(pq, leaf.bmin, leaf.size)) {
      if (an.valid && point_in_cube(pq, an.bmin, an.size))
        leaf = descend_leaf_sparse(s, pq, ch.node_base, an.idx, an.bmin, an.size);
      else
        leaf = descend_leaf_sparse(s, pq, ch.node_base, 0u, rb, rs);
      const AnchorNode na = anchor_from_leaf(s, leaf, ch.node_base);
      if (na.valid && (!an.valid || na.key != an.key)) an = na;
      have_leaf = true;
    }
    const CubeSlab slab = cube_slab_inv(ro, inv, leaf.bmin, leaf.size);
    const float t_leave = slab.t_exit;
    if (leaf.mat == MAT_AIR) {
      if (!opt.geom_only) {
        const uint32_t lod = grass_lod_from_t(tcur);
        float lim = grass_probe_max_leaf;
        if (lod == 1u) lim = 4.0f * vs;
        else if (lod == 2u) lim = 2.0f * vs;
        if (leaf.size <= lim) {
          const float t0p = fmax_(t_enter, tcur - eps_step);
          const float t1p = fmin_(t_leave, t_exit);
          if (t1p >= t0p) {
            const GrassHit gh = probe_grass_columns_xz_dda(s, ro, rd, inv, t0p, t1p, rb, ov, vs, ch.colinfo_base,
                                                           time_s, strength);
            if (gh.hit) {
              const uint32_t nd = leaf.has_node ? ch.node_base + leaf.idx_local : INVALID;
              return ChunkTraceResult{make_hit(MAT_GRASS, gh.t, gh.n, rb, rs, ch, nd, leaf.bmin, leaf.size),
                                      an.valid, an.key};
            }
          }
        }
      }
      const ExitFaceRes ex = exit_face_from_slab_safe(rd, slab);
      tcur = fmax_(t_leave, tcur) + eps_step;
      if (tcur > t_exit) break;
      if (ex.amb != 0u) { have_leaf = false; continue; }
      const uint32_t face = ex.face;
      const v3 pn = ro + rd * tcur;
      const v3 pqn = pn + ray_eps_vec(rd, 1e-4f * vs);
      if (leaf.has_node) {
        const uint32_t nidx = rope_face(s, ch.node_base + leaf.idx_local, face);
        if (nidx == INVALID) { have_leaf = false; continue; }
        const uint32_t nk = node_at(s, ch.node_base, nidx).key;
        const v4 c = node_cube_from_key(rb, rs, nk);
        leaf = descend_leaf_sparse(s, pqn, ch.node_base, nidx, V3(c.x, c.y, c.z), c.w);
        const AnchorNode na = anchor_from_leaf(s, leaf, ch.node_base);
        if (na.valid && (!an.valid || na.key != an.key)) an = na;
        have_leaf = true;
        continue;
      }
      if (leaf.has_anchor) {
        if (point_in_cube(pqn, leaf.anchor_bmin, leaf.anchor_size)) {
          leaf = descend_leaf_sparse(s, pqn, ch.node_base, leaf.anchor_idx, leaf.anchor_bmin, leaf.anchor_size);
          have_leaf = true;
          continue;
        }
        const uint32_t nidx2 = rope_face(s, ch.node_base + leaf.anchor_idx, face);
        if (nidx2 == INVALID) { have_leaf = false; continue; }
        const uint32_t nk2 = node_at(s, ch.node_base, nidx2).key;
        const v4 c2 = node_cube_from_key(rb, rs, nk2);
        leaf = descend_leaf_sparse(s, pqn, ch.node_base, nidx2, V3(c2.x, c2.y, c2.z), c2.w);
        const AnchorNode na = anchor_from_leaf(s, leaf, ch.node_base);
        if (na.valid && (!an.valid || na.key != an.key)) an = na;
        have_leaf = true;
        continue;
      }
      have_leaf = false;
      continue;
    }
    if (leaf.mat == MAT_LEAF && !opt.geom_only) {
      const float tmin_iter = fmax_(t_enter, tcur - eps_step);
      const BoxHit h2 = leaf_displaced_cube_hit(s, ro, rd, leaf.bmin, leaf.size, time_s, strength, tmin_iter, t_exit);
      if (h2.hit)
        return ChunkTraceResult{make_hit(MAT_LEAF, h2.t, h2.n, rb, rs, ch, ch.node_base + leaf.idx_local, leaf.bmin,
                                         leaf.size),
                                an.valid, an.key};
      tcur = fmax_(t_leave, tcur) + eps_step;
      have_leaf = false;
      continue;
    }
    const float tmin_iter = fmax_(t_enter, tcur - eps_step);
    const BoxHit bh = cube_hit_normal_from_slab(rd, slab, tmin_iter, t_exit);
    if (bh.hit) {
      const uint32_t nd = ch.node_base + leaf.idx_local;
      if (!opt.geom_only && leaf.mat == MAT_GRASS) {
        const v3 hp = ro + rd * bh.t;
        GrassCell cell = pick_grass_cell_in_chunk_with_bias(hp, bh.n, rb, ov, vs, (int32_t)s.cam->chunk_size);
        if (ch.colinfo_base != INVALID) {
          int32_t lx = to_i32(std::floor((hp.x - rb.x) / vs)), lz = to_i32(std::floor((hp.z - rb.z) / vs));
          lx = clampi(lx, 0, 63);
          lz = clampi(lz, 0, 63);
          const ColInfo ci = colinfo_decode(colinfo_entry_u16(s, ch.colinfo_base, (uint32_t)lx, (uint32_t)lz));
          if (ci.valid && ci.mat == MAT_GRASS) {
            const v3 id = V3((float)(ov.x + lx), (float)(ov.y + (int32_t)ci.y_vox), (float)(ov.z + lz));
            cell = GrassCell{id * vs, id};
          }
        }
        const float pad = (GRASS_LAYER_HEIGHT_VOX + 1.0f) * vs;
        const float tmn = fmax_(t_enter, bh.t - 0.01f * vs);
        const float tmx = fmin_(bh.t + pad, t_exit + pad);
        const GrassHit gh = try_grass_slab_hit(s, ro, rd, tmn, tmx, cell.bmin_m, cell.id_vox, vs, time_s, strength);
        if (gh.hit)
          return ChunkTraceResult{make_hit(MAT_GRASS, gh.t, gh.n, rb, rs, ch, nd, leaf.bmin, leaf.size), an.valid,
                                  an.key};
      }
      return ChunkTraceResult{make_hit(leaf.mat, bh.t, bh.n, rb, rs, ch, nd, leaf.bmin, leaf.size), an.valid, an.key};
    }
    tcur = fmax_(t_leave, tcur) + eps_step;
    have_leaf = false;
  }
  return ChunkTraceResult{miss_hitgeom(), an.valid, an.key};
}

ChunkTraceResult trace_chunk_interval_stream_macro(const Scene& s, v3 ro, v3 rd, v3 inv, const vxe_chunk_meta& ch,
                                                   float t0_in, float t1_in, bool use_anchor, uint32_t anchor_key_in,
                                                   const TraceOpts& opt) {  // chunk_trace.wgsl:592-667
  const float vs = vs_(s);
  const v3 rb = V3((float)ch.origin[0], (float)ch.origin[1], (float)ch.origin[2]) * vs;
  const float rs = (float)s.cam->chunk_size * vs;
  const float eps_step = 1e-4f * vs;
  float tcur = fmax_(t0_in, 0.0f) + eps_step;
  const float t_end = t1_in;
  uint32_t anchor_key = anchor_key_in;
  bool anchor_valid = use_anchor;
  if (ch.macro_base == INVALID)
    return trace_chunk_rope_interval_nomacro(s, ro, rd, inv, ch, tcur, t_end, anchor_valid, anchor_key, opt);
  MacroDDAState ms = macro_dda_init(ro, rd, inv, tcur, rb, rs, ch.macro_base);
  if (!ms.enabled)
    return trace_chunk_rope_interval_nomacro(s, ro, rd, inv, ch, tcur, t_end, anchor_valid, anchor_key, opt);
  for (uint32_t i = 0; i < 128u; ++i) {
    if (tcur >= t_end) break;
    macro_dda_sync(ms, tcur);
    const MacroStep st = macro_dda_current(s, ms, ch.macro_base);
    if (!st.valid) break;
    const float t_cell_exit = fmin_(st.t_exit, t_end);
    if (st.empty) {
      tcur = t_cell_exit + eps_step;
      if (ms.enabled && tcur >= st.t_exit) macro_dda_step(ms);
      continue;
    }
    const ChunkTraceResult h =
        trace_chunk_rope_interval_nomacro(s, ro, rd, inv, ch, tcur, t_cell_exit, anchor_valid, anchor_key, opt);
    if (h.hit.hit != 0u) return h;
    anchor_valid = h.anchor_valid;
    anchor_key = h.anchor_key;
    tcur = t_cell_exit + eps_step;
    if (ms.enabled && tcur >= st.t_exit) macro_dda_step(ms);
  }
  return ChunkTraceResult{miss_hitgeom(), anchor_valid, anchor_key};
}

struct VoxTraceResult {
  bool in_grid;
  HitGeom best;
  float t_exit;
  bool anchor_valid;
  uint32_t anchor_key;
  i3 anchor_chunk;
};

struct TileList {
  uint32_t count;  // raw count after atomics (may exceed 192)
  uint32_t slots[MAX_TILE_CHUNKS];
  float enter[MAX_TILE_CHUNKS];
};

void tile_add_candidate(const Scene& s, TileList& tl, uint32_t slot, float cell_enter) {  // chunk_trace.wgsl:1007-1026
  if (slot < s.cam->chunk_count) {
    if (chunk_at(s, slot).macro_empty != 0u) return;
  }
  for (uint32_t i = 0; i < tl.count && i < MAX_TILE_CHUNKS; ++i) {
    if (tl.slots[i] == slot) {
      tl.enter[i] = fmin_(tl.enter[i], cell_enter);
      return;
    }
  }
  const uint32_t idx = tl.count++;
  if (idx < MAX_TILE_CHUNKS) {
    tl.slots[idx] = slot;
    tl.enter[idx] = cell_enter;
  }
}

// Visits the chunk-grid cells crossed by a ray (chunk_trace.wgsl:1028-1151).
template <class F>
void chunk_grid_dda(const Scene& s, v3 ro, v3 rd, float t_min, float t_max, F&& visit) {
  if (s.cam->chunk_count == 0u) return;
  const float vsz = vs_(s);
  const float cs = (float)s.cam->chunk_size * vsz;
  const int32_t* go = s.cam->grid_origin_chunk;
  const uint32_t* gd = s.cam->grid_dims;
  const v3 gb0 = V3((float)go[0], (float)go[1], (float)go[2]) * cs;
  const v3 gb1 = gb0 + V3((float)gd[0], (float)gd[1], (float)gd[2]) * cs;
  const v2 rtg = intersect_aabb(ro, rd, gb0, gb1);
  const float t_enter = fmax_(fmax_(rtg.x, 0.0f), t_min);
  const float t_exit = fmin_(fmin_(rtg.y, FOG_MAX_DIST), t_max);
  if (t_exit < t_enter) return;
  const float start_t = t_enter + PRIMARY_NUDGE_VOXEL_FRAC * vsz;
  const v3 p0 = ro + rd * start_t;
  const i3 c = chunk_coord_from_pos(p0, cs);
  const int32_t nx = (int32_t)gd[0], ny = (int32_t)gd[1], nz = (int32_t)gd[2];
  int32_t lcx = c.x - go[0], lcy = c.y - go[1], lcz = c.z - go[2];
  if (lcx < 0 || lcy < 0 || lcz < 0 || lcx >= nx || lcy >= ny || lcz >= nz) return;
  const int32_t sy = nx, sz = nx * ny;
  int32_t idx = (lcz * ny + lcy) * nx + lcx;
  float t_local = 0.0f;
  const float t_exit_local = fmax_(t_exit - start_t, 0.0f);
  const v3 inv = safe_inv3(rd);
  const int32_t stx = rd.x > 0.0f ? 1 : -1, sty = rd.y > 0.0f ? 1 : -1, stz = rd.z > 0.0f ? 1 : -1;
  const float bx = rd.x > 0.0f ? (float)(c.x + 1) * cs : (float)c.x * cs;
  const float by = rd.y > 0.0f ? (float)(c.y + 1) * cs : (float)c.y * cs;
  const float bz = rd.z > 0.0f ? (float)(c.z + 1) * cs : (float)c.z * cs;
  float tMaxX = (bx - p0.x) * inv.x, tMaxY = (by - p0.y) * inv.y, tMaxZ = (bz - p0.z) * inv.z;
  const float tDX = std::fabs(cs * inv.x), tDY = std::fabs(cs * inv.y), tDZ = std::fabs(cs * inv.z);
  if (std::fabs(rd.x) < EPS_INV) tMaxX = BIG;
  if (std::fabs(rd.y) < EPS_INV) tMaxY = BIG;
  if (std::fabs(rd.z) < EPS_INV) tMaxZ = BIG;
  const int32_t dix = rd.x > 0.0f ? 1 : -1, diy = rd.y > 0.0f ? sy : -sy, diz = rd.z > 0.0f ? sz : -sz;
  int32_t rx = 0, ry = 0, rz = 0;
  if (std::fabs(rd.x) >= EPS_INV) rx = stx > 0 ? (nx - 1 - lcx) : lcx;
  if (std::fabs(rd.y) >= EPS_INV) ry = sty > 0 ? (ny - 1 - lcy) : lcy;
  if (std::fabs(rd.z) >= EPS_INV) rz = stz > 0 ? (nz - 1 - lcz) : lcz;
  const uint32_t max_steps = std::min((uint32_t)(rx + ry + rz) + 1u, 512u);
  for (uint32_t st = 0; st < max_steps; ++st) {
    if (t_local > t_exit_local) break;
    const uint32_t slot = grid_at(s, (uint32_t)idx);
    if (slot != INVALID && slot < s.cam->chunk_count) {
      if (visit(slot, start_t + t_local)) return;
    }
    const float tn = fmin_(tMaxX, fmin_(tMaxY, tMaxZ));
    const float e = 1e-6f * fmax_(1.0f, std::fabs(tn));
    if (std::fabs(tMaxX - tn) <= e) { lcx += stx; idx += dix; tMaxX += tDX; }
    if (std::fabs(tMaxY - tn) <= e) { lcy += sty; idx += diy; tMaxY += tDY; }
    if (std::fabs(tMaxZ - tn) <= e) { lcz += stz; idx += diz; tMaxZ += tDZ; }
    t_local = tn;
    if (lcx < 0 || lcy < 0 || lcz < 0 || lcx >= nx || lcy >= ny || lcz >= nz) break;
  }
}

void tile_sort_candidates_by_enter(TileList& tl, uint32_t count) {  // chunk_trace.wgsl:1153-1175
  if (count <= 1u) return;
  const uint32_t limit = std::min(count, PRIMARY_MAX_TILE_CHUNKS);
  if (limit <= 1u) return;
  for (uint32_t i = 0; i + 1u < limit; ++i) {
    uint32_t mi = i;
    float mt = tl.enter[i];
    for (uint32_t j = i + 1u; j < limit; ++j)
      if (tl.enter[j] < mt) { mt = tl.enter[j]; mi = j; }
    if (mi != i) {
      std::swap(tl.slots[i], tl.slots[mi]);
      std::swap(tl.enter[i], tl.enter[mi]);
    }
  }
}

// The per-workgroup candidate gather of main_primary (ray_main.wgsl:179-197).
uint32_t build_tile(const Scene& s, uint32_t wgx, uint32_t wgy, TileList& tl) {
  tl.count = 0;
  if (s.cam->chunk_count != 0u) {
    const v2 base = V2((float)(wgx * TILE_SIZE), (float)(wgy * TILE_SIZE));
    const v3 ro = cam_pos(s);
    auto add = [&](uint32_t slot, float te) { tile_add_candidate(s, tl, slot, te); return false; };
    chunk_grid_dda(s, ro, ray_dir_from_pixel(s, base + V2(4.5f, 4.5f)), 0.0f, FOG_MAX_DIST, add);
    chunk_grid_dda(s, ro, ray_dir_from_pixel(s, base + V2(1.5f, 1.5f)), 0.0f, FOG_MAX_DIST, add);
  }
  const uint32_t raw = std::min(tl.count, MAX_TILE_CHUNKS);
  tile_sort_candidates_by_enter(tl, raw);
  return std::min(raw, PRIMARY_MAX_TILE_CHUNKS);
}

inline bool chunk_coords_neighbor(i3 a, i3 b) {  // chunk_trace.wgsl:1000-1005
  return std::abs(a.x - b.x) <= 1 && std::abs(a.y - b.y) <= 1 && std::abs(a.z - b.z) <= 1;
}

bool chunk_heightfield_early_skip(const Scene& s, v3 ro, v3 rd, float t_enter, float t_exit, const vxe_chunk_meta& ch,
                                  float vs) {  // chunk_trace.wgsl:1310-1352
  if (ch.colinfo_base == INVALID) return false;
  if (rd.y >= 0.0f) return false;
  const float y0 = ro.y + rd.y * t_enter, y1 = ro.y + rd.y * t_exit;
  const float seg_y_min = fmin_(y0, y1);
  const v3 rb = V3((float)ch.origin[0], (float)ch.origin[1], (float)ch.origin[2]) * vs;
  const float seg_len = fmax_(t_exit - t_enter, 0.0f);
  const float dt = seg_len * (1.0f / 3.0f);
  for (uint32_t i = 0; i < 4u; ++i) {
    const float t = t_enter + (float)i * dt;
    const v3 p = ro + rd * t;
    const int32_t lx = clampi(to_i32(std::floor((p.x - rb.x) / vs)), 0, 63);
    const int32_t lz = clampi(to_i32(std::floor((p.z - rb.z) / vs)), 0, 63);
    const ColInfo ci = colinfo_decode(colinfo_entry_u16(s, ch.colinfo_base, (uint32_t)lx, (uint32_t)lz));
    if (!ci.valid) continue;
    const float top_y = rb.y + ((float)ci.y_vox + 1.0f) * vs;
    if (seg_y_min <= top_y + 1e-3f * vs) return false;
  }
  return true;
}

VoxTraceResult trace_scene_voxels_candidates(const Scene& s, const TileList& tl, v3 ro, v3 rd, float t_min,
                                             float t_max, bool anchor_valid_in, i3 anchor_chunk_in,
                                             uint32_t anchor_key_in, uint32_t cand_count) {
  // chunk_trace.wgsl:1177-1265
  VoxTraceResult none{false, miss_hitgeom(), 0.0f, false, INVALID, i3{0, 0, 0}};
  if (s.cam->chunk_count == 0u) return none;
  const float vsz = vs_(s);
  const float cs = (float)s.cam->chunk_size * vsz;
  const int32_t* go = s.cam->grid_origin_chunk;
  const uint32_t* gd = s.cam->grid_dims;
  const v3 gb0 = V3((float)go[0], (float)go[1], (float)go[2]) * cs;
  const v3 gb1 = gb0 + V3((float)gd[0], (float)gd[1], (float)gd[2]) * cs;
  const v2 rtg = intersect_aabb(ro, rd, gb0, gb1);
  const float t_enter = fmax_(fmax_(rtg.x, 0.0f), t_min);
  const float t_exit = fmin_(fmin_(rtg.y, FOG_MAX_DIST), t_max);
  if (t_exit < t_enter) return none;
  HitGeom best = miss_hitgeom();
  bool bav = false;
  uint32_t bak = INVALID;
  i3 bac{0, 0, 0};
  const v3 inv = safe_inv3(rd);
  const float rs = (float)s.cam->chunk_size * vsz;
  const uint32_t maxc = std::min(cand_count, MAX_TILE_CHUNKS);
  const TraceOpts opt{false};
  for (uint32_t i = 0; i < maxc; ++i) {
    const uint32_t slot = tl.slots[i];
    if (slot == INVALID || slot >= s.cam->chunk_count) continue;
    const vxe_chunk_meta ch = chunk_at(s, slot);
    if (ch.macro_empty != 0u) continue;
    const v3 rb = V3((float)ch.origin[0], (float)ch.origin[1], (float)ch.origin[2]) * vsz;
    const v2 rt = intersect_aabb(ro, rd, rb, rb + V3s(rs));
    const float ce = fmax_(rt.x, t_enter), cx = fmin_(rt.y, t_exit);
    if (cx < ce) continue;
    if (best.hit != 0u && ce >= best.t) continue;
    if (chunk_heightfield_early_skip(s, ro, rd, ce, cx, ch, vsz)) continue;
    const int32_t csz = (int32_t)s.cam->chunk_size;
    const i3 cc{ch.origin[0] / csz, ch.origin[1] / csz, ch.origin[2] / csz};
    const bool ua = anchor_valid_in && chunk_coords_neighbor(cc, anchor_chunk_in);
    const uint32_t aku = ua ? anchor_key_in : INVALID;
    const ChunkTraceResult h = trace_chunk_interval_stream_macro(s, ro, rd, inv, ch, ce, cx, ua, aku, opt);
    if (h.hit.hit != 0u && h.hit.t < best.t) {
      best = h.hit;
      bav = h.anchor_valid;
      bak = h.anchor_key;
      bac = cc;
    }
  }
  return VoxTraceResult{true, best, t_exit, bav, bak, bac};
}

// ---------------------------------------------------------------------------
// clipmap.wgsl
// ---------------------------------------------------------------------------
inline int32_t imod(int32_t a, int32_t m) {
  int32_t r = a % m;
  if (r < 0) r += m;
  return r;
}
inline v2 clip_st(const Scene& s, v2 xz, uint32_t level) {  // clipmap.wgsl:317-327
  const float* p = s.clip->level[level];
  const float cell = fmax_(p[2], 1e-6f);
  const v2 uv = (xz - V2(p[0], p[1])) / V2(cell, cell);
  return uv - V2(0.5f, 0.5f);
}
struct HSample { float h; bool ok; };
HSample clip_height_at_level_ok(const Scene& s, v2 xz, uint32_t level) {  // clipmap.wgsl:34-52
  const int32_t res = std::max((int32_t)s.clip->res, 1);
  const v2 st = clip_st(s, xz, level);
  const int32_t ix = to_i32(std::floor(st.x)), iz = to_i32(std::floor(st.y));
  if (ix < 0 || iz < 0 || ix >= res || iz >= res) return HSample{0.0f, false};
  const int32_t sx = imod(ix + (int32_t)s.clip->offset[level][0], res);
  const int32_t sz = imod(iz + (int32_t)s.clip->offset[level][1], res);
  return HSample{clip_texel(s, sx, sz, level), true};
}
float clip_height_texel(const Scene& s, uint32_t level, int32_t ix, int32_t iz) {  // clipmap.wgsl:55-67
  const int32_t res = std::max((int32_t)s.clip->res, 1);
  if (ix < 0 || iz < 0 || ix >= res || iz >= res) return -BIG;
  const int32_t sx = imod(ix + (int32_t)s.clip->offset[level][0], res);
  const int32_t sz = imod(iz + (int32_t)s.clip->offset[level][1], res);
  return clip_texel(s, sx, sz, level);
}
float clip_height_at_level(const Scene& s, v2 xz, uint32_t level) {  // clipmap.wgsl:71-108
  const int32_t res = std::max((int32_t)s.clip->res, 1);
  const float* p = s.clip->level[level];
  const float cell = fmax_(p[2], 1e-6f);
  const v2 uv = (xz - V2(p[0], p[1])) / V2(cell, cell);
  const v2 st = uv - V2(0.5f, 0.5f);
  const int32_t ix0 = to_i32(std::floor(st.x)), iz0 = to_i32(std::floor(st.y));
  const int32_t ix1 = ix0 + 1, iz1 = iz0 + 1;
  if (ix0 < 0 || iz0 < 0 || ix1 >= res || iz1 >= res) return -BIG;
  const float fx = fract(st.x), fz = fract(st.y);
  const float h00 = clip_height_texel(s, level, ix0, iz0), h10 = clip_height_texel(s, level, ix1, iz0);
  const float h01 = clip_height_texel(s, level, ix0, iz1), h11 = clip_height_texel(s, level, ix1, iz1);
  const float lim = -0.5f * BIG;
  if (h00 <= lim || h10 <= lim || h01 <= lim || h11 <= lim) return -BIG;
  return mixf(mixf(h00, h10, fx), mixf(h01, h11, fx), fz);
}
float clip_height_at_level_nearest(const Scene& s, v2 xz, uint32_t level) {  // clipmap.wgsl:110-130
  const int32_t res = std::max((int32_t)s.clip->res, 1);
  const float* p = s.clip->level[level];
  const float cell = fmax_(p[2], 1e-6f);
  const v2 uv = (xz - V2(p[0], p[1])) / V2(cell, cell);
  const v2 st = uv - V2(0.5f, 0.5f);
  const int32_t ix = to_i32(std::floor(st.x + 0.5f)), iz = to_i32(std::floor(st.y + 0.5f));
  const int32_t sx = imod(ix + (int32_t)s.clip->offset[level][0], res);
  const int32_t sz = imod(iz + (int32_t)s.clip->offset[level][1], res);
  return clip_texel(s, sx, sz, level);
}
v3 clip_normal_at_level_2tap(const Scene& s, v2 xz, uint32_t level) {  // clipmap.wgsl:132-147
  const float cell = s.clip->level[level][2];
  const HSample h0 = clip_height_at_level_ok(s, xz, level);
  const HSample hx = clip_height_at_level_ok(s, xz + V2(cell, 0.0f), level);
  const HSample hz = clip_height_at_level_ok(s, xz + V2(0.0f, cell), level);
  if (!h0.ok || !hx.ok || !hz.ok) return V3(0.0f, 1.0f, 0.0f);
  const float dhx = (hx.h - h0.h) / fmax_(cell, 1e-4f), dhz = (hz.h - h0.h) / fmax_(cell, 1e-4f);
  return normalize(V3(-dhx, 1.0f, -dhz));
}
bool clip_level_contains(const Scene& s, v2 xz, uint32_t level, int32_t guard) {  // clipmap.wgsl:277-292
  const int32_t res = std::max((int32_t)s.clip->res, 1);
  const v2 st = clip_st(s, xz, level);
  const int32_t ix0 = to_i32(std::floor(st.x)), iz0 = to_i32(std::floor(st.y));
  return ix0 >= guard && iz0 >= guard && ix0 + 1 < res - guard && iz0 + 1 < res - guard;
}
uint32_t clip_best_level(const Scene& s, v2 xz, int32_t guard) {  // clipmap.wgsl:295-301
  const uint32_t n = std::min(s.clip->levels, CLIP_LEVELS_MAX);
  for (uint32_t i = 0; i < n; ++i)
    if (clip_level_contains(s, xz, i, guard)) return i;
  return std::max(n, 1u) - 1u;
}
uint32_t clip_ensure_contains(const Scene& s, v2 xz, uint32_t lvl_in, int32_t guard) {  // clipmap.wgsl:304-315
  const uint32_t n = std::min(s.clip->levels, CLIP_LEVELS_MAX);
  if (n == 0u) return 0u;
  uint32_t lvl = std::min(lvl_in, n - 1u);
  for (;;) {
    if (clip_level_contains(s, xz, lvl, guard) || lvl >= n - 1u) break;
    lvl += 1u;
  }
  return lvl;
}
struct ClipHit { bool hit; float t; v3 n; uint32_t mat; };

ClipHit clip_trace_heightfield(const Scene& s, v3 ro, v3 rd, float t_min, float t_max) {  // clipmap.wgsl:156-243
  const ClipHit miss{false, BIG, V3s(0.0f), MAT_AIR};
  if (s.clip->levels == 0u) return miss;
  if (rd.y >= -1e-4f) return miss;
  const int32_t guard = 2;
  float t = fmax_(t_min, 0.0f);
  v3 p = ro + rd * t;
  uint32_t lvl = clip_best_level(s, V2(p.x, p.z), guard);
  const float h0 = clip_height_at_level_nearest(s, V2(p.x, p.z), lvl);
  if (h0 <= -0.5f * BIG) return miss;
  float s_prev = p.y - h0;
  float t_prev = t;
  for (uint32_t i = 0; i < HF_MAX_STEPS; ++i) {
    if (t > t_max) break;
    p = ro + rd * t;
    lvl = clip_ensure_contains(s, V2(p.x, p.z), lvl, guard);
    const float h = clip_height_at_level_nearest(s, V2(p.x, p.z), lvl);
    if (h <= -0.5f * BIG) return miss;
    const float sd = p.y - h;
    if (sd <= 0.0f && s_prev > 0.0f) {
      float a = t_prev, b = t;
      for (uint32_t k = 0; k < HF_BISECT; ++k) {
        const float m = 0.5f * (a + b);
        const v3 pm = ro + rd * m;
        const float hm = clip_height_at_level(s, V2(pm.x, pm.z), lvl);
        if (hm <= -0.5f * BIG) return miss;
        if (pm.y - hm > 0.0f) a = m; else b = m;
      }
      const float th = 0.5f * (a + b);
      const v3 ph = ro + rd * th;
      return ClipHit{true, th, clip_normal_at_level_2tap(s, V2(ph.x, ph.z), lvl), MAT_GRASS};
    }
    s_prev = sd;
    t_prev = t;
    const float vy = fmax_(-rd.y, 0.12f);
    const float vh = fmax_(length(V2(rd.x, rd.z)), 1e-4f);
    const float dt_y = std::fabs(sd) / vy;
    const float cell = s.clip->level[lvl][2];
    const float dt_xz = (6.0f * cell) / vh;
    float dt = fmin_(dt_y, dt_xz);
    dt = clampf(dt, 0.6f, HF_DT_MAX);
    t = t + dt;
  }
  return miss;
}

inline float material_variation_clip(v3 p, float cell, float strength) {  // clipmap.wgsl:247-250
  return (hash31(vfloor(p / cell)) - 0.5f) * strength;
}
v3 apply_material_variation_clip(v3 base, uint32_t mat, v3 hp) {  // clipmap.wgsl:252-275
  v3 c = base;
  if (mat == MAT_GRASS) {
    const float v = material_variation_clip(hp, 3.0f, 1.0f) + material_variation_clip(hp, 0.75f, 0.35f);
    c = c + V3(0.10f * v, 0.18f * v, 0.06f * v);
    c = c * (1.0f + 0.06f * v);
    c = vclamp(c, V3s(0.0f), V3s(2.0f));
  } else if (mat == MAT_DIRT) {
    const float v = material_variation_clip(hp, 1.5f, 0.8f);
    c = c + V3(0.05f * v, 0.03f * v, 0.01f * v);
    c = c * (1.0f + 0.08f * v);
    c = vclamp(c, V3s(0.0f), V3s(2.0f));
  } else if (mat == MAT_STONE) {
    const float v = material_variation_clip(hp, 2.0f, 0.9f);
    c = c * (1.0f + 0.10f * v);
    c = vclamp(c, V3s(0.0f), V3s(2.0f));
  }
  return c;
}

// ---------------------------------------------------------------------------
// phase.wgsl / fog.wgsl / sky.wgsl / clouds.wgsl
// ---------------------------------------------------------------------------
inline float phase_mie(float costh) {  // phase.wgsl:5-10
  const float g = PHASE_G, gg = g * g;
  const float denom = powf_(1.0f + gg - 2.0f * g * costh, 1.5f);
  return INV_4PI * (1.0f - gg) / fmax_(denom, 1e-3f);
}
inline float phase_blended(float costh) { return mixf(INV_4PI, phase_mie(costh), PHASE_MIE_W); }

inline v3 fog_color_from_sky(v3 rd, v3 sky) {  // fog.wgsl:5-12
  const float up = clampf(rd.y * 0.5f + 0.5f, 0.0f, 1.0f);
  return vmix(FOG_COLOR_GROUND, vmin(sky, V3s(0.45f)), FOG_COLOR_SKY_BLEND * up);
}
inline v3 fog_inscatter(v3 rd, v3 fogc) {  // fog.wgsl:15-19
  const float mu = clampf(dot(rd, SUN_DIR), 0.0f, 1.0f);
  const float ss = powf_(mu, 8.0f);
  return fogc + SUN_COLOR * (0.35f * ss);
}
inline float fog_density_primary(const Scene& s) { return fmax_(s.cam->voxel_params[3] * FOG_PRIMARY_SCALE, 0.0f); }
inline float fog_density_godray(const Scene& s) { return fmax_(s.cam->voxel_params[3] * FOG_GODRAY_SCALE, 0.0f); }
float fog_optical_depth_with_base(float base, v3 ro, v3 rd, float t) {  // fog.wgsl:31-45
  if (base <= 0.0f) return 0.0f;
  const float k = FOG_HEIGHT_FALLOFF, y0 = ro.y, dy = rd.y;
  if (std::fabs(dy) < 1e-4f) return base * expf_(-k * y0) * t;
  const float a = expf_(-k * y0);
  const float b = expf_(-k * (y0 + dy * t));
  return base * (a - b) / (k * dy);
}
v3 apply_fog(const Scene& s, v3 surface, v3 ro, v3 rd, float t_scene, v3 sky) {  // fog.wgsl:57-71
  const float od = fmax_(fog_optical_depth_with_base(fog_density_primary(s), ro, rd, t_scene), 0.0f);
  const float T = expf_(-od);
  const v3 ins = fog_inscatter(rd, fog_color_from_sky(rd, sky));
  return surface * T + ins * (1.0f - T);
}

v3 sky_bg(v3 rd) {  // sky.wgsl:5-25
  const float t0 = smooth(-0.10f, 0.85f, rd.y);
  v3 col = vmix(V3(0.05f, 0.08f, 0.12f), V3(0.55f, 0.75f, 0.95f), t0);
  const float th = 1.0f - smooth(-0.20f, 0.18f, std::fabs(rd.y));
  col = col + V3(0.80f, 0.75f, 0.70f) * (0.12f * th);
  const float tz = smooth(0.15f, 1.00f, rd.y);
  col = col + V3(0.20f, 0.35f, 0.60f) * (0.05f * tz);
  return col * SKY_EXPOSURE;
}
v3 sky_sun(v3 rd) {  // sky.wgsl:27-41
  const float mu = clampf(dot(rd, SUN_DIR), -1.0f, 1.0f);
  const float mu_inner = cosf_(0.009f);
  const float mu_outer = cosf_(0.009f + 0.004f);
  const float disc = smooth(mu_outer, mu_inner, mu);
  const float glow = smooth(0.70f, 0.98f, mu);
  const float halo = 0.03f * expf_(-2500.0f * fmax_(0.0f, 1.0f - mu));
  return SUN_COLOR * SUN_INTENSITY * (disc + halo + 0.04f * glow);
}

inline float cloud_height01(float y) {  // clouds.wgsl:5-15
  const float t = clampf((y - CLOUD_BASE_H) / fmax_(CLOUD_TOP_H - CLOUD_BASE_H, 1e-3f), 0.0f, 1.0f);
  return smooth(0.00f, 0.12f, t) * (1.0f - smooth(0.78f, 1.00f, t));
}
inline float cloud_coverage_at_xz(v2 xz, float time_s) {  // clouds.wgsl:18-31
  const v2 uv = xz * CLOUD_UV_SCALE + V2(CLOUD_WIND_X, CLOUD_WIND_Y) * time_s;
  const float field = 0.65f * fbm(uv) + 0.35f * fbm(uv * 2.3f + V2(13.2f, 7.1f));
  return smooth(CLOUD_COVERAGE, CLOUD_COVERAGE + CLOUD_SOFTNESS, field);
}
float cloud_density(v3 p, float time_s) {  // clouds.wgsl:34-65
  if (p.y <= CLOUD_BASE_H || p.y >= CLOUD_TOP_H) return 0.0f;
  const float h = cloud_height01(p.y);
  if (h <= 0.0f) return 0.0f;
  const float cov = cloud_coverage_at_xz(V2(p.x, p.z), time_s);
  if (cov <= 0.001f) return 0.0f;
  v2 uv = V2(p.x, p.z) * CLOUD_UV_SCALE + V2(CLOUD_WIND_X, CLOUD_WIND_Y) * time_s;
  uv = uv + V2(0.003f * p.y, 0.003f * p.y);
  const float base = fbm(uv * 1.2f);
  const float det = fbm(uv * 3.7f + V2(0.11f * p.y, -0.07f * p.y));
  float d = mixf(base, det, CLOUD_DETAIL_W);
  d = smooth(0.45f, 0.95f, d);
  d = powf_(d, CLOUD_PUFF_POW);
  d = d * cov;
  d = d * h;
  return clampf(d, 0.0f, 1.0f);
}
float cloud_light_transmittance(v3 p, float time_s) {  // clouds.wgsl:68-90
  const float tmax = (CLOUD_TOP_H - p.y) / fmax_(SUN_DIR_Y, 1e-3f);
  if (tmax <= 0.0f) return 1.0f;
  const float dt = tmax / (float)CLOUD_STEPS_LIGHT;
  float od = 0.0f;
  for (uint32_t i = 0; i < CLOUD_STEPS_LIGHT; ++i) {
    const float ti = ((float)i + 0.5f) * dt;
    od += cloud_density(p + SUN_DIR * ti, time_s) * dt;
  }
  return expf_(-CLOUD_DENSITY * od * CLOUD_SHADOW_ABSORB);
}
float cloud_sun_transmittance_fast(const Scene& s, v3 p, v3 sd) {  // clouds.wgsl:134-165
  if (sd.y <= 0.01f) return 1.0f;
  const float t0 = (CLOUD_BASE_H - p.y) / sd.y, t1 = (CLOUD_TOP_H - p.y) / sd.y;
  const float ta = fmin_(t0, t1), tb = fmax_(t0, t1);
  const float ts = fmax_(ta, 0.0f), te = fmax_(tb, 0.0f);
  if (te <= ts) return 1.0f;
  const float time_s = s.cam->voxel_params[1];
  const float dt = (te - ts) / 2.0f;
  float od = 0.0f;
  for (uint32_t i = 0; i < 2u; ++i) {
    const float ti = ts + ((float)i + 0.5f) * dt;
    od += cloud_density(p + sd * ti, time_s) * dt;
  }
  return expf_(-CLOUD_DENSITY * od * CLOUD_SHADOW_ABSORB);
}
float cloud_density_godray(v3 p, float time_s) {  // clouds.wgsl:167-182
  if (p.y <= CLOUD_BASE_H || p.y >= CLOUD_TOP_H) return 0.0f;
  const float h = cloud_height01(p.y);
  if (h <= 0.0f) return 0.0f;
  const v2 uv = V2(p.x, p.z) * CLOUD_UV_SCALE + V2(CLOUD_WIND_X, CLOUD_WIND_Y) * time_s;
  const float n0 = value_noise(uv);
  const float n1 = value_noise(uv * 2.0f + V2(17.0f, 9.0f));
  const float field = 0.70f * n0 + 0.30f * n1;
  return smooth(CLOUD_COVERAGE, CLOUD_COVERAGE + CLOUD_SOFTNESS, field) * h;
}
float cloud_sun_transmittance_godray(const Scene& s, v3 p, v3 sd) {  // clouds.wgsl:184-214
  if (sd.y <= 0.01f) return 1.0f;
  const float t0 = (CLOUD_BASE_H - p.y) / sd.y, t1 = (CLOUD_TOP_H - p.y) / sd.y;
  const float ta = fmin_(t0, t1), tb = fmax_(t0, t1);
  if (tb <= 0.0f) return 1.0f;
  const float ts = fmax_(ta, 0.0f), te = tb;
  if (te <= ts) return 1.0f;
  const float time_s = s.cam->voxel_params[1];
  const float tm = ts + 0.5f * (te - ts);
  const float dens = cloud_density_godray(p + sd * tm, time_s);
  return expf_(-CLOUD_DENSITY * dens * (te - ts) * CLOUD_SHADOW_ABSORB);
}

v3 sky_color(const Scene& s, v3 rd) {  // sky.wgsl:43-137
  const v3 bg = sky_bg(rd);
  const v3 sun = sky_sun(rd);
  float T_view = 1.0f;
  v3 acc = V3s(0.0f);
  if (rd.y > 0.01f) {
    const v3 ro = cam_pos(s);
    const float time_s = s.cam->voxel_params[1];
    const float t0 = (CLOUD_BASE_H - ro.y) / rd.y, t1 = (CLOUD_TOP_H - ro.y) / rd.y;
    float te = fmin_(t0, t1);
    const float tx = fmax_(t0, t1);
    te = fmax_(te, 0.0f);
    if (tx > te) {
      const float horizon2 = clampf((rd.y - CLOUD_HORIZON_Y0) / CLOUD_HORIZON_Y1, 0.0f, 1.0f);
      const float dt = (tx - te) / (float)CLOUD_STEPS_VIEW;
      const float phase = phase_blended(dot(rd, SUN_DIR));
      for (uint32_t i = 0; i < CLOUD_STEPS_VIEW; ++i) {
        const float ti = te + ((float)i + 0.5f) * dt;
        const v3 p = ro + rd * ti;
        float dens = cloud_density(p, time_s);
        dens = dens * horizon2;
        if (dens > 1e-4f) {
          const float Tl = cloud_light_transmittance(p, time_s);
          const float toward = clampf(dot(rd, SUN_DIR), 0.0f, 1.0f);
          const float silver = powf_(toward, CLOUD_SILVER_POW) * CLOUD_SILVER_STR;
          const v3 cc = vmix(V3(0.72f, 0.74f, 0.76f), V3s(1.0f), silver);
          const float tau = CLOUD_DENSITY * dens * dt;
          const float a = 1.0f - expf_(-tau);
          const v3 scatter = cc * (SUN_COLOR * SUN_INTENSITY) * (phase * Tl);
          acc = acc + scatter * (T_view * a);
          T_view = T_view * (1.0f - a);
          if (T_view < 0.02f) break;
        }
      }
    }
  }
  v3 col = bg * T_view + acc;
  float T_sun = 1.0f;
  if (rd.y > 0.01f) {
    T_sun = powf_(clampf(T_view, 0.0f, 1.0f), CLOUD_SUN_DISC_DIM_POW);
    T_sun = fmax_(T_sun, CLOUD_SUN_DISC_DIM_FLOOR);
  }
  return col + sun * T_sun;
}

// ---------------------------------------------------------------------------
// shadows.wgsl
// ---------------------------------------------------------------------------
float trace_chunk_shadow_trans_interval(const Scene& s, v3 ro, v3 rd, const vxe_chunk_meta& ch, float t_enter,
                                        float t_exit) {  // shadows.wgsl:4-82
  const float vs = vs_(s);
  const float nudge = 0.20f * vs;
  const v3 rb = V3((float)ch.origin[0], (float)ch.origin[1], (float)ch.origin[2]) * vs;
  const float rs = (float)s.cam->chunk_size * vs;
  float tcur = fmax_(t_enter, 0.0f) + nudge;
  const v3 inv = safe_inv3(rd);
  float trans = 1.0f;
  for (uint32_t i = 0; i < VSM_STEPS; ++i) {
    if (tcur > t_exit) break;
    if (trans < MIN_TRANS) break;
    const v3 p = ro + rd * tcur;
    const v3 pq = p + ray_eps_vec(rd, 1e-4f * vs);
    const LeafQuery q = query_leaf_at(s, pq, rb, rs, ch.node_base, ch.macro_base);
    const CubeSlab slab = cube_slab_inv(ro, inv, q.bmin, q.size);
    const float t_leave = slab.t_exit;
    if (q.mat != MAT_AIR) {
      if (q.mat == MAT_LEAF) {
        const v3 center = q.bmin + V3s(0.5f * q.size);
        const float d = length(center - cam_pos(s));
        if (d < LEAF_LOD_DISP_END) {
          const BoxHit h2 = leaf_displaced_cube_hit(s, ro, rd, q.bmin, q.size, s.cam->voxel_params[1],
                                                    s.cam->voxel_params[2], tcur - nudge, t_exit);
          if (h2.hit) trans *= LEAF_LIGHT_TRANSMIT;
        } else {
          trans *= LEAF_LIGHT_TRANSMIT;
        }
        tcur = fmax_(t_leave, tcur) + nudge;
        continue;
      }
      if (q.mat == MAT_GRASS) {
        trans *= GRASS_LIGHT_TRANSMIT;
        tcur = fmax_(t_leave, tcur) + nudge;
        continue;
      }
      return 0.0f;
    }
    tcur = fmax_(t_leave, tcur) + nudge;
  }
  return trans;
}

float sun_transmittance_geom_only(const Scene& s, v3 p, v3 sd) {  // shadows.wgsl:85-186
  const float vs = vs_(s);
  const float nudge = 0.18f * vs;
  const float cs = (float)s.cam->chunk_size * vs;
  const int32_t* go = s.cam->grid_origin_chunk;
  const uint32_t* gd = s.cam->grid_dims;
  const v3 gb0 = V3((float)go[0], (float)go[1], (float)go[2]) * cs;
  const v3 gb1 = gb0 + V3((float)gd[0], (float)gd[1], (float)gd[2]) * cs;
  const float bias = fmax_(SHADOW_BIAS, 0.50f * vs);
  const v3 ro = p + sd * bias;
  const v3 rd = sd;
  const v2 rtg = intersect_aabb(ro, rd, gb0, gb1);
  const float t_enter = fmax_(rtg.x, 0.0f), t_exit = rtg.y;
  if (t_exit < t_enter) return 1.0f;
  const float start_t = t_enter + nudge;
  const v3 p0 = ro + rd * start_t;
  float t_local = 0.0f;
  const float t_exit_local = fmax_(t_exit - start_t, 0.0f);
  const i3 c = chunk_coord_from_pos(p0, cs);
  int32_t cx = c.x, cy = c.y, cz = c.z;
  const v3 inv = safe_inv3(rd);
  const int32_t stx = rd.x > 0.0f ? 1 : -1, sty = rd.y > 0.0f ? 1 : -1, stz = rd.z > 0.0f ? 1 : -1;
  const float bx = rd.x > 0.0f ? (float)(cx + 1) * cs : (float)cx * cs;
  const float by = rd.y > 0.0f ? (float)(cy + 1) * cs : (float)cy * cs;
  const float bz = rd.z > 0.0f ? (float)(cz + 1) * cs : (float)cz * cs;
  float tMaxX = (bx - p0.x) * inv.x, tMaxY = (by - p0.y) * inv.y, tMaxZ = (bz - p0.z) * inv.z;
  const float tDX = std::fabs(cs * inv.x), tDY = std::fabs(cs * inv.y), tDZ = std::fabs(cs * inv.z);
  if (std::fabs(rd.x) < EPS_INV) tMaxX = BIG;
  if (std::fabs(rd.y) < EPS_INV) tMaxY = BIG;
  if (std::fabs(rd.z) < EPS_INV) tMaxZ = BIG;
  float trans = 1.0f;
  const uint32_t max_steps = std::min((gd[0] + gd[1] + gd[2]) * 6u + 8u, 512u);
  const int32_t gx1 = go[0] + (int32_t)gd[0], gy1 = go[1] + (int32_t)gd[1], gz1 = go[2] + (int32_t)gd[2];
  for (uint32_t st = 0; st < max_steps; ++st) {
    if (t_local > t_exit_local) break;
    if (trans < MIN_TRANS) break;
    const float tn = fmin_(tMaxX, fmin_(tMaxY, tMaxZ));
    const uint32_t slot = grid_lookup_slot(s, cx, cy, cz);
    if (slot != INVALID && slot < s.cam->chunk_count) {
      const vxe_chunk_meta ch2 = chunk_at(s, slot);
      const float ce = start_t + t_local;
      const float cx2 = start_t + fmin_(tn, t_exit_local);
      trans *= trace_chunk_shadow_trans_interval(s, ro, rd, ch2, ce, cx2);
      if (trans < MIN_TRANS) break;
    }
    if (tMaxX < tMaxY) {
      if (tMaxX < tMaxZ) { cx += stx; t_local = tMaxX; tMaxX += tDX; }
      else { cz += stz; t_local = tMaxZ; tMaxZ += tDZ; }
    } else {
      if (tMaxY < tMaxZ) { cy += sty; t_local = tMaxY; tMaxY += tDY; }
      else { cz += stz; t_local = tMaxZ; tMaxZ += tDZ; }
    }
    if (cx < go[0] || cy < go[1] || cz < go[2] || cx >= gx1 || cy >= gy1 || cz >= gz1) break;
  }
  return trans;
}

// ---------------------------------------------------------------------------
// light.wgsl
// ---------------------------------------------------------------------------
inline uint32_t hash3_i32(i3 p) {  // light.wgsl:18-23
  return hash_u32(((uint32_t)p.x * 73856093u) ^ ((uint32_t)p.y * 19349663u) ^ ((uint32_t)p.z * 83492791u));
}
inline v3 rot_about_axis(v3 v, v3 axis, float ang) {  // light.wgsl:32-37
  const v3 a = normalize(axis);
  const float sn = sinf_(ang), c = cosf_(ang);
  return v * c + cross(a, v) * sn + a * dot(a, v) * (1.0f - c);
}
inline v3 sphere_dir_local(uint32_t i, uint32_t count) {  // light.wgsl:48-56
  const float fi = (float)i;
  const float cf = fmax_(1.0f, (float)count);
  const float golden = 2.399963229728653f;
  const float y = 1.0f - 2.0f * ((fi + 0.5f) / cf);
  const float r = std::sqrt(fmax_(0.0f, 1.0f - y * y));
  const float phi = golden * fi;
  return V3(cosf_(phi) * r, sinf_(phi) * r, y);
}

v4 dda_hit_light(const Scene& s, v3 p0, v3 dir, uint32_t max_steps, float vs) {  // light.wgsl:65-121
  const v3 gpos = p0 / fmax_(vs, 1e-6f);
  const v3 fl = vfloor(gpos);
  i3 cell{to_i32(fl.x), to_i32(fl.y), to_i32(fl.z)};
  const i3 step{dir.x >= 0.0f ? 1 : -1, dir.y >= 0.0f ? 1 : -1, dir.z >= 0.0f ? 1 : -1};
  const v3 nb = V3((float)(cell.x + (dir.x >= 0.0f ? 1 : 0)), (float)(cell.y + (dir.y >= 0.0f ? 1 : 0)),
                   (float)(cell.z + (dir.z >= 0.0f ? 1 : 0)));
  const v3 inv = V3(std::fabs(dir.x) > 1e-6f ? 1.0f / std::fabs(dir.x) : 1e30f,
                    std::fabs(dir.y) > 1e-6f ? 1.0f / std::fabs(dir.y) : 1e30f,
                    std::fabs(dir.z) > 1e-6f ? 1.0f / std::fabs(dir.z) : 1e30f);
  v3 tMax = V3((nb.x - gpos.x) * inv.x, (nb.y - gpos.y) * inv.y, (nb.z - gpos.z) * inv.z);
  const v3 tDelta = inv;
  for (uint32_t i = 0; i < max_steps; ++i) {
    const v3 c = V3((float)cell.x + 0.5f, (float)cell.y + 0.5f, (float)cell.z + 0.5f) * vs;
    const LeafQuery lf = query_leaf_world(s, c);
    if (lf.mat == MAT_LIGHT) return v4{c.x, c.y, c.z, 1.0f};
    if (lf.mat != MAT_AIR) return v4{0.0f, 0.0f, 0.0f, 0.0f};
    if (tMax.x < tMax.y) {
      if (tMax.x < tMax.z) { cell.x += step.x; tMax.x += tDelta.x; }
      else { cell.z += step.z; tMax.z += tDelta.z; }
    } else {
      if (tMax.y < tMax.z) { cell.y += step.y; tMax.y += tDelta.y; }
      else { cell.z += step.z; tMax.z += tDelta.z; }
    }
  }
  return v4{0.0f, 0.0f, 0.0f, 0.0f};
}

inline v3 material_emission(uint32_t m) {  // shading.wgsl:211-216
  if (m == MAT_LIGHT) return V3(1.0f, 0.95f, 0.75f) * 18.0f;
  return V3s(0.0f);
}

v3 gather_voxel_lights(const Scene& s, v3 hp, v3 n, v3 rb) {  // light.wgsl:127-211
  uint32_t hits = 0;
  const float vs = vs_(s);
  const v3 p0 = hp + n * (0.75f * vs);
  // make_tbn (light.wgsl:25-30): columns t, b, n
  const v3 up = std::fabs(n.y) > 0.9f ? V3(1.0f, 0.0f, 0.0f) : V3(0.0f, 1.0f, 0.0f);
  const v3 tt = normalize(cross(up, n));
  const v3 bb = normalize(cross(n, tt));
  const v3 sv = vfloor((hp - rb) / fmax_(vs, 1e-6f));
  const uint32_t h0 = hash3_i32(i3{to_i32(sv.x), to_i32(sv.y), to_i32(sv.z)});
  const uint32_t h1 = hash_u32(h0);
  const uint32_t h2 = hash_u32(h1 ^ (s.cam->frame_index * 747796405u));
  const float rot = 6.28318530718f * ((float)(h2 & 1023u) / 1024.0f);
  const float soft_r = LIGHT_SOFT_RADIUS_VOX * vs, soft_r2 = soft_r * soft_r;
  const float min_r = LIGHT_NEAR_CLAMP_VOX * vs, min_r2 = min_r * min_r;
  const float range_m = LIGHT_RANGE_VOX * vs, range2 = range_m * range_m;
  const v3 Le = material_emission(MAT_LIGHT);
  v3 sum = V3s(0.0f);
  for (uint32_t i = 0; i < LIGHT_RAYS; ++i) {
    const v3 sl = normalize(sphere_dir_local(i, LIGHT_RAYS));
    v3 ldir = normalize(tt * sl.x + bb * sl.y + n * sl.z);
    ldir = normalize(rot_about_axis(ldir, n, rot));
    const v4 hit = dda_hit_light(s, p0, ldir, LIGHT_MAX_DIST_VOX, vs);
    if (hit.w > 0.5f) {
      hits += 1u;
      const v3 L = V3(hit.x, hit.y, hit.z) - hp;
      const float r2 = fmax_(dot(L, L), min_r2);
      const float r = std::sqrt(r2);
      const v3 lw = L / r;
      const float ndl = clampf((dot(n, lw) + LIGHT_WRAP) / (1.0f + LIGHT_WRAP), 0.0f, 1.0f);
      float att = clampf(1.0f - (r2 / fmax_(range2, 1e-6f)), 0.0f, 1.0f);
      att = att * att;
      const float falloff = 1.0f / (r2 + soft_r2);
      sum = sum + Le * (LIGHT_DIRECT_GAIN * ndl * falloff * att);
      if (r2 < 0.35f * range2) {
        const float bounce = LIGHT_INDIRECT_GAIN * falloff * att;
        sum = sum + Le * (0.25f * bounce);
      }
      if (hits >= LIGHT_EARLY_HITS) break;
    }
  }
  const float denom = fmax_(1.0f, (float)LIGHT_RAYS);
  return sum * (1.0f / denom);
}

// ---------------------------------------------------------------------------
// shading.wgsl
// ---------------------------------------------------------------------------
inline v3 color_for_material(uint32_t m) {  // shading.wgsl:7-16
  if (m == MAT_AIR) return V3s(0.0f);
  if (m == MAT_GRASS) return V3(0.18f, 0.75f, 0.18f);
  if (m == MAT_DIRT) return V3(0.45f, 0.30f, 0.15f);
  if (m == MAT_STONE) return V3(0.50f, 0.50f, 0.55f);
  if (m == MAT_WOOD) return V3(0.38f, 0.26f, 0.14f);
  if (m == MAT_LEAF) return V3(0.10f, 0.55f, 0.12f);
  if (m == MAT_LIGHT) return V3(1.0f, 0.95f, 0.75f);
  return V3(1.0f, 0.0f, 1.0f);
}
inline v3 hemi_ambient(v3 n, v3 sky_up) {  // shading.wgsl:18-22
  return vmix(FOG_COLOR_GROUND, sky_up, clampf(n.y * 0.5f + 0.5f, 0.0f, 1.0f));
}
v3 apply_material_variation(v3 base, uint32_t mat, v3 hp) {  // shading.wgsl:24-50
  v3 c = base;
  const float v = ALBEDO_VAR_GAIN * ((hash31(vfloor(hp / 0.05f)) - 0.5f) * 2.0f);
  if (mat == MAT_GRASS) {
    c = c + V3(0.02f * v, 0.05f * v, 0.01f * v);
    c = c * (1.0f + 0.06f * v);
  } else if (mat == MAT_DIRT) {
    c = c + V3(0.04f * v, 0.02f * v, 0.01f * v);
    c = c * (1.0f + 0.08f * v);
  } else if (mat == MAT_STONE) {
    c = c * (1.0f + 0.10f * v);
  } else if (mat == MAT_WOOD) {
    c = c + V3(0.05f * v, 0.02f * v, 0.00f * v);
    c = c * (1.0f + 0.07f * v);
  } else if (mat == MAT_LEAF) {
    c = c + V3(0.00f * v, 0.03f * v, 0.00f * v);
    c = c * (1.0f + 0.04f * v);
  }
  return vclamp(c, V3s(0.0f), V3s(1.5f));
}
v2 grass_wind_dir_xz(v3 p, float time_s) {  // shading.wgsl:52-59
  const v3 w = wind_field(p, time_s);
  v2 dir = V2(w.x, w.z) + V2(0.6f, 0.2f);
  if (dot(dir, dir) < 1e-4f) dir = V2(0.7f, 0.25f);
  return normalize(dir);
}
float grass_blade_slivers(v3 pw, float time_s, float freq, float detail) {  // shading.wgsl:61-88
  const v2 dir = grass_wind_dir_xz(pw, time_s);
  const v2 perp = V2(-dir.y, dir.x);
  const v2 pxz = V2(pw.x, pw.z);
  const v2 p = V2(dot(pxz, dir), dot(pxz, perp)) * freq;
  const v2 cell = vfloor(p);
  const v2 f = vfract(p);
  const float h0 = hash31(V3(cell.x, cell.y, 11.3f));
  const float h1 = hash31(V3(cell.x + 3.7f, cell.y + 7.1f, 5.9f));
  const float angle = (h0 - 0.5f) * 0.35f;
  const float ca = cosf_(angle), sa = sinf_(angle);
  const v2 pr = V2(f.x * ca - f.y * sa, f.x * sa + f.y * ca);
  const float center = 0.5f + (h1 - 0.5f) * 0.6f;
  const float u = clampf(pr.x, 0.0f, 1.0f);
  const float taper = mixf(0.065f, 0.012f, powf_(u, 1.8f));
  const float width = taper * mixf(0.75f, 1.25f, h0);
  const float aa = mixf(1.6f, 0.6f, detail) / freq;
  const float dist = std::fabs(pr.y - center);
  const float sliver = smooth(width + aa, width - aa, dist);
  const float lm = smooth(0.0f, 0.15f, u) * smooth(1.0f, 0.75f, u);
  return sliver * lm;
}
float grass_blade_field(v3 p, float time_s, float t) {  // shading.wgsl:90-98
  const float detail = 1.0f - smooth(18.0f, 55.0f, t);
  const float low = grass_blade_slivers(p, time_s, 9.0f, detail * 0.6f);
  const float high = grass_blade_slivers(p + V3(1.7f, 0.0f, 2.3f), time_s, 18.0f, detail);
  const float blend = mixf(0.15f, 1.0f, detail);
  return mixf(low, 0.5f * (low + high), blend);
}
v3 grass_top_albedo(const Scene& s, v3 base, v3 hp, float t) {  // shading.wgsl:100-122
  const float vs = vs_(s);
  const float tip = clampf(fract(hp.y / fmax_(vs, 1e-6f)), 0.0f, 1.0f);
  const float blade = grass_blade_field(hp, s.cam->voxel_params[1], t);
  const v2 hxz = V2(hp.x, hp.z);
  const float patches = fbm(hxz * 0.08f);
  const float clumps = fbm(hxz * 0.35f + V2(12.3f, 7.1f));
  const float density = smooth(0.25f, 0.75f, patches) * smooth(0.20f, 0.80f, clumps);
  const float coverage = blade * density;
  const v3 cool = base * V3(0.78f, 0.90f, 0.82f);
  const v3 warm = base * V3(1.08f, 1.16f, 0.92f) + V3(0.02f, 0.04f, 0.01f);
  const float grad = smooth(0.0f, 1.0f, tip);
  const v3 blade_col = vmix(cool, warm, grad);
  v3 out = vmix(base * 0.85f, blade_col, coverage);
  const float bs = mixf(0.68f, 1.0f, grad + 0.25f * coverage);
  out = out * bs;
  return vmax(out, V3s(0.02f));
}
inline v3 base_albedo(uint32_t mat, v3 hp, float t) {  // shading.wgsl:124-130
  v3 b = color_for_material(mat);
  if (t <= FAR_SHADING_DIST) b = apply_material_variation(b, mat, hp);
  return b;
}
float macro_occ_at_ws(const Scene& s, v3 p, v3 rb, float rs, uint32_t macro_base) {  // shading.wgsl:132-154
  if (macro_base == INVALID) return 0.0f;
  const v3 lp = p - rb;
  if (lp.x < 0.0f || lp.y < 0.0f || lp.z < 0.0f || lp.x >= rs || lp.y >= rs || lp.z >= rs) return 0.0f;
  const float cell = macro_cell_size(rs);
  const uint32_t mx = clampu(to_u32(std::floor(lp.x / cell)), 0u, 7u);
  const uint32_t my = clampu(to_u32(std::floor(lp.y / cell)), 0u, 7u);
  const uint32_t mz = clampu(to_u32(std::floor(lp.z / cell)), 0u, 7u);
  return macro_test(s, macro_base, macro_bit_index(mx, my, mz)) ? 1.0f : 0.0f;
}
float voxel_ao_local(const Scene& s, v3 hp, v3 n, v3 rb, float rs, uint32_t macro_base) {  // shading.wgsl:157-184
  const float r = 0.75f * vs_(s);
  const v3 up = std::fabs(n.y) > 0.9f ? V3(1.0f, 0.0f, 0.0f) : V3(0.0f, 1.0f, 0.0f);
  const v3 t = normalize(cross(up, n));
  const v3 b = normalize(cross(n, t));
  float occ = 0.0f;
  occ += macro_occ_at_ws(s, hp + t * r, rb, rs, macro_base);
  occ += macro_occ_at_ws(s, hp - t * r, rb, rs, macro_base);
  occ += macro_occ_at_ws(s, hp + b * r, rb, rs, macro_base);
  occ += macro_occ_at_ws(s, hp - b * r, rb, rs, macro_base);
  return clampf(1.0f - 0.70f * (occ * 0.25f), 0.35f, 1.0f);
}
inline float material_roughness(uint32_t m) {
  if (m == MAT_STONE) return 0.45f;
  if (m == MAT_WOOD) return 0.70f;
  if (m == MAT_LEAF) return 0.80f;
  if (m == MAT_GRASS) return 0.85f;
  if (m == MAT_DIRT) return 0.90f;
  if (m == MAT_LIGHT) return 0.25f;
  return 0.90f;
}
inline float material_f0(uint32_t m) {
  if (m == MAT_STONE) return 0.04f;
  if (m == MAT_WOOD) return 0.03f;
  if (m == MAT_LEAF) return 0.05f;
  if (m == MAT_GRASS) return 0.04f;
  if (m == MAT_DIRT) return 0.02f;
  if (m == MAT_LIGHT) return 0.08f;
  return 0.02f;
}

v3 shade_hit(const Scene& s, v3 ro, v3 rd, const HitGeom& hg, v3 sky_up, float sun_shadow) {  // shading.wgsl:257-362
  const v3 hp = ro + rd * hg.t;
  v3 base = base_albedo(hg.mat, hp, hg.t);
  if (hg.mat == MAT_GRASS) {
    base = grass_top_albedo(s, base, hp, hg.t);
    const float ndl = dot(hg.n, SUN_DIR);
    const float wrap = 0.35f;
    const float diff_wrap = clampf((ndl + wrap) / (1.0f + wrap), 0.0f, 1.0f);
    const float back = powf_(clampf(dot(-SUN_DIR, hg.n), 0.0f, 1.0f), 1.6f);
    const float vg = powf_(1.0f - fmax_(dot(normalize(-rd), hg.n), 0.0f), 2.0f);
    base = base + V3(0.18f, 0.34f, 0.10f) * (0.22f * back + 0.10f * vg * back);
    base = base * (0.90f + 0.10f * diff_wrap);
  }
  const float vs = vs_(s);
  const v3 hps = hp + hg.n * (0.75f * vs);
  const float Tc = cloud_sun_transmittance_fast(s, hps, SUN_DIR);
  const float sun_vis = Tc * clampf(sun_shadow, 0.0f, 1.0f);
  const float diff = fmax_(dot(hg.n, SUN_DIR), 0.0f);
  float ao = 1.0f;
  if (hg.hit != 0u && hg.t <= VOXEL_AO_MAX_DIST) ao = voxel_ao_local(s, hp, hg.n, hg.root_bmin, hg.root_size, hg.macro_base);
  const v3 amb_col = hemi_ambient(hg.n, sky_up);
  const float amb_strength = hg.mat == MAT_LEAF ? 0.13f : 0.10f;
  const float ao_term = powf_(clampf(ao, 0.0f, 1.0f), 1.0f);
  v3 ambient = amb_col * amb_strength * ao_term;
  if (hg.mat == MAT_STONE) ambient = ambient * V3(0.92f, 0.95f, 1.05f);
  float dapple = 1.0f;
  if (hg.mat == MAT_LEAF && hg.t <= FAR_SHADING_DIST) {
    const float ts = s.cam->voxel_params[1];
    const float d0 = sinf_(dot(V2(hp.x, hp.z), V2(3.0f, 2.2f)) + ts * 3.5f);
    const float d1 = sinf_(dot(V2(hp.x, hp.z), V2(6.5f, 4.1f)) - ts * 6.0f);
    dapple = 0.90f + 0.10f * (0.6f * d0 + 0.4f * d1);
  }
  v3 spec_col = V3s(0.0f);
  if (hg.t <= FAR_SHADING_DIST) {
    const v3 v = normalize(-rd);
    const v3 h = normalize(v + SUN_DIR);
    const float ndv = fmax_(dot(hg.n, v), 0.0f), ndh = fmax_(dot(hg.n, h), 0.0f);
    const float shin = mixf(8.0f, 96.0f, 1.0f - material_roughness(hg.mat));
    const float spec = powf_(ndh, shin);
    const float f0 = material_f0(hg.mat);
    const float fres = f0 + (1.0f - f0) * powf_(1.0f - clampf(ndv, 0.0f, 1.0f), 5.0f);
    spec_col = SUN_COLOR * SUN_INTENSITY * spec * fres * sun_vis;
  }
  float grass_ts = 1.0f;
  if (hg.mat == MAT_GRASS) {
    const GrassCell cell = grass_cell_from_world(hp, rd, hg.root_bmin, vs, (int32_t)s.cam->chunk_size);
    grass_ts = grass_self_shadow(s, hp, cell.bmin_m, cell.id_vox, s.cam->voxel_params[1], s.cam->voxel_params[2],
                                 grass_lod_from_t(hg.t));
  }
  const v3 direct = SUN_COLOR * SUN_INTENSITY * (0.35f * diff + 0.65f * diff * diff) * sun_vis * dapple * grass_ts;
  return base * (ambient + direct) + spec_col * 0.20f + material_emission(hg.mat);
}

v3 shade_clip_hit(const Scene& s, v3 ro, v3 rd, const ClipHit& ch, v3 sky_up) {  // shading.wgsl:364-434
  const v3 hp = ro + rd * ch.t;
  v3 base = color_for_material(ch.mat);
  if (ch.t <= FAR_SHADING_DIST) base = apply_material_variation_clip(base, ch.mat, hp);
  if (ch.mat == MAT_GRASS) base = grass_top_albedo(s, base, hp, ch.t);
  const float vs = vs_(s);
  const v3 hps = hp + ch.n * (0.75f * vs);
  const float vis = cloud_sun_transmittance_fast(s, hps, SUN_DIR);
  const float diff = fmax_(dot(ch.n, SUN_DIR), 0.0f);
  float ao = 1.0f;
  if (ch.mat == MAT_GRASS && ch.t <= FAR_SHADING_DIST) {
    const uint32_t lvl = clip_best_level(s, V2(hp.x, hp.z), 2);
    const float cell = s.clip->level[lvl][2];
    const v2 hxz = V2(hp.x, hp.z);
    const float h0 = clip_height_at_level(s, hxz, lvl);
    const float hx1 = clip_height_at_level(s, hxz + V2(cell, 0.0f), lvl);
    const float hx0 = clip_height_at_level(s, hxz + V2(-cell, 0.0f), lvl);
    const float hz1 = clip_height_at_level(s, hxz + V2(0.0f, cell), lvl);
    const float hz0 = clip_height_at_level(s, hxz + V2(0.0f, -cell), lvl);
    const float occ = fmax_(0.0f, hx1 - h0) + fmax_(0.0f, hx0 - h0) + fmax_(0.0f, hz1 - h0) + fmax_(0.0f, hz0 - h0);
    ao = clampf(1.0f - 0.65f * occ / fmax_(cell, 1e-3f), 0.45f, 1.0f);
  }
  const v3 ambient = hemi_ambient(ch.n, sky_up) * 0.10f * ao;
  const v3 direct = SUN_COLOR * SUN_INTENSITY * (diff * diff) * vis;
  v3 spec_col = V3s(0.0f);
  if (ch.t <= FAR_SHADING_DIST) {
    const v3 vd = normalize(-rd);
    const v3 hd = normalize(vd + SUN_DIR);
    const float ndv = fmax_(dot(ch.n, vd), 0.0f), ndh = fmax_(dot(ch.n, hd), 0.0f);
    float rough = 0.85f;
    if (ch.mat == MAT_STONE) rough = 0.50f;
    if (ch.mat == MAT_DIRT) rough = 0.90f;
    if (ch.mat == MAT_GRASS) rough = 0.88f;
    const float shin = mixf(8.0f, 96.0f, 1.0f - rough);
    const float spec = powf_(ndh, shin);
    float f0 = 0.03f;
    if (ch.mat == MAT_STONE) f0 = 0.04f;
    const float fres = f0 + (1.0f - f0) * powf_(1.0f - clampf(ndv, 0.0f, 1.0f), 5.0f);
    spec_col = SUN_COLOR * SUN_INTENSITY * spec * fres * vis;
  }
  return base * (ambient + direct) + spec_col * 0.18f;
}

// ---------------------------------------------------------------------------
// Frame images
// ---------------------------------------------------------------------------
struct FrameIO {
  uint32_t iw, ih, pw, ph;
  // inputs (history)
  const uint32_t* primary_hist_in;  // iw*ih*4 (raw bits)
  const float* shadow_in;           // iw*ih
  const float* local_hist_in;       // iw*ih*4
  const float* godray_hist_in;      // iw*ih*4
  const float* output_hist_in;      // pw*ph*4
  // outputs
  float* color;                // iw*ih*4
  float* depth;                // iw*ih
  float* local;                // iw*ih*4
  uint32_t* primary_hist_out;  // iw*ih*4
  float* shadow_out;           // iw*ih
  float* local_hist_out;       // iw*ih*4
  float* godray_out;           // iw*ih*4
  float* output_pre_taa;       // pw*ph*4
  float* output;               // pw*ph*4
  float* output_hist_out;      // pw*ph*4
  vxe_hit* hits;               // iw*ih (optional)
  // profile_counts (ray_main.wgsl:32-74): VOXEL, GRASS, HDR, FOG, SHADOW,
  // added to when cam.profile_flags & 1 (optional)
  uint32_t* profile;
};

// profile_inc / profile_add (ray_main.wgsl:64-74)
enum : uint32_t { PROFILE_VOXEL = 0, PROFILE_GRASS = 1, PROFILE_HDR = 2, PROFILE_FOG = 3, PROFILE_SHADOW = 4 };
inline void profile_add(const Scene& s, const FrameIO& io, uint32_t idx, uint32_t v) {
  if (io.profile && (s.cam->profile_flags & 1u) != 0u) __atomic_fetch_add(&io.profile[idx], v, __ATOMIC_RELAXED);
}
// fog_profile_weight (ray_main.wgsl:89-93)
inline uint32_t fog_profile_weight(float t_scene) {
  const float fog_norm = clampf(t_scene / FOG_MAX_DIST, 0.0f, 1.0f);
  return std::max(1u, to_u32(fog_norm * 256.0f));
}

inline v4 load4(const float* img, uint32_t w, int32_t x, int32_t y) {
  const float* p = img + ((size_t)y * w + (uint32_t)x) * 4;
  return v4{p[0], p[1], p[2], p[3]};
}
inline void store4(float* img, uint32_t w, int32_t x, int32_t y, v4 v) {
  float* p = img + ((size_t)y * w + (uint32_t)x) * 4;
  p[0] = v.x; p[1] = v.y; p[2] = v.z; p[3] = v.w;
}
// nearest + clamp-to-edge sample texel index
inline int32_t nearest_idx(float u, uint32_t n) { return clampi(to_i32(std::floor(u * (float)n)), 0, (int32_t)n - 1); }

inline uint32_t pack_i16x2(int32_t a, int32_t b) { return ((uint32_t)a & 0xFFFFu) | (((uint32_t)b & 0xFFFFu) << 16); }
inline int32_t unpack_i16(uint32_t v) {
  const int32_t s = (int32_t)(v & 0xFFFFu);
  return (v & 0x8000u) != 0u ? s - 0x10000 : s;
}

inline uint32_t face_from_n(v3 n) {
  const float ax = std::fabs(n.x), ay = std::fabs(n.y), az = std::fabs(n.z);
  if (ax >= ay && ax >= az) return n.x > 0.0f ? 0u : 1u;
  if (ay >= az) return n.y > 0.0f ? 2u : 3u;
  return n.z > 0.0f ? 4u : 5u;
}

void fill_hit(vxe_hit* h, const HitGeom& g, v3 ro, v3 rd, float vs, bool voxel_hit) {
  std::memset(h, 0, sizeof(*h));
  h->t = g.t;
  h->node = g.node;
  h->mat = g.mat;
  h->face = face_from_n(g.n);
  const v3 p = ro + rd * g.t;
  if (voxel_hit) {
    const v3 lr = (p - g.root_bmin) / vs;
    const v3 lmin = (g.leaf_bmin - g.root_bmin) / vs;
    const int32_t l0x = to_i32(std::floor(lmin.x + 0.5f)), l0y = to_i32(std::floor(lmin.y + 0.5f)),
                  l0z = to_i32(std::floor(lmin.z + 0.5f));
    const int32_t ls = to_i32(std::floor(g.leaf_size / vs + 0.5f));
    const int32_t ox = to_i32(std::floor(g.root_bmin.x / vs + 0.5f)), oy = to_i32(std::floor(g.root_bmin.y / vs + 0.5f)),
                  oz = to_i32(std::floor(g.root_bmin.z / vs + 0.5f));
    h->voxel[0] = ox + clampi(to_i32(std::floor(lr.x)), l0x, l0x + ls - 1);
    h->voxel[1] = oy + clampi(to_i32(std::floor(lr.y)), l0y, l0y + ls - 1);
    h->voxel[2] = oz + clampi(to_i32(std::floor(lr.z)), l0z, l0z + ls - 1);
  } else {
    h->voxel[0] = to_i32(std::floor(p.x / vs));
    h->voxel[1] = to_i32(std::floor(p.y / vs));
    h->voxel[2] = to_i32(std::floor(p.z / vs));
  }
}

void fill_miss(vxe_hit* h) {
  std::memset(h, 0, sizeof(*h));
  h->t = BIG;
  h->node = INVALID;
  h->face = 255u;
}

// main_primary for one pixel (ray_main.wgsl:163-517); the tile list was built
// by build_tile for this pixel's 8x8 workgroup.  Local TAA (taa.wgsl:26-69)
// is applied in the same call since it reads only this pixel.
void primary_pixel(const Scene& s, const FrameIO& io, const TileList& tl, uint32_t tile_count, uint32_t gx,
                   uint32_t gy) {
  const uint32_t W = io.iw, H = io.ih;
  const v3 sky_up = sky_bg(V3(0.0f, 1.0f, 0.0f));
  const v2 res = V2((float)W, (float)H);
  const v2 px = V2((float)gx + 0.5f, (float)gy + 0.5f);
  const uint32_t frame = s.cam->frame_index;
  const uint32_t seed = (gx * 1973u) ^ (gy * 9277u) ^ (frame * 26699u);
  const v3 ro = cam_pos(s);
  const v3 rd = ray_dir_from_pixel(s, px);
  const int32_t ix = (int32_t)gx, iy = (int32_t)gy;
  const size_t pix = (size_t)gy * W + gx;
  v3 local_out = V3s(0.0f);
  float local_w = 0.0f;
  float t_store = 0.0f;
  float shadow_out = 1.0f;
  const float vs = vs_(s);
  vxe_hit hit_rec;
  fill_miss(&hit_rec);

  auto write_common = [&](v3 col, float depth, uint32_t hx, uint32_t hy, uint32_t hz, uint32_t hw) {
    store4(io.color, W, ix, iy, v4{col.x, col.y, col.z, 1.0f});
    io.depth[pix] = depth;
    store4(io.local, W, ix, iy, v4{local_out.x, local_out.y, local_out.z, local_w});
    uint32_t* hp = io.primary_hist_out + pix * 4;
    hp[0] = hx; hp[1] = hy; hp[2] = hz; hp[3] = hw;
    io.shadow_out[pix] = shadow_out;
    if (io.hits) io.hits[pix] = hit_rec;
  };

  auto heightfield_or_sky = [&]() {
    ClipHit hf = clip_trace_heightfield(s, ro, rd, 0.0f, FOG_MAX_DIST);
    if (hf.hit) {
      if (hf.mat == MAT_GRASS) {
        const v3 hp = ro + rd * hf.t;
        const GrassCell cell = grass_cell_from_world_global(hp, rd, vs);
        const v3 gb = V3(cell.bmin_m.x, hp.y - vs, cell.bmin_m.z);
        const GrassHit gh = try_grass_slab_hit(s, ro, rd, 0.0f, hf.t, gb, cell.id_vox, vs, s.cam->voxel_params[1],
                                               s.cam->voxel_params[2]);
        if (gh.hit) {
          hf.t = gh.t;
          hf.n = gh.n;
          profile_add(s, io, PROFILE_GRASS, 1u);
        }
      }
      // shade_heightfield (ray_main.wgsl:100-114)
      profile_add(s, io, PROFILE_HDR, 1u);
      const v3 surface = shade_clip_hit(s, ro, rd, hf, sky_up);
      const float t_scene = fmin_(hf.t, FOG_MAX_DIST);
      const v3 col = apply_fog(s, surface, ro, rd, t_scene, sky_bg(rd));
      profile_add(s, io, PROFILE_FOG, fog_profile_weight(t_scene));
      t_store = t_scene;
      HitGeom g = miss_hitgeom();
      g.hit = 1; g.t = hf.t; g.n = hf.n; g.mat = hf.mat;
      fill_hit(&hit_rec, g, ro, rd, vs, false);
      write_common(col, t_scene, f_bits(t_store), 0u, 0u, 0u);
      return;
    }
    const v3 sky = sky_color(s, rd);
    write_common(sky, FOG_MAX_DIST, f_bits(t_store), 0u, 0u, 0u);
  };

  if (s.cam->chunk_count == 0u) {
    // no voxel chunks (ray_main.wgsl:219-231): the heightfield is traced but
    // not used; the pixel is sky
    const v3 sky = sky_color(s, rd);
    write_common(sky, FOG_MAX_DIST, f_bits(t_store), 0u, 0u, 0u);
  } else {
    float t_hist = 0.0f;
    bool hist_valid = false;
    uint32_t hak = INVALID;
    i3 hac{0, 0, 0};
    const bool has_tc = tile_count != 0u;
    const v2 uv = px / res;
    if (has_tc) {
      const uint32_t* hg = io.primary_hist_in + pix * 4;
      const float t_guess = bits_f(hg[0]);
      if (t_guess > 1e-3f) {
        const v3 p_ws = ro + rd * t_guess;
        const v2 uvp = prev_uv_from_world(s, p_ws);
        if (in_unit_square(uvp)) {
          const int32_t sx = nearest_idx(uvp.x, W), sy = nearest_idx(uvp.y, H);
          const uint32_t* hpv = io.primary_hist_in + ((size_t)sy * W + (uint32_t)sx) * 4;
          const float t_prev = bits_f(hpv[0]);
          const float rel = std::fabs(t_prev - t_guess) / fmax_(t_guess, 1e-3f);
          const float depth_ok = 1.0f - smooth(PRIMARY_HIT_DEPTH_REL0, PRIMARY_HIT_DEPTH_REL1, rel);
          const float vel = length((uvp - uv) * res);
          const float motion_ok = 1.0f - smooth(PRIMARY_HIT_MOTION_PX0, PRIMARY_HIT_MOTION_PX1, vel);
          if (t_prev > 1e-3f && depth_ok > 0.5f && motion_ok > 0.5f) {
            t_hist = t_prev;
            hist_valid = true;
            const uint32_t pz = hpv[3];
            if ((pz & 0x80000000u) != 0u) {
              hak = hpv[1];
              const uint32_t pxy = hpv[2];
              hac = i3{unpack_i16(pxy), unpack_i16(pxy >> 16), unpack_i16(pz)};
            }
          }
        }
      }
    }
    const float t_start = fmax_(t_hist - PRIMARY_HIT_MARGIN, 0.0f);
    const float t_end = fmin_(t_hist + PRIMARY_HIT_WINDOW, FOG_MAX_DIST);
    const Counters c_before = *s.ctr;
    // trace_primary_voxels (ray_main.wgsl:116-161)
    VoxTraceResult vt{false, miss_hitgeom(), 0.0f, false, INVALID, i3{0, 0, 0}};
    if (has_tc) {
      bool done = false;
      if (hist_valid) {
        profile_add(s, io, PROFILE_VOXEL, std::max(1u, tile_count));
        const VoxTraceResult h = trace_scene_voxels_candidates(s, tl, ro, rd, t_start, t_end, hak != INVALID, hac,
                                                               hak, tile_count);
        if (h.best.hit != 0u) { vt = h; done = true; }
      }
      if (!done) {
        profile_add(s, io, PROFILE_VOXEL, std::max(1u, tile_count));
        vt = trace_scene_voxels_candidates(s, tl, ro, rd, 0.0f, FOG_MAX_DIST, false, i3{0, 0, 0}, INVALID, tile_count);
      }
    }
    if (s.trace_ctr) {
      Counters& t = *s.trace_ctr;
      const Counters& c = *s.ctr;
      t.node_loads += c.node_loads - c_before.node_loads;
      t.rope_loads += c.rope_loads - c_before.rope_loads;
      t.meta_loads += c.meta_loads - c_before.meta_loads;
      t.grid_loads += c.grid_loads - c_before.grid_loads;
      t.macro_loads += c.macro_loads - c_before.macro_loads;
      t.colinfo_loads += c.colinfo_loads - c_before.colinfo_loads;
      t.clip_loads += c.clip_loads - c_before.clip_loads;
      t.oob += c.oob - c_before.oob;
    }
    if (!vt.in_grid || vt.best.hit == 0u) {
      heightfield_or_sky();
    } else {
      HitGeom best = vt.best;
      if (best.mat == MAT_GRASS) {
        const int32_t csv = (int32_t)s.cam->chunk_size;
        const i3 ov{to_i32(std::floor(best.root_bmin.x / vs + 0.5f)), to_i32(std::floor(best.root_bmin.y / vs + 0.5f)),
                    to_i32(std::floor(best.root_bmin.z / vs + 0.5f))};
        const v3 hp = ro + rd * best.t;
        const GrassCell cell = pick_grass_cell_in_chunk_with_bias(hp, rd, best.root_bmin, ov, vs, csv);
        const GrassHit gh = try_grass_slab_hit(s, ro, rd, 0.0f, best.t, cell.bmin_m, cell.id_vox, vs,
                                               s.cam->voxel_params[1], s.cam->voxel_params[2]);
        if (gh.hit) {
          best.t = gh.t;
          best.n = gh.n;
          profile_add(s, io, PROFILE_GRASS, 1u);
        }
      }
      const v3 hp = ro + rd * best.t;
      const v3 hps = hp + best.n * (0.75f * vs);
      profile_add(s, io, PROFILE_SHADOW, (seed & SHADOW_SUBSAMPLE_MASK) == 0u ? 2u : 1u);
      if ((seed & SHADOW_SUBSAMPLE_MASK) == 0u) {
        float sh = io.shadow_in[pix];
        const v2 uvp = prev_uv_from_world(s, hp);
        if (in_unit_square(uvp)) {
          const int32_t ppx = clampi(to_i32(uvp.x * (float)W), 0, (int32_t)W - 1);
          const int32_t ppy = clampi(to_i32(uvp.y * (float)H), 0, (int32_t)H - 1);
          sh = io.shadow_in[(size_t)ppy * W + (uint32_t)ppx];
        }
        sh = clampf(sh, 0.0f, 1.0f);
        const float cur = sun_transmittance_geom_only(s, hps, SUN_DIR);
        shadow_out = mixf(sh, cur, SHADOW_TAA_ALPHA);
      } else {
        shadow_out = clampf(io.shadow_in[pix], 0.0f, 1.0f);
      }
      // shade_hit_split (shading.wgsl:224-255)
      const v3 base_hdr = shade_hit(s, ro, rd, best, sky_up, shadow_out);
      if (best.hit != 0u && best.mat != MAT_LIGHT && best.t <= LOCAL_LIGHT_MAX_DIST) {
        const v3 hpl = ro + rd * best.t;
        const v3 alb = base_albedo(best.mat, hpl, best.t);
        local_out = gather_voxel_lights(s, hpl, best.n, best.root_bmin) * alb;
        local_w = 1.0f;
      }
      profile_add(s, io, PROFILE_HDR, 2u);
      const float t_scene = fmin_(best.t, FOG_MAX_DIST);
      const v3 col = apply_fog(s, base_hdr, ro, rd, t_scene, sky_bg(rd));
      profile_add(s, io, PROFILE_FOG, fog_profile_weight(t_scene));
      t_store = t_scene;
      uint32_t pxy = 0, pz = 0, ak = 0;
      if (vt.anchor_valid) {
        pxy = pack_i16x2(vt.anchor_chunk.x, vt.anchor_chunk.y);
        pz = pack_i16x2(vt.anchor_chunk.z, 0) | 0x80000000u;
        ak = vt.anchor_key;
      }
      fill_hit(&hit_rec, best, ro, rd, vs, true);
      write_common(col, t_scene, f_bits(t_store), ak, pxy, pz);
    }
  }
  // main_local_taa (taa.wgsl:26-69): nearest sample at the pixel centre is this pixel.
  const v4 cur4 = load4(io.local, W, ix, iy);
  const v4 hist4 = load4(io.local_hist_in, W, ix, iy);
  const v3 cur = V3(cur4.x, cur4.y, cur4.z);
  const float w_in = cur4.w;
  const bool hist_ok = !is_bad(V3(hist4.x, hist4.y, hist4.z));
  const v3 hist = hist_ok ? V3(hist4.x, hist4.y, hist4.z) : V3s(0.0f);
  const float conf0 = hist_ok ? hist4.w : 0.0f;
  const bool has_sample = w_in > 0.0f && !is_bad(cur);
  const float k = has_sample ? LOCAL_TAA_ALPHA * clampf(w_in, 0.0f, 1.0f) : 0.0f;
  const v3 ol = vmix(hist, cur, k);
  const float conf1 = has_sample ? fmin_(1.0f, conf0 + k) : conf0;
  store4(io.local_hist_out, W, ix, iy, v4{ol.x, ol.y, ol.z, conf1});
}

// ---------------------------------------------------------------------------
// godrays.wgsl
// ---------------------------------------------------------------------------
inline float approx_pow_0p75(float x) { const float y = clampf(x, 0.0f, 1.0f); return mixf(y, std::sqrt(y), 0.5f); }
inline float approx_pow_0p55(float x) { const float y = clampf(x, 0.0f, 1.0f); return mixf(std::sqrt(y), y, 0.20f); }
inline float exp_neg_fast(float xin) { const float x = fmax_(xin, 0.0f); return 1.0f / (1.0f + x + 0.48f * (x * x)); }
inline uint32_t godray_steps_for_tend(float t_end) {  // godrays.wgsl:30-43
  const float raw = std::ceil(t_end * GODRAY_STEPS_PER_METER);
  uint32_t sN = to_u32(clampf(raw, (float)GODRAY_MIN_STEPS, (float)GODRAY_STEPS_FAST));
  sN = ((sN + (GODRAY_STEP_Q - 1u)) / GODRAY_STEP_Q) * GODRAY_STEP_Q;
  return std::min(sN, GODRAY_STEPS_FAST);
}

v3 godray_integrate_1(const Scene& s, v3 ro, v3 rd, float t_end, float j, float j_phase) {  // godrays.wgsl:45-216
  const float base = fog_density_godray(s);
  if (base <= 0.0f || t_end <= 0.0f) return V3s(0.0f);
  const float phase = phase_blended(dot(rd, SUN_DIR));
  const float mu = dot(rd, SUN_DIR);
  const float view_gate = 0.10f + 0.90f * smooth(0.0f, 0.20f, mu);
  const uint32_t steps = godray_steps_for_tend(t_end);
  const float dt = t_end / (float)steps;
  const float a_ts = 1.0f - expf_(-dt * 3.0f);
  const float a_shaft = 1.0f - expf_(-dt * 5.0f);
  float ts = 1.0f, sh = 0.0f;
  v3 sum = V3s(0.0f);
  const float k = FOG_HEIGHT_FALLOFF, y0 = ro.y, dy = rd.y;
  const float f = clampf(0.5f + j_phase, 0.0f, 1.0f);
  const float omf = 1.0f - f;
  float Tv_acc = 1.0f;
  const bool horiz = std::fabs(dy) < 1e-4f;
  float tts_h = 1.0f, tte_h = 1.0f, inv_kdy = 0.0f, B = 0.0f, r_f = 1.0f, r_rem = 1.0f;
  if (horiz) {
    const float a = expf_(-k * y0);
    const float dc = base * a;
    tts_h = exp_neg_fast(dc * dt * f);
    tte_h = exp_neg_fast(dc * dt * omf);
  } else {
    inv_kdy = 1.0f / (k * dy);
    B = expf_(-k * y0);
    r_f = expf_(-k * dy * dt * f);
    r_rem = expf_(-k * dy * dt * omf);
  }
  float Ts_geom = 1.0f;
  for (uint32_t i = 0; i < steps; ++i) {
    const float ti = ((float)i + 0.5f + j_phase) * dt;
    if (ti + j * dt > t_end) break;
    const v3 p = ro + rd * ti;
    if (horiz) {
      Tv_acc *= tts_h;
    } else {
      const float Bs = B * r_f;
      const float dod = base * (B - Bs) * inv_kdy;
      Tv_acc *= exp_neg_fast(fmax_(dod, 0.0f));
    }
    const float Tv = Tv_acc;
    if (Tv < GODRAY_TV_CUTOFF) break;
    if ((i & 3u) == 0u) Ts_geom = sun_transmittance_geom_only(s, p, SUN_DIR);
    const float Tc = cloud_sun_transmittance_godray(s, p, SUN_DIR);
    const float Tc_vol = mixf(1.0f, Tc, CLOUD_GODRAY_W);
    const float Ts_soft = approx_pow_0p75(clampf(Ts_geom, 0.0f, 1.0f));
    const float haze_ramp = 1.0f - expf_(-ti / GODRAY_HAZE_NEAR_FADE);
    const float height_term = fmax_(expf_(-GODRAY_SCATTER_HEIGHT_FALLOFF * p.y), GODRAY_SCATTER_MIN_FRAC);
    const float dens = base * height_term;
    const v3 cf = (SUN_COLOR * SUN_INTENSITY) * (dens * dt) * Tv * phase * Tc_vol * 0.70f;
    const float ts_prev = ts;
    ts = mixf(ts, Ts_soft, a_ts);
    const float dTs = fmax_(0.0f, ts_prev - Ts_soft);
    float shaft = smooth(GODRAY_EDGE0, GODRAY_EDGE1, dTs);
    shaft = shaft * (1.0f - Ts_soft);
    shaft = approx_pow_0p55(clampf(shaft, 0.0f, 1.0f));
    sh = mixf(sh, shaft, a_shaft);
    shaft = sh;
    const float edge_boost = 1.0f + GODRAY_EDGE_ENERGY_BOOST * shaft;
    const float gate = smooth(0.35f, 0.80f, ts);
    const float haze = GODRAY_BASE_HAZE * haze_ramp * (ts * ts);
    const float w = clampf(haze + (1.0f - haze) * (shaft * gate), 0.0f, 1.0f);
    sum = sum + cf * view_gate * edge_boost * (ts * w);
    if (horiz) {
      Tv_acc *= tte_h;
    } else {
      const float Bs = B * r_f;
      const float Be = Bs * r_rem;
      const float dod2 = base * (Bs - Be) * inv_kdy;
      Tv_acc *= exp_neg_fast(fmax_(dod2, 0.0f));
      B = Be;
    }
  }
  v3 g = sum * GODRAY_ENERGY_BOOST;
  g = g / (g + V3s(GODRAY_KNEE_INTEGRATE));
  return g;
}

inline v3 godray_decompress(v3 c) {
  const v3 den = vmax(V3s(1.0f) - c, V3s(1e-4f));
  return (c * 0.25f) / den;
}
inline v3 godray_compress(v3 l) { return l / (l + V3s(0.25f)); }

// compute_godray_pixel (godrays.wgsl:241-356)
v4 godray_pixel(const Scene& s, const float* depth, const float* hist, uint32_t W, uint32_t H, uint32_t gx, uint32_t gy) {
  const int32_t Wi = (int32_t)W, Hi = (int32_t)H;
  const v3 ro = cam_pos(s);
  const int32_t x = (int32_t)gx, y = (int32_t)gy;
  const v2 qpx = V2((float)gx, (float)gy);
  const float fi = (float)(s.cam->frame_index & 1023u);
  const v2 fj = V2(fi, fi * 1.371f);
  auto D = [&](int32_t xx, int32_t yy) { return depth[(size_t)yy * W + (uint32_t)xx]; };
  const float t_c = D(x, y);
  const float t_l = D(clampi(x - 1, 0, Wi - 1), y), t_r = D(clampi(x + 1, 0, Wi - 1), y);
  const float t_u = D(x, clampi(y - 1, 0, Hi - 1)), t_d = D(x, clampi(y + 1, 0, Hi - 1));
  const float dmin = fmin_(t_c, fmin_(fmin_(t_l, t_r), fmin_(t_u, t_d)));
  const float dmax = fmax_(t_c, fmax_(fmax_(t_l, t_r), fmax_(t_u, t_d)));
  const float span = (dmax - dmin) / fmax_(dmin, 1e-3f);
  const float stable = 1.0f - smooth(0.06f, 0.30f, span);
  const float t_hist = dmin;
  const float j4 = 0.20f * (hash12(qpx * J0_SCALE + fj) - 0.5f);
  const float j_phase = hash12(qpx * 0.91f + fj * 0.73f + V2(31.7f, 12.3f)) - 0.5f;
  const float qstep = 0.03f;
  const float dq = (hash12(qpx * 1.37f + fj * 1.19f + V2(9.2f, 1.1f)) - 0.5f) * qstep;
  const v2 j_rd = V2(hash12(qpx + fj + V2(1.7f, 9.2f)) - 0.5f, hash12(qpx + fj * 1.13f + V2(8.3f, 2.1f)) - 0.5f);
  const float t_end = fmin_(std::floor((t_c + dq) / qstep) * qstep, GODRAY_MAX_DIST);
  const bool fog_ok = fog_density_godray(s) > 0.0f;
  const v2 pxc = V2((float)gx + 0.5f, (float)gy + 0.5f) + j_rd * 0.35f;
  const v3 rd = ray_dir_from_pixel(s, pxc);
  v3 cur = V3s(0.0f);
  if (fog_ok && t_end > 0.0f) cur = godray_integrate_1(s, ro, rd, t_end, j4, j_phase);
  const v3 p_ws = ro + rd * t_hist;
  const v2 uvp = prev_uv_from_world(s, p_ws);
  v3 hl = cur;
  float hv = 0.0f;
  const v2 hdf = V2((float)W, (float)H);
  const v2 uvc = V2((float)gx + 0.5f, (float)gy + 0.5f) / hdf;
  if (in_unit_square(uvp)) {
    const v4 h = load4(hist, W, nearest_idx(uvp.x, W), nearest_idx(uvp.y, H));
    const float hd = h.w;
    hl = godray_decompress(V3(h.x, h.y, h.z));
    const float rel = std::fabs(hd - t_hist) / fmax_(t_hist, 1e-3f);
    const float dok = 1.0f - smooth(0.08f, 0.20f, rel);
    const float dsane = hd > 1e-3f ? 1.0f : 0.0f;
    const float vel = length((uvp - uvc) * hdf);
    const float mok = 1.0f - smooth(0.75f, 2.50f, vel);
    hv = dok * dsane * mok;
  }
  const float delta = length(cur - hl);
  const float energy = fmax_(length(cur), 1e-3f);
  const float drel = delta / (0.05f + energy);
  const float react = smooth(0.10f, 0.45f, drel);
  const float cs = mixf(0.55f, 0.18f, stable);
  const v3 cw = vmax(cur * cs, V3s(0.015f));
  const v3 hc = vclamp(hl, cur - cw, cur + cw);
  const float hwb = mixf(0.25f, 0.92f, stable);
  const float hw = mixf(hwb, 0.03f, react) * hv;
  const v3 ol = vmix(cur, hc, hw);
  const v3 oc = godray_compress(vmax(ol, V3s(0.0f)));
  return v4{oc.x, oc.y, oc.z, t_hist};
}

// ---------------------------------------------------------------------------
// composite.wgsl + main_composite (ray_main.wgsl:537-573) + main_composite_taa (taa.wgsl:82-110)
// ---------------------------------------------------------------------------
inline v3 bright_extract_hue(v3 x, float thresh) {
  const float l = dot(x, V3(0.2126f, 0.7152f, 0.0722f));
  const float over = fmax_(l - thresh, 0.0f);
  return x * (over / fmax_(l, 1e-4f));
}
inline v3 hable(v3 x) {
  const float A = 0.22f, B = 0.30f, C = 0.10f, D = 0.20f, E = 0.01f, F = 0.30f;
  auto one = [&](float v) {
    const float num = v * (A * v + C * B) + D * E;
    const float den = v * (A * v + B) + D * F;
    return num / fmax_(den, 1e-6f) - E / F;
  };
  return V3(one(x.x), one(x.y), one(x.z));
}
inline v3 tonemap_white(v3 x, float wp) {
  const v3 w = hable(V3s(wp));
  const v3 invw = V3s(1.0f) / vmax(w, V3s(1e-6f));
  return hable(x) * invw;
}

void composite_pixel(const Scene& s, const FrameIO& io, uint32_t gx, uint32_t gy) {
  const uint32_t RW = io.iw, RH = io.ih, PW = io.pw, PH = io.ph;
  const v2 pp = V2((float)gx + 0.5f, (float)gy + 0.5f);
  const v2 rdim = V2((float)s.cam->render_present_px[0], (float)s.cam->render_present_px[1]);
  const v2 pdim = V2((float)s.cam->render_present_px[2], (float)s.cam->render_present_px[3]);
  const v2 px_render = (pp / pdim) * rdim;
  const int32_t ipr_x = clampi(to_i32(std::floor(px_render.x)), 0, to_i32(rdim.x) - 1);
  const int32_t ipr_y = clampi(to_i32(std::floor(px_render.y)), 0, to_i32(rdim.y) - 1);
  // composite_pixel_mapped (composite.wgsl:18-204)
  const int32_t rwi = (int32_t)RW, rhi = (int32_t)RH;
  const v2 rdf = V2((float)RW, (float)RH);
  const int32_t irx = clampi(ipr_x, 0, rwi - 1), iry = clampi(ipr_y, 0, rhi - 1);
  const v4 b4 = load4(io.color, RW, irx, iry);
  const v3 base = V3(b4.x, b4.y, b4.z);
  const v2 fdf = rdf;  // depth_full = internal depth
  const v2 px_full = px_render * (fdf / rdf);
  const int32_t ifx = clampi(to_i32(std::floor(px_full.x)), 0, rwi - 1);
  const int32_t ify = clampi(to_i32(std::floor(px_full.y)), 0, rhi - 1);
  const v2 uv_full = (px_full + V2(0.5f, 0.5f)) / fdf;
  auto DEP = [&](int32_t x, int32_t y) { return io.depth[(size_t)y * RW + (uint32_t)x]; };
  const float d0 = DEP(ifx, ify);
  const v2 gdf = V2((float)RW, (float)RH);
  const v2 du = V2(1.0f / gdf.x, 0.0f), dv = V2(0.0f, 1.0f / gdf.y);
  auto G = [&](v2 uv) {
    const v4 c = load4(io.godray_out, RW, nearest_idx(uv.x, RW), nearest_idx(uv.y, RH));
    return godray_decompress(V3(c.x, c.y, c.z));
  };
  const v3 gC = G(uv_full), gE = G(uv_full + du), gW = G(uv_full - du), gN = G(uv_full + dv), gS = G(uv_full - dv);
  const float dE = DEP(std::min(ifx + 1, rwi - 1), ify), dW = DEP(std::max(ifx - 1, 0), ify);
  const float dN = DEP(ifx, std::min(ify + 1, rhi - 1)), dS = DEP(ifx, std::max(ify - 1, 0));
  const float tol = 0.02f + 0.06f * smooth(10.0f, 80.0f, d0);
  const float wE = 1.0f - smooth(0.0f, tol, std::fabs(dE - d0));
  const float wW = 1.0f - smooth(0.0f, tol, std::fabs(dW - d0));
  const float wN = 1.0f - smooth(0.0f, tol, std::fabs(dN - d0));
  const float wS = 1.0f - smooth(0.0f, tol, std::fabs(dS - d0));
  const float wsum = fmax_(wE + wW + wN + wS, 1e-4f);
  const v3 blur = (gE * wE + gW * wW + gN * wN + gS * wS) / wsum;
  v3 god = vmax(gC + (gC - blur) * COMPOSITE_SHARPEN, V3s(0.0f));
  god = vmax(god - V3s(GODRAY_BLACK_LEVEL), V3s(0.0f));
  god = god / (god + V3s(GODRAY_KNEE_COMPOSITE));
  const float god_far = smooth(GODRAY_FADE_NEAR, GODRAY_FADE_FAR, d0);
  const float god_scale = GODRAY_COMPOSITE_SCALE * mixf(1.0f, 0.25f, god_far);
  const v3 lum_w = V3(0.2126f, 0.7152f, 0.0722f);
  const v3 sun_hue = normalize(vmax(SUN_COLOR, V3s(1e-4f)));
  const float g_lum = fmax_(dot(god, lum_w), 0.0f);
  const v3 god_sun = sun_hue * g_lum;
  god = vmix(god, god_sun, 0.55f * god_far);
  god = god * vmix(V3s(1.0f), V3(1.08f, 1.03f, 0.92f), god_far);
  v3 hdr = vmax(base + god * god_scale, V3s(0.0f));
  {
    const float bt = 1.4f;
    const float bk = 0.12f * mixf(1.0f, 0.0f, god_far);
    const v3 b0 = bright_extract_hue(hdr, bt);
    auto C = [&](int32_t x, int32_t y) { const v4 c = load4(io.color, RW, x, y); return vmax(V3(c.x, c.y, c.z), V3s(0.0f)); };
    const v3 hx1 = C(clampi(irx + 2, 0, rwi - 1), iry), hx0 = C(clampi(irx - 2, 0, rwi - 1), iry);
    const v3 hy1 = C(irx, clampi(iry + 2, 0, rhi - 1)), hy0 = C(irx, clampi(iry - 2, 0, rhi - 1));
    const v3 bloom = (b0 + bright_extract_hue(hx1, bt) + bright_extract_hue(hx0, bt) + bright_extract_hue(hy1, bt) +
                      bright_extract_hue(hy0, bt)) /
                     5.0f;
    const v3 bmax = vmax(hdr, V3s(0.0f)) * 0.35f;
    hdr = hdr + vmin(bloom, bmax) * bk;
  }
  const float l_hdr = fmax_(dot(hdr, lum_w), 1e-6f);
  const float t_sat = smooth(30.0f, 100.0f, d0);
  float sat = 1.00f + 0.55f * t_sat;
  const float hi = smooth(1.6f, 6.0f, l_hdr);
  sat = mixf(sat, 1.0f, 0.55f * hi);
  hdr = vmix(V3s(l_hdr), hdr, sat);
  hdr = hdr * 1.10f;
  hdr = hdr * V3(1.0f + 0.03f, 1.0f, 1.0f - 0.03f);
  hdr = (hdr - V3s(0.18f)) * 1.05f + V3s(0.18f);
  hdr = vmax(hdr, V3s(0.0f));
  v3 c = tonemap_white(hdr * POST_EXPOSURE, 6.0f);
  c = vclamp(c, V3s(0.0f), V3s(1.0f));
  c = V3(powf_(c.x, 0.98f), powf_(c.y, 0.98f), powf_(c.z, 0.98f));
  const float fi = (float)(s.cam->frame_index & 255u);
  const float n0 = hash12(px_render + V2(fi, 0.0f)) - 0.5f;
  const float n1 = hash12(px_render * 0.73f + V2(0.0f, fi)) - 0.5f;
  const float n = 0.6f * n0 + 0.4f * n1;
  c = c + V3s(n / 1536.0f);
  const v3 cc = vclamp(c, V3s(0.0f), V3s(1.0f));
  const float ge = 1.0f / 2.2f;
  const v3 ldr = V3(powf_(cc.x, ge), powf_(cc.y, ge), powf_(cc.z, ge));
  // + local_hist (ray_main.wgsl:558-569)
  const v2 uv_r = px_render * V2(1.0f / (float)RW, 1.0f / (float)RH);
  const v4 lh = load4(io.local_hist_out, RW, nearest_idx(uv_r.x, RW), nearest_idx(uv_r.y, RH));
  const v3 fin = ldr + V3(lh.x, lh.y, lh.z);
  const int32_t ox = (int32_t)gx, oy = (int32_t)gy;
  if (io.output_pre_taa) store4(io.output_pre_taa, PW, ox, oy, v4{fin.x, fin.y, fin.z, 1.0f});
  // main_composite_taa (taa.wgsl:82-110): reads composite_in at this pixel only.
  v3 taa = fin;
  if (s.cam->frame_index > 1u) {
    const float depth = DEP(ipr_x, ipr_y);
    const v3 rdv = ray_dir_from_pixel(s, px_render);
    const v3 p_ws = cam_pos(s) + rdv * depth;
    const v2 uvp = prev_uv_from_world(s, p_ws);
    if (in_unit_square(uvp)) {
      const v4 h = load4(io.output_hist_in, PW, nearest_idx(uvp.x, PW), nearest_idx(uvp.y, PH));
      taa = vmix(V3(h.x, h.y, h.z), taa, COMPOSITE_TAA_ALPHA);
    }
  }
  store4(io.output, PW, ox, oy, v4{taa.x, taa.y, taa.z, 1.0f});
  store4(io.output_hist_out, PW, ox, oy, v4{taa.x, taa.y, taa.z, 1.0f});
}

template <class F>
void parallel_rows(uint32_t rows, int threads, F&& f) {
  if (threads <= 1 || rows < 2) {
    f(0u, rows, 0);
    return;
  }
  std::vector<std::thread> ts;
  std::atomic<uint32_t> next{0};
  for (int t = 0; t < threads; ++t)
    ts.emplace_back([&, t]() {
      for (;;) {
        const uint32_t r = next.fetch_add(1);
        if (r >= rows) break;
        f(r, r + 1, t);
      }
    });
  for (auto& th : ts) th.join();
}

}  // namespace

// ===========================================================================
// C ABI of the oracle (for ctypes)
// ===========================================================================
extern "C" {

typedef struct ora_scene {
  const vxe_camera_gpu* cam;
  const vxe_chunk_meta* chunks;
  uint64_t chunks_n;
  const vxe_node* nodes;
  uint64_t nodes_n;
  const uint32_t* grid;
  uint64_t grid_n;
  const uint32_t* macro_words;
  uint64_t macro_n;
  const vxe_node_ropes* ropes;
  uint64_t ropes_n;
  const uint32_t* colinfo;
  uint64_t colinfo_n;
  const vxe_clipmap_gpu* clip;
  const float* clip_tex;
  uint32_t clip_layers, clip_res;
  uint32_t godray_macro_alias;
  uint32_t _pad;
} ora_scene;

typedef struct ora_counters {
  uint64_t node_loads, rope_loads, meta_loads, grid_loads, macro_loads, colinfo_loads, clip_loads, oob;
} ora_counters;

static Scene make_scene(const ora_scene* o, Counters* c, bool godray) {
  Scene s;
  s.cam = o->cam;
  s.chunks = o->chunks; s.chunks_n = o->chunks_n;
  s.nodes = o->nodes; s.nodes_n = o->nodes_n;
  s.grid = o->grid; s.grid_n = o->grid_n;
  if (godray && o->godray_macro_alias) {
    s.macro = reinterpret_cast<const uint32_t*>(o->ropes);
    s.macro_n = o->ropes_n * 8u;
  } else {
    s.macro = o->macro_words; s.macro_n = o->macro_n;
  }
  s.ropes = o->ropes; s.ropes_n = o->ropes_n;
  s.colinfo = o->colinfo; s.colinfo_n = o->colinfo_n;
  s.clip = o->clip; s.clip_tex = o->clip_tex; s.clip_layers = o->clip_layers; s.clip_res = o->clip_res;
  s.ctr = c;
  return s;
}

static void add_ctr(ora_counters* out, const Counters& c) {
  if (!out) return;
  out->node_loads += c.node_loads; out->rope_loads += c.rope_loads; out->meta_loads += c.meta_loads;
  out->grid_loads += c.grid_loads; out->macro_loads += c.macro_loads; out->colinfo_loads += c.colinfo_loads;
  out->clip_loads += c.clip_loads; out->oob += c.oob;
}

// One full frame: primary (+local TAA), godray, composite (+composite TAA).
// `io` arrays follow the layout documented in FrameIO.
int ora_render_frame(const ora_scene* sc, FrameIO* io, int threads, ora_counters* primary_ctr,
                     ora_counters* godray_ctr, ora_counters* trace_ctr) {
  if (!sc || !io) return 1;
  const int nt = threads < 1 ? 1 : threads;
  const uint32_t tiles_x = (io->iw + 7) / 8, tiles_y = (io->ih + 7) / 8;
  // primary: per tile row (tile lists are per 8x8 workgroup)
  std::vector<Counters> pc((size_t)nt);
  std::vector<Counters> tc((size_t)nt);
  parallel_rows(tiles_y, nt, [&](uint32_t r0, uint32_t r1, int t) {
    Scene s = make_scene(sc, &pc[(size_t)t], false);
    s.trace_ctr = &tc[(size_t)t];
    TileList tl;
    for (uint32_t ty = r0; ty < r1; ++ty)
      for (uint32_t tx = 0; tx < tiles_x; ++tx) {
        const uint32_t cnt = build_tile(s, tx, ty, tl);
        for (uint32_t y = ty * 8; y < std::min(ty * 8 + 8, io->ih); ++y)
          for (uint32_t x = tx * 8; x < std::min(tx * 8 + 8, io->iw); ++x) primary_pixel(s, *io, tl, cnt, x, y);
      }
  });
  for (auto& c : pc) add_ctr(primary_ctr, c);
  for (auto& c : tc) add_ctr(trace_ctr, c);
  std::vector<Counters> gc((size_t)nt);
  parallel_rows(io->ih, nt, [&](uint32_t r0, uint32_t r1, int t) {
    const Scene s = make_scene(sc, &gc[(size_t)t], true);
    for (uint32_t y = r0; y < r1; ++y)
      for (uint32_t x = 0; x < io->iw; ++x) {
        const v4 o = godray_pixel(s, io->depth, io->godray_hist_in, io->iw, io->ih, x, y);
        store4(io->godray_out, io->iw, (int32_t)x, (int32_t)y, o);
      }
  });
  for (auto& c : gc) add_ctr(godray_ctr, c);
  std::vector<Counters> cc((size_t)nt);
  parallel_rows(io->ph, nt, [&](uint32_t r0, uint32_t r1, int t) {
    const Scene s = make_scene(sc, &cc[(size_t)t], false);
    for (uint32_t y = r0; y < r1; ++y)
      for (uint32_t x = 0; x < io->pw; ++x) composite_pixel(s, *io, x, y);
  });
  return 0;
}

// Primary pass only over a row range [y0, y1) of tiles (for bounded CPU baselines).
int ora_primary_rows(const ora_scene* sc, FrameIO* io, uint32_t tile_y0, uint32_t tile_y1, int threads,
                     ora_counters* ctr) {
  if (!sc || !io) return 1;
  const int nt = threads < 1 ? 1 : threads;
  const uint32_t tiles_x = (io->iw + 7) / 8;
  const uint32_t tiles_y = (io->ih + 7) / 8;
  tile_y1 = std::min(tile_y1, tiles_y);
  if (tile_y0 >= tile_y1) return 0;
  std::vector<Counters> pc((size_t)nt);
  parallel_rows(tile_y1 - tile_y0, nt, [&](uint32_t r0, uint32_t r1, int t) {
    const Scene s = make_scene(sc, &pc[(size_t)t], false);
    TileList tl;
    for (uint32_t ty = tile_y0 + r0; ty < tile_y0 + r1; ++ty)
      for (uint32_t tx = 0; tx < tiles_x; ++tx) {
        const uint32_t cnt = build_tile(s, tx, ty, tl);
        for (uint32_t y = ty * 8; y < std::min(ty * 8 + 8, io->ih); ++y)
          for (uint32_t x = tx * 8; x < std::min(tx * 8 + 8, io->iw); ++x) primary_pixel(s, *io, tl, cnt, x, y);
      }
  });
  for (auto& c : pc) add_ctr(ctr, c);
  return 0;
}

// Per-tile candidate lists (count after clamping to 24, then the slots).
int ora_tile_lists(const ora_scene* sc, uint32_t iw, uint32_t ih, uint32_t* counts, uint32_t* slots24) {
  Counters c;
  const Scene s = make_scene(sc, &c, false);
  const uint32_t tx = (iw + 7) / 8, ty = (ih + 7) / 8;
  TileList tl;
  for (uint32_t y = 0; y < ty; ++y)
    for (uint32_t x = 0; x < tx; ++x) {
      const uint32_t n = build_tile(s, x, y, tl);
      const size_t t = (size_t)y * tx + x;
      counts[t] = n;
      for (uint32_t i = 0; i < PRIMARY_MAX_TILE_CHUNKS; ++i) slots24[t * PRIMARY_MAX_TILE_CHUNKS + i] = i < n ? tl.slots[i] : INVALID;
    }
  return 0;
}

// Ray queries: per-ray chunk-grid DDA, voxel geometry only, first hit.
int ora_trace_rays(const ora_scene* sc, const float* o, const float* d, uint32_t n, float tmax, vxe_hit* out,
                   int threads, ora_counters* ctr) {
  if (!sc) return 1;
  const int nt = threads < 1 ? 1 : threads;
  std::vector<Counters> pc((size_t)nt);
  const uint32_t rows = (n + 255) / 256;
  parallel_rows(rows, nt, [&](uint32_t r0, uint32_t r1, int t) {
    const Scene s = make_scene(sc, &pc[(size_t)t], false);
    const TraceOpts opt{true};
    for (uint32_t i = r0 * 256; i < std::min(r1 * 256, n); ++i) {
      const v3 ro = V3(o[3 * i], o[3 * i + 1], o[3 * i + 2]);
      const v3 rd = V3(d[3 * i], d[3 * i + 1], d[3 * i + 2]);
      const v3 inv = safe_inv3(rd);
      HitGeom best = miss_hitgeom();
      const float vs = vs_(s);
      const float rs = (float)s.cam->chunk_size * vs;
      chunk_grid_dda(s, ro, rd, 0.0f, tmax, [&](uint32_t slot, float) {
        const vxe_chunk_meta ch = chunk_at(s, slot);
        if (ch.macro_empty != 0u) return false;
        const v3 rb = V3((float)ch.origin[0], (float)ch.origin[1], (float)ch.origin[2]) * vs;
        const v2 rt = intersect_aabb(ro, rd, rb, rb + V3s(rs));
        const float ce = fmax_(rt.x, 0.0f), cx = fmin_(rt.y, fmin_(tmax, FOG_MAX_DIST));
        if (cx < ce) return false;
        const ChunkTraceResult h = trace_chunk_interval_stream_macro(s, ro, rd, inv, ch, ce, cx, false, INVALID, opt);
        if (h.hit.hit != 0u) { best = h.hit; return true; }
        return false;
      });
      if (best.hit) fill_hit(&out[i], best, ro, rd, vs, true);
      else fill_miss(&out[i]);
    }
  });
  for (auto& c : pc) add_ctr(ctr, c);
  return 0;
}

// Deterministic math probes (for tests of include/vxe/detmath.h).
void ora_detmath(int which, const float* x, const float* y, float* out, uint32_t n) {
  for (uint32_t i = 0; i < n; ++i) {
    switch (which) {
      case 0: out[i] = vxe_sinf(x[i]); break;
      case 1: out[i] = vxe_cosf(x[i]); break;
      case 2: out[i] = vxe_expf(x[i]); break;
      case 3: out[i] = vxe_powf(x[i], y[i]); break;
      case 4: out[i] = fmin_(x[i], y[i]); break;
      default: out[i] = fmax_(x[i], y[i]); break;
    }
  }
}

uint64_t ora_sizeof_frameio(void) { return sizeof(FrameIO); }

// Grass march pieces on host inputs (the device counterpart is
// vxe_debug_grass): which 0 = try_grass_slab_hit, 17 floats in (ro, rd,
// t_min, t_max, cb, id, voxel size, time, strength) -> 5 out (hit, t, n);
// which 1 = grass_sdf_lod, 13 floats in (p, cb, id, voxel size, time,
// strength, lod) -> 1 out.
void ora_debug_grass(int which, uint32_t n, const float* in, float* out) {
  Counters c;
  vxe_camera_gpu cam;
  std::memset(&cam, 0, sizeof cam);
  Scene s;
  std::memset((void*)&s, 0, sizeof s);
  s.cam = &cam;
  s.ctr = &c;
  for (uint32_t i = 0; i < n; ++i) {
    if (which == 0) {
      const float* a = in + (size_t)i * 17;
      cam.voxel_params[0] = a[14];
      cam.voxel_params[1] = a[15];
      cam.voxel_params[2] = a[16];
      const GrassHit g = try_grass_slab_hit(s, V3(a[0], a[1], a[2]), V3(a[3], a[4], a[5]), a[6], a[7],
                                            V3(a[8], a[9], a[10]), V3(a[11], a[12], a[13]), a[14], a[15], a[16]);
      float* o = out + (size_t)i * 5;
      o[0] = g.hit ? 1.0f : 0.0f;
      o[1] = g.t;
      o[2] = g.n.x;
      o[3] = g.n.y;
      o[4] = g.n.z;
    } else {
      const float* a = in + (size_t)i * 13;
      cam.voxel_params[0] = a[9];
      cam.voxel_params[1] = a[10];
      cam.voxel_params[2] = a[11];
      out[i] = grass_sdf_lod(s, V3(a[0], a[1], a[2]), V3(a[3], a[4], a[5]), V3(a[6], a[7], a[8]), a[10], a[11],
                             (uint32_t)a[12]);
    }
  }
}


// Pin interface (test infrastructure): the oracle's restatements of the
// reference's scene-reading helpers (sun shadow march, godray integral,
// local-light gather, leaf query, clipmap heightfield march and samples) over
// the world and clipmap of `sc`, in the flat-slot
// layout of oracle_shading_eval.  Returns -1 for a name it does not know.
int ora_scene_eval(const ora_scene* sc, const char* name, const float* in, float* out, uint32_t n) {
  if (!sc) return 1;
  Counters ctr;
  const Scene s = make_scene(sc, &ctr, false);
  const std::string nm(name);
  unsigned iw = 0;
  if (nm == "sun_transmittance_geom_only") iw = 6;
  else if (nm == "godray_integrate_1") iw = 9;
  else if (nm == "gather_voxel_lights") iw = 12;
  else if (nm == "query_leaf_world") iw = 3;
  else if (nm == "clip_trace_heightfield") iw = 8;
  else if (nm == "clip_height_at_level" || nm == "clip_height_at_level_nearest") iw = 3;
  else return -1;
  for (uint32_t k = 0; k < n; ++k) {
    const float* a = in + (size_t)k * iw;
    if (nm == "sun_transmittance_geom_only") {
      out[k] = sun_transmittance_geom_only(s, V3(a[0], a[1], a[2]), V3(a[3], a[4], a[5]));
    } else if (nm == "godray_integrate_1") {
      const v3 r = godray_integrate_1(s, V3(a[0], a[1], a[2]), V3(a[3], a[4], a[5]), a[6], a[7], a[8]);
      out[3 * k] = r.x, out[3 * k + 1] = r.y, out[3 * k + 2] = r.z;
    } else if (nm == "gather_voxel_lights") {  // root_size, node_base and macro_base are not read
      const v3 r = gather_voxel_lights(s, V3(a[0], a[1], a[2]), V3(a[3], a[4], a[5]), V3(a[6], a[7], a[8]));
      out[3 * k] = r.x, out[3 * k + 1] = r.y, out[3 * k + 2] = r.z;
    } else if (nm == "clip_trace_heightfield") {
      const ClipHit h = clip_trace_heightfield(s, V3(a[0], a[1], a[2]), V3(a[3], a[4], a[5]), a[6], a[7]);
      float* o = out + (size_t)k * 6;
      const uint32_t hit = h.hit ? 1u : 0u;
      std::memcpy(o, &hit, 4);
      o[1] = h.t, o[2] = h.n.x, o[3] = h.n.y, o[4] = h.n.z;
      std::memcpy(o + 5, &h.mat, 4);
    } else if (nm == "clip_height_at_level" || nm == "clip_height_at_level_nearest") {
      uint32_t level;
      std::memcpy(&level, a + 2, 4);
      out[k] = nm == "clip_height_at_level" ? clip_height_at_level(s, V2(a[0], a[1]), level)
                                            : clip_height_at_level_nearest(s, V2(a[0], a[1]), level);
    } else {
      const LeafQuery q = query_leaf_world(s, V3(a[0], a[1], a[2]));
      float* o = out + (size_t)k * 5;
      o[0] = q.bmin.x, o[1] = q.bmin.y, o[2] = q.bmin.z, o[3] = q.size;
      std::memcpy(o + 4, &q.mat, 4);
    }
  }
  return ctr.oob != 0 ? 2 : 0;
}

// Pin interface (test infrastructure): the cold primary voxel trace of the 64
// pixels of tile (tx, ty) -- build_tile (main_primary's lane-0 candidate
// list, ray_main.wgsl:179-197), then each pixel's
// trace_scene_voxels_candidates from t = 0 without an anchor
// (ray_main.wgsl:148-158) -- in the slot layout of the library
// oracle/wgsl_to_cpp.py builds from the reference's own WGSL: 64 x 16 slots,
// row-major pixels: in_grid (u32), hit (u32), mat (u32), t, n (3),
// root_bmin (3), root_size, t_exit, anchor_valid (u32), anchor_key (u32),
// anchor_chunk.xy (i32).  Returns the tile's candidate count.
int ora_primary_tile(const ora_scene* sc, uint32_t tx, uint32_t ty, float* out) {
  if (!sc) return -1;
  Counters ctr;
  const Scene s = make_scene(sc, &ctr, false);
  TileList tl;
  const uint32_t count = build_tile(s, tx, ty, tl);
  auto putu = [](float*& o, uint32_t x) { std::memcpy(o++, &x, 4); };
  for (uint32_t k = 0; k < 64u; ++k) {
    const uint32_t gx = tx * 8u + (k & 7u), gy = ty * 8u + (k >> 3);
    const v3 rd = ray_dir_from_pixel(s, V2((float)gx + 0.5f, (float)gy + 0.5f));
    const VoxTraceResult r =
        trace_scene_voxels_candidates(s, tl, cam_pos(s), rd, 0.0f, FOG_MAX_DIST, false, i3{0, 0, 0}, INVALID, count);
    float* o = out + (size_t)k * 16;
    putu(o, r.in_grid ? 1u : 0u);
    putu(o, r.best.hit);
    putu(o, r.best.mat);
    *o++ = r.best.t;
    *o++ = r.best.n.x, *o++ = r.best.n.y, *o++ = r.best.n.z;
    *o++ = r.best.root_bmin.x, *o++ = r.best.root_bmin.y, *o++ = r.best.root_bmin.z;
    *o++ = r.best.root_size;
    *o++ = r.t_exit;
    putu(o, r.anchor_valid ? 1u : 0u);
    putu(o, r.anchor_key);
    putu(o, (uint32_t)r.anchor_chunk.x);
    putu(o, (uint32_t)r.anchor_chunk.y);
  }
  return (int)count;
}

// Pin interface (test infrastructure): one chunk walk,
// trace_chunk_interval_stream_macro (chunk_trace.wgsl:592-667) with the
// grass probes of the primary trace, per ray, in the slot layout of the
// library oracle/wgsl_to_cpp.py builds from the reference's own WGSL:
//   rays: n x 12 slots: ro (3), rd (3), t0, t1, slot (u32 bits),
//         use_anchor (u32), anchor_key (u32), unused
//   out:  n x 16 slots: hit (u32), mat (u32), t, n (3), root_bmin (3),
//         root_size, node_base (u32), macro_base (u32), anchor_valid (u32),
//         anchor_key (u32), two unused
int ora_trace_chunk(const ora_scene* sc, const float* rays, float* out, uint32_t n) {
  if (!sc) return 1;
  Counters ctr;
  const Scene s = make_scene(sc, &ctr, false);
  const TraceOpts opt{false};
  auto putu = [](float*& o, uint32_t x) { std::memcpy(o++, &x, 4); };
  for (uint32_t k = 0; k < n; ++k) {
    const float* p = rays + (size_t)k * 12;
    float* o = out + (size_t)k * 16;
    const v3 ro = V3(p[0], p[1], p[2]), rd = V3(p[3], p[4], p[5]);
    uint32_t slot, use_anchor, key;
    std::memcpy(&slot, p + 8, 4);
    std::memcpy(&use_anchor, p + 9, 4);
    std::memcpy(&key, p + 10, 4);
    const ChunkTraceResult r =
        trace_chunk_interval_stream_macro(s, ro, rd, safe_inv3(rd), chunk_at(s, slot), p[6], p[7], use_anchor != 0u, key, opt);
    putu(o, r.hit.hit);
    putu(o, r.hit.mat);
    *o++ = r.hit.t;
    *o++ = r.hit.n.x;
    *o++ = r.hit.n.y;
    *o++ = r.hit.n.z;
    *o++ = r.hit.root_bmin.x;
    *o++ = r.hit.root_bmin.y;
    *o++ = r.hit.root_bmin.z;
    *o++ = r.hit.root_size;
    putu(o, r.hit.node_base);
    putu(o, r.hit.macro_base);
    putu(o, r.anchor_valid ? 1u : 0u);
    putu(o, r.anchor_key);
    *o++ = 0.0f;
    *o++ = 0.0f;
  }
  return ctr.oob != 0 ? 2 : 0;
}

// Pin interface (test infrastructure): the oracle's restatements of the
// reference's pure shading helpers behind the flat-slot calling convention of
// the library oracle/wgsl_to_cpp.py builds from the reference's own WGSL, so a
// test compares the two function by function.  Parameters and results are
// float slots (vecN = N slots; u32 passes its bit pattern); cam_pos4 and
// voxel_params4 stand in for the camera uniform.  Returns -1 for a name it
// does not know.
int oracle_shading_eval(const char* name, const float* in, float* out, unsigned n, const float* cam_pos4,
                        const float* voxel_params4) {
  vxe_camera_gpu cam;
  std::memset(&cam, 0, sizeof cam);
  for (int k = 0; k < 4; ++k) {
    cam.cam_pos[k] = cam_pos4[k];
    cam.voxel_params[k] = voxel_params4[k];
  }
  Counters ctr;
  Scene sc{};
  sc.cam = &cam;
  sc.ctr = &ctr;
  const Scene& s = sc;
  auto f1 = [](const float*& a) { return *a++; };
  auto v2_ = [](const float*& a) { const v2 r{a[0], a[1]}; a += 2; return r; };
  auto v3_ = [](const float*& a) { const v3 r{a[0], a[1], a[2]}; a += 3; return r; };
  auto u1 = [](const float*& a) { uint32_t u; std::memcpy(&u, a++, 4); return u; };
  auto put1 = [](float*& o, float x) { *o++ = x; };
  auto putu = [](float*& o, uint32_t x) { std::memcpy(o++, &x, 4); };
  auto put2 = [](float*& o, v2 x) { *o++ = x.x; *o++ = x.y; };
  auto put3 = [](float*& o, v3 x) { *o++ = x.x; *o++ = x.y; *o++ = x.z; };
  auto put4 = [](float*& o, v4 x) { *o++ = x.x; *o++ = x.y; *o++ = x.z; *o++ = x.w; };
  struct Entry {
    const char* name;
    unsigned in_w, out_w;
  };
  static const Entry widths[] = {
      {"hash_u32", 1, 1}, {"hash12", 2, 1}, {"hash31", 3, 1}, {"value_noise", 2, 1}, {"fbm", 2, 1},
      {"hash1", 3, 1}, {"wind_field", 4, 3}, {"clamp_len", 4, 3}, {"grass_wind_xz", 5, 2},
      {"grass_blade_params", 4, 4}, {"sdf_box", 9, 1}, {"phase_mie", 1, 1}, {"phase_blended", 1, 1},
      {"sky_bg", 3, 3}, {"sky_sun", 3, 3}, {"sky_color", 3, 3}, {"fog_color_from_sky", 6, 3},
      {"fog_inscatter", 6, 3}, {"fog_optical_depth_with_base", 8, 1}, {"apply_fog", 13, 3},
      {"cloud_height01", 1, 1}, {"cloud_coverage_at_xz", 3, 1}, {"cloud_density", 4, 1},
      {"cloud_light_transmittance", 4, 1}, {"cloud_sun_transmittance_fast", 6, 1}, {"cloud_density_godray", 4, 1},
      {"cloud_sun_transmittance_godray", 6, 1}, {"tonemap_filmic_hable", 3, 3}, {"tonemap_filmic_white_scale", 4, 3},
      {"bright_extract_hue", 4, 3}, {"intersect_aabb", 12, 2}, {"safe_inv", 1, 1}, {"ray_eps_vec", 4, 3},
      {"macro_cell_size", 1, 1}, {"grass_lod_from_t", 1, 1}, {"hemi_ambient", 6, 3}, {"color_for_material", 1, 3},
      {"apply_material_variation", 7, 3}, {"grass_wind_dir_xz", 4, 2}, {"grass_blade_slivers", 6, 1},
      {"grass_blade_field", 5, 1}, {"grass_top_albedo", 7, 3}, {"base_albedo", 5, 3}, {"material_roughness", 1, 1},
      {"material_f0", 1, 1}, {"material_emission", 1, 3}, {"approx_pow_0p75", 1, 1}, {"approx_pow_0p55", 1, 1},
      {"exp_neg_fast", 1, 1}, {"godray_steps_for_tend", 1, 1}, {"godray_decompress", 3, 3},
      {"godray_compress", 3, 3}, {"rot_about_axis", 7, 3}, {"sphere_dir_local", 2, 3}};
  const Entry* e = nullptr;
  for (const Entry& w : widths)
    if (!std::strcmp(w.name, name)) e = &w;
  if (!e) return -1;
  const std::string nm(name);
  for (unsigned k = 0; k < n; ++k) {
    const float* a = in + (size_t)k * e->in_w;
    float* o = out + (size_t)k * e->out_w;
    if (nm == "hash_u32") putu(o, hash_u32(u1(a)));
    else if (nm == "hash12") put1(o, hash12(v2_(a)));
    else if (nm == "hash31") put1(o, hash31(v3_(a)));
    else if (nm == "value_noise") put1(o, value_noise(v2_(a)));
    else if (nm == "fbm") put1(o, fbm(v2_(a)));
    else if (nm == "hash1") put1(o, hash1(v3_(a)));
    else if (nm == "wind_field") { const v3 p = v3_(a); put3(o, wind_field(p, f1(a))); }
    else if (nm == "clamp_len") { const v3 v = v3_(a); put3(o, clamp_len(v, f1(a))); }
    else if (nm == "grass_wind_xz") { const v3 r = v3_(a); const float t = f1(a); put2(o, grass_wind_xz(r, t, f1(a))); }
    else if (nm == "grass_blade_params") { const v3 id = v3_(a); put4(o, grass_blade_params(id, u1(a))); }
    else if (nm == "sdf_box") { const v3 p = v3_(a), c = v3_(a); put1(o, sdf_box(p, c, v3_(a))); }
    else if (nm == "phase_mie") put1(o, phase_mie(f1(a)));
    else if (nm == "phase_blended") put1(o, phase_blended(f1(a)));
    else if (nm == "sky_bg") put3(o, sky_bg(v3_(a)));
    else if (nm == "sky_sun") put3(o, sky_sun(v3_(a)));
    else if (nm == "sky_color") put3(o, sky_color(s, v3_(a)));
    else if (nm == "fog_color_from_sky") { const v3 rd = v3_(a); put3(o, fog_color_from_sky(rd, v3_(a))); }
    else if (nm == "fog_inscatter") { const v3 rd = v3_(a); put3(o, fog_inscatter(rd, v3_(a))); }
    else if (nm == "fog_optical_depth_with_base") {
      const float b = f1(a);
      const v3 ro = v3_(a), rd = v3_(a);
      put1(o, fog_optical_depth_with_base(b, ro, rd, f1(a)));
    } else if (nm == "apply_fog") {
      const v3 su = v3_(a), ro = v3_(a), rd = v3_(a);
      const float t = f1(a);
      put3(o, apply_fog(s, su, ro, rd, t, v3_(a)));
    } else if (nm == "cloud_height01") put1(o, cloud_height01(f1(a)));
    else if (nm == "cloud_coverage_at_xz") { const v2 xz = v2_(a); put1(o, cloud_coverage_at_xz(xz, f1(a))); }
    else if (nm == "cloud_density") { const v3 p = v3_(a); put1(o, cloud_density(p, f1(a))); }
    else if (nm == "cloud_light_transmittance") { const v3 p = v3_(a); put1(o, cloud_light_transmittance(p, f1(a))); }
    else if (nm == "cloud_sun_transmittance_fast") { const v3 p = v3_(a); put1(o, cloud_sun_transmittance_fast(s, p, v3_(a))); }
    else if (nm == "cloud_density_godray") { const v3 p = v3_(a); put1(o, cloud_density_godray(p, f1(a))); }
    else if (nm == "cloud_sun_transmittance_godray") { const v3 p = v3_(a); put1(o, cloud_sun_transmittance_godray(s, p, v3_(a))); }
    else if (nm == "tonemap_filmic_hable") put3(o, hable(v3_(a)));
    else if (nm == "tonemap_filmic_white_scale") { const v3 x = v3_(a); put3(o, tonemap_white(x, f1(a))); }
    else if (nm == "bright_extract_hue") { const v3 x = v3_(a); put3(o, bright_extract_hue(x, f1(a))); }
    else if (nm == "intersect_aabb") {
      const v3 ro = v3_(a), rd = v3_(a), b0 = v3_(a);
      put2(o, intersect_aabb(ro, rd, b0, v3_(a)));
    } else if (nm == "safe_inv") put1(o, safe_inv(f1(a)));
    else if (nm == "ray_eps_vec") { const v3 rd = v3_(a); put3(o, ray_eps_vec(rd, f1(a))); }
    else if (nm == "macro_cell_size") put1(o, macro_cell_size(f1(a)));
    else if (nm == "grass_lod_from_t") putu(o, grass_lod_from_t(f1(a)));
    else if (nm == "hemi_ambient") { const v3 nn = v3_(a); put3(o, hemi_ambient(nn, v3_(a))); }
    else if (nm == "color_for_material") put3(o, color_for_material(u1(a)));
    else if (nm == "apply_material_variation") {
      const v3 b = v3_(a);
      const uint32_t m = u1(a);
      put3(o, apply_material_variation(b, m, v3_(a)));
    } else if (nm == "grass_wind_dir_xz") { const v3 p = v3_(a); put2(o, grass_wind_dir_xz(p, f1(a))); }
    else if (nm == "grass_blade_slivers") {
      const v3 p = v3_(a);
      const float t = f1(a), fr = f1(a);
      put1(o, grass_blade_slivers(p, t, fr, f1(a)));
    } else if (nm == "grass_blade_field") { const v3 p = v3_(a); const float t = f1(a); put1(o, grass_blade_field(p, t, f1(a))); }
    else if (nm == "grass_top_albedo") { const v3 b = v3_(a), hp = v3_(a); put3(o, grass_top_albedo(s, b, hp, f1(a))); }
    else if (nm == "base_albedo") { const uint32_t m = u1(a); const v3 hp = v3_(a); put3(o, base_albedo(m, hp, f1(a))); }
    else if (nm == "material_roughness") put1(o, material_roughness(u1(a)));
    else if (nm == "material_f0") put1(o, material_f0(u1(a)));
    else if (nm == "material_emission") put3(o, material_emission(u1(a)));
    else if (nm == "approx_pow_0p75") put1(o, approx_pow_0p75(f1(a)));
    else if (nm == "approx_pow_0p55") put1(o, approx_pow_0p55(f1(a)));
    else if (nm == "exp_neg_fast") put1(o, exp_neg_fast(f1(a)));
    else if (nm == "godray_steps_for_tend") putu(o, godray_steps_for_tend(f1(a)));
    else if (nm == "godray_decompress") put3(o, godray_decompress(v3_(a)));
    else if (nm == "godray_compress") put3(o, godray_compress(v3_(a)));
    else if (nm == "rot_about_axis") { const v3 v = v3_(a), ax = v3_(a); put3(o, rot_about_axis(v, ax, f1(a))); }
    else if (nm == "sphere_dir_local") { const uint32_t i = u1(a); put3(o, sphere_dir_local(i, u1(a))); }
  }
  return 0;
}


}  // extern "C"
