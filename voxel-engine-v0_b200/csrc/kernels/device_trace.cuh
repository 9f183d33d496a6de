// device_trace.cuh -- device restatement of the reference WGSL ray functions.
//
// One device function per WGSL function of src/shaders/{common,clipmap}.wgsl
// and src/shaders/ray/*.wgsl (each cites its source lines).  The float
// operation sequence of every function matches the CPU oracle op for op, so
// outputs compare bit for bit.  Loads go through the bounds-checked accessors
// of device_common.cuh (16-byte node records, one rope word per exit).
#pragma once

#include "device_common.cuh"

namespace vxe {
namespace dev {

// Constants (common.wgsl:16-332)
constexpr float SUN_DIR_X = 0.61237244f, SUN_DIR_Y = 0.5f, SUN_DIR_Z = 0.61237244f;
constexpr float SHADOW_BIAS = 2e-4f;
constexpr uint32_t VSM_STEPS = 16;
constexpr float LEAF_LIGHT_TRANSMIT = 0.50f, GRASS_LIGHT_TRANSMIT = 0.70f, MIN_TRANS = 0.03f;
constexpr float GODRAY_ENERGY_BOOST = 8.0f, GODRAY_KNEE_INTEGRATE = 0.35f, GODRAY_COMPOSITE_SCALE = 6.5f;
constexpr float GODRAY_FADE_NEAR = 40.0f, GODRAY_FADE_FAR = 80.0f, GODRAY_KNEE_COMPOSITE = 0.25f;
constexpr float FOG_HEIGHT_FALLOFF = 0.18f, FOG_PRIMARY_SCALE = 0.02f,
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
constexpr uint32_t MACRO_DIM = 8, PRIMARY_MAX_TILE_CHUNKS = 24;


// ---------------------------------------------------------------------------
// common.wgsl helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ float macro_cell_size(float root_size) { return root_size / (float)MACRO_DIM; }  // common.wgsl:426
__device__ __forceinline__ uint32_t macro_bit_index(uint32_t mx, uint32_t my, uint32_t mz) {                 // common.wgsl:431
  return mx + MACRO_DIM * (my + MACRO_DIM * mz);
}
__device__ __forceinline__ bool macro_test(const Scene& s, uint32_t macro_base, uint32_t bit) {  // common.wgsl:435-440
  const uint32_t w = bit >> 5, b = bit & 31u;
  return (macro_word(s, macro_base + w) & (1u << b)) != 0u;
}
__device__ __forceinline__ float safe_inv(float x) { return fabsf(x) < EPS_INV ? BIG : 1.0f / x; }  // common.wgsl:442
__device__ __forceinline__ v3 safe_inv3(v3 r) { return V3(safe_inv(r.x), safe_inv(r.y), safe_inv(r.z)); }

__device__ __forceinline__ v3 ray_dir_from_pixel(const Scene& s, v2 px) {  // common.wgsl:456-459
  const vxe_camera_gpu* c = s.cam;
  const v3 d = V3(c->ray00[0] + px.x * c->ray_dx[0] + px.y * c->ray_dy[0],
                  c->ray00[1] + px.x * c->ray_dx[1] + px.y * c->ray_dy[1],
                  c->ray00[2] + px.x * c->ray_dx[2] + px.y * c->ray_dy[2]);
  return normalize(d);
}

__device__ __forceinline__ v2 prev_uv_from_world(const Scene& s, v3 p) {  // common.wgsl:461-467
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

__device__ v2 intersect_aabb(v3 ro, v3 rd, v3 bmin, v3 bmax) {  // common.wgsl:473-510
  const float eps = 1e-8f;
  float t_enter = -1e30f, t_exit = 1e30f;
  const float r[3] = {ro.x, ro.y, ro.z}, d[3] = {rd.x, rd.y, rd.z};
  const float lo[3] = {bmin.x, bmin.y, bmin.z}, hi[3] = {bmax.x, bmax.y, bmax.z};
  for (int a = 0; a < 3; ++a) {
    if (fabsf(d[a]) < eps) {
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

__device__ __forceinline__ uint32_t child_rank(uint32_t mask, uint32_t ci) {  // common.wgsl:512-516
  return (uint32_t)__popc(mask & ((1u << ci) - 1u));
}

__device__ uint32_t grid_lookup_slot(const Scene& s, int32_t cx, int32_t cy, int32_t cz) {  // common.wgsl:518-541
  const int32_t ix = cx - s.cam->grid_origin_chunk[0], iy = cy - s.cam->grid_origin_chunk[1],
                iz = cz - s.cam->grid_origin_chunk[2];
  if (ix < 0 || iy < 0 || iz < 0) return INVALID;
  const uint32_t nx = s.cam->grid_dims[0], ny = s.cam->grid_dims[1], nz = s.cam->grid_dims[2];
  if ((uint32_t)ix >= nx || (uint32_t)iy >= ny || (uint32_t)iz >= nz) return INVALID;
  return grid_at(s, (uint32_t)iz * ny * nx + (uint32_t)iy * nx + (uint32_t)ix);
}

__device__ __forceinline__ i3 chunk_coord_from_pos(v3 p, float cs) {  // common.wgsl:543-554
  const float eps = 1e-6f * cs;
  const float px = p.x - signf(p.x) * eps, py = p.y - signf(p.y) * eps, pz = p.z - signf(p.z) * eps;
  return i3{to_i32(floorf(px / cs)), to_i32(floorf(py / cs)), to_i32(floorf(pz / cs))};
}

__device__ __forceinline__ uint32_t chunk_max_depth(const Scene& s) {  // common.wgsl:569-572
  return 31u - (uint32_t)__clz(s.cam->chunk_size);
}

// Hashes / noise (common.wgsl:595-662)
__device__ __forceinline__ uint32_t hash_u32(uint32_t v) {
  v ^= v >> 16;
  v *= 0x7feb352du;
  v ^= v >> 15;
  v *= 0x846ca68bu;
  v ^= v >> 16;
  return v;
}
__device__ __forceinline__ uint32_t hash2_u32(uint32_t x, uint32_t y) { return hash_u32(x * 0x8da6b343u ^ y * 0xd8163841u); }
__device__ __forceinline__ uint32_t hash3_u32(uint32_t x, uint32_t y, uint32_t z) {
  return hash_u32(x * 0x8da6b343u ^ y * 0xd8163841u ^ z * 0xcb1ab31fu);
}
constexpr float U32_TO_F01 = 1.0f / 4294967296.0f;
__device__ __forceinline__ float hash12(v2 p) {
  const uint32_t ix = (uint32_t)to_i32(floorf(p.x)), iy = (uint32_t)to_i32(floorf(p.y));
  return (float)hash2_u32(ix, iy) * U32_TO_F01;
}
__device__ __forceinline__ float hash31(v3 p) {
  const uint32_t ix = (uint32_t)to_i32(floorf(p.x)), iy = (uint32_t)to_i32(floorf(p.y)),
                 iz = (uint32_t)to_i32(floorf(p.z));
  return (float)hash3_u32(ix, iy, iz) * U32_TO_F01;
}
__device__ __noinline__ float value_noise(v2 p) {
  const v2 i = vfloor(p), f = vfract(p);
  const float a = hash12(i), b = hash12(i + V2(1.0f, 0.0f)), c = hash12(i + V2(0.0f, 1.0f)),
              d = hash12(i + V2(1.0f, 1.0f));
  const v2 u = V2(f.x * f.x * (3.0f - 2.0f * f.x), f.y * f.y * (3.0f - 2.0f * f.y));
  const float x1 = mixf(a, b, u.x), x2 = mixf(c, d, u.x);
  return mixf(x1, x2, u.y);
}
__device__ __noinline__ float fbm(v2 p) {
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

__device__ __forceinline__ bool is_bad(v3 v) {  // common.wgsl:692-706
  auto bad = [](float x) { return x != x || fabsf(x) > 1.0e30f; };
  return bad(v.x) || bad(v.y) || bad(v.z);
}
__device__ __forceinline__ v3 ray_eps_vec(v3 rd, float e) {  // common.wgsl:708-715
  return V3(rd.x >= 0.0f ? e : -e, rd.y >= 0.0f ? e : -e, rd.z >= 0.0f ? e : -e);
}

// ---------------------------------------------------------------------------
// aabb.wgsl
// ---------------------------------------------------------------------------
struct CubeSlab { v3 tminv, tmaxv; float t_enter, t_exit; };

__device__ CubeSlab cube_slab_inv(v3 ro, v3 inv, v3 bmin, float size) {  // aabb.wgsl:16-84
  const v3 bmax = bmin + V3s(size);
  v3 t0 = (bmin - ro) * inv, t1 = (bmax - ro) * inv;
  const float INV_PARALLEL = 1e20f;
  const CubeSlab miss{V3s(BIG), V3s(-BIG), BIG, -BIG};
  if (fabsf(inv.x) > INV_PARALLEL) {
    if (ro.x < bmin.x || ro.x >= bmax.x) return miss;
    t0.x = -BIG; t1.x = BIG;
  }
  if (fabsf(inv.y) > INV_PARALLEL) {
    if (ro.y < bmin.y || ro.y >= bmax.y) return miss;
    t0.y = -BIG; t1.y = BIG;
  }
  if (fabsf(inv.z) > INV_PARALLEL) {
    if (ro.z < bmin.z || ro.z >= bmax.z) return miss;
    t0.z = -BIG; t1.z = BIG;
  }
  const v3 tminv = vmin(t0, t1), tmaxv = vmax(t0, t1);
  return CubeSlab{tminv, tmaxv, max3(tminv), min3(tmaxv)};
}

struct BoxHit { bool hit; float t, t_exit; v3 n; };

__device__ BoxHit cube_hit_normal_from_slab(v3 rd, const CubeSlab& slab, float t_min, float t_max) {  // aabb.wgsl:95-141
  const float t0 = fmax_(slab.t_enter, t_min);
  if (slab.t_exit < t0 || t0 > t_max) return BoxHit{false, BIG, slab.t_exit, V3s(0.0f)};
  const float te = slab.t_enter;
  const float eps = 1e-5f * fmax_(1.0f, fabsf(te));
  const bool mx = fabsf(slab.tminv.x - te) <= eps, my = fabsf(slab.tminv.y - te) <= eps,
             mz = fabsf(slab.tminv.z - te) <= eps;
  uint32_t axis = 0;
  if (mx || my || mz) {
    float best = -1.0f;
    if (mx) { best = fabsf(rd.x); axis = 0; }
    if (my && fabsf(rd.y) > best) { best = fabsf(rd.y); axis = 1; }
    if (mz && fabsf(rd.z) > best) { best = fabsf(rd.z); axis = 2; }
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

__device__ __forceinline__ BoxHit aabb_hit_normal_inv(v3 ro, v3 rd, v3 inv, v3 bmin, float size, float tmin, float tmax) {
  return cube_hit_normal_from_slab(rd, cube_slab_inv(ro, inv, bmin, size), tmin, tmax);
}

// ---------------------------------------------------------------------------
// svo_query.wgsl
// ---------------------------------------------------------------------------
struct LeafQuery { v3 bmin; float size; uint32_t mat; };

__device__ __noinline__ LeafQuery query_leaf_at(const Scene& s, v3 p, v3 root_bmin, float root_size, uint32_t node_base,
                        uint32_t macro_base) {  // svo_query.wgsl:11-108
  uint32_t idx = node_base;
  v3 bmin = root_bmin;
  float size = root_size;
  if (macro_base != INVALID) {
    const float cell = macro_cell_size(root_size);
    const v3 lp = p - root_bmin;
    if (lp.x < 0.0f || lp.y < 0.0f || lp.z < 0.0f || lp.x >= root_size || lp.y >= root_size || lp.z >= root_size)
      return LeafQuery{root_bmin, root_size, MAT_AIR};
    const int32_t mx = to_i32(floorf(lp.x / cell)), my = to_i32(floorf(lp.y / cell)),
                  mz = to_i32(floorf(lp.z / cell));
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

__device__ __noinline__ LeafQuery query_leaf_world(const Scene& s, v3 p) {  // svo_query.wgsl:270-291
  const float vs = vs_(s);
  const float cs = (float)s.cam->chunk_size * vs;
  const i3 c = chunk_coord_from_pos(p, cs);
  const uint32_t slot = grid_lookup_slot(s, c.x, c.y, c.z);
  if (slot == INVALID || slot >= s.cam->chunk_count) return LeafQuery{p, vs, MAT_AIR};
  const Meta ch = meta_at(s, slot);
  const v3 rb = V3((float)ch.ox, (float)ch.oy, (float)ch.oz) * vs;
  return query_leaf_at(s, p, rb, (float)s.cam->chunk_size * vs, ch.node_base, ch.macro_base);
}

// ---------------------------------------------------------------------------
// wind.wgsl / leaves.wgsl
// ---------------------------------------------------------------------------
__device__ __forceinline__ float hash1(v3 p) { return fract(sinf_(dot(p, V3(127.1f, 311.7f, 74.7f))) * 43758.5453f); }

__device__ __noinline__ v3 wind_field(v3 pos, float t) {  // wind.wgsl:10-36
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

__device__ __forceinline__ v3 clamp_len(v3 v, float max_len) {  // wind.wgsl:38-42
  const float l2 = dot(v, v);
  if (l2 <= max_len * max_len) return v;
  return v * (max_len / sqrtf(l2));
}

__device__ __noinline__ v3 leaf_cube_offset(const Scene& s, v3 bmin, float size, float time_s, float strength) {  // leaves.wgsl:5-18
  const v3 center = bmin + V3s(0.5f * size);
  const float d = length(center - cam_pos(s));
  const float fade = smooth(LEAF_LOD_DISP_START, LEAF_LOD_DISP_END, d);
  const float se = strength * (1.0f - fade);
  v3 w = wind_field(center, time_s) * se;
  w = V3(w.x, LEAF_VERTICAL_REDUCE * w.y, w.z);
  const float amp = LEAF_OFFSET_AMP * size;
  return clamp_len(w * amp, LEAF_OFFSET_MAX_FRAC * size);
}

__device__ __noinline__ BoxHit leaf_displaced_cube_hit(const Scene& s, v3 ro, v3 rd, v3 bmin, float size, float time_s, float strength,
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

__device__ GrassCell pick_grass_cell_in_chunk_with_bias(v3 hp, v3 bias_dir, v3 root_bmin, i3 origin_vox, float vs,
                                            int32_t csv) {  // grass.wgsl:10-44
  const float root_size_m = (float)csv * vs;
  const float bias = 0.05f * vs;
  v3 lxz = (hp - root_bmin) - bias_dir * bias;
  lxz.x = clampf(lxz.x, 0.0f, root_size_m - 1e-6f);
  lxz.z = clampf(lxz.z, 0.0f, root_size_m - 1e-6f);
  const float y_in = (hp - bias_dir * bias).y - 1e-4f * vs;
  const float ly = clampf(y_in - root_bmin.y, 0.0f, root_size_m - 1e-6f);
  int32_t ix = to_i32(floorf(lxz.x / vs)), iy = to_i32(floorf(ly / vs)), iz = to_i32(floorf(lxz.z / vs));
  ix = clampi(ix, 0, csv - 1);
  iy = clampi(iy, 0, csv - 1);
  iz = clampi(iz, 0, csv - 1);
  const v3 bmin = root_bmin + V3((float)ix, (float)iy, (float)iz) * vs;
  const v3 id = V3((float)(origin_vox.x + ix), (float)(origin_vox.y + iy), (float)(origin_vox.z + iz));
  return GrassCell{bmin, id};
}

__device__ GrassCell grass_cell_from_world(v3 hp, v3 rd, v3 root_bmin, float vs, int32_t csv) {  // grass.wgsl:64-84
  const i3 o{to_i32(floorf(root_bmin.x / vs)), to_i32(floorf(root_bmin.y / vs)),
             to_i32(floorf(root_bmin.z / vs))};
  return pick_grass_cell_in_chunk_with_bias(hp, rd, root_bmin, o, vs, csv);
}

__device__ GrassCell grass_cell_from_world_global(v3 hp, v3 rd, float vs) {  // grass.wgsl:86-104
  const float bias = 0.05f * vs;
  const v3 p = hp - rd * bias;
  const float py = p.y - 1e-4f * vs;
  const int32_t ix = to_i32(floorf(p.x / vs)), iy = to_i32(floorf(py / vs)), iz = to_i32(floorf(p.z / vs));
  const v3 id = V3((float)ix, (float)iy, (float)iz);
  return GrassCell{id * vs, id};
}

__device__ __forceinline__ float sdf_box(v3 p, v3 c, v3 b) {  // grass.wgsl:106-111
  const v3 q = vabs(p - c) - b;
  const float outside = length(vmax(q, V3s(0.0f)));
  const float inside = fmin_(fmax_(q.x, fmax_(q.y, q.z)), 0.0f);
  return outside + inside;
}

__device__ __forceinline__ v3 ortho_basis_x(v3 n) {  // grass.wgsl:120-126 (column 0)
  const v3 up = fabsf(n.y) > 0.999f ? V3(1.0f, 0.0f, 0.0f) : V3(0.0f, 1.0f, 0.0f);
  return normalize(cross(up, n));
}

__device__ __forceinline__ v4 grass_blade_params(v3 id, uint32_t i) {  // grass.wgsl:353-368
  const float fi = (float)i;
  const float h0 = hash31(id + V3(fi * 7.3f, 1.1f, 2.9f));
  const float h1 = hash31(id + V3(fi * 3.7f, 8.4f, 0.6f));
  return v4{fract(h0 * 1.61803398875f), fract(h0 * 2.41421356237f), fract(h0 * 3.14159265359f),
            0.35f + 0.65f * (h1 * h1)};
}

__device__ __forceinline__ v2 grass_wind_xz(v3 root, float t, float strength) {  // grass.wgsl:185-189
  const v3 w = wind_field(root, t) * strength;
  return V2(w.x, w.z);
}

__device__ __noinline__ float grass_sdf_lod(const Scene& s, v3 p, v3 cb, v3 id, float time_s, float strength, uint32_t lod) {
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
  uint32_t segs = to_u32(fmax_(3.0f, floorf(GRASS_VOXEL_SEGS)));
  if (lod == 1u) {
    blade_count = min(blade_count, GRASS_BLADE_COUNT_MID);
    segs = min(segs, GRASS_SEGS_MID);
  } else if (lod == 2u) {
    blade_count = min(blade_count, GRASS_BLADE_COUNT_FAR);
    segs = min(segs, GRASS_SEGS_FAR);
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
      else S = S * (1.0f / sqrtf(s2));
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

// ---------------------------------------------------------------------------
// Per-cell grass blade geometry.  grass_sdf_lod derives every blade's root,
// wind bend, lean, radius, side axis and per-segment taper from the cell id
// alone (10 sin/cos + 2 wind fields per blade, a pow per segment); only the
// final box distance depends on the query point.  A march, its 6-tap normal
// and the self-shadow march evaluate the same cell up to 13 times, so the
// invariants are computed once per cell, lazily (after the point-dependent
// rejects pass), with the identical float operation sequence.
// ---------------------------------------------------------------------------
struct GrassBladeGeom {
  v3 root;
  v2 w_xz, lean_dir;
  float lean_amt, r0;
  v3 side_hint;
};

struct GrassCellGeom {
  bool built;
  uint32_t blade_count, segs;
  float blade_len, inv_segs;
  GrassBladeGeom blade[3];
  float taper[6];
  uint64_t rec;     // table record the cell was loaded from (~0: derived)
  uint32_t frames;  // lod-0 segment frames of the record: 0 unknown, 1 ready, 2 none
};

// One blade segment's box frame (grass.wgsl:300-345): everything of the
// segment's box SDF that does not depend on the point.
struct GrassSegFrame {
  v3 mid, S, T, N;
  float half_w, half_h;
};

__device__ __forceinline__ GrassSegFrame grass_seg_frame(const GrassBladeGeom& B, float blade_len, float inv_segs,
                                                         float taper, uint32_t sg) {
  const float t01a = (float)sg * inv_segs;
  const float t01b = ((float)sg + 1.0f) * inv_segs;
  const float ya = t01a * blade_len, yb = t01b * blade_len;
  const float seg_h = yb - ya;
  const float bend_a = (blade_len * t01a) * (0.55f + 0.45f * t01a);
  const float bend_b = (blade_len * t01b) * (0.55f + 0.45f * t01b);
  const v2 bva = B.w_xz * t01a + B.lean_dir * B.lean_amt;
  const v2 bvb = B.w_xz * t01b + B.lean_dir * B.lean_amt;
  const v2 offa = bva * bend_a, offb = bvb * bend_b;
  const v3 pa = B.root + V3(offa.x, ya, offa.y);
  const v3 pb = B.root + V3(offb.x, yb, offb.y);
  GrassSegFrame f;
  f.T = normalize(pb - pa);
  v3 S = B.side_hint - f.T * dot(B.side_hint, f.T);
  const float s2 = dot(S, S);
  if (s2 < 1e-6f) S = ortho_basis_x(f.T);
  else S = S * (1.0f / sqrtf(s2));
  f.S = S;
  f.N = cross(f.T, S);
  f.mid = 0.5f * (pa + pb);
  f.half_w = B.r0 * taper * 0.7f;
  f.half_h = 0.5f * seg_h;
  return f;
}

__device__ __forceinline__ float grass_seg_sdf(const GrassSegFrame& f, v3 p) {
  const v3 d = p - f.mid;
  const v3 local = V3(dot(d, f.S), dot(d, f.T), dot(d, f.N));
  return sdf_box(local, V3s(0.0f), V3(f.half_w, f.half_h, f.half_w));
}

// Blade length of cell `id` (grass.wgsl:216).
__device__ __forceinline__ float grass_blade_len(const Scene& s, v3 id) {
  const float layer_h = GRASS_LAYER_HEIGHT_VOX * vs_(s);
  return layer_h * (0.65f + 0.35f * hash31(id + V3(9.1f, 3.7f, 5.2f)));
}

// The point-independent part of blade i of cell (cb, id) (grass.wgsl:243-298).
__device__ __noinline__ void grass_blade_geom(const Scene& s, v3 cb, v3 id, float time_s, float strength, uint32_t i,
                                              GrassBladeGeom& B) {
  const float vs = vs_(s);
  const float top_y = cb.y + vs;
  const float clump_r = 0.18f * vs;
  const float base_r = (GRASS_VOXEL_THICKNESS_VOX * vs) * 0.85f;
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
  B.root = V3(root_xz.x, top_y, root_xz.y);
  B.w_xz = 0.35f * grass_wind_xz(B.root + V3(0.0f, ph, 0.0f), time_s, strength);
  const float lean_ang = TAU * fract(u0 * 1.73f + v0 * 2.11f);
  B.lean_dir = V2(cosf_(lean_ang), sinf_(lean_ang));
  B.lean_amt = 0.10f + 0.25f * (v0 * v0);
  B.r0 = base_r * mixf(0.85f, 1.35f, wR);
  const float roll = TAU * (0.15f * ph + 0.10f * wR);
  const v2 roll_dir = V2(cosf_(roll), sinf_(roll));
  B.side_hint = normalize(V3(B.lean_dir.x * roll_dir.x - B.lean_dir.y * roll_dir.y, 0.12f,
                             B.lean_dir.x * roll_dir.y + B.lean_dir.y * roll_dir.x));
}

// Segment taper of a blade with `segs` segments (grass.wgsl:335-339).
__device__ __forceinline__ float grass_taper_value(float inv_segs, uint32_t sg) {
  const float t01a = (float)sg * inv_segs;
  const float t01b = ((float)sg + 1.0f) * inv_segs;
  const float tmid = 0.5f * (t01a + t01b);
  const float taper_shape = powf_(clampf(1.0f - tmid, 0.0f, 1.0f), 3.0f);
  return mixf(GRASS_VOXEL_TAPER, 1.0f, taper_shape);
}

__device__ __forceinline__ uint32_t grass_lod_segs(uint32_t lod) {
  uint32_t segs = to_u32(fmax_(3.0f, floorf(GRASS_VOXEL_SEGS)));
  if (lod == 1u) segs = min(segs, GRASS_SEGS_MID);
  else if (lod == 2u) segs = min(segs, GRASS_SEGS_FAR);
  return segs;
}

// Per-frame grass cell table: one record of GRASS_REC_F4 float4 per column
// (slot * 4096 + lz * 64 + lx) of every resident chunk, written each frame by
// k_grass_cells for the column's top cell when that cell is grass:
//   [0]            blade_len, cell id (x, y, z)      (id NaN: no grass top)
//   [1 + 3b .. 3b + 3]  blade b: root.xyz, w_xz.x | w_xz.y, lean_dir.xy,
//                       lean_amt | r0, side_hint.xyz
// Values are produced by the same functions as the in-march build, so a
// record and a fresh build are bit-identical.
constexpr uint32_t GRASS_REC_F4 = 10u;
constexpr uint32_t GRASS_TAPER_N = 18u;
// Lod-0 segment frames of a record (blade-major, 3 blades x 6 segments):
// (mid, half_w), (S, half_h), (T, 0) per segment; N = cross(T, S).
constexpr uint32_t GRASS_FRAME_SEGS = 18u;
constexpr uint32_t GRASS_FRAME_F4 = 3u * GRASS_FRAME_SEGS;

__device__ __forceinline__ void grass_rec_store(float4* r, float blade_len, v3 id, const GrassBladeGeom* B) {
  r[0] = make_float4(blade_len, id.x, id.y, id.z);
  for (uint32_t b = 0; b < GRASS_BLADE_COUNT; ++b) {
    r[1 + 3 * b] = make_float4(B[b].root.x, B[b].root.y, B[b].root.z, B[b].w_xz.x);
    r[2 + 3 * b] = make_float4(B[b].w_xz.y, B[b].lean_dir.x, B[b].lean_dir.y, B[b].lean_amt);
    r[3 + 3 * b] = make_float4(B[b].r0, B[b].side_hint.x, B[b].side_hint.y, B[b].side_hint.z);
  }
}

// Loads cell (cb, id) from the table when the pass has one, the column's
// record is this cell and cb is the id * vs the record was built from (some
// callers derive cb from the chunk origin instead, which may differ in the
// last bit); false means "derive it".
__device__ __noinline__ bool grass_table_load(const Scene& s, v3 cb, v3 id, GrassCellGeom& G) {
  if (s.grass_rec == nullptr) return false;
  const v3 cb_rec = id * vs_(s);
  if (__float_as_uint(cb_rec.x) != __float_as_uint(cb.x) || __float_as_uint(cb_rec.y) != __float_as_uint(cb.y) ||
      __float_as_uint(cb_rec.z) != __float_as_uint(cb.z))
    return false;
  const int32_t cs = (int32_t)s.cam->chunk_size;
  if (cs <= 0) return false;
  const int32_t wx = __float2int_rz(id.x), wy = __float2int_rz(id.y), wz = __float2int_rz(id.z);
  auto fdiv = [cs](int32_t a) { return a >= 0 ? a / cs : -((-a + cs - 1) / cs); };
  const uint32_t slot = grid_lookup_slot(s, fdiv(wx), fdiv(wy), fdiv(wz));
  if (slot == INVALID || slot >= s.cam->chunk_count) return false;
  const Meta m = meta_at(s, slot);
  const int32_t lx = wx - m.ox, lz = wz - m.oz;
  if (lx < 0 || lx > 63 || lz < 0 || lz > 63) return false;
  const uint64_t e = (uint64_t)slot * 4096u + (uint64_t)(lz * 64 + lx);
  if (e >= s.grass_rec_n) return false;
  const float4* r = s.grass_rec + e * GRASS_REC_F4;
  const float4 h = r[0];
  if (__float_as_uint(h.y) != __float_as_uint(id.x) || __float_as_uint(h.z) != __float_as_uint(id.y) ||
      __float_as_uint(h.w) != __float_as_uint(id.z))
    return false;
  G.rec = e;
  G.blade_len = h.x;
  for (uint32_t b = 0; b < G.blade_count; ++b) {
    const float4 a = r[1 + 3 * b], c = r[2 + 3 * b], d = r[3 + 3 * b];
    GrassBladeGeom& B = G.blade[b];
    B.root = V3(a.x, a.y, a.z);
    B.w_xz = V2(a.w, c.x);
    B.lean_dir = V2(c.y, c.z);
    B.lean_amt = c.w;
    B.r0 = d.x;
    B.side_hint = V3(d.y, d.z, d.w);
  }
  return true;
}

__device__ __noinline__ void grass_cell_build(const Scene& s, v3 cb, v3 id, float time_s, float strength, uint32_t lod,
                                              GrassCellGeom& G) {
  uint32_t blade_count = GRASS_BLADE_COUNT;
  if (lod == 1u) blade_count = min(blade_count, GRASS_BLADE_COUNT_MID);
  else if (lod == 2u) blade_count = min(blade_count, GRASS_BLADE_COUNT_FAR);
  const uint32_t segs = grass_lod_segs(lod);
  G.blade_count = blade_count;
  G.segs = segs;
  G.inv_segs = 1.0f / fmax_((float)segs, 1.0f);
  G.rec = ~0ull;
  G.frames = 2u;
  if (s.grass_taper != nullptr && lod < 3u) {
    for (uint32_t sg = 0; sg < segs; ++sg) G.taper[sg] = s.grass_taper[lod * 6u + sg];
  } else {
    for (uint32_t sg = 0; sg < segs; ++sg) G.taper[sg] = grass_taper_value(G.inv_segs, sg);
  }
  if (!grass_table_load(s, cb, id, G)) {
    G.blade_len = grass_blade_len(s, id);
    for (uint32_t i = 0; i < blade_count; ++i) grass_blade_geom(s, cb, id, time_s, strength, i, G.blade[i]);
  } else if (lod == 0u && s.grass_state != nullptr && blade_count * segs == GRASS_FRAME_SEGS) {
    G.frames = 0u;
  }
  G.built = true;
}

__device__ __forceinline__ uint32_t ld_acquire_gpu(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release_gpu(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Makes the record's lod-0 segment frames usable: ready already, or built
// here by the first lane to claim them (the same grass_seg_frame values every
// march would compute).  A lane that finds another one building them goes on
// without (false) and asks again at its next evaluation; nothing waits.
__device__ __noinline__ bool grass_frames_ready(const Scene& s, GrassCellGeom& G) {
  uint32_t* st = s.grass_state + G.rec;
  const uint32_t v = ld_acquire_gpu(st);
  if (v == 2u) {
    G.frames = 1u;
    return true;
  }
  if (v != 0u || atomicCAS(st, 0u, 1u) != 0u) return false;
  float4* F = s.grass_frames + G.rec * GRASS_FRAME_F4;
  for (uint32_t i = 0; i < G.blade_count; ++i)
    for (uint32_t sg = 0; sg < G.segs; ++sg) {
      const GrassSegFrame f = grass_seg_frame(G.blade[i], G.blade_len, G.inv_segs, G.taper[sg], sg);
      float4* o = F + 3u * (i * G.segs + sg);
      o[0] = make_float4(f.mid.x, f.mid.y, f.mid.z, f.half_w);
      o[1] = make_float4(f.S.x, f.S.y, f.S.z, f.half_h);
      o[2] = make_float4(f.T.x, f.T.y, f.T.z, 0.0f);
    }
  st_release_gpu(st, 2u);
  G.frames = 1u;
  return true;
}

// grass_sdf_lod (grass.wgsl:192-350) over the cached cell geometry.
__device__ __noinline__ float grass_sdf_cached(const Scene& s, v3 p, v3 cb, v3 id, float time_s, float strength,
                                               uint32_t lod, GrassCellGeom& G) {
  const float vs = vs_(s);
  const float top_y = cb.y + vs;
  const float layer_h = GRASS_LAYER_HEIGHT_VOX * vs;
  const float y01 = (p.y - top_y) / fmax_(layer_h, 1e-6f);
  if (y01 < 0.0f || y01 > 1.0f) return BIG;
  const float over = GRASS_OVERHANG_VOX * vs;
  if (p.x < cb.x - over || p.x > cb.x + vs + over || p.z < cb.z - over || p.z > cb.z + vs + over) return BIG;
  if (!G.built) grass_cell_build(s, cb, id, time_s, strength, lod, G);
  float dmin = BIG;
  if (G.frames == 1u || (G.frames == 0u && grass_frames_ready(s, G))) {
    const float4* F = s.grass_frames + G.rec * GRASS_FRAME_F4;
#pragma unroll 6
    for (uint32_t k = 0; k < GRASS_FRAME_SEGS; ++k) {
      const float4 a = F[3u * k], b = F[3u * k + 1u], c = F[3u * k + 2u];
      GrassSegFrame f;
      f.mid = V3(a.x, a.y, a.z);
      f.S = V3(b.x, b.y, b.z);
      f.T = V3(c.x, c.y, c.z);
      f.N = cross(f.T, f.S);
      f.half_w = a.w;
      f.half_h = b.w;
      dmin = fmin_(dmin, grass_seg_sdf(f, p));
    }
    return dmin;
  }
  for (uint32_t i = 0; i < G.blade_count; ++i)
    for (uint32_t sg = 0; sg < G.segs; ++sg)
      dmin = fmin_(dmin, grass_seg_sdf(grass_seg_frame(G.blade[i], G.blade_len, G.inv_segs, G.taper[sg], sg), p));
  return dmin;
}

__device__ __noinline__ v3 grass_sdf_normal_lod(const Scene& s, v3 p, v3 cb, v3 id, float time_s, float strength,
                                                uint32_t lod, GrassCellGeom& G) {
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
  const float dx = grass_sdf_cached(s, p + V3(e, 0.0f, 0.0f), cb, id, time_s, strength, lod, G) -
                   grass_sdf_cached(s, p - V3(e, 0.0f, 0.0f), cb, id, time_s, strength, lod, G);
  const float dy = grass_sdf_cached(s, p + V3(0.0f, e, 0.0f), cb, id, time_s, strength, lod, G) -
                   grass_sdf_cached(s, p - V3(0.0f, e, 0.0f), cb, id, time_s, strength, lod, G);
  const float dz = grass_sdf_cached(s, p + V3(0.0f, 0.0f, e), cb, id, time_s, strength, lod, G) -
                   grass_sdf_cached(s, p - V3(0.0f, 0.0f, e), cb, id, time_s, strength, lod, G);
  return normalize(V3(dx, dy, dz));
}

__device__ __noinline__ float grass_self_shadow(const Scene& s, v3 hp, v3 cb, v3 id, float time_s, float strength, uint32_t lod) {
  // grass.wgsl:410-447
  const float vs = vs_(s);
  GrassCellGeom G;
  G.built = false;
  v3 p = hp + SUN_DIR * (0.02f * vs);
  const float max_dist = (0.55f + 0.35f * (float)lod) * vs;
  const uint32_t steps = lod != 0u ? 4u : 6u;
  const float dt = max_dist / (float)steps;
  float occ = 0.0f;
  for (uint32_t i = 0; i < steps; ++i) {
    const float d = grass_sdf_cached(s, p, cb, id, time_s, strength, lod, G);
    occ += clampf(1.0f - d / (0.05f * vs), 0.0f, 1.0f);
    p = p + SUN_DIR * dt;
  }
  return expf_(-0.35f * occ);
}

__device__ __forceinline__ uint32_t grass_lod_from_t(float t) {  // grass.wgsl:540-545
  if (t >= GRASS_LOD_FAR_START) return 2u;
  if (t >= GRASS_LOD_MID_START) return 1u;
  return 0u;
}

__device__ __noinline__ GrassHit grass_layer_trace_lod(const Scene& s, v3 ro, v3 rd, float t_start, float t_end, v3 cb, v3 id, float time_s,
                               float strength, uint32_t lod) {  // grass.wgsl:456-491
  const float vs = vs_(s);
  GrassCellGeom G;
  G.built = false;
  float t = t_start;
  uint32_t steps = GRASS_TRACE_STEPS;
  if (lod == 1u) steps = GRASS_TRACE_STEPS_MID;
  if (lod == 2u) steps = GRASS_TRACE_STEPS_FAR;
  for (uint32_t i = 0; i < steps; ++i) {
    if (t > t_end) break;
    const v3 p = ro + rd * t;
    const float d = grass_sdf_cached(s, p, cb, id, time_s, strength, lod, G);
    if (d < GRASS_HIT_EPS_VOX * vs) {
      return GrassHit{true, t, grass_sdf_normal_lod(s, p, cb, id, time_s, strength, lod, G)};
    }
    t += fmax_(d, GRASS_STEP_MIN_VOX * vs);
  }
  return GrassHit{false, BIG, V3s(0.0f)};
}

// The part of [t_min, t_max] inside the cell's grass slab and before the
// cell's own voxel (grass.wgsl:494-535); empty when t1 <= t0.
__device__ __forceinline__ v2 grass_slab_interval(v3 ro, v3 rd, float t_min, float t_max, v3 cb, float vs) {
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
  return V2(t0, t1);
}

__device__ __noinline__ GrassHit try_grass_slab_hit(const Scene& s, v3 ro, v3 rd, float t_min, float t_max, v3 cb, v3 id, float vs,
                            float time_s, float strength) {  // grass.wgsl:494-538
  const v2 iv = grass_slab_interval(ro, rd, t_min, t_max, cb, vs);
  if (iv.y <= iv.x) return GrassHit{false, BIG, V3s(0.0f)};
  return grass_layer_trace_lod(s, ro, rd, iv.x, iv.y, cb, id, time_s, strength, grass_lod_from_t(iv.x));
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

__device__ __forceinline__ HitGeom miss_hitgeom() {  // chunk_trace.wgsl:40-51
  HitGeom h;
  h.hit = 0; h.mat = MAT_AIR; h.t = BIG; h.n = V3s(0.0f); h.root_bmin = V3s(0.0f); h.root_size = 0.0f;
  h.node_base = 0; h.macro_base = INVALID; h.node = INVALID; h.leaf_bmin = V3s(0.0f); h.leaf_size = 0.0f;
  return h;
}

// A chunk walk's result.  `gov`: the hit is a grass voxel whose blade march
// (grass_on_voxel_hit over [gov_t0, gov_t1]) the walk left to a later pass;
// that march may replace the hit's t and n.
struct ChunkTraceResult {
  HitGeom hit;
  bool anchor_valid;
  uint32_t anchor_key;
  bool gov = false;
  float gov_t0 = 0.0f, gov_t1 = 0.0f;  // the walk's interval, for the march
  float gov_lo = 0.0f, gov_hi = 0.0f;  // the march's slab interval: its hit t lies in it
};

__device__ __forceinline__ bool point_in_cube(v3 p, v3 bmin, float size) {  // chunk_trace.wgsl:54-59
  const v3 bmax = bmin + V3s(size);
  return p.x >= bmin.x && p.x < bmax.x && p.y >= bmin.y && p.y < bmax.y && p.z >= bmin.z && p.z < bmax.z;
}

__device__ __forceinline__ uint32_t node_level(uint32_t k) { return (k >> 18) & 7u; }
__device__ __forceinline__ uint32_t node_x(uint32_t k) { return k & 63u; }
__device__ __forceinline__ uint32_t node_y(uint32_t k) { return (k >> 6) & 63u; }
__device__ __forceinline__ uint32_t node_z(uint32_t k) { return (k >> 12) & 63u; }

__device__ __forceinline__ v4 node_cube_from_key(v3 rb, float rs, uint32_t key) {  // chunk_trace.wgsl:123-128
  const float sz = rs / (float)(1u << node_level(key));
  const v3 b = rb + V3((float)node_x(key), (float)node_y(key), (float)node_z(key)) * sz;
  return v4{b.x, b.y, b.z, sz};
}

struct AnchorNode { bool valid; uint32_t idx; v3 bmin; float size; uint32_t key; };

__device__ __noinline__ AnchorNode anchor_from_key(const Scene& s, uint32_t node_base, v3 rb, float rs, uint32_t key) {
  // chunk_trace.wgsl:138-191
  if (key == INVALID) return AnchorNode{false, 0, V3s(0.0f), 0.0f, INVALID};
  const uint32_t lvl = min(node_level(key), chunk_max_depth(s));
  const uint32_t tx = node_x(key), ty = node_y(key), tz = node_z(key);
  uint32_t idx = 0;
  v3 bmin = rb;
  float size = rs;
  for (uint32_t d = 0; d < 32; ++d) {
    if (d >= lvl) return AnchorNode{true, idx, bmin, size, node_key(s, node_base, idx)};
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
  return AnchorNode{true, idx, bmin, size, node_key(s, node_base, idx)};
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

__device__ AnchorNode anchor_from_leaf(const Scene& s, const LeafState& l, uint32_t node_base) {  // chunk_trace.wgsl:193-203
  if (l.has_node) return AnchorNode{true, l.idx_local, l.bmin, l.size, node_key(s, node_base, l.idx_local)};
  if (l.has_anchor)
    return AnchorNode{true, l.anchor_idx, l.anchor_bmin, l.anchor_size, node_key(s, node_base, l.anchor_idx)};
  return AnchorNode{false, 0, V3s(0.0f), 0.0f, INVALID};
}

struct ExitFaceRes { uint32_t face, amb; };

__device__ ExitFaceRes exit_face_from_slab_safe(v3 rd, const CubeSlab& slab) {  // chunk_trace.wgsl:233-272
  const float te = slab.t_exit;
  const float eps = 1e-5f * fmax_(1.0f, fabsf(te));
  const bool mx = fabsf(rd.x) >= EPS_INV && fabsf(slab.tmaxv.x - te) <= eps;
  const bool my = fabsf(rd.y) >= EPS_INV && fabsf(slab.tmaxv.y - te) <= eps;
  const bool mz = fabsf(rd.z) >= EPS_INV && fabsf(slab.tmaxv.z - te) <= eps;
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

__device__ __forceinline__ LeafState descend_leaf_sparse(const Scene& s, v3 p, uint32_t node_base, uint32_t start_idx, v3 start_bmin,
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

__device__ __noinline__ LeafState descend_leaf_sparse_ool(const Scene& s, v3 p, uint32_t node_base, uint32_t start_idx,
                                                         v3 start_bmin, float start_size) {
  return descend_leaf_sparse(s, p, node_base, start_idx, start_bmin, start_size);
}

struct MacroDDAState {
  bool enabled;
  int32_t mx, my, mz, step_x, step_y, step_z;
  float tMaxX, tMaxY, tMaxZ, tDeltaX, tDeltaY, tDeltaZ, cell;
};

__device__ __forceinline__ MacroDDAState macro_dda_init(v3 ro, v3 rd, v3 inv, float tcur, v3 rb, float rs, uint32_t macro_base) {
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
  const int32_t mx = to_i32(floorf(lp.x / cell)), my = to_i32(floorf(lp.y / cell)),
                mz = to_i32(floorf(lp.z / cell));
  if (mx < 0 || my < 0 || mz < 0 || mx >= 8 || my >= 8 || mz >= 8) return st;
  st.enabled = true;
  st.mx = mx; st.my = my; st.mz = mz;
  st.step_x = rd.x > 0.0f ? 1 : -1;
  st.step_y = rd.y > 0.0f ? 1 : -1;
  st.step_z = rd.z > 0.0f ? 1 : -1;
  st.tDeltaX = fabsf(cell * inv.x);
  st.tDeltaY = fabsf(cell * inv.y);
  st.tDeltaZ = fabsf(cell * inv.z);
  st.cell = cell;
  if (fabsf(rd.x) >= EPS_INV) {
    const float bx = rb.x + (float)(mx + (rd.x > 0.0f ? 1 : 0)) * cell;
    st.tMaxX = tcur + (bx - p.x) * inv.x;
  }
  if (fabsf(rd.y) >= EPS_INV) {
    const float by = rb.y + (float)(my + (rd.y > 0.0f ? 1 : 0)) * cell;
    st.tMaxY = tcur + (by - p.y) * inv.y;
  }
  if (fabsf(rd.z) >= EPS_INV) {
    const float bz = rb.z + (float)(mz + (rd.z > 0.0f ? 1 : 0)) * cell;
    st.tMaxZ = tcur + (bz - p.z) * inv.z;
  }
  return st;
}

__device__ __forceinline__ float macro_dda_t_exit(const MacroDDAState& st) { return fmin_(st.tMaxX, fmin_(st.tMaxY, st.tMaxZ)); }

__device__ void macro_dda_step(MacroDDAState& st) {  // chunk_trace.wgsl:536-559
  const float tn = macro_dda_t_exit(st);
  const float e = 1e-6f * fmax_(1.0f, fabsf(tn));
  if (fabsf(st.tMaxX - tn) <= e) { st.mx += st.step_x; st.tMaxX += st.tDeltaX; }
  if (fabsf(st.tMaxY - tn) <= e) { st.my += st.step_y; st.tMaxY += st.tDeltaY; }
  if (fabsf(st.tMaxZ - tn) <= e) { st.mz += st.step_z; st.tMaxZ += st.tDeltaZ; }
  if (st.mx < 0 || st.my < 0 || st.mz < 0 || st.mx >= 8 || st.my >= 8 || st.mz >= 8) st.enabled = false;
}

__device__ void macro_dda_sync(MacroDDAState& st, float tcur) {  // chunk_trace.wgsl:561-568
  for (uint32_t i = 0; i < 32; ++i) {
    if (!st.enabled) break;
    if (tcur < macro_dda_t_exit(st)) break;
    macro_dda_step(st);
  }
}

struct MacroStep { bool valid, empty; float t_exit; };

__device__ MacroStep macro_dda_current(const Scene& s, const MacroDDAState& st, uint32_t macro_base) {  // chunk_trace.wgsl:570-587
  MacroStep o{st.enabled, false, macro_dda_t_exit(st)};
  if (!st.enabled || macro_base == INVALID) { o.valid = false; return o; }
  o.empty = !macro_test(s, macro_base, macro_bit_index((uint32_t)st.mx, (uint32_t)st.my, (uint32_t)st.mz));
  return o;
}

// colinfo (chunk_trace.wgsl:1284-1308)
__device__ __forceinline__ uint32_t colinfo_entry_u16(const Scene& s, uint32_t base, uint32_t lx, uint32_t lz) {
  const uint32_t idx = lz * 64u + lx;
  const uint32_t word = colinfo_word(s, base + (idx >> 1));
  return (idx & 1u) == 0u ? (word & 0xFFFFu) : ((word >> 16) & 0xFFFFu);
}
struct ColInfo { bool valid; uint32_t y_vox, mat; };
__device__ __forceinline__ ColInfo colinfo_decode(uint32_t e) {
  const uint32_t y8 = e & 0xFFu, m8 = (e >> 8) & 0xFFu;
  if (y8 == 255u) return ColInfo{false, 0, 0};
  return ColInfo{true, y8, m8};
}

// The column DDA of probe_grass_columns_xz_dda (chunk_trace.wgsl:1358-1504):
// calls visit(it, t, tNext, id) for every grass column (in DDA order, `it`
// the iteration) whose grass slab the ray segment [t, tNext] overlaps in y;
// stops when visit returns true.
template <class F>
__device__ __forceinline__ void grass_columns_dda(const Scene& s, v3 ro, v3 rd, v3 inv, float t0_in, float t1_in,
                                                  v3 rb, i3 origin_vox, float vs, uint32_t colinfo_base, F&& visit) {
  const float t0 = t0_in, t1 = t1_in;
  if (t1 <= t0) return;
  const float eps = 1e-4f * vs;
  float t = t0 + eps;
  if (t > t1) t = t0;
  v3 p = ro + rd * t;
  int32_t lx = to_i32(floorf((p.x - rb.x) / vs)), lz = to_i32(floorf((p.z - rb.z) / vs));
  lx = clampi(lx, 0, 63);
  lz = clampi(lz, 0, 63);
  const int32_t stepX = rd.x > 0.0f ? 1 : -1, stepZ = rd.z > 0.0f ? 1 : -1;
  float tMaxX = BIG, tDeltaX = BIG, tMaxZ = BIG, tDeltaZ = BIG;
  if (fabsf(rd.x) >= EPS_INV) {
    const float nextX = rb.x + (float)(stepX > 0 ? lx + 1 : lx) * vs;
    tMaxX = t + (nextX - p.x) * inv.x;
    tDeltaX = vs * fabsf(inv.x);
  }
  if (fabsf(rd.z) >= EPS_INV) {
    const float nextZ = rb.z + (float)(stepZ > 0 ? lz + 1 : lz) * vs;
    tMaxZ = t + (nextZ - p.z) * inv.z;
    tDeltaZ = vs * fabsf(inv.z);
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
        if (visit(it, t, tNext, id)) return;
      }
    }
    if (tNext >= t1) break;
    const float tStep = fmin_(tMaxX, tMaxZ);
    const float epsTie = 1e-6f * fmax_(1.0f, fabsf(tStep));
    if (fabsf(tMaxX - tStep) <= epsTie) { lx += stepX; tMaxX += tDeltaX; }
    if (fabsf(tMaxZ - tStep) <= epsTie) { lz += stepZ; tMaxZ += tDeltaZ; }
    t = tStep + eps;
    if (lx < 0 || lx > 63 || lz < 0 || lz > 63) break;
    p = ro + rd * t;
  }
}

__device__ __noinline__ GrassHit probe_grass_columns_xz_dda(const Scene& s, v3 ro, v3 rd, v3 inv, float t0_in, float t1_in, v3 rb,
                                    i3 origin_vox, float vs, uint32_t colinfo_base, float time_s,
                                    float strength) {  // chunk_trace.wgsl:1358-1504
  GrassHit out{false, BIG, V3s(0.0f)};
  grass_columns_dda(s, ro, rd, inv, t0_in, t1_in, rb, origin_vox, vs, colinfo_base,
                    [&](uint32_t, float t, float tNext, v3 id) {
                      const GrassHit gh = try_grass_slab_hit(s, ro, rd, t, tNext, id * vs, id, vs, time_s, strength);
                      if (gh.hit) out = gh;
                      return gh.hit;
                    });
  return out;
}

struct TraceOpts { bool geom_only; };

__device__ __forceinline__ HitGeom make_hit(uint32_t mat, float t, v3 n, v3 rb, float rs, const Meta& ch, uint32_t node,
                        v3 lb, float ls) {
  HitGeom o = miss_hitgeom();
  o.hit = 1; o.t = t; o.mat = mat; o.n = n; o.root_bmin = rb; o.root_size = rs; o.node_base = ch.node_base;
  o.macro_base = ch.macro_base; o.node = node; o.leaf_bmin = lb; o.leaf_size = ls;
  return o;
}

// ---------------------------------------------------------------------------
// Grass column probes of the leaf walk.
//
// The walk (chunk_trace.wgsl:669-961) probes the grass columns of every small
// air leaf it crosses and ends the chunk at the first probe that hits.  The
// probes are most of the primary trace's work and are reached by single lanes
// deep inside divergent walks, so the wavefront schedule runs them apart:
//   PROBE_RECORD  the walk stores each probe (interval, chunk, and the leaf and
//                 anchor state a hit record needs) and goes on as if it missed;
//   k_probe_dda   runs each stored probe's column DDA, one lane each, and
//                 stores one task per grass slab it meets;
//   k_slab_eval   marches every slab, one lane each;
//   resolve       rebuilds the candidate loop's answer from the parts.
// Why the parts suffice: the candidate loop keeps the nearest chunk result
// (earliest chunk on ties) and a chunk's result is its first probe hit, else
// its voxel hit.  A chunk walk does not depend on the loop's best so far, so
// every chunk the reference walks is walked identically here (here fewer
// chunks are skipped, as probe hits never lower the best).  Along one walk
// probe intervals follow each other in t (up to rounding where one leaf's exit
// meets the next: k_slab_pick sends those rare pixels to the inline walk), so
// a chunk's first probe hit is also its nearest; the answer is therefore
// the nearer of the nearest probe hit over all chunks (key: t, chunk, probe,
// column) and the walk's voxel answer, unless the voxel answer wins while its own chunk had a probe hit
// (its grass-slab refinement reached below that hit): such pixels, and pixels
// whose probes did not all fit the buffers, walk again with inline probes.
// PROBE_INLINE is the reference order (megakernel, batches, queries, that
// fallback).
// ---------------------------------------------------------------------------
enum : uint32_t { PROBE_INLINE = 0u, PROBE_RECORD = 1u };
// The walk functions take the mode as a template argument (PM) so that a
// kernel holds only the probe code it runs; PROBE_DYNAMIC reads ph.mode.
constexpr uint32_t PROBE_DYNAMIC = 2u;

// A stored probe: three 16-byte words, written and read as vectors.
struct __align__(16) ProbeRec {
  uint32_t pixel, slot;
  float t0, t1;
  uint32_t tag;         // probe order (20 bits; PROBE_SEQ_LOST: beyond what it counts) | candidate index << 20
                        // | trace phase << 25 (0 hint window, 1 full) | anchor valid << 26
  uint32_t node;        // hit-record leaf node (INVALID: implicit leaf)
  uint32_t anchor_key;
  float leaf_size;
  float leaf_bmin[3];
  uint32_t _pad;
};
constexpr uint32_t PROBE_SEQ_LOST = 0xFFFFFu;

// A grass slab to march (16 B): its probe, the column (x, z within the
// probe's chunk, the column top's y within the chunk) and the column DDA
// step, and the part of the step's interval inside the slab
// (grass_slab_interval).  The cell id is the chunk origin + those offsets,
// the same integers the column DDA converted.
__device__ __forceinline__ uint4 slab_task(uint32_t probe, uint32_t it, float t, float t_next, v3 id, const Meta& ch) {
  const uint32_t lx = (uint32_t)((int32_t)id.x - ch.ox), ly = (uint32_t)((int32_t)id.y - ch.oy),
                 lz = (uint32_t)((int32_t)id.z - ch.oz);
  return make_uint4(probe, (lx & 63u) | ((lz & 63u) << 6) | ((ly & 63u) << 12) | ((it & 63u) << 18),
                    __float_as_uint(t), __float_as_uint(t_next));
}
__device__ __forceinline__ uint32_t slab_task_step(const uint4& a) { return (a.y >> 18) & 63u; }
__device__ __forceinline__ v3 slab_task_cell(const uint4& a, const Meta& ch) {
  return V3((float)(ch.ox + (int32_t)(a.y & 63u)), (float)(ch.oy + (int32_t)((a.y >> 12) & 63u)),
            (float)(ch.oz + (int32_t)((a.y >> 6) & 63u)));
}
__device__ __forceinline__ uint32_t probe_seq(const ProbeRec& r) { return r.tag & 0xFFFFFu; }
__device__ __forceinline__ uint32_t probe_cand(const ProbeRec& r) { return (r.tag >> 20) & 31u; }
__device__ __forceinline__ uint32_t probe_phase(const ProbeRec& r) { return (r.tag >> 25) & 1u; }
__device__ __forceinline__ bool probe_anchor_valid(const ProbeRec& r) { return ((r.tag >> 26) & 1u) != 0u; }

struct ProbeHook {
  uint32_t mode;
  uint32_t seq;        // probes met so far, in walk order
  uint32_t slot;       // chunk slot of the walk in progress
  uint32_t cand;       // its index in the candidate list
  uint32_t phase;      // 0 hint-window trace, 1 full trace
  uint32_t first_phase;  // phase the primary trace started in (2: it did not trace)
  uint32_t best_cand;  // candidate index of the trace's current best (INVALID: none)
  uint32_t pixel;
  uint32_t recorded;   // probes stored
  bool defer_gov;      // leave the blade march of a grass-voxel hit to a later pass
  ProbeRec* recs;
  uint32_t* rec_count;
  uint32_t rec_cap;
};

__device__ __forceinline__ ProbeHook probe_hook_inline() {
  ProbeHook h;
  h.mode = PROBE_INLINE;
  h.seq = 0u;
  h.slot = INVALID;
  h.cand = 0u;
  h.phase = 1u;
  h.first_phase = 2u;
  h.best_cand = INVALID;
  h.pixel = 0u;
  h.recorded = 0u;
  h.defer_gov = false;
  h.recs = nullptr;
  h.rec_count = nullptr;
  h.rec_cap = 0u;
  return h;
}

// Stores this lane's probe; lanes that reach the store together share one
// atomic.
__device__ __forceinline__ void probe_record(ProbeHook& ph, float t0, float t1, uint32_t node, v3 leaf_bmin,
                                             float leaf_size, bool anchor_valid, uint32_t anchor_key) {
  if (ph.recs == nullptr) return;  // counting only
  const uint32_t mask = __activemask();
  const uint32_t lane = threadIdx.x & 31u, leader = __ffs(mask) - 1u;
  uint32_t base = 0u;
  if (lane == leader) base = atomicAdd(ph.rec_count, (uint32_t)__popc(mask));
  base = __shfl_sync(mask, base, leader);
  const uint32_t idx = base + (uint32_t)__popc(mask & ((1u << lane) - 1u));
  if (idx < ph.rec_cap) {
    const uint32_t tag = min(ph.seq, PROBE_SEQ_LOST) | ((ph.cand & 31u) << 20) | ((ph.phase & 1u) << 25) |
                         (anchor_valid ? (1u << 26) : 0u);
    uint4* d = reinterpret_cast<uint4*>(ph.recs + idx);
    d[0] = make_uint4(ph.pixel, ph.slot, __float_as_uint(t0), __float_as_uint(t1));
    d[1] = make_uint4(tag, node, anchor_key, __float_as_uint(leaf_size));
    d[2] = make_uint4(__float_as_uint(leaf_bmin.x), __float_as_uint(leaf_bmin.y), __float_as_uint(leaf_bmin.z), 0u);
    ++ph.recorded;
  }
}

// The blades on top of a grass voxel the walk hit at (t, n)
// (chunk_trace.wgsl:917-950): the cell from the hit point, corrected by the
// column's colinfo top, then its grass slab from just before the hit.  This
// part gives the cell and the slab interval the march would cover
// (try_grass_slab_hit's first step); empty when y <= x.
__device__ __forceinline__ v2 grass_on_voxel_interval(const Scene& s, v3 ro, v3 rd, const Meta& ch, float t, v3 n,
                                                     float t_enter, float t_exit, GrassCell* cell_out) {
  const float vs = vs_(s);
  const v3 rb = V3((float)ch.ox, (float)ch.oy, (float)ch.oz) * vs;
  const i3 ov{ch.ox, ch.oy, ch.oz};
  const v3 hp = ro + rd * t;
  GrassCell cell = pick_grass_cell_in_chunk_with_bias(hp, n, rb, ov, vs, (int32_t)s.cam->chunk_size);
  if (ch.colinfo_base != INVALID) {
    int32_t lx = to_i32(floorf((hp.x - rb.x) / vs)), lz = to_i32(floorf((hp.z - rb.z) / vs));
    lx = clampi(lx, 0, 63);
    lz = clampi(lz, 0, 63);
    const ColInfo ci = colinfo_decode(colinfo_entry_u16(s, ch.colinfo_base, (uint32_t)lx, (uint32_t)lz));
    if (ci.valid && ci.mat == MAT_GRASS) {
      const v3 id = V3((float)(ov.x + lx), (float)(ov.y + (int32_t)ci.y_vox), (float)(ov.z + lz));
      cell = GrassCell{id * vs, id};
    }
  }
  const float pad = (GRASS_LAYER_HEIGHT_VOX + 1.0f) * vs;
  const float tmn = fmax_(t_enter, t - 0.01f * vs);
  const float tmx = fmin_(t + pad, t_exit + pad);
  *cell_out = cell;
  return grass_slab_interval(ro, rd, tmn, tmx, cell.bmin_m, vs);
}

// ... and the march over it (try_grass_slab_hit).
__device__ __noinline__ GrassHit grass_on_voxel_hit(const Scene& s, v3 ro, v3 rd, const Meta& ch, float t, v3 n,
                                                    float t_enter, float t_exit) {
  GrassCell cell;
  const v2 iv = grass_on_voxel_interval(s, ro, rd, ch, t, n, t_enter, t_exit, &cell);
  if (iv.y <= iv.x) return GrassHit{false, BIG, V3s(0.0f)};
  return grass_layer_trace_lod(s, ro, rd, iv.x, iv.y, cell.bmin_m, cell.id_vox, s.cam->voxel_params[1],
                               s.cam->voxel_params[2], grass_lod_from_t(iv.x));
}

template <uint32_t PM>
__device__ __forceinline__ ChunkTraceResult trace_chunk_rope_interval_nomacro(const Scene& s, v3 ro, v3 rd, v3 inv, const Meta& ch,
                                                   float t_enter, float t_exit, bool use_anchor,
                                                   uint32_t anchor_key, const TraceOpts& opt, ProbeHook& ph) {
  // chunk_trace.wgsl:669-961
  const float vs = vs_(s);
  const v3 rb = V3((float)ch.ox, (float)ch.oy, (float)ch.oz) * vs;
  const float rs = (float)s.cam->chunk_size * vs;
  const float eps_step = 1e-4f * vs;
  float tcur = fmax_(t_enter, 0.0f) + eps_step;
  AnchorNode an{false, 0, V3s(0.0f), 0.0f, INVALID};
  if (use_anchor) an = anchor_from_key(s, ch.node_base, rb, rs, anchor_key);
  const float grass_probe_max_leaf = 8.0f * vs;
  const i3 ov{ch.ox, ch.oy, ch.oz};
  const float time_s = s.cam->voxel_params[1], strength = s.cam->voxel_params[2];
  bool have_leaf = false;
  LeafState leaf{};
  // A descent chosen at the end of an air step (rope neighbour or anchor) is
  // made at the top of the next iteration, at the same point, so that the walk
  // has one descent site.
  bool pend = false, pend_anchor = false;
  uint32_t pend_idx = 0u;
  v3 pend_bmin = V3s(0.0f);
  float pend_size = 0.0f;
  const uint32_t MAX_ITERS = 128u + s.cam->chunk_size * 2u;
  for (uint32_t it = 0; it < MAX_ITERS; ++it) {
    if (tcur > t_exit) break;
    const v3 p = ro + rd * tcur;
    const v3 pq = p + ray_eps_vec(rd, 1e-4f * vs);
    // the pending descent (the one the reference makes at the end of the
    // previous iteration), then the reference's check at the top of an
    // iteration: a re-descent from the anchor or the root when the leaf does
    // not hold the point.  That re-descent is not checked again.
    for (uint32_t pass = 0; pass < 2u; ++pass) {
      uint32_t si;
      v3 sb;
      float ss;
      bool upd = true;
      const bool pending = pend;
      if (pend) {
        si = pend_idx;
        sb = pend_bmin;
        ss = pend_size;
        upd = pend_anchor;
        pend = false;
      } else if (!have_leaf || !point_in_cube(pq, leaf.bmin, leaf.size)) {
        const bool use_an = an.valid && point_in_cube(pq, an.bmin, an.size);
        si = use_an ? an.idx : 0u;
        sb = use_an ? an.bmin : rb;
        ss = use_an ? an.size : rs;
      } else {
        break;
      }
      leaf = descend_leaf_sparse(s, pq, ch.node_base, si, sb, ss);
      if (upd) {
        const AnchorNode na = anchor_from_leaf(s, leaf, ch.node_base);
        if (na.valid && (!an.valid || na.key != an.key)) an = na;
      }
      have_leaf = true;
      if (!pending) break;
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
            GrassHit gh{false, BIG, V3s(0.0f)};
            const bool rec = PM == PROBE_DYNAMIC ? ph.mode == PROBE_RECORD : PM == PROBE_RECORD;
            if (rec)
              probe_record(ph, t0p, t1p, leaf.has_node ? ch.node_base + leaf.idx_local : INVALID, leaf.bmin,
                           leaf.size, an.valid, an.key);
            else
              gh = probe_grass_columns_xz_dda(s, ro, rd, inv, t0p, t1p, rb, ov, vs, ch.colinfo_base, time_s, strength);
            ++ph.seq;
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
      // the next point (ro + rd * tcur + nudge) is the next iteration's pq
      if (!leaf.has_node && !leaf.has_anchor) {
        have_leaf = false;
        continue;
      }
      if (!leaf.has_node) {
        // an implicit air leaf: back into its anchor when the point is there
        const v3 pqn = (ro + rd * tcur) + ray_eps_vec(rd, 1e-4f * vs);
        if (point_in_cube(pqn, leaf.anchor_bmin, leaf.anchor_size)) {
          pend = true;
          pend_anchor = false;
          pend_idx = leaf.anchor_idx;
          pend_bmin = leaf.anchor_bmin;
          pend_size = leaf.anchor_size;
          continue;
        }
      }
      // the rope of the leaf's node, or of the implicit leaf's anchor
      const uint32_t nidx = rope_face(s, ch.node_base + (leaf.has_node ? leaf.idx_local : leaf.anchor_idx), face);
      if (nidx == INVALID) { have_leaf = false; continue; }
      const v4 c = node_cube_from_key(rb, rs, node_key(s, ch.node_base, nidx));
      pend = true;
      pend_anchor = true;
      pend_idx = nidx;
      pend_bmin = V3(c.x, c.y, c.z);
      pend_size = c.w;
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
      if (!opt.geom_only && leaf.mat == MAT_GRASS && ph.defer_gov) {
        // the march is left to k_gov_eval; its hit t lies in the slab
        // interval, and an empty interval is no hit
        ChunkTraceResult r{make_hit(leaf.mat, bh.t, bh.n, rb, rs, ch, nd, leaf.bmin, leaf.size), an.valid, an.key};
        GrassCell cell;
        const v2 iv = grass_on_voxel_interval(s, ro, rd, ch, bh.t, bh.n, t_enter, t_exit, &cell);
        if (iv.y > iv.x) {
          r.gov = true;
          r.gov_t0 = t_enter;
          r.gov_t1 = t_exit;
          r.gov_lo = iv.x;
          r.gov_hi = iv.y;
        }
        return r;
      }
      if (!opt.geom_only && leaf.mat == MAT_GRASS) {
        const GrassHit gh = grass_on_voxel_hit(s, ro, rd, ch, bh.t, bh.n, t_enter, t_exit);
        if (gh.hit)
          return ChunkTraceResult{make_hit(MAT_GRASS, gh.t, gh.n, rb, rs, ch, nd, leaf.bmin, leaf.size), an.valid,
                                  an.key};
      }
      return ChunkTraceResult{make_hit(leaf.mat, bh.t, bh.n, rb, rs, ch, nd, leaf.bmin, leaf.size), an.valid, an.key};
    }
    tcur = fmax_(t_leave, tcur) + eps_step;
    have_leaf = false;
  }
  if (pend && pend_anchor) {
    // the iteration limit ended the walk right after choosing a descent: the
    // descent still updates the anchor the walk returns
    const v3 pq = (ro + rd * tcur) + ray_eps_vec(rd, 1e-4f * vs);
    const LeafState l2 = descend_leaf_sparse_ool(s, pq, ch.node_base, pend_idx, pend_bmin, pend_size);
    const AnchorNode na = anchor_from_leaf(s, l2, ch.node_base);
    if (na.valid && (!an.valid || na.key != an.key)) an = na;
  }
  return ChunkTraceResult{miss_hitgeom(), an.valid, an.key};
}

template <uint32_t PM>
__device__ __forceinline__ ChunkTraceResult trace_chunk_interval_stream_macro(const Scene& s, v3 ro, v3 rd, v3 inv, const Meta& ch,
                                                   float t0_in, float t1_in, bool use_anchor, uint32_t anchor_key_in,
                                                   const TraceOpts& opt, ProbeHook& ph) {  // chunk_trace.wgsl:592-667
  const float vs = vs_(s);
  const v3 rb = V3((float)ch.ox, (float)ch.oy, (float)ch.oz) * vs;
  const float rs = (float)s.cam->chunk_size * vs;
  const float eps_step = 1e-4f * vs;
  float tcur = fmax_(t0_in, 0.0f) + eps_step;
  const float t_end = t1_in;
  uint32_t anchor_key = anchor_key_in;
  bool anchor_valid = use_anchor;
  MacroDDAState ms;
  ms.enabled = false;
  if (ch.macro_base != INVALID) ms = macro_dda_init(ro, rd, inv, tcur, rb, rs, ch.macro_base);
  // Without a usable macro grid the whole interval is one segment.  One call
  // site for the leaf walk keeps it inlined once.
  const bool whole = !ms.enabled;
  for (uint32_t i = 0; i < 128u; ++i) {
    float seg_end = t_end, cell_exit = t_end;
    bool empty = false;
    if (!whole) {
      if (tcur >= t_end) break;
      macro_dda_sync(ms, tcur);
      const MacroStep st = macro_dda_current(s, ms, ch.macro_base);
      if (!st.valid) break;
      cell_exit = st.t_exit;
      seg_end = fmin_(st.t_exit, t_end);
      empty = st.empty;
    }
    if (!empty) {
      const ChunkTraceResult h =
          trace_chunk_rope_interval_nomacro<PM>(s, ro, rd, inv, ch, tcur, seg_end, anchor_valid, anchor_key, opt, ph);
      if (whole || h.hit.hit != 0u) return h;
      anchor_valid = h.anchor_valid;
      anchor_key = h.anchor_key;
    }
    tcur = seg_end + eps_step;
    if (ms.enabled && tcur >= cell_exit) macro_dda_step(ms);
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
  // deferred blade march of the answer (ChunkTraceResult::gov): 0 none,
  // 1 pending (its interval and chunk slot below), 2 another chunk's result
  // could win once the marches are known (the pixel walks again)
  uint32_t gov_state = 0u;
  float gov_t0 = 0.0f, gov_t1 = 0.0f;
  uint32_t gov_slot = 0u;
};

// Visits the chunk-grid cells crossed by a ray (chunk_trace.wgsl:1028-1151).
template <class F>
__device__ __forceinline__ void chunk_grid_dda(const Scene& s, v3 ro, v3 rd, float t_min, float t_max, F&& visit) {
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
  const float tDX = fabsf(cs * inv.x), tDY = fabsf(cs * inv.y), tDZ = fabsf(cs * inv.z);
  if (fabsf(rd.x) < EPS_INV) tMaxX = BIG;
  if (fabsf(rd.y) < EPS_INV) tMaxY = BIG;
  if (fabsf(rd.z) < EPS_INV) tMaxZ = BIG;
  const int32_t dix = rd.x > 0.0f ? 1 : -1, diy = rd.y > 0.0f ? sy : -sy, diz = rd.z > 0.0f ? sz : -sz;
  int32_t rx = 0, ry = 0, rz = 0;
  if (fabsf(rd.x) >= EPS_INV) rx = stx > 0 ? (nx - 1 - lcx) : lcx;
  if (fabsf(rd.y) >= EPS_INV) ry = sty > 0 ? (ny - 1 - lcy) : lcy;
  if (fabsf(rd.z) >= EPS_INV) rz = stz > 0 ? (nz - 1 - lcz) : lcz;
  const uint32_t max_steps = min((uint32_t)(rx + ry + rz) + 1u, 512u);
  for (uint32_t st = 0; st < max_steps; ++st) {
    if (t_local > t_exit_local) break;
    const uint32_t slot = grid_at(s, (uint32_t)idx);
    if (slot != INVALID && slot < s.cam->chunk_count) {
      if (visit(slot, start_t + t_local)) return;
    }
    const float tn = fmin_(tMaxX, fmin_(tMaxY, tMaxZ));
    const float e = 1e-6f * fmax_(1.0f, fabsf(tn));
    if (fabsf(tMaxX - tn) <= e) { lcx += stx; idx += dix; tMaxX += tDX; }
    if (fabsf(tMaxY - tn) <= e) { lcy += sty; idx += diy; tMaxY += tDY; }
    if (fabsf(tMaxZ - tn) <= e) { lcz += stz; idx += diz; tMaxZ += tDZ; }
    t_local = tn;
    if (lcx < 0 || lcy < 0 || lcz < 0 || lcx >= nx || lcy >= ny || lcz >= nz) break;
  }
}

__device__ __forceinline__ bool chunk_coords_neighbor(i3 a, i3 b) {  // chunk_trace.wgsl:1000-1005
  return abs(a.x - b.x) <= 1 && abs(a.y - b.y) <= 1 && abs(a.z - b.z) <= 1;
}

__device__ __noinline__ bool chunk_heightfield_early_skip(const Scene& s, v3 ro, v3 rd, float t_enter, float t_exit, const Meta& ch,
                                  float vs) {  // chunk_trace.wgsl:1310-1352
  if (ch.colinfo_base == INVALID) return false;
  if (rd.y >= 0.0f) return false;
  const float y0 = ro.y + rd.y * t_enter, y1 = ro.y + rd.y * t_exit;
  const float seg_y_min = fmin_(y0, y1);
  const v3 rb = V3((float)ch.ox, (float)ch.oy, (float)ch.oz) * vs;
  const float seg_len = fmax_(t_exit - t_enter, 0.0f);
  const float dt = seg_len * (1.0f / 3.0f);
  for (uint32_t i = 0; i < 4u; ++i) {
    const float t = t_enter + (float)i * dt;
    const v3 p = ro + rd * t;
    const int32_t lx = clampi(to_i32(floorf((p.x - rb.x) / vs)), 0, 63);
    const int32_t lz = clampi(to_i32(floorf((p.z - rb.z) / vs)), 0, 63);
    const ColInfo ci = colinfo_decode(colinfo_entry_u16(s, ch.colinfo_base, (uint32_t)lx, (uint32_t)lz));
    if (!ci.valid) continue;
    const float top_y = rb.y + ((float)ci.y_vox + 1.0f) * vs;
    if (seg_y_min <= top_y + 1e-3f * vs) return false;
  }
  return true;
}

// ---------------------------------------------------------------------------
// clipmap.wgsl
// ---------------------------------------------------------------------------
__device__ __forceinline__ int32_t imod(int32_t a, int32_t m) {
  int32_t r = a % m;
  if (r < 0) r += m;
  return r;
}
__device__ __forceinline__ v2 clip_st(const Scene& s, v2 xz, uint32_t level) {  // clipmap.wgsl:317-327
  const float* p = s.clip->level[level];
  const float cell = fmax_(p[2], 1e-6f);
  const v2 uv = (xz - V2(p[0], p[1])) / V2(cell, cell);
  return uv - V2(0.5f, 0.5f);
}
struct HSample { float h; bool ok; };
__device__ HSample clip_height_at_level_ok(const Scene& s, v2 xz, uint32_t level) {  // clipmap.wgsl:34-52
  const int32_t res = max((int32_t)s.clip->res, 1);
  const v2 st = clip_st(s, xz, level);
  const int32_t ix = to_i32(floorf(st.x)), iz = to_i32(floorf(st.y));
  if (ix < 0 || iz < 0 || ix >= res || iz >= res) return HSample{0.0f, false};
  const int32_t sx = imod(ix + (int32_t)s.clip->offset[level][0], res);
  const int32_t sz = imod(iz + (int32_t)s.clip->offset[level][1], res);
  return HSample{clip_texel(s, sx, sz, level), true};
}
__device__ float clip_height_texel(const Scene& s, uint32_t level, int32_t ix, int32_t iz) {  // clipmap.wgsl:55-67
  const int32_t res = max((int32_t)s.clip->res, 1);
  if (ix < 0 || iz < 0 || ix >= res || iz >= res) return -BIG;
  const int32_t sx = imod(ix + (int32_t)s.clip->offset[level][0], res);
  const int32_t sz = imod(iz + (int32_t)s.clip->offset[level][1], res);
  return clip_texel(s, sx, sz, level);
}
__device__ __noinline__ float clip_height_at_level(const Scene& s, v2 xz, uint32_t level) {  // clipmap.wgsl:71-108
  const int32_t res = max((int32_t)s.clip->res, 1);
  const float* p = s.clip->level[level];
  const float cell = fmax_(p[2], 1e-6f);
  const v2 uv = (xz - V2(p[0], p[1])) / V2(cell, cell);
  const v2 st = uv - V2(0.5f, 0.5f);
  const int32_t ix0 = to_i32(floorf(st.x)), iz0 = to_i32(floorf(st.y));
  const int32_t ix1 = ix0 + 1, iz1 = iz0 + 1;
  if (ix0 < 0 || iz0 < 0 || ix1 >= res || iz1 >= res) return -BIG;
  const float fx = fract(st.x), fz = fract(st.y);
  const float h00 = clip_height_texel(s, level, ix0, iz0), h10 = clip_height_texel(s, level, ix1, iz0);
  const float h01 = clip_height_texel(s, level, ix0, iz1), h11 = clip_height_texel(s, level, ix1, iz1);
  const float lim = -0.5f * BIG;
  if (h00 <= lim || h10 <= lim || h01 <= lim || h11 <= lim) return -BIG;
  return mixf(mixf(h00, h10, fx), mixf(h01, h11, fx), fz);
}
__device__ float clip_height_at_level_nearest(const Scene& s, v2 xz, uint32_t level) {  // clipmap.wgsl:110-130
  const int32_t res = max((int32_t)s.clip->res, 1);
  const float* p = s.clip->level[level];
  const float cell = fmax_(p[2], 1e-6f);
  const v2 uv = (xz - V2(p[0], p[1])) / V2(cell, cell);
  const v2 st = uv - V2(0.5f, 0.5f);
  const int32_t ix = to_i32(floorf(st.x + 0.5f)), iz = to_i32(floorf(st.y + 0.5f));
  const int32_t sx = imod(ix + (int32_t)s.clip->offset[level][0], res);
  const int32_t sz = imod(iz + (int32_t)s.clip->offset[level][1], res);
  return clip_texel(s, sx, sz, level);
}
__device__ __noinline__ v3 clip_normal_at_level_2tap(const Scene& s, v2 xz, uint32_t level) {  // clipmap.wgsl:132-147
  const float cell = s.clip->level[level][2];
  const HSample h0 = clip_height_at_level_ok(s, xz, level);
  const HSample hx = clip_height_at_level_ok(s, xz + V2(cell, 0.0f), level);
  const HSample hz = clip_height_at_level_ok(s, xz + V2(0.0f, cell), level);
  if (!h0.ok || !hx.ok || !hz.ok) return V3(0.0f, 1.0f, 0.0f);
  const float dhx = (hx.h - h0.h) / fmax_(cell, 1e-4f), dhz = (hz.h - h0.h) / fmax_(cell, 1e-4f);
  return normalize(V3(-dhx, 1.0f, -dhz));
}
__device__ bool clip_level_contains(const Scene& s, v2 xz, uint32_t level, int32_t guard) {  // clipmap.wgsl:277-292
  const int32_t res = max((int32_t)s.clip->res, 1);
  const v2 st = clip_st(s, xz, level);
  const int32_t ix0 = to_i32(floorf(st.x)), iz0 = to_i32(floorf(st.y));
  return ix0 >= guard && iz0 >= guard && ix0 + 1 < res - guard && iz0 + 1 < res - guard;
}
__device__ __noinline__ uint32_t clip_best_level(const Scene& s, v2 xz, int32_t guard) {  // clipmap.wgsl:295-301
  const uint32_t n = min(s.clip->levels, CLIP_LEVELS_MAX);
  for (uint32_t i = 0; i < n; ++i)
    if (clip_level_contains(s, xz, i, guard)) return i;
  return max(n, 1u) - 1u;
}
__device__ __noinline__ uint32_t clip_ensure_contains(const Scene& s, v2 xz, uint32_t lvl_in, int32_t guard) {  // clipmap.wgsl:304-315
  const uint32_t n = min(s.clip->levels, CLIP_LEVELS_MAX);
  if (n == 0u) return 0u;
  uint32_t lvl = min(lvl_in, n - 1u);
  for (;;) {
    if (clip_level_contains(s, xz, lvl, guard) || lvl >= n - 1u) break;
    lvl += 1u;
  }
  return lvl;
}
struct ClipHit { bool hit; float t; v3 n; uint32_t mat; };

__device__ __noinline__ ClipHit clip_trace_heightfield(const Scene& s, v3 ro, v3 rd, float t_min, float t_max) {  // clipmap.wgsl:156-243
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
    const float dt_y = fabsf(sd) / vy;
    const float cell = s.clip->level[lvl][2];
    const float dt_xz = (6.0f * cell) / vh;
    float dt = fmin_(dt_y, dt_xz);
    dt = clampf(dt, 0.6f, HF_DT_MAX);
    t = t + dt;
  }
  return miss;
}

__device__ __forceinline__ float material_variation_clip(v3 p, float cell, float strength) {  // clipmap.wgsl:247-250
  return (hash31(vfloor(p / cell)) - 0.5f) * strength;
}
__device__ __noinline__ v3 apply_material_variation_clip(v3 base, uint32_t mat, v3 hp) {  // clipmap.wgsl:252-275
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
__device__ __forceinline__ float phase_mie(float costh) {  // phase.wgsl:5-10
  const float g = PHASE_G, gg = g * g;
  const float denom = powf_(1.0f + gg - 2.0f * g * costh, 1.5f);
  return INV_4PI * (1.0f - gg) / fmax_(denom, 1e-3f);
}
__device__ __forceinline__ float phase_blended(float costh) { return mixf(INV_4PI, phase_mie(costh), PHASE_MIE_W); }

__device__ __forceinline__ v3 fog_color_from_sky(v3 rd, v3 sky) {  // fog.wgsl:5-12
  const float up = clampf(rd.y * 0.5f + 0.5f, 0.0f, 1.0f);
  return vmix(FOG_COLOR_GROUND, vmin(sky, V3s(0.45f)), FOG_COLOR_SKY_BLEND * up);
}
__device__ __forceinline__ v3 fog_inscatter(v3 rd, v3 fogc) {  // fog.wgsl:15-19
  const float mu = clampf(dot(rd, SUN_DIR), 0.0f, 1.0f);
  const float ss = powf_(mu, 8.0f);
  return fogc + SUN_COLOR * (0.35f * ss);
}
__device__ __forceinline__ float fog_density_primary(const Scene& s) { return fmax_(s.cam->voxel_params[3] * FOG_PRIMARY_SCALE, 0.0f); }
__device__ __forceinline__ float fog_density_godray(const Scene& s) { return fmax_(s.cam->voxel_params[3] * FOG_GODRAY_SCALE, 0.0f); }
__device__ float fog_optical_depth_with_base(float base, v3 ro, v3 rd, float t) {  // fog.wgsl:31-45
  if (base <= 0.0f) return 0.0f;
  const float k = FOG_HEIGHT_FALLOFF, y0 = ro.y, dy = rd.y;
  if (fabsf(dy) < 1e-4f) return base * expf_(-k * y0) * t;
  const float a = expf_(-k * y0);
  const float b = expf_(-k * (y0 + dy * t));
  return base * (a - b) / (k * dy);
}
__device__ __noinline__ v3 apply_fog(const Scene& s, v3 surface, v3 ro, v3 rd, float t_scene, v3 sky) {  // fog.wgsl:57-71
  const float od = fmax_(fog_optical_depth_with_base(fog_density_primary(s), ro, rd, t_scene), 0.0f);
  const float T = expf_(-od);
  const v3 ins = fog_inscatter(rd, fog_color_from_sky(rd, sky));
  return surface * T + ins * (1.0f - T);
}

__device__ __noinline__ v3 sky_bg(v3 rd) {  // sky.wgsl:5-25
  const float t0 = smooth(-0.10f, 0.85f, rd.y);
  v3 col = vmix(V3(0.05f, 0.08f, 0.12f), V3(0.55f, 0.75f, 0.95f), t0);
  const float th = 1.0f - smooth(-0.20f, 0.18f, fabsf(rd.y));
  col = col + V3(0.80f, 0.75f, 0.70f) * (0.12f * th);
  const float tz = smooth(0.15f, 1.00f, rd.y);
  col = col + V3(0.20f, 0.35f, 0.60f) * (0.05f * tz);
  return col * SKY_EXPOSURE;
}
__device__ __noinline__ v3 sky_sun(v3 rd) {  // sky.wgsl:27-41
  const float mu = clampf(dot(rd, SUN_DIR), -1.0f, 1.0f);
  const float mu_inner = cosf_(0.009f);
  const float mu_outer = cosf_(0.009f + 0.004f);
  const float disc = smooth(mu_outer, mu_inner, mu);
  const float glow = smooth(0.70f, 0.98f, mu);
  const float halo = 0.03f * expf_(-2500.0f * fmax_(0.0f, 1.0f - mu));
  return SUN_COLOR * SUN_INTENSITY * (disc + halo + 0.04f * glow);
}

__device__ __forceinline__ float cloud_height01(float y) {  // clouds.wgsl:5-15
  const float t = clampf((y - CLOUD_BASE_H) / fmax_(CLOUD_TOP_H - CLOUD_BASE_H, 1e-3f), 0.0f, 1.0f);
  return smooth(0.00f, 0.12f, t) * (1.0f - smooth(0.78f, 1.00f, t));
}
__device__ __forceinline__ float cloud_coverage_at_xz(v2 xz, float time_s) {  // clouds.wgsl:18-31
  const v2 uv = xz * CLOUD_UV_SCALE + V2(CLOUD_WIND_X, CLOUD_WIND_Y) * time_s;
  const float field = 0.65f * fbm(uv) + 0.35f * fbm(uv * 2.3f + V2(13.2f, 7.1f));
  return smooth(CLOUD_COVERAGE, CLOUD_COVERAGE + CLOUD_SOFTNESS, field);
}
__device__ __noinline__ float cloud_density(v3 p, float time_s) {  // clouds.wgsl:34-65
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
__device__ __noinline__ float cloud_light_transmittance(v3 p, float time_s) {  // clouds.wgsl:68-90
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
__device__ __noinline__ float cloud_sun_transmittance_fast(const Scene& s, v3 p, v3 sd) {  // clouds.wgsl:134-165
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
__device__ __noinline__ float cloud_density_godray(v3 p, float time_s) {  // clouds.wgsl:167-182
  if (p.y <= CLOUD_BASE_H || p.y >= CLOUD_TOP_H) return 0.0f;
  const float h = cloud_height01(p.y);
  if (h <= 0.0f) return 0.0f;
  const v2 uv = V2(p.x, p.z) * CLOUD_UV_SCALE + V2(CLOUD_WIND_X, CLOUD_WIND_Y) * time_s;
  const float n0 = value_noise(uv);
  const float n1 = value_noise(uv * 2.0f + V2(17.0f, 9.0f));
  const float field = 0.70f * n0 + 0.30f * n1;
  return smooth(CLOUD_COVERAGE, CLOUD_COVERAGE + CLOUD_SOFTNESS, field) * h;
}
__device__ __noinline__ float cloud_sun_transmittance_godray(const Scene& s, v3 p, v3 sd) {  // clouds.wgsl:184-214
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

__device__ __noinline__ v3 sky_color(const Scene& s, v3 rd) {  // sky.wgsl:43-137
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
__device__ __noinline__ float trace_chunk_shadow_trans_interval(const Scene& s, v3 ro, v3 rd, const Meta& ch, float t_enter,
                                        float t_exit) {  // shadows.wgsl:4-82
  const float vs = vs_(s);
  const float nudge = 0.20f * vs;
  const v3 rb = V3((float)ch.ox, (float)ch.oy, (float)ch.oz) * vs;
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

__device__ __noinline__ float sun_transmittance_geom_only(const Scene& s, v3 p, v3 sd) {  // shadows.wgsl:85-186
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
  const float tDX = fabsf(cs * inv.x), tDY = fabsf(cs * inv.y), tDZ = fabsf(cs * inv.z);
  if (fabsf(rd.x) < EPS_INV) tMaxX = BIG;
  if (fabsf(rd.y) < EPS_INV) tMaxY = BIG;
  if (fabsf(rd.z) < EPS_INV) tMaxZ = BIG;
  float trans = 1.0f;
  const uint32_t max_steps = min((gd[0] + gd[1] + gd[2]) * 6u + 8u, 512u);
  const int32_t gx1 = go[0] + (int32_t)gd[0], gy1 = go[1] + (int32_t)gd[1], gz1 = go[2] + (int32_t)gd[2];
  for (uint32_t st = 0; st < max_steps; ++st) {
    if (t_local > t_exit_local) break;
    if (trans < MIN_TRANS) break;
    const float tn = fmin_(tMaxX, fmin_(tMaxY, tMaxZ));
    const uint32_t slot = grid_lookup_slot(s, cx, cy, cz);
    if (slot != INVALID && slot < s.cam->chunk_count) {
      const Meta ch2 = meta_at(s, slot);
      const float ce = start_t + t_local;
      const float cx2 = start_t + fmin_(tn, t_exit_local);
      // A rising ray that enters the chunk a voxel above its top solid leaf
      // meets only air there: the chunk's factor is exactly 1.
      const bool above = s.slot_top != nullptr && rd.y > 0.0f && slot < s.metas_n &&
                         ro.y + rd.y * fmax_(ce, 0.0f) >= ((float)ch2.oy + (float)__ldg(&s.slot_top[slot]) + 1.0f) * vs;
      if (!above) trans *= trace_chunk_shadow_trans_interval(s, ro, rd, ch2, ce, cx2);
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
__device__ __forceinline__ uint32_t hash3_i32(i3 p) {  // light.wgsl:18-23
  return hash_u32(((uint32_t)p.x * 73856093u) ^ ((uint32_t)p.y * 19349663u) ^ ((uint32_t)p.z * 83492791u));
}
__device__ __forceinline__ v3 rot_about_axis(v3 v, v3 axis, float ang) {  // light.wgsl:32-37
  const v3 a = normalize(axis);
  const float sn = sinf_(ang), c = cosf_(ang);
  return v * c + cross(a, v) * sn + a * dot(a, v) * (1.0f - c);
}
__device__ __forceinline__ v3 sphere_dir_local(uint32_t i, uint32_t count) {  // light.wgsl:48-56
  const float fi = (float)i;
  const float cf = fmax_(1.0f, (float)count);
  const float golden = 2.399963229728653f;
  const float y = 1.0f - 2.0f * ((fi + 0.5f) / cf);
  const float r = sqrtf(fmax_(0.0f, 1.0f - y * y));
  const float phi = golden * fi;
  return V3(cosf_(phi) * r, sinf_(phi) * r, y);
}

__device__ __noinline__ v4 dda_hit_light(const Scene& s, v3 p0, v3 dir, uint32_t max_steps, float vs) {  // light.wgsl:65-121
  const v3 gpos = p0 / fmax_(vs, 1e-6f);
  const v3 fl = vfloor(gpos);
  i3 cell{to_i32(fl.x), to_i32(fl.y), to_i32(fl.z)};
  const i3 step{dir.x >= 0.0f ? 1 : -1, dir.y >= 0.0f ? 1 : -1, dir.z >= 0.0f ? 1 : -1};
  const v3 nb = V3((float)(cell.x + (dir.x >= 0.0f ? 1 : 0)), (float)(cell.y + (dir.y >= 0.0f ? 1 : 0)),
                   (float)(cell.z + (dir.z >= 0.0f ? 1 : 0)));
  const v3 inv = V3(fabsf(dir.x) > 1e-6f ? 1.0f / fabsf(dir.x) : 1e30f,
                    fabsf(dir.y) > 1e-6f ? 1.0f / fabsf(dir.y) : 1e30f,
                    fabsf(dir.z) > 1e-6f ? 1.0f / fabsf(dir.z) : 1e30f);
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

__device__ __forceinline__ v3 material_emission(uint32_t m) {  // shading.wgsl:211-216
  if (m == MAT_LIGHT) return V3(1.0f, 0.95f, 0.75f) * 18.0f;
  return V3s(0.0f);
}

// gather_voxel_lights (light.wgsl:127-211) in three parts so that its eight
// rays can also run on eight lanes: the per-pixel frame, one ray's direction,
// and the in-order accumulation (ray results do not depend on each other;
// only the accumulation stops early, after LIGHT_EARLY_HITS hits).
struct LightFrame {
  v3 p0, tt, bb;
  float rot;
};

__device__ __forceinline__ LightFrame light_frame(const Scene& s, v3 hp, v3 n, v3 rb) {  // light.wgsl:127-151
  const float vs = vs_(s);
  LightFrame F;
  F.p0 = hp + n * (0.75f * vs);
  // make_tbn (light.wgsl:25-30): columns t, b, n
  const v3 up = fabsf(n.y) > 0.9f ? V3(1.0f, 0.0f, 0.0f) : V3(0.0f, 1.0f, 0.0f);
  F.tt = normalize(cross(up, n));
  F.bb = normalize(cross(n, F.tt));
  const v3 sv = vfloor((hp - rb) / fmax_(vs, 1e-6f));
  const uint32_t h0 = hash3_i32(i3{to_i32(sv.x), to_i32(sv.y), to_i32(sv.z)});
  const uint32_t h1 = hash_u32(h0);
  const uint32_t h2 = hash_u32(h1 ^ (s.cam->frame_index * 747796405u));
  F.rot = 6.28318530718f * ((float)(h2 & 1023u) / 1024.0f);
  return F;
}

__device__ __forceinline__ v3 light_ray_dir(const LightFrame& F, v3 n, uint32_t i) {  // light.wgsl:167-169
  const v3 sl = normalize(sphere_dir_local(i, LIGHT_RAYS));
  const v3 ldir = normalize(F.tt * sl.x + F.bb * sl.y + n * sl.z);
  return normalize(rot_about_axis(ldir, n, F.rot));
}

// Adds ray result `hit` (dda_hit_light) to `sum`; true when the gather stops.
__device__ __forceinline__ bool light_accum(const Scene& s, v3 hp, v3 n, v4 hit, uint32_t& hits, v3& sum) {
  if (!(hit.w > 0.5f)) return false;  // light.wgsl:172-205
  const float vs = vs_(s);
  const float soft_r = LIGHT_SOFT_RADIUS_VOX * vs, soft_r2 = soft_r * soft_r;
  const float min_r = LIGHT_NEAR_CLAMP_VOX * vs, min_r2 = min_r * min_r;
  const float range_m = LIGHT_RANGE_VOX * vs, range2 = range_m * range_m;
  const v3 Le = material_emission(MAT_LIGHT);
  hits += 1u;
  const v3 L = V3(hit.x, hit.y, hit.z) - hp;
  const float r2 = fmax_(dot(L, L), min_r2);
  const float r = sqrtf(r2);
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
  return hits >= LIGHT_EARLY_HITS;
}

__device__ __forceinline__ v3 light_finish(v3 sum) {  // light.wgsl:207-210
  const float denom = fmax_(1.0f, (float)LIGHT_RAYS);
  return sum * (1.0f / denom);
}

// False when no chunk within reach of dda_hit_light from p0 (at most
// LIGHT_MAX_DIST_VOX cells, each step one cell along one axis) holds a LIGHT
// leaf: every light ray then ends on a solid voxel, in air or outside the
// grid, and the gather adds nothing.  The cell box gets one cell of margin
// for the half-cell offset of the query points.
__device__ __noinline__ bool lights_possible(const Scene& s, v3 p0) {
  if (s.slot_lights == nullptr) return true;
  const v3 fl = vfloor(p0 / fmax_(vs_(s), 1e-6f));
  const int32_t cs = (int32_t)s.cam->chunk_size;
  if (cs <= 0) return true;
  const int32_t r = (int32_t)LIGHT_MAX_DIST_VOX + 1;
  auto fdiv = [cs](int32_t a) { return a >= 0 ? a / cs : -((-a + cs - 1) / cs); };
  const int32_t cx = to_i32(fl.x), cy = to_i32(fl.y), cz = to_i32(fl.z);
  for (int32_t z = fdiv(cz - r); z <= fdiv(cz + r); ++z)
    for (int32_t y = fdiv(cy - r); y <= fdiv(cy + r); ++y)
      for (int32_t x = fdiv(cx - r); x <= fdiv(cx + r); ++x) {
        const uint32_t slot = grid_lookup_slot(s, x, y, z);
        if (slot != INVALID && slot < s.cam->chunk_count && slot < s.metas_n && __ldg(&s.slot_lights[slot]) != 0u)
          return true;
      }
  return false;
}

__device__ __noinline__ v3 gather_voxel_lights(const Scene& s, v3 hp, v3 n, v3 rb) {  // light.wgsl:127-211
  const LightFrame F = light_frame(s, hp, n, rb);
  uint32_t hits = 0;
  v3 sum = V3s(0.0f);
  if (!lights_possible(s, F.p0)) return light_finish(sum);
  for (uint32_t i = 0; i < LIGHT_RAYS; ++i) {
    const v4 hit = dda_hit_light(s, F.p0, light_ray_dir(F, n, i), LIGHT_MAX_DIST_VOX, vs_(s));
    if (light_accum(s, hp, n, hit, hits, sum)) break;
  }
  return light_finish(sum);
}

// ---------------------------------------------------------------------------
// shading.wgsl
// ---------------------------------------------------------------------------
__device__ __forceinline__ v3 color_for_material(uint32_t m) {  // shading.wgsl:7-16
  if (m == MAT_AIR) return V3s(0.0f);
  if (m == MAT_GRASS) return V3(0.18f, 0.75f, 0.18f);
  if (m == MAT_DIRT) return V3(0.45f, 0.30f, 0.15f);
  if (m == MAT_STONE) return V3(0.50f, 0.50f, 0.55f);
  if (m == MAT_WOOD) return V3(0.38f, 0.26f, 0.14f);
  if (m == MAT_LEAF) return V3(0.10f, 0.55f, 0.12f);
  if (m == MAT_LIGHT) return V3(1.0f, 0.95f, 0.75f);
  return V3(1.0f, 0.0f, 1.0f);
}
__device__ __forceinline__ v3 hemi_ambient(v3 n, v3 sky_up) {  // shading.wgsl:18-22
  return vmix(FOG_COLOR_GROUND, sky_up, clampf(n.y * 0.5f + 0.5f, 0.0f, 1.0f));
}
__device__ __noinline__ v3 apply_material_variation(v3 base, uint32_t mat, v3 hp) {  // shading.wgsl:24-50
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
__device__ __noinline__ v2 grass_wind_dir_xz(v3 p, float time_s) {  // shading.wgsl:52-59
  const v3 w = wind_field(p, time_s);
  v2 dir = V2(w.x, w.z) + V2(0.6f, 0.2f);
  if (dot(dir, dir) < 1e-4f) dir = V2(0.7f, 0.25f);
  return normalize(dir);
}
__device__ __noinline__ float grass_blade_slivers(v3 pw, float time_s, float freq, float detail) {  // shading.wgsl:61-88
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
  const float dist = fabsf(pr.y - center);
  const float sliver = smooth(width + aa, width - aa, dist);
  const float lm = smooth(0.0f, 0.15f, u) * smooth(1.0f, 0.75f, u);
  return sliver * lm;
}
__device__ __noinline__ float grass_blade_field(v3 p, float time_s, float t) {  // shading.wgsl:90-98
  const float detail = 1.0f - smooth(18.0f, 55.0f, t);
  const float low = grass_blade_slivers(p, time_s, 9.0f, detail * 0.6f);
  const float high = grass_blade_slivers(p + V3(1.7f, 0.0f, 2.3f), time_s, 18.0f, detail);
  const float blend = mixf(0.15f, 1.0f, detail);
  return mixf(low, 0.5f * (low + high), blend);
}
__device__ __noinline__ v3 grass_top_albedo(const Scene& s, v3 base, v3 hp, float t) {  // shading.wgsl:100-122
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
__device__ __forceinline__ v3 base_albedo(uint32_t mat, v3 hp, float t) {  // shading.wgsl:124-130
  v3 b = color_for_material(mat);
  if (t <= FAR_SHADING_DIST) b = apply_material_variation(b, mat, hp);
  return b;
}
__device__ float macro_occ_at_ws(const Scene& s, v3 p, v3 rb, float rs, uint32_t macro_base) {  // shading.wgsl:132-154
  if (macro_base == INVALID) return 0.0f;
  const v3 lp = p - rb;
  if (lp.x < 0.0f || lp.y < 0.0f || lp.z < 0.0f || lp.x >= rs || lp.y >= rs || lp.z >= rs) return 0.0f;
  const float cell = macro_cell_size(rs);
  const uint32_t mx = clampu(to_u32(floorf(lp.x / cell)), 0u, 7u);
  const uint32_t my = clampu(to_u32(floorf(lp.y / cell)), 0u, 7u);
  const uint32_t mz = clampu(to_u32(floorf(lp.z / cell)), 0u, 7u);
  return macro_test(s, macro_base, macro_bit_index(mx, my, mz)) ? 1.0f : 0.0f;
}
__device__ __noinline__ float voxel_ao_local(const Scene& s, v3 hp, v3 n, v3 rb, float rs, uint32_t macro_base) {  // shading.wgsl:157-184
  const float r = 0.75f * vs_(s);
  const v3 up = fabsf(n.y) > 0.9f ? V3(1.0f, 0.0f, 0.0f) : V3(0.0f, 1.0f, 0.0f);
  const v3 t = normalize(cross(up, n));
  const v3 b = normalize(cross(n, t));
  float occ = 0.0f;
  occ += macro_occ_at_ws(s, hp + t * r, rb, rs, macro_base);
  occ += macro_occ_at_ws(s, hp - t * r, rb, rs, macro_base);
  occ += macro_occ_at_ws(s, hp + b * r, rb, rs, macro_base);
  occ += macro_occ_at_ws(s, hp - b * r, rb, rs, macro_base);
  return clampf(1.0f - 0.70f * (occ * 0.25f), 0.35f, 1.0f);
}
__device__ __forceinline__ float material_roughness(uint32_t m) {
  if (m == MAT_STONE) return 0.45f;
  if (m == MAT_WOOD) return 0.70f;
  if (m == MAT_LEAF) return 0.80f;
  if (m == MAT_GRASS) return 0.85f;
  if (m == MAT_DIRT) return 0.90f;
  if (m == MAT_LIGHT) return 0.25f;
  return 0.90f;
}
__device__ __forceinline__ float material_f0(uint32_t m) {
  if (m == MAT_STONE) return 0.04f;
  if (m == MAT_WOOD) return 0.03f;
  if (m == MAT_LEAF) return 0.05f;
  if (m == MAT_GRASS) return 0.04f;
  if (m == MAT_DIRT) return 0.02f;
  if (m == MAT_LIGHT) return 0.08f;
  return 0.02f;
}

__device__ __noinline__ v3 shade_hit(const Scene& s, v3 ro, v3 rd, const HitGeom& hg, v3 sky_up, float sun_shadow) {  // shading.wgsl:257-362
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

__device__ __noinline__ v3 shade_clip_hit(const Scene& s, v3 ro, v3 rd, const ClipHit& ch, v3 sky_up) {  // shading.wgsl:364-434
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
// godrays.wgsl
// ---------------------------------------------------------------------------
__device__ __forceinline__ float approx_pow_0p75(float x) { const float y = clampf(x, 0.0f, 1.0f); return mixf(y, sqrtf(y), 0.5f); }
__device__ __forceinline__ float approx_pow_0p55(float x) { const float y = clampf(x, 0.0f, 1.0f); return mixf(sqrtf(y), y, 0.20f); }
__device__ __forceinline__ float exp_neg_fast(float xin) { const float x = fmax_(xin, 0.0f); return 1.0f / (1.0f + x + 0.48f * (x * x)); }
__device__ __forceinline__ uint32_t godray_steps_for_tend(float t_end) {  // godrays.wgsl:30-43
  const float raw = ceilf(t_end * GODRAY_STEPS_PER_METER);
  uint32_t sN = to_u32(clampf(raw, (float)GODRAY_MIN_STEPS, (float)GODRAY_STEPS_FAST));
  sN = ((sN + (GODRAY_STEP_Q - 1u)) / GODRAY_STEP_Q) * GODRAY_STEP_Q;
  return min(sN, GODRAY_STEPS_FAST);
}

__device__ __noinline__ v3 godray_integrate_1(const Scene& s, v3 ro, v3 rd, float t_end, float j, float j_phase) {  // godrays.wgsl:45-216
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
  const bool horiz = fabsf(dy) < 1e-4f;
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

__device__ __forceinline__ v3 godray_decompress(v3 c) {
  const v3 den = vmax(V3s(1.0f) - c, V3s(1e-4f));
  return (c * 0.25f) / den;
}
__device__ __forceinline__ v3 godray_compress(v3 l) { return l / (l + V3s(0.25f)); }

__device__ __forceinline__ v3 bright_extract_hue(v3 x, float thresh) {
  const float l = dot(x, V3(0.2126f, 0.7152f, 0.0722f));
  const float over = fmax_(l - thresh, 0.0f);
  return x * (over / fmax_(l, 1e-4f));
}
__device__ __forceinline__ v3 hable(v3 x) {
  const float A = 0.22f, B = 0.30f, C = 0.10f, D = 0.20f, E = 0.01f, F = 0.30f;
  auto one = [&](float v) {
    const float num = v * (A * v + C * B) + D * E;
    const float den = v * (A * v + B) + D * F;
    return num / fmax_(den, 1e-6f) - E / F;
  };
  return V3(one(x.x), one(x.y), one(x.z));
}
__device__ __forceinline__ v3 tonemap_white(v3 x, float wp) {
  const v3 w = hable(V3s(wp));
  const v3 invw = V3s(1.0f) / vmax(w, V3s(1e-6f));
  return hable(x) * invw;
}


}  // namespace dev
}  // namespace vxe
