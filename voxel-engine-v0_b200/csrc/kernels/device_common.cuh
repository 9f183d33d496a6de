// device_common.cuh -- scalar helpers, bindings and loads for the vxe kernels.
//
// Float semantics follow the WGSL spec (common.wgsl helpers): mix = a*(1-t)+b*t,
// smoothstep = t*t*(3-2t), clamp = min(max()), normalize(v) = v*(1/sqrt(dot)),
// saturating f32->int conversions.  Compiled with -fmad=false -prec-div=true
// -prec-sqrt=true so every operation is one IEEE binary32 op, which is what the
// CPU oracle evaluates too; transcendental functions come from detmath.h.
#pragma once

#include <cstdint>

#include "vxe/detmath.h"
#include "vxe/vxe.h"

namespace vxe {
namespace dev {

// ---------------------------------------------------------------------------
// Constants (common.wgsl:16-332)
// ---------------------------------------------------------------------------
constexpr uint32_t INVALID = 0xFFFFFFFFu;
constexpr uint32_t LEAF = 0xFFFFFFFFu;
constexpr float BIG = 1e30f;
constexpr float EPS_INV = 1e-8f;
constexpr uint32_t MAT_AIR = 0, MAT_GRASS = 1, MAT_DIRT = 2, MAT_STONE = 3, MAT_WOOD = 4, MAT_LEAF = 5,
                   MAT_LIGHT = 6;
constexpr float SUN_X = 0.61237244f, SUN_Y = 0.5f, SUN_Z = 0.61237244f;
constexpr float SUN_INTENSITY = 5.0f;
constexpr float FOG_MAX_DIST = 120.0f;
constexpr uint32_t MAX_TILE_CHUNKS = 192, TILE_CANDS = 24, TILE_SIZE = 8;

// Error word bits (vxe_read_error_word).
constexpr uint32_t ERR_NODE = 1u << 0, ERR_ROPE = 1u << 1, ERR_META = 1u << 2, ERR_GRID = 1u << 3,
                   ERR_MACRO = 1u << 4, ERR_COLINFO = 1u << 5, ERR_CLIP = 1u << 6;

// ---------------------------------------------------------------------------
// Scalars
// ---------------------------------------------------------------------------
__device__ __forceinline__ float fmin_(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ float fmax_(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
__device__ __forceinline__ float mixf(float a, float b, float t) {
  return __fadd_rn(__fmul_rn(a, __fsub_rn(1.0f, t)), __fmul_rn(b, t));
}
__device__ __forceinline__ float smooth(float e0, float e1, float x) {
  const float t = clampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}
__device__ __forceinline__ float fract(float x) { return x - floorf(x); }
__device__ __forceinline__ float signf(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }
__device__ __forceinline__ int32_t to_i32(float f) { return __float2int_rz(f); }
__device__ __forceinline__ uint32_t to_u32(float f) { return __float2uint_rz(f); }
__device__ __forceinline__ int32_t clampi(int32_t x, int32_t lo, int32_t hi) { return min(max(x, lo), hi); }
__device__ __forceinline__ uint32_t clampu(uint32_t x, uint32_t lo, uint32_t hi) { return min(max(x, lo), hi); }
__device__ __forceinline__ float sinf_(float x) { return vxe_sinf(x); }
__device__ __forceinline__ float cosf_(float x) { return vxe_cosf(x); }
__device__ __forceinline__ float expf_(float x) { return vxe_expf(x); }
__device__ __forceinline__ float powf_(float x, float y) { return vxe_powf(x, y); }

struct v2 { float x, y; };
struct v3 { float x, y, z; };
struct v4 { float x, y, z, w; };
struct i3 { int32_t x, y, z; };

__device__ __forceinline__ v2 V2(float x, float y) { return v2{x, y}; }
__device__ __forceinline__ v3 V3(float x, float y, float z) { return v3{x, y, z}; }
__device__ __forceinline__ v3 V3s(float s) { return v3{s, s, s}; }
__device__ __forceinline__ v2 operator+(v2 a, v2 b) { return {a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ v2 operator-(v2 a, v2 b) { return {a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ v2 operator*(v2 a, v2 b) { return {a.x * b.x, a.y * b.y}; }
__device__ __forceinline__ v2 operator*(v2 a, float s) { return {a.x * s, a.y * s}; }
__device__ __forceinline__ v2 operator*(float s, v2 a) { return {s * a.x, s * a.y}; }
__device__ __forceinline__ v2 operator/(v2 a, v2 b) { return {a.x / b.x, a.y / b.y}; }
__device__ __forceinline__ v3 operator+(v3 a, v3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ v3 operator-(v3 a, v3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ v3 operator-(v3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ v3 operator*(v3 a, v3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ v3 operator*(v3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ v3 operator*(float s, v3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ v3 operator/(v3 a, v3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
__device__ __forceinline__ v3 operator/(v3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ float dot(v2 a, v2 b) { return a.x * b.x + a.y * b.y; }
__device__ __forceinline__ float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float length(v2 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ float length(v3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ v2 normalize(v2 a) { const float inv = 1.0f / sqrtf(dot(a, a)); return a * inv; }
__device__ __forceinline__ v3 normalize(v3 a) { const float inv = 1.0f / sqrtf(dot(a, a)); return a * inv; }
__device__ __forceinline__ v3 cross(v3 a, v3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ v3 vmin(v3 a, v3 b) { return {fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)}; }
__device__ __forceinline__ v3 vmax(v3 a, v3 b) { return {fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)}; }
__device__ __forceinline__ v3 vabs(v3 a) { return {fabsf(a.x), fabsf(a.y), fabsf(a.z)}; }
__device__ __forceinline__ v3 vfloor(v3 a) { return {floorf(a.x), floorf(a.y), floorf(a.z)}; }
__device__ __forceinline__ v2 vfloor(v2 a) { return {floorf(a.x), floorf(a.y)}; }
__device__ __forceinline__ v2 vfract(v2 a) { return {fract(a.x), fract(a.y)}; }
__device__ __forceinline__ v3 vclamp(v3 x, v3 lo, v3 hi) { return vmin(vmax(x, lo), hi); }
__device__ __forceinline__ v3 vmix(v3 a, v3 b, float t) { return {mixf(a.x, b.x, t), mixf(a.y, b.y, t), mixf(a.z, b.z, t)}; }
__device__ __forceinline__ float max3(v3 v) { return fmaxf(v.x, fmaxf(v.y, v.z)); }
__device__ __forceinline__ float min3(v3 v) { return fminf(v.x, fminf(v.y, v.z)); }
__device__ __forceinline__ bool in_unit_square(v2 uv) { return uv.x >= 0.0f && uv.y >= 0.0f && uv.x <= 1.0f && uv.y <= 1.0f; }

#define SUN_DIR V3(SUN_X, SUN_Y, SUN_Z)
#define SUN_COLOR V3(1.0f, 0.94f, 0.72f)
#define FOG_COLOR_GROUND V3(0.40f, 0.42f, 0.45f)

// ---------------------------------------------------------------------------
// Bindings
// ---------------------------------------------------------------------------
struct Meta {
  int32_t ox, oy, oz;
  uint32_t node_base, macro_base, colinfo_base, macro_empty;
};

struct Scene {
  const vxe_camera_gpu* cam;  // grid-constant parameter space
  const vxe_clipmap_gpu* clip;
  const uint4* __restrict__ nodes;
  uint64_t nodes_n;
  const uint32_t* __restrict__ ropes;  // 8 words per node
  uint64_t ropes_n;
  const uint4* __restrict__ metas;  // 3 x uint4 per slot
  uint64_t metas_n;
  const uint32_t* __restrict__ grid;
  uint64_t grid_n;
  const uint32_t* __restrict__ macro;  // words as bound for the pass
  uint64_t macro_n;
  const uint32_t* __restrict__ colinfo;
  uint64_t colinfo_n;
  const float* __restrict__ clip_tex;
  uint32_t clip_layers, clip_res;
  uint32_t* err;
  // Per-frame grass cell table (10 x float4 per column, slot * 4096 + column)
  // and blade taper per LOD (3 x 6); null when the pass has none.
  const float4* __restrict__ grass_rec;
  uint64_t grass_rec_n;
  const float* __restrict__ grass_taper;
  // Lod-0 blade segment frames of the table's records (GRASS_FRAME_F4 float4
  // each), filled in by the first march that needs them in a frame, and their
  // state (0 not built, 1 being built, 2 ready); null when the pass has none.
  // Written during passes, so never read through the read-only path.
  uint32_t* grass_state;
  float4* grass_frames;
  // Per chunk slot: 1 when the slot's nodes hold a LIGHT leaf (written with
  // the slot's uploads and meta writes); null when the pass has none.
  const uint32_t* __restrict__ slot_lights;
  // Per chunk slot: the top (exclusive, in voxels above the chunk origin) of
  // the slot's non-air leaves, 0 when the slot holds none; null when the pass
  // has none.
  const uint32_t* __restrict__ slot_top;
};

struct Node { uint32_t child_base, child_mask, material, key; };

__device__ __forceinline__ void flag(const Scene& s, uint32_t bit) { atomicOr(s.err, bit); }

// Reads of the world's records at data-derived indices.  Two builds of the
// library differ only here:
//   VXE_DEVICE_CHECKS 0 (libvxe.so): every index is clamped into its buffer:
//     no branch and no atomic on the traversal's hot path, never a read
//     outside the buffers; records that point outside their chunk give wrong
//     images but no fault (the robust-access behaviour WGSL allows);
//   VXE_DEVICE_CHECKS 1 (libvxe_checked.so): an index outside its buffer
//     reads as a zero record and sets a bit of the context's error word
//     (vxe_read_error_word; vxe_render_frame returns VXE_ERR_BOUNDS).
// Records that are in range give the same values in both builds.
#ifndef VXE_DEVICE_CHECKS
#define VXE_DEVICE_CHECKS 0
#endif
#if VXE_DEVICE_CHECKS
__device__ __forceinline__ Node node_global(const Scene& s, uint32_t gi) {
  if (gi >= s.nodes_n) { flag(s, ERR_NODE); return Node{0u, 0u, 0u, 0u}; }
  const uint4 n = __ldg(&s.nodes[gi]);
  return Node{n.x, n.y, n.z, n.w};
}
__device__ __forceinline__ uint32_t node_key(const Scene& s, uint32_t base, uint32_t local) {
  const uint32_t gi = base + local;
  if (gi >= s.nodes_n) { flag(s, ERR_NODE); return 0u; }
  return __ldg(&s.nodes[gi].w);
}
__device__ __forceinline__ Meta meta_at(const Scene& s, uint32_t slot) {
  if (slot >= s.metas_n) { flag(s, ERR_META); return Meta{0, 0, 0, 0u, 0u, 0u, 0u}; }
  const uint4 a = __ldg(&s.metas[(size_t)slot * 3u]);
  const uint4 b = __ldg(&s.metas[(size_t)slot * 3u + 1u]);
  const uint32_t e = __ldg(&s.metas[(size_t)slot * 3u + 2u].x);
  return Meta{(int32_t)a.x, (int32_t)a.y, (int32_t)a.z, b.x, b.z, b.w, e};
}
__device__ __forceinline__ uint32_t meta_empty(const Scene& s, uint32_t slot) {
  if (slot >= s.metas_n) { flag(s, ERR_META); return 0u; }
  return __ldg(&s.metas[(size_t)slot * 3u + 2u].x);
}
__device__ __forceinline__ uint32_t grid_at(const Scene& s, uint32_t idx) {
  if (idx >= s.grid_n) { flag(s, ERR_GRID); return 0u; }
  return __ldg(&s.grid[idx]);
}
__device__ __forceinline__ uint32_t macro_word(const Scene& s, uint32_t idx) {
  if (idx >= s.macro_n) { flag(s, ERR_MACRO); return 0u; }
  return __ldg(&s.macro[idx]);
}
__device__ __forceinline__ uint32_t colinfo_word(const Scene& s, uint32_t idx) {
  if (idx >= s.colinfo_n) { flag(s, ERR_COLINFO); return 0u; }
  return __ldg(&s.colinfo[idx]);
}
__device__ __forceinline__ uint32_t rope_face(const Scene& s, uint32_t gi, uint32_t face) {
  if (gi >= s.ropes_n) { flag(s, ERR_ROPE); return 0u; }
  return __ldg(&s.ropes[(size_t)gi * 8u + face]);
}
__device__ __forceinline__ float clip_texel(const Scene& s, int32_t sx, int32_t sz, uint32_t level) {
  if (level >= s.clip_layers || sx < 0 || sz < 0 || (uint32_t)sx >= s.clip_res || (uint32_t)sz >= s.clip_res) {
    flag(s, ERR_CLIP);
    return 0.0f;
  }
  return __ldg(&s.clip_tex[((size_t)level * s.clip_res + (uint32_t)sz) * s.clip_res + (uint32_t)sx]);
}
#else
// (every buffer holds at least one record: the context's capacities and the
// scene-view checks guarantee n >= 1)
__device__ __forceinline__ uint64_t clamp_index(uint64_t i, uint64_t n) { return i < n ? i : n - 1u; }
__device__ __forceinline__ Node node_global(const Scene& s, uint32_t gi) {
  const uint4 n = __ldg(&s.nodes[clamp_index(gi, s.nodes_n)]);
  return Node{n.x, n.y, n.z, n.w};
}
__device__ __forceinline__ uint32_t node_key(const Scene& s, uint32_t base, uint32_t local) {
  return __ldg(&s.nodes[clamp_index(base + local, s.nodes_n)].w);
}
__device__ __forceinline__ Meta meta_at(const Scene& s, uint32_t slot) {
  const size_t i = (size_t)clamp_index(slot, s.metas_n) * 3u;
  const uint4 a = __ldg(&s.metas[i]);
  const uint4 b = __ldg(&s.metas[i + 1u]);
  const uint32_t e = __ldg(&s.metas[i + 2u].x);
  return Meta{(int32_t)a.x, (int32_t)a.y, (int32_t)a.z, b.x, b.z, b.w, e};
}
__device__ __forceinline__ uint32_t meta_empty(const Scene& s, uint32_t slot) {
  return __ldg(&s.metas[(size_t)clamp_index(slot, s.metas_n) * 3u + 2u].x);
}
__device__ __forceinline__ uint32_t grid_at(const Scene& s, uint32_t idx) { return __ldg(&s.grid[clamp_index(idx, s.grid_n)]); }
__device__ __forceinline__ uint32_t macro_word(const Scene& s, uint32_t idx) {
  return __ldg(&s.macro[clamp_index(idx, s.macro_n)]);
}
__device__ __forceinline__ uint32_t colinfo_word(const Scene& s, uint32_t idx) {
  return __ldg(&s.colinfo[clamp_index(idx, s.colinfo_n)]);
}
__device__ __forceinline__ uint32_t rope_face(const Scene& s, uint32_t gi, uint32_t face) {
  return __ldg(&s.ropes[(size_t)clamp_index(gi, s.ropes_n) * 8u + face]);
}
__device__ __forceinline__ float clip_texel(const Scene& s, int32_t sx, int32_t sz, uint32_t level) {
  if (s.clip_layers == 0u || s.clip_res == 0u) return 0.0f;  // no clipmap texture
  const uint32_t r1 = s.clip_res - 1u;
  const uint32_t l = min(level, s.clip_layers - 1u), x = min((uint32_t)max(sx, 0), r1),
                 z = min((uint32_t)max(sz, 0), r1);
  return __ldg(&s.clip_tex[((size_t)l * s.clip_res + z) * s.clip_res + x]);
}
#endif
__device__ __forceinline__ Node node_at(const Scene& s, uint32_t base, uint32_t local) { return node_global(s, base + local); }

__device__ __forceinline__ v3 cam_pos(const Scene& s) { return V3(s.cam->cam_pos[0], s.cam->cam_pos[1], s.cam->cam_pos[2]); }
__device__ __forceinline__ float vs_(const Scene& s) { return s.cam->voxel_params[0]; }

}  // namespace dev
}  // namespace vxe
