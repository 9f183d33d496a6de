// frame_kernels.cuh -- the frame passes as sm_100a kernels.
//
//   k_tiles      per 8x8 logical tile: two probe-ray chunk-grid DDAs, dedup,
//                partial selection sort (ray_main.wgsl:179-197,
//                chunk_trace.wgsl:1007-1175).  Runs as its own launch so the
//                primary launch shape is free of the 8x8 workgroup.
//   k_primary    main_primary (ray_main.wgsl:163-517) with main_local_taa
//                (taa.wgsl:26-69) fused into the epilogue: local TAA reads only
//                the same pixel, so local_img never round-trips through HBM.
//   k_godray     main_godray (ray_main.wgsl:520-535, godrays.wgsl:241-356).
//   k_composite  main_composite (ray_main.wgsl:537-573, composite.wgsl) with
//                main_composite_taa (taa.wgsl:82-110) fused: it reads only the
//                composite output of the same pixel.
//   k_query      ray queries: per-ray chunk DDA, voxel geometry only.
#pragma once

#include "device_trace.cuh"

namespace vxe {
namespace dev {

struct FrameArgs {
  vxe_camera_gpu cam;
  vxe_clipmap_gpu clip;
  const uint4* nodes;
  uint64_t nodes_n;
  const uint32_t* ropes;
  uint64_t ropes_n;
  const uint4* metas;
  uint64_t metas_n;
  const uint32_t* grid;
  uint64_t grid_n;
  const uint32_t* macro;
  uint64_t macro_n;
  const uint32_t* colinfo;
  uint64_t colinfo_n;
  const float* clip_tex;
  uint32_t clip_layers, clip_res;
  uint32_t* err;
  uint32_t godray_alias;
  uint32_t iw, ih, pw, ph;
  uint32_t* tile_count;  // tiles
  uint32_t* tile_slots;  // tiles * 24
  const uint4* hist_in;
  uint4* hist_out;
  const float* shadow_in;
  float* shadow_out;
  const float4* local_hist_in;
  float4* local_hist_out;
  float4* color;
  float* depth;
  float4* local;  // optional (debug intermediates)
  const float4* god_in;
  float4* god_out;
  float4* pre_taa;  // optional (debug intermediates)
  float4* output;
  const float4* out_hist_in;
  float4* out_hist_out;
  uint4* hits;  // optional, 2 x uint4 per pixel (vxe_hit)
  // wavefront primary: per-pixel trace results + class queues
  uint4* pix_hit;     // 5 x uint4 per pixel (PixHit), written for voxel hits
  uint32_t* q_vox;    // pixel ids with a voxel hit
  uint32_t* q_far;    // pixel ids for heightfield / sky
  uint32_t* q_count;  // [0] voxel, [1] far, [2] fresh shadow, [3] light gather, [4] probes, [5] pending,
                      // [6] slab tasks, [7] slab hits, [8] far pixels queued by the walk
  uint32_t* q_shadow;  // voxel pixels that trace a fresh sun shadow this frame
  uint32_t* q_light;   // voxel pixels that gather local lights
  float* px_shadow;    // fresh sun transmittance per pixel (q_shadow pixels)
  float4* px_light;    // light gather result per pixel (q_light pixels)
  // deferred grass column probes (PROBE_RECORD -> k_probe_dda -> k_slab_eval
  // -> k_slab_pick -> k_primary_resolve)
  ProbeRec* probe_recs;           // stored probes, q_count[4] of them (capped)
  uint32_t probe_cap;
  uint4* slab_tasks;              // one uint4 (slab_task) per grass column slab to march, q_count[6] of them
  float4* slab_res;               // per slab task: hit t, normal (written on hits)
  uint32_t* slab_hits;            // slab tasks that hit, q_count[7] of them
  uint32_t slab_cap;
  unsigned long long* px_first;   // per pixel: nearest probe hit key (slab_key), ~0 = none
  uint32_t* px_task;              // per pixel: the slab task with that key
  uint2* px_mask;                 // per pixel: candidate chunks with a probe hit, hint / full trace
  uint2* px_probe;                // per pixel: walk summary (probe_summary) | probes stored
  uint4* px_gov = nullptr;        // per pending pixel: deferred blade march of its answer (gov_state,
                                  // interval, chunk slot); 3 / 4 once k_gov_eval ran it (hit / miss)
  uint32_t* q_pending;            // pixels whose walk met probes, q_count[5] of them
  // per-frame grass cell table: written by k_grass_cells, read by the rest
  float4* grass_rec;
  uint64_t grass_rec_n;  // records (slots * 4096)
  float* grass_taper;    // 3 LODs x 6 segments
  uint32_t* grass_state;  // per record: lod-0 segment frames built?
  float4* grass_frames;   // per record: the frames
  const uint32_t* slot_lights;  // per slot: holds a LIGHT leaf
  const uint32_t* slot_top;     // per slot: top of its non-air leaves (voxels)
  uint32_t grass_slot0;  // k_grass_cells: first slot of the launch
  uint32_t* grass_list;    // grass columns of the last full build (k_grass_cells appends; null: no list)
  uint32_t* grass_list_n;  // their count
  // profile_counts (ray_main.wgsl:32-74): VOXEL, GRASS, HDR, FOG, SHADOW,
  // added to when cam.profile_flags & 1 (null: not counted)
  uint32_t* profile;
  // Godray integrals of the walk's far pixels, made beside the probe passes
  // (k_godray_far; w = 1 where made, cleared each frame); null: none.
  float4* god_pre = nullptr;
};

// profile_inc / profile_add (ray_main.wgsl:64-74).  The flag is uniform over
// the launch (a kernel parameter), so with it off this is one predicated
// branch.
enum : uint32_t { PROFILE_VOXEL = 0u, PROFILE_GRASS = 1u, PROFILE_HDR = 2u, PROFILE_FOG = 3u, PROFILE_SHADOW = 4u };
__device__ __forceinline__ void profile_add(const FrameArgs& A, uint32_t idx, uint32_t v) {
  if (A.profile != nullptr && (A.cam.profile_flags & 1u) != 0u) atomicAdd(&A.profile[idx], v);
}
// fog_profile_weight (ray_main.wgsl:89-93)
__device__ __forceinline__ uint32_t fog_profile_weight(float t_scene) {
  const float fog_norm = clampf(t_scene / FOG_MAX_DIST, 0.0f, 1.0f);
  return max(1u, to_u32(fog_norm * 256.0f));
}

// The arguments of up to kMaxViewsPerLaunch views' frames, rendered by one
// launch of each pass: blockIdx.z selects the view.
constexpr uint32_t kMaxViewsPerLaunch = 8u;
struct FrameArgsViews {
  FrameArgs v[kMaxViewsPerLaunch];
};

__device__ __forceinline__ Scene make_scene(const FrameArgs& A, bool godray) {
  Scene s;
  s.cam = &A.cam;
  s.clip = &A.clip;
  s.nodes = A.nodes;
  s.nodes_n = A.nodes_n;
  s.ropes = A.ropes;
  s.ropes_n = A.ropes_n;
  s.metas = A.metas;
  s.metas_n = A.metas_n;
  s.grid = A.grid;
  s.grid_n = A.grid_n;
  if (godray && A.godray_alias) {
    // Reference binding mismatch: main_godray's macro_occ reads the rope buffer.
    s.macro = A.ropes;
    s.macro_n = A.ropes_n * 8u;
  } else {
    s.macro = A.macro;
    s.macro_n = A.macro_n;
  }
  s.colinfo = A.colinfo;
  s.colinfo_n = A.colinfo_n;
  s.clip_tex = A.clip_tex;
  s.clip_layers = A.clip_layers;
  s.clip_res = A.clip_res;
  s.err = A.err;
  s.grass_rec = A.grass_rec;
  s.grass_rec_n = A.grass_rec_n;
  s.grass_taper = A.grass_taper;
  s.grass_state = A.grass_rec ? A.grass_state : nullptr;
  s.grass_frames = A.grass_rec ? A.grass_frames : nullptr;
  s.slot_lights = A.slot_lights;
  s.slot_top = A.slot_top;
  return s;
}

// ---------------------------------------------------------------------------
// Per-frame grass cell table (see GRASS_REC_F4): one thread per column of
// every resident chunk; grass column tops get their blade geometry for this
// frame's wind, every other column a NaN id so no stale record can match.
// Thread 0 also writes the per-LOD blade taper.
// ---------------------------------------------------------------------------
constexpr int GRASS_CELL_THREADS = 128;

// Record g (slot g >> 12, column g & 4095) for this camera's wind; with
// `list`, grass columns also append g to the grass column list.
__device__ __forceinline__ void grass_column_build(const FrameArgs& A, const Scene& s, uint64_t g, bool list) {
  const uint32_t slot = (uint32_t)(g >> 12), col = (uint32_t)(g & 4095u);
  if (slot >= A.cam.chunk_count || (uint64_t)slot * 4096u >= A.grass_rec_n) return;
  float4* r = A.grass_rec + g * GRASS_REC_F4;
  if (A.grass_state) A.grass_state[g] = 0u;  // this frame's segment frames are built on first use
  const Meta m = meta_at(s, slot);
  const float nan = __uint_as_float(0x7FC00000u);
  if (m.colinfo_base == INVALID) {
    r[0] = make_float4(0.0f, nan, nan, nan);
    return;
  }
  const uint32_t lx = col & 63u, lz = col >> 6;
  const ColInfo ci = colinfo_decode(colinfo_entry_u16(s, m.colinfo_base, lx, lz));
  if (!(ci.valid && ci.mat == MAT_GRASS)) {
    r[0] = make_float4(0.0f, nan, nan, nan);
    return;
  }
  if (list) {  // warp-aggregated append
    const uint32_t mask = __activemask(), lane = threadIdx.x & 31u, leader = __ffs(mask) - 1u;
    uint32_t base = 0u;
    if (lane == leader) base = atomicAdd(A.grass_list_n, (uint32_t)__popc(mask));
    base = __shfl_sync(mask, base, leader);
    A.grass_list[base + __popc(mask & ((1u << lane) - 1u))] = (uint32_t)g;
  }
  // The cell the column probe and the grass-voxel hit derive
  // (chunk_trace.wgsl:1434-1445).
  const float vs = vs_(s);
  const v3 id = V3((float)(m.ox + (int32_t)lx), (float)(m.oy + (int32_t)ci.y_vox), (float)(m.oz + (int32_t)lz));
  const v3 cb = id * vs;
  const float time_s = A.cam.voxel_params[1], strength = A.cam.voxel_params[2];
  GrassBladeGeom B[GRASS_BLADE_COUNT];
  for (uint32_t i = 0; i < GRASS_BLADE_COUNT; ++i) grass_blade_geom(s, cb, id, time_s, strength, i, B[i]);
  const float blade_len = grass_blade_len(s, id);
  grass_rec_store(r, blade_len, id, B);
  // Columns within the lod-0 range of this camera also get their segment
  // frames now (the values grass_frames_ready would build on first use).
  if (A.grass_state && A.grass_frames &&
      length(cb + V3s(0.5f * vs) - cam_pos(s)) < GRASS_LOD_MID_START + 1.0f + 4.0f * vs) {
    const uint32_t segs = grass_lod_segs(0u);
    const float inv_segs = 1.0f / fmax_((float)segs, 1.0f);
    float4* F = A.grass_frames + g * GRASS_FRAME_F4;
    for (uint32_t i = 0; i < GRASS_BLADE_COUNT; ++i)
      for (uint32_t sg = 0; sg < segs; ++sg) {
        const GrassSegFrame f = grass_seg_frame(B[i], blade_len, inv_segs, grass_taper_value(inv_segs, sg), sg);
        float4* o = F + 3u * (i * segs + sg);
        o[0] = make_float4(f.mid.x, f.mid.y, f.mid.z, f.half_w);
        o[1] = make_float4(f.S.x, f.S.y, f.S.z, f.half_h);
        o[2] = make_float4(f.T.x, f.T.y, f.T.z, 0.0f);
      }
    A.grass_state[g] = 2u;
  }
}

// Every column of slots [grass_slot0, ...): one thread per column; with a
// grass list, the grass columns are appended to it.  Thread 0 also writes the
// per-LOD blade taper.
__global__ void __launch_bounds__(GRASS_CELL_THREADS) k_grass_cells(const __grid_constant__ FrameArgs A) {
  const uint64_t g = (uint64_t)A.grass_slot0 * 4096u + (uint64_t)blockIdx.x * GRASS_CELL_THREADS + threadIdx.x;
  const Scene s = make_scene(A, false);
  if (g == 0u) {
    for (uint32_t lod = 0; lod < 3u; ++lod) {
      const uint32_t segs = grass_lod_segs(lod);
      const float inv_segs = 1.0f / fmax_((float)segs, 1.0f);
      for (uint32_t sg = 0; sg < 6u; ++sg) A.grass_taper[lod * 6u + sg] = sg < segs ? grass_taper_value(inv_segs, sg) : 0.0f;
    }
  }
  grass_column_build(A, s, g, A.grass_list != nullptr);
}

// A new wind over an unchanged world: only the grass columns (the list of
// the last full build) change; every other record keeps its NaN id.
__global__ void __launch_bounds__(GRASS_CELL_THREADS) k_grass_wind(const __grid_constant__ FrameArgs A) {
  const Scene s = make_scene(A, false);
  const uint32_t n = *A.grass_list_n;
  for (uint32_t i = blockIdx.x * GRASS_CELL_THREADS + threadIdx.x; i < n; i += gridDim.x * GRASS_CELL_THREADS)
    grass_column_build(A, s, A.grass_list[i], false);
}

// ---------------------------------------------------------------------------
// Per-slot flags: one block per slot of [slot0, slot0 + gridDim.x), over
// the node records of its meta's range: whether one is a LIGHT leaf, and the
// top of the non-air leaves (a leaf's cube from its key: coordinates in units
// of the cube size 2^(log2(chunk) - level)).  Every point of the chunk above
// that top is in an air leaf, an implicit air child or an empty macro cell.
// ---------------------------------------------------------------------------
constexpr int SLOT_LIGHT_THREADS = 256;

__global__ void __launch_bounds__(SLOT_LIGHT_THREADS) k_slot_lights(const uint4* metas, uint64_t metas_n,
                                                                     const uint4* nodes, uint64_t nodes_n,
                                                                     uint32_t slot0, uint32_t chunk_size,
                                                                     uint32_t* out, uint32_t* top_out) {
  __shared__ uint32_t top_s;
  const uint32_t slot = slot0 + blockIdx.x;
  if (slot >= metas_n) return;
  if (threadIdx.x == 0) top_s = 0u;
  __syncthreads();
  const uint4 b = metas[(size_t)slot * 3u + 1u];  // node_base, node_count, macro_base, colinfo_base
  int any = 0;
  uint32_t top = 0u;
  for (uint32_t i = threadIdx.x; i < b.y; i += SLOT_LIGHT_THREADS) {
    const uint64_t gi = (uint64_t)b.x + i;
    if (gi >= nodes_n) break;
    const uint4 n = nodes[gi];
    any |= (n.x == LEAF && n.z == MAT_LIGHT) ? 1 : 0;
    if (n.x == LEAF && n.z != MAT_AIR) {
      const uint32_t lvl = (n.w >> 18) & 7u, y = (n.w >> 6) & 63u;
      top = max(top, (y + 1u) * (chunk_size >> lvl));
    }
  }
  atomicMax(&top_s, top);
  any = __syncthreads_or(any);
  if (threadIdx.x == 0) {
    out[slot] = any ? 1u : 0u;
    top_out[slot] = top_s;
  }
}

// ---------------------------------------------------------------------------
// Tile candidate lists
// ---------------------------------------------------------------------------
constexpr int TILE_THREADS = 32;
#define TILE_THREADS_DECL 32

// Candidate list of logical tile (tx, ty) for this lane; `sl` / `en` are the
// block's [MAX_TILE_CHUNKS][TILE_THREADS] shared scratch.  Writes the clamped
// count and 24 slots (INVALID-padded) to out_count / out_slots.
__device__ __noinline__ void build_tile_list(const Scene& s, uint32_t tx, uint32_t ty, uint32_t lane,
                                             uint32_t (*sl)[TILE_THREADS_DECL], float (*en)[TILE_THREADS_DECL],
                                             uint32_t* out_count, uint32_t* out_slots) {
  uint32_t count = 0;
  if (s.cam->chunk_count != 0u) {
    const v2 base = V2((float)(tx * TILE_SIZE), (float)(ty * TILE_SIZE));
    const v3 ro = cam_pos(s);
    auto add = [&](uint32_t slot, float te) -> bool {
      // tile_add_candidate (chunk_trace.wgsl:1007-1026)
      if (slot < s.cam->chunk_count && meta_empty(s, slot) != 0u) return false;
      for (uint32_t i = 0; i < count && i < MAX_TILE_CHUNKS; ++i) {
        if (sl[i][lane] == slot) {
          en[i][lane] = fminf(en[i][lane], te);
          return false;
        }
      }
      const uint32_t idx = count++;
      if (idx < MAX_TILE_CHUNKS) {
        sl[idx][lane] = slot;
        en[idx][lane] = te;
      }
      return false;
    };
    chunk_grid_dda(s, ro, ray_dir_from_pixel(s, base + V2(4.5f, 4.5f)), 0.0f, FOG_MAX_DIST, add);
    chunk_grid_dda(s, ro, ray_dir_from_pixel(s, base + V2(1.5f, 1.5f)), 0.0f, FOG_MAX_DIST, add);
  }
  const uint32_t raw = min(count, MAX_TILE_CHUNKS);
  const uint32_t limit = min(raw, TILE_CANDS);
  // tile_sort_candidates_by_enter (chunk_trace.wgsl:1153-1175): selection sort of the first 24.
  if (raw > 1u && limit > 1u) {
    for (uint32_t i = 0; i + 1u < limit; ++i) {
      uint32_t mi = i;
      float mt = en[i][lane];
      for (uint32_t j = i + 1u; j < limit; ++j) {
        const float e = en[j][lane];
        if (e < mt) { mt = e; mi = j; }
      }
      if (mi != i) {
        const uint32_t ts = sl[i][lane];
        const float tt = en[i][lane];
        sl[i][lane] = sl[mi][lane];
        en[i][lane] = en[mi][lane];
        sl[mi][lane] = ts;
        en[mi][lane] = tt;
      }
    }
  }
  *out_count = limit;
  for (uint32_t i = 0; i < TILE_CANDS; ++i) out_slots[i] = i < limit ? sl[i][lane] : INVALID;
}

__device__ __forceinline__ void k_tiles_body(const FrameArgs& A) {
  __shared__ uint32_t sl[MAX_TILE_CHUNKS][TILE_THREADS];
  __shared__ float en[MAX_TILE_CHUNKS][TILE_THREADS];
  const uint32_t lane = threadIdx.x;
  const uint32_t tiles_x = (A.iw + 7u) / 8u, tiles_y = (A.ih + 7u) / 8u;
  const uint32_t tile = blockIdx.x * TILE_THREADS + lane;
  if (tile >= tiles_x * tiles_y) return;
  const Scene s = make_scene(A, false);
  build_tile_list(s, tile % tiles_x, tile / tiles_x, lane, sl, en, &A.tile_count[tile],
                  &A.tile_slots[(size_t)tile * TILE_CANDS]);
}
__global__ void __launch_bounds__(TILE_THREADS) k_tiles(const __grid_constant__ FrameArgs A) { k_tiles_body(A); }
__global__ void __launch_bounds__(TILE_THREADS) k_tiles_views(const __grid_constant__ FrameArgsViews V) {
  k_tiles_body(V.v[blockIdx.z]);
}

// trace_scene_voxels_candidates (chunk_trace.wgsl:1177-1265) over a tile list
// staged in shared memory (slots + their ChunkMeta records).
template <uint32_t PM>
__device__ VoxTraceResult trace_candidates(const Scene& s, const uint32_t* cslot, const Meta* cmeta, v3 ro, v3 rd,
                                           float t_min, float t_max, bool anchor_valid_in, i3 anchor_chunk_in,
                                           uint32_t anchor_key_in, uint32_t cand_count, ProbeHook& ph) {
  VoxTraceResult none{false, miss_hitgeom(), 0.0f, false, INVALID, i3{0, 0, 0}};
  ph.best_cand = INVALID;
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
  const uint32_t maxc = min(cand_count, MAX_TILE_CHUNKS);
  const TraceOpts opt{false};
  // With a deferred blade march (ChunkTraceResult::gov) a chunk's final t is
  // its voxel hit's or one in the march's slab interval: only bounded.  The
  // skip test takes the nearest upper bound, so every chunk the reference
  // walks is walked here; the answer is decided at the end when no other
  // chunk's lower bound reaches its upper bound (with no deferred march
  // these are the plain t's and this is the reference's loop).
  float skip_t = BIG;
  float lo_gov = BIG, lo_plain = BIG;  // lowest final t of the other chunks, deferred / plain
  bool a_gov = false;
  float a_t0 = 0.0f, a_t1 = 0.0f, a_hi = 0.0f, a_lo = 0.0f;
  uint32_t a_slot = 0u;
  for (uint32_t i = 0; i < maxc; ++i) {
    const uint32_t slot = cslot[i];
    if (slot == INVALID || slot >= s.cam->chunk_count) continue;
    const Meta ch = cmeta ? cmeta[i] : meta_at(s, slot);
    if (ch.macro_empty != 0u) continue;
    const v3 rb = V3((float)ch.ox, (float)ch.oy, (float)ch.oz) * vsz;
    const v2 rt = intersect_aabb(ro, rd, rb, rb + V3s(rs));
    const float ce = fmax_(rt.x, t_enter), cx = fmin_(rt.y, t_exit);
    if (cx < ce) continue;
    if (ce >= skip_t) continue;
    if (chunk_heightfield_early_skip(s, ro, rd, ce, cx, ch, vsz)) continue;
    const int32_t csz = (int32_t)s.cam->chunk_size;
    const i3 cc{ch.ox / csz, ch.oy / csz, ch.oz / csz};
    const bool ua = anchor_valid_in && chunk_coords_neighbor(cc, anchor_chunk_in);
    const uint32_t aku = ua ? anchor_key_in : INVALID;
    ph.slot = slot;
    ph.cand = i;
    const ChunkTraceResult h = trace_chunk_interval_stream_macro<PM>(s, ro, rd, inv, ch, ce, cx, ua, aku, opt, ph);
    if (h.hit.hit == 0u) continue;
    const float lo = h.gov ? fmin_(h.hit.t, h.gov_lo) : h.hit.t;
    const float hi = h.gov ? fmax_(h.hit.t, h.gov_hi) : h.hit.t;
    skip_t = fmin_(skip_t, hi);
    if (h.hit.t < best.t) {
      if (best.hit != 0u) {  // the previous answer becomes another chunk
        if (a_gov) lo_gov = fmin_(lo_gov, a_lo);
        else lo_plain = fmin_(lo_plain, best.t);
      }
      best = h.hit;
      bav = h.anchor_valid;
      bak = h.anchor_key;
      bac = cc;
      ph.best_cand = i;
      a_gov = h.gov;
      a_t0 = h.gov_t0;
      a_t1 = h.gov_t1;
      a_lo = lo;
      a_hi = hi;
      a_slot = slot;
    } else if (h.gov) {
      lo_gov = fmin_(lo_gov, lo);
    } else {
      lo_plain = fmin_(lo_plain, h.hit.t);
    }
  }
  VoxTraceResult r{true, best, t_exit, bav, bak, bac};
  if (best.hit != 0u) {
    const float up = a_gov ? a_hi : best.t;
    if (lo_gov <= up || (a_gov && lo_plain <= up)) r.gov_state = 2u;
    else if (a_gov) r.gov_state = 1u;
    r.gov_t0 = a_t0;
    r.gov_t1 = a_t1;
    r.gov_slot = a_slot;
  }
  return r;
}

// ---------------------------------------------------------------------------
// Hit records
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t face_from_n(v3 n) {
  const float ax = fabsf(n.x), ay = fabsf(n.y), az = fabsf(n.z);
  if (ax >= ay && ax >= az) return n.x > 0.0f ? 0u : 1u;
  if (ay >= az) return n.y > 0.0f ? 2u : 3u;
  return n.z > 0.0f ? 4u : 5u;
}

struct HitRec {
  float t;
  uint32_t node;
  int32_t vx, vy, vz;
  uint32_t face, mat;
};

__device__ __forceinline__ HitRec miss_rec() { return HitRec{BIG, INVALID, 0, 0, 0, 255u, 0u}; }

__device__ HitRec make_rec(const HitGeom& g, v3 ro, v3 rd, float vs, bool voxel_hit) {
  HitRec h;
  h.t = g.t;
  h.node = g.node;
  h.mat = g.mat;
  h.face = face_from_n(g.n);
  const v3 p = ro + rd * g.t;
  if (voxel_hit) {
    const v3 lr = (p - g.root_bmin) / vs;
    const v3 lmin = (g.leaf_bmin - g.root_bmin) / vs;
    const int32_t l0x = to_i32(floorf(lmin.x + 0.5f)), l0y = to_i32(floorf(lmin.y + 0.5f)),
                  l0z = to_i32(floorf(lmin.z + 0.5f));
    const int32_t ls = to_i32(floorf(g.leaf_size / vs + 0.5f));
    const int32_t ox = to_i32(floorf(g.root_bmin.x / vs + 0.5f)), oy = to_i32(floorf(g.root_bmin.y / vs + 0.5f)),
                  oz = to_i32(floorf(g.root_bmin.z / vs + 0.5f));
    h.vx = ox + clampi(to_i32(floorf(lr.x)), l0x, l0x + ls - 1);
    h.vy = oy + clampi(to_i32(floorf(lr.y)), l0y, l0y + ls - 1);
    h.vz = oz + clampi(to_i32(floorf(lr.z)), l0z, l0z + ls - 1);
  } else {
    h.vx = to_i32(floorf(p.x / vs));
    h.vy = to_i32(floorf(p.y / vs));
    h.vz = to_i32(floorf(p.z / vs));
  }
  return h;
}

__device__ __forceinline__ void store_rec(uint4* dst, const HitRec& h) {
  dst[0] = make_uint4(__float_as_uint(h.t), h.node, (uint32_t)h.vx, (uint32_t)h.vy);
  dst[1] = make_uint4((uint32_t)h.vz, h.face, h.mat, 0u);
}

__device__ __forceinline__ uint32_t pack_i16x2(int32_t a, int32_t b) {
  return ((uint32_t)a & 0xFFFFu) | (((uint32_t)b & 0xFFFFu) << 16);
}
__device__ __forceinline__ int32_t unpack_i16(uint32_t v) {
  const int32_t s = (int32_t)(v & 0xFFFFu);
  return (v & 0x8000u) != 0u ? s - 0x10000 : s;
}
__device__ __forceinline__ int32_t nearest_idx(float u, uint32_t n) {
  return clampi(to_i32(floorf(u * (float)n)), 0, (int32_t)n - 1);
}
__device__ __forceinline__ v3 xyz(float4 v) { return V3(v.x, v.y, v.z); }

// ---------------------------------------------------------------------------
// Primary pass (+ fused local TAA)
//
// Two schedules of the same per-pixel function:
//   k_primary            one thread per pixel does trace + shading (megakernel);
//   k_primary_trace  ->  k_shade_vox / k_shade_far  (wavefront): the trace
//       kernel classifies each pixel (voxel hit vs heightfield/sky) into a
//       queue with warp-aggregated atomics and stores the hit; each shading
//       kernel then runs over one class only, so sky cloud marches, terrain
//       marches and voxel shading no longer share warps.  Queue order does not
//       matter: every pixel's result depends only on its own inputs.
// ---------------------------------------------------------------------------
constexpr int PRIMARY_THREADS = 128;  // two 8x8 logical tiles per block
constexpr int SHADE_THREADS = 128;
// Blocks per SM the heavier shading kernels are compiled for (48 registers a
// thread instead of 96-128, a few spills: measured 0.11 ms faster per 1080p
// frame than without the bound; 6, 8 and 10 blocks gave 0.05, 0.09, 0.11).
constexpr int SHADE_MIN_BLOCKS = 10;
// Blocks per SM of the blade-march kernels (64 registers a thread instead of
// 80: more marches in flight, measured 0.08 ms faster per 1080p frame).
constexpr int SLAB_MIN_BLOCKS = 8;

struct PrimaryCtx {
  uint32_t gx, gy;
  size_t pix;
  v2 px;
  uint32_t seed;
  v3 ro, rd;
};

__device__ __forceinline__ PrimaryCtx primary_ctx(const Scene& s, uint32_t gx, uint32_t gy, uint32_t W) {
  PrimaryCtx c;
  c.gx = gx;
  c.gy = gy;
  c.pix = (size_t)gy * W + gx;
  c.px = V2((float)gx + 0.5f, (float)gy + 0.5f);
  c.seed = (gx * 1973u) ^ (gy * 9277u) ^ (s.cam->frame_index * 26699u);
  c.ro = cam_pos(s);
  c.rd = ray_dir_from_pixel(s, c.px);
  return c;
}

// The primary-hit history hint (ray_main.wgsl:274-318): the previous hit
// distance at this pixel, accepted when its reprojection agrees in depth and
// motion; with it the window the first trace phase searches and the anchor.
struct PrimaryHint {
  bool valid;
  float t_start, t_end;
  uint32_t anchor_key;  // INVALID: none
  i3 anchor_chunk;
};

__device__ __forceinline__ PrimaryHint primary_hint(const Scene& s, const FrameArgs& A, const PrimaryCtx& c) {
  const uint32_t W = A.iw, H = A.ih;
  const v2 res = V2((float)W, (float)H);
  float t_hist = 0.0f;
  PrimaryHint h{false, 0.0f, 0.0f, INVALID, i3{0, 0, 0}};
  const v2 uv = c.px / res;
  const float t_guess = __uint_as_float(A.hist_in[c.pix].x);
  if (t_guess > 1e-3f) {
    const v3 p_ws = c.ro + c.rd * t_guess;
    const v2 uvp = prev_uv_from_world(s, p_ws);
    if (in_unit_square(uvp)) {
      const int32_t sx = nearest_idx(uvp.x, W), sy = nearest_idx(uvp.y, H);
      const uint4 hp = A.hist_in[(size_t)sy * W + (uint32_t)sx];
      const float t_prev = __uint_as_float(hp.x);
      const float rel = fabsf(t_prev - t_guess) / fmax_(t_guess, 1e-3f);
      const float depth_ok = 1.0f - smooth(PRIMARY_HIT_DEPTH_REL0, PRIMARY_HIT_DEPTH_REL1, rel);
      const float vel = length((uvp - uv) * res);
      const float motion_ok = 1.0f - smooth(PRIMARY_HIT_MOTION_PX0, PRIMARY_HIT_MOTION_PX1, vel);
      if (t_prev > 1e-3f && depth_ok > 0.5f && motion_ok > 0.5f) {
        t_hist = t_prev;
        h.valid = true;
        if ((hp.w & 0x80000000u) != 0u) {
          h.anchor_key = hp.y;
          h.anchor_chunk = i3{unpack_i16(hp.z), unpack_i16(hp.z >> 16), unpack_i16(hp.w)};
        }
      }
    }
  }
  h.t_start = fmax_(t_hist - PRIMARY_HIT_MARGIN, 0.0f);
  h.t_end = fmin_(t_hist + PRIMARY_HIT_WINDOW, FOG_MAX_DIST);
  return h;
}

// History hint + voxel trace (ray_main.wgsl:274-325 and trace_primary_voxels :116-161).
template <uint32_t PM>
__device__ __noinline__ VoxTraceResult primary_trace(const Scene& s, const FrameArgs& A, const PrimaryCtx& c,
                                                     const uint32_t* cslot, const Meta* cmeta, uint32_t tile_count,
                                                     ProbeHook& ph) {
  VoxTraceResult vt{false, miss_hitgeom(), 0.0f, false, INVALID, i3{0, 0, 0}};
  if (s.cam->chunk_count == 0u || tile_count == 0u) return vt;
  const PrimaryHint hh = primary_hint(s, A, c);
  // phase 0: the hint window (when the history is valid); phase 1: the full
  // trace when phase 0 found nothing.  One call site keeps one copy of the walk.
  ph.first_phase = hh.valid ? 0u : 1u;
  for (uint32_t phase = ph.first_phase;; ++phase) {
    const bool w = phase == 0u;
    ph.phase = phase;
    const VoxTraceResult h =
        trace_candidates<PM>(s, cslot, cmeta, c.ro, c.rd, w ? hh.t_start : 0.0f, w ? hh.t_end : FOG_MAX_DIST,
                             w && hh.anchor_key != INVALID, w ? hh.anchor_chunk : i3{0, 0, 0},
                             w ? hh.anchor_key : INVALID, tile_count, ph);
    if (!w || h.best.hit != 0u) return h;
  }
}

// PROFILE_VOXEL of trace_primary_voxels (ray_main.wgsl:130-148): the tile's
// candidate count once per trace phase run; `last_phase` is the phase that
// gave the answer (1 when none did).
__device__ __forceinline__ void profile_voxel(const FrameArgs& A, uint32_t first_phase, uint32_t last_phase,
                                              uint32_t tile_count) {
  if (first_phase > 1u) return;
  profile_add(A, PROFILE_VOXEL, max(1u, tile_count) * (last_phase - first_phase + 1u));
}

// main_local_taa (taa.wgsl:26-69) for one pixel, fused after its shading.
__device__ __forceinline__ void local_taa_store(const FrameArgs& A, size_t pix, v3 local_out, float local_w) {
  if (A.local) A.local[pix] = make_float4(local_out.x, local_out.y, local_out.z, local_w);
  const float4 h4 = A.local_hist_in[pix];
  const bool hist_ok = !is_bad(xyz(h4));
  const v3 hl = hist_ok ? xyz(h4) : V3s(0.0f);
  const float conf0 = hist_ok ? h4.w : 0.0f;
  const bool has_sample = local_w > 0.0f && !is_bad(local_out);
  const float k = has_sample ? LOCAL_TAA_ALPHA * clampf(local_w, 0.0f, 1.0f) : 0.0f;
  const v3 ol = vmix(hl, local_out, k);
  const float conf1 = has_sample ? fmin_(1.0f, conf0 + k) : conf0;
  A.local_hist_out[pix] = make_float4(ol.x, ol.y, ol.z, conf1);
}

// Voxel-hit shading (ray_main.wgsl:374-471) + outputs, in the parts the
// wavefront schedule runs as separate kernels:
//   grass_refine         grass-on-voxel slab march (may move t and n)
//   shadow_blend         1/8 of the pixels per frame: reprojected shadow
//                        history mixed with a fresh sun transmittance
//   gather_voxel_lights  local light gather (8 rays)
//   shade_voxel_final    surface shading, fog, outputs, fused local TAA.
__device__ __forceinline__ bool grass_refine(const Scene& s, const PrimaryCtx& c, HitGeom& best) {
  if (best.mat != MAT_GRASS) return false;
  const float vs = vs_(s);
  const int32_t csv = (int32_t)s.cam->chunk_size;
  const i3 ov{to_i32(floorf(best.root_bmin.x / vs + 0.5f)), to_i32(floorf(best.root_bmin.y / vs + 0.5f)),
              to_i32(floorf(best.root_bmin.z / vs + 0.5f))};
  const v3 hp = c.ro + c.rd * best.t;
  const GrassCell cell = pick_grass_cell_in_chunk_with_bias(hp, c.rd, best.root_bmin, ov, vs, csv);
  const GrassHit gh = try_grass_slab_hit(s, c.ro, c.rd, 0.0f, best.t, cell.bmin_m, cell.id_vox, vs,
                                         s.cam->voxel_params[1], s.cam->voxel_params[2]);
  if (gh.hit) { best.t = gh.t; best.n = gh.n; }
  return gh.hit;
}

__device__ __forceinline__ bool shadow_fresh(const PrimaryCtx& c) { return (c.seed & SHADOW_SUBSAMPLE_MASK) == 0u; }
__device__ __forceinline__ bool lights_wanted(const HitGeom& best) {
  return best.hit != 0u && best.mat != MAT_LIGHT && best.t <= LOCAL_LIGHT_MAX_DIST;
}
__device__ __forceinline__ v3 shadow_origin(const Scene& s, const PrimaryCtx& c, const HitGeom& best) {
  return (c.ro + c.rd * best.t) + best.n * (0.75f * vs_(s));
}

// Shadow for a pixel whose fresh transmittance is `cur` (shadow_fresh).
__device__ __forceinline__ float shadow_blend(const Scene& s, const FrameArgs& A, const PrimaryCtx& c, v3 hp, float cur) {
  const uint32_t W = A.iw, H = A.ih;
  float sh = A.shadow_in[c.pix];
  const v2 uvp = prev_uv_from_world(s, hp);
  if (in_unit_square(uvp)) {
    const int32_t ppx = clampi(to_i32(uvp.x * (float)W), 0, (int32_t)W - 1);
    const int32_t ppy = clampi(to_i32(uvp.y * (float)H), 0, (int32_t)H - 1);
    sh = A.shadow_in[(size_t)ppy * W + (uint32_t)ppx];
  }
  sh = clampf(sh, 0.0f, 1.0f);
  return mixf(sh, cur, SHADOW_TAA_ALPHA);
}

// `light` is gather_voxel_lights' result when lights_wanted(best).
// `depth_written`: k_shade_prep already stored this pixel's depth.
__device__ __noinline__ void shade_voxel_final(const Scene& s, const FrameArgs& A, const PrimaryCtx& c,
                                               const HitGeom& best, float shadow_out, v3 light, bool anchor_valid,
                                               uint32_t anchor_key, i3 anchor_chunk, bool depth_written) {
  const float vs = vs_(s);
  const v3 ro = c.ro, rd = c.rd;
  const v3 sky_up = sky_bg(V3(0.0f, 1.0f, 0.0f));
  const v3 base_hdr = shade_hit(s, ro, rd, best, sky_up, shadow_out);
  v3 local_out = V3s(0.0f);
  float local_w = 0.0f;
  if (lights_wanted(best)) {
    const v3 hpl = ro + rd * best.t;
    const v3 alb = base_albedo(best.mat, hpl, best.t);
    local_out = light * alb;
    local_w = 1.0f;
  }
  const float t_scene = fmin_(best.t, FOG_MAX_DIST);
  const v3 col = apply_fog(s, base_hdr, ro, rd, t_scene, sky_bg(rd));
  profile_add(A, PROFILE_SHADOW, shadow_fresh(c) ? 2u : 1u);
  profile_add(A, PROFILE_HDR, 2u);
  profile_add(A, PROFILE_FOG, fog_profile_weight(t_scene));
  uint32_t pxy = 0u, pz = 0u, ak = 0u;
  if (anchor_valid) {
    pxy = pack_i16x2(anchor_chunk.x, anchor_chunk.y);
    pz = pack_i16x2(anchor_chunk.z, 0) | 0x80000000u;
    ak = anchor_key;
  }
  A.color[c.pix] = make_float4(col.x, col.y, col.z, 1.0f);
  if (!depth_written) A.depth[c.pix] = t_scene;
  A.hist_out[c.pix] = make_uint4(__float_as_uint(t_scene), ak, pxy, pz);
  A.shadow_out[c.pix] = shadow_out;
  if (A.hits) store_rec(A.hits + c.pix * 2u, make_rec(best, ro, rd, vs, true));
  local_taa_store(A, c.pix, local_out, local_w);
}

// The whole voxel-hit shading of one pixel (megakernel schedule).
__device__ __noinline__ void shade_voxel_pixel(const Scene& s, const FrameArgs& A, const PrimaryCtx& c, HitGeom best,
                                               bool anchor_valid, uint32_t anchor_key, i3 anchor_chunk) {
  if (grass_refine(s, c, best)) profile_add(A, PROFILE_GRASS, 1u);
  float shadow_out;
  if (shadow_fresh(c)) {
    const float cur = sun_transmittance_geom_only(s, shadow_origin(s, c, best), SUN_DIR);
    shadow_out = shadow_blend(s, A, c, c.ro + c.rd * best.t, cur);
  } else {
    shadow_out = clampf(A.shadow_in[c.pix], 0.0f, 1.0f);
  }
  v3 light = V3s(0.0f);
  if (lights_wanted(best)) light = gather_voxel_lights(s, c.ro + c.rd * best.t, best.n, best.root_bmin);
  shade_voxel_final(s, A, c, best, shadow_out, light, anchor_valid, anchor_key, anchor_chunk, false);
}

// Heightfield then sky (ray_main.wgsl:224-269 / 327-372 / 473-516) + outputs.
__device__ __noinline__ void shade_far_pixel(const Scene& s, const FrameArgs& A, const PrimaryCtx& c) {
  const float vs = vs_(s);
  const v3 ro = c.ro, rd = c.rd;
  HitRec rec = miss_rec();
  v3 col;
  float depth, t_store = 0.0f;
  // With no voxel chunks the reference traces the heightfield but draws sky
  // (ray_main.wgsl:219-231).
  ClipHit hf{false, BIG, V3s(0.0f), MAT_AIR};
  if (s.cam->chunk_count != 0u) hf = clip_trace_heightfield(s, ro, rd, 0.0f, FOG_MAX_DIST);
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
        profile_add(A, PROFILE_GRASS, 1u);
      }
    }
    const v3 surface = shade_clip_hit(s, ro, rd, hf, sky_bg(V3(0.0f, 1.0f, 0.0f)));
    const float t_scene = fmin_(hf.t, FOG_MAX_DIST);
    col = apply_fog(s, surface, ro, rd, t_scene, sky_bg(rd));
    profile_add(A, PROFILE_HDR, 1u);
    profile_add(A, PROFILE_FOG, fog_profile_weight(t_scene));
    depth = t_scene;
    t_store = t_scene;
    HitGeom g = miss_hitgeom();
    g.hit = 1u;
    g.t = hf.t;
    g.n = hf.n;
    g.mat = hf.mat;
    rec = make_rec(g, ro, rd, vs, false);
  } else {
    col = sky_color(s, rd);
    depth = FOG_MAX_DIST;
  }
  A.color[c.pix] = make_float4(col.x, col.y, col.z, 1.0f);
  A.depth[c.pix] = depth;
  A.hist_out[c.pix] = make_uint4(__float_as_uint(t_store), 0u, 0u, 0u);
  A.shadow_out[c.pix] = 1.0f;
  if (A.hits) store_rec(A.hits + c.pix * 2u, rec);
  local_taa_store(A, c.pix, V3s(0.0f), 0.0f);
}

// Stages a block's two tile candidate lists (slots + ChunkMeta) in shared memory.
__device__ __forceinline__ void stage_tiles(const Scene& s, const FrameArgs& A, uint32_t (*cslot)[TILE_CANDS],
                                            Meta (*cmeta)[TILE_CANDS], uint32_t* ccount) {
  const uint32_t tid = threadIdx.x;
  const uint32_t tiles_x = (A.iw + 7u) / 8u;
  if (tid < 2u * TILE_CANDS) {
    const uint32_t t = tid / TILE_CANDS, i = tid % TILE_CANDS;
    const uint32_t tx = blockIdx.x * 2u + t;
    uint32_t n = 0u, slot = INVALID;
    if (tx < tiles_x) {
      const size_t tile = (size_t)blockIdx.y * tiles_x + tx;
      n = A.tile_count[tile];
      slot = A.tile_slots[tile * TILE_CANDS + i];
    }
    if (i == 0u) ccount[t] = n;
    cslot[t][i] = slot;
    if (i < n && slot != INVALID && slot < s.cam->chunk_count) cmeta[t][i] = meta_at(s, slot);
  }
  __syncthreads();
}

// Pixel of this thread in the two-tile block layout (warps of 8x4 pixels).
__device__ __forceinline__ bool block_pixel(const FrameArgs& A, uint32_t* t, uint32_t* gx, uint32_t* gy) {
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const uint32_t tiles_x = (A.iw + 7u) / 8u;
  *t = warp >> 1;
  const uint32_t tx = blockIdx.x * 2u + *t;
  *gx = tx * 8u + (lane & 7u);
  *gy = blockIdx.y * 8u + (warp & 1u) * 4u + (lane >> 3);
  return tx < tiles_x && *gx < A.iw && *gy < A.ih;
}

__global__ void __launch_bounds__(PRIMARY_THREADS) k_primary(const __grid_constant__ FrameArgs A) {
  __shared__ uint32_t cslot[2][TILE_CANDS];
  __shared__ Meta cmeta[2][TILE_CANDS];
  __shared__ uint32_t ccount[2];
  const Scene s = make_scene(A, false);
  stage_tiles(s, A, cslot, cmeta, ccount);
  uint32_t t, gx, gy;
  if (!block_pixel(A, &t, &gx, &gy)) return;
  const PrimaryCtx c = primary_ctx(s, gx, gy, A.iw);
  ProbeHook ph = probe_hook_inline();
  const VoxTraceResult vt = primary_trace<PROBE_INLINE>(s, A, c, cslot[t], cmeta[t], ccount[t], ph);
  profile_voxel(A, ph.first_phase, ph.phase, ccount[t]);
  if (vt.in_grid && vt.best.hit != 0u) shade_voxel_pixel(s, A, c, vt.best, vt.anchor_valid, vt.anchor_key, vt.anchor_chunk);
  else shade_far_pixel(s, A, c);
}

// PixHit: the fields of HitGeom + anchor the shading kernel needs (5 x uint4).
__device__ __forceinline__ void store_pixhit(uint4* dst, const HitGeom& g, const VoxTraceResult& vt) {
  dst[0] = make_uint4(__float_as_uint(g.t), __float_as_uint(g.n.x), __float_as_uint(g.n.y), __float_as_uint(g.n.z));
  dst[1] = make_uint4(__float_as_uint(g.root_bmin.x), __float_as_uint(g.root_bmin.y), __float_as_uint(g.root_bmin.z),
                      g.mat);
  dst[2] = make_uint4(g.node_base, g.macro_base, g.node, __float_as_uint(g.leaf_size));
  dst[3] = make_uint4(__float_as_uint(g.leaf_bmin.x), __float_as_uint(g.leaf_bmin.y), __float_as_uint(g.leaf_bmin.z),
                      vt.anchor_valid ? 1u : 0u);
  dst[4] = make_uint4(vt.anchor_key, (uint32_t)vt.anchor_chunk.x, (uint32_t)vt.anchor_chunk.y,
                      (uint32_t)vt.anchor_chunk.z);
}

__device__ __forceinline__ void enqueue(uint32_t* q, uint32_t* counter, bool mine, uint32_t value) {
  const uint32_t mask = __ballot_sync(0xFFFFFFFFu, mine);
  if (!mine) return;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t leader = __ffs(mask) - 1u;
  uint32_t base = 0u;
  if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
  base = __shfl_sync(mask, base, leader);
  q[base + __popc(mask & ((1u << lane) - 1u))] = value;
}

__device__ __forceinline__ uint32_t warp_uniform_end(uint32_t n) { return (n + 31u) & ~31u; }

// Walk summary of a pixel that met probes (px_probe.x): probes met (24 bits),
// candidate index of the voxel answer, its trace phase, whether the trace
// began with the hint window, voxel-hit bit.
__device__ __forceinline__ uint32_t probe_summary(uint32_t met, uint32_t best_cand, uint32_t phase, bool hinted,
                                                  bool vox) {
  return min(met, 0xFFFFFFu) | ((best_cand & 31u) << 24) | ((phase & 1u) << 29) | (hinted ? 0x40000000u : 0u) |
         (vox ? 0x80000000u : 0u);
}

// Order of probe hits: trace phase (hint window first), t, candidate index,
// probe order, column order.  t >= 0, so its bits order like its value.
__device__ __forceinline__ unsigned long long slab_key(uint32_t phase, float t, uint32_t cand, uint32_t seq,
                                                      uint32_t it) {
  return ((unsigned long long)(phase & 1u) << 62) | ((unsigned long long)__float_as_uint(t) << 31) |
         ((unsigned long long)(cand & 31u) << 26) | ((unsigned long long)(seq & 0xFFFFFu) << 6) |
         (unsigned long long)(it & 63u);
}

// The end of a pixel's walk in record mode: the voxel answer's PixHit, and
// for pixels that met probes the walk summary (the rest is final).
__device__ __forceinline__ void walk_finish(const FrameArgs& A, uint32_t pix, const VoxTraceResult& vt,
                                            const ProbeHook& ph, uint32_t tile_count, bool* vox, bool* pend) {
  *vox = vt.in_grid && vt.best.hit != 0u;
  if (*vox) store_pixhit(A.pix_hit + (size_t)pix * 5u, vt.best, vt);
  const uint32_t gs = *vox ? vt.gov_state : 0u;
  *pend = ph.seq != 0u || gs != 0u;
  if (*pend) {
    A.px_gov[pix] = make_uint4(gs, __float_as_uint(vt.gov_t0), __float_as_uint(vt.gov_t1), vt.gov_slot);
    // more probes than the summary counts: every stored one is still used,
    // the pixel just walks again
    const uint32_t stored = ph.seq > 0xFFFFFFu ? 0u : ph.recorded;
    A.px_probe[pix] = make_uint2(probe_summary(ph.seq, ph.best_cand, ph.phase, ph.first_phase == 0u, *vox), stored);
  } else {
    profile_voxel(A, ph.first_phase, ph.phase, tile_count);  // the walk is the reference's (no probe met)
  }
}

__device__ __forceinline__ ProbeHook probe_hook_record(const FrameArgs& A, uint32_t pix) {
  ProbeHook ph = probe_hook_inline();
  ph.mode = PROBE_RECORD;
  ph.pixel = pix;
  ph.recs = A.probe_recs;
  ph.rec_count = &A.q_count[4];
  ph.rec_cap = A.probe_cap;
  ph.defer_gov = A.px_gov != nullptr;
  return ph;
}

// Voxel walk with the grass column probes stored, not evaluated (both trace
// phases: the hint window, then the full trace when the window held no voxel
// hit).  Pixels that met no probe are final here; the rest wait for
// k_probe_dda, k_slab_eval, k_slab_pick and k_primary_resolve.  (Running the
// full-trace phase as a second launch over a compacted queue of the pixels
// that need it was measured slower: 2.49 vs 2.32 ms per 1080p frame.)
__device__ __forceinline__ void k_primary_trace_body(const FrameArgs& A) {
  // a block beyond this view's tiles (a launch over views of different sizes)
  if (blockIdx.x * 2u >= (A.iw + 7u) / 8u || blockIdx.y >= (A.ih + 7u) / 8u) return;
  __shared__ uint32_t cslot[2][TILE_CANDS];
  __shared__ Meta cmeta[2][TILE_CANDS];
  __shared__ uint32_t ccount[2];
  const Scene s = make_scene(A, false);
  stage_tiles(s, A, cslot, cmeta, ccount);
  uint32_t t, gx, gy;
  const bool active = block_pixel(A, &t, &gx, &gy);
  bool vox = false, pend = false, full = false;
  uint32_t pix = 0u;
  if (active) {
    const PrimaryCtx c = primary_ctx(s, gx, gy, A.iw);
    pix = (uint32_t)c.pix;
    ProbeHook ph = probe_hook_record(A, pix);
    const VoxTraceResult vt = primary_trace<PROBE_RECORD>(s, A, c, cslot[t], cmeta[t], ccount[t], ph);
    walk_finish(A, pix, vt, ph, ccount[t], &vox, &pend);
    full = ph.first_phase <= 1u && ph.phase == 1u;
  }
  enqueue(A.q_vox, &A.q_count[0], active && vox && !pend, pix);
  enqueue(A.q_far, &A.q_count[1], active && !vox && !pend, pix);
  enqueue(A.q_pending, &A.q_count[5], active && pend, pix);
  const uint32_t nfull = __popc(__ballot_sync(0xFFFFFFFFu, full));  // frame statistics
  if ((threadIdx.x & 31u) == 0u && nfull != 0u) atomicAdd(&A.q_count[10], nfull);
}
__global__ void __launch_bounds__(PRIMARY_THREADS) k_primary_trace(const __grid_constant__ FrameArgs A) { k_primary_trace_body(A); }
__global__ void __launch_bounds__(PRIMARY_THREADS) k_primary_trace_views(const __grid_constant__ FrameArgsViews V) {
  k_primary_trace_body(V.v[blockIdx.z]);
}

// One lane per stored probe: the probe's column DDA with the walk's
// arguments, storing one task per grass slab it would march.  A probe whose
// tasks do not all fit sends its pixel to the inline walk (stored count 0).
__device__ __forceinline__ void k_probe_dda_body(const FrameArgs& A) {
  const Scene s = make_scene(A, false);
  const uint32_t n = min(A.q_count[4], A.probe_cap);
  const float vs = vs_(s);
  for (uint32_t i = blockIdx.x * SHADE_THREADS + threadIdx.x; i < n; i += gridDim.x * SHADE_THREADS) {
    const ProbeRec r = A.probe_recs[i];
    const PrimaryCtx c = primary_ctx(s, r.pixel % A.iw, r.pixel / A.iw, A.iw);
    const Meta ch = meta_at(s, r.slot);
    const v3 rb = V3((float)ch.ox, (float)ch.oy, (float)ch.oz) * vs;
    const i3 ov{ch.ox, ch.oy, ch.oz};
    bool lost = probe_seq(r) == PROBE_SEQ_LOST;
    grass_columns_dda(s, c.ro, c.rd, safe_inv3(c.rd), r.t0, r.t1, rb, ov, vs, ch.colinfo_base,
                      [&](uint32_t it, float t, float tNext, v3 id) {
                        // the part of the column step inside the cell's grass
                        // slab (try_grass_slab_hit's first step): an empty one
                        // is no task
                        const v2 iv = grass_slab_interval(c.ro, c.rd, t, tNext, id * vs, vs);
                        if (iv.y <= iv.x) return false;
                        const uint32_t j = atomicAdd(&A.q_count[6], 1u);
                        if (j < A.slab_cap) {
                          A.slab_tasks[j] = slab_task(i, it, iv.x, iv.y, id, ch);
                        } else {
                          lost = true;
                        }
                        return false;
                      });
    if (lost) atomicMin(&A.px_probe[r.pixel].y, 0u);
  }
}
__global__ void __launch_bounds__(SHADE_THREADS) k_probe_dda(const __grid_constant__ FrameArgs A) { k_probe_dda_body(A); }
__global__ void __launch_bounds__(SHADE_THREADS) k_probe_dda_views(const __grid_constant__ FrameArgsViews V) {
  k_probe_dda_body(V.v[blockIdx.z]);
}

// One lane per grass slab: try_grass_slab_hit (the blade march).  A hit
// lowers its pixel's nearest-hit key and marks its chunk.
__device__ __forceinline__ void k_slab_eval_body(const FrameArgs& A) {
  const Scene s = make_scene(A, false);
  const uint32_t n = min(A.q_count[6], A.slab_cap);
  const float vs = vs_(s);
  const float time_s = s.cam->voxel_params[1], strength = s.cam->voxel_params[2];
  for (uint32_t j = blockIdx.x * SHADE_THREADS + threadIdx.x; j < n; j += gridDim.x * SHADE_THREADS) {
    const uint4 a = A.slab_tasks[j];
    const ProbeRec r = A.probe_recs[a.x];
    const PrimaryCtx c = primary_ctx(s, r.pixel % A.iw, r.pixel / A.iw, A.iw);
    const v3 id = slab_task_cell(a, meta_at(s, r.slot));
    const float t0 = __uint_as_float(a.z);  // the slab interval (non-empty)
    const GrassHit gh = grass_layer_trace_lod(s, c.ro, c.rd, t0, __uint_as_float(a.w), id * vs, id, time_s, strength,
                                              grass_lod_from_t(t0));
    if (gh.hit) {
      if (__float_as_uint(gh.t) & 0x80000000u) {  // not ordered by the key: walk again
        atomicMin(&A.px_probe[r.pixel].y, 0u);
        continue;
      }
      const uint32_t cand = probe_cand(r), phase = probe_phase(r);
      A.slab_res[j] = make_float4(gh.t, gh.n.x, gh.n.y, gh.n.z);
      atomicMin(&A.px_first[r.pixel], slab_key(phase, gh.t, cand, probe_seq(r), slab_task_step(a)));
      atomicOr(phase ? &A.px_mask[r.pixel].y : &A.px_mask[r.pixel].x, 1u << (cand & 31u));
      A.slab_hits[atomicAdd(&A.q_count[7], 1u)] = j;
    }
  }
}
__global__ void __launch_bounds__(SHADE_THREADS, SLAB_MIN_BLOCKS) k_slab_eval(const __grid_constant__ FrameArgs A) { k_slab_eval_body(A); }
__global__ void __launch_bounds__(SHADE_THREADS, SLAB_MIN_BLOCKS) k_slab_eval_views(const __grid_constant__ FrameArgsViews V) {
  k_slab_eval_body(V.v[blockIdx.z]);
}

// True when hit `key` cannot stand for its chunk: an earlier probe of the
// same chunk and trace phase also hit.  Successive probe intervals meet at a
// leaf exit only up to rounding (t_leave + eps - eps), so in that rare case a
// later probe's hit may be nearer than the chunk's first one, which is the
// one the reference keeps.
__device__ __forceinline__ bool slab_hit_shadows_first(unsigned long long first, unsigned long long key) {
  const unsigned long long chunk_mask = (1ull << 62) | (31ull << 26);  // phase, candidate
  const unsigned long long seq_mask = 0xFFFFFull << 6;
  return first != ~0ull && (key & chunk_mask) == (first & chunk_mask) && (key & seq_mask) < (first & seq_mask);
}

// Finds, per pixel, the slab task whose key is the pixel's nearest; pixels
// where that hit is not its chunk's first are sent to the inline walk.
__device__ __forceinline__ void k_slab_pick_body(const FrameArgs& A) {
  const uint32_t n = min(A.q_count[7], A.slab_cap);
  for (uint32_t i = blockIdx.x * SHADE_THREADS + threadIdx.x; i < n; i += gridDim.x * SHADE_THREADS) {
    const uint32_t j = A.slab_hits[i];
    const uint4 a = A.slab_tasks[j];
    const ProbeRec r = A.probe_recs[a.x];
    const unsigned long long key =
        slab_key(probe_phase(r), A.slab_res[j].x, probe_cand(r), probe_seq(r), slab_task_step(a));
    const unsigned long long first = A.px_first[r.pixel];
    if (key == first) A.px_task[r.pixel] = j;
    else if (slab_hit_shadows_first(first, key)) atomicMin(&A.px_probe[r.pixel].y, 0u);
  }
}
__global__ void __launch_bounds__(SHADE_THREADS) k_slab_pick(const __grid_constant__ FrameArgs A) { k_slab_pick_body(A); }
__global__ void __launch_bounds__(SHADE_THREADS) k_slab_pick_views(const __grid_constant__ FrameArgsViews V) {
  k_slab_pick_body(V.v[blockIdx.z]);
}

// The blade marches the walk deferred (grass_on_voxel_hit of a grass-voxel
// answer, px_gov state 1), one lane per pending pixel: a hit replaces the
// answer's t and n in its PixHit record (state 3), a miss keeps the voxel
// hit (state 4).
__device__ __forceinline__ void k_gov_eval_body(const FrameArgs& A) {
  if (A.px_gov == nullptr) return;
  const Scene s = make_scene(A, false);
  const uint32_t n = A.q_count[5];
  for (uint32_t i = blockIdx.x * SHADE_THREADS + threadIdx.x; i < n; i += gridDim.x * SHADE_THREADS) {
    const uint32_t pix = A.q_pending[i];
    const uint4 gv = A.px_gov[pix];
    if (gv.x != 1u) continue;
    uint4* rec = A.pix_hit + (size_t)pix * 5u;
    const uint4 h0 = rec[0];
    const PrimaryCtx c = primary_ctx(s, pix % A.iw, pix / A.iw, A.iw);
    const GrassHit gh = grass_on_voxel_hit(s, c.ro, c.rd, meta_at(s, gv.w), __uint_as_float(h0.x),
                                           V3(__uint_as_float(h0.y), __uint_as_float(h0.z), __uint_as_float(h0.w)),
                                           __uint_as_float(gv.y), __uint_as_float(gv.z));
    if (gh.hit)
      rec[0] = make_uint4(__float_as_uint(gh.t), __float_as_uint(gh.n.x), __float_as_uint(gh.n.y),
                          __float_as_uint(gh.n.z));
    A.px_gov[pix].x = gh.hit ? 3u : 4u;
  }
}
__global__ void __launch_bounds__(SHADE_THREADS, SLAB_MIN_BLOCKS) k_gov_eval(const __grid_constant__ FrameArgs A) {
  k_gov_eval_body(A);
}
__global__ void __launch_bounds__(SHADE_THREADS, SLAB_MIN_BLOCKS) k_gov_eval_views(const __grid_constant__ FrameArgsViews V) {
  k_gov_eval_body(V.v[blockIdx.z]);
}

// Pixels that met probes: the nearer of the nearest probe hit and the voxel
// answer (see the comment above ProbeRec), or, when that cannot be decided
// from the parts, the reference walk with inline probes.
__device__ __forceinline__ void k_primary_resolve_body(const FrameArgs& A) {
  const Scene s = make_scene(A, false);
  const uint32_t n = A.q_count[5], end = warp_uniform_end(n);
  const uint32_t tiles_x = (A.iw + 7u) / 8u;
  const float vs = vs_(s);
  for (uint32_t i = blockIdx.x * SHADE_THREADS + threadIdx.x; i < end; i += gridDim.x * SHADE_THREADS) {
    bool active = i < n, vox = false;
    uint32_t pix = 0u;
    if (active) {
      pix = A.q_pending[i];
      const uint2 pp = A.px_probe[pix];
      const uint32_t met = pp.x & 0xFFFFFFu;
      uint32_t vcand = (pp.x >> 24) & 31u, vphase = (pp.x >> 29) & 1u;
      uint32_t first_phase = (pp.x & 0x40000000u) != 0u ? 0u : 1u;
      vox = (pp.x >> 31) != 0u;
      if (A.px_gov != nullptr && A.px_gov[pix].x == 2u) {
        // A deferred blade march left the voxel answer open: the walk again
        // with its blade marches inline (probes only counted; their hits are
        // the first walk's) gives the voxel answer, with the same probes
        // before it.
        const uint32_t gx = pix % A.iw, gy = pix / A.iw;
        const size_t tile = (size_t)(gy >> 3) * tiles_x + (gx >> 3);
        const PrimaryCtx c = primary_ctx(s, gx, gy, A.iw);
        ProbeHook ph = probe_hook_inline();
        ph.mode = PROBE_RECORD;  // recs stay null: probes are counted, not stored
        ph.pixel = pix;
        const VoxTraceResult vt = primary_trace<PROBE_RECORD>(s, A, c, A.tile_slots + tile * TILE_CANDS, nullptr,
                                                              A.tile_count[tile], ph);
        vox = vt.in_grid && vt.best.hit != 0u;
        if (vox) store_pixhit(A.pix_hit + (size_t)pix * 5u, vt.best, vt);
        vcand = ph.best_cand & 31u;  // as probe_summary keeps it
        vphase = ph.phase & 1u;
        first_phase = ph.first_phase;
      }
      uint32_t answer_phase = vphase;  // phase of the answer (1 when there is none)
      const unsigned long long first = A.px_first[pix];
      bool walk = pp.y < met;  // some probes were not evaluated
      if (!walk && first != ~0ull) {
        const uint32_t j = A.px_task[pix];
        const float4 res = A.slab_res[j];
        const ProbeRec r = A.probe_recs[A.slab_tasks[j].x];
        const uint32_t pcand = probe_cand(r), pphase = probe_phase(r);
        bool probe_wins = true;
        if (vox && pphase == vphase) {
          const float vt = __uint_as_float(A.pix_hit[(size_t)pix * 5u].x);
          probe_wins = res.x < vt || (res.x == vt && pcand <= vcand);
        }
        if (probe_wins) {
          answer_phase = pphase;
          const Meta ch = meta_at(s, r.slot);
          const v3 rb = V3((float)ch.ox, (float)ch.oy, (float)ch.oz) * vs;
          const float rs = (float)s.cam->chunk_size * vs;
          const int32_t csz = (int32_t)s.cam->chunk_size;
          const HitGeom g = make_hit(MAT_GRASS, res.x, V3(res.y, res.z, res.w), rb, rs, ch, r.node,
                                     V3(r.leaf_bmin[0], r.leaf_bmin[1], r.leaf_bmin[2]), r.leaf_size);
          const VoxTraceResult vr{true, g, 0.0f, probe_anchor_valid(r), r.anchor_key,
                                  i3{ch.ox / csz, ch.oy / csz, ch.oz / csz}};
          store_pixhit(A.pix_hit + (size_t)pix * 5u, g, vr);
          vox = true;
        } else {
          // the voxel answer's own chunk had a probe hit: undecided here
          const uint2 pm = A.px_mask[pix];
          walk = (((vphase ? pm.y : pm.x) >> vcand) & 1u) != 0u;
        }
      }
      const uint32_t gx = pix % A.iw, gy = pix / A.iw;
      const size_t tile = (size_t)(gy >> 3) * tiles_x + (gx >> 3);
      if (walk) {
        atomicAdd(&A.q_count[9], 1u);
        const PrimaryCtx c = primary_ctx(s, gx, gy, A.iw);
        ProbeHook ph = probe_hook_inline();
        const VoxTraceResult vt = primary_trace<PROBE_INLINE>(s, A, c, A.tile_slots + tile * TILE_CANDS, nullptr,
                                                A.tile_count[tile], ph);
        vox = vt.in_grid && vt.best.hit != 0u;
        if (vox) store_pixhit(A.pix_hit + (size_t)pix * 5u, vt.best, vt);
        profile_voxel(A, ph.first_phase, ph.phase, A.tile_count[tile]);
      } else {
        profile_voxel(A, first_phase, vox ? answer_phase : 1u, A.tile_count[tile]);
      }
    }
    enqueue(A.q_vox, &A.q_count[0], active && vox, pix);
    enqueue(A.q_far, &A.q_count[1], active && !vox, pix);
  }
}
__global__ void __launch_bounds__(SHADE_THREADS) k_primary_resolve(const __grid_constant__ FrameArgs A) { k_primary_resolve_body(A); }
__global__ void __launch_bounds__(SHADE_THREADS) k_primary_resolve_views(const __grid_constant__ FrameArgsViews V) {
  k_primary_resolve_body(V.v[blockIdx.z]);
}

__device__ __forceinline__ HitGeom load_pixhit(const Scene& s, const uint4* src) {
  const uint4 a = src[0], b = src[1], d = src[2], e = src[3];
  HitGeom g = miss_hitgeom();
  g.hit = 1u;
  g.t = __uint_as_float(a.x);
  g.n = V3(__uint_as_float(a.y), __uint_as_float(a.z), __uint_as_float(a.w));
  g.root_bmin = V3(__uint_as_float(b.x), __uint_as_float(b.y), __uint_as_float(b.z));
  g.mat = b.w;
  g.root_size = (float)s.cam->chunk_size * vs_(s);
  g.node_base = d.x;
  g.macro_base = d.y;
  g.node = d.z;
  g.leaf_size = __uint_as_float(d.w);
  g.leaf_bmin = V3(__uint_as_float(e.x), __uint_as_float(e.y), __uint_as_float(e.z));
  return g;
}

// Voxel-hit shading, wavefront schedule: prep (grass refine + classify) ->
// fresh shadows | light gathers -> final.  Each kernel walks its queue with
// a grid-stride loop whose trip count is uniform per warp (queues are read on
// the device), so the warp-wide enqueue and shuffles see every lane.

__device__ __forceinline__ void k_shade_prep_body(const FrameArgs& A) {
  const Scene s = make_scene(A, false);
  const uint32_t n = A.q_count[0], end = warp_uniform_end(n);
  for (uint32_t i = blockIdx.x * SHADE_THREADS + threadIdx.x; i < end; i += gridDim.x * SHADE_THREADS) {
    bool fresh = false, light = false;
    uint32_t pix = 0u;
    if (i < n) {
      pix = A.q_vox[i];
      const PrimaryCtx c = primary_ctx(s, pix % A.iw, pix / A.iw, A.iw);
      uint4* src = A.pix_hit + (size_t)pix * 5u;
      HitGeom g = load_pixhit(s, src);
      if (g.mat == MAT_GRASS) {
        if (grass_refine(s, c, g)) profile_add(A, PROFILE_GRASS, 1u);
        src[0] = make_uint4(__float_as_uint(g.t), __float_as_uint(g.n.x), __float_as_uint(g.n.y),
                            __float_as_uint(g.n.z));
      }
      A.depth[pix] = fmin_(g.t, FOG_MAX_DIST);  // final: godray may start before k_shade_vox
      fresh = shadow_fresh(c);
      light = lights_wanted(g);
      if (light && !lights_possible(s, (c.ro + c.rd * g.t) + g.n * (0.75f * vs_(s)))) {
        // no LIGHT voxel within the gather's reach: its exact result, +0
        const v3 r = light_finish(V3s(0.0f));
        A.px_light[pix] = make_float4(r.x, r.y, r.z, 0.0f);
        light = false;
      }
    }
    enqueue(A.q_shadow, &A.q_count[2], fresh, pix);
    enqueue(A.q_light, &A.q_count[3], light, pix);
  }
}
__global__ void __launch_bounds__(SHADE_THREADS, SHADE_MIN_BLOCKS) k_shade_prep(const __grid_constant__ FrameArgs A) { k_shade_prep_body(A); }
__global__ void __launch_bounds__(SHADE_THREADS, SHADE_MIN_BLOCKS) k_shade_prep_views(const __grid_constant__ FrameArgsViews V) {
  k_shade_prep_body(V.v[blockIdx.z]);
}

__device__ __forceinline__ void k_shade_shadow_body(const FrameArgs& A) {
  const Scene s = make_scene(A, false);
  const uint32_t n = A.q_count[2];
  for (uint32_t i = blockIdx.x * SHADE_THREADS + threadIdx.x; i < n; i += gridDim.x * SHADE_THREADS) {
    const uint32_t pix = A.q_shadow[i];
    const PrimaryCtx c = primary_ctx(s, pix % A.iw, pix / A.iw, A.iw);
    const HitGeom g = load_pixhit(s, A.pix_hit + (size_t)pix * 5u);
    A.px_shadow[pix] = sun_transmittance_geom_only(s, shadow_origin(s, c, g), SUN_DIR);
  }
}
__global__ void __launch_bounds__(SHADE_THREADS) k_shade_shadow(const __grid_constant__ FrameArgs A) { k_shade_shadow_body(A); }
__global__ void __launch_bounds__(SHADE_THREADS) k_shade_shadow_views(const __grid_constant__ FrameArgsViews V) {
  k_shade_shadow_body(V.v[blockIdx.z]);
}

// Eight lanes per pixel, one light ray each; the group's first lane adds the
// eight results in ray order (the reference loop's order and early stop).
__device__ __forceinline__ void k_shade_lights_body(const FrameArgs& A) {
  const Scene s = make_scene(A, false);
  const uint32_t lane = threadIdx.x & 31u, ray = lane & 7u, group0 = lane & ~7u;
  const uint32_t n = A.q_count[3], groups = n * 8u, end = warp_uniform_end(groups);
  for (uint32_t i = blockIdx.x * SHADE_THREADS + threadIdx.x; i < end; i += gridDim.x * SHADE_THREADS) {
    const bool active = i < groups;
    uint32_t pix = 0u;
    v3 hp = V3s(0.0f), nrm = V3(0.0f, 1.0f, 0.0f);
    v4 hit = v4{0.0f, 0.0f, 0.0f, 0.0f};
    if (active) {
      pix = A.q_light[i >> 3];
      const PrimaryCtx c = primary_ctx(s, pix % A.iw, pix / A.iw, A.iw);
      const HitGeom g = load_pixhit(s, A.pix_hit + (size_t)pix * 5u);
      hp = c.ro + c.rd * g.t;
      nrm = g.n;
      const LightFrame F = light_frame(s, hp, nrm, g.root_bmin);
      hit = dda_hit_light(s, F.p0, light_ray_dir(F, nrm, ray), LIGHT_MAX_DIST_VOX, vs_(s));
    }
    v4 h[LIGHT_RAYS];
    for (uint32_t k = 0; k < LIGHT_RAYS; ++k) {
      h[k].x = __shfl_sync(0xFFFFFFFFu, hit.x, group0 + k);
      h[k].y = __shfl_sync(0xFFFFFFFFu, hit.y, group0 + k);
      h[k].z = __shfl_sync(0xFFFFFFFFu, hit.z, group0 + k);
      h[k].w = __shfl_sync(0xFFFFFFFFu, hit.w, group0 + k);
    }
    if (active && ray == 0u) {
      uint32_t hits = 0u;
      v3 sum = V3s(0.0f);
      for (uint32_t k = 0; k < LIGHT_RAYS; ++k)
        if (light_accum(s, hp, nrm, h[k], hits, sum)) break;
      const v3 r = light_finish(sum);
      A.px_light[pix] = make_float4(r.x, r.y, r.z, 0.0f);
    }
  }
}
__global__ void __launch_bounds__(SHADE_THREADS) k_shade_lights(const __grid_constant__ FrameArgs A) { k_shade_lights_body(A); }
__global__ void __launch_bounds__(SHADE_THREADS) k_shade_lights_views(const __grid_constant__ FrameArgsViews V) {
  k_shade_lights_body(V.v[blockIdx.z]);
}

__device__ __forceinline__ void k_shade_vox_body(const FrameArgs& A) {
  const Scene s = make_scene(A, false);
  const uint32_t n = A.q_count[0];
  for (uint32_t i = blockIdx.x * SHADE_THREADS + threadIdx.x; i < n; i += gridDim.x * SHADE_THREADS) {
    const uint32_t pix = A.q_vox[i];
    const PrimaryCtx c = primary_ctx(s, pix % A.iw, pix / A.iw, A.iw);
    const uint4* src = A.pix_hit + (size_t)pix * 5u;
    const HitGeom g = load_pixhit(s, src);  // t and n as refined by k_shade_prep
    const uint4 e = src[3], f = src[4];
    const float shadow_out = shadow_fresh(c) ? shadow_blend(s, A, c, c.ro + c.rd * g.t, A.px_shadow[pix])
                                             : clampf(A.shadow_in[c.pix], 0.0f, 1.0f);
    v3 light = V3s(0.0f);
    if (lights_wanted(g)) {
      const float4 l = A.px_light[pix];
      light = V3(l.x, l.y, l.z);
    }
    shade_voxel_final(s, A, c, g, shadow_out, light, e.w != 0u, f.x, i3{(int32_t)f.y, (int32_t)f.z, (int32_t)f.w},
                      true);
  }
}
__global__ void __launch_bounds__(SHADE_THREADS, SHADE_MIN_BLOCKS) k_shade_vox(const __grid_constant__ FrameArgs A) { k_shade_vox_body(A); }
__global__ void __launch_bounds__(SHADE_THREADS, SHADE_MIN_BLOCKS) k_shade_vox_views(const __grid_constant__ FrameArgsViews V) {
  k_shade_vox_body(V.v[blockIdx.z]);
}

// PART 0: the far pixels the walk queued (q_count[8], copied right after the
// walk), shaded while the grass probes resolve; PART 1: those the resolve
// queued after them; PART 2: the whole queue.
template <int PART>
__device__ __forceinline__ void k_shade_far_body(const FrameArgs& A) {
  const Scene s = make_scene(A, false);
  const uint32_t first = PART == 1 ? A.q_count[8] : 0u;
  const uint32_t n = PART == 0 ? A.q_count[8] : A.q_count[1];
  for (uint32_t i = first + blockIdx.x * SHADE_THREADS + threadIdx.x; i < n; i += gridDim.x * SHADE_THREADS) {
    const uint32_t pix = A.q_far[i];
    const PrimaryCtx c = primary_ctx(s, pix % A.iw, pix / A.iw, A.iw);
    shade_far_pixel(s, A, c);
  }
}
template <int PART>
__global__ void __launch_bounds__(SHADE_THREADS, SHADE_MIN_BLOCKS) k_shade_far(const __grid_constant__ FrameArgs A) { k_shade_far_body<PART>(A); }
template <int PART>
__global__ void __launch_bounds__(SHADE_THREADS, SHADE_MIN_BLOCKS) k_shade_far_views(const __grid_constant__ FrameArgsViews V) {
  k_shade_far_body<PART>(V.v[blockIdx.z]);
}

// ---------------------------------------------------------------------------
// Godray pass
// ---------------------------------------------------------------------------
constexpr int POST_THREADS_X = 32, POST_THREADS_Y = 4;

// The godray ray of pixel (gx, gy) with depth t_c (main_godray,
// ray_main.wgsl:520-535): the jittered direction and march length.
struct GodrayPixel {
  v3 ro, rd;
  float t_end, j4, j_phase;
  bool fog_ok;
};
__device__ __forceinline__ GodrayPixel godray_pixel(const Scene& s, uint32_t gx, uint32_t gy, float t_c) {
  GodrayPixel g;
  g.ro = cam_pos(s);
  const v2 qpx = V2((float)gx, (float)gy);
  const float fi = (float)(s.cam->frame_index & 1023u);
  const v2 fj = V2(fi, fi * 1.371f);
  g.j4 = 0.20f * (hash12(qpx * J0_SCALE + fj) - 0.5f);
  g.j_phase = hash12(qpx * 0.91f + fj * 0.73f + V2(31.7f, 12.3f)) - 0.5f;
  const float qstep = 0.03f;
  const float dq = (hash12(qpx * 1.37f + fj * 1.19f + V2(9.2f, 1.1f)) - 0.5f) * qstep;
  const v2 j_rd = V2(hash12(qpx + fj + V2(1.7f, 9.2f)) - 0.5f, hash12(qpx + fj * 1.13f + V2(8.3f, 2.1f)) - 0.5f);
  g.t_end = fmin_(floorf((t_c + dq) / qstep) * qstep, GODRAY_MAX_DIST);
  g.fog_ok = fog_density_godray(s) > 0.0f;
  const v2 pxc = V2((float)gx + 0.5f, (float)gy + 0.5f) + j_rd * 0.35f;
  g.rd = ray_dir_from_pixel(s, pxc);
  return g;
}
// Its in-scatter.
__device__ __forceinline__ v3 godray_pixel_integral(const Scene& s, const GodrayPixel& g) {
  if (g.fog_ok && g.t_end > 0.0f) return godray_integrate_1(s, g.ro, g.rd, g.t_end, g.j4, g.j_phase);
  return V3s(0.0f);
}

__device__ __forceinline__ void k_godray_body(const FrameArgs& A) {
  const uint32_t gx = blockIdx.x * POST_THREADS_X + threadIdx.x;
  const uint32_t gy = blockIdx.y * POST_THREADS_Y + threadIdx.y;
  if (gx >= A.iw || gy >= A.ih) return;
  const Scene s = make_scene(A, true);
  const uint32_t W = A.iw, H = A.ih;
  const int32_t Wi = (int32_t)W, Hi = (int32_t)H;
  const v3 ro = cam_pos(s);
  const int32_t x = (int32_t)gx, y = (int32_t)gy;
  const float* D = A.depth;
  const float t_c = D[(size_t)y * W + x];
  const float t_l = D[(size_t)y * W + clampi(x - 1, 0, Wi - 1)], t_r = D[(size_t)y * W + clampi(x + 1, 0, Wi - 1)];
  const float t_u = D[(size_t)clampi(y - 1, 0, Hi - 1) * W + x], t_d = D[(size_t)clampi(y + 1, 0, Hi - 1) * W + x];
  const float dmin = fmin_(t_c, fmin_(fmin_(t_l, t_r), fmin_(t_u, t_d)));
  const float dmax = fmax_(t_c, fmax_(fmax_(t_l, t_r), fmax_(t_u, t_d)));
  const float span = (dmax - dmin) / fmax_(dmin, 1e-3f);
  const float stable = 1.0f - smooth(0.06f, 0.30f, span);
  const float t_hist = dmin;
  const GodrayPixel g = godray_pixel(s, gx, gy, t_c);
  const float4 pre = A.god_pre ? A.god_pre[(size_t)gy * W + gx] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  // made beside the probe passes for a far pixel of the walk
  const v3 cur = pre.w != 0.0f ? V3(pre.x, pre.y, pre.z) : godray_pixel_integral(s, g);
  const v3 p_ws = ro + g.rd * t_hist;
  const v2 uvp = prev_uv_from_world(s, p_ws);
  v3 hl = cur;
  float hv = 0.0f;
  const v2 hdf = V2((float)W, (float)H);
  const v2 uvc = V2((float)gx + 0.5f, (float)gy + 0.5f) / hdf;
  if (in_unit_square(uvp)) {
    const float4 h = A.god_in[(size_t)nearest_idx(uvp.y, H) * W + (uint32_t)nearest_idx(uvp.x, W)];
    const float hd = h.w;
    hl = godray_decompress(xyz(h));
    const float rel = fabsf(hd - t_hist) / fmax_(t_hist, 1e-3f);
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
  A.god_out[(size_t)gy * W + gx] = make_float4(oc.x, oc.y, oc.z, t_hist);
}

// The godray integrals of the walk's far pixels (queue entries [0,
// q_count[8]) of q_far), whose depths k_shade_far<0> has made final: run on
// the side stream beside the probe passes, read by k_godray.
__device__ __forceinline__ void k_godray_far_body(const FrameArgs& A) {
  if (A.god_pre == nullptr) return;
  const Scene s = make_scene(A, true);
  const uint32_t n = A.q_count[8];
  for (uint32_t i = blockIdx.x * SHADE_THREADS + threadIdx.x; i < n; i += gridDim.x * SHADE_THREADS) {
    const uint32_t pix = A.q_far[i];
    const v3 cur = godray_pixel_integral(s, godray_pixel(s, pix % A.iw, pix / A.iw, A.depth[pix]));
    A.god_pre[pix] = make_float4(cur.x, cur.y, cur.z, 1.0f);
  }
}
__global__ void __launch_bounds__(SHADE_THREADS) k_godray_far(const __grid_constant__ FrameArgs A) { k_godray_far_body(A); }
__global__ void __launch_bounds__(SHADE_THREADS) k_godray_far_views(const __grid_constant__ FrameArgsViews V) {
  k_godray_far_body(V.v[blockIdx.z]);
}
__global__ void __launch_bounds__(POST_THREADS_X* POST_THREADS_Y) k_godray(const __grid_constant__ FrameArgs A) { k_godray_body(A); }
__global__ void __launch_bounds__(POST_THREADS_X* POST_THREADS_Y) k_godray_views(const __grid_constant__ FrameArgsViews V) {
  k_godray_body(V.v[blockIdx.z]);
}

// ---------------------------------------------------------------------------
// Composite pass (+ fused composite TAA)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void k_composite_body(const FrameArgs& A) {
  const uint32_t gx = blockIdx.x * POST_THREADS_X + threadIdx.x;
  const uint32_t gy = blockIdx.y * POST_THREADS_Y + threadIdx.y;
  if (gx >= A.pw || gy >= A.ph) return;
  const Scene s = make_scene(A, false);
  const uint32_t RW = A.iw, RH = A.ih, PW = A.pw, PH = A.ph;
  const v2 pp = V2((float)gx + 0.5f, (float)gy + 0.5f);
  const v2 rdim = V2((float)s.cam->render_present_px[0], (float)s.cam->render_present_px[1]);
  const v2 pdim = V2((float)s.cam->render_present_px[2], (float)s.cam->render_present_px[3]);
  const v2 px_render = (pp / pdim) * rdim;
  const int32_t ipr_x = clampi(to_i32(floorf(px_render.x)), 0, to_i32(rdim.x) - 1);
  const int32_t ipr_y = clampi(to_i32(floorf(px_render.y)), 0, to_i32(rdim.y) - 1);
  const int32_t rwi = (int32_t)RW, rhi = (int32_t)RH;
  const v2 rdf = V2((float)RW, (float)RH);
  const int32_t irx = clampi(ipr_x, 0, rwi - 1), iry = clampi(ipr_y, 0, rhi - 1);
  auto C4 = [&](int32_t xx, int32_t yy) { return A.color[(size_t)yy * RW + (uint32_t)xx]; };
  auto DEP = [&](int32_t xx, int32_t yy) { return A.depth[(size_t)yy * RW + (uint32_t)xx]; };
  const v3 base = xyz(C4(irx, iry));
  const v2 fdf = rdf;
  const v2 px_full = px_render * (fdf / rdf);
  const int32_t ifx = clampi(to_i32(floorf(px_full.x)), 0, rwi - 1);
  const int32_t ify = clampi(to_i32(floorf(px_full.y)), 0, rhi - 1);
  const v2 uv_full = (px_full + V2(0.5f, 0.5f)) / fdf;
  const float d0 = DEP(ifx, ify);
  const v2 gdf = V2((float)RW, (float)RH);
  const v2 du = V2(1.0f / gdf.x, 0.0f), dv = V2(0.0f, 1.0f / gdf.y);
  auto G = [&](v2 uv) {
    const float4 c = A.god_out[(size_t)nearest_idx(uv.y, RH) * RW + (uint32_t)nearest_idx(uv.x, RW)];
    return godray_decompress(xyz(c));
  };
  const v3 gC = G(uv_full), gE = G(uv_full + du), gW = G(uv_full - du), gN = G(uv_full + dv), gS = G(uv_full - dv);
  const float dE = DEP(min(ifx + 1, rwi - 1), ify), dW = DEP(max(ifx - 1, 0), ify);
  const float dN = DEP(ifx, min(ify + 1, rhi - 1)), dS = DEP(ifx, max(ify - 1, 0));
  const float tol = 0.02f + 0.06f * smooth(10.0f, 80.0f, d0);
  const float wE = 1.0f - smooth(0.0f, tol, fabsf(dE - d0));
  const float wW = 1.0f - smooth(0.0f, tol, fabsf(dW - d0));
  const float wN = 1.0f - smooth(0.0f, tol, fabsf(dN - d0));
  const float wS = 1.0f - smooth(0.0f, tol, fabsf(dS - d0));
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
    const v3 hx1 = vmax(xyz(C4(clampi(irx + 2, 0, rwi - 1), iry)), V3s(0.0f));
    const v3 hx0 = vmax(xyz(C4(clampi(irx - 2, 0, rwi - 1), iry)), V3s(0.0f));
    const v3 hy1 = vmax(xyz(C4(irx, clampi(iry + 2, 0, rhi - 1))), V3s(0.0f));
    const v3 hy0 = vmax(xyz(C4(irx, clampi(iry - 2, 0, rhi - 1))), V3s(0.0f));
    const v3 bloom = (b0 + bright_extract_hue(hx1, bt) + bright_extract_hue(hx0, bt) + bright_extract_hue(hy1, bt) +
                      bright_extract_hue(hy0, bt)) /
                     5.0f;
    const v3 bmx = vmax(hdr, V3s(0.0f)) * 0.35f;
    hdr = hdr + vmin(bloom, bmx) * bk;
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
  const v2 uv_r = px_render * V2(1.0f / (float)RW, 1.0f / (float)RH);
  const float4 lh = A.local_hist_out[(size_t)nearest_idx(uv_r.y, RH) * RW + (uint32_t)nearest_idx(uv_r.x, RW)];
  const v3 fin = ldr + xyz(lh);
  const size_t opix = (size_t)gy * PW + gx;
  if (A.pre_taa) A.pre_taa[opix] = make_float4(fin.x, fin.y, fin.z, 1.0f);
  v3 taa = fin;
  if (s.cam->frame_index > 1u) {
    const float dd = DEP(ipr_x, ipr_y);
    const v3 rdv = ray_dir_from_pixel(s, px_render);
    const v3 p_ws = cam_pos(s) + rdv * dd;
    const v2 uvp = prev_uv_from_world(s, p_ws);
    if (in_unit_square(uvp)) {
      const float4 h = A.out_hist_in[(size_t)nearest_idx(uvp.y, PH) * PW + (uint32_t)nearest_idx(uvp.x, PW)];
      taa = vmix(xyz(h), taa, COMPOSITE_TAA_ALPHA);
    }
  }
  const float4 o = make_float4(taa.x, taa.y, taa.z, 1.0f);
  A.output[opix] = o;
  A.out_hist_out[opix] = o;
}
__global__ void __launch_bounds__(POST_THREADS_X* POST_THREADS_Y) k_composite(const __grid_constant__ FrameArgs A) { k_composite_body(A); }
__global__ void __launch_bounds__(POST_THREADS_X* POST_THREADS_Y) k_composite_views(const __grid_constant__ FrameArgsViews V) {
  k_composite_body(V.v[blockIdx.z]);
}

// ---------------------------------------------------------------------------
// Ray queries
// ---------------------------------------------------------------------------
struct QueryArgs {
  vxe_camera_gpu cam;  // only chunk_size, chunk_count, voxel_params, grid fields are read
  vxe_clipmap_gpu clip;
  const uint4* nodes;
  uint64_t nodes_n;
  const uint32_t* ropes;
  uint64_t ropes_n;
  const uint4* metas;
  uint64_t metas_n;
  const uint32_t* grid;
  uint64_t grid_n;
  const uint32_t* macro;
  uint64_t macro_n;
  const uint32_t* colinfo;
  uint64_t colinfo_n;
  uint32_t* err;
  const float* origins;
  const float* dirs;
  uint32_t n;
  float tmax;
  uint4* out;  // 2 x uint4 per ray
};

__device__ __forceinline__ Scene make_query_scene(const QueryArgs& Q) {
  Scene s;
  s.cam = &Q.cam;
  s.clip = &Q.clip;
  s.nodes = Q.nodes;
  s.nodes_n = Q.nodes_n;
  s.ropes = Q.ropes;
  s.ropes_n = Q.ropes_n;
  s.metas = Q.metas;
  s.metas_n = Q.metas_n;
  s.grid = Q.grid;
  s.grid_n = Q.grid_n;
  s.macro = Q.macro;
  s.macro_n = Q.macro_n;
  s.colinfo = Q.colinfo;
  s.colinfo_n = Q.colinfo_n;
  s.clip_tex = nullptr;
  s.clip_layers = 0;
  s.clip_res = 0;
  s.err = Q.err;
  s.grass_rec = nullptr;
  s.grass_rec_n = 0;
  s.grass_state = nullptr;
  s.grass_frames = nullptr;
  s.slot_lights = nullptr;
  s.slot_top = nullptr;
  s.grass_taper = nullptr;
  return s;
}

// One ray: chunk DDA front to back, first hit wins (cells are disjoint in t).
__device__ __forceinline__ HitRec trace_query_ray(const Scene& s, v3 ro, v3 rd, float tmax) {
  const v3 inv = safe_inv3(rd);
  HitGeom best = miss_hitgeom();
  const float vs = vs_(s);
  const float rs = (float)s.cam->chunk_size * vs;
  const TraceOpts opt{true};
  chunk_grid_dda(s, ro, rd, 0.0f, tmax, [&](uint32_t slot, float) -> bool {
    const Meta ch = meta_at(s, slot);
    if (ch.macro_empty != 0u) return false;
    const v3 rb = V3((float)ch.ox, (float)ch.oy, (float)ch.oz) * vs;
    const v2 rt = intersect_aabb(ro, rd, rb, rb + V3s(rs));
    const float ce = fmax_(rt.x, 0.0f), cx = fmin_(rt.y, fmin_(tmax, FOG_MAX_DIST));
    if (cx < ce) return false;
    ProbeHook ph = probe_hook_inline();
    const ChunkTraceResult h =
        trace_chunk_interval_stream_macro<PROBE_INLINE>(s, ro, rd, inv, ch, ce, cx, false, INVALID, opt, ph);
    if (h.hit.hit != 0u) {
      best = h.hit;
      return true;
    }
    return false;
  });
  if (best.hit) return make_rec(best, ro, rd, vs, true);
  return miss_rec();
}

constexpr int QUERY_THREADS = 128;

__global__ void __launch_bounds__(QUERY_THREADS) k_query(const __grid_constant__ QueryArgs Q) {
  const uint32_t i = blockIdx.x * QUERY_THREADS + threadIdx.x;
  if (i >= Q.n) return;
  const Scene s = make_query_scene(Q);
  const v3 ro = V3(Q.origins[3 * i], Q.origins[3 * i + 1], Q.origins[3 * i + 2]);
  const v3 rd = V3(Q.dirs[3 * i], Q.dirs[3 * i + 1], Q.dirs[3 * i + 2]);
  store_rec(Q.out + (size_t)i * 2u, trace_query_ray(s, ro, rd, Q.tmax));
}

}  // namespace dev
}  // namespace vxe
