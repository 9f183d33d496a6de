// batch_kernels.cuh -- many uneven requests traced by one persistent kernel.
//
// A batch mixes viewport requests (primary hit records of a cold frame, the
// records vxe_render_frame writes on its first frame after vxe_resize) and
// ray-query batches (voxel geometry only, as vxe_trace_rays).  Work is cut
// into items:
//   viewport  a rect of (tile_w * rays_per_thread) x tile_h pixels,
//   query     128 * rays_per_thread rays,
// numbered in request order.  Every warp of a grid sized to fill the GPU pops
// items from one atomic counter until the batch is drained, so small and large
// requests share the machine with no per-request launch and no tail between
// requests.  Logical 8x8 candidate tiles stay per viewport pixel (x/8, y/8),
// independent of the item shape, so results do not depend on the tuning.
// The batch sizes live in a device-side header: one captured CUDA graph
// serves every batch that fits the allocated capacities.
#pragma once

#include "frame_kernels.cuh"

namespace vxe {
namespace dev {

struct BatchReq {  // 80 B
  uint32_t kind;        // 0 viewport, 1 query
  uint32_t w, h;        // viewport size; w = ray count for queries
  uint32_t tiles_x;     // viewport: logical 8x8 tiles per row
  uint32_t tile_base;   // viewport: first tile in the batch tile arrays
  uint32_t item_begin;  // first work item of this request
  uint32_t items_x;     // viewport: items per row
  uint32_t cam;         // index into the camera array
  const float* o;       // query origins (3 floats per ray)
  const float* d;       // query directions
  uint4* out;           // 2 x uint4 per record
  float tmax;
  uint32_t ray_base;    // first ray in the batch's viewport ray numbering (queries: the next viewport's)
  uint32_t q_base;      // first ray in the batch's query ray numbering (viewports: the next query's)
  uint32_t _pad[3];
};

struct BatchHeader {
  uint32_t n_reqs, total_tiles, n_items, tile_w, tile_h, rpt, tile_reqs, vp_rays;
  // coherent queries: items >= vp_items take query rays in sorted order
  uint32_t vp_items, q_rays, nbins, sorted;
};

struct BatchArgs {
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
  const BatchHeader* hdr;
  const BatchReq* reqs;
  const vxe_camera_gpu* cams;
  uint32_t* tile_count;
  uint32_t* tile_slots;
  uint32_t* head;       // [0] item counter, [1] tile counter
  uint32_t req_first;   // plain mode: the one request a launch serves
  uint32_t plain;       // 1: item = blockIdx-derived, no queue
  // grass cell table, valid for cameras with this wind time / strength
  const float4* grass_rec;
  uint64_t grass_rec_n;
  const float* grass_taper;
  uint32_t* grass_state;
  float4* grass_frames;
  uint32_t grass_time_bits, grass_strength_bits;
  // deferred grass probes of viewport rays (persistent and graph modes), the
  // frame's scheme over the batch's viewport ray numbering (BatchReq::ray_base)
  uint32_t defer;
  ProbeRec* probe_recs;
  uint32_t probe_cap;
  uint4* slab_tasks;
  float4* slab_res;
  uint32_t* slab_hits;
  uint32_t slab_cap;
  uint32_t ray_cap;               // per-ray arrays' capacity
  unsigned long long* px_first;
  uint32_t* px_task;
  uint2* px_mask;
  uint2* px_probe;
  uint4* px_hit;                  // 4 x uint4 per ray: voxel answer of a ray that met probes or needs refining
  uint32_t* q_pending;
  uint32_t* q_refine;             // rays whose answer is a grass voxel (grass-slab refinement)
  uint32_t* q_far;                // rays without a voxel answer (heightfield)
  uint32_t* dcount;               // [0] probes, [1] pending rays, [2] slab tasks, [3] slab hits, [4] refine, [5] far
  // coherent queries: query rays binned by (origin chunk, direction octant)
  uint32_t* q_keys;               // bin of each query ray
  uint32_t* q_perm;               // query rays in bin order
  uint32_t* bin_count;            // per bin: rays, then (after the scan) the next free position
};

constexpr int BATCH_THREADS = 128;
constexpr int MAX_BATCH_REQS = 1024;

__device__ __forceinline__ Scene batch_scene(const BatchArgs& B, const vxe_camera_gpu* cam) {
  Scene s;
  s.cam = cam;
  s.clip = &B.clip;
  s.nodes = B.nodes;
  s.nodes_n = B.nodes_n;
  s.ropes = B.ropes;
  s.ropes_n = B.ropes_n;
  s.metas = B.metas;
  s.metas_n = B.metas_n;
  s.grid = B.grid;
  s.grid_n = B.grid_n;
  s.macro = B.macro;
  s.macro_n = B.macro_n;
  s.colinfo = B.colinfo;
  s.colinfo_n = B.colinfo_n;
  s.clip_tex = B.clip_tex;
  s.clip_layers = B.clip_layers;
  s.clip_res = B.clip_res;
  s.err = B.err;
  const bool table = B.grass_rec != nullptr && __float_as_uint(cam->voxel_params[1]) == B.grass_time_bits &&
                     __float_as_uint(cam->voxel_params[2]) == B.grass_strength_bits;
  s.grass_rec = table ? B.grass_rec : nullptr;
  s.grass_rec_n = table ? B.grass_rec_n : 0;
  s.grass_taper = table ? B.grass_taper : nullptr;
  s.grass_state = table ? B.grass_state : nullptr;
  s.grass_frames = table ? B.grass_frames : nullptr;
  s.slot_lights = nullptr;
  s.slot_top = nullptr;
  return s;
}

// Last request whose first element (item or tile, via `key`) is <= x.
template <class K>
__device__ __forceinline__ uint32_t find_req(const BatchReq* reqs, uint32_t n, uint32_t x, K key) {
  uint32_t lo = 0, hi = n;  // invariant: key(reqs[lo]) <= x
  while (hi - lo > 1u) {
    const uint32_t mid = (lo + hi) >> 1;
    if (key(reqs[mid]) <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Voxel trace of one cold viewport pixel (no history hint); PM the probe mode.
template <uint32_t PM>
__device__ __noinline__ VoxTraceResult viewport_trace(const Scene& s, const uint32_t* tile_count,
                                                      const uint32_t* tile_slots, uint32_t tiles_x, uint32_t gx,
                                                      uint32_t gy, ProbeHook& ph) {
  const v3 ro = cam_pos(s);
  const v3 rd = ray_dir_from_pixel(s, V2((float)gx + 0.5f, (float)gy + 0.5f));
  const size_t tile = (size_t)(gy >> 3) * tiles_x + (gx >> 3);
  const uint32_t cnt = tile_count[tile];
  VoxTraceResult vt{false, miss_hitgeom(), 0.0f, false, INVALID, i3{0, 0, 0}};
  ph.best_cand = INVALID;
  if (s.cam->chunk_count != 0u && cnt != 0u)
    vt = trace_candidates<PM>(s, tile_slots + tile * TILE_CANDS, nullptr, ro, rd, 0.0f, FOG_MAX_DIST, false,
                          i3{0, 0, 0}, INVALID, cnt, ph);
  return vt;
}

// Record of voxel hit `best` (grass voxels get main_primary's grass-slab
// refinement first).
__device__ __noinline__ HitRec viewport_voxel_rec(const Scene& s, uint32_t gx, uint32_t gy, HitGeom best) {
  const float vs = vs_(s);
  const v3 ro = cam_pos(s);
  const v3 rd = ray_dir_from_pixel(s, V2((float)gx + 0.5f, (float)gy + 0.5f));
  if (best.mat == MAT_GRASS) {
    const i3 ov{to_i32(floorf(best.root_bmin.x / vs + 0.5f)), to_i32(floorf(best.root_bmin.y / vs + 0.5f)),
                to_i32(floorf(best.root_bmin.z / vs + 0.5f))};
    const v3 hp = ro + rd * best.t;
    const GrassCell cell =
        pick_grass_cell_in_chunk_with_bias(hp, rd, best.root_bmin, ov, vs, (int32_t)s.cam->chunk_size);
    const GrassHit gh = try_grass_slab_hit(s, ro, rd, 0.0f, best.t, cell.bmin_m, cell.id_vox, vs,
                                           s.cam->voxel_params[1], s.cam->voxel_params[2]);
    if (gh.hit) { best.t = gh.t; best.n = gh.n; }
  }
  return make_rec(best, ro, rd, vs, true);
}

// Record of a ray without a voxel hit: the heightfield (main_primary's
// fallback, with its grass refinement) or a miss.
__device__ __noinline__ HitRec viewport_far_rec(const Scene& s, uint32_t gx, uint32_t gy) {
  const float vs = vs_(s);
  const v3 ro = cam_pos(s);
  const v3 rd = ray_dir_from_pixel(s, V2((float)gx + 0.5f, (float)gy + 0.5f));
  if (s.cam->chunk_count == 0u) return miss_rec();  // no chunks: sky (ray_main.wgsl:219-231)
  ClipHit hf = clip_trace_heightfield(s, ro, rd, 0.0f, FOG_MAX_DIST);
  if (!hf.hit) return miss_rec();
  if (hf.mat == MAT_GRASS) {
    const v3 hp = ro + rd * hf.t;
    const GrassCell cell = grass_cell_from_world_global(hp, rd, vs);
    const v3 gb = V3(cell.bmin_m.x, hp.y - vs, cell.bmin_m.z);
    const GrassHit gh = try_grass_slab_hit(s, ro, rd, 0.0f, hf.t, gb, cell.id_vox, vs, s.cam->voxel_params[1],
                                           s.cam->voxel_params[2]);
    if (gh.hit) { hf.t = gh.t; hf.n = gh.n; }
  }
  HitGeom g = miss_hitgeom();
  g.hit = 1u;
  g.t = hf.t;
  g.n = hf.n;
  g.mat = hf.mat;
  return make_rec(g, ro, rd, vs, false);
}

__device__ __forceinline__ HitRec viewport_finish(const Scene& s, uint32_t gx, uint32_t gy, bool voxel,
                                                  const HitGeom& best) {
  return voxel ? viewport_voxel_rec(s, gx, gy, best) : viewport_far_rec(s, gx, gy);
}

// Cold-frame primary hit record of one viewport pixel: voxel trace without a
// history hint, then main_primary's grass refinement or heightfield fallback.
__device__ __forceinline__ HitRec viewport_pixel_hit(const Scene& s, const uint32_t* tile_count,
                                                     const uint32_t* tile_slots, uint32_t tiles_x, uint32_t gx,
                                                     uint32_t gy, ProbeHook& ph) {
  const VoxTraceResult vt = viewport_trace<PROBE_INLINE>(s, tile_count, tile_slots, tiles_x, gx, gy, ph);
  return viewport_finish(s, gx, gy, vt.in_grid && vt.best.hit != 0u, vt.best);
}

// Persistent candidate-tile builder over every viewport tile of the batch.
__global__ void __launch_bounds__(TILE_THREADS) k_batch_tiles(const __grid_constant__ BatchArgs B) {
  __shared__ uint32_t sl[MAX_TILE_CHUNKS][TILE_THREADS];
  __shared__ float en[MAX_TILE_CHUNKS][TILE_THREADS];
  const BatchHeader H = *B.hdr;
  const uint32_t lane = threadIdx.x;
  const uint32_t first = B.plain ? B.req_first : 0u;
  const uint32_t nreq = B.plain ? 1u : H.tile_reqs;
  const uint32_t total = B.plain ? B.reqs[first].tiles_x * ((B.reqs[first].h + 7u) / 8u) : H.total_tiles;
  for (uint32_t t = blockIdx.x * TILE_THREADS + lane; t < total; t += gridDim.x * TILE_THREADS) {
    const uint32_t gt = B.plain ? B.reqs[first].tile_base + t : t;
    const uint32_t r = B.plain ? first : find_req(B.reqs, nreq, gt, [](const BatchReq& q) { return q.tile_base; });
    const BatchReq q = B.reqs[r];
    const Scene s = batch_scene(B, &B.cams[q.cam]);
    const uint32_t local = gt - q.tile_base;
    build_tile_list(s, local % q.tiles_x, local / q.tiles_x, lane, sl, en, &B.tile_count[gt],
                    &B.tile_slots[(size_t)gt * TILE_CANDS]);
  }
}

__device__ __forceinline__ void store_rec_at(uint4* out, size_t i, const HitRec& h) { store_rec(out + i * 2u, h); }

// Appends `value` to queue q; the lanes that arrive together share one atomic.
__device__ __forceinline__ void enqueue_active(uint32_t* q, uint32_t* counter, uint32_t value) {
  const uint32_t mask = __activemask();
  const uint32_t lane = threadIdx.x & 31u, leader = __ffs(mask) - 1u;
  uint32_t base = 0u;
  if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
  base = __shfl_sync(mask, base, leader);
  q[base + (uint32_t)__popc(mask & ((1u << lane) - 1u))] = value;
}

__device__ __forceinline__ void store_hitgeom(uint4* dst, const HitGeom& g) {
  dst[0] = make_uint4(__float_as_uint(g.t), __float_as_uint(g.n.x), __float_as_uint(g.n.y), __float_as_uint(g.n.z));
  dst[1] = make_uint4(__float_as_uint(g.root_bmin.x), __float_as_uint(g.root_bmin.y), __float_as_uint(g.root_bmin.z),
                      g.mat);
  dst[2] = make_uint4(g.node_base, g.macro_base, g.node, __float_as_uint(g.leaf_size));
  dst[3] = make_uint4(__float_as_uint(g.leaf_bmin.x), __float_as_uint(g.leaf_bmin.y), __float_as_uint(g.leaf_bmin.z),
                      0u);
}

// Finishes a decided viewport ray (deferred mode): a non-grass voxel hit is
// written at once, a grass voxel hit waits for k_batch_refine, a ray without
// a voxel hit for k_batch_far.
__device__ __forceinline__ void batch_finish(const BatchArgs& B, const Scene& s, const BatchReq& q, uint32_t ray,
                                             uint32_t gx, uint32_t gy, bool vox, const HitGeom& best) {
  if (vox && best.mat != MAT_GRASS) {
    store_rec_at(q.out, (size_t)gy * q.w + gx, viewport_voxel_rec(s, gx, gy, best));
  } else if (vox) {
    store_hitgeom(B.px_hit + (size_t)ray * 4u, best);
    enqueue_active(B.q_refine, &B.dcount[4], ray);
  } else {
    enqueue_active(B.q_far, &B.dcount[5], ray);
  }
}

// Processes one work item with the calling warp; DEFER: viewport rays record
// their grass probes for the deferred passes (else they probe inline).
template <bool DEFER>
__device__ __forceinline__ void batch_item(const BatchArgs& B, const BatchHeader& H, const BatchReq& q,
                                           const Scene& s, uint32_t local, uint32_t lane) {
  if (q.kind == 0u) {
    const uint32_t rw = H.tile_w * H.rpt, rh = H.tile_h;
    const uint32_t x0 = (local % q.items_x) * rw, y0 = (local / q.items_x) * rh;
    for (uint32_t k = lane; k < rw * rh; k += 32u) {
      const uint32_t gx = x0 + k % rw, gy = y0 + k / rw;
      if (gx >= q.w || gy >= q.h) continue;
      ProbeHook ph = probe_hook_inline();
      const uint32_t ray = q.ray_base + gy * q.w + gx;
      if (DEFER) {
        ph.mode = PROBE_RECORD;
        ph.pixel = ray;
        ph.recs = B.probe_recs;
        ph.rec_count = &B.dcount[0];
        ph.rec_cap = B.probe_cap;
      }
      const VoxTraceResult vt = viewport_trace<DEFER ? PROBE_RECORD : PROBE_INLINE>(s, B.tile_count + q.tile_base,
                                               B.tile_slots + (size_t)q.tile_base * TILE_CANDS, q.tiles_x, gx, gy, ph);
      const bool vox = vt.in_grid && vt.best.hit != 0u;
      if (!DEFER) {
        store_rec_at(q.out, (size_t)gy * q.w + gx, viewport_finish(s, gx, gy, vox, vt.best));
      } else if (ph.seq != 0u) {  // met probes: k_batch_resolve decides
        if (vox) store_hitgeom(B.px_hit + (size_t)ray * 4u, vt.best);
        const uint32_t stored = ph.seq > 0xFFFFFFu ? 0u : ph.recorded;
        B.px_probe[ray] = make_uint2(probe_summary(ph.seq, ph.best_cand, ph.phase, ph.first_phase == 0u, vox), stored);
        enqueue_active(B.q_pending, &B.dcount[1], ray);
      } else {
        batch_finish(B, s, q, ray, gx, gy, vox, vt.best);
      }
    }
  } else {
    const uint32_t per = 128u * H.rpt;
    const uint32_t r0 = local * per;
    for (uint32_t k = lane; k < per; k += 32u) {
      const uint32_t i = r0 + k;
      if (i >= q.w) break;
      const v3 ro = V3(q.o[3 * (size_t)i], q.o[3 * (size_t)i + 1], q.o[3 * (size_t)i + 2]);
      const v3 rd = V3(q.d[3 * (size_t)i], q.d[3 * (size_t)i + 1], q.d[3 * (size_t)i + 2]);
      store_rec_at(q.out, i, trace_query_ray(s, ro, rd, q.tmax));
    }
  }
}

// Query rays in bin order (coherent mode): item k takes sorted positions
// [k * 128 * rpt, ...); each lane finds its ray's request by the query base.
__device__ __forceinline__ void batch_sorted_queries(const BatchArgs& B, const BatchHeader& H, uint32_t k,
                                                     uint32_t lane) {
  const uint32_t per = 128u * H.rpt;
  for (uint32_t j = lane; j < per; j += 32u) {
    const uint32_t pos = k * per + j;
    if (pos >= H.q_rays) break;
    const uint32_t ray = B.q_perm[pos];
    const uint32_t r = find_req(B.reqs, H.n_reqs, ray, [](const BatchReq& q) { return q.q_base; });
    const BatchReq& q = B.reqs[r];
    const uint32_t i = ray - q.q_base;
    const Scene s = batch_scene(B, &B.cams[0]);
    const v3 ro = V3(q.o[3 * (size_t)i], q.o[3 * (size_t)i + 1], q.o[3 * (size_t)i + 2]);
    const v3 rd = V3(q.d[3 * (size_t)i], q.d[3 * (size_t)i + 1], q.d[3 * (size_t)i + 2]);
    store_rec_at(q.out, i, trace_query_ray(s, ro, rd, q.tmax));
  }
}

// The persistent work-queue kernel (plain = 0) or one request per launch
// with one warp per item (plain = 1, the per-request baseline).
// DEFER must equal B.defer (one instantiation per probe mode).
template <bool DEFER>
__global__ void __launch_bounds__(BATCH_THREADS) k_batch_trace(const __grid_constant__ BatchArgs B) {
  __shared__ vxe_camera_gpu wcam[BATCH_THREADS / 32];
  __shared__ uint32_t wcam_id[BATCH_THREADS / 32];
  const BatchHeader H = *B.hdr;
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  if (lane == 0) wcam_id[warp] = 0xFFFFFFFFu;
  __syncwarp();
  auto load_cam = [&](uint32_t cam) {
    if (wcam_id[warp] != cam) {
      const uint32_t* src = reinterpret_cast<const uint32_t*>(&B.cams[cam]);
      uint32_t* dst = reinterpret_cast<uint32_t*>(&wcam[warp]);
      for (uint32_t k = lane; k < sizeof(vxe_camera_gpu) / 4u; k += 32u) dst[k] = src[k];
      __syncwarp();
      if (lane == 0) wcam_id[warp] = cam;
      __syncwarp();
    }
  };
  if (B.plain) {
    const BatchReq q = B.reqs[B.req_first];
    const uint32_t local = blockIdx.x * (BATCH_THREADS / 32) + warp;
    const uint32_t n_local = (B.req_first + 1 < H.n_reqs ? B.reqs[B.req_first + 1].item_begin : H.n_items) - q.item_begin;
    if (local >= n_local) return;
    load_cam(q.cam);
    const Scene s = batch_scene(B, &wcam[warp]);
    batch_item<DEFER>(B, H, q, s, local, lane);
    return;
  }
  for (;;) {
    uint32_t item = 0;
    if (lane == 0) item = atomicAdd(&B.head[0], 1u);
    item = __shfl_sync(0xFFFFFFFFu, item, 0);
    if (item >= H.n_items) break;
    if (H.sorted && item >= H.vp_items) {
      batch_sorted_queries(B, H, item - H.vp_items, lane);
      continue;
    }
    const uint32_t r = find_req(B.reqs, H.n_reqs, item, [](const BatchReq& q) { return q.item_begin; });
    const BatchReq q = B.reqs[r];
    load_cam(q.cam);
    const Scene s = batch_scene(B, &wcam[warp]);
    batch_item<DEFER>(B, H, q, s, item - q.item_begin, lane);
  }
}

// ---------------------------------------------------------------------------
// Deferred grass probes of viewport rays: the frame's k_probe_dda /
// k_slab_eval / k_slab_pick / k_primary_resolve over the batch's viewport
// rays (one trace phase: cold rays have no hint window).
// ---------------------------------------------------------------------------
struct BatchRay {
  const BatchReq* q;
  uint32_t gx, gy;
};

__device__ __forceinline__ BatchRay batch_ray(const BatchArgs& B, uint32_t n_reqs, uint32_t ray) {
  // ray_base never decreases over the requests and a query repeats the next
  // viewport's base, so the last request whose base is <= ray is a viewport.
  const uint32_t r = find_req(B.reqs, n_reqs, ray, [](const BatchReq& q) { return q.ray_base; });
  const BatchReq* q = &B.reqs[r];
  const uint32_t local = ray - q->ray_base;
  return BatchRay{q, local % q->w, local / q->w};
}

__global__ void __launch_bounds__(BATCH_THREADS) k_batch_defer_clear(const __grid_constant__ BatchArgs B) {
  const uint32_t n = min(B.hdr->vp_rays, B.ray_cap);
  for (uint32_t i = blockIdx.x * BATCH_THREADS + threadIdx.x; i < n; i += gridDim.x * BATCH_THREADS) {
    B.px_first[i] = ~0ull;
    B.px_mask[i] = make_uint2(0u, 0u);
  }
}

__global__ void __launch_bounds__(BATCH_THREADS) k_batch_probe_dda(const __grid_constant__ BatchArgs B) {
  const uint32_t n_reqs = B.hdr->n_reqs;
  const uint32_t n = min(B.dcount[0], B.probe_cap);
  for (uint32_t i = blockIdx.x * BATCH_THREADS + threadIdx.x; i < n; i += gridDim.x * BATCH_THREADS) {
    const ProbeRec r = B.probe_recs[i];
    const BatchRay br = batch_ray(B, n_reqs, r.pixel);
    const Scene s = batch_scene(B, &B.cams[br.q->cam]);
    const float vs = vs_(s);
    const v3 ro = cam_pos(s);
    const v3 rd = ray_dir_from_pixel(s, V2((float)br.gx + 0.5f, (float)br.gy + 0.5f));
    const Meta ch = meta_at(s, r.slot);
    const v3 rb = V3((float)ch.ox, (float)ch.oy, (float)ch.oz) * vs;
    const i3 ov{ch.ox, ch.oy, ch.oz};
    bool lost = probe_seq(r) == PROBE_SEQ_LOST;
    grass_columns_dda(s, ro, rd, safe_inv3(rd), r.t0, r.t1, rb, ov, vs, ch.colinfo_base,
                      [&](uint32_t it, float t, float tNext, v3 id) {
                        // the part of the column step inside the cell's grass
                        // slab (try_grass_slab_hit's first step): an empty one
                        // is no task
                        const v2 iv = grass_slab_interval(ro, rd, t, tNext, id * vs, vs);
                        if (iv.y <= iv.x) return false;
                        const uint32_t j = atomicAdd(&B.dcount[2], 1u);
                        if (j < B.slab_cap) {
                          B.slab_tasks[j] = slab_task(i, it, iv.x, iv.y, id, ch);
                        } else {
                          lost = true;
                        }
                        return false;
                      });
    if (lost) atomicMin(&B.px_probe[r.pixel].y, 0u);
  }
}

__global__ void __launch_bounds__(BATCH_THREADS, SLAB_MIN_BLOCKS) k_batch_slab_eval(const __grid_constant__ BatchArgs B) {
  const uint32_t n_reqs = B.hdr->n_reqs;
  const uint32_t n = min(B.dcount[2], B.slab_cap);
  for (uint32_t j = blockIdx.x * BATCH_THREADS + threadIdx.x; j < n; j += gridDim.x * BATCH_THREADS) {
    const uint4 a = B.slab_tasks[j];
    const ProbeRec r = B.probe_recs[a.x];
    const BatchRay br = batch_ray(B, n_reqs, r.pixel);
    const Scene s = batch_scene(B, &B.cams[br.q->cam]);
    const float vs = vs_(s);
    const v3 ro = cam_pos(s);
    const v3 rd = ray_dir_from_pixel(s, V2((float)br.gx + 0.5f, (float)br.gy + 0.5f));
    const v3 id = slab_task_cell(a, meta_at(s, r.slot));
    const float t0 = __uint_as_float(a.z);  // the slab interval (non-empty)
    const GrassHit gh = grass_layer_trace_lod(s, ro, rd, t0, __uint_as_float(a.w), id * vs, id, s.cam->voxel_params[1],
                                              s.cam->voxel_params[2], grass_lod_from_t(t0));
    if (gh.hit) {
      if (__float_as_uint(gh.t) & 0x80000000u) {
        atomicMin(&B.px_probe[r.pixel].y, 0u);
        continue;
      }
      const uint32_t cand = probe_cand(r), phase = probe_phase(r);
      B.slab_res[j] = make_float4(gh.t, gh.n.x, gh.n.y, gh.n.z);
      atomicMin(&B.px_first[r.pixel], slab_key(phase, gh.t, cand, probe_seq(r), slab_task_step(a)));
      atomicOr(phase ? &B.px_mask[r.pixel].y : &B.px_mask[r.pixel].x, 1u << (cand & 31u));
      B.slab_hits[atomicAdd(&B.dcount[3], 1u)] = j;
    }
  }
}

__global__ void __launch_bounds__(BATCH_THREADS) k_batch_slab_pick(const __grid_constant__ BatchArgs B) {
  const uint32_t n = min(B.dcount[3], B.slab_cap);
  for (uint32_t i = blockIdx.x * BATCH_THREADS + threadIdx.x; i < n; i += gridDim.x * BATCH_THREADS) {
    const uint32_t j = B.slab_hits[i];
    const uint4 a = B.slab_tasks[j];
    const ProbeRec r = B.probe_recs[a.x];
    const unsigned long long key = slab_key(probe_phase(r), B.slab_res[j].x, probe_cand(r), probe_seq(r), slab_task_step(a));
    const unsigned long long first = B.px_first[r.pixel];
    if (key == first) B.px_task[r.pixel] = j;
    else if (slab_hit_shadows_first(first, key)) atomicMin(&B.px_probe[r.pixel].y, 0u);
  }
}

// Rays that met probes: the nearer of the nearest probe hit and the voxel
// answer, or the reference walk with inline probes when the parts cannot
// decide.
__global__ void __launch_bounds__(BATCH_THREADS) k_batch_resolve(const __grid_constant__ BatchArgs B) {
  const uint32_t n_reqs = B.hdr->n_reqs;
  const uint32_t n = B.dcount[1];
  for (uint32_t i = blockIdx.x * BATCH_THREADS + threadIdx.x; i < n; i += gridDim.x * BATCH_THREADS) {
    const uint32_t ray = B.q_pending[i];
    const uint2 pp = B.px_probe[ray];
    const unsigned long long first = B.px_first[ray];
    const uint32_t met = pp.x & 0xFFFFFFu, vcand = (pp.x >> 24) & 31u, vphase = (pp.x >> 29) & 1u;
    const bool vox = (pp.x >> 31) != 0u;
    const BatchRay br = batch_ray(B, n_reqs, ray);
    const BatchReq& q = *br.q;
    const Scene s = batch_scene(B, &B.cams[q.cam]);
    bool walk = pp.y < met;
    if (!walk && first != ~0ull) {
      const uint32_t j = B.px_task[ray];
      const float4 res = B.slab_res[j];
      const ProbeRec r = B.probe_recs[B.slab_tasks[j].x];
      const uint32_t pcand = probe_cand(r), pphase = probe_phase(r);
      bool probe_wins = true;
      if (vox && pphase == vphase) {
        const float vt = __uint_as_float(B.px_hit[(size_t)ray * 4u].x);
        probe_wins = res.x < vt || (res.x == vt && pcand <= vcand);
      }
      if (probe_wins) {
        const float vs = vs_(s);
        const Meta ch = meta_at(s, r.slot);
        const v3 rb = V3((float)ch.ox, (float)ch.oy, (float)ch.oz) * vs;
        const HitGeom g = make_hit(MAT_GRASS, res.x, V3(res.y, res.z, res.w), rb, (float)s.cam->chunk_size * vs, ch,
                                   r.node, V3(r.leaf_bmin[0], r.leaf_bmin[1], r.leaf_bmin[2]), r.leaf_size);
        batch_finish(B, s, q, ray, br.gx, br.gy, true, g);
        continue;
      }
      const uint2 pm = B.px_mask[ray];
      walk = (((vphase ? pm.y : pm.x) >> vcand) & 1u) != 0u;
    }
    if (walk) {
      ProbeHook ph = probe_hook_inline();
      const HitRec h = viewport_pixel_hit(s, B.tile_count + q.tile_base,
                                          B.tile_slots + (size_t)q.tile_base * TILE_CANDS, q.tiles_x, br.gx, br.gy, ph);
      store_rec_at(q.out, (size_t)br.gy * q.w + br.gx, h);
      continue;
    }
    // no probe hit, or the voxel answer is nearer: the walk's answer stands
    const HitGeom best = vox ? load_pixhit(s, B.px_hit + (size_t)ray * 4u) : miss_hitgeom();
    batch_finish(B, s, q, ray, br.gx, br.gy, vox, best);
  }
}

__global__ void __launch_bounds__(BATCH_THREADS) k_batch_refine(const __grid_constant__ BatchArgs B) {
  const uint32_t n_reqs = B.hdr->n_reqs;
  const uint32_t n = B.dcount[4];
  for (uint32_t i = blockIdx.x * BATCH_THREADS + threadIdx.x; i < n; i += gridDim.x * BATCH_THREADS) {
    const uint32_t ray = B.q_refine[i];
    const BatchRay br = batch_ray(B, n_reqs, ray);
    const Scene s = batch_scene(B, &B.cams[br.q->cam]);
    const HitGeom best = load_pixhit(s, B.px_hit + (size_t)ray * 4u);
    store_rec_at(br.q->out, (size_t)br.gy * br.q->w + br.gx, viewport_voxel_rec(s, br.gx, br.gy, best));
  }
}

__global__ void __launch_bounds__(BATCH_THREADS) k_batch_far(const __grid_constant__ BatchArgs B) {
  const uint32_t n_reqs = B.hdr->n_reqs;
  const uint32_t n = B.dcount[5];
  for (uint32_t i = blockIdx.x * BATCH_THREADS + threadIdx.x; i < n; i += gridDim.x * BATCH_THREADS) {
    const uint32_t ray = B.q_far[i];
    const BatchRay br = batch_ray(B, n_reqs, ray);
    const Scene s = batch_scene(B, &B.cams[br.q->cam]);
    store_rec_at(br.q->out, (size_t)br.gy * br.q->w + br.gx, viewport_far_rec(s, br.gx, br.gy));
  }
}

// ---------------------------------------------------------------------------
// Coherent queries: query rays are binned by origin chunk (world grid cell,
// clamped into the grid) and direction octant, and traced in bin order, so a
// warp's rays start in the same chunk heading the same way.  Each ray's
// record is its own; only the order of work changes.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t query_bin(const vxe_camera_gpu& cam, v3 o, v3 d) {
  const float cs = (float)cam.chunk_size * cam.voxel_params[0];
  const int32_t c[3] = {__float2int_rd(o.x / cs) - cam.grid_origin_chunk[0],
                        __float2int_rd(o.y / cs) - cam.grid_origin_chunk[1],
                        __float2int_rd(o.z / cs) - cam.grid_origin_chunk[2]};
  uint32_t idx[3];
  for (int k = 0; k < 3; ++k) idx[k] = (uint32_t)min(max(c[k], 0), (int32_t)max(cam.grid_dims[k], 1u) - 1);
  const uint32_t cell = (idx[2] * max(cam.grid_dims[1], 1u) + idx[1]) * max(cam.grid_dims[0], 1u) + idx[0];
  const uint32_t oct = (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
  return cell * 8u + oct;
}

__global__ void __launch_bounds__(BATCH_THREADS) k_qsort_count(const __grid_constant__ BatchArgs B) {
  const BatchHeader& H = *B.hdr;
  const uint32_t n = H.q_rays, n_reqs = H.n_reqs, nbins = H.nbins;
  for (uint32_t ray = blockIdx.x * BATCH_THREADS + threadIdx.x; ray < n; ray += gridDim.x * BATCH_THREADS) {
    const uint32_t r = find_req(B.reqs, n_reqs, ray, [](const BatchReq& q) { return q.q_base; });
    const BatchReq& q = B.reqs[r];
    const uint32_t i = ray - q.q_base;
    const v3 o = V3(q.o[3 * (size_t)i], q.o[3 * (size_t)i + 1], q.o[3 * (size_t)i + 2]);
    const v3 d = V3(q.d[3 * (size_t)i], q.d[3 * (size_t)i + 1], q.d[3 * (size_t)i + 2]);
    const uint32_t bin = min(query_bin(B.cams[0], o, d), nbins - 1u);
    B.q_keys[ray] = bin;
    atomicAdd(&B.bin_count[bin], 1u);
  }
}

// Exclusive scan of the bin counts in place (one block).
constexpr int QSCAN_THREADS = 1024;
__global__ void __launch_bounds__(QSCAN_THREADS) k_qsort_scan(const __grid_constant__ BatchArgs B) {
  __shared__ uint32_t part[QSCAN_THREADS];
  const uint32_t nbins = B.hdr->nbins;
  const uint32_t per = (nbins + QSCAN_THREADS - 1) / QSCAN_THREADS;
  const uint32_t b0 = threadIdx.x * per, b1 = min(b0 + per, nbins);
  uint32_t sum = 0u;
  for (uint32_t b = b0; b < b1; ++b) sum += B.bin_count[b];
  part[threadIdx.x] = sum;
  __syncthreads();
  for (uint32_t off = 1; off < QSCAN_THREADS; off <<= 1) {
    const uint32_t v = threadIdx.x >= off ? part[threadIdx.x - off] : 0u;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  uint32_t run = part[threadIdx.x] - sum;  // exclusive prefix of this thread's range
  for (uint32_t b = b0; b < b1; ++b) {
    const uint32_t c = B.bin_count[b];
    B.bin_count[b] = run;
    run += c;
  }
}

__global__ void __launch_bounds__(BATCH_THREADS) k_qsort_scatter(const __grid_constant__ BatchArgs B) {
  const uint32_t n = B.hdr->q_rays;
  for (uint32_t ray = blockIdx.x * BATCH_THREADS + threadIdx.x; ray < n; ray += gridDim.x * BATCH_THREADS)
    B.q_perm[atomicAdd(&B.bin_count[B.q_keys[ray]], 1u)] = ray;
}

}  // namespace dev
}  // namespace vxe
