// vxe_api.cu -- C ABI of the B200 passes (declared in include/vxe/vxe.h).
//
// A vxe_ctx owns every device resource of one renderer instance, like the
// reference `Renderer` (render/state/mod.rs:34-709):
//   arenas   nodes (16 B), ropes (32 B), ChunkMeta slots (48 B), macro words,
//            colinfo words, chunk grid, clipmap layers;
//   images   internal-size color / depth / histories, present-size output and
//            output history, per-tile candidate lists;
//   streams  a compute stream for the passes and an upload stream whose copies
//            are ordered before the next frame by an event.
// The ping-pong wiring mirrors Renderer::encode_compute (render/state/mod.rs:
// 329-446): the primary pass reads hist[ping] and writes hist[pong]; godray
// reads godray[ping] and writes godray[pong]; composite reads godray[pong] and
// local_hist[pong]; composite TAA reads out_hist[ping] and writes
// out_hist[pong]; then ping = pong.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "kernels/batch_kernels.cuh"
#include "common/terrain_noise.h"
#include "kernels/frame_kernels.cuh"
#include "kernels/build_kernels.cuh"
#include "vxe/vxe.h"

using vxe::dev::FrameArgs;
using vxe::dev::QueryArgs;

namespace {

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  bool pooled = false;  // from the context's stream-ordered pool
};

enum Img {
  IMG_COLOR, IMG_DEPTH, IMG_LOCAL, IMG_HIST0, IMG_HIST1, IMG_SHADOW0, IMG_SHADOW1, IMG_LHIST0, IMG_LHIST1,
  IMG_GOD0, IMG_GOD1, IMG_PRE_TAA, IMG_OUTPUT, IMG_OHIST0, IMG_OHIST1, IMG_HITS, IMG_TILE_COUNT, IMG_TILE_SLOTS,
  IMG_PIXHIT, IMG_QVOX, IMG_QFAR, IMG_QCOUNT, IMG_QSHADOW, IMG_QLIGHT, IMG_PXSHADOW, IMG_PXLIGHT,
  IMG_PROBE_RECS, IMG_SLAB_TASKS, IMG_SLAB_RES, IMG_SLAB_HITS, IMG_PXFIRST, IMG_PXPROBE, IMG_PXMASK, IMG_PXTASK,
  IMG_QPENDING, IMG_GODPRE, IMG_PXGOV,
  IMG_N
};

// The per-frame grass cell table, shared by the frame stream and the batch
// lanes.  Its contents depend on the chunk records and on the camera's wind
// time, wind strength, voxel size and chunk count (the tag).  A pass whose
// camera matches the tag reads it as is; otherwise its stream rebuilds it
// after every earlier reader on every stream has finished, so no pass sees a
// table change under it.  Chunk uploads refresh the records of the uploaded
// slots on the upload stream, with the same ordering as the chunk data.
constexpr int kGrassReaders = 1 + VXE_BATCH_LANES;  // compute stream, lanes

struct GrassTable {
  DevBuf rec, taper, state, frames, list, list_n;
  bool list_valid = false;  // the grass column list matches the world's data
  bool valid = false;
  uint32_t time_bits = 0, strength_bits = 0, vs_bits = 0, chunk_count = 0;
  vxe_camera_gpu cam{};  // camera of the last full build (for slot refreshes)
  cudaEvent_t built = nullptr;
  bool built_recorded = false;
  cudaEvent_t reader[kGrassReaders] = {};
  bool reader_used[kGrassReaders] = {};
};

// One frame pipeline's images, ping-pong state, timing events and captured
// graph: the context's own frame, and one per viewport session (vxe_view).
struct FrameState {
  DevBuf img[IMG_N];
  uint32_t iw = 0, ih = 0, pw = 0, ph = 0;
  int ping = 0;
  // frame events: start, grass table, tiles, trace, shading, godray, composite,
  // then the walk kernel's own start and end
  cudaEvent_t ev[9] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  bool timed = false, timed_trace = false;
  // the frame as a captured CUDA graph
  cudaGraph_t fgraph = nullptr;
  cudaGraphExec_t fgraph_exec = nullptr;
  std::vector<cudaGraphNode_t> fgraph_nodes;
  uint64_t fgraph_key[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  // set by launch_frame while an asynchronous read of the output image is in
  // flight: the composite (its writer) waits for it, the earlier passes do not
  cudaEvent_t composite_wait = nullptr;
  // set by launch_frame when the grass cell table is (re)built on the side
  // stream beside the walk: the first pass that reads the table (the blade
  // marches) waits for it, the walk and the probe DDAs do not
  cudaEvent_t table_wait = nullptr;
};

// A second stream a frame forks to (far-pixel shading beside the probe
// resolve and the voxel shading) and joins back before the godray pass.
struct SideStream {
  cudaStream_t s = nullptr;
  cudaEvent_t fork = nullptr, mid = nullptr, prep = nullptr, join = nullptr;
  cudaEvent_t pre = nullptr, table = nullptr;  // frame start -> side, grass table ready -> compute
};

struct BatchLane {
  cudaStream_t stream = nullptr;
  SideStream side;
  DevBuf hdr, reqs, cams, tile_count, tile_slots, head;
  // deferred grass probes of viewport rays: per-ray arrays for ray_cap rays,
  // probe records and slab tasks in proportion, counters
  DevBuf probe_recs, slab_tasks, slab_res, slab_hits, px_first, px_task, px_mask, px_probe, px_hit, q_pending,
      q_refine, q_far, dcount;
  uint32_t ray_cap = 0;
  // coherent queries: bin of each query ray, rays in bin order, bin counters
  DevBuf q_keys, q_perm, bin_count;
  uint32_t q_cap = 0;
  void* stage = nullptr;  // pinned: header | requests | cameras
  cudaGraphExec_t graph = nullptr;
  uint32_t graph_key[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  vxe_clipmap_gpu graph_clip{};  // clipmap uniform baked into the captured launches
  cudaEvent_t ev[2] = {nullptr, nullptr};
  bool busy = false;
  uint64_t rays = 0;
  uint32_t items = 0, tiles = 0;
  // per-frame working buffers (tile lists, queues, probe and slab records)
  // of the viewport sessions rendered on this lane, sized for the largest
  FrameState scratch;
  // one set per view of a multi-view launch (vxe_view_render_batch_async)
  FrameState mscratch[vxe::dev::kMaxViewsPerLaunch];
};

}  // namespace

struct vxe_ctx {
  vxe_config cfg{};
  uint32_t flags = 0;
  std::string err;
  int device = 0;
  cudaStream_t compute = nullptr, upload = nullptr;
  cudaEvent_t upload_done = nullptr;
  bool upload_pending = false;
  // arenas
  DevBuf nodes, ropes, metas, macro, colinfo, grid, clip_tex, errword;
  DevBuf slot_lights;  // per slot: holds a LIGHT leaf (k_slot_lights)
  DevBuf slot_top;     // per slot: top of its non-air leaves, voxels (k_slot_lights)
  DevBuf profile;      // profile_counts of the context's frames (5 words)
  // caps on the wavefront's stored grass probes and slab tasks (0: the buffers' sizes)
  uint32_t probe_limit = 0, slab_limit = 0;
  // chunk builder: per-chunk scratch (materials, ground minima, level-5 cell
  // states and child offsets, solid counts) and events around its two kernels
  // asynchronous image reads: a copy stream and one event per ticket slot;
  // out_pending / any_pending: the last output / other image copy not yet
  // waited for by a frame
  cudaStream_t copy = nullptr;
  cudaEvent_t copy_ev[8] = {};
  uint64_t copy_seq = 0;
  bool out_pending = false, any_pending = false;
  cudaEvent_t out_ev = nullptr, any_ev = nullptr;
  DevBuf build_scratch;
  DevBuf build_places;  // vxe_build_place records of a resident build
  DevBuf move_buf;      // vxe_slot_move records
  cudaEvent_t build_ev[3] = {};
  bool build_timed = false;
  GrassTable gt;
  FrameState fr;  // the context's own frame
  SideStream side;  // its fork stream
  vxe_camera_gpu cam{};
  vxe_clipmap_gpu clip{};
  // query scratch
  DevBuf q_in, q_out;
  // batches: independent lanes (stream, pinned staging, descriptors, tile
  // lists, queue heads, captured graph) so several batches can be in flight
  BatchLane lanes[VXE_BATCH_LANES];
  int b_trace_grid = 0, b_tile_grid = 0;
  int shade_wave = 148 * 16;  // blocks of the grid-stride shading kernels
  bool upload_recorded = false;
  // Stream-ordered pool for lane and view buffers: growing or freeing them
  // never waits for the device (cudaFree would wait for every stream).
  cudaMemPool_t pool = nullptr;
  cudaStream_t aux = nullptr;  // zero-fills new views' images
  // Pinned staging for world writes: blocks filled in turn; a block is
  // refilled only after the copies queued from it have run.
  struct StageBlock {
    char* p = nullptr;
    cudaEvent_t ev = nullptr;
    bool rec = false;
  };
  std::vector<StageBlock> ring;
  size_t ring_off = 0;
  size_t ring_cur = 0;
  // where the compute stream and each lane stood at the last world write
  cudaEvent_t rd_ev[1 + VXE_BATCH_LANES] = {};
};

struct vxe_view {
  FrameState fr;
  cudaStream_t last_stream = nullptr;  // stream of the view's last frame
  cudaEvent_t done = nullptr;          // orders frames that move between lanes
};

namespace {

vxe_status stage_block_add(vxe_ctx* c);

vxe_status fail(vxe_ctx* c, vxe_status st, const char* fmt, ...) {
  if (c) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    c->err = buf;
  }
  return st;
}

#define CK(call)                                                                              \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      return fail(c, e_ == cudaErrorMemoryAllocation ? VXE_ERR_OOM : VXE_ERR_DEVICE, "%s: %s", #call, \
                  cudaGetErrorString(e_));                                                    \
  } while (0)

// Fills device memory and waits for it.  A plain cudaMemset runs on the
// legacy default stream, which the context's non-blocking streams do not wait
// for: a pass launched right after could write the buffer first and then see
// its results overwritten.
cudaError_t fill_sync(void* p, int value, size_t bytes) {
  cudaError_t e = cudaMemsetAsync(p, value, bytes, cudaStreamLegacy);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(cudaStreamLegacy);
}

vxe_status alloc(vxe_ctx* c, DevBuf& b, size_t bytes) {
  if (b.p) {
    cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
  }
  b.pooled = false;
  if (bytes == 0) return VXE_OK;
  CK(cudaMalloc(&b.p, bytes));
  b.bytes = bytes;
  CK(fill_sync(b.p, 0, bytes));
  return VXE_OK;
}

// Releases a buffer; a pooled one after the work queued on `st` so far.
void release(DevBuf& b, cudaStream_t st = nullptr) {
  if (b.p) {
    if (b.pooled)
      cudaFreeAsync(b.p, st ? st : cudaStreamLegacy);
    else
      cudaFree(b.p);
  }
  b.p = nullptr;
  b.bytes = 0;
  b.pooled = false;
}

// Stream-ordered (re)allocation from the context's pool, zero-filled on `st`.
vxe_status alloc_on(vxe_ctx* c, DevBuf& b, size_t bytes, cudaStream_t st) {
  release(b, st);
  if (bytes == 0) return VXE_OK;
  CK(cudaMallocFromPoolAsync(&b.p, bytes, c->pool, st));
  b.bytes = bytes;
  b.pooled = true;
  CK(cudaMemsetAsync(b.p, 0, bytes, st));
  return VXE_OK;
}

// Stored grass column probes per internal pixel (the walk meets about four
// per pixel on grassland; pixels past the cap replay their walk).
constexpr size_t kProbesPerPixel = 8;
// Grass slab marches those probes ask for, per internal pixel.
constexpr size_t kSlabsPerPixel = 4;

size_t img_bytes(const FrameState& F, int i) {
  const size_t in = (size_t)F.iw * F.ih, pn = (size_t)F.pw * F.ph;
  const size_t tiles = (size_t)((F.iw + 7) / 8) * ((F.ih + 7) / 8);
  switch (i) {
    case IMG_COLOR: case IMG_LOCAL: case IMG_LHIST0: case IMG_LHIST1: case IMG_GOD0: case IMG_GOD1:
    case IMG_HIST0: case IMG_HIST1:
      return in * 16;
    case IMG_DEPTH: case IMG_SHADOW0: case IMG_SHADOW1:
      return in * 4;
    case IMG_PRE_TAA: case IMG_OUTPUT: case IMG_OHIST0: case IMG_OHIST1:
      return pn * 16;
    case IMG_HITS:
      return in * 32;
    case IMG_TILE_COUNT:
      return tiles * 4;
    case IMG_TILE_SLOTS:
      return tiles * 4 * VXE_PRIMARY_MAX_TILE_CHUNKS;
    case IMG_PIXHIT:
      return in * 80;
    case IMG_QVOX: case IMG_QFAR: case IMG_QSHADOW: case IMG_QLIGHT: case IMG_PXSHADOW: case IMG_QPENDING:
      return in * 4;
    case IMG_PROBE_RECS:
      return in * kProbesPerPixel * sizeof(vxe::dev::ProbeRec);
    case IMG_SLAB_TASKS:
      return in * kSlabsPerPixel * 16;
    case IMG_SLAB_RES:
      return in * kSlabsPerPixel * 16;
    case IMG_SLAB_HITS:
      return in * kSlabsPerPixel * 4;
    case IMG_PXTASK:
      return in * 4;
    case IMG_PXFIRST: case IMG_PXPROBE: case IMG_PXMASK:
      return in * 8;
    case IMG_PXLIGHT: case IMG_GODPRE: case IMG_PXGOV:
      return in * 16;
    case IMG_QCOUNT:
      return 64;
    default:
      return 0;
  }
}

bool img_enabled(const vxe_ctx* c, int i) {
  if (i == IMG_LOCAL || i == IMG_PRE_TAA) return (c->flags & VXE_FLAG_DEBUG_INTERMEDIATES) != 0;
  if (i == IMG_HITS) return (c->flags & VXE_FLAG_HIT_RECORDS) != 0;
  return true;
}

// Per-frame working buffers of the wavefront (tile lists, queues, probe and
// slab records): a frame's contents only, nothing carried to the next frame.
// A view borrows them from the lane it renders on; the rest of a frame state
// (outputs and histories) is its own.
bool img_is_scratch(int i) {
  return i == IMG_TILE_COUNT || i == IMG_TILE_SLOTS || i >= IMG_PIXHIT;
}

enum ImgSet { IMG_SET_ALL, IMG_SET_OWN, IMG_SET_SCRATCH };

bool img_in_set(int i, ImgSet set) {
  return set == IMG_SET_ALL || (set == IMG_SET_SCRATCH) == img_is_scratch(i);
}

// Allocates and zero-fills a frame state's images: synchronously, or with
// `st`, stream-ordered from the pool.
vxe_status alloc_images(vxe_ctx* c, FrameState& F, ImgSet set = IMG_SET_ALL, cudaStream_t st = nullptr) {
  for (int i = 0; i < IMG_N; ++i) {
    const size_t b = img_enabled(c, i) && img_in_set(i, set) ? img_bytes(F, i) : 0;
    if (b != F.img[i].bytes || (b != 0) != (F.img[i].p != nullptr)) {
      vxe_status rc = st ? alloc_on(c, F.img[i], b, st) : alloc(c, F.img[i], b);
      if (rc != VXE_OK) return rc;
    } else if (F.img[i].p) {
      if ((st ? cudaMemsetAsync(F.img[i].p, 0, b, st) : fill_sync(F.img[i].p, 0, b)) != cudaSuccess)
        return fail(c, VXE_ERR_DEVICE, "memset failed");
    }
  }
  F.ping = 0;
  return VXE_OK;
}

// Maps the public image id to the buffer index under the current ping.
int map_image(const FrameState& F, vxe_image im) {
  const int p = F.ping, q = 1 - F.ping;
  switch (im) {
    case VXE_IMG_COLOR: return IMG_COLOR;
    case VXE_IMG_DEPTH: return IMG_DEPTH;
    case VXE_IMG_LOCAL: return IMG_LOCAL;
    case VXE_IMG_PRIMARY_HIST_IN: return IMG_HIST0 + p;
    case VXE_IMG_PRIMARY_HIST_OUT: return IMG_HIST0 + q;
    case VXE_IMG_SHADOW_IN: return IMG_SHADOW0 + p;
    case VXE_IMG_SHADOW_OUT: return IMG_SHADOW0 + q;
    case VXE_IMG_LOCAL_HIST_IN: return IMG_LHIST0 + p;
    case VXE_IMG_LOCAL_HIST_OUT: return IMG_LHIST0 + q;
    case VXE_IMG_GODRAY_IN: return IMG_GOD0 + p;
    case VXE_IMG_GODRAY_OUT: return IMG_GOD0 + q;
    case VXE_IMG_OUTPUT_PRE_TAA: return IMG_PRE_TAA;
    case VXE_IMG_OUTPUT: return IMG_OUTPUT;
    case VXE_IMG_OUTPUT_HIST_IN: return IMG_OHIST0 + p;
    case VXE_IMG_OUTPUT_HIST_OUT: return IMG_OHIST0 + q;
    case VXE_IMG_HITS: return IMG_HITS;
    default: return -1;
  }
}

void fill_scene_args(const vxe_ctx* c, FrameArgs& A) {
  std::memset(&A, 0, sizeof A);
  A.cam = c->cam;
  A.clip = c->clip;
  A.nodes = (const uint4*)c->nodes.p;
  A.nodes_n = c->cfg.node_capacity;
  A.ropes = (const uint32_t*)c->ropes.p;
  A.ropes_n = c->cfg.node_capacity;
  A.metas = (const uint4*)c->metas.p;
  A.metas_n = c->cfg.chunk_capacity;
  A.grid = (const uint32_t*)c->grid.p;
  A.grid_n = c->cfg.grid_capacity;
  A.macro = (const uint32_t*)c->macro.p;
  A.macro_n = (uint64_t)c->cfg.chunk_capacity * VXE_MACRO_WORDS_PER_CHUNK;
  A.colinfo = (const uint32_t*)c->colinfo.p;
  A.colinfo_n = (uint64_t)c->cfg.chunk_capacity * VXE_COLINFO_WORDS_PER_CHUNK;
  A.clip_tex = (const float*)c->clip_tex.p;
  A.clip_layers = c->cfg.clip_levels;
  A.clip_res = c->cfg.clip_res;
  A.err = (uint32_t*)c->errword.p;
  A.godray_alias = (c->flags & VXE_FLAG_GODRAY_MACRO_ALIAS) ? 1u : 0u;
  A.slot_lights = (const uint32_t*)c->slot_lights.p;
  A.slot_top = (const uint32_t*)c->slot_top.p;
}

// Recomputes the light flags of slots [first, first + n) on the upload
// stream, after the writes queued there.
vxe_status slot_lights_refresh(vxe_ctx* c, uint32_t first, uint32_t n) {
  if (n == 0 || !c->slot_lights.p) return VXE_OK;
  vxe::dev::k_slot_lights<<<n, vxe::dev::SLOT_LIGHT_THREADS, 0, c->upload>>>(
      (const uint4*)c->metas.p, c->cfg.chunk_capacity, (const uint4*)c->nodes.p, c->cfg.node_capacity, first, 64u,
      (uint32_t*)c->slot_lights.p, (uint32_t*)c->slot_top.p);
  CK(cudaGetLastError());
  return VXE_OK;
}

uint32_t fbits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}

void grass_table_args(const vxe_ctx* c, FrameArgs& A) {
  A.grass_rec = (float4*)c->gt.rec.p;
  A.grass_rec_n = (uint64_t)c->cfg.chunk_capacity * 4096u;
  A.grass_state = (uint32_t*)c->gt.state.p;
  A.grass_frames = (float4*)c->gt.frames.p;
  A.grass_taper = (float*)c->gt.taper.p;
}

// Records of slots [slot0, slot0 + n) for camera `cam` on stream `st`.
vxe_status grass_table_fill(vxe_ctx* c, cudaStream_t st, const vxe_camera_gpu& cam, uint32_t slot0, uint32_t n,
                            bool list = false) {
  using namespace vxe::dev;
  if (n == 0) return VXE_OK;
  FrameArgs A;
  fill_scene_args(c, A);
  A.cam = cam;
  grass_table_args(c, A);
  A.grass_slot0 = slot0;
  if (list) {
    A.grass_list = (uint32_t*)c->gt.list.p;
    A.grass_list_n = (uint32_t*)c->gt.list_n.p;
    CK(cudaMemsetAsync(c->gt.list_n.p, 0, 4, st));
  }
  const uint64_t threads = (uint64_t)n * 4096u;
  k_grass_cells<<<(unsigned)((threads + GRASS_CELL_THREADS - 1) / GRASS_CELL_THREADS), GRASS_CELL_THREADS, 0, st>>>(A);
  CK(cudaGetLastError());
  return VXE_OK;
}

// Makes the table valid on stream `st` for `cam`; *use tells whether the
// pass may read it.  `reader` is the stream's index (0 compute, 1+ lanes).
vxe_status grass_table_acquire(vxe_ctx* c, cudaStream_t st, int reader, const vxe_camera_gpu& cam, bool* use) {
  *use = false;
  GrassTable& T = c->gt;
  if (!T.rec.p || (c->flags & VXE_FLAG_NO_GRASS_TABLE) || cam.chunk_count == 0 ||
      cam.chunk_count > c->cfg.chunk_capacity)
    return VXE_OK;
  const uint32_t tb = fbits(cam.voxel_params[1]), sb = fbits(cam.voxel_params[2]), vb = fbits(cam.voxel_params[0]);
  const bool same = T.valid && T.time_bits == tb && T.strength_bits == sb && T.vs_bits == vb &&
                    T.chunk_count == cam.chunk_count;
  if (!same) {
    for (int i = 0; i < kGrassReaders; ++i)
      if (T.reader_used[i]) CK(cudaStreamWaitEvent(st, T.reader[i], 0));
    if (T.built_recorded) CK(cudaStreamWaitEvent(st, T.built, 0));
    vxe_status s2 = VXE_OK;
    if (T.valid && T.list_valid && T.vs_bits == vb && T.chunk_count == cam.chunk_count) {
      // only the wind changed: rebuild the grass columns of the list
      FrameArgs A;
      fill_scene_args(c, A);
      A.cam = cam;
      grass_table_args(c, A);
      A.grass_list = (uint32_t*)T.list.p;
      A.grass_list_n = (uint32_t*)T.list_n.p;
      vxe::dev::k_grass_wind<<<c->shade_wave, vxe::dev::GRASS_CELL_THREADS, 0, st>>>(A);
      CK(cudaGetLastError());
    } else {
      s2 = grass_table_fill(c, st, cam, 0u, cam.chunk_count, true);
      T.list_valid = true;
    }
    if (s2 != VXE_OK) return s2;
    T.valid = true;
    T.time_bits = tb;
    T.strength_bits = sb;
    T.vs_bits = vb;
    T.chunk_count = cam.chunk_count;
    T.cam = cam;
  } else if (T.built_recorded) {
    CK(cudaStreamWaitEvent(st, T.built, 0));
  }
  CK(cudaEventRecord(T.built, st));
  T.built_recorded = true;
  *use = true;
  return VXE_OK;
}

// After chunk uploads: rebuild the records of the uploaded slots on the
// upload stream, ordered after the copies (and after the last full build).
// `slots`: sorted, without repeats.
vxe_status grass_table_refresh(vxe_ctx* c, const std::vector<uint32_t>& slots) {
  GrassTable& T = c->gt;
  if (!T.valid || slots.empty()) return VXE_OK;
  T.list_valid = false;  // the next wind change rebuilds every column
  if (T.built_recorded) CK(cudaStreamWaitEvent(c->upload, T.built, 0));
  for (size_t i = 0; i < slots.size() && slots[i] < T.chunk_count;) {  // one launch per run of consecutive slots
    size_t j = i + 1;
    while (j < slots.size() && slots[j] == slots[j - 1] + 1 && slots[j] < T.chunk_count) ++j;
    vxe_status st = grass_table_fill(c, c->upload, T.cam, slots[i], (uint32_t)(j - i));
    if (st != VXE_OK) return st;
    i = j;
  }
  return VXE_OK;
}

// Marks the end of a pass that read the table on stream `st`.
vxe_status grass_table_release(vxe_ctx* c, cudaStream_t st, int reader) {
  CK(cudaEventRecord(c->gt.reader[reader], st));
  c->gt.reader_used[reader] = true;
  return VXE_OK;
}

vxe_status frame_validate(vxe_ctx* c, const FrameState& F, const vxe_camera_gpu& cam) {
  if (F.iw == 0 || F.pw == 0) return fail(c, VXE_ERR_INVALID_ARG, "vxe_resize must be called before rendering");
  if (cam.render_present_px[0] != F.iw || cam.render_present_px[1] != F.ih ||
      cam.render_present_px[2] != F.pw || cam.render_present_px[3] != F.ph)
    return fail(c, VXE_ERR_INVALID_ARG, "camera render_present_px (%u,%u,%u,%u) does not match images (%u,%u,%u,%u)",
                cam.render_present_px[0], cam.render_present_px[1], cam.render_present_px[2],
                cam.render_present_px[3], F.iw, F.ih, F.pw, F.ph);
  if (cam.chunk_size != 64u) return fail(c, VXE_ERR_INVALID_ARG, "chunk_size must be 64 (colinfo layout)");
  if ((uint64_t)cam.grid_dims[0] * cam.grid_dims[1] * cam.grid_dims[2] > c->cfg.grid_capacity)
    return fail(c, VXE_ERR_CAPACITY, "grid_dims exceed grid capacity");
  if (cam.chunk_count > c->cfg.chunk_capacity) return fail(c, VXE_ERR_CAPACITY, "chunk_count exceeds capacity");
  if (c->clip.levels > c->cfg.clip_levels && c->clip.levels != 0)
    return fail(c, VXE_ERR_CAPACITY, "clipmap levels exceed allocated layers");
  if (c->clip.levels != 0 && c->clip.res != c->cfg.clip_res)
    return fail(c, VXE_ERR_INVALID_ARG, "clipmap res %u != allocated %u", c->clip.res, c->cfg.clip_res);
  return VXE_OK;
}

// `S` holds the per-frame working buffers (F itself, or a lane's for a view).
void frame_fill(vxe_ctx* c, FrameState& F, const vxe_camera_gpu& cam, FrameArgs& A, const FrameState* S = nullptr) {
  if (!S) S = &F;
  fill_scene_args(c, A);
  A.cam = cam;
  const int p = F.ping, q = 1 - F.ping;
  A.iw = F.iw;
  A.ih = F.ih;
  A.pw = F.pw;
  A.ph = F.ph;
  A.tile_count = (uint32_t*)S->img[IMG_TILE_COUNT].p;
  A.tile_slots = (uint32_t*)S->img[IMG_TILE_SLOTS].p;
  A.hist_in = (const uint4*)F.img[IMG_HIST0 + p].p;
  A.hist_out = (uint4*)F.img[IMG_HIST0 + q].p;
  A.shadow_in = (const float*)F.img[IMG_SHADOW0 + p].p;
  A.shadow_out = (float*)F.img[IMG_SHADOW0 + q].p;
  A.local_hist_in = (const float4*)F.img[IMG_LHIST0 + p].p;
  A.local_hist_out = (float4*)F.img[IMG_LHIST0 + q].p;
  A.color = (float4*)F.img[IMG_COLOR].p;
  A.depth = (float*)F.img[IMG_DEPTH].p;
  A.local = (float4*)F.img[IMG_LOCAL].p;
  A.god_in = (const float4*)F.img[IMG_GOD0 + p].p;
  A.god_out = (float4*)F.img[IMG_GOD0 + q].p;
  A.pre_taa = (float4*)F.img[IMG_PRE_TAA].p;
  A.output = (float4*)F.img[IMG_OUTPUT].p;
  A.out_hist_in = (const float4*)F.img[IMG_OHIST0 + p].p;
  A.out_hist_out = (float4*)F.img[IMG_OHIST0 + q].p;
  A.hits = (uint4*)F.img[IMG_HITS].p;
  A.pix_hit = (uint4*)S->img[IMG_PIXHIT].p;
  A.q_vox = (uint32_t*)S->img[IMG_QVOX].p;
  A.q_far = (uint32_t*)S->img[IMG_QFAR].p;
  A.q_count = (uint32_t*)S->img[IMG_QCOUNT].p;
  A.q_shadow = (uint32_t*)S->img[IMG_QSHADOW].p;
  A.q_light = (uint32_t*)S->img[IMG_QLIGHT].p;
  A.px_shadow = (float*)S->img[IMG_PXSHADOW].p;
  A.px_light = (float4*)S->img[IMG_PXLIGHT].p;
  A.probe_recs = (vxe::dev::ProbeRec*)S->img[IMG_PROBE_RECS].p;
  A.probe_cap = (uint32_t)std::min<size_t>(S->img[IMG_PROBE_RECS].bytes / sizeof(vxe::dev::ProbeRec), 0xFFFFFFFFu);
  if (c->probe_limit) A.probe_cap = std::min(A.probe_cap, c->probe_limit);
  A.slab_tasks = (uint4*)S->img[IMG_SLAB_TASKS].p;
  A.slab_res = (float4*)S->img[IMG_SLAB_RES].p;
  A.slab_cap = (uint32_t)std::min<size_t>(S->img[IMG_SLAB_TASKS].bytes / 16u, 0xFFFFFFFFu);
  if (c->slab_limit) A.slab_cap = std::min(A.slab_cap, c->slab_limit);
  A.px_first = (unsigned long long*)S->img[IMG_PXFIRST].p;
  A.px_probe = (uint2*)S->img[IMG_PXPROBE].p;
  A.slab_hits = (uint32_t*)S->img[IMG_SLAB_HITS].p;
  A.px_task = (uint32_t*)S->img[IMG_PXTASK].p;
  A.px_mask = (uint2*)S->img[IMG_PXMASK].p;
  // the wavefront walk leaves grass-voxel blade marches to k_gov_eval
  A.px_gov = (c->flags & VXE_FLAG_PRIMARY_MEGAKERNEL) ? nullptr : (uint4*)S->img[IMG_PXGOV].p;
  A.q_pending = (uint32_t*)S->img[IMG_QPENDING].p;
  A.god_pre = (c->flags & VXE_FLAG_PRIMARY_MEGAKERNEL) ? nullptr : (float4*)S->img[IMG_GODPRE].p;
}

// The frame's launches on the compute stream (captured as-is by the graph
// path; `timed` adds the per-pass events).
vxe_status side_ready(vxe_ctx* c, SideStream& S) {
  if (S.s) return VXE_OK;
  CK(cudaStreamCreateWithFlags(&S.s, cudaStreamNonBlocking));
  for (cudaEvent_t* e : {&S.fork, &S.mid, &S.prep, &S.join, &S.pre, &S.table})
    CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  return VXE_OK;
}

void side_release(SideStream& S) {
  if (S.s) {
    cudaStreamSynchronize(S.s);
    cudaStreamDestroy(S.s);
  }
  for (cudaEvent_t e : {S.fork, S.mid, S.prep, S.join, S.pre, S.table})
    if (e) cudaEventDestroy(e);
  S = SideStream{};
}

vxe_status frame_enqueue(vxe_ctx* c, FrameState& F, const FrameArgs& A, bool timed, cudaStream_t st,
                         SideStream* side) {
  const uint32_t tiles_x = (F.iw + 7) / 8, tiles_y = (F.ih + 7) / 8;
  const uint32_t tiles = tiles_x * tiles_y;
  const uint32_t npix = F.iw * F.ih;
  using namespace vxe::dev;
  if (timed) CK(cudaEventRecord(F.ev[1], st));
  k_tiles<<<(tiles + TILE_THREADS - 1) / TILE_THREADS, TILE_THREADS, 0, st>>>(A);
  if (timed) CK(cudaEventRecord(F.ev[2], st));
  if (c->flags & VXE_FLAG_PRIMARY_MEGAKERNEL) {
    k_primary<<<dim3((tiles_x + 1) / 2, tiles_y), PRIMARY_THREADS, 0, st>>>(A);
    if (timed) CK(cudaEventRecord(F.ev[3], st));
  } else {
    // Queue lengths stay on the device: each kernel after the walk runs over
    // its queue with a grid-stride loop over at most a full wave of blocks.
    auto grid = [&](uint64_t threads) {
      return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((threads + SHADE_THREADS - 1) / SHADE_THREADS,
                                                                (uint64_t)c->shade_wave));
    };
    CK(cudaMemsetAsync(A.q_count, 0, 64, st));
    vxe_status sr;
    if (side && (sr = side_ready(c, *side)) != VXE_OK) return sr;
    CK(cudaMemsetAsync(A.px_first, 0xFF, (size_t)npix * 8u, st));
    CK(cudaMemsetAsync(A.px_mask, 0, (size_t)npix * 8u, st));
    if (A.god_pre) CK(cudaMemsetAsync(A.god_pre, 0, (size_t)npix * 16u, st));
    if (timed) CK(cudaEventRecord(F.ev[7], st));
    k_primary_trace<<<dim3((tiles_x + 1) / 2, tiles_y), PRIMARY_THREADS, 0, st>>>(A);
    if (timed) CK(cudaEventRecord(F.ev[8], st));
    if (side) {  // the walk's far pixels shade beside the probe passes
      CK(cudaMemcpyAsync(A.q_count + 8, A.q_count + 1, 4, cudaMemcpyDeviceToDevice, st));
      CK(cudaEventRecord(side->fork, st));
      CK(cudaStreamWaitEvent(side->s, side->fork, 0));
      k_shade_far<0><<<grid(npix), SHADE_THREADS, 0, side->s>>>(A);
      // their godray integrals too, while the compute stream runs the probes
      k_godray_far<<<grid(npix), SHADE_THREADS, 0, side->s>>>(A);
    }
    k_probe_dda<<<grid((uint64_t)npix * kProbesPerPixel), SHADE_THREADS, 0, st>>>(A);
    if (F.table_wait) CK(cudaStreamWaitEvent(st, F.table_wait, 0));
    k_slab_eval<<<grid((uint64_t)npix * kSlabsPerPixel), SHADE_THREADS, 0, st>>>(A);
    k_slab_pick<<<grid(npix), SHADE_THREADS, 0, st>>>(A);
    k_gov_eval<<<grid(npix), SHADE_THREADS, 0, st>>>(A);
    k_primary_resolve<<<grid(npix), SHADE_THREADS, 0, st>>>(A);
    if (timed) CK(cudaEventRecord(F.ev[3], st));
    if (side) {  // the far pixels the resolve queued, beside the voxel shading
      CK(cudaEventRecord(side->mid, st));
      CK(cudaStreamWaitEvent(side->s, side->mid, 0));
      k_shade_far<1><<<grid(npix), SHADE_THREADS, 0, side->s>>>(A);
    }
    k_shade_prep<<<grid(npix), SHADE_THREADS, 0, st>>>(A);
    if (side) {
      // Every depth is final here (voxel pixels' from k_shade_prep, far
      // pixels' from k_shade_far), and godray reads nothing else the shading
      // writes: it runs beside the rest of the voxel shading.
      CK(cudaEventRecord(side->prep, st));
      CK(cudaStreamWaitEvent(side->s, side->prep, 0));
      if (timed) CK(cudaEventRecord(F.ev[4], side->s));
      k_godray<<<dim3((F.iw + POST_THREADS_X - 1) / POST_THREADS_X, (F.ih + POST_THREADS_Y - 1) / POST_THREADS_Y),
                 dim3(POST_THREADS_X, POST_THREADS_Y), 0, side->s>>>(A);
      if (timed) CK(cudaEventRecord(F.ev[5], side->s));
      CK(cudaEventRecord(side->join, side->s));
    }
    k_shade_shadow<<<grid(npix), SHADE_THREADS, 0, st>>>(A);
    k_shade_lights<<<grid((uint64_t)npix * 8u), SHADE_THREADS, 0, st>>>(A);
    k_shade_vox<<<grid(npix), SHADE_THREADS, 0, st>>>(A);
    if (side)
      CK(cudaStreamWaitEvent(st, side->join, 0));
    else
      k_shade_far<2><<<grid(npix), SHADE_THREADS, 0, st>>>(A);
  }
  if (!side || (c->flags & VXE_FLAG_PRIMARY_MEGAKERNEL)) {
    if (timed) CK(cudaEventRecord(F.ev[4], st));
    k_godray<<<dim3((F.iw + POST_THREADS_X - 1) / POST_THREADS_X, (F.ih + POST_THREADS_Y - 1) / POST_THREADS_Y),
               dim3(POST_THREADS_X, POST_THREADS_Y), 0, st>>>(A);
    if (timed) CK(cudaEventRecord(F.ev[5], st));
  }
  if (F.composite_wait) CK(cudaStreamWaitEvent(st, F.composite_wait, 0));
  k_composite<<<dim3((F.pw + POST_THREADS_X - 1) / POST_THREADS_X, (F.ph + POST_THREADS_Y - 1) / POST_THREADS_Y),
                dim3(POST_THREADS_X, POST_THREADS_Y), 0, st>>>(A);
  if (timed) CK(cudaEventRecord(F.ev[6], st));
  CK(cudaGetLastError());
  return VXE_OK;
}

// The wavefront frame of n views (vxe_view_render_batch_async): each pass is
// one launch over all of them (blockIdx.z = view), sized for the largest.
vxe_status views_enqueue(vxe_ctx* c, const vxe::dev::FrameArgsViews& V, uint32_t n, uint32_t max_iw,
                         uint32_t max_ih, uint32_t max_pw, uint32_t max_ph, uint64_t max_pix, cudaStream_t st,
                         SideStream* side) {
  using namespace vxe::dev;
  const uint32_t tiles_x = (max_iw + 7) / 8, tiles_y = (max_ih + 7) / 8;
  const uint32_t per_view = std::max<uint32_t>(1u, (uint32_t)c->shade_wave / n);
  auto grid = [&](uint64_t threads) {
    return dim3((unsigned)std::max<uint64_t>(1, std::min<uint64_t>((threads + SHADE_THREADS - 1) / SHADE_THREADS,
                                                                    (uint64_t)per_view)),
                1, n);
  };
  for (uint32_t i = 0; i < n; ++i) {
    const FrameArgs& A = V.v[i];
    const size_t npix = (size_t)A.iw * A.ih;
    CK(cudaMemsetAsync(A.q_count, 0, 64, st));
    CK(cudaMemsetAsync(A.px_first, 0xFF, npix * 8u, st));
    CK(cudaMemsetAsync(A.px_mask, 0, npix * 8u, st));
    if (A.god_pre) CK(cudaMemsetAsync(A.god_pre, 0, npix * 16u, st));
  }
  vxe_status sr = side_ready(c, *side);
  if (sr != VXE_OK) return sr;
  k_tiles_views<<<dim3((tiles_x * tiles_y + TILE_THREADS - 1) / TILE_THREADS, 1, n), TILE_THREADS, 0, st>>>(V);
  k_primary_trace_views<<<dim3((tiles_x + 1) / 2, tiles_y, n), PRIMARY_THREADS, 0, st>>>(V);
  for (uint32_t i = 0; i < n; ++i)  // the walk's far pixels shade beside the probe passes
    CK(cudaMemcpyAsync(V.v[i].q_count + 8, V.v[i].q_count + 1, 4, cudaMemcpyDeviceToDevice, st));
  CK(cudaEventRecord(side->fork, st));
  CK(cudaStreamWaitEvent(side->s, side->fork, 0));
  k_shade_far_views<0><<<grid(max_pix), SHADE_THREADS, 0, side->s>>>(V);
  k_godray_far_views<<<grid(max_pix), SHADE_THREADS, 0, side->s>>>(V);
  k_probe_dda_views<<<grid(max_pix * kProbesPerPixel), SHADE_THREADS, 0, st>>>(V);
  k_slab_eval_views<<<grid(max_pix * kSlabsPerPixel), SHADE_THREADS, 0, st>>>(V);
  k_slab_pick_views<<<grid(max_pix), SHADE_THREADS, 0, st>>>(V);
  k_gov_eval_views<<<grid(max_pix), SHADE_THREADS, 0, st>>>(V);
  k_primary_resolve_views<<<grid(max_pix), SHADE_THREADS, 0, st>>>(V);
  CK(cudaEventRecord(side->mid, st));
  CK(cudaStreamWaitEvent(side->s, side->mid, 0));
  k_shade_far_views<1><<<grid(max_pix), SHADE_THREADS, 0, side->s>>>(V);
  k_shade_prep_views<<<grid(max_pix), SHADE_THREADS, 0, st>>>(V);
  CK(cudaEventRecord(side->prep, st));
  CK(cudaStreamWaitEvent(side->s, side->prep, 0));
  k_godray_views<<<dim3((max_iw + POST_THREADS_X - 1) / POST_THREADS_X, (max_ih + POST_THREADS_Y - 1) / POST_THREADS_Y, n),
                   dim3(POST_THREADS_X, POST_THREADS_Y), 0, side->s>>>(V);
  CK(cudaEventRecord(side->join, side->s));
  k_shade_shadow_views<<<grid(max_pix), SHADE_THREADS, 0, st>>>(V);
  k_shade_lights_views<<<grid(max_pix * 8u), SHADE_THREADS, 0, st>>>(V);
  k_shade_vox_views<<<grid(max_pix), SHADE_THREADS, 0, st>>>(V);
  CK(cudaStreamWaitEvent(st, side->join, 0));
  k_composite_views<<<dim3((max_pw + POST_THREADS_X - 1) / POST_THREADS_X, (max_ph + POST_THREADS_Y - 1) / POST_THREADS_Y,
                           n),
                      dim3(POST_THREADS_X, POST_THREADS_Y), 0, st>>>(V);
  CK(cudaGetLastError());
  return VXE_OK;
}

vxe_status launch_frame(vxe_ctx* c, bool timed) {
  vxe_status st = frame_validate(c, c->fr, c->cam);
  if (st != VXE_OK) return st;
  if (c->upload_recorded) CK(cudaStreamWaitEvent(c->compute, c->upload_done, 0));
  if (c->any_pending) {  // an image other than the output: before any pass
    CK(cudaStreamWaitEvent(c->compute, c->any_ev, 0));
    c->any_pending = false;
  }
  FrameArgs A;
  frame_fill(c, c->fr, c->cam, A);
  A.profile = (uint32_t*)c->profile.p;
  if (timed) CK(cudaEventRecord(c->fr.ev[0], c->compute));
  // In the wavefront schedule the walk reads nothing of the grass cell table
  // (its blade marches are deferred), so the table's per-frame rebuild runs
  // on the side stream beside the tile lists and the walk; the blade marches
  // wait for it.
  const bool table_beside = !(c->flags & VXE_FLAG_PRIMARY_MEGAKERNEL);
  cudaStream_t gst = c->compute;
  if (table_beside) {
    if ((st = side_ready(c, c->side)) != VXE_OK) return st;
    CK(cudaEventRecord(c->side.pre, c->compute));
    CK(cudaStreamWaitEvent(c->side.s, c->side.pre, 0));
    gst = c->side.s;
  }
  bool use_grass = false;
  if ((st = grass_table_acquire(c, gst, 0, c->cam, &use_grass)) != VXE_OK) return st;
  if (use_grass) grass_table_args(c, A);
  if (table_beside) CK(cudaEventRecord(c->side.table, gst));
  c->fr.table_wait = table_beside ? c->side.table : nullptr;
  c->fr.composite_wait = c->out_pending ? c->out_ev : nullptr;
  st = frame_enqueue(c, c->fr, A, timed, c->compute, &c->side);
  c->fr.composite_wait = nullptr;
  c->fr.table_wait = nullptr;
  if (st != VXE_OK) return st;
  c->out_pending = false;
  if (use_grass && (st = grass_table_release(c, c->compute, 0)) != VXE_OK) return st;
  c->fr.timed = timed;
  c->fr.timed_trace = timed && !(c->flags & VXE_FLAG_PRIMARY_MEGAKERNEL);
  c->fr.ping = 1 - c->fr.ping;
  return VXE_OK;
}

// The frame as one CUDA graph: captured on first use and again whenever the
// launch shapes or the buffers of its memset nodes change (resize, schedule,
// grass table use); every other frame only rewrites the kernel nodes'
// argument (camera, clipmap uniform, ping-pong images) and relaunches.  The
// grass cell table's (re)build is launched before the graph, outside it.
vxe_status launch_frame_graph(vxe_ctx* c, FrameState& F, const vxe_camera_gpu& cam, cudaStream_t st, int reader) {
  vxe_status rc = frame_validate(c, F, cam);
  if (rc != VXE_OK) return rc;
  if (c->upload_recorded) CK(cudaStreamWaitEvent(st, c->upload_done, 0));
  if (&F == &c->fr) {  // asynchronous reads of the context's images land first
    if (c->out_pending) CK(cudaStreamWaitEvent(st, c->out_ev, 0));
    if (c->any_pending) CK(cudaStreamWaitEvent(st, c->any_ev, 0));
    c->out_pending = c->any_pending = false;
  }
  FrameArgs A;
  frame_fill(c, F, cam, A);
  if (&F == &c->fr) A.profile = (uint32_t*)c->profile.p;
  bool use_grass = false;
  if ((rc = grass_table_acquire(c, st, reader, cam, &use_grass)) != VXE_OK) return rc;
  if (use_grass) grass_table_args(c, A);
  const uint64_t key[8] = {F.iw, F.ih, F.pw, F.ph,
                           (uint64_t)(c->flags & VXE_FLAG_PRIMARY_MEGAKERNEL) | (use_grass ? 2u : 0u),
                           (uint64_t)c->shade_wave, (uint64_t)(uintptr_t)A.q_count, (uint64_t)(uintptr_t)A.px_first};
  if (!F.fgraph_exec || std::memcmp(key, F.fgraph_key, sizeof key) != 0) {
    if (F.fgraph_exec) cudaGraphExecDestroy(F.fgraph_exec);
    if (F.fgraph) cudaGraphDestroy(F.fgraph);
    F.fgraph_exec = nullptr;
    F.fgraph = nullptr;
    F.fgraph_nodes.clear();
    if (st == c->compute && (rc = side_ready(c, c->side)) != VXE_OK) return rc;  // created outside the capture
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    rc = frame_enqueue(c, F, A, false, st, st == c->compute ? &c->side : nullptr);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &g);
    if (rc != VXE_OK) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return fail(c, VXE_ERR_DEVICE, "frame graph capture: %s", cudaGetErrorString(e));
    F.fgraph = g;
    size_t n = 0;
    CK(cudaGraphGetNodes(g, nullptr, &n));
    std::vector<cudaGraphNode_t> nodes(n);
    if (n) CK(cudaGraphGetNodes(g, nodes.data(), &n));
    for (cudaGraphNode_t nd : nodes) {
      cudaGraphNodeType t;
      CK(cudaGraphNodeGetType(nd, &t));
      if (t == cudaGraphNodeTypeKernel) F.fgraph_nodes.push_back(nd);
    }
    CK(cudaGraphInstantiate(&F.fgraph_exec, g, 0));
    std::memcpy(F.fgraph_key, key, sizeof key);
  } else {
    // every frame kernel takes the one FrameArgs
    void* args[1] = {(void*)&A};
    for (cudaGraphNode_t nd : F.fgraph_nodes) {
      cudaKernelNodeParams kp;
      CK(cudaGraphKernelNodeGetParams(nd, &kp));
      kp.kernelParams = args;
      kp.extra = nullptr;
      CK(cudaGraphExecKernelNodeSetParams(F.fgraph_exec, nd, &kp));
    }
  }
  CK(cudaGraphLaunch(F.fgraph_exec, st));
  if (use_grass && (rc = grass_table_release(c, st, reader)) != VXE_OK) return rc;
  F.timed = false;
  F.timed_trace = false;
  F.ping = 1 - F.ping;
  return VXE_OK;
}

// internal = round(present * scale).max(1) (render/state/mod.rs:239-241);
// f32::round rounds half away from zero, like std::round.
void set_dims(FrameState& F, uint32_t present_w, uint32_t present_h, float render_scale) {
  const float fw = (float)present_w * render_scale, fh = (float)present_h * render_scale;
  F.iw = (uint32_t)std::max(1.0f, std::round(fw));
  F.ih = (uint32_t)std::max(1.0f, std::round(fh));
  F.pw = present_w;
  F.ph = present_h;
}

void release_frame_state(FrameState& F, cudaStream_t st = nullptr) {
  if (F.fgraph_exec) cudaGraphExecDestroy(F.fgraph_exec);
  if (F.fgraph) cudaGraphDestroy(F.fgraph);
  F.fgraph_exec = nullptr;
  F.fgraph = nullptr;
  F.fgraph_nodes.clear();
  for (auto& b : F.img) release(b, st);
}

void frame_out(vxe_ctx* c, vxe_frame_out* out) {
  if (!out) return;
  out->color = (float*)c->fr.img[IMG_COLOR].p;
  out->depth = (float*)c->fr.img[IMG_DEPTH].p;
  out->godray = (float*)c->fr.img[IMG_GOD0 + c->fr.ping].p;  // written this frame (ping already flipped)
  out->output = (float*)c->fr.img[IMG_OUTPUT].p;
  out->internal_w = c->fr.iw;
  out->internal_h = c->fr.ih;
  out->present_w = c->fr.pw;
  out->present_h = c->fr.ph;
}

}  // namespace

extern "C" {

vxe_status vxe_create(const vxe_config* cfg, vxe_ctx** out) {
  if (!cfg || !out) return VXE_ERR_INVALID_ARG;
  *out = nullptr;
  if (cfg->node_capacity == 0 || cfg->chunk_capacity == 0 || cfg->grid_capacity == 0 ||
      cfg->clip_levels > VXE_CLIP_LEVELS_MAX)
    return VXE_ERR_INVALID_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= cfg->device || cfg->device < 0) return VXE_ERR_NO_DEVICE;
  auto* c = new (std::nothrow) vxe_ctx();
  if (!c) return VXE_ERR_OOM;
  c->cfg = *cfg;
  c->flags = cfg->flags;
  c->device = cfg->device;
  vxe_status st = VXE_OK;
  auto bail = [&](vxe_status s) {
    vxe_destroy(c);
    return s;
  };
  if (cudaSetDevice(c->device) != cudaSuccess) return bail(VXE_ERR_DEVICE);
  if (cudaStreamCreateWithFlags(&c->compute, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->upload, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->upload_done, cudaEventDisableTiming) != cudaSuccess)
    return bail(VXE_ERR_DEVICE);
  for (auto& e : c->fr.ev)
    if (cudaEventCreate(&e) != cudaSuccess) return bail(VXE_ERR_DEVICE);
  {
    cudaMemPoolProps pp{};
    pp.allocType = cudaMemAllocationTypePinned;
    pp.handleTypes = cudaMemHandleTypeNone;
    pp.location.type = cudaMemLocationTypeDevice;
    pp.location.id = c->device;
    if (cudaMemPoolCreate(&c->pool, &pp) != cudaSuccess) return bail(VXE_ERR_DEVICE);
    // keep freed blocks for the next view or lane growth
    uint64_t keep = ~0ull;
    if (cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess)
      return bail(VXE_ERR_DEVICE);
  }
  const uint64_t nc = cfg->node_capacity, cc = cfg->chunk_capacity;
  if ((st = alloc(c, c->nodes, nc * 16)) != VXE_OK) return bail(st);
  if ((st = alloc(c, c->ropes, nc * 32)) != VXE_OK) return bail(st);
  if ((st = alloc(c, c->metas, cc * 48)) != VXE_OK) return bail(st);
  if ((st = alloc(c, c->macro, cc * VXE_MACRO_WORDS_PER_CHUNK * 4)) != VXE_OK) return bail(st);
  if ((st = alloc(c, c->colinfo, cc * VXE_COLINFO_WORDS_PER_CHUNK * 4)) != VXE_OK) return bail(st);
  if ((st = alloc(c, c->grid, (uint64_t)cfg->grid_capacity * 4)) != VXE_OK) return bail(st);
  if (fill_sync(c->grid.p, 0xFF, c->grid.bytes) != cudaSuccess) return bail(VXE_ERR_DEVICE);
  const uint64_t clip_bytes = (uint64_t)cfg->clip_levels * cfg->clip_res * cfg->clip_res * 4;
  if ((st = alloc(c, c->clip_tex, clip_bytes)) != VXE_OK) return bail(st);
  if ((st = alloc(c, c->errword, 4)) != VXE_OK) return bail(st);
  if ((st = alloc(c, c->slot_lights, cc * 4)) != VXE_OK) return bail(st);
  if ((st = alloc(c, c->slot_top, cc * 4)) != VXE_OK) return bail(st);
  if ((st = alloc(c, c->profile, 32)) != VXE_OK) return bail(st);
  if (fill_sync(c->profile.p, 0, 32) != cudaSuccess) return bail(VXE_ERR_DEVICE);
  if (!(cfg->flags & VXE_FLAG_NO_GRASS_TABLE)) {
    if ((st = alloc(c, c->gt.rec, cc * 4096u * vxe::dev::GRASS_REC_F4 * 16u)) != VXE_OK) return bail(st);
    if ((st = alloc(c, c->gt.taper, vxe::dev::GRASS_TAPER_N * 4u)) != VXE_OK) return bail(st);
    if ((st = alloc(c, c->gt.state, cc * 4096u * 4u)) != VXE_OK) return bail(st);
    if ((st = alloc(c, c->gt.list, cc * 4096u * 4u)) != VXE_OK) return bail(st);
    if ((st = alloc(c, c->gt.list_n, 4)) != VXE_OK) return bail(st);
    if ((st = alloc(c, c->gt.frames, cc * 4096u * vxe::dev::GRASS_FRAME_F4 * 16u)) != VXE_OK) return bail(st);
  }
  if (cudaEventCreateWithFlags(&c->gt.built, cudaEventDisableTiming) != cudaSuccess) return bail(VXE_ERR_DEVICE);
  for (auto& e : c->gt.reader)
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return bail(VXE_ERR_DEVICE);
  c->cam.chunk_size = 64u;
  {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device) == cudaSuccess && sms > 0)
      c->shade_wave = sms * 16;
  }
  // two pinned staging blocks up front: a stream's first chunk uploads need
  // them, and allocating pinned memory then would hold the host for ms
  for (int i = 0; i < 2; ++i) {
    const vxe_status sb = stage_block_add(c);
    if (sb != VXE_OK) return bail(sb);
  }
  *out = c;
  return VXE_OK;
}

void vxe_destroy(vxe_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->compute) cudaStreamSynchronize(c->compute);
  if (c->upload) cudaStreamSynchronize(c->upload);
  if (c->copy) {
    cudaStreamSynchronize(c->copy);
    cudaStreamDestroy(c->copy);
  }
  for (auto& e : c->copy_ev)
    if (e) cudaEventDestroy(e);
  if (c->fr.fgraph_exec) cudaGraphExecDestroy(c->fr.fgraph_exec);
  if (c->fr.fgraph) cudaGraphDestroy(c->fr.fgraph);
  for (auto& L : c->lanes)  // lanes read the arenas: drain them before freeing
    if (L.stream) cudaStreamSynchronize(L.stream);
  for (auto* b : {&c->nodes, &c->ropes, &c->metas, &c->macro, &c->colinfo, &c->grid, &c->clip_tex, &c->errword, &c->slot_lights, &c->slot_top, &c->profile, &c->build_scratch, &c->build_places, &c->move_buf,
                  &c->q_in, &c->q_out, &c->gt.rec, &c->gt.taper, &c->gt.state, &c->gt.frames,
                  &c->gt.list, &c->gt.list_n})
    release(*b);
  for (auto& L : c->lanes) {
    if (L.stream) cudaStreamSynchronize(L.stream);
    for (auto* b : {&L.hdr, &L.reqs, &L.cams, &L.tile_count, &L.tile_slots, &L.head, &L.probe_recs, &L.slab_tasks,
                    &L.slab_res, &L.slab_hits, &L.px_first, &L.px_task, &L.px_mask, &L.px_probe, &L.px_hit,
                    &L.q_pending, &L.q_refine, &L.q_far, &L.dcount, &L.q_keys, &L.q_perm, &L.bin_count})
      release(*b, L.stream);
    release_frame_state(L.scratch, L.stream);
    for (auto& m : L.mscratch) release_frame_state(m, L.stream);
    if (L.stream) cudaStreamSynchronize(L.stream);
    side_release(L.side);
    if (L.graph) cudaGraphExecDestroy(L.graph);
    if (L.stage) cudaFreeHost(L.stage);
    for (auto& e : L.ev)
      if (e) cudaEventDestroy(e);
    if (L.stream) cudaStreamDestroy(L.stream);
  }
  if (c->aux) {
    cudaStreamSynchronize(c->aux);
    cudaStreamDestroy(c->aux);
  }
  for (auto& e : c->build_ev)
    if (e) cudaEventDestroy(e);
  if (c->pool) cudaMemPoolDestroy(c->pool);
  for (auto& e : c->rd_ev)
    if (e) cudaEventDestroy(e);
  if (c->upload) cudaStreamSynchronize(c->upload);
  for (auto& b : c->ring) {
    cudaFreeHost(b.p);
    if (b.ev) cudaEventDestroy(b.ev);
  }
  for (auto& b : c->fr.img) release(b);
  for (auto& e : c->fr.ev)
    if (e) cudaEventDestroy(e);
  if (c->gt.built) cudaEventDestroy(c->gt.built);
  for (auto& e : c->gt.reader)
    if (e) cudaEventDestroy(e);
  if (c->upload_done) cudaEventDestroy(c->upload_done);
  side_release(c->side);
  if (c->compute) cudaStreamDestroy(c->compute);
  if (c->upload) cudaStreamDestroy(c->upload);
  delete c;
}

const char* vxe_last_error(const vxe_ctx* c) { return c ? c->err.c_str() : "null context"; }

uint32_t vxe_get_flags(const vxe_ctx* c) { return c ? c->flags : 0u; }

vxe_status vxe_set_flags(vxe_ctx* c, uint32_t flags) {
  if (!c) return VXE_ERR_INVALID_ARG;
  const uint32_t img_bits = VXE_FLAG_DEBUG_INTERMEDIATES | VXE_FLAG_HIT_RECORDS;
  const bool realloc = ((flags ^ c->flags) & img_bits) != 0;
  c->flags = flags;
  if (realloc && c->fr.iw != 0) {
    cudaSetDevice(c->device);
    // Only (de)allocate the optional images; histories are kept.
    for (int i : {IMG_LOCAL, IMG_PRE_TAA, IMG_HITS}) {
      const size_t b = img_enabled(c, i) ? img_bytes(c->fr, i) : 0;
      if (b != c->fr.img[i].bytes) {
        vxe_status st = alloc(c, c->fr.img[i], b);
        if (st != VXE_OK) return st;
      }
    }
  }
  return VXE_OK;
}

vxe_status vxe_resize(vxe_ctx* c, uint32_t present_w, uint32_t present_h, float render_scale) {
  if (!c || present_w == 0 || present_h == 0 || !(render_scale > 0.0f) || render_scale > 4.0f)
    return fail(c, VXE_ERR_INVALID_ARG, "bad resize arguments");
  cudaSetDevice(c->device);
  CK(cudaStreamSynchronize(c->compute));
  if (c->copy) CK(cudaStreamSynchronize(c->copy));
  set_dims(c->fr, present_w, present_h, render_scale);
  return alloc_images(c, c->fr);
}

vxe_status vxe_get_internal_dims(const vxe_ctx* c, uint32_t* w, uint32_t* h) {
  if (!c || !w || !h) return VXE_ERR_INVALID_ARG;
  *w = c->fr.iw;
  *h = c->fr.ih;
  return VXE_OK;
}

}  // extern "C"

namespace {

constexpr size_t kStageBlock = (size_t)16 << 20;
constexpr size_t kStageBlocksMax = 16;  // 256 MB of pinned staging at most

vxe_status stage_block_add(vxe_ctx* c) {
  vxe_ctx::StageBlock b;
  CK(cudaMallocHost((void**)&b.p, kStageBlock));
  if (cudaEventCreateWithFlags(&b.ev, cudaEventDisableTiming) != cudaSuccess) {
    cudaFreeHost(b.p);
    return fail(c, VXE_ERR_DEVICE, "staging event");
  }
  c->ring.push_back(b);
  return VXE_OK;
}

// Queues a host-to-device copy on the upload stream through the pinned
// staging blocks: the host returns once the bytes are in pinned memory (a
// pageable cudaMemcpyAsync would hold the host until the copy has run).
// World writes wait for the passes in flight, so with a deep queue the next
// block may still be in use: another block is added rather than waiting,
// up to the cap.
vxe_status ring_copy(vxe_ctx* c, void* dst, const void* src, size_t bytes) {
  vxe_status rs;
  if (c->ring.empty() && (rs = stage_block_add(c)) != VXE_OK) return rs;
  char* d = (char*)dst;
  const char* h = (const char*)src;
  while (bytes) {
    if (c->ring_off >= kStageBlock) {  // this block is full: move to a free one
      vxe_ctx::StageBlock& cur = c->ring[c->ring_cur];
      CK(cudaEventRecord(cur.ev, c->upload));
      cur.rec = true;
      const size_t next = (c->ring_cur + 1) % c->ring.size();
      vxe_ctx::StageBlock& nb = c->ring[next];
      const cudaError_t q = nb.rec ? cudaEventQuery(nb.ev) : cudaSuccess;
      if (q != cudaSuccess && q != cudaErrorNotReady) return fail(c, VXE_ERR_DEVICE, "staging event query");
      if (q == cudaErrorNotReady && c->ring.size() < kStageBlocksMax) {
        if ((rs = stage_block_add(c)) != VXE_OK) return rs;
        // the new block goes after the current one, so blocks stay in fill order
        std::rotate(c->ring.begin() + c->ring_cur + 1, c->ring.end() - 1, c->ring.end());
        c->ring_cur = c->ring_cur + 1;
      } else {
        if (q == cudaErrorNotReady) CK(cudaEventSynchronize(nb.ev));
        c->ring_cur = next;
      }
      c->ring_off = 0;
    }
    const size_t n = std::min(bytes, kStageBlock - c->ring_off);
    char* stage = c->ring[c->ring_cur].p + c->ring_off;
    std::memcpy(stage, h, n);
    CK(cudaMemcpyAsync(d, stage, n, cudaMemcpyHostToDevice, c->upload));
    c->ring_off = (c->ring_off + n + 15) & ~(size_t)15;
    d += n;
    h += n;
    bytes -= n;
  }
  return VXE_OK;
}

// World writes (chunk data, metas, grid, clipmap texels) are ordered after
// every pass already enqueued on the compute stream and the lanes, and before
// every pass enqueued later (which waits for upload_done): a frame in flight
// reads the world as it was when the frame was enqueued, like a queue write
// between two submissions in the reference.  Nothing here waits on the host.
vxe_status upload_after_readers(vxe_ctx* c) {
  cudaStream_t streams[1 + VXE_BATCH_LANES];
  streams[0] = c->compute;
  for (int l = 0; l < VXE_BATCH_LANES; ++l) streams[1 + l] = c->lanes[l].stream;
  for (int k = 0; k < 1 + VXE_BATCH_LANES; ++k) {
    if (!streams[k]) continue;
    if (!c->rd_ev[k]) CK(cudaEventCreateWithFlags(&c->rd_ev[k], cudaEventDisableTiming));
    CK(cudaEventRecord(c->rd_ev[k], streams[k]));
    CK(cudaStreamWaitEvent(c->upload, c->rd_ev[k], 0));
  }
  return VXE_OK;
}

}  // namespace

namespace {
// After chunk records of `slots` were written on the upload stream: their
// grass cell records and light flags are refreshed on the same stream and
// the next pass on any stream waits for all of it.
vxe_status chunks_written(vxe_ctx* c, std::vector<uint32_t>& slots) {
  std::sort(slots.begin(), slots.end());
  slots.erase(std::unique(slots.begin(), slots.end()), slots.end());
  vxe_status st = grass_table_refresh(c, slots);
  if (st != VXE_OK) return st;
  for (size_t i = 0; i < slots.size();) {  // one launch per run of consecutive slots
    size_t j = i + 1;
    while (j < slots.size() && slots[j] == slots[j - 1] + 1) ++j;
    if ((st = slot_lights_refresh(c, slots[i], (uint32_t)(j - i))) != VXE_OK) return st;
    i = j;
  }
  CK(cudaEventRecord(c->upload_done, c->upload));
  c->upload_pending = true;
  c->upload_recorded = true;
  return VXE_OK;
}
}  // namespace

extern "C" {

vxe_status vxe_upload_chunks(vxe_ctx* c, const vxe_chunk_upload* ups, uint32_t n) {
  if (!c || (n && !ups)) return fail(c, VXE_ERR_INVALID_ARG, "null uploads");
  cudaSetDevice(c->device);
  const bool silent = (c->flags & VXE_FLAG_SILENT_CAPACITY_SKIP) != 0;
  if (!(c->flags & VXE_FLAG_UPLOADS_UNORDERED)) {
    vxe_status ws = upload_after_readers(c);
    if (ws != VXE_OK) return ws;
  }
  for (uint32_t i = 0; i < n; ++i) {
    const vxe_chunk_upload& u = ups[i];
    const uint64_t mb = (uint64_t)u.meta.macro_base, cb = (uint64_t)u.meta.colinfo_base;
    const bool fits = u.slot < c->cfg.chunk_capacity && (uint64_t)u.node_base + u.node_count <= c->cfg.node_capacity &&
                      mb + VXE_MACRO_WORDS_PER_CHUNK <= (uint64_t)c->cfg.chunk_capacity * VXE_MACRO_WORDS_PER_CHUNK &&
                      cb + VXE_COLINFO_WORDS_PER_CHUNK <= (uint64_t)c->cfg.chunk_capacity * VXE_COLINFO_WORDS_PER_CHUNK &&
                      u.meta.node_base == u.node_base;
    if (!fits) {
      if (silent) continue;
      return fail(c, VXE_ERR_CAPACITY, "upload %u (slot %u, node_base %u, count %u) exceeds capacity", i, u.slot,
                  u.node_base, u.node_count);
    }
    if (u.node_count && (!u.nodes || !u.ropes)) return fail(c, VXE_ERR_INVALID_ARG, "upload %u has no node data", i);
    vxe_status rs;
    if ((rs = ring_copy(c, (char*)c->metas.p + (size_t)u.slot * 48, &u.meta, 48)) != VXE_OK) return rs;
    if (u.node_count) {
      if ((rs = ring_copy(c, (char*)c->nodes.p + (size_t)u.node_base * 16, u.nodes, (size_t)u.node_count * 16)) !=
          VXE_OK)
        return rs;
      if ((rs = ring_copy(c, (char*)c->ropes.p + (size_t)u.node_base * 32, u.ropes, (size_t)u.node_count * 32)) !=
          VXE_OK)
        return rs;
    }
    if (u.macro_words &&
        (rs = ring_copy(c, (char*)c->macro.p + mb * 4, u.macro_words, VXE_MACRO_WORDS_PER_CHUNK * 4)) != VXE_OK)
      return rs;
    if (u.colinfo_words &&
        (rs = ring_copy(c, (char*)c->colinfo.p + cb * 4, u.colinfo_words, VXE_COLINFO_WORDS_PER_CHUNK * 4)) != VXE_OK)
      return rs;
  }
  std::vector<uint32_t> slots;
  slots.reserve(n);
  for (uint32_t i = 0; i < n; ++i)
    if (ups[i].slot < c->cfg.chunk_capacity) slots.push_back(ups[i].slot);
  return chunks_written(c, slots);
}

vxe_status vxe_write_meta(vxe_ctx* c, uint32_t first, const vxe_chunk_meta* metas, uint32_t n) {
  if (!c || (n && !metas)) return fail(c, VXE_ERR_INVALID_ARG, "null metas");
  if ((uint64_t)first + n > c->cfg.chunk_capacity) return fail(c, VXE_ERR_CAPACITY, "meta run exceeds capacity");
  cudaSetDevice(c->device);
  vxe_status ws = upload_after_readers(c);
  if (ws != VXE_OK) return ws;
  if (n && (ws = ring_copy(c, (char*)c->metas.p + (size_t)first * 48, metas, (size_t)n * 48)) != VXE_OK) return ws;
  if ((ws = slot_lights_refresh(c, first, n)) != VXE_OK) return ws;
  // a slot's records follow its meta (origin, colinfo base)
  if (n && c->gt.valid) {
    c->gt.list_valid = false;  // the next wind change rebuilds every column
    if (c->gt.built_recorded) CK(cudaStreamWaitEvent(c->upload, c->gt.built, 0));
    const uint32_t hi = std::min(first + n, c->gt.chunk_count);
    if (hi > first) {
      vxe_status gst = grass_table_fill(c, c->upload, c->gt.cam, first, hi - first);
      if (gst != VXE_OK) return gst;
    }
  }
  CK(cudaEventRecord(c->upload_done, c->upload));
  c->upload_pending = true;
  c->upload_recorded = true;
  return VXE_OK;
}

vxe_status vxe_write_grid(vxe_ctx* c, const uint32_t* grid, uint32_t n) {
  if (!c || (n && !grid)) return fail(c, VXE_ERR_INVALID_ARG, "null grid");
  if (n > c->cfg.grid_capacity) return fail(c, VXE_ERR_CAPACITY, "grid of %u cells exceeds capacity %u", n, c->cfg.grid_capacity);
  cudaSetDevice(c->device);
  vxe_status ws = upload_after_readers(c);
  if (ws != VXE_OK) return ws;
  if (n && (ws = ring_copy(c, c->grid.p, grid, (size_t)n * 4)) != VXE_OK) return ws;
  CK(cudaEventRecord(c->upload_done, c->upload));
  c->upload_pending = true;
  c->upload_recorded = true;
  return VXE_OK;
}

vxe_status vxe_write_camera(vxe_ctx* c, const vxe_camera_gpu* cam) {
  if (!c || !cam) return fail(c, VXE_ERR_INVALID_ARG, "null camera");
  c->cam = *cam;
  return VXE_OK;
}

}  // extern "C"

namespace {

// The texels of up to VXE_CLIP_PATCHES_MAX clipmap patches: patch k covers
// texels [first[k], first[k + 1]) of the launch, row-major in its rectangle.
struct ClipPlan {
  vxe_world_params world;
  float* tex;
  uint32_t res, n;
  uint32_t first[VXE_CLIP_PATCHES_MAX + 1];
  vxe_clip_patch_geom g[VXE_CLIP_PATCHES_MAX];
};

__global__ void __launch_bounds__(256) k_clip_patches(const __grid_constant__ ClipPlan P) {
  const uint32_t total = P.first[P.n];
  for (uint32_t t = blockIdx.x * 256u + threadIdx.x; t < total; t += gridDim.x * 256u) {
    uint32_t k = 0;
    while (k + 1u < P.n && t >= P.first[k + 1u]) ++k;
    const vxe_clip_patch_geom& g = P.g[k];
    const uint32_t i = t - P.first[k], x = i % g.w, z = i / g.w;
    // Patches are uploaded in order and a later one may cover the same
    // storage texel (an x strip and a z strip of one level meet at a corner):
    // the last one covering it writes it.
    const uint32_t sx = g.x + x, sz = g.y + z;
    bool later = false;
    for (uint32_t j = k + 1u; j < P.n && !later; ++j) {
      const vxe_clip_patch_geom& h = P.g[j];
      later = h.level == g.level && sx >= h.x && sx < h.x + h.w && sz >= h.y && sz < h.y + h.h;
    }
    if (later) continue;
    // the texel centre as clipmap.rs emits it
    const float wz = g.oz_m + ((float)(g.lz0 + z) + 0.5f) * g.cell_m;
    const float wx = g.ox_m + ((float)(g.lx0 + x) + 0.5f) * g.cell_m;
    P.tex[((size_t)g.level * P.res + sz) * P.res + sx] = vxe::terrain::clip_sample(P.world, wx, wz);
  }
}

}  // namespace

extern "C" {

vxe_status vxe_clipmap_update_device(vxe_ctx* c, vxe_clipmap_state* s, float cam_x, float cam_z) {
  if (!c || !s) return fail(c, VXE_ERR_INVALID_ARG, "null clipmap arguments");
  cudaSetDevice(c->device);
  ClipPlan P;
  std::memset(&P, 0, sizeof P);
  vxe_clipmap_gpu params;
  const vxe_clip_patch_geom* geoms = nullptr;
  uint32_t n = 0;
  vxe_status st = vxe_clipmap_plan(s, cam_x, cam_z, &params, &geoms, &n, &P.world);
  if (st != VXE_OK) return fail(c, st, "vxe_clipmap_plan failed");
  if (params.levels > c->cfg.clip_levels || (params.levels != 0 && params.res != c->cfg.clip_res))
    return fail(c, VXE_ERR_CAPACITY, "clipmap %u x %u^2 does not fit the context's %u x %u^2", params.levels,
                params.res, c->cfg.clip_levels, c->cfg.clip_res);
  if (n > VXE_CLIP_PATCHES_MAX) return fail(c, VXE_ERR_CAPACITY, "%u clipmap patches > %u", n, VXE_CLIP_PATCHES_MAX);
  P.tex = (float*)c->clip_tex.p;
  P.res = c->cfg.clip_res;
  P.n = n;
  uint64_t total = 0;
  for (uint32_t k = 0; k < n; ++k) {
    P.g[k] = geoms[k];
    P.first[k] = (uint32_t)total;
    total += (uint64_t)geoms[k].w * geoms[k].h;
  }
  P.first[n] = (uint32_t)total;
  if ((st = upload_after_readers(c)) != VXE_OK) return st;
  if (total) {
    const unsigned grid = (unsigned)std::min<uint64_t>((total + 255) / 256, (uint64_t)c->shade_wave);
    k_clip_patches<<<grid, 256, 0, c->upload>>>(P);
    CK(cudaGetLastError());
  }
  c->clip = params;
  CK(cudaEventRecord(c->upload_done, c->upload));
  c->upload_pending = true;
  c->upload_recorded = true;
  return VXE_OK;
}

vxe_status vxe_read_clipmap(vxe_ctx* c, float* host, size_t bytes) {
  if (!c || !host) return fail(c, VXE_ERR_INVALID_ARG, "null clipmap read arguments");
  if (bytes != c->clip_tex.bytes) return fail(c, VXE_ERR_INVALID_ARG, "clipmap is %zu bytes, got %zu", c->clip_tex.bytes, bytes);
  cudaSetDevice(c->device);
  CK(cudaStreamSynchronize(c->upload));
  if (bytes) CK(cudaMemcpy(host, c->clip_tex.p, bytes, cudaMemcpyDeviceToHost));
  return VXE_OK;
}

vxe_status vxe_write_clipmap(vxe_ctx* c, const vxe_clipmap_gpu* params, const vxe_clip_patch* patches, uint32_t n) {
  if (!c || !params || (n && !patches)) return fail(c, VXE_ERR_INVALID_ARG, "null clipmap arguments");
  cudaSetDevice(c->device);
  const uint32_t res = c->cfg.clip_res;
  for (uint32_t i = 0; i < n; ++i) {
    const vxe_clip_patch& p = patches[i];
    if (p.level >= c->cfg.clip_levels || (uint64_t)p.x + p.w > res || (uint64_t)p.y + p.h > res || !p.data)
      return fail(c, VXE_ERR_CAPACITY, "clip patch %u out of range", i);
  }
  vxe_status ws = upload_after_readers(c);
  if (ws != VXE_OK) return ws;
  for (uint32_t i = 0; i < n; ++i) {
    const vxe_clip_patch& p = patches[i];
    if (p.w == 0 || p.h == 0) continue;
    char* dst = (char*)c->clip_tex.p + (((size_t)p.level * res + p.y) * res + p.x) * 4;
    CK(cudaMemcpy2DAsync(dst, (size_t)res * 4, p.data, (size_t)p.w * 4, (size_t)p.w * 4, p.h, cudaMemcpyHostToDevice,
                         c->upload));
  }
  c->clip = *params;
  CK(cudaEventRecord(c->upload_done, c->upload));
  c->upload_pending = true;
  c->upload_recorded = true;
  return VXE_OK;
}

vxe_status vxe_render_frame_async(vxe_ctx* c, vxe_frame_out* out) {
  if (!c) return VXE_ERR_INVALID_ARG;
  cudaSetDevice(c->device);
  vxe_status st = launch_frame(c, true);
  if (st != VXE_OK) return st;
  frame_out(c, out);
  return VXE_OK;
}

vxe_status vxe_render_frame(vxe_ctx* c, vxe_frame_out* out) {
  vxe_status st = vxe_render_frame_async(c, out);
  if (st != VXE_OK) return st;
  CK(cudaStreamSynchronize(c->compute));
  uint32_t word = 0;
  CK(cudaMemcpy(&word, c->errword.p, 4, cudaMemcpyDeviceToHost));
  if (word) return fail(c, VXE_ERR_BOUNDS, "device bounds check tripped (error word 0x%x)", word);
  return VXE_OK;
}

vxe_status vxe_render_frame_graph(vxe_ctx* c, vxe_frame_out* out) {
  if (!c) return VXE_ERR_INVALID_ARG;
  cudaSetDevice(c->device);
  vxe_status st = launch_frame_graph(c, c->fr, c->cam, c->compute, 0);
  if (st != VXE_OK) return st;
  frame_out(c, out);
  CK(cudaStreamSynchronize(c->compute));
  uint32_t word = 0;
  CK(cudaMemcpy(&word, c->errword.p, 4, cudaMemcpyDeviceToHost));
  if (word) return fail(c, VXE_ERR_BOUNDS, "device bounds check tripped (error word 0x%x)", word);
  return VXE_OK;
}

vxe_status vxe_synchronize(vxe_ctx* c) {
  if (!c) return VXE_ERR_INVALID_ARG;
  cudaSetDevice(c->device);
  CK(cudaStreamSynchronize(c->compute));
  CK(cudaStreamSynchronize(c->upload));
  if (c->copy) CK(cudaStreamSynchronize(c->copy));
  return VXE_OK;
}

vxe_status vxe_get_timings(vxe_ctx* c, vxe_timings* t) {
  if (!c || !t) return VXE_ERR_INVALID_ARG;
  std::memset(t, 0, sizeof *t);
  if (!c->fr.timed) return VXE_OK;
  cudaSetDevice(c->device);
  CK(cudaEventSynchronize(c->fr.ev[6]));
  float ms[6];
  for (int i = 0; i < 6; ++i) CK(cudaEventElapsedTime(&ms[i], c->fr.ev[i], c->fr.ev[i + 1]));
  t->grass_cells = ms[0];
  t->tiles = (double)ms[0] + ms[1];
  t->primary_trace = c->fr.timed_trace ? ms[2] : 0.0;
  if (c->fr.timed_trace) {
    float mk = 0.0f;
    CK(cudaEventElapsedTime(&mk, c->fr.ev[7], c->fr.ev[8]));
    t->trace_kernel = mk;
  }
  t->primary = (double)ms[2] + ms[3];
  t->godray = ms[4];
  t->composite = ms[5];
  t->total = (double)ms[0] + ms[1] + ms[2] + ms[3] + ms[4] + ms[5];
  return VXE_OK;
}

vxe_status vxe_image_size(const vxe_ctx* c, vxe_image im, size_t* bytes) {
  if (!c || !bytes) return VXE_ERR_INVALID_ARG;
  const int i = map_image(c->fr, im);
  if (i < 0) return VXE_ERR_INVALID_ARG;
  *bytes = c->fr.img[i].bytes;
  return VXE_OK;
}

vxe_status vxe_read_image(vxe_ctx* c, vxe_image im, void* host, size_t bytes) {
  if (!c || !host) return VXE_ERR_INVALID_ARG;
  const int i = map_image(c->fr, im);
  if (i < 0 || !c->fr.img[i].p) return fail(c, VXE_ERR_INVALID_ARG, "image %d not available", (int)im);
  if (bytes != c->fr.img[i].bytes) return fail(c, VXE_ERR_INVALID_ARG, "image %d is %zu bytes, got %zu", (int)im, c->fr.img[i].bytes, bytes);
  cudaSetDevice(c->device);
  CK(cudaStreamSynchronize(c->compute));
  CK(cudaMemcpy(host, c->fr.img[i].p, bytes, cudaMemcpyDeviceToHost));
  return VXE_OK;
}

vxe_status vxe_read_image_async(vxe_ctx* c, vxe_image im, void* host, size_t bytes, uint64_t* ticket) {
  if (!c || !host) return VXE_ERR_INVALID_ARG;
  const int i = map_image(c->fr, im);
  if (i < 0 || !c->fr.img[i].p) return fail(c, VXE_ERR_INVALID_ARG, "image %d not available", (int)im);
  if (bytes != c->fr.img[i].bytes) return fail(c, VXE_ERR_INVALID_ARG, "image %d is %zu bytes, got %zu", (int)im, c->fr.img[i].bytes, bytes);
  cudaSetDevice(c->device);
  if (!c->copy) CK(cudaStreamCreateWithFlags(&c->copy, cudaStreamNonBlocking));
  for (auto& e : c->copy_ev)
    if (!e) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  cudaEvent_t& slot = c->copy_ev[c->copy_seq % 8];
  CK(cudaEventRecord(slot, c->compute));  // after the frame work queued so far
  CK(cudaStreamWaitEvent(c->copy, slot, 0));
  CK(cudaMemcpyAsync(host, c->fr.img[i].p, bytes, cudaMemcpyDeviceToHost, c->copy));
  CK(cudaEventRecord(slot, c->copy));
  if (i == IMG_OUTPUT) {
    c->out_ev = slot;
    c->out_pending = true;
  } else {
    c->any_ev = slot;
    c->any_pending = true;
  }
  if (ticket) *ticket = c->copy_seq;
  ++c->copy_seq;
  return VXE_OK;
}

vxe_status vxe_read_image_wait(vxe_ctx* c, uint64_t ticket) {
  if (!c) return VXE_ERR_INVALID_ARG;
  if (ticket >= c->copy_seq) return fail(c, VXE_ERR_INVALID_ARG, "no image read %llu queued", (unsigned long long)ticket);
  cudaSetDevice(c->device);
  // copies run in order on one stream: a slot re-recorded by a later copy
  // completes after this one
  CK(cudaEventSynchronize(c->copy_ev[ticket % 8]));
  return VXE_OK;
}

vxe_status vxe_write_image(vxe_ctx* c, vxe_image im, const void* host, size_t bytes) {
  if (!c || !host) return VXE_ERR_INVALID_ARG;
  const int i = map_image(c->fr, im);
  if (i < 0 || !c->fr.img[i].p) return fail(c, VXE_ERR_INVALID_ARG, "image %d not available", (int)im);
  if (bytes != c->fr.img[i].bytes) return fail(c, VXE_ERR_INVALID_ARG, "image %d is %zu bytes, got %zu", (int)im, c->fr.img[i].bytes, bytes);
  cudaSetDevice(c->device);
  CK(cudaStreamSynchronize(c->compute));
  if (c->copy) CK(cudaStreamSynchronize(c->copy));  // an asynchronous read of this image may be in flight
  CK(cudaMemcpy(c->fr.img[i].p, host, bytes, cudaMemcpyHostToDevice));
  CK(cudaStreamSynchronize(cudaStreamLegacy));  // a pageable copy may still be landing
  return VXE_OK;
}

vxe_status vxe_read_error_word(vxe_ctx* c, uint32_t* word) {
  if (!c || !word) return VXE_ERR_INVALID_ARG;
  cudaSetDevice(c->device);
  CK(cudaStreamSynchronize(c->compute));
  CK(cudaStreamSynchronize(c->upload));  // resident builds report here too
  CK(cudaMemcpy(word, c->errword.p, 4, cudaMemcpyDeviceToHost));
  CK(fill_sync(c->errword.p, 0, 4));
  return VXE_OK;
}

vxe_status vxe_set_record_limits(vxe_ctx* c, uint32_t probe_records, uint32_t slab_tasks) {
  if (!c) return VXE_ERR_INVALID_ARG;
  c->probe_limit = probe_records;
  c->slab_limit = slab_tasks;
  return VXE_OK;
}

vxe_status vxe_get_frame_stats(vxe_ctx* c, vxe_frame_stats* out) {
  if (!c || !out) return VXE_ERR_INVALID_ARG;
  std::memset(out, 0, sizeof *out);
  if (!c->fr.img[IMG_QCOUNT].p || (c->flags & VXE_FLAG_PRIMARY_MEGAKERNEL)) return VXE_OK;
  cudaSetDevice(c->device);
  CK(cudaStreamSynchronize(c->compute));
  uint32_t q[16];
  CK(cudaMemcpy(q, c->fr.img[IMG_QCOUNT].p, sizeof q, cudaMemcpyDeviceToHost));
  out->voxel_pixels = q[0];
  out->far_pixels = q[1];
  out->probes = q[4];
  out->pending_pixels = q[5];
  out->slab_tasks = q[6];
  out->slab_hits = q[7];
  out->rewalk_pixels = q[9];
  out->full_trace_pixels = q[10];
  return VXE_OK;
}

vxe_status vxe_reset_profile_counts(vxe_ctx* c) {
  if (!c) return VXE_ERR_INVALID_ARG;
  cudaSetDevice(c->device);
  CK(cudaMemsetAsync(c->profile.p, 0, c->profile.bytes, c->compute));  // after the frames enqueued so far
  return VXE_OK;
}

vxe_status vxe_read_profile_counts(vxe_ctx* c, uint32_t counts[VXE_PROFILE_COUNT]) {
  if (!c || !counts) return VXE_ERR_INVALID_ARG;
  cudaSetDevice(c->device);
  CK(cudaStreamSynchronize(c->compute));
  CK(cudaMemcpy(counts, c->profile.p, VXE_PROFILE_COUNT * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  return VXE_OK;
}

static void fill_query_args(const vxe_ctx* c, QueryArgs& Q) {
  std::memset(&Q, 0, sizeof Q);
  Q.cam = c->cam;
  Q.clip = c->clip;
  Q.nodes = (const uint4*)c->nodes.p;
  Q.nodes_n = c->cfg.node_capacity;
  Q.ropes = (const uint32_t*)c->ropes.p;
  Q.ropes_n = c->cfg.node_capacity;
  Q.metas = (const uint4*)c->metas.p;
  Q.metas_n = c->cfg.chunk_capacity;
  Q.grid = (const uint32_t*)c->grid.p;
  Q.grid_n = c->cfg.grid_capacity;
  Q.macro = (const uint32_t*)c->macro.p;
  Q.macro_n = (uint64_t)c->cfg.chunk_capacity * VXE_MACRO_WORDS_PER_CHUNK;
  Q.colinfo = (const uint32_t*)c->colinfo.p;
  Q.colinfo_n = (uint64_t)c->cfg.chunk_capacity * VXE_COLINFO_WORDS_PER_CHUNK;
  Q.err = (uint32_t*)c->errword.p;
}

}  // extern "C"

namespace {

__global__ void __launch_bounds__(256) k_solid_voxels(const __grid_constant__ vxe::dev::FrameArgs A, const int32_t* vox,
                                                      uint32_t n, vxe_world_params wp, uint32_t has_world,
                                                      uint8_t* out) {
  using namespace vxe::dev;
  const Scene s = make_scene(A, false);
  const int32_t cs = (int32_t)s.cam->chunk_size;
  auto fdiv = [cs](int32_t a) { return a >= 0 ? a / cs : -((-a + cs - 1) / cs); };
  for (uint32_t i = blockIdx.x * 256u + threadIdx.x; i < n; i += gridDim.x * 256u) {
    const int32_t vx = vox[3u * i], vy = vox[3u * i + 1u], vz = vox[3u * i + 2u];
    const int32_t cx = fdiv(vx), cy = fdiv(vy), cz = fdiv(vz);
    const uint32_t slot = grid_lookup_slot(s, cx, cy, cz);
    uint8_t solid = 0u;
    if (slot != INVALID && slot < s.cam->chunk_count) {
      const Meta m = meta_at(s, slot);
      const uint32_t lx = (uint32_t)(vx - cx * cs), lz = (uint32_t)(vz - cz * cs);
      const int32_t ly = vy - cy * cs;
      const uint32_t top = colinfo_entry_u16(s, m.colinfo_base, lx, lz) & 0xFFu;
      solid = (top != 255u && ly <= (int32_t)top) ? 1u : 0u;
    } else if (has_world) {
      solid = vy <= vxe::terrain::ground(wp, vx, vz) ? 1u : 0u;
    }
    out[i] = solid;
  }
}

}  // namespace

namespace {
// Dense-slot moves in order, one CTA: a slot's meta record (its macro and
// colinfo bases follow the slot), 16 macro words and 2048 colinfo words.
__global__ void __launch_bounds__(1024) k_move_slots(const uint2* moves, uint32_t n, uint4* metas, uint32_t* macro,
                                                    uint32_t* colinfo) {
  const uint32_t t = threadIdx.x;
  for (uint32_t m = 0; m < n; ++m) {
    const uint2 mv = moves[m];
    if (t < VXE_MACRO_WORDS_PER_CHUNK)
      macro[(size_t)mv.y * VXE_MACRO_WORDS_PER_CHUNK + t] = macro[(size_t)mv.x * VXE_MACRO_WORDS_PER_CHUNK + t];
    for (uint32_t i = t; i < VXE_COLINFO_WORDS_PER_CHUNK; i += 1024u)
      colinfo[(size_t)mv.y * VXE_COLINFO_WORDS_PER_CHUNK + i] = colinfo[(size_t)mv.x * VXE_COLINFO_WORDS_PER_CHUNK + i];
    if (t < 3u) {
      uint4 w = metas[(size_t)mv.x * 3u + t];
      if (t == 1u) {
        w.z = mv.y * VXE_MACRO_WORDS_PER_CHUNK;
        w.w = mv.y * VXE_COLINFO_WORDS_PER_CHUNK;
      }
      metas[(size_t)mv.y * 3u + t] = w;
    }
    __syncthreads();  // a later move may read this one's destination
  }
}
}  // namespace

namespace {
// The cave test of the seeded world, s / 1.5 > threshold with s = n1 + 0.5 n2
// in [0, 1.5), is monotone in s: returns the least binary64 s >= 0 that
// passes (bisection over the ordered bit patterns of [0, 2]), +inf when none.
double cave_s_min(double thr) {
  auto pass = [thr](double v) { return v / 1.5 > thr; };
  if (pass(0.0)) return 0.0;
  if (!pass(2.0)) return INFINITY;
  uint64_t lo, hi;
  const double zero = 0.0, two = 2.0;
  std::memcpy(&lo, &zero, 8);
  std::memcpy(&hi, &two, 8);
  while (hi - lo > 1) {
    const uint64_t mid = lo + (hi - lo) / 2;
    double v;
    std::memcpy(&v, &mid, 8);
    if (pass(v)) hi = mid;
    else lo = mid;
  }
  double r;
  std::memcpy(&r, &hi, 8);
  return r;
}
}  // namespace

namespace {
// Scratch, events and the two builder kernels on the world-write stream.
vxe_status build_launch(vxe_ctx* c, vxe::build::BuildArgs& B, uint32_t n) {
  namespace vb = vxe::build;
  // per chunk: materials, level-1 ground minima, level-5 states and child
  // offsets, solid counts of the 16 column blocks
  constexpr size_t kPerChunk = (size_t)vb::kVoxels + 1024 * 4 + (size_t)vb::kCells5 * 8 + 16 * 4;
  const size_t need = kPerChunk * n;
  if (c->build_scratch.bytes < need) {
    vxe_status st = alloc(c, c->build_scratch, need);
    if (st != VXE_OK) return st;
  }
  if (!c->build_ev[0]) {  // first build on this context: events, and the octree kernel's staging size
    for (auto& e : c->build_ev) CK(cudaEventCreate(&e));
    CK(cudaFuncSetAttribute(vb::k_build_svo, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vb::kStageBytes));
  }
  B.cave_smin = cave_s_min((double)B.wp.cave_threshold);
  B.n = n;
  char* base = (char*)c->build_scratch.p;
  B.mat = (uint8_t*)base;
  base += (size_t)vb::kVoxels * n;
  B.st5 = (uint32_t*)base;
  base += (size_t)vb::kCells5 * 4 * n;
  B.kb5 = (uint32_t*)base;
  base += (size_t)vb::kCells5 * 4 * n;
  B.mip1 = (int32_t*)base;
  base += (size_t)1024 * 4 * n;
  B.solid_part = (uint32_t*)base;
  cudaStream_t st = c->upload;
  CK(cudaEventRecord(c->build_ev[0], st));
  vb::k_build_columns<<<n * 16u, 256, 0, st>>>(B);
  CK(cudaGetLastError());
  CK(cudaEventRecord(c->build_ev[1], st));
  vb::k_build_svo<<<n, vb::SVO_THREADS, vb::kStageBytes, st>>>(B);
  CK(cudaGetLastError());
  CK(cudaEventRecord(c->build_ev[2], st));
  c->build_timed = true;
  return VXE_OK;
}
}  // namespace

extern "C" {

vxe_status vxe_solid_voxels_device(vxe_ctx* c, const int32_t* d_vox, uint32_t n, const vxe_world_params* world,
                                   uint8_t* d_out) {
  if (!c || (n && (!d_vox || !d_out))) return fail(c, VXE_ERR_INVALID_ARG, "null solidity buffers");
  if (n == 0) return VXE_OK;
  if (c->cam.chunk_size != 64u) return fail(c, VXE_ERR_INVALID_ARG, "chunk_size must be 64 (colinfo layout)");
  cudaSetDevice(c->device);
  if (c->upload_recorded) CK(cudaStreamWaitEvent(c->compute, c->upload_done, 0));
  vxe::dev::FrameArgs A;
  fill_scene_args(c, A);
  vxe_world_params wp;
  std::memset(&wp, 0, sizeof wp);
  if (world) wp = *world;
  const unsigned grid = (unsigned)std::min<uint64_t>(((uint64_t)n + 255) / 256, (uint64_t)c->shade_wave);
  k_solid_voxels<<<grid, 256, 0, c->compute>>>(A, d_vox, n, wp, world ? 1u : 0u, d_out);
  CK(cudaGetLastError());
  return VXE_OK;
}

vxe_status vxe_build_chunks_device(vxe_ctx* c, const vxe_world_params* world, const int32_t* d_coords, uint32_t n,
                                   uint32_t node_cap, vxe_node* d_nodes, vxe_node_ropes* d_ropes, uint32_t* d_macro,
                                   uint32_t* d_colinfo, uint32_t* d_counts) {
  namespace vb = vxe::build;
  if (!c || !world) return fail(c, VXE_ERR_INVALID_ARG, "null builder arguments");
  if (n == 0) return VXE_OK;
  if (!d_coords || !d_macro || !d_colinfo || !d_counts || (node_cap && (!d_nodes || !d_ropes)))
    return fail(c, VXE_ERR_INVALID_ARG, "null builder buffers");
  if (n > VXE_BUILD_BATCH_MAX) return fail(c, VXE_ERR_CAPACITY, "%u chunks > %u per build call", n, VXE_BUILD_BATCH_MAX);
  if (node_cap > VXE_BUILD_NODE_CAP_MAX)
    return fail(c, VXE_ERR_INVALID_ARG, "node_cap %u > %u", node_cap, VXE_BUILD_NODE_CAP_MAX);
  cudaSetDevice(c->device);
  vb::BuildArgs B;
  std::memset(&B, 0, sizeof B);
  B.wp = *world;
  B.coords = d_coords;
  B.node_cap = node_cap;
  B.nodes = d_nodes;
  B.ropes = d_ropes;
  B.macro = d_macro;
  B.colinfo = d_colinfo;
  B.counts = d_counts;
  return build_launch(c, B, n);
}

vxe_status vxe_build_chunks_resident(vxe_ctx* c, const vxe_world_params* world, const vxe_build_place* places,
                                     uint32_t n) {
  namespace vb = vxe::build;
  if (!c || !world || (n && !places)) return fail(c, VXE_ERR_INVALID_ARG, "null resident build arguments");
  if (n == 0) return VXE_OK;
  if (n > VXE_BUILD_BATCH_MAX) return fail(c, VXE_ERR_CAPACITY, "%u chunks > %u per build call", n, VXE_BUILD_BATCH_MAX);
  std::vector<uint32_t> slots(n);
  std::vector<std::pair<uint64_t, uint64_t>> ranges(n);
  for (uint32_t i = 0; i < n; ++i) {
    const vxe_build_place& pl = places[i];
    if (pl.slot >= c->cfg.chunk_capacity || (uint64_t)pl.node_base + pl.node_count > c->cfg.node_capacity ||
        pl.node_count > VXE_BUILD_NODE_CAP_MAX)
      return fail(c, VXE_ERR_CAPACITY, "place %u (slot %u, node_base %u, count %u) exceeds capacity", i, pl.slot,
                  pl.node_base, pl.node_count);
    slots[i] = pl.slot;
    ranges[i] = {pl.node_base, (uint64_t)pl.node_base + pl.node_count};
  }
  std::vector<uint32_t> sorted = slots;
  std::sort(sorted.begin(), sorted.end());
  if (std::adjacent_find(sorted.begin(), sorted.end()) != sorted.end())
    return fail(c, VXE_ERR_INVALID_ARG, "two places share a slot");
  std::sort(ranges.begin(), ranges.end());
  for (uint32_t i = 1; i < n; ++i)
    if (ranges[i].first < ranges[i - 1].second) return fail(c, VXE_ERR_INVALID_ARG, "two places share arena nodes");
  cudaSetDevice(c->device);
  if (!(c->flags & VXE_FLAG_UPLOADS_UNORDERED)) {
    vxe_status ws = upload_after_readers(c);
    if (ws != VXE_OK) return ws;
  }
  const size_t pbytes = sizeof(vxe_build_place) * n;
  if (c->build_places.bytes < pbytes) {
    vxe_status st = alloc(c, c->build_places, sizeof(vxe_build_place) * VXE_BUILD_BATCH_MAX);
    if (st != VXE_OK) return st;
  }
  vxe_status st = ring_copy(c, c->build_places.p, places, pbytes);
  if (st != VXE_OK) return st;
  vb::BuildArgs B;
  std::memset(&B, 0, sizeof B);
  B.wp = *world;
  B.place = (const vxe_build_place*)c->build_places.p;
  B.nodes = (vxe_node*)c->nodes.p;
  B.ropes = (vxe_node_ropes*)c->ropes.p;
  B.macro = (uint32_t*)c->macro.p;
  B.colinfo = (uint32_t*)c->colinfo.p;
  B.metas = (vxe_chunk_meta*)c->metas.p;
  B.error_word = (uint32_t*)c->errword.p;
  if ((st = build_launch(c, B, n)) != VXE_OK) return st;
  return chunks_written(c, slots);
}

vxe_status vxe_move_slots(vxe_ctx* c, const vxe_slot_move* moves, uint32_t n) {
  if (!c || (n && !moves)) return fail(c, VXE_ERR_INVALID_ARG, "null slot moves");
  if (n == 0) return VXE_OK;
  if (n > VXE_MOVE_SLOTS_MAX) return fail(c, VXE_ERR_CAPACITY, "%u slot moves > %u per call", n, VXE_MOVE_SLOTS_MAX);
  std::vector<uint32_t> dst(n);
  for (uint32_t i = 0; i < n; ++i) {
    if (moves[i].from >= c->cfg.chunk_capacity || moves[i].to >= c->cfg.chunk_capacity)
      return fail(c, VXE_ERR_CAPACITY, "slot move %u (%u -> %u) outside %u slots", i, moves[i].from, moves[i].to,
                  c->cfg.chunk_capacity);
    dst[i] = moves[i].to;
  }
  cudaSetDevice(c->device);
  if (!(c->flags & VXE_FLAG_UPLOADS_UNORDERED)) {
    vxe_status ws = upload_after_readers(c);
    if (ws != VXE_OK) return ws;
  }
  if (c->move_buf.bytes < sizeof(vxe_slot_move) * n) {
    vxe_status st = alloc(c, c->move_buf, sizeof(vxe_slot_move) * VXE_MOVE_SLOTS_MAX);
    if (st != VXE_OK) return st;
  }
  vxe_status st = ring_copy(c, c->move_buf.p, moves, sizeof(vxe_slot_move) * n);
  if (st != VXE_OK) return st;
  k_move_slots<<<1, 1024, 0, c->upload>>>((const uint2*)c->move_buf.p, n, (uint4*)c->metas.p, (uint32_t*)c->macro.p,
                                          (uint32_t*)c->colinfo.p);
  CK(cudaGetLastError());
  return chunks_written(c, dst);
}

vxe_status vxe_get_build_timings(vxe_ctx* c, vxe_build_timings* t) {
  if (!c || !t) return fail(c, VXE_ERR_INVALID_ARG, "null build timings");
  std::memset(t, 0, sizeof *t);
  if (!c->build_timed) return VXE_OK;
  cudaSetDevice(c->device);
  CK(cudaEventSynchronize(c->build_ev[2]));
  float ms[2];
  for (int i = 0; i < 2; ++i) CK(cudaEventElapsedTime(&ms[i], c->build_ev[i], c->build_ev[i + 1]));
  t->columns = ms[0];
  t->svo = ms[1];
  return VXE_OK;
}

vxe_status vxe_trace_rays_device(vxe_ctx* c, const float* d_o, const float* d_d, uint32_t n, float tmax, vxe_hit* d_out) {
  if (!c || (n && (!d_o || !d_d || !d_out))) return fail(c, VXE_ERR_INVALID_ARG, "null ray buffers");
  if (n == 0) return VXE_OK;
  cudaSetDevice(c->device);
  if (c->upload_recorded) CK(cudaStreamWaitEvent(c->compute, c->upload_done, 0));
  QueryArgs Q;
  fill_query_args(c, Q);
  Q.origins = d_o;
  Q.dirs = d_d;
  Q.n = n;
  Q.tmax = tmax;
  Q.out = (uint4*)d_out;
  using namespace vxe::dev;
  k_query<<<(n + QUERY_THREADS - 1) / QUERY_THREADS, QUERY_THREADS, 0, c->compute>>>(Q);
  CK(cudaGetLastError());
  return VXE_OK;
}

vxe_status vxe_trace_rays(vxe_ctx* c, const float* o, const float* d, uint32_t n, float tmax, vxe_hit* out) {
  if (!c || (n && (!o || !d || !out))) return fail(c, VXE_ERR_INVALID_ARG, "null ray buffers");
  if (n == 0) return VXE_OK;
  cudaSetDevice(c->device);
  const size_t in_bytes = (size_t)n * 24, out_bytes = (size_t)n * sizeof(vxe_hit);
  vxe_status st;
  if (c->q_in.bytes < in_bytes && (st = alloc(c, c->q_in, in_bytes)) != VXE_OK) return st;
  if (c->q_out.bytes < out_bytes && (st = alloc(c, c->q_out, out_bytes)) != VXE_OK) return st;
  float* din = (float*)c->q_in.p;
  CK(cudaMemcpyAsync(din, o, (size_t)n * 12, cudaMemcpyHostToDevice, c->compute));
  CK(cudaMemcpyAsync(din + (size_t)n * 3, d, (size_t)n * 12, cudaMemcpyHostToDevice, c->compute));
  st = vxe_trace_rays_device(c, din, din + (size_t)n * 3, n, tmax, (vxe_hit*)c->q_out.p);
  if (st != VXE_OK) return st;
  CK(cudaMemcpyAsync(out, c->q_out.p, out_bytes, cudaMemcpyDeviceToHost, c->compute));
  CK(cudaStreamSynchronize(c->compute));
  return VXE_OK;
}

}  // extern "C"

namespace {

using vxe::dev::BatchArgs;
using vxe::dev::BatchHeader;
using vxe::dev::BatchReq;

constexpr size_t kStageHdr = 0, kStageReqs = 64,
                 kStageCams = kStageReqs + (size_t)VXE_MAX_BATCH_REQUESTS * sizeof(BatchReq),
                 kStageBytes = kStageCams + (size_t)(VXE_MAX_BATCH_REQUESTS + 1) * sizeof(vxe_camera_gpu);

// Stored probes and slab tasks per viewport ray of a batch; rays past the
// budget walk again with inline probes.
constexpr uint32_t kBatchProbesPerRay = 4, kBatchSlabsPerRay = 2;

vxe_status lane_resources(vxe_ctx* c, BatchLane& L, uint32_t tiles, uint32_t vp_rays, uint32_t q_rays) {
  vxe_status st;
  if (!L.stage) {
    if (cudaMallocHost(&L.stage, kStageBytes) != cudaSuccess) return fail(c, VXE_ERR_OOM, "pinned staging");
    CK(cudaStreamCreateWithFlags(&L.stream, cudaStreamNonBlocking));
    if ((st = alloc_on(c, L.hdr, sizeof(BatchHeader), L.stream)) != VXE_OK) return st;
    if ((st = alloc_on(c, L.reqs, (size_t)VXE_MAX_BATCH_REQUESTS * sizeof(BatchReq), L.stream)) != VXE_OK) return st;
    if ((st = alloc_on(c, L.cams, (size_t)(VXE_MAX_BATCH_REQUESTS + 1) * sizeof(vxe_camera_gpu), L.stream)) != VXE_OK) return st;
    if ((st = alloc_on(c, L.head, 16, L.stream)) != VXE_OK) return st;
    for (auto& e : L.ev) CK(cudaEventCreate(&e));
  }
  if (c->b_trace_grid == 0) {
    // Persistent grids: every SM filled to the kernels' occupancy limit.
    int sms = 0, tb = 0, lb = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
    int tb0 = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&tb, vxe::dev::k_batch_trace<true>, vxe::dev::BATCH_THREADS, 0));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&tb0, vxe::dev::k_batch_trace<false>, vxe::dev::BATCH_THREADS, 0));
    tb = std::min(tb, tb0);  // the persistent grid fills every SM for either instantiation
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&lb, vxe::dev::k_batch_tiles, vxe::dev::TILE_THREADS, 0));
    c->b_trace_grid = sms * std::max(tb, 1);
    c->b_tile_grid = sms * std::max(lb, 1);
  }
  if (vp_rays > L.ray_cap) {
    const uint64_t cap = std::min<uint64_t>(std::max<uint64_t>((uint64_t)vp_rays + vp_rays / 2, 1u << 16),
                                            0x3FFFFFFFu / kBatchProbesPerRay);
    if ((st = alloc_on(c, L.px_first, cap * 8, L.stream)) != VXE_OK) return st;
    if ((st = alloc_on(c, L.px_mask, cap * 8, L.stream)) != VXE_OK) return st;
    if ((st = alloc_on(c, L.px_probe, cap * 8, L.stream)) != VXE_OK) return st;
    if ((st = alloc_on(c, L.px_task, cap * 4, L.stream)) != VXE_OK) return st;
    if ((st = alloc_on(c, L.px_hit, cap * 64, L.stream)) != VXE_OK) return st;
    if ((st = alloc_on(c, L.q_pending, cap * 4, L.stream)) != VXE_OK) return st;
    if ((st = alloc_on(c, L.q_refine, cap * 4, L.stream)) != VXE_OK) return st;
    if ((st = alloc_on(c, L.q_far, cap * 4, L.stream)) != VXE_OK) return st;
    if ((st = alloc_on(c, L.probe_recs, cap * kBatchProbesPerRay * sizeof(vxe::dev::ProbeRec), L.stream)) != VXE_OK) return st;
    if ((st = alloc_on(c, L.slab_tasks, cap * kBatchSlabsPerRay * 16, L.stream)) != VXE_OK) return st;
    if ((st = alloc_on(c, L.slab_res, cap * kBatchSlabsPerRay * 16, L.stream)) != VXE_OK) return st;
    if ((st = alloc_on(c, L.slab_hits, cap * kBatchSlabsPerRay * 4, L.stream)) != VXE_OK) return st;
    if (!L.dcount.p && (st = alloc_on(c, L.dcount, 32, L.stream)) != VXE_OK) return st;
    L.ray_cap = (uint32_t)cap;
    if (L.graph) {  // the captured launches hold the old pointers
      cudaGraphExecDestroy(L.graph);
      L.graph = nullptr;
    }
  }
  if (q_rays > L.q_cap) {
    const uint64_t cap = std::max<uint64_t>((uint64_t)q_rays + q_rays / 2, 1u << 16);
    if ((st = alloc_on(c, L.q_keys, cap * 4, L.stream)) != VXE_OK) return st;
    if ((st = alloc_on(c, L.q_perm, cap * 4, L.stream)) != VXE_OK) return st;
    if (!L.bin_count.p && (st = alloc_on(c, L.bin_count, (size_t)std::max(c->cfg.grid_capacity, 1u) * 8u * 4u, L.stream)) != VXE_OK)
      return st;
    L.q_cap = (uint32_t)cap;
    if (L.graph) {
      cudaGraphExecDestroy(L.graph);
      L.graph = nullptr;
    }
  }
  if ((size_t)tiles * 4 > L.tile_count.bytes) {
    // grow by 1.5x so a stream of slightly larger batches does not reallocate every time
    const size_t cap = std::max<size_t>((size_t)tiles + tiles / 2, 4096);
    if ((st = alloc_on(c, L.tile_count, cap * 4, L.stream)) != VXE_OK) return st;
    if ((st = alloc_on(c, L.tile_slots, cap * 4 * VXE_PRIMARY_MAX_TILE_CHUNKS, L.stream)) != VXE_OK) return st;
    if (L.graph) {
      cudaGraphExecDestroy(L.graph);
      L.graph = nullptr;
    }
  }
  return VXE_OK;
}

BatchArgs batch_args(const vxe_ctx* c, const BatchLane& L) {
  BatchArgs B;
  std::memset(&B, 0, sizeof B);
  B.clip = c->clip;
  B.nodes = (const uint4*)c->nodes.p;
  B.nodes_n = c->cfg.node_capacity;
  B.ropes = (const uint32_t*)c->ropes.p;
  B.ropes_n = c->cfg.node_capacity;
  B.metas = (const uint4*)c->metas.p;
  B.metas_n = c->cfg.chunk_capacity;
  B.grid = (const uint32_t*)c->grid.p;
  B.grid_n = c->cfg.grid_capacity;
  B.macro = (const uint32_t*)c->macro.p;
  B.macro_n = (uint64_t)c->cfg.chunk_capacity * VXE_MACRO_WORDS_PER_CHUNK;
  B.colinfo = (const uint32_t*)c->colinfo.p;
  B.colinfo_n = (uint64_t)c->cfg.chunk_capacity * VXE_COLINFO_WORDS_PER_CHUNK;
  B.clip_tex = (const float*)c->clip_tex.p;
  B.clip_layers = c->cfg.clip_levels;
  B.clip_res = c->cfg.clip_res;
  B.err = (uint32_t*)c->errword.p;
  B.hdr = (const BatchHeader*)L.hdr.p;
  B.reqs = (const BatchReq*)L.reqs.p;
  B.cams = (const vxe_camera_gpu*)L.cams.p;
  B.tile_count = (uint32_t*)L.tile_count.p;
  B.tile_slots = (uint32_t*)L.tile_slots.p;
  B.head = (uint32_t*)L.head.p;
  B.probe_recs = (vxe::dev::ProbeRec*)L.probe_recs.p;
  B.probe_cap = L.ray_cap * kBatchProbesPerRay;
  if (c->probe_limit) B.probe_cap = std::min(B.probe_cap, c->probe_limit);
  B.slab_tasks = (uint4*)L.slab_tasks.p;
  B.slab_res = (float4*)L.slab_res.p;
  B.slab_hits = (uint32_t*)L.slab_hits.p;
  B.slab_cap = L.ray_cap * kBatchSlabsPerRay;
  if (c->slab_limit) B.slab_cap = std::min(B.slab_cap, c->slab_limit);
  B.ray_cap = L.ray_cap;
  B.px_first = (unsigned long long*)L.px_first.p;
  B.px_task = (uint32_t*)L.px_task.p;
  B.px_mask = (uint2*)L.px_mask.p;
  B.px_probe = (uint2*)L.px_probe.p;
  B.px_hit = (uint4*)L.px_hit.p;
  B.q_pending = (uint32_t*)L.q_pending.p;
  B.q_refine = (uint32_t*)L.q_refine.p;
  B.q_far = (uint32_t*)L.q_far.p;
  B.q_keys = (uint32_t*)L.q_keys.p;
  B.q_perm = (uint32_t*)L.q_perm.p;
  B.bin_count = (uint32_t*)L.bin_count.p;
  B.dcount = (uint32_t*)L.dcount.p;
  return B;
}

vxe_status launch_persistent(vxe_ctx* c, BatchLane& L, const BatchArgs& B, bool sorted) {
  using namespace vxe::dev;
  CK(cudaMemcpyAsync(L.hdr.p, (char*)L.stage + kStageHdr, sizeof(BatchHeader), cudaMemcpyHostToDevice, L.stream));
  CK(cudaMemcpyAsync(L.reqs.p, (char*)L.stage + kStageReqs, kStageCams - kStageReqs, cudaMemcpyHostToDevice,
                     L.stream));
  CK(cudaMemcpyAsync(L.cams.p, (char*)L.stage + kStageCams, kStageBytes - kStageCams, cudaMemcpyHostToDevice,
                     L.stream));
  CK(cudaMemsetAsync(L.head.p, 0, 16, L.stream));
  if (B.defer) {
    CK(cudaMemsetAsync(L.dcount.p, 0, 32, L.stream));
    k_batch_defer_clear<<<c->shade_wave, BATCH_THREADS, 0, L.stream>>>(B);
  }
  if (sorted) {
    CK(cudaMemsetAsync(L.bin_count.p, 0, L.bin_count.bytes, L.stream));
    k_qsort_count<<<c->shade_wave, BATCH_THREADS, 0, L.stream>>>(B);
    k_qsort_scan<<<1, QSCAN_THREADS, 0, L.stream>>>(B);
    k_qsort_scatter<<<c->shade_wave, BATCH_THREADS, 0, L.stream>>>(B);
  }
  k_batch_tiles<<<c->b_tile_grid, TILE_THREADS, 0, L.stream>>>(B);
  if (B.defer)
    k_batch_trace<true><<<c->b_trace_grid, BATCH_THREADS, 0, L.stream>>>(B);
  else
    k_batch_trace<false><<<c->b_trace_grid, BATCH_THREADS, 0, L.stream>>>(B);
  if (B.defer) {
    k_batch_probe_dda<<<c->shade_wave, BATCH_THREADS, 0, L.stream>>>(B);
    k_batch_slab_eval<<<c->shade_wave, BATCH_THREADS, 0, L.stream>>>(B);
    k_batch_slab_pick<<<c->shade_wave, BATCH_THREADS, 0, L.stream>>>(B);
    k_batch_resolve<<<c->shade_wave, BATCH_THREADS, 0, L.stream>>>(B);
    k_batch_refine<<<c->shade_wave, BATCH_THREADS, 0, L.stream>>>(B);
    k_batch_far<<<c->shade_wave, BATCH_THREADS, 0, L.stream>>>(B);
  }
  CK(cudaGetLastError());
  return VXE_OK;
}

}  // namespace

extern "C" {

vxe_status vxe_submit_batch_async(vxe_ctx* c, uint32_t lane, const vxe_request* reqs, uint32_t n,
                                  const vxe_batch_options* opt) {
  using namespace vxe::dev;
  if (!c || (n && !reqs) || !opt) return fail(c, VXE_ERR_INVALID_ARG, "null batch arguments");
  if (lane >= VXE_BATCH_LANES) return fail(c, VXE_ERR_INVALID_ARG, "lane %u >= %u", lane, VXE_BATCH_LANES);
  BatchLane& L = c->lanes[lane];
  if (L.busy) return fail(c, VXE_ERR_INVALID_ARG, "lane %u still has a batch in flight", lane);
  if (n > VXE_MAX_BATCH_REQUESTS) return fail(c, VXE_ERR_CAPACITY, "batch of %u requests > %u", n, VXE_MAX_BATCH_REQUESTS);
  const uint32_t tw = opt->tile_w, th = opt->tile_h, rpt = opt->rays_per_thread;
  if (tw == 0 || th == 0 || rpt == 0 || rpt > 8 || tw * th * rpt > 4096 || opt->mode > VXE_BATCH_GRAPH)
    return fail(c, VXE_ERR_INVALID_ARG, "bad batch options");
  cudaSetDevice(c->device);
  // Host-side descriptors (requests keep their order; tiles and items are
  // numbered in request order so the device finds a request by binary search).
  uint32_t tiles = 0, items = 0;
  uint64_t rays = 0, vp_rays = 0, q_rays = 0;
  // Coherent queries (persistent and graph modes): query rays are traced in
  // bin order after every viewport item instead of as per-request items.
  bool sorted = false;
  if (opt->mode != VXE_BATCH_PLAIN)
    for (uint32_t i = 0; i < n; ++i) sorted = sorted || reqs[i].kind == VXE_REQ_QUERY;
  std::vector<BatchReq> R(n);
  for (uint32_t i = 0; i < n; ++i) {
    const vxe_request& q = reqs[i];
    BatchReq& r = R[i];
    std::memset(&r, 0, sizeof r);
    r.kind = q.kind;
    r.out = (uint4*)q.d_out;
    r.tile_base = tiles;
    r.item_begin = items;
    r.ray_base = (uint32_t)vp_rays;  // a query repeats the next viewport's base
    r.q_base = (uint32_t)q_rays;     // a viewport repeats the next query's base
    if (!q.d_out) return fail(c, VXE_ERR_INVALID_ARG, "request %u has no output", i);
    if (q.kind == VXE_REQ_VIEWPORT) {
      if (q.width == 0 || q.height == 0 || q.camera.render_present_px[0] != q.width ||
          q.camera.render_present_px[1] != q.height)
        return fail(c, VXE_ERR_INVALID_ARG, "viewport %u size / camera mismatch", i);
      r.w = q.width;
      r.h = q.height;
      r.tiles_x = (q.width + 7) / 8;
      r.items_x = (q.width + tw * rpt - 1) / (tw * rpt);
      r.cam = i + 1;
      tiles += r.tiles_x * ((q.height + 7) / 8);
      items += r.items_x * ((q.height + th - 1) / th);
      rays += (uint64_t)q.width * q.height;
      vp_rays += (uint64_t)q.width * q.height;
      if (vp_rays > 0x3FFFFFFFull) return fail(c, VXE_ERR_CAPACITY, "batch of more than 2^30 viewport rays");
    } else if (q.kind == VXE_REQ_QUERY) {
      if (q.ray_count == 0 || !q.d_origins || !q.d_dirs) return fail(c, VXE_ERR_INVALID_ARG, "query %u empty", i);
      r.w = q.ray_count;
      r.o = q.d_origins;
      r.d = q.d_dirs;
      r.tmax = q.tmax;
      r.cam = 0;
      if (!sorted) items += (q.ray_count + 128 * rpt - 1) / (128 * rpt);
      rays += q.ray_count;
      q_rays += q.ray_count;
      if (q_rays > 0x3FFFFFFFull) return fail(c, VXE_ERR_CAPACITY, "batch of more than 2^30 query rays");
    } else {
      return fail(c, VXE_ERR_INVALID_ARG, "request %u kind %u", i, q.kind);
    }
  }
  // Deferred grass probes in the persistent and graph modes; the plain mode
  // is the per-request single-launch baseline with the reference's inline
  // probes.
  const bool defer = opt->mode != VXE_BATCH_PLAIN && vp_rays != 0;
  const uint32_t vp_items = items;
  if (sorted) items += (uint32_t)((q_rays + 128u * rpt - 1) / (128u * rpt));
  vxe_status st = lane_resources(c, L, tiles, defer ? (uint32_t)vp_rays : 0u, sorted ? (uint32_t)q_rays : 0u);
  if (st != VXE_OK) return st;
  if (c->upload_recorded) CK(cudaStreamWaitEvent(L.stream, c->upload_done, 0));
  const uint32_t nbins = std::max(c->cfg.grid_capacity, 1u) * 8u;
  BatchHeader H{n, tiles, items, tw, th, rpt, n, (uint32_t)vp_rays, vp_items, (uint32_t)q_rays, nbins, sorted ? 1u : 0u};
  std::memcpy((char*)L.stage + kStageHdr, &H, sizeof H);
  if (n) std::memcpy((char*)L.stage + kStageReqs, R.data(), n * sizeof(BatchReq));
  auto* cams = (vxe_camera_gpu*)((char*)L.stage + kStageCams);
  cams[0] = c->cam;  // world camera for queries
  for (uint32_t i = 0; i < n; ++i) {
    if (reqs[i].kind != VXE_REQ_VIEWPORT) continue;
    vxe_camera_gpu v = reqs[i].camera;
    // the world is the context's
    v.chunk_size = c->cam.chunk_size;
    v.chunk_count = c->cam.chunk_count;
    for (int k = 0; k < 4; ++k) {
      v.grid_origin_chunk[k] = c->cam.grid_origin_chunk[k];
      v.grid_dims[k] = c->cam.grid_dims[k];
    }
    cams[i + 1] = v;
  }
  BatchArgs B = batch_args(c, L);
  B.defer = defer ? 1u : 0u;
  CK(cudaEventRecord(L.ev[0], L.stream));
  // Grass cell table for the wind of the first viewport's camera (requests
  // with another wind time / strength derive their cells in the march).
  const vxe_camera_gpu* gcam = &cams[0];
  for (uint32_t i = 0; i < n; ++i)
    if (reqs[i].kind == VXE_REQ_VIEWPORT) {
      gcam = &cams[i + 1];
      break;
    }
  bool use_grass = false;
  if ((st = grass_table_acquire(c, L.stream, 1 + (int)lane, *gcam, &use_grass)) != VXE_OK) return st;
  if (use_grass) {
    B.grass_rec = (const float4*)c->gt.rec.p;
    B.grass_rec_n = (uint64_t)c->cfg.chunk_capacity * 4096u;
    B.grass_state = (uint32_t*)c->gt.state.p;
    B.grass_frames = (float4*)c->gt.frames.p;
    B.grass_taper = (const float*)c->gt.taper.p;
    B.grass_time_bits = fbits(gcam->voxel_params[1]);
    B.grass_strength_bits = fbits(gcam->voxel_params[2]);
  }
  if (opt->mode == VXE_BATCH_PLAIN) {
    CK(cudaMemcpyAsync(L.hdr.p, (char*)L.stage + kStageHdr, sizeof H, cudaMemcpyHostToDevice, L.stream));
    CK(cudaMemcpyAsync(L.reqs.p, (char*)L.stage + kStageReqs, n * sizeof(BatchReq), cudaMemcpyHostToDevice, L.stream));
    CK(cudaMemcpyAsync(L.cams.p, cams, (n + 1) * sizeof(vxe_camera_gpu), cudaMemcpyHostToDevice, L.stream));
    B.plain = 1;
    for (uint32_t i = 0; i < n; ++i) {
      B.req_first = i;
      const uint32_t n_items = (i + 1 < n ? R[i + 1].item_begin : items) - R[i].item_begin;
      if (R[i].kind == VXE_REQ_VIEWPORT) {
        const uint32_t t = R[i].tiles_x * ((R[i].h + 7) / 8);
        k_batch_tiles<<<(t + TILE_THREADS - 1) / TILE_THREADS, TILE_THREADS, 0, L.stream>>>(B);
      }
      k_batch_trace<false><<<(n_items + BATCH_THREADS / 32 - 1) / (BATCH_THREADS / 32), BATCH_THREADS, 0, L.stream>>>(B);
    }
    CK(cudaGetLastError());
  } else if (opt->mode == VXE_BATCH_PERSISTENT) {
    if ((st = launch_persistent(c, L, B, sorted)) != VXE_OK) return st;
  } else {
    // Captured once per tile-buffer allocation and clipmap uniform; later
    // batches only rewrite the pinned staging the graph's copies read.
    const uint32_t key[9] = {(uint32_t)(uintptr_t)L.tile_count.p, (uint32_t)((uintptr_t)L.tile_count.p >> 32),
                             (uint32_t)c->cfg.clip_levels, c->clip.levels, c->clip.res, 1u,
                             (use_grass ? 1u : 0u) | (B.defer ? 2u : 0u) | (sorted ? 4u : 0u), B.grass_time_bits,
                             B.grass_strength_bits};
    const bool same = L.graph != nullptr && std::memcmp(key, L.graph_key, sizeof key) == 0 &&
                      std::memcmp(&L.graph_clip, &B.clip, sizeof B.clip) == 0;
    if (!same) {
      if (L.graph) {
        cudaGraphExecDestroy(L.graph);
        L.graph = nullptr;
      }
      cudaGraph_t g = nullptr;
      CK(cudaStreamBeginCapture(L.stream, cudaStreamCaptureModeThreadLocal));
      st = launch_persistent(c, L, B, sorted);
      cudaError_t e = cudaStreamEndCapture(L.stream, &g);
      if (st != VXE_OK) return st;
      if (e != cudaSuccess) return fail(c, VXE_ERR_DEVICE, "graph capture: %s", cudaGetErrorString(e));
      e = cudaGraphInstantiate(&L.graph, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return fail(c, VXE_ERR_DEVICE, "graph instantiate: %s", cudaGetErrorString(e));
      std::memcpy(L.graph_key, key, sizeof key);
      L.graph_clip = B.clip;
    }
    CK(cudaGraphLaunch(L.graph, L.stream));
  }
  if (use_grass && (st = grass_table_release(c, L.stream, 1 + (int)lane)) != VXE_OK) return st;
  CK(cudaEventRecord(L.ev[1], L.stream));
  L.busy = true;
  L.rays = rays;
  L.items = items;
  L.tiles = tiles;
  return VXE_OK;
}

vxe_status vxe_batch_wait(vxe_ctx* c, uint32_t lane, int block, vxe_batch_stats* stats) {
  if (!c || lane >= VXE_BATCH_LANES) return fail(c, VXE_ERR_INVALID_ARG, "bad lane");
  BatchLane& L = c->lanes[lane];
  if (!L.busy) return fail(c, VXE_ERR_INVALID_ARG, "lane %u has no batch", lane);
  cudaSetDevice(c->device);
  if (!block) {
    const cudaError_t q = cudaEventQuery(L.ev[1]);
    if (q == cudaErrorNotReady) return VXE_NOT_READY;
    if (q != cudaSuccess) return fail(c, VXE_ERR_DEVICE, "batch: %s", cudaGetErrorString(q));
  } else {
    CK(cudaEventSynchronize(L.ev[1]));
  }
  L.busy = false;
  float ms = 0.0f;
  CK(cudaEventElapsedTime(&ms, L.ev[0], L.ev[1]));
  if (stats) {
    stats->ms = ms;
    stats->rays = L.rays;
    stats->items = L.items;
    stats->tiles = L.tiles;
  }
  uint32_t word = 0;
  CK(cudaMemcpy(&word, c->errword.p, 4, cudaMemcpyDeviceToHost));
  if (word) return fail(c, VXE_ERR_BOUNDS, "device bounds check tripped (error word 0x%x)", word);
  return VXE_OK;
}

vxe_status vxe_submit_batch(vxe_ctx* c, const vxe_request* reqs, uint32_t n, const vxe_batch_options* opt,
                            vxe_batch_stats* stats) {
  vxe_status st = vxe_submit_batch_async(c, 0, reqs, n, opt);
  if (st != VXE_OK) return st;
  return vxe_batch_wait(c, 0, 1, stats);
}


// ---------------------------------------------------------------------------
// Viewport sessions
// ---------------------------------------------------------------------------
vxe_status lane_ready(vxe_ctx* c, uint32_t lane) {
  if (lane >= VXE_BATCH_LANES) return fail(c, VXE_ERR_INVALID_ARG, "lane %u >= %u", lane, VXE_BATCH_LANES);
  return lane_resources(c, c->lanes[lane], 0u, 0u, 0u);
}

// Grows the lane's per-frame working buffers to cover an iw x ih frame.  The
// lane's queued frames may still use the old buffers: those are freed after
// them, in stream order.
vxe_status lane_scratch(vxe_ctx* c, BatchLane& L, uint32_t iw, uint32_t ih, FrameState* set = nullptr) {
  FrameState& S = set ? *set : L.scratch;
  if (S.img[IMG_PIXHIT].p && S.iw >= iw && S.ih >= ih) return VXE_OK;
  S.iw = S.pw = std::max(S.iw, iw);
  S.ih = S.ph = std::max(S.ih, ih);
  return alloc_images(c, S, IMG_SET_SCRATCH, L.stream);  // the old ones are freed in stream order
}

uint64_t vxe_view_bytes(const vxe_ctx* c, uint32_t present_w, uint32_t present_h, float render_scale) {
  if (!c || present_w == 0 || present_h == 0 || !(render_scale > 0.0f)) return 0;
  FrameState F;
  set_dims(F, present_w, present_h, render_scale);
  uint64_t total = 0;
  for (int i = 0; i < IMG_N; ++i)
    if (img_enabled(c, i) && !img_is_scratch(i)) total += img_bytes(F, i);
  return total;
}

uint64_t vxe_view_lane_bytes(const vxe_ctx* c, uint32_t present_w, uint32_t present_h, float render_scale) {
  if (!c || present_w == 0 || present_h == 0 || !(render_scale > 0.0f)) return 0;
  FrameState F;
  set_dims(F, present_w, present_h, render_scale);
  uint64_t total = 0;
  for (int i = 0; i < IMG_N; ++i)
    if (img_enabled(c, i) && img_is_scratch(i)) total += img_bytes(F, i);
  return total;
}

vxe_status vxe_view_create(vxe_ctx* c, uint32_t present_w, uint32_t present_h, float render_scale, vxe_view** out) {
  if (!c || !out || present_w == 0 || present_h == 0 || !(render_scale > 0.0f) || render_scale > 4.0f)
    return fail(c, VXE_ERR_INVALID_ARG, "bad view arguments");
  *out = nullptr;
  cudaSetDevice(c->device);
  if (!c->aux) CK(cudaStreamCreateWithFlags(&c->aux, cudaStreamNonBlocking));
  auto* v = new (std::nothrow) vxe_view();
  if (!v) return fail(c, VXE_ERR_OOM, "view");
  set_dims(v->fr, present_w, present_h, render_scale);
  if (cudaEventCreateWithFlags(&v->done, cudaEventDisableTiming) != cudaSuccess) {
    delete v;
    return fail(c, VXE_ERR_DEVICE, "view event");
  }
  // images from the pool, zero-filled on the aux stream; the first frame
  // waits for the fill like a frame that follows one on another lane
  vxe_status st = alloc_images(c, v->fr, IMG_SET_OWN, c->aux);
  if (st != VXE_OK) {
    release_frame_state(v->fr, c->aux);
    cudaEventDestroy(v->done);
    delete v;
    return st;
  }
  v->last_stream = c->aux;
  *out = v;
  return VXE_OK;
}

vxe_status vxe_view_render_async(vxe_ctx* c, vxe_view* v, uint32_t lane, const vxe_camera_gpu* cam) {
  if (!c || !v || !cam) return fail(c, VXE_ERR_INVALID_ARG, "null view arguments");
  cudaSetDevice(c->device);
  vxe_status st = lane_ready(c, lane);
  if (st != VXE_OK) return st;
  BatchLane& L = c->lanes[lane];
  // a view's frames run in order: follow its previous frame's lane
  if (v->last_stream && v->last_stream != L.stream) {
    CK(cudaEventRecord(v->done, v->last_stream));
    CK(cudaStreamWaitEvent(L.stream, v->done, 0));
  }
  vxe_camera_gpu vc = *cam;
  vc.chunk_size = c->cam.chunk_size;
  vc.chunk_count = c->cam.chunk_count;
  for (int k = 0; k < 4; ++k) {
    vc.grid_origin_chunk[k] = c->cam.grid_origin_chunk[k];
    vc.grid_dims[k] = c->cam.grid_dims[k];
  }
  if ((st = frame_validate(c, v->fr, vc)) != VXE_OK) return st;
  for (int i = 0; i < IMG_N; ++i)
    if (!img_is_scratch(i) && img_enabled(c, i) != (v->fr.img[i].p != nullptr))
      return fail(c, VXE_ERR_INVALID_ARG, "view was created under other image flags");
  if ((st = lane_scratch(c, L, v->fr.iw, v->fr.ih)) != VXE_OK) return st;
  if (!L.busy) CK(cudaEventRecord(L.ev[0], L.stream));
  if (c->upload_recorded) CK(cudaStreamWaitEvent(L.stream, c->upload_done, 0));
  // The view's own outputs and histories, the lane's working buffers; plain
  // launches (a view's graph would be re-captured whenever it changes lanes).
  FrameArgs A;
  frame_fill(c, v->fr, vc, A, &L.scratch);
  bool use_grass = false;
  const int reader = 1 + (int)lane;
  if ((st = grass_table_acquire(c, L.stream, reader, vc, &use_grass)) != VXE_OK) return st;
  if (use_grass) grass_table_args(c, A);
  if ((st = frame_enqueue(c, v->fr, A, false, L.stream, &L.side)) != VXE_OK) return st;
  if (use_grass && (st = grass_table_release(c, L.stream, reader)) != VXE_OK) return st;
  v->fr.ping = 1 - v->fr.ping;
  CK(cudaEventRecord(L.ev[1], L.stream));
  if (!L.busy) {
    L.rays = 0;
    L.items = 0;
    L.tiles = 0;
  }
  L.busy = true;
  L.rays += (uint64_t)v->fr.iw * v->fr.ih;
  v->last_stream = L.stream;
  return VXE_OK;
}

vxe_status vxe_view_render_batch_async(vxe_ctx* c, vxe_view* const* views, const vxe_camera_gpu* cams, uint32_t n,
                                       uint32_t lane) {
  using namespace vxe::dev;
  if (!c || (n && (!views || !cams))) return fail(c, VXE_ERR_INVALID_ARG, "null view arguments");
  if (n == 0) return VXE_OK;
  if (n > kMaxViewsPerLaunch)
    return fail(c, VXE_ERR_CAPACITY, "%u views in one launch > %u", n, kMaxViewsPerLaunch);
  if (c->flags & VXE_FLAG_PRIMARY_MEGAKERNEL) {  // the one-kernel schedule renders view by view
    for (uint32_t i = 0; i < n; ++i) {
      const vxe_status st = vxe_view_render_async(c, views[i], lane, &cams[i]);
      if (st != VXE_OK) return st;
    }
    return VXE_OK;
  }
  cudaSetDevice(c->device);
  vxe_status st = lane_ready(c, lane);
  if (st != VXE_OK) return st;
  BatchLane& L = c->lanes[lane];
  std::vector<vxe_camera_gpu> vc(n);
  for (uint32_t i = 0; i < n; ++i) {
    vxe_view* v = views[i];
    if (!v) return fail(c, VXE_ERR_INVALID_ARG, "null view %u", i);
    for (uint32_t j = 0; j < i; ++j)
      if (views[j] == v) return fail(c, VXE_ERR_INVALID_ARG, "view %u appears twice in one launch", i);
    vc[i] = cams[i];
    vc[i].chunk_size = c->cam.chunk_size;
    vc[i].chunk_count = c->cam.chunk_count;
    for (int k = 0; k < 4; ++k) {
      vc[i].grid_origin_chunk[k] = c->cam.grid_origin_chunk[k];
      vc[i].grid_dims[k] = c->cam.grid_dims[k];
    }
    if ((st = frame_validate(c, v->fr, vc[i])) != VXE_OK) return st;
    for (int k = 0; k < IMG_N; ++k)
      if (!img_is_scratch(k) && img_enabled(c, k) != (v->fr.img[k].p != nullptr))
        return fail(c, VXE_ERR_INVALID_ARG, "view %u was created under other image flags", i);
  }
  for (uint32_t i = 0; i < n; ++i)
    if ((st = lane_scratch(c, L, views[i]->fr.iw, views[i]->fr.ih, &L.mscratch[i])) != VXE_OK) return st;
  if (!L.busy) CK(cudaEventRecord(L.ev[0], L.stream));
  if (c->upload_recorded) CK(cudaStreamWaitEvent(L.stream, c->upload_done, 0));
  for (uint32_t i = 0; i < n; ++i) {  // each view's frames run in order
    vxe_view* v = views[i];
    if (v->last_stream && v->last_stream != L.stream) {
      CK(cudaEventRecord(v->done, v->last_stream));
      CK(cudaStreamWaitEvent(L.stream, v->done, 0));
    }
  }
  // The grass cell table serves the launch when every view's camera matches
  // its tag (same wind); otherwise the marches derive their cells.
  const int reader = 1 + (int)lane;
  bool use_grass = false;
  if ((st = grass_table_acquire(c, L.stream, reader, vc[0], &use_grass)) != VXE_OK) return st;
  for (uint32_t i = 1; i < n && use_grass; ++i)
    use_grass = vc[i].voxel_params[0] == vc[0].voxel_params[0] && vc[i].voxel_params[1] == vc[0].voxel_params[1] &&
                vc[i].voxel_params[2] == vc[0].voxel_params[2] && vc[i].chunk_count == vc[0].chunk_count;
  auto* V = new (std::nothrow) FrameArgsViews;  // 12 KB: off the stack
  if (!V) return fail(c, VXE_ERR_OOM, "view arguments");
  std::unique_ptr<FrameArgsViews> hold(V);
  std::memset(V, 0, sizeof *V);
  uint32_t max_iw = 0, max_ih = 0, max_pw = 0, max_ph = 0;
  uint64_t max_pix = 0, rays = 0;
  for (uint32_t i = 0; i < n; ++i) {
    FrameState& F = views[i]->fr;
    frame_fill(c, F, vc[i], V->v[i], &L.mscratch[i]);
    if (use_grass) grass_table_args(c, V->v[i]);
    max_iw = std::max(max_iw, F.iw);
    max_ih = std::max(max_ih, F.ih);
    max_pw = std::max(max_pw, F.pw);
    max_ph = std::max(max_ph, F.ph);
    max_pix = std::max<uint64_t>(max_pix, (uint64_t)F.iw * F.ih);
    rays += (uint64_t)F.iw * F.ih;
  }
  if ((st = views_enqueue(c, *V, n, max_iw, max_ih, max_pw, max_ph, max_pix, L.stream, &L.side)) != VXE_OK)
    return st;
  if ((st = grass_table_release(c, L.stream, reader)) != VXE_OK) return st;
  for (uint32_t i = 0; i < n; ++i) {
    views[i]->fr.ping = 1 - views[i]->fr.ping;
    views[i]->last_stream = L.stream;
  }
  CK(cudaEventRecord(L.ev[1], L.stream));
  if (!L.busy) {
    L.rays = 0;
    L.items = 0;
    L.tiles = 0;
  }
  L.busy = true;
  L.rays += rays;
  return VXE_OK;
}

vxe_status vxe_view_read_image(vxe_ctx* c, vxe_view* v, int image, void* host, size_t bytes) {
  if (!c || !v || !host) return fail(c, VXE_ERR_INVALID_ARG, "null view arguments");
  const int i = map_image(v->fr, (vxe_image)image);
  if (i < 0 || !v->fr.img[i].p) return fail(c, VXE_ERR_INVALID_ARG, "image %d not available", image);
  if (bytes != v->fr.img[i].bytes)
    return fail(c, VXE_ERR_INVALID_ARG, "image %d is %zu bytes, got %zu", image, v->fr.img[i].bytes, bytes);
  cudaSetDevice(c->device);
  if (v->last_stream) CK(cudaStreamSynchronize(v->last_stream));
  CK(cudaMemcpy(host, v->fr.img[i].p, bytes, cudaMemcpyDeviceToHost));
  return VXE_OK;
}

vxe_status vxe_view_destroy(vxe_ctx* c, vxe_view* v) {
  if (!c || !v) return VXE_ERR_INVALID_ARG;
  cudaSetDevice(c->device);
  release_frame_state(v->fr, v->last_stream);  // freed after the view's last frame
  if (v->done) cudaEventDestroy(v->done);
  delete v;
  return VXE_OK;
}

}  // extern "C"

namespace {
__global__ void k_detmath(int which, const float* x, const float* y, float* out, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float r;
  switch (which) {
    case 0: r = vxe_sinf(x[i]); break;
    case 1: r = vxe_cosf(x[i]); break;
    case 2: r = vxe_expf(x[i]); break;
    case 3: r = vxe_powf(x[i], y[i]); break;
    case 4: r = fminf(x[i], y[i]); break;
    default: r = fmaxf(x[i], y[i]); break;
  }
  out[i] = r;
}
}  // namespace

extern "C" vxe_status vxe_debug_detmath(int which, const float* x, const float* y, float* out, uint32_t n) {
  if (!x || !y || !out) return VXE_ERR_INVALID_ARG;
  if (n == 0) return VXE_OK;
  float* d = nullptr;
  if (cudaMalloc(&d, (size_t)n * 12) != cudaSuccess) return VXE_ERR_OOM;
  vxe_status st = VXE_OK;
  if (cudaMemcpy(d, x, (size_t)n * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(d + n, y, (size_t)n * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
    st = VXE_ERR_DEVICE;
  } else {
    k_detmath<<<(n + 255) / 256, 256>>>(which, d, d + n, d + 2 * (size_t)n, n);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpy(out, d + 2 * (size_t)n, (size_t)n * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
      st = VXE_ERR_DEVICE;
  }
  cudaFree(d);
  return st;
}

namespace {
// One grass march (which 0) or SDF evaluation (which 1) per thread on
// caller inputs, for host/device comparisons (vxe_debug_grass).
__global__ void k_debug_grass(int which, const float* in, float* out, uint32_t n) {
  using namespace vxe::dev;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  vxe_camera_gpu cam;
  memset(&cam, 0, sizeof cam);
  Scene s;
  memset(&s, 0, sizeof s);
  s.cam = &cam;
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
}  // namespace

extern "C" vxe_status vxe_debug_grass(int which, uint32_t n, const float* in, float* out) {
  if (!in || !out || which < 0 || which > 1) return VXE_ERR_INVALID_ARG;
  if (n == 0) return VXE_OK;
  const size_t nin = (size_t)n * (which == 0 ? 17u : 13u), nout = (size_t)n * (which == 0 ? 5u : 1u);
  float* d = nullptr;
  if (cudaMalloc(&d, (nin + nout) * 4) != cudaSuccess) return VXE_ERR_OOM;
  vxe_status st = VXE_OK;
  if (cudaMemcpy(d, in, nin * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
    st = VXE_ERR_DEVICE;
  } else {
    k_debug_grass<<<(n + 127) / 128, 128>>>(which, d, d + nin, n);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpy(out, d + nin, nout * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
      st = VXE_ERR_DEVICE;
  }
  cudaFree(d);
  return st;
}

// L2 read bandwidth: every thread reads 16-byte words of an L2-resident
// buffer in a grid-stride loop (consecutive lanes, consecutive words), so
// after the first pass each launch streams the buffer from L2.
__global__ void __launch_bounds__(512) k_l2_read(const uint4* __restrict__ p, size_t n, uint32_t* sink) {
  uint32_t acc = 0u;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const uint4 v = __ldcg(p + i);
    acc ^= v.x ^ v.y ^ v.z ^ v.w;
  }
  if (acc == 0x9E3779B9u) sink[0] = acc;  // keeps the loads; the buffer is zero, so never taken
}

extern "C" vxe_status vxe_measure_l2_bandwidth(int device, uint64_t bytes, uint32_t launches, double* gbs) {
  if (!gbs || bytes < (1u << 20) || launches == 0) return VXE_ERR_INVALID_ARG;
  *gbs = 0.0;
  if (cudaSetDevice(device) != cudaSuccess) return VXE_ERR_NO_DEVICE;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || sms <= 0)
    return VXE_ERR_DEVICE;
  void* buf = nullptr;
  if (cudaMalloc(&buf, bytes + 256) != cudaSuccess) return VXE_ERR_OOM;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  vxe_status st = VXE_OK;
  const size_t n = bytes / 16;
  const unsigned grid = (unsigned)sms * 4u;  // 4 blocks of 512 threads per SM
  uint32_t* sink = (uint32_t*)((char*)buf + bytes);
  if (cudaMemset(buf, 0, bytes + 256) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
      cudaEventCreate(&e1) != cudaSuccess) {
    st = VXE_ERR_DEVICE;
  } else {
    for (int w = 0; w < 3; ++w) k_l2_read<<<grid, 512>>>((const uint4*)buf, n, sink);  // resident in L2
    cudaEventRecord(e0);
    for (uint32_t i = 0; i < launches; ++i) k_l2_read<<<grid, 512>>>((const uint4*)buf, n, sink);
    cudaEventRecord(e1);
    float ms = 0.0f;
    if (cudaGetLastError() != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
        cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess || ms <= 0.0f)
      st = VXE_ERR_DEVICE;
    else
      *gbs = (double)(n * 16) * launches / (ms * 1e-3) / 1e9;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(buf);
  return st;
}

// ===========================================================================
// Allocation-free primary hit records (vxe_trace_primary_hits_noalloc)
// ===========================================================================
#include <mutex>

namespace {

// Scratch of the allocation-free entry point: word 0 is the device error
// word, the per-tile candidate counts start at word 64 (256 B), the 24-slot
// lists follow.  Sized for VXE_NOALLOC_MAX_TILES tiles (3.7 MB); every device
// that loads the library holds it until the process exits.
constexpr size_t kNoallocCountOff = 64;
constexpr size_t kNoallocSlotOff = kNoallocCountOff + VXE_NOALLOC_MAX_TILES;
constexpr size_t kNoallocWords = kNoallocSlotOff + (size_t)VXE_NOALLOC_MAX_TILES * VXE_PRIMARY_MAX_TILE_CHUNKS;
static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoallocWords];

// In host code g_noalloc_scratch is only a stand-in symbol, not a device
// address; the address is resolved per device with that device current, and
// again when the device's context changed since (after cudaDeviceReset the
// module loads again, possibly at another address).
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
uint32_t* g_noalloc_addr[kMaxDevices] = {};
void* g_noalloc_ctx[kMaxDevices] = {};

// The current driver context (cuCtxGetCurrent through the runtime's entry
// point lookup, so the library needs no link against the driver library);
// null if it cannot be had.
void* current_context() {
  using GetCurrent = int (*)(void**);
  static GetCurrent fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return (GetCurrent)f;
  }();
  void* ctx = nullptr;
  if (!fn || fn(&ctx) != 0) return nullptr;
  return ctx;
}

vxe_status noalloc_scratch(int dev, uint32_t** out) {
  if (dev < 0 || dev >= kMaxDevices) return VXE_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  void* ctx = current_context();
  if (!g_noalloc_addr[dev] || !ctx || ctx != g_noalloc_ctx[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return VXE_ERR_DEVICE;
    g_noalloc_addr[dev] = (uint32_t*)p;
    g_noalloc_ctx[dev] = ctx;
  }
  *out = g_noalloc_addr[dev];
  return VXE_OK;
}

// Per-pixel hit record of a cold frame: the primary trace without history,
// then the grass refinement / heightfield fallback of main_primary
// (ray_main.wgsl:224-269, 327-411, 473-498), as the frame pass records them.
__global__ void __launch_bounds__(vxe::dev::PRIMARY_THREADS) k_hits_noalloc(const __grid_constant__ FrameArgs A) {
  using namespace vxe::dev;
  __shared__ uint32_t cslot[2][TILE_CANDS];
  __shared__ Meta cmeta[2][TILE_CANDS];
  __shared__ uint32_t ccount[2];
  const Scene s = make_scene(A, false);
  stage_tiles(s, A, cslot, cmeta, ccount);
  uint32_t t, gx, gy;
  if (!block_pixel(A, &t, &gx, &gy)) return;
  const PrimaryCtx c = primary_ctx(s, gx, gy, A.iw);
  const float vs = vs_(s);
  const v3 ro = c.ro, rd = c.rd;
  VoxTraceResult vt{false, miss_hitgeom(), 0.0f, false, INVALID, i3{0, 0, 0}};
  ProbeHook ph = probe_hook_inline();
  if (s.cam->chunk_count != 0u && ccount[t] != 0u)
    vt = trace_candidates<PROBE_INLINE>(s, cslot[t], cmeta[t], ro, rd, 0.0f, FOG_MAX_DIST, false, i3{0, 0, 0}, INVALID,
                                        ccount[t], ph);
  HitRec rec = miss_rec();
  if (vt.in_grid && vt.best.hit != 0u) {
    HitGeom best = vt.best;
    if (best.mat == MAT_GRASS) {
      const i3 ov{to_i32(floorf(best.root_bmin.x / vs + 0.5f)), to_i32(floorf(best.root_bmin.y / vs + 0.5f)),
                  to_i32(floorf(best.root_bmin.z / vs + 0.5f))};
      const v3 hp = ro + rd * best.t;
      const GrassCell cell = pick_grass_cell_in_chunk_with_bias(hp, rd, best.root_bmin, ov, vs, (int32_t)s.cam->chunk_size);
      const GrassHit gh = try_grass_slab_hit(s, ro, rd, 0.0f, best.t, cell.bmin_m, cell.id_vox, vs,
                                             s.cam->voxel_params[1], s.cam->voxel_params[2]);
      if (gh.hit) { best.t = gh.t; best.n = gh.n; }
    }
    rec = make_rec(best, ro, rd, vs, true);
  } else if (s.cam->chunk_count != 0u) {  // no chunks: sky (ray_main.wgsl:219-231)
    ClipHit hf = clip_trace_heightfield(s, ro, rd, 0.0f, FOG_MAX_DIST);
    if (hf.hit) {
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
      rec = make_rec(g, ro, rd, vs, false);
    }
  }
  store_rec(A.hits + c.pix * 2u, rec);
}

}  // namespace

extern "C" vxe_status vxe_trace_primary_hits_noalloc(const vxe_scene_view* sv, const vxe_camera_gpu* cam,
                                                     const vxe_clipmap_gpu* clip, vxe_hit* d_hits, void* stream) {
  using namespace vxe::dev;
  if (!sv || !cam || !clip || !d_hits || !sv->nodes || !sv->ropes || !sv->metas || !sv->macro_words ||
      !sv->colinfo_words || !sv->grid || sv->node_count == 0 || sv->chunk_capacity == 0 || sv->grid_cells == 0)
    return VXE_ERR_INVALID_ARG;
  const uint32_t iw = cam->render_present_px[0], ih = cam->render_present_px[1];
  if (iw == 0 || ih == 0 || cam->chunk_size != 64u) return VXE_ERR_INVALID_ARG;
  const uint64_t tiles_x = (iw + 7) / 8, tiles_y = (ih + 7) / 8;
  if (tiles_x * tiles_y > VXE_NOALLOC_MAX_TILES) return VXE_ERR_CAPACITY;
  if ((uint64_t)cam->grid_dims[0] * cam->grid_dims[1] * cam->grid_dims[2] > sv->grid_cells) return VXE_ERR_CAPACITY;
  if (cam->chunk_count > sv->chunk_capacity) return VXE_ERR_CAPACITY;
  if (clip->levels != 0 && (!sv->clip_tex || clip->levels > sv->clip_layers || clip->res != sv->clip_res))
    return VXE_ERR_INVALID_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return VXE_ERR_NO_DEVICE;
  // An error the caller left pending is not this call's: report it without
  // launching, and leave it for the caller (peek does not clear it).
  if (cudaPeekAtLastError() != cudaSuccess) return VXE_ERR_DEVICE;
  uint32_t* scratch = nullptr;
  vxe_status st = noalloc_scratch(dev, &scratch);
  if (st != VXE_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  FrameArgs A;
  std::memset(&A, 0, sizeof A);
  A.cam = *cam;
  A.clip = *clip;
  A.nodes = (const uint4*)sv->nodes;
  A.nodes_n = sv->node_count;
  A.ropes = (const uint32_t*)sv->ropes;
  A.ropes_n = sv->node_count;
  A.metas = (const uint4*)sv->metas;
  A.metas_n = sv->chunk_capacity;
  A.grid = sv->grid;
  A.grid_n = sv->grid_cells;
  A.macro = sv->macro_words;
  A.macro_n = (uint64_t)sv->chunk_capacity * VXE_MACRO_WORDS_PER_CHUNK;
  A.colinfo = sv->colinfo_words;
  A.colinfo_n = (uint64_t)sv->chunk_capacity * VXE_COLINFO_WORDS_PER_CHUNK;
  A.clip_tex = sv->clip_tex;
  A.clip_layers = sv->clip_tex ? sv->clip_layers : 0u;
  A.clip_res = sv->clip_res;
  A.err = scratch;  // word 0, cleared below: it must start at zero
  A.iw = iw;
  A.ih = ih;
  A.tile_count = scratch + kNoallocCountOff;  // fully rewritten by k_tiles every call
  A.tile_slots = scratch + kNoallocSlotOff;
  A.hits = (uint4*)d_hits;
  if (cudaMemsetAsync(scratch, 0, 4, s) != cudaSuccess) return VXE_ERR_DEVICE;
  const uint32_t tiles = (uint32_t)(tiles_x * tiles_y);
  k_tiles<<<(tiles + TILE_THREADS - 1) / TILE_THREADS, TILE_THREADS, 0, s>>>(A);
  k_hits_noalloc<<<dim3((uint32_t)(tiles_x + 1) / 2, (uint32_t)tiles_y), PRIMARY_THREADS, 0, s>>>(A);
  if (cudaGetLastError() != cudaSuccess) return VXE_ERR_DEVICE;
  if (cudaStreamSynchronize(s) != cudaSuccess) return VXE_ERR_DEVICE;
  uint32_t word = 0;
  if (cudaMemcpy(&word, scratch, 4, cudaMemcpyDeviceToHost) != cudaSuccess) return VXE_ERR_DEVICE;
  return word ? VXE_ERR_BOUNDS : VXE_OK;
}
