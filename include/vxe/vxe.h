/*
 * vxe.h -- C ABI of the B200-native primary / godray / composite passes.
 *
 * Drop-in boundary for voxel-engine-v0's compute frame.  Every struct below is
 * byte-identical to the Rust `#[repr(C)]` POD that the reference uploads with
 * `queue.write_buffer`, so a Rust host can pass its existing slices straight
 * through `extern "C"`.  Every entry point cites the reference method it
 * replaces (paths relative to the reference project root).
 *
 * Conventions
 *  - All calls return vxe_status; vxe_last_error(ctx) gives a message.
 *  - A vxe_ctx is externally synchronised (one host thread at a time), the
 *    same contract as the reference `Renderer` (render/state/mod.rs:34-709).
 *  - Host pointers are borrowed for the duration of the call only.
 *  - Device pointers returned in vxe_frame_out stay valid until the next
 *    vxe_render_frame / vxe_resize / vxe_destroy on the same ctx.
 *
 * Device bounds checks
 *  The passes read node, rope, meta, grid, macro, colinfo and clipmap
 *  records at indices taken from other records.  Two builds of this library
 *  export the same entry points and differ only in those reads:
 *  - libvxe.so clamps every such index into its buffer: never a read outside
 *    the buffers, no branch on the traversal's hot path (the checks cost
 *    about a fifth of a 1080p frame and half of the walk kernel's time);
 *    records that point outside their chunk give wrong images and no error
 *    report;
 *  - libvxe_checked.so reads a zero record for an index outside its buffer
 *    and sets a bit of the context's error word (vxe_read_error_word;
 *    vxe_render_frame and the allocation-free entry point then return
 *    VXE_ERR_BOUNDS).
 *  Valid records give identical results with either.  Use the checked build
 *  to validate a new producer's records.
 */
#ifndef VXE_VXE_H
#define VXE_VXE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Status codes                                                              */
/* ------------------------------------------------------------------------ */
typedef enum vxe_status {
  VXE_OK = 0,
  VXE_ERR_INVALID_ARG = 1,
  VXE_ERR_CAPACITY = 2,   /* upload exceeds an arena (reference skips silently) */
  VXE_ERR_OOM = 3,        /* device allocation failed                          */
  VXE_ERR_TIMEOUT = 4,    /* a bounded device wait gave up                      */
  VXE_ERR_DEVICE = 5,     /* CUDA runtime error                                 */
  VXE_ERR_BOUNDS = 6,     /* device-side bounds check tripped (error word set)  */
  VXE_ERR_NO_DEVICE = 7,  /* no CUDA device / extension unusable                */
  VXE_NOT_READY = 8       /* asynchronous work still running (not an error)     */
} vxe_status;

/* ------------------------------------------------------------------------ */
/* Constants (common.wgsl:16-19, 416-420; app/config.rs:5-51)                */
/* ------------------------------------------------------------------------ */
#define VXE_INVALID_U32 0xFFFFFFFFu
#define VXE_LEAF_U32 0xFFFFFFFFu
#define VXE_MACRO_WORDS_PER_CHUNK 16u
#define VXE_COLINFO_WORDS_PER_CHUNK 2048u
#define VXE_CHUNK_SIZE 64u
#define VXE_CLIP_LEVELS_MAX 16u
#define VXE_TILE_SIZE 8u
#define VXE_MAX_TILE_CHUNKS 192u
#define VXE_PRIMARY_MAX_TILE_CHUNKS 24u

enum {
  VXE_MAT_AIR = 0, VXE_MAT_GRASS = 1, VXE_MAT_DIRT = 2, VXE_MAT_STONE = 3,
  VXE_MAT_WOOD = 4, VXE_MAT_LEAF = 5, VXE_MAT_LIGHT = 6
};

/* ------------------------------------------------------------------------ */
/* GPU records (render/gpu_types.rs)                                         */
/* ------------------------------------------------------------------------ */

/* NodeGpu (render/gpu_types.rs:13-20, common.wgsl:338-343): 16 B. */
typedef struct vxe_node {
  uint32_t child_base; /* local index of first packed child, or VXE_LEAF_U32 */
  uint32_t child_mask; /* bit ci = x | y<<1 | z<<2                           */
  uint32_t material;
  uint32_t key;        /* x | y<<6 | z<<12 | level<<18 (svo/builder_svo.rs:22-35) */
} vxe_node;

/* NodeRopesGpu (render/gpu_types.rs:22-33): 32 B, local neighbour indices. */
typedef struct vxe_node_ropes {
  uint32_t px, nx, py, ny, pz, nz, _pad0, _pad1;
} vxe_node_ropes;

/* ChunkMetaGpu (render/gpu_types.rs:36-48): 48 B. */
typedef struct vxe_chunk_meta {
  int32_t origin[4];     /* chunk origin in voxels, w = 0 */
  uint32_t node_base;    /* global arena index of the chunk's root */
  uint32_t node_count;
  uint32_t macro_base;   /* slot * 16 */
  uint32_t colinfo_base; /* slot * 2048 */
  uint32_t macro_empty;  /* 1 when all 512 macro bits are 0 */
  uint32_t _pad0, _pad1, _pad2;
} vxe_chunk_meta;

/* CameraGpu (render/gpu_types.rs:50-86): 464 B, matrices column-major. */
typedef struct vxe_camera_gpu {
  float view_inv[4][4];
  float proj_inv[4][4];
  float view_proj[4][4];
  float prev_view_proj[4][4];
  float cam_pos[4];
  float ray00[4];
  float ray_dx[4];
  float ray_dy[4];
  uint32_t chunk_size;
  uint32_t chunk_count;
  uint32_t max_steps;
  uint32_t frame_index;
  float voxel_params[4];      /* [voxel_size, time_s, wind_strength, fog_density] */
  int32_t grid_origin_chunk[4];
  uint32_t grid_dims[4];
  uint32_t render_present_px[4]; /* internal w,h ; present w,h */
  uint32_t profile_flags;
  uint32_t _pad_profile[3];
  uint32_t _pad0[4];
  uint32_t _pad1[4];
  uint32_t _pad2[4];
} vxe_camera_gpu;

/* ClipmapGpu (render/gpu_types.rs:103-138): 528 B. */
typedef struct vxe_clipmap_gpu {
  uint32_t levels;
  uint32_t res;
  float base_cell_m;
  float _pad0;
  float level[VXE_CLIP_LEVELS_MAX][4];     /* origin_x_m, origin_z_m, cell_m, 0 */
  uint32_t offset[VXE_CLIP_LEVELS_MAX][4]; /* off_x, off_z, 0, 0 (texels)      */
} vxe_clipmap_gpu;

/* ClipmapUpload (clipmap.rs:35-42): a sub-rectangle of one level layer. */
typedef struct vxe_clip_patch {
  uint32_t level, x, y, w, h;
  const float* data; /* w*h floats, row-major */
} vxe_clip_patch;

/* ChunkUpload (streaming/types.rs:87-103). */
typedef struct vxe_chunk_upload {
  uint32_t slot;
  vxe_chunk_meta meta;
  uint32_t node_base;
  uint32_t node_count;
  const vxe_node* nodes;          /* node_count records */
  const vxe_node_ropes* ropes;    /* node_count records */
  const uint32_t* macro_words;    /* 16 words            */
  const uint32_t* colinfo_words;  /* 2048 words          */
} vxe_chunk_upload;

/* ------------------------------------------------------------------------ */
/* Context                                                                   */
/* ------------------------------------------------------------------------ */
typedef struct vxe_ctx vxe_ctx;

enum {
  /* The reference binds the scene group for main_godray with macro_occ at
   * binding 8 while the shader reads binding 9 (render/state/bindgroups.rs:
   * 116-156 vs shaders/common.wgsl:407-409), so godray shadow marches read
   * rope words as macro bits.  Set = reproduce that aliasing (default). */
  VXE_FLAG_GODRAY_MACRO_ALIAS = 1u << 0,
  /* Reference render/state/mod.rs:538-565 silently skips uploads that do not
   * fit; set to keep that behaviour, clear to get VXE_ERR_CAPACITY. */
  VXE_FLAG_SILENT_CAPACITY_SKIP = 1u << 1,
  /* Write per-pixel hit records (t, node, voxel, face, mat) from the primary
   * pass (the reference has no such output; see vxe_hit). */
  VXE_FLAG_HIT_RECORDS = 1u << 2,
  /* Keep the intermediate images (local_img, output_pre_taa) that the fused
   * kernels otherwise never materialise; used by parity tests. */
  VXE_FLAG_DEBUG_INTERMEDIATES = 1u << 3,
  /* (bit 4 is unused: device bounds checks are a build of the library,
   * see "Device bounds checks" above) */
  /* Run the primary pass as one kernel per pixel (trace + shading) instead of
   * the default wavefront (trace kernel -> per-class shading kernels).  Both
   * produce identical images. */
  VXE_FLAG_PRIMARY_MEGAKERNEL = 1u << 5,
  /* Do not keep the per-frame grass cell table (blade roots, wind bend,
   * lean, radius and side axis of every grass column top, 160 B per column of
   * every chunk slot).  Without it each grass march derives its cell's blades
   * itself, as the reference shader does; images are identical either way.
   * Read at vxe_create (the table is allocated there) and per frame.  The
   * table also caches, per frame, the lod-0 blade segment frames of the
   * columns that grass marches visit (864 B per column). */
  VXE_FLAG_NO_GRASS_TABLE = 1u << 6,
  /* vxe_upload_chunks copies are ordered before every pass enqueued after
   * the call but not after the passes already in flight (a world write is
   * otherwise ordered after both, like a queue write between submissions).
   * For callers whose uploads only write chunk slots and node ranges that no
   * pass in flight reads -- freshly allocated slots of a streaming loader --
   * or rewrite them with identical contents.  Grid, meta and clipmap writes
   * stay ordered. */
  VXE_FLAG_UPLOADS_UNORDERED = 1u << 7
};

typedef struct vxe_config {
  uint32_t node_capacity;    /* NodeGpu records in the arena (ropes: same)   */
  uint32_t chunk_capacity;   /* ChunkMetaGpu slots                           */
  uint32_t grid_capacity;    /* chunk_grid cells                             */
  uint32_t clip_levels;      /* clipmap layers allocated (<= 16)             */
  uint32_t clip_res;         /* clipmap texture side                         */
  uint32_t flags;            /* VXE_FLAG_*                                    */
  int32_t device;            /* CUDA ordinal                                 */
  uint32_t _reserved;
} vxe_config;

/* Renderer::new (render/state/mod.rs:147-267). */
vxe_status vxe_create(const vxe_config* cfg, vxe_ctx** out);
void vxe_destroy(vxe_ctx* ctx);
const char* vxe_last_error(const vxe_ctx* ctx);
uint32_t vxe_get_flags(const vxe_ctx* ctx);
vxe_status vxe_set_flags(vxe_ctx* ctx, uint32_t flags);

/* Renderer::resize_output (render/state/mod.rs:297-308): recreates the images
 * (internal = round(present*render_scale)) and resets histories + ping. */
vxe_status vxe_resize(vxe_ctx* ctx, uint32_t present_w, uint32_t present_h, float render_scale);
vxe_status vxe_get_internal_dims(const vxe_ctx* ctx, uint32_t* w, uint32_t* h);

/* Renderer::apply_chunk_uploads (render/state/mod.rs:514-582).  Copies are
 * issued on the upload stream and ordered before the next frame by an event. */
vxe_status vxe_upload_chunks(vxe_ctx* ctx, const vxe_chunk_upload* ups, uint32_t n);
/* Meta-only rewrite of slots [first, first+n) (render/state/mod.rs:104-144). */
vxe_status vxe_write_meta(vxe_ctx* ctx, uint32_t first_slot, const vxe_chunk_meta* metas, uint32_t n);
/* Renderer::write_chunk_grid (render/state/mod.rs:310-317). */
vxe_status vxe_write_grid(vxe_ctx* ctx, const uint32_t* grid, uint32_t n);
/* Renderer::write_camera (render/state/mod.rs:319-322). */
vxe_status vxe_write_camera(vxe_ctx* ctx, const vxe_camera_gpu* cam);
/* Renderer::write_clipmap_updates (render/state/mod.rs:586-634): patches
 * first, then the uniform, both ordered before the next frame. */
vxe_status vxe_write_clipmap(vxe_ctx* ctx, const vxe_clipmap_gpu* params,
                             const vxe_clip_patch* patches, uint32_t n);

/* Outputs of one frame (device pointers, ctx-owned). */
typedef struct vxe_frame_out {
  float* color;        /* internal w*h RGBA32F  (color_img)      */
  float* depth;        /* internal w*h R32F     (depth_img)      */
  float* godray;       /* internal w*h RGBA32F  (godray[pong])   */
  float* output;       /* present  w*h RGBA32F  (output_tex)     */
  uint32_t internal_w, internal_h, present_w, present_h;
} vxe_frame_out;

/* Renderer::encode_compute (render/state/mod.rs:329-446): primary, local
 * TAA, godray, composite, composite TAA with the reference ping-pong; plain
 * launches on the ctx compute stream.  Synchronous unless `async` != 0. */
vxe_status vxe_render_frame(vxe_ctx* ctx, vxe_frame_out* out);
vxe_status vxe_render_frame_async(vxe_ctx* ctx, vxe_frame_out* out);
/* Same frame replayed from a CUDA graph captured on first use (per size). */
vxe_status vxe_render_frame_graph(vxe_ctx* ctx, vxe_frame_out* out);
vxe_status vxe_synchronize(vxe_ctx* ctx);

/* Hit record (no reference counterpart; defined by this project):
 *   node  = global arena index of the leaf that produced the hit, or
 *           VXE_INVALID_U32 for implicit-air grass hits and heightfield hits
 *   voxel = world voxel containing the hit point, clamped to the leaf cube
 *   face  = 0..5 (+X,-X,+Y,-Y,+Z,-Z) of the dominant normal axis, 255 = miss
 *   mat   = HitGeom.mat (chunk_trace.wgsl:15-32); 0 on miss               */
typedef struct vxe_hit {
  float t;
  uint32_t node;
  int32_t voxel[3];
  uint32_t face;
  uint32_t mat;
  uint32_t _pad;
} vxe_hit;

/* Ray queries (picking / physics): per-ray chunk-grid DDA over the resident
 * world, voxel geometry only, first hit within [0, tmax].  Host arrays of
 * n*3 floats; result written to host `out`.  The reference does this on the
 * CPU (app/app.rs:847-961). */
vxe_status vxe_trace_rays(vxe_ctx* ctx, const float* origins, const float* dirs, uint32_t n,
                          float tmax, vxe_hit* out);
/* Same, device pointers in and out, launched on the compute stream. */
vxe_status vxe_trace_rays_device(vxe_ctx* ctx, const float* d_origins, const float* d_dirs,
                                 uint32_t n, float tmax, vxe_hit* d_out);


/* Batched requests (no reference counterpart; the reference renders one
 * viewport per frame and answers picking queries on the CPU).  A viewport
 * request yields the primary hit records of a cold frame (the records
 * vxe_render_frame writes with VXE_FLAG_HIT_RECORDS on its first frame after
 * vxe_resize); a query request yields vxe_trace_rays records.  The world
 * (chunk_count, grid) is the context's: write it with vxe_write_camera first. */
enum { VXE_REQ_VIEWPORT = 0, VXE_REQ_QUERY = 1 };
typedef struct vxe_request {
  uint32_t kind;
  uint32_t width, height;      /* viewport: internal size = camera.render_present_px[0..1] */
  uint32_t ray_count;          /* query */
  vxe_camera_gpu camera;       /* viewport pose / projection */
  const float* d_origins;      /* query: device, 3 floats per ray */
  const float* d_dirs;         /* query: device, 3 floats per ray */
  float tmax;                  /* query */
  uint32_t _pad;
  vxe_hit* d_out;              /* device: width*height or ray_count records */
} vxe_request;

enum {
  VXE_BATCH_PERSISTENT = 0,    /* one persistent kernel over an atomic work queue */
  VXE_BATCH_PLAIN = 1,         /* one launch (or two) per request, back to back */
  VXE_BATCH_GRAPH = 2          /* the persistent launch replayed from a CUDA graph */
};
typedef struct vxe_batch_options {
  uint32_t tile_w, tile_h;     /* viewport work item: (tile_w * rays_per_thread) x tile_h pixels */
  uint32_t rays_per_thread;    /* 1..4; query work item = 128 * rays_per_thread rays */
  uint32_t mode;               /* VXE_BATCH_* */
} vxe_batch_options;

typedef struct vxe_batch_stats {
  double ms;                   /* device time of the batch (CUDA events) */
  uint64_t rays;               /* viewport pixels + query rays */
  uint32_t items, tiles;
} vxe_batch_stats;

#define VXE_MAX_BATCH_REQUESTS 256u
#define VXE_BATCH_LANES 4u
/* Traces n (<= VXE_MAX_BATCH_REQUESTS) requests; returns when they are done
 * (lane 0). */
vxe_status vxe_submit_batch(vxe_ctx* ctx, const vxe_request* reqs, uint32_t n, const vxe_batch_options* opt,
                            vxe_batch_stats* stats);
/* Asynchronous form: each of the VXE_BATCH_LANES lanes owns a stream, staging
 * and scratch, so up to that many batches are in flight and overlap on the
 * device.  vxe_batch_wait(block = 0) returns VXE_NOT_READY while the lane's
 * batch runs; after it returns VXE_OK the lane takes a new batch. */
vxe_status vxe_submit_batch_async(vxe_ctx* ctx, uint32_t lane, const vxe_request* reqs, uint32_t n,
                                  const vxe_batch_options* opt);
vxe_status vxe_batch_wait(vxe_ctx* ctx, uint32_t lane, int block, vxe_batch_stats* stats);

/* Viewport sessions (serving; no counterpart in the reference, whose
 * Renderer owns exactly one frame pipeline).  A view owns what one client's
 * frames carry from frame to frame -- internal and present images, the
 * primary-hit, shadow, local-light, godray and output histories and their
 * ping-pong state -- and renders from the context's world (arenas, grid,
 * clipmap, grass table).  A frame's working buffers (tile lists, shading
 * queues, grass probe and slab records) belong to the lane it renders on,
 * sized for the largest view that lane has rendered.  Its frames are
 * exactly the frames vxe_render_frame renders from the same camera sequence
 * after vxe_resize (render/state/mod.rs:297-308, 329-446).
 *   vxe_view_bytes          device bytes a view of that size holds (admission;
 *                           the lane's working buffers are not included)
 *   vxe_view_lane_bytes     device bytes of a lane's working buffers for
 *                           views up to that size
 *   vxe_view_create         allocates it (histories start at zero)
 *   vxe_view_render_async   one frame on a batch lane's stream; it may follow
 *                           a batch on the same lane, and vxe_batch_wait then
 *                           waits for both.  A view larger than any before on
 *                           that lane first waits for the lane and grows its
 *                           working buffers.  The camera's world fields
 *                           (chunk size and count, grid origin and dims) are
 *                           taken from the context's camera.
 *   vxe_view_read_image     waits for the view's last frame, copies an image
 *   vxe_view_destroy        frees it after its last frame (stream-ordered;
 *                           does not wait)
 * A view's images and a lane's buffers come from a stream-ordered pool of
 * the context: creating, growing and freeing them never waits for the
 * device.  A view rendered after vxe_set_flags changed the image flags
 * (VXE_FLAG_DEBUG_INTERMEDIATES, VXE_FLAG_HIT_RECORDS) is refused. */
typedef struct vxe_view vxe_view;
uint64_t vxe_view_bytes(const vxe_ctx* ctx, uint32_t present_w, uint32_t present_h, float render_scale);
uint64_t vxe_view_lane_bytes(const vxe_ctx* ctx, uint32_t present_w, uint32_t present_h, float render_scale);
vxe_status vxe_view_create(vxe_ctx* ctx, uint32_t present_w, uint32_t present_h, float render_scale,
                           vxe_view** out);
vxe_status vxe_view_render_async(vxe_ctx* ctx, vxe_view* view, uint32_t lane, const vxe_camera_gpu* camera);
/* One frame of each of n (<= VXE_MAX_VIEWS_PER_LAUNCH) distinct views on a
 * lane, every pass launched once for all of them: small views fill the GPU
 * together instead of one small launch after another.  Each view's frame is
 * the one vxe_view_render_async renders for the same camera; the lane holds
 * one set of working buffers per view of the launch. */
#define VXE_MAX_VIEWS_PER_LAUNCH 8u
vxe_status vxe_view_render_batch_async(vxe_ctx* ctx, vxe_view* const* views, const vxe_camera_gpu* cameras,
                                       uint32_t n, uint32_t lane);
vxe_status vxe_view_read_image(vxe_ctx* ctx, vxe_view* view, int image, void* host, size_t bytes);
vxe_status vxe_view_destroy(vxe_ctx* ctx, vxe_view* view);

/* GpuTimingsMs (render/state/mod.rs:22-31) minus blit; CUDA events of the last
 * frame.  local_taa and composite_taa are fused into primary / composite and
 * report 0.  Extra fields (no reference counterpart): primary_trace is the
 * trace kernel inside `primary` (the rest of `primary` is shading) and
 * grass_cells the per-frame grass cell table, which `tiles` includes. */
typedef struct vxe_timings {
  double primary, local_taa, godray, composite, composite_taa, tiles, total;
  /* extras: the trace stage of the wavefront schedule (walk, probe column
   * DDAs, slab marches, pick, resolve), the grass table build, and the walk
   * kernel (k_primary_trace) alone */
  double primary_trace, grass_cells, trace_kernel;
} vxe_timings;
vxe_status vxe_get_timings(vxe_ctx* ctx, vxe_timings* out);

/* Images that can be read / written for teacher-forced parity runs. */
typedef enum vxe_image {
  VXE_IMG_COLOR = 0, VXE_IMG_DEPTH = 1, VXE_IMG_LOCAL = 2,
  VXE_IMG_PRIMARY_HIST_IN = 3, VXE_IMG_PRIMARY_HIST_OUT = 4,
  VXE_IMG_SHADOW_IN = 5, VXE_IMG_SHADOW_OUT = 6,
  VXE_IMG_LOCAL_HIST_IN = 7, VXE_IMG_LOCAL_HIST_OUT = 8,
  VXE_IMG_GODRAY_IN = 9, VXE_IMG_GODRAY_OUT = 10,
  VXE_IMG_OUTPUT_PRE_TAA = 11, VXE_IMG_OUTPUT = 12,
  VXE_IMG_OUTPUT_HIST_IN = 13, VXE_IMG_OUTPUT_HIST_OUT = 14,
  VXE_IMG_HITS = 15,
  VXE_IMG_COUNT = 16
} vxe_image;
/* "IN" = the history the next frame reads, "OUT" = the one it writes. */
vxe_status vxe_image_size(const vxe_ctx* ctx, vxe_image img, size_t* bytes);
vxe_status vxe_read_image(vxe_ctx* ctx, vxe_image img, void* host, size_t bytes);
/* Asynchronous read-back (none in the reference, whose output goes to the
 * swapchain; the pipelined counterpart of vxe_read_image): queues a copy of
 * `img` -- as the frames queued so far leave
 * it -- into `host` on a copy stream and returns a ticket.  The next frame's
 * write of that image waits for the copy: for VXE_IMG_OUTPUT only its final
 * composite pass does, so the copy overlaps that frame's earlier passes; for
 * any other image the whole next frame does.  `host` must stay valid until
 * the copy has landed; pinned memory (cudaHostAlloc) makes the copy
 * asynchronous.  vxe_read_image_wait blocks until the copy of `ticket` has
 * landed; vxe_synchronize waits for all of them. */
vxe_status vxe_read_image_async(vxe_ctx* ctx, vxe_image img, void* host, size_t bytes, uint64_t* ticket);
vxe_status vxe_read_image_wait(vxe_ctx* ctx, uint64_t ticket);
vxe_status vxe_write_image(vxe_ctx* ctx, vxe_image img, const void* host, size_t bytes);

/* Device error word (bounds checks / bounded waits); cleared on read. */
vxe_status vxe_read_error_word(vxe_ctx* ctx, uint32_t* word);

/* Primary-pass work counters (ray_main.wgsl:32-74, binding 17
 * `profile_counts`): while the camera's profile_flags has bit 0 set, each
 * frame of the context adds, per pixel, what main_primary's profile_inc /
 * profile_add calls add -- VOXEL: the tile's candidate count per voxel trace
 * phase run; GRASS: 1 per grass-slab refinement that hit; HDR: 1 per
 * heightfield shade, 2 per voxel shade; FOG: fog_profile_weight(t) per shaded
 * pixel; SHADOW: 2 per fresh sun shadow, 1 per reused one.  The counts
 * accumulate over frames until reset.
 *   vxe_reset_profile_counts  Renderer::reset_primary_profile_counts
 *                             (render/state/mod.rs:448-455); ordered after the
 *                             frames already enqueued
 *   vxe_read_profile_counts   Renderer::encode_primary_profile_readback +
 *                             read_primary_profile_counts_blocking
 *                             (render/state/mod.rs:457-491); waits for the
 *                             context's frames */
#define VXE_PROFILE_COUNT 5u
enum { VXE_PROFILE_VOXEL = 0, VXE_PROFILE_GRASS = 1, VXE_PROFILE_HDR = 2, VXE_PROFILE_FOG = 3,
       VXE_PROFILE_SHADOW = 4 };
vxe_status vxe_reset_profile_counts(vxe_ctx* ctx);
vxe_status vxe_read_profile_counts(vxe_ctx* ctx, uint32_t counts[VXE_PROFILE_COUNT]);

/* Wavefront record limits (no reference counterpart).  The trace stage
 * stores every grass-column probe the voxel walk meets and every grass slab a
 * probe's column DDA finds, and marches them in kernels of their own; a pixel
 * whose records do not all fit walks again with the probes inline (the
 * reference's order), with the same result.  These cap the records stored
 * per frame or batch below the buffers' sizes (0 = the buffer size): a knob
 * for tests of the re-walk path and for runs with smaller buffers. */
vxe_status vxe_set_record_limits(vxe_ctx* ctx, uint32_t probe_records, uint32_t slab_tasks);

/* Work counts of the context's last frame (no reference counterpart; waits
 * for the frame).  Wavefront schedule only: zeros with
 * VXE_FLAG_PRIMARY_MEGAKERNEL. */
typedef struct vxe_frame_stats {
  uint32_t voxel_pixels;    /* pixels shaded as voxel hits */
  uint32_t far_pixels;      /* pixels shaded as heightfield or sky */
  uint32_t probes;          /* grass-column probes the walk met (stored or not) */
  uint32_t pending_pixels;  /* pixels whose walk met probes */
  uint32_t slab_tasks;      /* grass slabs found by the probes' column DDAs */
  uint32_t slab_hits;       /* slabs whose march hit */
  uint32_t rewalk_pixels;   /* pending pixels walked again with inline probes */
  uint32_t full_trace_pixels; /* pixels whose walk ran the full trace (no valid
                                 history hint, or nothing in its window) */
} vxe_frame_stats;
vxe_status vxe_get_frame_stats(vxe_ctx* ctx, vxe_frame_stats* out);

/* Scene buffers the caller already holds on the device, in the layouts of the
 * structs above (used by vxe_trace_primary_hits_noalloc). */
typedef struct vxe_scene_view {
  const vxe_node* nodes;          /* node_count NodeGpu records                 */
  const vxe_node_ropes* ropes;    /* node_count NodeRopesGpu records            */
  uint64_t node_count;
  const vxe_chunk_meta* metas;    /* chunk_capacity slots                       */
  const uint32_t* macro_words;    /* chunk_capacity * 16                        */
  const uint32_t* colinfo_words;  /* chunk_capacity * 2048                      */
  uint32_t chunk_capacity;
  uint32_t grid_cells;            /* cells of `grid`                            */
  const uint32_t* grid;
  const float* clip_tex;          /* clip_layers * clip_res^2 R32F, or NULL     */
  uint32_t clip_layers, clip_res;
} vxe_scene_view;

/* No reference counterpart.  Primary hit records of one cold frame (no history
 * hint), identical to the records vxe_render_frame writes with
 * VXE_FLAG_HIT_RECORDS on the first frame after vxe_resize, for callers that
 * must not allocate device memory: hosts whose frame loop runs under an
 * allocation-free policy, and engines whose device memory all comes from their
 * own allocator (for example buffers shared with a graphics API), where a
 * cudaMalloc from inside a plugin is not allowed.  It allocates nothing: its
 * scratch (per-tile candidate lists and a device error word) is a fixed
 * file-scope device array of VXE_NOALLOC_MAX_TILES tiles, which every GPU that
 * loads the library holds until exit.  Internal sizes whose tile count
 * (ceil(w/8) * ceil(h/8)) exceeds the maximum return VXE_ERR_CAPACITY.
 *   scene / cam / clip: host structs; the buffers inside `scene` and `d_hits`
 *     (w*h records, w,h = cam->render_present_px[0..1]) are device pointers.
 *   stream: a cudaStream_t (NULL = legacy default stream).  The call returns
 *     after the work on `stream` has finished.
 * The first call on a device resolves the scratch address on that device (so
 * does the first call after the device's context was re-created, e.g. after
 * cudaDeviceReset) and should come before any stream capture.  A CUDA error
 * already pending on the calling thread is reported as VXE_ERR_DEVICE before
 * anything is launched, and left pending.  Calls share the one scratch array,
 * so calls that overlap on the GPU (different streams, threads or devices
 * sharing a context) race; serialise them. */
#define VXE_NOALLOC_MAX_TILES 36864u
vxe_status vxe_trace_primary_hits_noalloc(const vxe_scene_view* scene, const vxe_camera_gpu* cam,
                                          const vxe_clipmap_gpu* clip, vxe_hit* d_hits, void* stream);

/* Diagnostic (no reference counterpart): evaluates the deterministic math
 * of detmath.h on the device for n host inputs; which = 0 sin, 1 cos, 2 exp,
 * 3 pow(x, y), 4 min(x, y), 5 max(x, y).  Used to prove host/device bit
 * equality of the functions every pass depends on. */
vxe_status vxe_debug_detmath(int which, const float* x, const float* y, float* out, uint32_t n);

/* Diagnostic (no reference counterpart): the grass blade march on the device
 * for n host inputs, without the per-frame cell table.  which = 0:
 * try_grass_slab_hit (grass.wgsl:494-538), 17 floats per input (ray origin
 * and direction, t_min, t_max, cell minimum corner, cell id, voxel size, wind
 * time, wind strength) -> 5 floats (hit, t, normal); which = 1:
 * grass_sdf_lod (grass.wgsl:192-350), 13 floats per input (point, cell
 * minimum corner, cell id, voxel size, wind time, wind strength, lod) -> 1
 * float.  Used to compare the march with the CPU restatement input by input. */
vxe_status vxe_debug_grass(int which, uint32_t n, const float* in, float* out);

/* Diagnostic (no reference counterpart): the device's L2 read bandwidth, the
 * roof of kernels whose working set stays in L2 (the world's node, rope,
 * meta, macro and colinfo records).  Reads an L2-resident buffer of `bytes`
 * (a few tens of MB; allocated and freed by the call) with 16-byte loads,
 * `launches` times after three warm-up launches; *gbs = bytes read / time
 * (CUDA events). */
vxe_status vxe_measure_l2_bandwidth(int device, uint64_t bytes, uint32_t launches, double* gbs);

/* ------------------------------------------------------------------------ */
/* Producer side (C++ port of src/svo, streaming meta, clipmap, camera)      */
/* ------------------------------------------------------------------------ */

/* Seeded synthetic world used for every benchmark configuration (the
 * reference's Perlin worldgen is replaced by project value noise). */
typedef struct vxe_world_params {
  uint32_t seed;
  int32_t height_min;       /* surface voxel y range [min, max] */
  int32_t height_max;
  int32_t dirt_depth;       /* dirt voxels below grass; also builder dirt_depth */
  uint32_t carve_mod;       /* solid voxel -> air when hash3 % carve_mod == 0 (0 = off) */
  float cave_threshold;     /* 3D value noise > threshold -> air (>= 1 = off) */
  float height_scale_vox;   /* lattice spacing of the height noise octave 0 */
  uint32_t features;        /* bit0 trees (wood+leaf), bit1 light voxels */
} vxe_world_params;

/* Physics solidity (ChunkManagerQuery::solid_voxel_at, physics/world_query.rs:
 * 80-112; the reference answers it on the CPU): for n voxel coordinates
 * (x, y, z int32 triples, device memory) out[i] = 1 when solid.  A voxel of a
 * chunk in the context's grid is solid at or below its column's colinfo top
 * (empty column: never); elsewhere, with `world` non-null, at or below the
 * seeded heightfield (the reference's fallback while a chunk streams in),
 * else 0.  Launched on the compute stream.  The reference consults every
 * resident or uploading chunk; here the chunks of the grid window. */
vxe_status vxe_solid_voxels_device(vxe_ctx* ctx, const int32_t* d_vox, uint32_t n, const vxe_world_params* world,
                                   uint8_t* d_out);

/* Chunk builder on the device.  The reference builds chunks on CPU worker
 * threads (build_chunk_svo_sparse_cancelable_with_scratch, svo/builder.rs:
 * 846-986, called from streaming/build_pool.rs:19-25); this runs the same
 * pipeline -- material fill, colinfo, macro bits, ground min-mip, octree with
 * stone / uniform collapse, ropes -- for n chunks at once and writes, for
 * chunk i of the n chunk coordinates (int32 x, y, z triples), exactly the
 * records vxe_build_chunk returns:
 *   d_nodes[i*node_cap ...], d_ropes[i*node_cap ...]   node_count records
 *   d_macro[i*16 ...], d_colinfo[i*2048 ...]
 *   d_counts[2i] = node_count, d_counts[2i+1] = solid_voxels.
 * All buffers are device memory.  A chunk whose node_count exceeds node_cap
 * gets its counts, macro and colinfo words but no nodes or ropes: build it
 * again with a larger cap (VXE_BUILD_NODE_CAP_MAX always fits; node_cap 0
 * only counts).  Launched on the context's world-write stream;
 * vxe_synchronize waits for it. */
#define VXE_BUILD_NODE_CAP_MAX 299593u /* 1 + 8 + 8^2 + ... + 8^6 */
#define VXE_BUILD_BATCH_MAX 2048u
vxe_status vxe_build_chunks_device(vxe_ctx* ctx, const vxe_world_params* world, const int32_t* d_coords, uint32_t n,
                                   uint32_t node_cap, vxe_node* d_nodes, vxe_node_ropes* d_ropes, uint32_t* d_macro,
                                   uint32_t* d_colinfo, uint32_t* d_counts);
/* Resident chunk builds: the same builder writing straight into the
 * context's world -- the device counterpart of building on the CPU and then
 * uploading (streaming/build_pool.rs -> streaming/upload.rs, ChunkUpload,
 * streaming/types.rs:87-103).  For each place: nodes and ropes at
 * [node_base, node_base + node_count), macro words at slot * 16, colinfo
 * words at slot * 2048 and the slot's meta record (origin, node_base, the
 * built node count, macro / colinfo bases, macro_empty).  node_count reserves
 * the arena range: take it from a counting build (vxe_build_chunks_device
 * with node_cap 0).  A chunk that needs more nodes than reserved gets no
 * nodes, an empty meta (node_count 0, macro_empty 1) and error word bit
 * VXE_ERR_WORD_BUILD.  Ordered like vxe_upload_chunks (after the frames and
 * batches in flight unless VXE_FLAG_UPLOADS_UNORDERED), with the same grass
 * table and light flag refresh of the written slots; the grid is written
 * with vxe_write_grid as for uploads. */
typedef struct vxe_build_place {
  int32_t cx, cy, cz;
  uint32_t slot;
  uint32_t node_base;
  uint32_t node_count;
} vxe_build_place;
#define VXE_ERR_WORD_BUILD (1u << 7)
vxe_status vxe_build_chunks_resident(vxe_ctx* ctx, const vxe_world_params* world, const vxe_build_place* places,
                                     uint32_t n);
/* Dense-slot moves on the device (the slot compaction of
 * streaming/manager/slots.rs:163-766: unloading a chunk moves the last slot
 * into its hole).  Moves run in order; each copies the slot's meta record
 * (macro / colinfo bases rewritten for the new slot), its 16 macro words and
 * 2048 colinfo words; node data stays where the arena holds it.  With
 * resident builds this keeps a streamed world entirely on the device (only
 * node counts come back to the host).  Ordered like vxe_upload_chunks, with
 * the grass / light refresh of the destination slots; the grid follows with
 * vxe_write_grid. */
typedef struct vxe_slot_move {
  uint32_t from, to;
} vxe_slot_move;
#define VXE_MOVE_SLOTS_MAX 4096u
vxe_status vxe_move_slots(vxe_ctx* ctx, const vxe_slot_move* moves, uint32_t n);
/* Device time (ms) of the last vxe_build_chunks_device / _resident call's kernels. */
typedef struct vxe_build_timings {
  double columns; /* ground, materials, colinfo, level-5 cell states */
  double svo;     /* octree levels 4..0, offsets, nodes, ropes, macro bits */
} vxe_build_timings;
vxe_status vxe_get_build_timings(vxe_ctx* ctx, vxe_build_timings* out);

typedef struct vxe_built_chunk {
  vxe_node* nodes;
  vxe_node_ropes* ropes;
  uint32_t node_count;
  uint32_t macro_words[VXE_MACRO_WORDS_PER_CHUNK];
  uint32_t colinfo_words[VXE_COLINFO_WORDS_PER_CHUNK];
  uint32_t solid_voxels;
} vxe_built_chunk;

/* build_chunk_svo_sparse_cancelable_with_scratch (svo/builder.rs:846-986). */
vxe_status vxe_build_chunk(const vxe_world_params* wp, int32_t cx, int32_t cy, int32_t cz,
                           vxe_built_chunk* out);
void vxe_free_chunk(vxe_built_chunk* c);
/* Dense material grid (layout y*64*64 + z*64 + x, svo/builder.rs:528-668). */
vxe_status vxe_chunk_materials(const vxe_world_params* wp, int32_t cx, int32_t cy, int32_t cz,
                               uint8_t* out_64cubed);
/* Ground height (surface voxel y) at a world voxel column. */
int32_t vxe_ground_height(const vxe_world_params* wp, int32_t wx, int32_t wz);

/* Build the SVO + ropes + macro + colinfo from a caller material grid. */
vxe_status vxe_build_from_materials(const uint8_t* material_64cubed, int32_t chunk_oy,
                                    const int32_t* ground_64x64, int32_t dirt_depth,
                                    vxe_built_chunk* out);

/* Camera packing (app/app.rs:411-511, app/camera.rs:95-111), double math
 * rounded to f32. */
typedef struct vxe_camera_params {
  float pos[3];
  float yaw, pitch;
  float fovy_rad, z_near, z_far;
  uint32_t present_w, present_h, internal_w, internal_h;
  uint32_t frame_index;
  uint32_t jitter;            /* 1 = halton(frame+1)-0.5 sub-pixel jitter */
  float time_s;
  uint32_t chunk_count;
  int32_t grid_origin_chunk[3];
  uint32_t grid_dims[3];
  uint32_t has_prev;          /* 0 -> prev_view_proj = view_proj */
  float prev_view_proj[4][4];
} vxe_camera_params;
vxe_status vxe_build_camera(const vxe_camera_params* p, vxe_camera_gpu* out);

/* Toroidal clipmap (clipmap.rs:182-577).  State lives in an opaque handle. */
typedef struct vxe_clipmap_state vxe_clipmap_state;
vxe_clipmap_state* vxe_clipmap_new(const vxe_world_params* wp, uint32_t levels, uint32_t res,
                                   float base_cell_m);
void vxe_clipmap_free(vxe_clipmap_state* s);
/* Computes the new params and patches for camera (x,z).  Patch data pointers
 * stay valid until the next update / free. */
vxe_status vxe_clipmap_update(vxe_clipmap_state* s, float cam_x, float cam_z,
                              vxe_clipmap_gpu* params, const vxe_clip_patch** patches,
                              uint32_t* n_patches);

/* A patch's placement without its texels: storage rectangle (as
 * vxe_clip_patch), first logical texel, and the level's origin and cell. */
typedef struct vxe_clip_patch_geom {
  uint32_t level, x, y, w, h;
  uint32_t lx0, lz0;
  float ox_m, oz_m, cell_m;
} vxe_clip_patch_geom;
#define VXE_CLIP_PATCHES_MAX 64 /* at most 4 per level (two wrapped strips per axis) */
/* vxe_clipmap_update's state step without evaluating texels: the params, the
 * patches' geometry and the world parameters the texels come from.  Geometry
 * stays valid until the next update / plan / free. */
vxe_status vxe_clipmap_plan(vxe_clipmap_state* s, float cam_x, float cam_z, vxe_clipmap_gpu* params,
                            const vxe_clip_patch_geom** geoms, uint32_t* n_geoms, vxe_world_params* world);
/* Clipmap patch generation on the device (no reference counterpart: the
 * reference computes patches on the CPU, clipmap.rs:182-577, and uploads them
 * with write_clipmap_updates): vxe_clipmap_plan, then the patches' texels are
 * evaluated by a kernel straight into the context's clipmap texture on the
 * upload stream, ordered like vxe_write_clipmap, and the params become the
 * context's clipmap uniform.  The texels equal vxe_clipmap_update's bit for
 * bit; no host texel data, no host-to-device copy. */
vxe_status vxe_clipmap_update_device(vxe_ctx* ctx, vxe_clipmap_state* s, float cam_x, float cam_z);
/* Copies the context's clipmap texture (levels x res x res floats) to host
 * memory, after the writes queued so far. */
vxe_status vxe_read_clipmap(vxe_ctx* ctx, float* host, size_t bytes);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* VXE_VXE_H */
