"""Translates the reference's WGSL shader functions into C++ (test
infrastructure for pinning the oracle; never part of the product).

The reference is Rust + WGSL: its shaders cannot run here (no graphics stack)
and its host cannot be built (no Rust toolchain).  Most of its shader code is
plain f32 / u32 arithmetic over structs and read-only storage buffers, though,
and WGSL's syntax for it is close to C++.  This script rewrites the functions
in EXPORTS, with their whole call closure, mechanically and at build time from
the shader sources where they lie, into oracle/_ref/ref_wgsl.cpp over
oracle/wgsl_shim.h (vector and matrix types, builtins with WGSL semantics,
storage buffers that read zero past their end), and compiles that into
oracle/_ref/libref_wgsl.so.  Nothing of the reference is committed:
oracle/_ref is git-ignored.  The rewrite is textual: declarations (let / var /
const), types, struct definitions and constructors (brace initialisation),
function pointers (`ptr<function, T>` -> `T*`), conversions, swizzles (.xy
.xz .xyz), f32 literals, and the scene bindings as globals.

The library exports
    int ref_wgsl_eval(const char* name, const float* in, float* out, unsigned n)
    int ref_wgsl_widths(const char* name, unsigned* in_w, unsigned* out_w)
    void ref_wgsl_set_cam(const float* cam_pos4, const float* voxel_params4)
over the exported functions with scalar and vector parameters: parameters
and results are flattened into float slots (vecN = N slots; u32 / i32 / bool
pass their bit patterns), n calls in a row; and, for the chunk walk,
    void ref_wgsl_set_scene(...)   (the world's host arrays and camera fields)
    int ref_wgsl_trace_chunk(const float* rays, float* out, unsigned n)
and for whole frames of the five compute passes,
    void ref_wgsl_set_clip(...)    (the clipmap uniform and layers)
    int ref_wgsl_primary_tile(uint32_t tx, uint32_t ty, float* out)
    int ref_wgsl_frame(uint32_t iw, uint32_t ih, uint32_t pw, uint32_t ph, float* const* images,
                       uint32_t threads)
The oracle exports the same interfaces over its own restatements
(oracle_shading_eval, ora_scene_eval, ora_trace_chunk, ora_primary_tile;
its frames through ora_render_frame), so a test compares the two.

Usage: python oracle/wgsl_to_cpp.py <reference shader dir> <out .cpp>
"""
from __future__ import annotations

import re
import sys
from pathlib import Path

FILES = ["common.wgsl", "ray/wind.wgsl", "ray/phase.wgsl", "ray/fog.wgsl", "ray/clouds.wgsl", "ray/sky.wgsl",
         "ray/composite.wgsl", "ray/grass.wgsl", "ray/shading.wgsl", "ray/godrays.wgsl", "ray/light.wgsl",
         "ray/aabb.wgsl", "ray/svo_query.wgsl", "ray/leaves.wgsl", "clipmap.wgsl", "ray/chunk_trace.wgsl",
         "ray/shadows.wgsl", "ray_main.wgsl", "taa.wgsl"]

# The functions the pin compares (each with its whole call closure).
EXPORTS = ["hash_u32", "hash12", "hash31", "value_noise", "fbm", "hash1", "wind_field", "clamp_len",
           "grass_wind_xz", "grass_blade_params", "sdf_box", "phase_mie", "phase_blended", "sky_bg", "sky_sun",
           "sky_color", "fog_color_from_sky", "fog_inscatter", "fog_optical_depth_with_base",
           "fog_transmittance_primary", "fog_transmittance_godray", "apply_fog", "cloud_height01",
           "cloud_coverage_at_xz", "cloud_density", "cloud_light_transmittance", "cloud_sun_transmittance_fast",
           "cloud_density_godray", "cloud_sun_transmittance_godray", "tonemap_filmic_hable",
           "tonemap_filmic_white_scale", "gamma_encode", "bright_extract_hue", "intersect_aabb", "safe_inv",
           "ray_eps_vec", "macro_cell_size", "grass_lod_from_t", "hemi_ambient", "color_for_material",
           "apply_material_variation", "grass_wind_dir_xz", "grass_blade_slivers", "grass_blade_field",
           "grass_top_albedo", "base_albedo", "material_roughness", "material_f0", "material_emission",
           "approx_pow_0p75", "approx_pow_0p55", "exp_neg_fast", "godray_steps_for_tend", "godray_decompress",
           "godray_compress", "rot_about_axis", "sphere_dir_local", "trace_chunk_interval_stream_macro",
           "sun_transmittance_geom_only", "godray_integrate_1", "gather_voxel_lights", "query_leaf_world",
           "clip_trace_heightfield", "clip_height_at_level", "clip_height_at_level_nearest",
           "tile_append_candidates_for_ray", "tile_sort_candidates_by_enter", "trace_scene_voxels_candidates",
           "ray_dir_from_pixel", "main_primary", "main_local_taa", "main_godray", "main_composite",
           "main_composite_taa"]

# The chunk walk (chunk_trace.wgsl, trace_chunk_interval_stream_macro) over a
# world the caller holds in host memory, in the layouts of include/vxe/vxe.h
# (which are the shader's structs byte for byte).
#   rays: n x 12 slots: ro (3), rd (3), t0, t1, slot (u32), use_anchor (u32),
#         anchor_key (u32), unused
#   out:  n x 16 slots: hit (u32), mat (u32), t, n (3), root_bmin (3),
#         root_size, node_base (u32), macro_base (u32), anchor_valid (u32),
#         anchor_key (u32), two unused
CHUNK_WALK_EXPORT = r"""
static_assert(sizeof(Node) == 16 && sizeof(NodeRopes) == 32 && sizeof(ChunkMeta) == 48, "buffer layouts");
extern "C" void ref_wgsl_set_scene(const void* chunk_metas, uint64_t chunks_n, const void* node_recs, uint64_t nodes_n,
                                   const uint32_t* grid, uint64_t grid_n, const uint32_t* macro_words,
                                   uint64_t macro_n, const void* rope_recs, uint64_t ropes_n,
                                   const uint32_t* colinfo_words, uint64_t colinfo_n, const vxe_camera_gpu* c) {
  wgsl::chunks = Buf<ChunkMeta>{(const ChunkMeta*)chunk_metas, chunks_n};
  wgsl::nodes = Buf<Node>{(const Node*)node_recs, nodes_n};
  wgsl::chunk_grid = Buf<uint32_t>{grid, grid_n};
  wgsl::macro_occ = Buf<uint32_t>{macro_words, macro_n};
  wgsl::node_ropes = Buf<NodeRopes>{(const NodeRopes*)rope_recs, ropes_n};
  wgsl::chunk_colinfo = Buf<uint32_t>{colinfo_words, colinfo_n};
  for (int i = 0; i < 4; ++i) {
    for (int j = 0; j < 4; ++j) {
      cam.view_inv.c[i][j] = c->view_inv[i][j];
      cam.proj_inv.c[i][j] = c->proj_inv[i][j];
      cam.view_proj.c[i][j] = c->view_proj[i][j];
      cam.prev_view_proj.c[i][j] = c->prev_view_proj[i][j];
    }
    cam.cam_pos[i] = c->cam_pos[i];
    cam.ray00[i] = c->ray00[i];
    cam.ray_dx[i] = c->ray_dx[i];
    cam.ray_dy[i] = c->ray_dy[i];
    cam.voxel_params[i] = c->voxel_params[i];
    cam.grid_origin_chunk[i] = c->grid_origin_chunk[i];
    cam.grid_dims[i] = c->grid_dims[i];
    cam.render_present_px[i] = c->render_present_px[i];
  }
  cam.chunk_size = c->chunk_size;
  cam.chunk_count = c->chunk_count;
  cam.max_steps = c->max_steps;
  cam.frame_index = c->frame_index;
  cam.profile_flags = c->profile_flags;
}
static_assert(sizeof(ClipmapParams) == 528, "clipmap uniform layout");
extern "C" void ref_wgsl_set_clip(const void* params528, const float* texels, int32_t res, int32_t layers) {
  std::memcpy(&clip, params528, sizeof clip);
  clip_height = Tex2DArrayF{texels, res, layers};
}
extern "C" int ref_wgsl_trace_chunk(const float* rays, float* out, unsigned n) {
  for (unsigned k = 0; k < n; ++k) {
    const float* p = rays + (size_t)k * 12;
    float* o = out + (size_t)k * 16;
    const vec3f ro = get_v<3>(p), rd = get_v<3>(p);
    const float t0 = get_f(p), t1 = get_f(p);
    const uint32_t slot = get_slot<uint32_t>(p), use_anchor = get_slot<uint32_t>(p), key = get_slot<uint32_t>(p);
    const vec3f inv = vec3f(safe_inv(rd.x), safe_inv(rd.y), safe_inv(rd.z));
    const ChunkTraceResult r = trace_chunk_interval_stream_macro(ro, rd, inv, wgsl::chunks[slot], t0, t1,
                                                                 use_anchor != 0u, key, 0u);
    put(o, r.hit.hit);
    put(o, r.hit.mat);
    put(o, r.hit.t);
    put(o, r.hit.n);
    put(o, r.hit.root_bmin);
    put(o, r.hit.root_size);
    put(o, r.hit.node_base);
    put(o, r.hit.macro_base);
    put(o, (uint32_t)(r.anchor_valid ? 1u : 0u));
    put(o, r.anchor_key);
    put(o, 0.0f);
    put(o, 0.0f);
  }
  return 0;
}
// The cold primary voxel trace of the 64 pixels of tile (tx, ty): the tile's
// candidate list built as main_primary's lane 0 builds it
// (ray_main.wgsl:179-197), then each pixel's
// trace_scene_voxels_candidates(ro, rd, 0, FOG_MAX_DIST, no anchor)
// (ray_main.wgsl:148-158).  out: 64 x 16 slots per tile, row-major pixels:
// in_grid (u32), hit (u32), mat (u32), t, n (3), root_bmin (3), root_size,
// t_exit, anchor_valid (u32), anchor_key (u32), anchor_chunk.xy (i32);
// returns the tile's candidate count.
extern "C" int ref_wgsl_primary_tile(uint32_t tx, uint32_t ty, float* out) {
  atomicStore(&WG_TILE_COUNT, 0u);
  if (cam.chunk_count != 0u) {
    const vec2f tile_base = vec2f(wgsl_f32(tx * TILE_SIZE), wgsl_f32(ty * TILE_SIZE));
    const vec3f ro_tile = cam.cam_pos.xyz();
    vec2f px = tile_base + vec2f(4.5f, 4.5f);
    tile_append_candidates_for_ray(ro_tile, ray_dir_from_pixel(px), 0.0f, FOG_MAX_DIST);
    px = tile_base + vec2f(1.5f, 1.5f);
    tile_append_candidates_for_ray(ro_tile, ray_dir_from_pixel(px), 0.0f, FOG_MAX_DIST);
  }
  const uint32_t raw_count = min(atomicLoad(&WG_TILE_COUNT), MAX_TILE_CHUNKS);
  tile_sort_candidates_by_enter(raw_count);
  const uint32_t count = min(raw_count, PRIMARY_MAX_TILE_CHUNKS);
  for (uint32_t k = 0; k < 64u; ++k) {
    const uint32_t gx = tx * 8u + (k & 7u), gy = ty * 8u + (k >> 3);
    const vec2f px = vec2f(wgsl_f32(gx) + 0.5f, wgsl_f32(gy) + 0.5f);
    const uint32_t seed = (gx * 1973u) ^ (gy * 9277u) ^ (cam.frame_index * 26699u);
    const VoxTraceResult r = trace_scene_voxels_candidates(cam.cam_pos.xyz(), ray_dir_from_pixel(px), 0.0f,
                                                           FOG_MAX_DIST, false, vec3i(0), INVALID_U32, count, seed);
    float* o = out + (size_t)k * 16;
    put(o, (uint32_t)(r.in_grid ? 1u : 0u));
    put(o, r.best.hit);
    put(o, r.best.mat);
    put(o, r.best.t);
    put(o, r.best.n);
    put(o, r.best.root_bmin);
    put(o, r.best.root_size);
    put(o, r.t_exit);
    put(o, (uint32_t)(r.anchor_valid ? 1u : 0u));
    put(o, r.anchor_key);
    put(o, r.anchor_chunk.x);
    put(o, r.anchor_chunk.y);
  }
  return (int)count;
}
"""

# One cold frame of the reference's compute passes in the order
# Renderer::encode_compute runs them (render/state/mod.rs:329-446):
# main_primary, main_local_taa, main_godray, main_composite,
# main_composite_taa, each over every pixel of its image; a workgroup of
# main_primary runs its 64 lanes one after another, lane 0 first, so the tile
# list lane 0 builds is there for the others (the barriers have nothing to
# wait for).  The images are the caller's host arrays, wired as the frame's
# bind groups wire them (render/state/bindgroups.rs): the godray and local
# TAA passes write their "out" images, which the composite reads.  The
# history inputs are the caller's (zero on a cold frame).  With more than one
# host thread each thread runs whole workgroups (workgroup memory is
# thread-local); the work counters of profile_flags are plain increments there,
# so they are exact only on one thread (the bench and the pin keep them off).
#   img[0..15]: color, depth, local, primary_hist_in, primary_hist_out,
#   shadow_hist_in, shadow_hist_out (buffer, rows padded to 256 B),
#   local_hist_in, local_hist_out, godray_hist_in, godray_out, pre_taa,
#   output_hist_in, output, output_hist_out (internal iw x ih, present
#   pw x ph)
FRAME_EXPORT = r"""
// Runs body(row) for rows [0, rows) on `threads` host threads (interleaved).
template <class F>
static void parallel_rows(uint32_t rows, uint32_t threads, F body) {
  if (threads <= 1u) {
    for (uint32_t r = 0; r < rows; ++r) body(r);
    return;
  }
  std::vector<std::thread> pool;
  for (uint32_t t = 0; t < threads; ++t)
    pool.emplace_back([=] {
      for (uint32_t r = t; r < rows; r += threads) body(r);
    });
  for (auto& th : pool) th.join();
}
// The work counters of main_primary (profile_counts: VOXEL, GRASS, HDR, FOG,
// SHADOW), accumulated while cam.profile_flags & 1; read into out5 and
// cleared.
extern "C" void ref_wgsl_take_profile(uint32_t* out5) {
  for (int i = 0; i < 5; ++i) {
    out5[i] = profile_counts.counts[i].v;
    profile_counts.counts[i].v = 0u;
  }
}
extern "C" int ref_wgsl_frame(uint32_t iw, uint32_t ih, uint32_t pw, uint32_t ph, float* const* img,
                              uint32_t threads) {
  auto t4 = [](float* p, uint32_t w, uint32_t h) { return Tex2D{p, (int32_t)w, (int32_t)h, 4}; };
  auto t1 = [](float* p, uint32_t w, uint32_t h) { return Tex2D{p, (int32_t)w, (int32_t)h, 1}; };
  color_img = t4(img[0], iw, ih);
  depth_img = t1(img[1], iw, ih);
  local_img = t4(img[2], iw, ih);
  primary_hist_tex = t4(img[3], iw, ih);
  primary_hist_out = t4(img[4], iw, ih);
  shadow_hist_in = t1(img[5], iw, ih);
  const uint64_t stride = (((uint64_t)iw * 4u + 255u) & ~(uint64_t)255u) / 4u;
  shadow_hist_out = RWBuf<float>{img[6], stride * ih};
  local_in_tex = t4(img[2], iw, ih);
  local_hist_in_tex = t4(img[7], iw, ih);
  local_hist_out = t4(img[8], iw, ih);
  depth_tex = t1(img[1], iw, ih);
  godray_hist_tex = t4(img[9], iw, ih);
  godray_out = t4(img[10], iw, ih);
  color_tex = t4(img[0], iw, ih);
  godray_tex = t4(img[10], iw, ih);
  out_img = t4(img[11], pw, ph);
  depth_full = t1(img[1], iw, ih);
  local_hist_tex = t4(img[8], iw, ih);
  composite_in_tex = t4(img[11], pw, ph);
  depth_full_tex = t1(img[1], iw, ih);
  hist_in_tex = t4(img[12], pw, ph);
  output_tex = t4(img[13], pw, ph);
  hist_out_tex = t4(img[14], pw, ph);
  parallel_rows((ih + 7u) / 8u, threads, [&](uint32_t wy) {
    for (uint32_t wx = 0; wx < (iw + 7u) / 8u; ++wx)
      for (uint32_t lid = 0; lid < 64u; ++lid)
        main_primary(vec3u(wx * 8u + (lid & 7u), wy * 8u + (lid >> 3), 0u), lid, vec3u(wx, wy, 0u));
  });
  parallel_rows(ih, threads, [&](uint32_t y) {
    for (uint32_t x = 0; x < iw; ++x) main_local_taa(vec3u(x, y, 0u));
  });
  // The godray pass binds scene_bg (render/state/bindgroups.rs:120-156):
  // macro_occ at binding 8, node_ropes at 9, colinfo at 10, while the shader
  // declares macro_occ at 9, node_ropes at 10 and chunk_colinfo at 11.
  const Buf<uint32_t> macro_keep = wgsl::macro_occ;
  const Buf<NodeRopes> ropes_keep = wgsl::node_ropes;
  const Buf<uint32_t> colinfo_keep = wgsl::chunk_colinfo;
  wgsl::macro_occ = Buf<uint32_t>{(const uint32_t*)ropes_keep.p, ropes_keep.n * 8u};
  wgsl::node_ropes = Buf<NodeRopes>{(const NodeRopes*)colinfo_keep.p, colinfo_keep.n / 8u};
  wgsl::chunk_colinfo = Buf<uint32_t>{};
  parallel_rows(ih, threads, [&](uint32_t y) {
    for (uint32_t x = 0; x < iw; ++x) main_godray(vec3u(x, y, 0u));
  });
  wgsl::macro_occ = macro_keep;
  wgsl::node_ropes = ropes_keep;
  wgsl::chunk_colinfo = colinfo_keep;
  parallel_rows(ph, threads, [&](uint32_t y) {
    for (uint32_t x = 0; x < pw; ++x) main_composite(vec3u(x, y, 0u));
  });
  parallel_rows(ph, threads, [&](uint32_t y) {
    for (uint32_t x = 0; x < pw; ++x) main_composite_taa(vec3u(x, y, 0u));
  });
  return 0;
}
"""

STRUCT_PUTS = []  # (struct name, field names) of flat structs, filled by main()

TYPE_MAP = {"f32": "float", "u32": "uint32_t", "i32": "int32_t", "bool": "bool"}
WIDTH = {"float": 1, "uint32_t": 1, "int32_t": 1, "bool": 1, "vec2f": 2, "vec3f": 3, "vec4f": 4}


def strip_comments(src: str) -> str:
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return re.sub(r"//[^\n]*", "", src)


def match_brace(src: str, i: int) -> int:
    """Index just past the brace block that opens at src[i] == '{'."""
    depth = 0
    for j in range(i, len(src)):
        if src[j] == "{":
            depth += 1
        elif src[j] == "}":
            depth -= 1
            if depth == 0:
                return j + 1
    raise ValueError("unbalanced braces")


def conv_type(t: str) -> str:
    t = t.strip()
    t = re.sub(r"\bvec([234])<f32>", r"vec\1f", t)
    t = re.sub(r"\bvec([234])<i32>", r"vec\1i", t)
    t = re.sub(r"\bvec([234])<u32>", r"vec\1u", t)
    t = re.sub(r"\bmat2x2<f32>", "mat2x2f", t)
    t = re.sub(r"\bmat4x4<f32>", "mat4x4f", t)
    t = re.sub(r"\bmat3x3<f32>", "mat3x3f", t)
    t = re.sub(r"\batomic<u32>", "atomic_u32", t)
    if t.startswith("texture_2d<"):
        return "const Tex2D&"
    if t.startswith("texture_storage_2d<"):
        return "Tex2D&"
    if t == "sampler":
        return "const Sampler&"
    pm = re.match(r"ptr<\s*function\s*,\s*(.+)>$", t)
    if pm:
        return conv_type(pm.group(1)) + "*"
    t = re.sub(r"\barray<\s*([^,>]+)\s*,\s*([^>]+)>", lambda m: f"std::array<{conv_type(m.group(1))}, {m.group(2).strip()}>", t)
    return TYPE_MAP.get(t, t)


def conv_expr(s: str) -> str:
    """WGSL statements / expressions -> C++ over wgsl_shim.h."""
    s = re.sub(r"\bvec([234])<f32>", r"vec\1f", s)
    s = re.sub(r"\bvec([234])<i32>", r"vec\1i", s)
    s = re.sub(r"\bvec([234])<u32>", r"vec\1u", s)
    s = re.sub(r"\bmat2x2<f32>", "mat2x2f", s)
    s = re.sub(r"\bmat3x3<f32>", "mat3x3f", s)
    s = re.sub(r"\bmat4x4<f32>", "mat4x4f", s)
    s = re.sub(r"\bbitcast<u32>\s*\(", "bitcast_u32(", s)
    s = re.sub(r"\bbitcast<f32>\s*\(", "bitcast_f32(", s)
    s = re.sub(r"\bbitcast<i32>\s*\(", "bitcast_i32(", s)
    # declarations
    s = re.sub(r"\blet\s+(\w+)\s*:\s*([^=;]+?)\s*=", lambda m: f"const {conv_type(m.group(2))} {m.group(1)} =", s)
    s = re.sub(r"\blet\s+(\w+)\s*=", r"const auto \1 =", s)
    s = re.sub(r"\bconst\s+(\w+)\s*:\s*([^=;]+?)\s*=", lambda m: f"const {conv_type(m.group(2))} {m.group(1)} =", s)
    s = re.sub(r"\bconst\s+(\w+)\s*=", r"const auto \1 =", s)
    s = re.sub(r"\bvar\s+(\w+)\s*:\s*([^=;]+?)\s*=", lambda m: f"{conv_type(m.group(2))} {m.group(1)} =", s)
    s = re.sub(r"\bvar\s+(\w+)\s*:\s*([^=;]+?)\s*;", lambda m: f"{conv_type(m.group(2))} {m.group(1)}{{}};", s)
    s = re.sub(r"\bvar\s+(\w+)\s*=", r"auto \1 =", s)
    # conversions, builtins with other C++ names, swizzles, loops
    s = re.sub(r"\bf32\s*\(", "wgsl_f32(", s)
    s = re.sub(r"\bu32\s*\(", "wgsl_u32(", s)
    s = re.sub(r"\bi32\s*\(", "wgsl_i32(", s)
    s = re.sub(r"\bf32\b", "float", s)
    s = re.sub(r"\bu32\b", "uint32_t", s)
    s = re.sub(r"\bi32\b", "int32_t", s)
    s = re.sub(r"\bselect\s*\(", "wgsl_select(", s)
    s = re.sub(r"\.(xyz|xz|xy)\b", r".\1()", s)
    s = re.sub(r"\bloop\s*\{", "for (;;) {", s)
    # literals: WGSL floats are f32 (C++ would make them double)
    s = re.sub(r"(?<![\w.])(\d+)i\b", r"\1", s)
    s = re.sub(r"(?<![\w.])(\d+)f\b", r"\1.0f", s)
    s = re.sub(r"(?<![\w.])(\d+\.\d*|\.\d+)([eE][-+]?\d+)?(?![\w.])", r"\1\2f", s)
    s = re.sub(r"(?<![\w.])(\d+)([eE][-+]?\d+)(?![\w.])", r"\1.0\2f", s)
    return s


def split_top(text: str, sep: str = ","):
    """Splits on `sep` outside <> and ()."""
    parts, depth, cur = [], 0, ""
    for ch in text:
        if ch in "<(":
            depth += 1
        elif ch in ">)":
            depth -= 1
        if ch == sep and depth == 0:
            parts.append(cur)
            cur = ""
        else:
            cur += ch
    parts.append(cur)
    return [q.strip() for q in parts if q.strip()]


def brace_ctors(s: str, names) -> str:
    """`S(a, b)` -> `S{a, b}` for every struct name S."""
    if not names:
        return s
    pat = re.compile(r"\b(" + "|".join(sorted(names, key=len, reverse=True)) + r")\s*\(")
    pos = 0
    while True:
        m = pat.search(s, pos)
        if not m:
            return s
        open_i = m.end() - 1
        depth = 0
        for j in range(open_i, len(s)):
            if s[j] == "(":
                depth += 1
            elif s[j] == ")":
                depth -= 1
                if depth == 0:
                    break
        s = s[:open_i] + "{" + s[open_i + 1:j] + "}" + s[j + 1:]
        pos = open_i + 1


def parse(shader_dir: Path):
    consts, fns, structs, bindings, wg_vars = [], {}, [], [], []
    for rel in FILES:
        src = strip_comments((shader_dir / rel).read_text())
        i = 0
        while i < len(src):
            m = re.compile(r"\s*(const|fn|struct|@|alias|override|var|enable)").match(src, i)
            if not m:
                i += 1
                continue
            kind = m.group(1)
            if kind == "const":
                end = src.index(";", m.end())
                cm = re.match(r"\s*const\s+(\w+)\s*(?::\s*([^=]+?))?\s*=\s*(.*)", src[i:end], flags=re.S)
                if cm:
                    consts.append((cm.group(1), cm.group(2), cm.group(3)))
                i = end + 1
            elif kind == "fn":
                fm = re.compile(r"\s*fn\s+(\w+)\s*\((.*?)\)\s*(?:->\s*([^{]+?))?\s*\{", re.S).match(src, i)
                end = match_brace(src, fm.end() - 1)
                fns[fm.group(1)] = (fm.group(2), fm.group(3), src[fm.end():end - 1], rel)
                i = end
            elif kind == "struct":
                sm = re.compile(r"\s*struct\s+(\w+)\s*\{").match(src, i)
                end = match_brace(src, sm.end() - 1)
                fields = []
                for fdecl in split_top(src[sm.end():end - 1]):
                    fname, fty = fdecl.split(":", 1)
                    fields.append((re.sub(r"@\w+(\([^)]*\))?", "", fname).strip(), fty.strip()))
                structs.append((sm.group(1), fields))
                i = end
            elif kind == "var" and re.compile(r"\s*var<(workgroup|private)>").match(src, i):
                vm = re.compile(r"\s*var<(?:workgroup|private)>\s+(\w+)\s*:\s*([^;]+);").match(src, i)
                wg_vars.append((vm.group(1), vm.group(2).strip()))
                i = vm.end()
            elif kind == "@" and re.compile(r"\s*@compute").match(src, i):
                i = re.compile(r"\s*@compute\s*@workgroup_size\([^)]*\)").match(src, i).end()
            elif kind == "@":
                bm = re.compile(r"\s*@group\(\d+\)\s*@binding\(\d+\)\s*var(<[^>]*>)?\s+(\w+)\s*:\s*([^;]+);",
                                re.S).match(src, i)
                if bm:
                    bindings.append((bm.group(1) or "", bm.group(2), bm.group(3).strip()))
                    i = bm.end()
                    continue
                end = src.find(";", m.end())
                brace = src.find("{", m.end())
                i = (end + 1) if end >= 0 and (brace < 0 or end < brace) else (match_brace(src, brace) if brace >= 0 else len(src))
            else:
                end = src.find(";", m.end())
                brace = src.find("{", m.end())
                i = (end + 1) if end >= 0 and (brace < 0 or end < brace) else (match_brace(src, brace) if brace >= 0 else len(src))
    return consts, fns, structs, bindings, wg_vars


def closure(fns, roots):
    out, todo = [], list(roots)
    while todo:
        f = todo.pop()
        if f in out or f not in fns:
            continue
        out.append(f)
        for callee in re.findall(r"\b(\w+)\s*\(", fns[f][2]):
            if callee in fns and callee not in out:
                todo.append(callee)
    return out


def params_of(ptext: str):
    ps = []
    for p in split_top(re.sub(r"@\w+\([^)]*\)", "", ptext)):
        name, ty = p.split(":", 1)
        ps.append((name.strip(), conv_type(ty)))
    return ps


def main(shader_dir: Path, out: Path) -> None:
    consts, fns, structs, bindings, wg_vars = parse(shader_dir)
    names = closure(fns, EXPORTS)
    snames = [n for n, _ in structs]
    lines = ["// Generated by oracle/wgsl_to_cpp.py from the reference's WGSL; not committed.",
             '#include "wgsl_shim.h"', '#include "vxe/vxe.h"', "#include <cstring>", "#include <thread>",
             "#include <vector>", "namespace wgsl {"]
    for name, ty, expr in consts:
        ty_c = conv_type(ty) if ty else "auto"
        lines.append(f"static const {ty_c} {name} = {brace_ctors(conv_expr(expr.strip()), snames)};")
    for sname, fields in structs:  # the shader's structs, member for member
        if any("texture" in t for _, t in fields):
            continue
        lines.append(f"struct {sname} {{ " + " ".join(f"{conv_type(t)} {f};" for f, t in fields) + " };")
    for space, bname, bty in bindings:  # storage buffers, the uniforms, images
        m = re.match(r"array<\s*(\w+)\s*>$", bty)
        if "read_write" in space and m:
            lines.append(f"static RWBuf<{conv_type(m.group(1))}> {bname};")
        elif "read_write" in space:
            lines.append(f"static {conv_type(bty)} {bname}{{}};")
        elif "storage" in space and m:
            lines.append(f"static Buf<{conv_type(m.group(1))}> {bname};")
        elif bty.startswith("texture_2d<") or bty.startswith("texture_storage_2d<"):
            lines.append(f"static Tex2D {bname};")
        elif bty == "sampler":
            lines.append(f"static Sampler {bname};")
        elif "uniform" in space:
            lines.append(f"static {conv_type(bty)} {bname}{{}};")
        elif bty.startswith("texture_2d_array<f32>"):
            lines.append(f"static Tex2DArrayF {bname};")
    for vname, vty in wg_vars:  # workgroup memory: each host thread runs whole workgroups
        lines.append(f"static thread_local {conv_type(vty)} {vname}{{}};")
    for sname, fields in structs:  # structs of flat fields can be results
        ftys = [conv_type(t) for _, t in fields]
        if fields and all(t in WIDTH for t in ftys) and not sname.startswith("_"):
            WIDTH[sname] = sum(WIDTH[t] for t in ftys)
            STRUCT_PUTS.append((sname, [f for f, _ in fields]))
    sigs = {}
    for f in names:
        ptext, ret, body, rel = fns[f]
        ps = params_of(ptext)
        rt = conv_type(ret) if ret else "void"
        sigs[f] = (ps, rt)
        lines.append(f"{rt} {f}({', '.join(f'{t} {n}' for n, t in ps)});")
    for f in names:
        ptext, ret, body, rel = fns[f]
        ps, rt = sigs[f]
        lines.append(f"// {rel}")
        lines.append(f"{rt} {f}({', '.join(f'{t} {n}' for n, t in ps)}) {{{brace_ctors(conv_expr(body), snames)}}}")
    lines.append("}  // namespace wgsl")
    # the flat-slot dispatcher
    lines += ["using namespace wgsl;",
              "template <class T> static T get_slot(const float*& p) { T v; std::memcpy(&v, p, 4); ++p; return v; }",
              "static float get_f(const float*& p) { return *p++; }",
              "template <int N> static vec<float, N> get_v(const float*& p) { vec<float, N> v; for (int i = 0; i < N; ++i) v[i] = *p++; return v; }",
              "static void put(float*& o, float v) { *o++ = v; }",
              "static void put(float*& o, uint32_t v) { std::memcpy(o++, &v, 4); }",
              "static void put(float*& o, int32_t v) { std::memcpy(o++, &v, 4); }",
              "static void put(float*& o, bool v) { const uint32_t u = v ? 1u : 0u; std::memcpy(o++, &u, 4); }",
              "template <int N> static void put(float*& o, const vec<float, N>& v) { for (int i = 0; i < N; ++i) *o++ = v[i]; }",
              *[f"static void put_struct(float*& o, const {n}& v) {{ " + " ".join(f"put(o, v.{f});" for f in fs) + " }"
                for n, fs in STRUCT_PUTS],
              'extern "C" void ref_wgsl_set_cam(const float* p, const float* vp) { for (int i = 0; i < 4; ++i) { cam.cam_pos[i] = p[i]; cam.voxel_params[i] = vp[i]; } }',
              'extern "C" int ref_wgsl_widths(const char* name, unsigned* in_w, unsigned* out_w) {']
    table = []
    for f in EXPORTS:
        if f not in sigs:
            continue
        ps, rt = sigs[f]
        if rt not in WIDTH or any(t not in WIDTH for _, t in ps):
            continue
        table.append(f)
        lines.append(f'  if (!std::strcmp(name, "{f}")) {{ *in_w = {sum(WIDTH[t] for _, t in ps)}; *out_w = {WIDTH[rt]}; return 0; }}')
    lines += ["  return -1;", "}",
              'extern "C" int ref_wgsl_eval(const char* name, const float* in, float* out, unsigned n) {',
              "  unsigned iw = 0, ow = 0;", "  if (ref_wgsl_widths(name, &iw, &ow) != 0) return -1;",
              "  for (unsigned k = 0; k < n; ++k) {",
              "    const float* p = in + (size_t)k * iw; float* o = out + (size_t)k * ow;"]
    for f in table:
        ps, rt = sigs[f]
        args = []
        for _, t in ps:
            if t == "float":
                args.append("get_f(p)")
            elif t in ("uint32_t", "int32_t"):
                args.append(f"get_slot<{t}>(p)")
            elif t == "bool":
                args.append("(get_slot<uint32_t>(p) != 0u)")
            else:
                args.append(f"get_v<{WIDTH[t]}>(p)")
        # arguments are read in order into locals first (evaluation order)
        decl = "; ".join(f"const auto a{i} = {a}" for i, a in enumerate(args))
        call = f"{f}({', '.join(f'a{i}' for i in range(len(args)))})"
        putter = "put_struct" if rt in dict(STRUCT_PUTS) else "put"
        lines.append(f'    if (!std::strcmp(name, "{f}")) {{ {decl}{";" if decl else ""} {putter}(o, {call}); continue; }}')
    lines += ["  }", "  return 0;", "}"]
    if "trace_chunk_interval_stream_macro" in sigs:
        lines += CHUNK_WALK_EXPORT.splitlines()
    if "main_primary" in sigs:
        lines += FRAME_EXPORT.splitlines()
    out.parent.mkdir(parents=True, exist_ok=True)
    out.write_text("\n".join(lines) + "\n")


if __name__ == "__main__":
    main(Path(sys.argv[1]), Path(sys.argv[2]))
