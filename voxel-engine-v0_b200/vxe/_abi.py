"""ctypes mirror of include/vxe/vxe.h (the C ABI of libvxe.so).

The structs here are byte-identical to the reference's GPU PODs
(render/gpu_types.rs); ``check_layout`` asserts the sizes the reference
relies on (NodeGpu 16 B, NodeRopesGpu 32 B, ChunkMetaGpu 48 B, CameraGpu 464 B,
ClipmapGpu 528 B).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libvxe.so"
# the same library with device bounds checks (zero records + error word for
# out-of-range indices instead of clamped reads)
CHECKED_LIB_PATH = Path(__file__).resolve().parent / "libvxe_checked.so"

VXE_OK = 0
STATUS_NAMES = {
    0: "VXE_OK", 1: "VXE_ERR_INVALID_ARG", 2: "VXE_ERR_CAPACITY", 3: "VXE_ERR_OOM", 4: "VXE_ERR_TIMEOUT",
    5: "VXE_ERR_DEVICE", 6: "VXE_ERR_BOUNDS", 7: "VXE_ERR_NO_DEVICE", 8: "VXE_NOT_READY",
}
VXE_NOT_READY = 8
BATCH_LANES = 4

INVALID_U32 = 0xFFFFFFFF
MACRO_WORDS_PER_CHUNK = 16
COLINFO_WORDS_PER_CHUNK = 2048
CHUNK_SIZE = 64
CLIP_LEVELS_MAX = 16

FLAG_GODRAY_MACRO_ALIAS = 1 << 0
FLAG_SILENT_CAPACITY_SKIP = 1 << 1
FLAG_HIT_RECORDS = 1 << 2
FLAG_DEBUG_INTERMEDIATES = 1 << 3
FLAG_PRIMARY_MEGAKERNEL = 1 << 5
FLAG_NO_GRASS_TABLE = 1 << 6
FLAG_UPLOADS_UNORDERED = 1 << 7

(IMG_COLOR, IMG_DEPTH, IMG_LOCAL, IMG_PRIMARY_HIST_IN, IMG_PRIMARY_HIST_OUT, IMG_SHADOW_IN, IMG_SHADOW_OUT,
 IMG_LOCAL_HIST_IN, IMG_LOCAL_HIST_OUT, IMG_GODRAY_IN, IMG_GODRAY_OUT, IMG_OUTPUT_PRE_TAA, IMG_OUTPUT,
 IMG_OUTPUT_HIST_IN, IMG_OUTPUT_HIST_OUT, IMG_HITS) = range(16)

NODE_DTYPE = np.dtype([("child_base", "<u4"), ("child_mask", "<u4"), ("material", "<u4"), ("key", "<u4")])
ROPES_DTYPE = np.dtype([(n, "<u4") for n in ("px", "nx", "py", "ny", "pz", "nz", "_pad0", "_pad1")])
HIT_DTYPE = np.dtype([("t", "<f4"), ("node", "<u4"), ("voxel", "<i4", (3,)), ("face", "<u4"), ("mat", "<u4"),
                      ("_pad", "<u4")])


class Node(C.Structure):
    _fields_ = [("child_base", C.c_uint32), ("child_mask", C.c_uint32), ("material", C.c_uint32), ("key", C.c_uint32)]


class NodeRopes(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in ("px", "nx", "py", "ny", "pz", "nz", "_pad0", "_pad1")]


class ChunkMeta(C.Structure):
    _fields_ = [("origin", C.c_int32 * 4), ("node_base", C.c_uint32), ("node_count", C.c_uint32),
                ("macro_base", C.c_uint32), ("colinfo_base", C.c_uint32), ("macro_empty", C.c_uint32),
                ("_pad0", C.c_uint32), ("_pad1", C.c_uint32), ("_pad2", C.c_uint32)]


Mat4 = (C.c_float * 4) * 4


class CameraGpu(C.Structure):
    _fields_ = [("view_inv", Mat4), ("proj_inv", Mat4), ("view_proj", Mat4), ("prev_view_proj", Mat4),
                ("cam_pos", C.c_float * 4), ("ray00", C.c_float * 4), ("ray_dx", C.c_float * 4),
                ("ray_dy", C.c_float * 4), ("chunk_size", C.c_uint32), ("chunk_count", C.c_uint32),
                ("max_steps", C.c_uint32), ("frame_index", C.c_uint32), ("voxel_params", C.c_float * 4),
                ("grid_origin_chunk", C.c_int32 * 4), ("grid_dims", C.c_uint32 * 4),
                ("render_present_px", C.c_uint32 * 4), ("profile_flags", C.c_uint32),
                ("_pad_profile", C.c_uint32 * 3), ("_pad0", C.c_uint32 * 4), ("_pad1", C.c_uint32 * 4),
                ("_pad2", C.c_uint32 * 4)]


class ClipmapGpu(C.Structure):
    _fields_ = [("levels", C.c_uint32), ("res", C.c_uint32), ("base_cell_m", C.c_float), ("_pad0", C.c_float),
                ("level", (C.c_float * 4) * CLIP_LEVELS_MAX), ("offset", (C.c_uint32 * 4) * CLIP_LEVELS_MAX)]


class ClipPatch(C.Structure):
    _fields_ = [("level", C.c_uint32), ("x", C.c_uint32), ("y", C.c_uint32), ("w", C.c_uint32), ("h", C.c_uint32),
                ("data", C.POINTER(C.c_float))]


class ChunkUpload(C.Structure):
    _fields_ = [("slot", C.c_uint32), ("meta", ChunkMeta), ("node_base", C.c_uint32), ("node_count", C.c_uint32),
                ("nodes", C.c_void_p), ("ropes", C.c_void_p), ("macro_words", C.c_void_p),
                ("colinfo_words", C.c_void_p)]


class Config(C.Structure):
    _fields_ = [("node_capacity", C.c_uint32), ("chunk_capacity", C.c_uint32), ("grid_capacity", C.c_uint32),
                ("clip_levels", C.c_uint32), ("clip_res", C.c_uint32), ("flags", C.c_uint32), ("device", C.c_int32),
                ("_reserved", C.c_uint32)]


class FrameOut(C.Structure):
    _fields_ = [("color", C.c_void_p), ("depth", C.c_void_p), ("godray", C.c_void_p), ("output", C.c_void_p),
                ("internal_w", C.c_uint32), ("internal_h", C.c_uint32), ("present_w", C.c_uint32),
                ("present_h", C.c_uint32)]


class Hit(C.Structure):
    _fields_ = [("t", C.c_float), ("node", C.c_uint32), ("voxel", C.c_int32 * 3), ("face", C.c_uint32),
                ("mat", C.c_uint32), ("_pad", C.c_uint32)]


class Timings(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("primary", "local_taa", "godray", "composite", "composite_taa", "tiles",
                                           "total", "primary_trace", "grass_cells", "trace_kernel")]


class ClipPatchGeom(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in ("level", "x", "y", "w", "h", "lx0", "lz0")] + \
               [(n, C.c_float) for n in ("ox_m", "oz_m", "cell_m")]


class BuildTimings(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("columns", "svo")]


class BuildPlace(C.Structure):
    _fields_ = [("cx", C.c_int32), ("cy", C.c_int32), ("cz", C.c_int32), ("slot", C.c_uint32),
                ("node_base", C.c_uint32), ("node_count", C.c_uint32)]


ERR_WORD_BUILD = 1 << 7


class SlotMove(C.Structure):
    _fields_ = [("from_", C.c_uint32), ("to", C.c_uint32)]
BUILD_NODE_CAP_MAX = 299593
BUILD_BATCH_MAX = 2048


class WorldParams(C.Structure):
    _fields_ = [("seed", C.c_uint32), ("height_min", C.c_int32), ("height_max", C.c_int32),
                ("dirt_depth", C.c_int32), ("carve_mod", C.c_uint32), ("cave_threshold", C.c_float),
                ("height_scale_vox", C.c_float), ("features", C.c_uint32)]


class BuiltChunk(C.Structure):
    _fields_ = [("nodes", C.POINTER(Node)), ("ropes", C.POINTER(NodeRopes)), ("node_count", C.c_uint32),
                ("macro_words", C.c_uint32 * MACRO_WORDS_PER_CHUNK),
                ("colinfo_words", C.c_uint32 * COLINFO_WORDS_PER_CHUNK), ("solid_voxels", C.c_uint32)]


class CameraParams(C.Structure):
    _fields_ = [("pos", C.c_float * 3), ("yaw", C.c_float), ("pitch", C.c_float), ("fovy_rad", C.c_float),
                ("z_near", C.c_float), ("z_far", C.c_float), ("present_w", C.c_uint32), ("present_h", C.c_uint32),
                ("internal_w", C.c_uint32), ("internal_h", C.c_uint32), ("frame_index", C.c_uint32),
                ("jitter", C.c_uint32), ("time_s", C.c_float), ("chunk_count", C.c_uint32),
                ("grid_origin_chunk", C.c_int32 * 3), ("grid_dims", C.c_uint32 * 3), ("has_prev", C.c_uint32),
                ("prev_view_proj", Mat4)]


class SceneView(C.Structure):
    _fields_ = [("nodes", C.c_void_p), ("ropes", C.c_void_p), ("node_count", C.c_uint64), ("metas", C.c_void_p),
                ("macro_words", C.c_void_p), ("colinfo_words", C.c_void_p), ("chunk_capacity", C.c_uint32),
                ("grid_cells", C.c_uint32), ("grid", C.c_void_p), ("clip_tex", C.c_void_p),
                ("clip_layers", C.c_uint32), ("clip_res", C.c_uint32)]


NOALLOC_MAX_TILES = 36864
PROFILE_COUNT = 5
PROFILE_VOXEL, PROFILE_GRASS, PROFILE_HDR, PROFILE_FOG, PROFILE_SHADOW = range(5)


class FrameStats(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in ("voxel_pixels", "far_pixels", "probes", "pending_pixels", "slab_tasks",
                                           "slab_hits", "rewalk_pixels", "full_trace_pixels")]

REQ_VIEWPORT, REQ_QUERY = 0, 1
BATCH_PERSISTENT, BATCH_PLAIN, BATCH_GRAPH = 0, 1, 2
MAX_BATCH_REQUESTS = 256
MAX_VIEWS_PER_LAUNCH = 8


class Request(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("width", C.c_uint32), ("height", C.c_uint32), ("ray_count", C.c_uint32),
                ("camera", CameraGpu), ("d_origins", C.c_void_p), ("d_dirs", C.c_void_p), ("tmax", C.c_float),
                ("_pad", C.c_uint32), ("d_out", C.c_void_p)]


class BatchOptions(C.Structure):
    _fields_ = [("tile_w", C.c_uint32), ("tile_h", C.c_uint32), ("rays_per_thread", C.c_uint32),
                ("mode", C.c_uint32)]


class BatchStats(C.Structure):
    _fields_ = [("ms", C.c_double), ("rays", C.c_uint64), ("items", C.c_uint32), ("tiles", C.c_uint32)]


# Every symbol include/vxe/vxe.h declares, with (restype, argtypes).
P = C.POINTER
SIGNATURES = {
    "vxe_create": (C.c_int, [P(Config), P(C.c_void_p)]),
    "vxe_destroy": (None, [C.c_void_p]),
    "vxe_last_error": (C.c_char_p, [C.c_void_p]),
    "vxe_get_flags": (C.c_uint32, [C.c_void_p]),
    "vxe_set_flags": (C.c_int, [C.c_void_p, C.c_uint32]),
    "vxe_resize": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_float]),
    "vxe_get_internal_dims": (C.c_int, [C.c_void_p, P(C.c_uint32), P(C.c_uint32)]),
    "vxe_upload_chunks": (C.c_int, [C.c_void_p, P(ChunkUpload), C.c_uint32]),
    "vxe_write_meta": (C.c_int, [C.c_void_p, C.c_uint32, P(ChunkMeta), C.c_uint32]),
    "vxe_write_grid": (C.c_int, [C.c_void_p, P(C.c_uint32), C.c_uint32]),
    "vxe_write_camera": (C.c_int, [C.c_void_p, P(CameraGpu)]),
    "vxe_write_clipmap": (C.c_int, [C.c_void_p, P(ClipmapGpu), P(ClipPatch), C.c_uint32]),
    "vxe_render_frame": (C.c_int, [C.c_void_p, P(FrameOut)]),
    "vxe_render_frame_async": (C.c_int, [C.c_void_p, P(FrameOut)]),
    "vxe_render_frame_graph": (C.c_int, [C.c_void_p, P(FrameOut)]),
    "vxe_synchronize": (C.c_int, [C.c_void_p]),
    "vxe_trace_rays": (C.c_int, [C.c_void_p, P(C.c_float), P(C.c_float), C.c_uint32, C.c_float, C.c_void_p]),
    "vxe_trace_rays_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_float, C.c_void_p]),
    "vxe_get_timings": (C.c_int, [C.c_void_p, P(Timings)]),
    "vxe_image_size": (C.c_int, [C.c_void_p, C.c_int, P(C.c_size_t)]),
    "vxe_read_image": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]),
    "vxe_write_image": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]),
    "vxe_read_error_word": (C.c_int, [C.c_void_p, P(C.c_uint32)]),
    "vxe_reset_profile_counts": (C.c_int, [C.c_void_p]),
    "vxe_read_profile_counts": (C.c_int, [C.c_void_p, C.c_void_p]),
    "vxe_set_record_limits": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32]),
    "vxe_get_frame_stats": (C.c_int, [C.c_void_p, P(FrameStats)]),
    "vxe_debug_grass": (C.c_int, [C.c_int, C.c_uint32, C.c_void_p, C.c_void_p]),
    "vxe_measure_l2_bandwidth": (C.c_int, [C.c_int, C.c_uint64, C.c_uint32, P(C.c_double)]),
    "vxe_debug_detmath": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]),
    "vxe_trace_primary_hits_noalloc": (C.c_int, [P(SceneView), P(CameraGpu), P(ClipmapGpu), C.c_void_p,
                                                  C.c_void_p]),
    "vxe_submit_batch": (C.c_int, [C.c_void_p, P(Request), C.c_uint32, P(BatchOptions), P(BatchStats)]),
    "vxe_submit_batch_async": (C.c_int, [C.c_void_p, C.c_uint32, P(Request), C.c_uint32, P(BatchOptions)]),
    "vxe_batch_wait": (C.c_int, [C.c_void_p, C.c_uint32, C.c_int, P(BatchStats)]),
    "vxe_view_bytes": (C.c_uint64, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_float]),
    "vxe_view_lane_bytes": (C.c_uint64, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_float]),
    "vxe_view_create": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_float, P(C.c_void_p)]),
    "vxe_view_render_async": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, P(CameraGpu)]),
    "vxe_view_render_batch_async": (C.c_int, [C.c_void_p, P(C.c_void_p), P(CameraGpu), C.c_uint32, C.c_uint32]),
    "vxe_view_read_image": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]),
    "vxe_view_destroy": (C.c_int, [C.c_void_p, C.c_void_p]),
    "vxe_build_chunk": (C.c_int, [P(WorldParams), C.c_int32, C.c_int32, C.c_int32, P(BuiltChunk)]),
    "vxe_free_chunk": (None, [P(BuiltChunk)]),
    "vxe_chunk_materials": (C.c_int, [P(WorldParams), C.c_int32, C.c_int32, C.c_int32, C.c_void_p]),
    "vxe_ground_height": (C.c_int32, [P(WorldParams), C.c_int32, C.c_int32]),
    "vxe_build_from_materials": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, P(BuiltChunk)]),
    "vxe_build_camera": (C.c_int, [P(CameraParams), P(CameraGpu)]),
    "vxe_clipmap_new": (C.c_void_p, [P(WorldParams), C.c_uint32, C.c_uint32, C.c_float]),
    "vxe_clipmap_free": (None, [C.c_void_p]),
    "vxe_clipmap_update": (C.c_int, [C.c_void_p, C.c_float, C.c_float, P(ClipmapGpu), P(P(ClipPatch)),
                                     P(C.c_uint32)]),
    "vxe_clipmap_plan": (C.c_int, [C.c_void_p, C.c_float, C.c_float, P(ClipmapGpu), P(P(ClipPatchGeom)),
                                   P(C.c_uint32), P(WorldParams)]),
    "vxe_clipmap_update_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_float, C.c_float]),
    "vxe_read_clipmap": (C.c_int, [C.c_void_p, P(C.c_float), C.c_size_t]),
    "vxe_solid_voxels_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, P(WorldParams), C.c_void_p]),
    "vxe_build_chunks_device": (C.c_int, [C.c_void_p, P(WorldParams), C.c_void_p, C.c_uint32, C.c_uint32,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "vxe_get_build_timings": (C.c_int, [C.c_void_p, P(BuildTimings)]),
    "vxe_build_chunks_resident": (C.c_int, [C.c_void_p, P(WorldParams), P(BuildPlace), C.c_uint32]),
    "vxe_read_image_async": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t, P(C.c_uint64)]),
    "vxe_read_image_wait": (C.c_int, [C.c_void_p, C.c_uint64]),
    "vxe_move_slots": (C.c_int, [C.c_void_p, P(SlotMove), C.c_uint32]),
}


class VxeError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str = ""):
        self.status = status
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}" + (f" ({msg})" if msg else ""))


_libs = {}


def lib(checked: bool = False) -> C.CDLL:
    """Loads libvxe.so (or, with `checked`, libvxe_checked.so).  There is no
    fallback: a missing library is an error."""
    path = CHECKED_LIB_PATH if checked else LIB_PATH
    if path not in _libs:
        if not path.exists():
            raise FileNotFoundError(f"{path} is missing; run `python voxel-engine-v0_b200/vxe_build.py` first")
        l = C.CDLL(str(path))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(l, name)
            fn.restype = res
            fn.argtypes = args
        _libs[path] = l
    return _libs[path]


# The host-side producers (chunk builder, camera packing, clipmap state) are
# plain C++ with no device code.  A process that must not map the CUDA library
# (a CPU-only consumer of the producers, such as a CPU timing of the passes)
# registers a host-only build of the same sources here.
HOST_SYMBOLS = ("vxe_build_chunk", "vxe_free_chunk", "vxe_chunk_materials", "vxe_ground_height",
                "vxe_build_from_materials", "vxe_build_camera", "vxe_clipmap_new", "vxe_clipmap_free",
                "vxe_clipmap_update", "vxe_clipmap_plan")
_host_lib = None


def use_host_library(path) -> C.CDLL:
    """Routes the host-side producer calls (HOST_SYMBOLS) to the library at
    `path`, a host-only build of the producer sources, instead of libvxe.so."""
    global _host_lib
    l = C.CDLL(str(path))
    for name in HOST_SYMBOLS:
        res, args = SIGNATURES[name]
        fn = getattr(l, name)
        fn.restype = res
        fn.argtypes = args
    _host_lib = l
    return l


def host_lib() -> C.CDLL:
    """The library serving the host-side producer calls: libvxe.so unless
    use_host_library() registered a host-only build."""
    return _host_lib if _host_lib is not None else lib()


def check_layout() -> None:
    sizes = {Node: 16, NodeRopes: 32, ChunkMeta: 48, CameraGpu: 464, ClipmapGpu: 528, Hit: 32}
    for t, n in sizes.items():
        assert C.sizeof(t) == n, f"{t.__name__} is {C.sizeof(t)} bytes, expected {n}"
    assert NODE_DTYPE.itemsize == 16 and ROPES_DTYPE.itemsize == 32 and HIT_DTYPE.itemsize == 32


check_layout()
