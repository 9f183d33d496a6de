"""Host-side mirror of the reference ``Renderer`` (render/state/mod.rs:34-709).

Same method set and argument meaning as the Rust renderer, forwarding to the
C ABI of libvxe.so (include/vxe/vxe.h).  Every call raises ``VxeError`` on a
non-OK status; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi as A
from .world import Upload, World


class Renderer:
    def __init__(self, width: int, height: int, render_scale: float = 0.5, *, node_capacity: int,
                 chunk_capacity: int, grid_capacity: int, clip_levels: int = 16, clip_res: int = 256,
                 flags: int = A.FLAG_GODRAY_MACRO_ALIAS, device: int = 0, checked: bool = False):
        """`checked`: run on libvxe_checked.so (device bounds checks reported
        in the error word) instead of libvxe.so (clamped reads)."""
        self._lib = A.lib(checked)
        self.checked = checked
        cfg = A.Config(node_capacity, chunk_capacity, grid_capacity, clip_levels, clip_res, flags, device, 0)
        h = C.c_void_p()
        st = self._lib.vxe_create(C.byref(cfg), C.byref(h))
        if st != A.VXE_OK:
            raise A.VxeError(st, "vxe_create")
        self._ctx = h
        self.clip_levels, self.clip_res = clip_levels, clip_res
        self.device = device
        self.render_scale = render_scale
        self.resize_output(width, height)

    # -- lifecycle --------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_ctx", None):
            self._lib.vxe_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int, where: str) -> None:
        if st != A.VXE_OK:
            msg = self._lib.vxe_last_error(self._ctx)
            raise A.VxeError(st, where, msg.decode() if msg else "")

    @property
    def flags(self) -> int:
        return int(self._lib.vxe_get_flags(self._ctx))

    def set_flags(self, flags: int) -> None:
        self._check(self._lib.vxe_set_flags(self._ctx, flags), "vxe_set_flags")

    def resize_output(self, width: int, height: int) -> None:
        self._check(self._lib.vxe_resize(self._ctx, width, height, self.render_scale), "vxe_resize")
        self.present = (width, height)
        w, h = C.c_uint32(), C.c_uint32()
        self._check(self._lib.vxe_get_internal_dims(self._ctx, C.byref(w), C.byref(h)), "vxe_get_internal_dims")
        self.internal = (w.value, h.value)

    def internal_dims(self):
        return self.internal

    # -- uploads ----------------------------------------------------------------
    def apply_chunk_uploads(self, uploads: list[Upload]) -> None:
        if not uploads:
            return
        arr = (A.ChunkUpload * len(uploads))()
        keep = []
        for i, u in enumerate(uploads):
            d = arr[i]
            d.slot = u.slot
            C.memmove(C.byref(d.meta), u.meta.ctypes.data, 48)
            d.node_base = u.node_base
            if u.data is not None:
                macro = np.ascontiguousarray(u.data.macro, dtype=np.uint32)
                colinfo = np.ascontiguousarray(u.data.colinfo, dtype=np.uint32)
                keep += [macro, colinfo]
                d.macro_words, d.colinfo_words = macro.ctypes.data, colinfo.ctypes.data
                if not u.rewrite:  # a slot rewrite leaves the node records where they are
                    nodes = np.ascontiguousarray(u.data.nodes)
                    ropes = np.ascontiguousarray(u.data.ropes)
                    keep += [nodes, ropes]
                    d.node_count = len(nodes)
                    d.nodes, d.ropes = nodes.ctypes.data, ropes.ctypes.data
        self._check(self._lib.vxe_upload_chunks(self._ctx, arr, len(uploads)), "vxe_upload_chunks")

    def upload_world(self, world: World, uploads: list[Upload]) -> None:
        self.apply_chunk_uploads(uploads)
        self.write_chunk_grid(world.grid)

    def write_chunk_grid(self, grid: np.ndarray) -> None:
        g = np.ascontiguousarray(grid, dtype=np.uint32)
        self._check(self._lib.vxe_write_grid(self._ctx, g.ctypes.data_as(C.POINTER(C.c_uint32)), g.size),
                    "vxe_write_grid")

    def write_camera(self, cam: A.CameraGpu) -> None:
        self._check(self._lib.vxe_write_camera(self._ctx, C.byref(cam)), "vxe_write_camera")

    def write_clipmap_updates(self, params: A.ClipmapGpu, patches) -> None:
        arr = (A.ClipPatch * max(1, len(patches)))()
        keep = []
        for i, (lvl, x, y, w, h, data) in enumerate(patches):
            d = np.ascontiguousarray(data, dtype=np.float32)
            keep.append(d)
            arr[i] = A.ClipPatch(lvl, x, y, w, h, d.ctypes.data_as(C.POINTER(C.c_float)))
        self._check(self._lib.vxe_write_clipmap(self._ctx, C.byref(params), arr, len(patches)), "vxe_write_clipmap")

    # -- frame ------------------------------------------------------------------
    def encode_compute(self, sync: bool = True) -> A.FrameOut:
        out = A.FrameOut()
        fn = self._lib.vxe_render_frame if sync else self._lib.vxe_render_frame_async
        self._check(fn(self._ctx, C.byref(out)), "vxe_render_frame")
        return out

    def render_frame_graph(self) -> A.FrameOut:
        out = A.FrameOut()
        self._check(self._lib.vxe_render_frame_graph(self._ctx, C.byref(out)), "vxe_render_frame_graph")
        return out

    def synchronize(self) -> None:
        self._check(self._lib.vxe_synchronize(self._ctx), "vxe_synchronize")

    def read_gpu_timings_ms_blocking(self) -> dict:
        t = A.Timings()
        self._check(self._lib.vxe_get_timings(self._ctx, C.byref(t)), "vxe_get_timings")
        return {k: getattr(t, k) for k, _ in A.Timings._fields_}

    def solid_voxels(self, vox, world_params=None):
        """Physics solidity of voxel coordinates `vox` (torch int32 tensor (n, 3) on
        this context's device); returns a torch uint8 tensor (1 = solid).
        `world_params` (A.WorldParams) enables the heightfield fallback."""
        import torch

        vox = vox.contiguous()
        out = torch.empty(vox.shape[0], dtype=torch.uint8, device=vox.device)
        wp = C.byref(world_params) if world_params is not None else None
        torch.cuda.current_stream().synchronize()
        self._check(self._lib.vxe_solid_voxels_device(self._ctx, vox.data_ptr(), vox.shape[0], wp, out.data_ptr()),
                    "vxe_solid_voxels_device")
        self.synchronize()
        return out

    @property
    def torch_device(self) -> str:
        """The torch device string of this context's GPU."""
        return f"cuda:{self.device}"

    def build_chunks(self, world_params, coords, node_cap=None):
        """Builds chunks on the device (the GPU counterpart of the chunk builder,
        svo/builder.rs:846-986).  `coords`: torch int32 tensor (n, 3) of chunk
        coordinates on this context's device, n <= BUILD_BATCH_MAX.  Returns a
        dict of device tensors: nodes (n, cap, 4) u32, ropes (n, cap, 8) u32,
        macro (n, 16), colinfo (n, 2048), counts (n, 2) = (node_count,
        solid_voxels); a chunk whose node_count exceeds `node_cap` carries no
        nodes or ropes (the default cap always fits)."""
        import torch

        coords = coords.to(torch.int32).contiguous()
        n = coords.shape[0]
        cap = A.BUILD_NODE_CAP_MAX if node_cap is None else int(node_cap)
        dev = coords.device
        out = {
            "nodes": torch.empty((n, cap, 4), dtype=torch.int32, device=dev),
            "ropes": torch.empty((n, cap, 8), dtype=torch.int32, device=dev),
            "macro": torch.empty((n, A.MACRO_WORDS_PER_CHUNK), dtype=torch.int32, device=dev),
            "colinfo": torch.empty((n, A.COLINFO_WORDS_PER_CHUNK), dtype=torch.int32, device=dev),
            "counts": torch.empty((n, 2), dtype=torch.int32, device=dev),
        }
        torch.cuda.current_stream().synchronize()
        self._check(self._lib.vxe_build_chunks_device(
            self._ctx, C.byref(world_params), coords.data_ptr(), n, cap, out["nodes"].data_ptr(),
            out["ropes"].data_ptr(), out["macro"].data_ptr(), out["colinfo"].data_ptr(), out["counts"].data_ptr()),
            "vxe_build_chunks_device")
        self.synchronize()
        return out

    def build_resident(self, world_params, places) -> None:
        """Builds chunks on the device straight into this context's world.
        `places`: (key, slot, node_base, node_count) tuples, node_count from a
        counting build (build_chunks(..., node_cap=0))."""
        arr = (A.BuildPlace * max(1, len(places)))()
        for i, (key, slot, base, n) in enumerate(places):
            arr[i] = A.BuildPlace(key[0], key[1], key[2], slot, base, n)
        self._check(self._lib.vxe_build_chunks_resident(self._ctx, C.byref(world_params), arr, len(places)),
                    "vxe_build_chunks_resident")

    def move_slots(self, moves) -> None:
        """Dense-slot moves on the device, in order: (from, to) pairs."""
        if not moves:
            return
        arr = (A.SlotMove * len(moves))(*[A.SlotMove(f, t) for f, t in moves])
        self._check(self._lib.vxe_move_slots(self._ctx, arr, len(moves)), "vxe_move_slots")

    def build_timings(self) -> dict:
        """Device milliseconds of the last build_chunks call, per kernel."""
        t = A.BuildTimings()
        self._check(self._lib.vxe_get_build_timings(self._ctx, C.byref(t)), "vxe_get_build_timings")
        return {"columns": t.columns, "svo": t.svo}

    def read_clipmap(self) -> np.ndarray:
        """The clipmap texture (levels, res, res) after the writes queued so far."""
        out = np.zeros((self.clip_levels, self.clip_res, self.clip_res), dtype=np.float32)
        self._check(self._lib.vxe_read_clipmap(self._ctx, out.ctypes.data_as(C.POINTER(C.c_float)), out.nbytes),
                    "vxe_read_clipmap")
        return out

    def read_error_word(self) -> int:
        w = C.c_uint32()
        self._check(self._lib.vxe_read_error_word(self._ctx, C.byref(w)), "vxe_read_error_word")
        return w.value

    # -- primary profile counters (render/state/mod.rs:448-491) -------------------
    def reset_primary_profile_counts(self) -> None:
        self._check(self._lib.vxe_reset_profile_counts(self._ctx), "vxe_reset_profile_counts")

    def read_primary_profile_counts_blocking(self) -> np.ndarray:
        """VOXEL, GRASS, HDR, FOG, SHADOW counts of the frames since the last reset."""
        out = np.zeros(A.PROFILE_COUNT, dtype=np.uint32)
        self._check(self._lib.vxe_read_profile_counts(self._ctx, out.ctypes.data), "vxe_read_profile_counts")
        return out

    # -- wavefront diagnostics ----------------------------------------------------
    def set_record_limits(self, probe_records: int = 0, slab_tasks: int = 0) -> None:
        self._check(self._lib.vxe_set_record_limits(self._ctx, probe_records, slab_tasks), "vxe_set_record_limits")

    def frame_stats(self) -> dict:
        st = A.FrameStats()
        self._check(self._lib.vxe_get_frame_stats(self._ctx, C.byref(st)), "vxe_get_frame_stats")
        return {k: int(getattr(st, k)) for k, _ in A.FrameStats._fields_ if not k.startswith("_")}

    # -- images -----------------------------------------------------------------
    _IMG_SHAPES = {
        A.IMG_COLOR: ("i", 4, np.float32), A.IMG_DEPTH: ("i", 1, np.float32), A.IMG_LOCAL: ("i", 4, np.float32),
        A.IMG_PRIMARY_HIST_IN: ("i", 4, np.uint32), A.IMG_PRIMARY_HIST_OUT: ("i", 4, np.uint32),
        A.IMG_SHADOW_IN: ("i", 1, np.float32), A.IMG_SHADOW_OUT: ("i", 1, np.float32),
        A.IMG_LOCAL_HIST_IN: ("i", 4, np.float32), A.IMG_LOCAL_HIST_OUT: ("i", 4, np.float32),
        A.IMG_GODRAY_IN: ("i", 4, np.float32), A.IMG_GODRAY_OUT: ("i", 4, np.float32),
        A.IMG_OUTPUT_PRE_TAA: ("p", 4, np.float32), A.IMG_OUTPUT: ("p", 4, np.float32),
        A.IMG_OUTPUT_HIST_IN: ("p", 4, np.float32), A.IMG_OUTPUT_HIST_OUT: ("p", 4, np.float32),
    }

    def read_image_async(self, img: int, out: np.ndarray) -> int:
        """Queues a copy of image `img` into `out` (pinned host memory for an
        asynchronous copy; keep it alive until the wait) and returns a ticket
        for read_image_wait.  The next frame's write of the image waits for
        the copy (for the output only its composite pass)."""
        t = C.c_uint64()
        self._check(self._lib.vxe_read_image_async(self._ctx, img, out.ctypes.data, out.nbytes, C.byref(t)),
                    "vxe_read_image_async")
        return t.value

    def read_image_wait(self, ticket: int) -> None:
        self._check(self._lib.vxe_read_image_wait(self._ctx, ticket), "vxe_read_image_wait")

    def read_image(self, img: int) -> np.ndarray:
        if img == A.IMG_HITS:
            w, h = self.internal
            arr = np.zeros(w * h, dtype=A.HIT_DTYPE)
        else:
            which, ch, dt = self._IMG_SHAPES[img]
            w, h = self.internal if which == "i" else self.present
            arr = np.zeros((h, w, ch) if ch > 1 else (h, w), dtype=dt)
        self._check(self._lib.vxe_read_image(self._ctx, img, arr.ctypes.data, arr.nbytes), "vxe_read_image")
        return arr

    def write_image(self, img: int, arr: np.ndarray) -> None:
        a = np.ascontiguousarray(arr)
        self._check(self._lib.vxe_write_image(self._ctx, img, a.ctypes.data, a.nbytes), "vxe_write_image")

    # -- batches ----------------------------------------------------------------
    def submit_batch(self, requests, tile=(8, 8), rays_per_thread=1, mode=A.BATCH_PERSISTENT) -> A.BatchStats:
        """Traces A.Request records (device outputs) in one batch; returns device timings."""
        n = len(requests)
        arr = (A.Request * max(n, 1))(*requests)
        opt = A.BatchOptions(tile[0], tile[1], rays_per_thread, mode)
        st = A.BatchStats()
        self._check(self._lib.vxe_submit_batch(self._ctx, arr, n, C.byref(opt), C.byref(st)), "vxe_submit_batch")
        return st

    def submit_batch_async(self, lane, requests, tile=(8, 8), rays_per_thread=1, mode=A.BATCH_PERSISTENT) -> None:
        n = len(requests)
        arr = (A.Request * max(n, 1))(*requests)
        opt = A.BatchOptions(tile[0], tile[1], rays_per_thread, mode)
        self._check(self._lib.vxe_submit_batch_async(self._ctx, lane, arr, n, C.byref(opt)), "vxe_submit_batch_async")

    def batch_wait(self, lane, block=True):
        """Returns BatchStats when the lane's batch is done, None while it still runs."""
        st = A.BatchStats()
        rc = self._lib.vxe_batch_wait(self._ctx, lane, 1 if block else 0, C.byref(st))
        if rc == A.VXE_NOT_READY:
            return None
        self._check(rc, "vxe_batch_wait")
        return st

    # -- viewport sessions --------------------------------------------------------
    def view_bytes(self, width: int, height: int, render_scale: float) -> int:
        return int(self._lib.vxe_view_bytes(self._ctx, width, height, render_scale))

    def view_lane_bytes(self, width: int, height: int, render_scale: float) -> int:
        """Bytes of one lane's per-frame working buffers for views up to this size."""
        return int(self._lib.vxe_view_lane_bytes(self._ctx, width, height, render_scale))

    def view(self, width: int, height: int, render_scale: float) -> "View":
        return View(self, width, height, render_scale)

    def render_views_async(self, lane: int, views_and_cameras) -> None:
        """One frame of each (view, camera) pair on `lane`, every pass launched
        once for up to MAX_VIEWS_PER_LAUNCH views (vxe_view_render_batch_async);
        longer lists go in several launches."""
        items = list(views_and_cameras)
        for i in range(0, len(items), A.MAX_VIEWS_PER_LAUNCH):
            part = items[i:i + A.MAX_VIEWS_PER_LAUNCH]
            hs = (C.c_void_p * len(part))(*[v._h.value for v, _ in part])
            cams = (A.CameraGpu * len(part))(*[cam for _, cam in part])
            self._check(self._lib.vxe_view_render_batch_async(self._ctx, hs, cams, len(part), lane),
                        "vxe_view_render_batch_async")

    # -- queries ----------------------------------------------------------------
    def trace_rays(self, origins: np.ndarray, dirs: np.ndarray, tmax: float) -> np.ndarray:
        o = np.ascontiguousarray(origins, dtype=np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(dirs, dtype=np.float32).reshape(-1, 3)
        assert o.shape == d.shape
        out = np.zeros(len(o), dtype=A.HIT_DTYPE)
        fp = C.POINTER(C.c_float)
        self._check(self._lib.vxe_trace_rays(self._ctx, o.ctypes.data_as(fp), d.ctypes.data_as(fp), len(o),
                                             float(tmax), out.ctypes.data), "vxe_trace_rays")
        return out


class View:
    """A viewport session: its own images and histories, rendered from the
    renderer's world on a batch lane (vxe_view_*)."""

    def __init__(self, renderer: Renderer, width: int, height: int, render_scale: float):
        self._r = renderer
        self.present = (width, height)
        # round(present * scale), halves away from zero, in binary32 (as vxe_resize)
        self.internal = tuple(max(1, int(np.floor(np.float32(v) * np.float32(render_scale) + np.float32(0.5))))
                              for v in (width, height))
        h = C.c_void_p()
        renderer._check(renderer._lib.vxe_view_create(renderer._ctx, width, height, render_scale, C.byref(h)),
                        "vxe_view_create")
        self._h = h

    def render_async(self, lane: int, cam: A.CameraGpu) -> None:
        self._r._check(self._r._lib.vxe_view_render_async(self._r._ctx, self._h, lane, C.byref(cam)),
                       "vxe_view_render_async")

    def read_image(self, img: int) -> np.ndarray:
        which, ch, dt = Renderer._IMG_SHAPES[img]
        w, h = self.internal if which == "i" else self.present
        arr = np.zeros((h, w, ch) if ch > 1 else (h, w), dtype=dt)
        self._r._check(self._r._lib.vxe_view_read_image(self._r._ctx, self._h, img, arr.ctypes.data, arr.nbytes),
                       "vxe_view_read_image")
        return arr

    def close(self) -> None:
        if getattr(self, "_h", None) and self._r._ctx:
            self._r._lib.vxe_view_destroy(self._r._ctx, self._h)
        self._h = None
