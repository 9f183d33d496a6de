"""TEST INFRASTRUCTURE ONLY -- ctypes driver of the CPU oracle (vxe_oracle.cpp).

Used by tests/, __graft_entry__.smoke() and bench.py's CPU baseline to check
the CUDA passes; the product never imports this module.  The oracle reads the
same host mirrors (World arrays, camera, clipmap layers) that are uploaded to
the device and keeps its own ping-pong histories, mirroring
Renderer::encode_compute (render/state/mod.rs:329-446).
"""
from __future__ import annotations

import ctypes as C
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent
sys.path.insert(0, str(REPO / "voxel-engine-v0_b200"))

from vxe import _abi as A  # noqa: E402

LIB_PATH = HERE / "liboracle_vxe.so"


class OraScene(C.Structure):
    _fields_ = [("cam", C.c_void_p), ("chunks", C.c_void_p), ("chunks_n", C.c_uint64), ("nodes", C.c_void_p),
                ("nodes_n", C.c_uint64), ("grid", C.c_void_p), ("grid_n", C.c_uint64), ("macro_words", C.c_void_p),
                ("macro_n", C.c_uint64), ("ropes", C.c_void_p), ("ropes_n", C.c_uint64), ("colinfo", C.c_void_p),
                ("colinfo_n", C.c_uint64), ("clip", C.c_void_p), ("clip_tex", C.c_void_p),
                ("clip_layers", C.c_uint32), ("clip_res", C.c_uint32), ("godray_macro_alias", C.c_uint32),
                ("_pad", C.c_uint32)]


class OraCounters(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("node_loads", "rope_loads", "meta_loads", "grid_loads", "macro_loads",
                                           "colinfo_loads", "clip_loads", "oob")]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class FrameIO(C.Structure):
    _fields_ = [("iw", C.c_uint32), ("ih", C.c_uint32), ("pw", C.c_uint32), ("ph", C.c_uint32)] + [
        (n, C.c_void_p) for n in ("primary_hist_in", "shadow_in", "local_hist_in", "godray_hist_in",
                                  "output_hist_in", "color", "depth", "local", "primary_hist_out", "shadow_out",
                                  "local_hist_out", "godray_out", "output_pre_taa", "output", "output_hist_out",
                                  "hits", "profile")]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(f"{LIB_PATH} missing; run voxel-engine-v0_b200/vxe_build.py")
        l = C.CDLL(str(LIB_PATH))
        l.ora_render_frame.restype = C.c_int
        l.ora_render_frame.argtypes = [C.POINTER(OraScene), C.POINTER(FrameIO), C.c_int, C.POINTER(OraCounters),
                                       C.POINTER(OraCounters), C.POINTER(OraCounters)]
        l.ora_primary_rows.restype = C.c_int
        l.ora_primary_rows.argtypes = [C.POINTER(OraScene), C.POINTER(FrameIO), C.c_uint32, C.c_uint32, C.c_int,
                                       C.POINTER(OraCounters)]
        l.ora_tile_lists.restype = C.c_int
        l.ora_tile_lists.argtypes = [C.POINTER(OraScene), C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p]
        l.ora_trace_rays.restype = C.c_int
        l.ora_trace_rays.argtypes = [C.POINTER(OraScene), C.c_void_p, C.c_void_p, C.c_uint32, C.c_float, C.c_void_p,
                                     C.c_int, C.POINTER(OraCounters)]
        l.ora_detmath.restype = None
        l.ora_detmath.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]
        l.ora_debug_grass.restype = None
        l.ora_debug_grass.argtypes = [C.c_int, C.c_uint32, C.c_void_p, C.c_void_p]
        l.ora_sizeof_frameio.restype = C.c_uint64
        assert l.ora_sizeof_frameio() == C.sizeof(FrameIO), "FrameIO layout mismatch"
        _lib = l
    return _lib


def default_threads() -> int:
    return max(1, os.cpu_count() or 1)


class OracleFrameRunner:
    """Runs frames on the CPU with the same ping-pong as the device context."""

    def __init__(self, world, internal, present, clip_tex=None, clip_res=256, godray_alias=True):
        self.world = world
        self.iw, self.ih = internal
        self.pw, self.ph = present
        self.clip_tex = clip_tex
        self.clip_res = clip_res
        self.godray_alias = godray_alias
        n, p = self.iw * self.ih, self.pw * self.ph
        z4 = lambda m: np.zeros((m, 4), dtype=np.float32)
        self.hist = [np.zeros((n, 4), dtype=np.uint32) for _ in range(2)]
        self.shadow = [np.zeros(n, dtype=np.float32) for _ in range(2)]
        self.lhist = [z4(n) for _ in range(2)]
        self.god = [z4(n) for _ in range(2)]
        self.ohist = [z4(p) for _ in range(2)]
        self.color, self.depth, self.local = z4(n), np.zeros(n, dtype=np.float32), z4(n)
        self.pre_taa, self.output = z4(p), z4(p)
        self.hits = np.zeros(n, dtype=A.HIT_DTYPE)
        # profile_counts (VOXEL, GRASS, HDR, FOG, SHADOW), accumulated over
        # frames rendered with cam.profile_flags & 1 until reset
        self.profile = np.zeros(5, dtype=np.uint32)
        self.ping = 0
        self.primary_ctr = OraCounters()
        self.godray_ctr = OraCounters()

    def scene(self, cam, clip_params, grid=None) -> OraScene:
        """`grid`: a chunk grid to read instead of the world's own (a window
        of the camera's grid dims over a world holding more slots)."""
        w = self.world
        g = w.grid if grid is None else np.ascontiguousarray(grid, dtype=np.uint32)
        self._grid_ref = g
        s = OraScene()
        s.cam = C.addressof(cam)
        s.chunks, s.chunks_n = w.metas.ctypes.data, w.metas.shape[0]
        s.nodes, s.nodes_n = w.nodes.ctypes.data, len(w.nodes)
        s.grid, s.grid_n = g.ctypes.data, len(g)
        s.macro_words, s.macro_n = w.macro.ctypes.data, len(w.macro)
        s.ropes, s.ropes_n = w.ropes.ctypes.data, len(w.ropes)
        s.colinfo, s.colinfo_n = w.colinfo.ctypes.data, len(w.colinfo)
        s.clip = C.addressof(clip_params)
        if self.clip_tex is not None:
            s.clip_tex = self.clip_tex.ctypes.data
            s.clip_layers = self.clip_tex.shape[0]
            s.clip_res = self.clip_tex.shape[1]
        s.godray_macro_alias = 1 if self.godray_alias else 0
        return s

    def render(self, cam, clip_params, threads: int | None = None, grid=None) -> None:
        p, q = self.ping, 1 - self.ping
        io = FrameIO(self.iw, self.ih, self.pw, self.ph)
        io.primary_hist_in = self.hist[p].ctypes.data
        io.shadow_in = self.shadow[p].ctypes.data
        io.local_hist_in = self.lhist[p].ctypes.data
        io.godray_hist_in = self.god[p].ctypes.data
        io.output_hist_in = self.ohist[p].ctypes.data
        io.color, io.depth, io.local = self.color.ctypes.data, self.depth.ctypes.data, self.local.ctypes.data
        io.primary_hist_out = self.hist[q].ctypes.data
        io.shadow_out = self.shadow[q].ctypes.data
        io.local_hist_out = self.lhist[q].ctypes.data
        io.godray_out = self.god[q].ctypes.data
        io.output_pre_taa, io.output = self.pre_taa.ctypes.data, self.output.ctypes.data
        io.output_hist_out = self.ohist[q].ctypes.data
        io.hits = self.hits.ctypes.data
        io.profile = self.profile.ctypes.data
        sc = self.scene(cam, clip_params, grid)
        self.primary_ctr = OraCounters()
        self.godray_ctr = OraCounters()
        self.trace_ctr = OraCounters()  # the voxel trace phase of the primary pass
        rc = lib().ora_render_frame(C.byref(sc), C.byref(io), threads or default_threads(),
                                    C.byref(self.primary_ctr), C.byref(self.godray_ctr), C.byref(self.trace_ctr))
        assert rc == 0
        self.ping = q

    def primary_rows(self, cam, clip_params, tile_y0: int, tile_y1: int, threads: int | None = None) -> int:
        """The primary pass (with local TAA) over tile rows [tile_y0, tile_y1)
        only, without touching the histories' ping-pong; returns the rays
        traced.  For bounded CPU timings."""
        p, q = self.ping, 1 - self.ping
        io = FrameIO(self.iw, self.ih, self.pw, self.ph)
        io.primary_hist_in = self.hist[p].ctypes.data
        io.shadow_in = self.shadow[p].ctypes.data
        io.local_hist_in = self.lhist[p].ctypes.data
        io.color, io.depth, io.local = self.color.ctypes.data, self.depth.ctypes.data, self.local.ctypes.data
        io.primary_hist_out = self.hist[q].ctypes.data
        io.shadow_out = self.shadow[q].ctypes.data
        io.local_hist_out = self.lhist[q].ctypes.data
        sc = self.scene(cam, clip_params)
        ctr = OraCounters()
        rc = lib().ora_primary_rows(C.byref(sc), C.byref(io), tile_y0, tile_y1, threads or default_threads(),
                                    C.byref(ctr))
        assert rc == 0
        y0, y1 = min(tile_y0 * 8, self.ih), min(tile_y1 * 8, self.ih)
        return (y1 - y0) * self.iw

    # Frame outputs after render() (the "IN" buffers of the next frame).
    def outputs(self) -> dict:
        p = self.ping
        return {"color": self.color, "depth": self.depth, "local": self.local, "primary_hist": self.hist[p],
                "shadow": self.shadow[p], "local_hist": self.lhist[p], "godray": self.god[p],
                "output_pre_taa": self.pre_taa, "output": self.output, "output_hist": self.ohist[p],
                "hits": self.hits}


def tile_lists(world, cam, clip_params, internal):
    iw, ih = internal
    tx, ty = (iw + 7) // 8, (ih + 7) // 8
    counts = np.zeros(tx * ty, dtype=np.uint32)
    slots = np.zeros((tx * ty, 24), dtype=np.uint32)
    r = OracleFrameRunner(world, internal, internal)
    sc = r.scene(cam, clip_params)
    lib().ora_tile_lists(C.byref(sc), iw, ih, counts.ctypes.data, slots.ctypes.data)
    return counts, slots


def trace_rays(world, cam, origins, dirs, tmax, threads=None):
    o = np.ascontiguousarray(origins, dtype=np.float32).reshape(-1, 3)
    d = np.ascontiguousarray(dirs, dtype=np.float32).reshape(-1, 3)
    out = np.zeros(len(o), dtype=A.HIT_DTYPE)
    r = OracleFrameRunner(world, (8, 8), (8, 8))
    clip = A.ClipmapGpu()
    sc = r.scene(cam, clip)
    ctr = OraCounters()
    rc = lib().ora_trace_rays(C.byref(sc), o.ctypes.data, d.ctypes.data, len(o), float(tmax), out.ctypes.data,
                              threads or default_threads(), C.byref(ctr))
    assert rc == 0
    return out, ctr.as_dict()


def detmath(which: int, x, y=None):
    x = np.ascontiguousarray(x, dtype=np.float32)
    y = np.ascontiguousarray(y if y is not None else np.zeros_like(x), dtype=np.float32)
    out = np.zeros_like(x)
    lib().ora_detmath(which, x.ctypes.data, y.ctypes.data, out.ctypes.data, len(x))
    return out


def debug_grass(which: int, inputs):
    """The oracle's grass march (0: try_grass_slab_hit, 17 floats per input ->
    5) or SDF (1: grass_sdf_lod, 13 floats -> 1) on host inputs."""
    a = np.ascontiguousarray(inputs, dtype=np.float32)
    n = a.shape[0]
    out = np.zeros((n, 5 if which == 0 else 1), dtype=np.float32)
    lib().ora_debug_grass(which, n, a.ctypes.data, out.ctypes.data)
    return out
