"""Drives a scene through both the CUDA context and the CPU oracle.

Every float image is compared for exact equality (+0 == -0, NaN == NaN):
the passes are specified to be bit-identical to the oracle, because both
evaluate the same IEEE binary32 op sequence with the same deterministic
transcendental functions.  Integer outputs (hit node / voxel / face / mat,
history bit patterns) must match bit for bit.
"""
from __future__ import annotations

import numpy as np

from oracle import oracle as O
from vxe import _abi as A
from vxe.renderer import Renderer
from vxe.scenes import FrameDriver


def float_mismatch(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    a = np.asarray(a, dtype=np.float32)
    b = np.asarray(b, dtype=np.float32)
    same = (a == b) | (np.isnan(a) & np.isnan(b))
    return ~same


def compare_frame(gpu: dict, ora: dict) -> dict:
    """Returns {image: mismatching element count} (empty when identical)."""
    bad = {}
    for k in ("color", "depth", "local", "shadow", "local_hist", "godray", "output_pre_taa", "output",
              "output_hist"):
        if k not in gpu:
            continue
        g = np.asarray(gpu[k]).reshape(-1)
        o = np.asarray(ora[k]).reshape(-1)
        m = int(float_mismatch(g, o).sum())
        if m:
            bad[k] = m
    if "primary_hist" in gpu:
        g = np.asarray(gpu["primary_hist"]).reshape(-1, 4)
        o = np.asarray(ora["primary_hist"]).reshape(-1, 4)
        m = int((g != o).any(axis=1).sum())
        if m:
            bad["primary_hist"] = m
    if "hits" in gpu:
        g, o = gpu["hits"], ora["hits"]
        m = int(((g["node"] != o["node"]) | (g["face"] != o["face"]) | (g["mat"] != o["mat"]) |
                 (g["voxel"] != o["voxel"]).any(axis=1) | float_mismatch(g["t"], o["t"])).sum())
        if m:
            bad["hits"] = m
    return bad


def read_gpu_frame(r: Renderer) -> dict:
    out = {
        "color": r.read_image(A.IMG_COLOR).reshape(-1, 4),
        "depth": r.read_image(A.IMG_DEPTH).reshape(-1),
        "primary_hist": r.read_image(A.IMG_PRIMARY_HIST_IN).reshape(-1, 4),
        "shadow": r.read_image(A.IMG_SHADOW_IN).reshape(-1),
        "local_hist": r.read_image(A.IMG_LOCAL_HIST_IN).reshape(-1, 4),
        "godray": r.read_image(A.IMG_GODRAY_IN).reshape(-1, 4),
        "output": r.read_image(A.IMG_OUTPUT).reshape(-1, 4),
        "output_hist": r.read_image(A.IMG_OUTPUT_HIST_IN).reshape(-1, 4),
    }
    if r.flags & A.FLAG_DEBUG_INTERMEDIATES:
        out["local"] = r.read_image(A.IMG_LOCAL).reshape(-1, 4)
        out["output_pre_taa"] = r.read_image(A.IMG_OUTPUT_PRE_TAA).reshape(-1, 4)
    if r.flags & A.FLAG_HIT_RECORDS:
        out["hits"] = r.read_image(A.IMG_HITS)
    return out


def make_renderer(scene, world, flags=A.FLAG_GODRAY_MACRO_ALIAS | A.FLAG_HIT_RECORDS | A.FLAG_DEBUG_INTERMEDIATES,
                  checked: bool = False):
    return Renderer(scene.present[0], scene.present[1], scene.render_scale, node_capacity=world.node_capacity,
                    chunk_capacity=world.chunk_capacity, grid_capacity=world.grid_capacity,
                    clip_levels=max(1, scene.clip_levels), clip_res=scene.clip_res, flags=flags, checked=checked)


def run_parity(scene, frames: int, threads: int | None = None, godray_alias: bool = True, on_frame=None,
               extra_flags: int = 0, graph: bool = False, flags: int | None = None, start_frame: int = 0,
               cam_hook=None, setup=None, budgeted: bool = False):
    """Renders `frames` frames on both sides; returns a list of per-frame mismatch dicts.

    `flags`: the context flags (default: hit records + debug intermediates +
    the godray alias, | extra_flags).  `start_frame`: first path frame.
    `cam_hook(cam)`: edits each frame's camera before both sides see it.
    `setup(renderer)`: called once after the world upload.  `budgeted`:
    chunk streaming under the per-frame upload budget (FrameDriver)."""
    drv = FrameDriver(scene, start_frame=start_frame, budgeted=budgeted)
    ups = drv.initial_uploads()
    if flags is None:
        flags = A.FLAG_HIT_RECORDS | A.FLAG_DEBUG_INTERMEDIATES | (A.FLAG_GODRAY_MACRO_ALIAS if godray_alias else 0)
        flags |= extra_flags
    godray_alias = bool(flags & A.FLAG_GODRAY_MACRO_ALIAS)
    r = make_renderer(scene, drv.world, flags)
    try:
        r.upload_world(drv.world, ups)
        if setup is not None:
            setup(r)
        ora = O.OracleFrameRunner(drv.world, scene.internal, scene.present,
                                  drv.clip.tex if drv.clip else None, scene.clip_res, godray_alias=godray_alias)
        results = []
        for _ in range(frames):
            uploads, grid_changed, clip, cam = drv.step()
            if uploads:
                r.apply_chunk_uploads(uploads)
            if grid_changed:
                r.write_chunk_grid(drv.world.grid)
            if clip is not None:
                params, patches = clip
                r.write_clipmap_updates(params, patches)
            else:
                params = drv.empty_clip()
                r.write_clipmap_updates(params, [])
            if cam_hook is not None:
                cam_hook(cam)
            r.write_camera(cam)
            if graph:
                r.render_frame_graph()
            else:
                r.encode_compute()
            ora.render(cam, params, threads=threads)
            g = read_gpu_frame(r)
            o = ora.outputs()
            bad = compare_frame(g, o)
            results.append(bad)
            if on_frame:
                on_frame(g, o, bad, r, ora)
        assert r.read_error_word() == 0
        return results
    finally:
        r.close()


def run_resident_parity(scene, frames, flags=A.FLAG_GODRAY_MACRO_ALIAS, threads=None):
    """The device-resident frames of a shifting path (vxe.scenes.ResidentPathDriver:
    every chunk the path visits uploaded once, grid windows rewritten at the
    shifts) for the path frames in `frames`, on both sides; per-frame mismatch
    dicts."""
    from vxe.scenes import ResidentPathDriver

    drv = ResidentPathDriver(scene)
    ups = drv.initial_uploads()
    w = drv.world
    r = Renderer(scene.present[0], scene.present[1], scene.render_scale, node_capacity=w.node_capacity,
                 chunk_capacity=w.chunk_capacity, grid_capacity=int(np.prod(scene.grid_dims)),
                 clip_levels=scene.clip_levels, clip_res=scene.clip_res, flags=flags)
    try:
        r.apply_chunk_uploads(ups)
        ora = O.OracleFrameRunner(w, scene.internal, scene.present, drv.clip.tex, scene.clip_res,
                                  godray_alias=bool(flags & A.FLAG_GODRAY_MACRO_ALIAS))
        grid = None
        results = []
        for f in frames:
            cam, params, patches, g = drv.inputs(f)
            if g is not None:
                grid = g
                r.write_chunk_grid(grid)
            r.write_clipmap_updates(params, patches)
            r.write_camera(cam)
            r.encode_compute()
            ora.render(cam, params, threads=threads, grid=grid)
            results.append(compare_frame(read_gpu_frame(r), ora.outputs()))
        assert r.read_error_word() == 0
        return results
    finally:
        r.close()
