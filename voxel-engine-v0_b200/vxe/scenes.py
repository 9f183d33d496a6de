"""Seeded synthetic workloads (the reference publishes no benchmark data).

* ``config1``: one 64^3 chunk (heights 8-48, grass/dirt(3)/stone, 2 % carved),
  pinhole 60 deg camera outside the chunk looking at its centre, 256x144 rays.
* ``config2``: 16x4x16 chunks with 3D value-noise caves (threshold 0.6), a
  5-level 256^2 toroidal clipmap, 1920x1080 present / 960x540 internal, a
  64-frame Catmull-Rom camera path at 0.15 m (1.5 voxels) per frame and a
  chunk-grid shift of +1 chunk in x every 16 frames.
* ``config5``: 32x8x32 chunks with caves above 0.5, a 6-level 512^2 clipmap,
  3840x2160 present / 1920x1080 internal, a 128-frame path.
* ``features``: a small world with caves, carving, trees (wood + leaves) and
  light voxels so every shading path (leaf displacement, grass, voxel lights)
  is exercised by the parity tests.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi as A
from .world import Clipmap, UploadQueue, World, WorldSpec, build_camera, ground_height


@dataclass
class Scene:
    name: str
    spec: WorldSpec
    grid_origin: tuple
    grid_dims: tuple
    present: tuple
    render_scale: float
    clip_levels: int
    clip_res: int
    frames: int
    node_capacity: int
    shift_every: int = 0          # frames between +1 chunk grid shifts in x (0 = never)
    path: object = None           # callable frame -> (pos, yaw, pitch)
    jitter: bool = True

    @property
    def internal(self):
        return (max(1, round(self.present[0] * self.render_scale)), max(1, round(self.present[1] * self.render_scale)))


def _look_at(pos, target):
    d = np.asarray(target, dtype=np.float64) - np.asarray(pos, dtype=np.float64)
    yaw = math.atan2(d[0], d[2])
    pitch = math.asin(d[1] / np.linalg.norm(d))
    return yaw, pitch


def config1(seed: int = 12345) -> Scene:
    spec = WorldSpec(seed=seed, height_min=8, height_max=48, dirt_depth=3, carve_mod=50, cave_threshold=2.0)
    rng = np.random.default_rng(seed)
    center = np.array([3.2, 3.2, 3.2])
    ang = rng.uniform(0, 2 * math.pi)
    elev = rng.uniform(0.35, 0.7)
    dist = rng.uniform(6.0, 7.5)
    pos = center + dist * np.array([math.cos(elev) * math.sin(ang), math.sin(elev), math.cos(elev) * math.cos(ang)])
    yaw, pitch = _look_at(pos, center)
    return Scene("config1", spec, (0, 0, 0), (1, 1, 1), (256, 144), 1.0, 0, 256, 1, node_capacity=1 << 18,
                 path=lambda f: (pos, yaw, pitch), jitter=False)


class CatmullRomPath:
    """Arc-length parameterised Catmull-Rom spline through seeded points."""

    def __init__(self, points, step_m: float, y_of=None):
        self.p = np.asarray(points, dtype=np.float64)
        self.step = step_m
        samples = []
        for i in range(1, len(self.p) - 2):
            p0, p1, p2, p3 = self.p[i - 1], self.p[i], self.p[i + 1], self.p[i + 2]
            for t in np.linspace(0.0, 1.0, 200, endpoint=False):
                t2, t3 = t * t, t * t * t
                samples.append(0.5 * ((2 * p1) + (-p0 + p2) * t + (2 * p0 - 5 * p1 + 4 * p2 - p3) * t2 +
                                      (-p0 + 3 * p1 - 3 * p2 + p3) * t3))
        self.s = np.asarray(samples)
        seg = np.linalg.norm(np.diff(self.s, axis=0), axis=1)
        self.cum = np.concatenate([[0.0], np.cumsum(seg)])

    def at(self, frame: int):
        d = min(frame * self.step, self.cum[-1] - 1e-6)
        i = int(np.searchsorted(self.cum, d, side="right") - 1)
        f = (d - self.cum[i]) / max(self.cum[i + 1] - self.cum[i], 1e-12)
        pos = self.s[i] * (1 - f) + self.s[i + 1] * f
        tang = self.s[i + 1] - self.s[i]
        yaw = math.atan2(tang[0], tang[2])
        return pos, yaw


def config2(seed: int = 12345, frames: int = 64, present=(1920, 1080), render_scale: float = 0.5) -> Scene:
    spec = WorldSpec(seed=seed, height_min=8, height_max=48, dirt_depth=3, carve_mod=0, cave_threshold=0.6)
    rng = np.random.default_rng(seed + 2)
    # Control points near the middle of the 102.4 m x 102.4 m world, heading +x.
    base = np.array([40.0, 7.5, 51.2])
    pts = [base + np.array([-6.0 + 4.0 * i, rng.uniform(-0.5, 0.5), rng.uniform(-3.0, 3.0)]) for i in range(8)]
    path = CatmullRomPath(pts, 0.15)

    def at(f):
        pos, yaw = path.at(f)
        return pos, yaw, -0.12

    return Scene("config2", spec, (0, 0, 0), (16, 4, 16), present, render_scale, 5, 256, frames,
                 node_capacity=12 << 20, shift_every=16, path=at)


def config5(seed: int = 12345, frames: int = 128, present=(3840, 2160), render_scale: float = 0.5) -> Scene:
    """32x8x32 chunks (204.8 x 51.2 x 204.8 m), 3D value-noise caves above 0.5, a
    6-level 512^2 clipmap, 3840x2160 present / 1920x1080 internal, a 128-frame
    Catmull-Rom path across the middle of the world."""
    spec = WorldSpec(seed=seed, height_min=8, height_max=48, dirt_depth=3, carve_mod=0, cave_threshold=0.5)
    rng = np.random.default_rng(seed + 5)
    base = np.array([70.0, 7.5, 102.4])
    pts = [base + np.array([-6.0 + 6.0 * i, rng.uniform(-0.5, 0.5), rng.uniform(-4.0, 4.0)]) for i in range(10)]
    path = CatmullRomPath(pts, 0.15)

    def at(f):
        pos, yaw = path.at(f)
        return pos, yaw, -0.12

    return Scene("config5", spec, (0, 0, 0), (32, 8, 32), present, render_scale, 6, 512, frames,
                 node_capacity=40 << 20, path=at)


def features(seed: int = 777, present=(128, 80)) -> Scene:
    spec = WorldSpec(seed=seed, height_min=10, height_max=30, dirt_depth=3, carve_mod=50, cave_threshold=0.62,
                     height_scale_vox=48.0, features=3)
    pos = np.array([5.5, 5.2, 1.0])
    target = np.array([7.0, 2.2, 6.4])
    yaw, pitch = _look_at(pos, target)

    def at(f):
        p = pos + np.array([0.05 * f, 0.0, 0.04 * f])
        return p, yaw + 0.01 * f, pitch

    return Scene("features", spec, (0, 0, 0), (3, 1, 3), present, 1.0, 3, 128, 4, node_capacity=1 << 21, path=at)


SCENES = {"config1": config1, "config2": config2, "config5": config5, "features": features}


class FrameDriver:
    """Produces per-frame inputs (uploads, grid, clipmap patches, camera) for a scene."""

    def __init__(self, scene: Scene, device_renderer=None, mirror: bool = True, start_frame: int = 0,
                 budgeted: bool = False):
        """`device_renderer`: keep the world on that renderer's device -- chunks
        built resident there, grid shifts by device slot moves (step() then
        returns no uploads and writes the grid itself).  `mirror`: the world
        keeps host copies of the node and rope arenas (World).  `start_frame`:
        the first path frame step() produces; the grid starts where the shifts
        of the earlier frames left it (histories start empty).  `budgeted`:
        host streaming through the reference's per-frame upload budget
        (UploadQueue.take_budgeted); chunks join the grid once uploaded."""
        self.scene = scene
        self.device = device_renderer
        self.last_shift = None  # (chunks built, slots moved) of the last device shift
        origin = tuple(scene.grid_origin)
        if scene.shift_every and start_frame > 0:
            origin = (origin[0] + (start_frame - 1) // scene.shift_every, origin[1], origin[2])
        self.queue = UploadQueue() if budgeted else None
        self.world = World(scene.spec, origin, scene.grid_dims, scene.node_capacity,
                           chunk_capacity=int(np.prod(scene.grid_dims)), mirror=mirror, queue=self.queue)
        self.clip = Clipmap(scene.spec, scene.clip_levels, scene.clip_res, 1.0) if scene.clip_levels else None
        self.prev_vp = None
        self.frame = start_frame

    def initial_uploads(self):
        if self.device is not None:
            self.world.populate_device(self.device)
            return []
        ups = self.world.populate()
        if self.queue is not None:  # the first frame's budget would leave chunks out: take them all now
            while len(self.queue):
                part = self.queue.take_budgeted(self.world)
                ups += part
                self.world.mark_uploaded(part)
        return ups

    def step(self):
        """Returns (uploads, grid_changed, clip (params, patches) or None, camera) for the next frame."""
        sc = self.scene
        f = self.frame
        uploads, grid_changed = [], False
        if sc.shift_every and f > 0 and f % sc.shift_every == 0:
            if self.device is not None:
                self.last_shift = self.world.shift_device(self.device, 1, 0, 0)
            else:
                uploads = self.world.shift(1, 0, 0)
                grid_changed = True
        if self.queue is not None and len(self.queue):
            uploads = self.queue.take_budgeted(self.world)
            self.world.mark_uploaded(uploads)
            grid_changed = True
        pos, yaw, pitch = sc.path(f)
        clip = None
        if self.clip is not None:
            clip = self.clip.update(float(pos[0]), float(pos[2]))
        cam = build_camera(pos, yaw, pitch, sc.present, sc.internal, frame_index=f + 1, time_s=f / 60.0,
                           world=self.world, jitter=sc.jitter, prev_view_proj=self.prev_vp)
        self.prev_vp = cam.view_proj
        self.frame += 1
        return uploads, grid_changed, clip, cam

    def empty_clip(self):
        p = A.ClipmapGpu()
        p.res = self.scene.clip_res
        return p


class ResidentPathDriver:
    """The frames of a shifting path over a world that holds every chunk the
    path visits: the grid window of frame f starts at x = f // shift_every, so
    a grid shift rewrites the grid and moves no chunk.  Frame f of the path is
    frame f % frames.  This is the device-resident workload: every chunk is
    uploaded once, before the frames."""

    def __init__(self, scene: Scene, shifts: int = 3):
        self.scene = scene
        nx, ny, nz = scene.grid_dims
        dims = (nx + shifts, ny, nz)
        self.world = World(scene.spec, scene.grid_origin, dims, scene.node_capacity, chunk_capacity=int(np.prod(dims)))
        self.clip = Clipmap(scene.spec, scene.clip_levels, scene.clip_res, 1.0)
        self.prev_vp = None
        self.last_ox = None

    def initial_uploads(self):
        return self.world.populate()

    def grid_window(self, ox: int) -> np.ndarray:
        """chunk_grid of the scene's grid dims at origin x = ox over the world's slots."""
        nx, ny, nz = self.scene.grid_dims
        g = np.full(nx * ny * nz, A.INVALID_U32, dtype=np.uint32)
        oy, oz = self.scene.grid_origin[1], self.scene.grid_origin[2]
        for iz in range(nz):
            for iy in range(ny):
                for ix in range(nx):
                    s = self.world.key_to_slot.get((ox + ix, oy + iy, oz + iz))
                    if s is not None:
                        g[(iz * ny + iy) * nx + ix] = s
        return g

    def inputs(self, step: int):
        """(camera, clipmap params, clipmap patches, grid or None when unchanged) of path frame step % frames."""
        sc = self.scene
        f = step % sc.frames
        ox = sc.grid_origin[0] + (f // sc.shift_every if sc.shift_every else 0)
        pos, yaw, pitch = sc.path(f)
        cam = build_camera(pos, yaw, pitch, sc.present, sc.internal, frame_index=f + 1, time_s=f / 60.0, world=None,
                           jitter=sc.jitter, prev_view_proj=self.prev_vp)
        cam.chunk_count = self.world.chunk_count
        cam.grid_origin_chunk[0], cam.grid_origin_chunk[1], cam.grid_origin_chunk[2] = \
            ox, sc.grid_origin[1], sc.grid_origin[2]
        cam.grid_dims[0], cam.grid_dims[1], cam.grid_dims[2] = sc.grid_dims
        self.prev_vp = cam.view_proj
        params, patches = self.clip.update(float(pos[0]), float(pos[2]))
        grid = None
        if ox != self.last_ox:
            grid = self.grid_window(ox)
            self.last_ox = ox
        return cam, params, patches, grid
