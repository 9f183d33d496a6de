"""Batched-launch workload (64 uneven requests) and the launch-shape autotuner.

Workload (seeded): 24 pinhole viewports with width and height uniform in
[128, 1920] x [128, 1080], poses inside the world looking at the terrain, and
40 incoherent ray-query batches with log-uniform sizes in [1e3, 1e6] rays,
origins uniform in the world AABB and directions uniform on the sphere,
tmax = 120 m.  Device buffers come from torch (plumbing only).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi as A
from .world import World, build_camera

TILE_SHAPES = [(8, 4), (8, 8), (16, 8), (32, 1)]
RAYS_PER_THREAD = [1, 2, 3, 4]


@dataclass
class Batch:
    requests: list                 # A.Request
    kinds: list
    sizes: list                    # records per request
    outputs: list = field(default_factory=list)   # torch uint8 tensors (32 B per record)
    inputs: list = field(default_factory=list)    # torch tensors kept alive
    cams: list = field(default_factory=list)

    @property
    def rays(self) -> int:
        return int(sum(self.sizes))


def make_batch(world: World, torch, seed: int = 3, n_viewports: int = 24, n_queries: int = 40,
               vp_range=((128, 1920), (128, 1080)), q_range=(1e3, 1e6), device="cuda") -> Batch:
    rng = np.random.default_rng(seed)
    lo, hi = world.world_aabb_m()
    reqs, kinds, sizes, outs, ins, cams = [], [], [], [], [], []
    order = ["v"] * n_viewports + ["q"] * n_queries
    rng.shuffle(order)
    for k in order:
        r = A.Request()
        if k == "v":
            w = int(rng.integers(vp_range[0][0], vp_range[0][1] + 1))
            h = int(rng.integers(vp_range[1][0], vp_range[1][1] + 1))
            pos = np.array([rng.uniform(lo[0] + 10, hi[0] - 10), rng.uniform(6.0, 12.0),
                            rng.uniform(lo[2] + 10, hi[2] - 10)])
            yaw = rng.uniform(0, 2 * math.pi)
            pitch = rng.uniform(-0.45, 0.05)
            cam = build_camera(pos, yaw, pitch, (w, h), (w, h), frame_index=1, time_s=0.0, world=world, jitter=False)
            r.kind, r.width, r.height = A.REQ_VIEWPORT, w, h
            r.camera = cam
            cams.append(cam)
            n = w * h
        else:
            n = int(round(math.exp(rng.uniform(math.log(q_range[0]), math.log(q_range[1])))))
            o = rng.uniform(lo, hi, size=(n, 3)).astype(np.float32)
            d = rng.normal(size=(n, 3))
            d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
            to = torch.from_numpy(o).to(device)
            td = torch.from_numpy(d).to(device)
            ins += [to, td]
            r.kind, r.ray_count, r.tmax = A.REQ_QUERY, n, 120.0
            r.d_origins, r.d_dirs = to.data_ptr(), td.data_ptr()
        out = torch.empty(n * 32, dtype=torch.uint8, device=device)
        r.d_out = out.data_ptr()
        outs.append(out)
        reqs.append(r)
        kinds.append(k)
        sizes.append(n)
    return Batch(reqs, kinds, sizes, outs, ins, cams)


def autotune(renderer, batch: Batch, repeats: int = 2, mode=A.BATCH_PERSISTENT):
    """Sweeps tile shapes x rays per thread; returns (best (tile, rpt), {config: ms})."""
    results = {}
    for tile in TILE_SHAPES:
        for rpt in RAYS_PER_THREAD:
            ms = min(renderer.submit_batch(batch.requests, tile, rpt, mode).ms for _ in range(repeats))
            results[(tile, rpt)] = ms
    best = min(results, key=results.get)
    return best, results
