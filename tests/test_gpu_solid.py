"""Physics solidity on the device against a host restatement of
ChunkManagerQuery::solid_voxel_at (physics/world_query.rs:80-112): colinfo
column tops for chunks of the grid, the seeded heightfield elsewhere."""
import ctypes as C

import numpy as np
import pytest

from vxe import _abi as A
from vxe import scenes
from vxe.renderer import Renderer
from vxe.scenes import FrameDriver

pytestmark = pytest.mark.gpu


def host_solid(world, wp, vox, with_world):
    out = np.zeros(len(vox), dtype=np.uint8)
    ox, oy, oz = world.grid_origin
    nx, ny, nz = world.grid_dims
    for i, (vx, vy, vz) in enumerate(vox.tolist()):
        cx, cy, cz = vx // 64, vy // 64, vz // 64
        lx, ly, lz = vx - cx * 64, vy - cy * 64, vz - cz * 64
        ix, iy, iz = cx - ox, cy - oy, cz - oz
        slot = A.INVALID_U32
        if 0 <= ix < nx and 0 <= iy < ny and 0 <= iz < nz:
            slot = int(world.grid[(iz * ny + iy) * nx + ix])
        if slot != A.INVALID_U32 and slot < world.chunk_count:
            col = lz * 64 + lx
            w = int(world.colinfo[slot * 2048 + (col >> 1)])
            v = (w & 0xFFFF) if (col & 1) == 0 else (w >> 16)
            top = v & 0xFF
            out[i] = 1 if (top != 255 and ly <= top) else 0
        elif with_world:
            out[i] = 1 if vy <= A.lib().vxe_ground_height(C.byref(wp), vx, vz) else 0
    return out


def test_solid_voxels_match_host():
    import torch

    sc = scenes.config2(present=(64, 36))
    drv = FrameDriver(sc)
    ups = drv.initial_uploads()
    _, _, clip, cam = drv.step()
    w = drv.world
    r = Renderer(64, 36, 1.0, node_capacity=w.node_capacity, chunk_capacity=w.chunk_capacity,
                 grid_capacity=w.grid_capacity, clip_levels=5, clip_res=256)
    try:
        r.upload_world(w, ups)
        r.write_camera(cam)
        rng = np.random.default_rng(11)
        # inside the grid (near the surface, 0..80 voxels up) and outside it
        inside = np.stack([rng.integers(0, 1024, 6000), rng.integers(-10, 80, 6000), rng.integers(0, 1024, 6000)], 1)
        outside = np.stack([rng.integers(-900, 2000, 3000), rng.integers(-20, 70, 3000),
                            rng.integers(-900, 2000, 3000)], 1)
        vox = np.concatenate([inside, outside]).astype(np.int32)
        wp = sc.spec.params()
        t = torch.from_numpy(vox).cuda()
        for world_params, with_world in ((wp, True), (None, False)):
            got = r.solid_voxels(t, world_params).cpu().numpy()
            ref = host_solid(w, wp, vox, with_world)
            assert np.array_equal(got, ref), int((got != ref).sum())
        assert 0.05 < got[:6000].mean() < 0.95  # both answers occur
    finally:
        r.close()
