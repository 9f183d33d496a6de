"""Viewport sessions: a view's frames equal the context's own frames for the
same camera sequence (bit-exact), on any lane, with frames moving between
lanes."""
import numpy as np
import pytest

from vxe import _abi as A
from vxe.renderer import Renderer
from vxe.scenes import FrameDriver, config2

pytestmark = pytest.mark.gpu


def test_view_frames_equal_context_frames():
    sc = config2(present=(320, 180))
    sc.shift_every = 2
    drv = FrameDriver(sc)
    ups = drv.initial_uploads()
    w = drv.world
    r = Renderer(sc.present[0], sc.present[1], sc.render_scale, node_capacity=w.node_capacity,
                 chunk_capacity=w.chunk_capacity, grid_capacity=w.grid_capacity, clip_levels=sc.clip_levels,
                 clip_res=sc.clip_res)
    v = None
    try:
        r.upload_world(w, ups)
        v = r.view(sc.present[0], sc.present[1], sc.render_scale)
        assert v.internal == r.internal
        assert r.view_bytes(*sc.present, sc.render_scale) > 0
        for f in range(4):
            u, g, clip, cam = drv.step()
            if u:
                r.apply_chunk_uploads(u)
            if g:
                r.write_chunk_grid(w.grid)
            r.write_clipmap_updates(*clip)
            r.write_camera(cam)
            r.encode_compute()
            v.render_async(f % 2, cam)  # alternate lanes: frames must stay in order
            for img in (A.IMG_OUTPUT, A.IMG_COLOR, A.IMG_DEPTH):
                a, b = r.read_image(img), v.read_image(img)
                assert a.tobytes() == b.tobytes(), (f, img)
            r.batch_wait(f % 2, block=True)
    finally:
        if v is not None:
            v.close()
        r.close()


def test_world_writes_wait_for_frames_in_flight():
    # A grid write issued while frames are queued on two lanes reaches the
    # device only after them: the frames enqueued before it see the old world,
    # the ones enqueued after it the new one -- the same images as rendering
    # one frame at a time with a full wait around the write.
    sc = config2(present=(640, 360))
    drv = FrameDriver(sc)
    ups = drv.initial_uploads()
    _, _, clip, cam = drv.step()
    w = drv.world
    r = Renderer(sc.present[0], sc.present[1], sc.render_scale, node_capacity=w.node_capacity,
                 chunk_capacity=w.chunk_capacity, grid_capacity=w.grid_capacity, clip_levels=sc.clip_levels,
                 clip_res=sc.clip_res)
    holes = w.grid.copy()
    holes[::3] = 0xFFFFFFFF  # every third cell unloaded
    views = []
    try:
        r.upload_world(w, ups)
        r.write_clipmap_updates(*clip)
        r.write_camera(cam)

        def render_all(sync):
            vs = [r.view(*sc.present, sc.render_scale) for _ in range(6)]
            views.extend(vs)
            for i, v in enumerate(vs[:3]):
                v.render_async(i % 2, cam)
                if sync:
                    r.batch_wait(i % 2, block=True)
            r.write_chunk_grid(holes)
            for i, v in enumerate(vs[3:]):
                v.render_async(i % 2, cam)
                if sync:
                    r.batch_wait(i % 2, block=True)
            r.write_chunk_grid(w.grid)
            if not sync:
                for lane in (0, 1):
                    r.batch_wait(lane, block=True)
            return [v.read_image(A.IMG_OUTPUT).tobytes() for v in vs]

        ref = render_all(sync=True)
        assert ref[0] != ref[3]  # the holes show
        got = render_all(sync=False)
        assert got == ref
    finally:
        for v in views:
            v.close()
        r.close()
