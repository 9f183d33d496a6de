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


def test_async_output_reads_equal_sync_reads():
    """Pipelined read-back: frame i's output copied on the copy stream while
    frame i+1 is queued behind it (the composite waits for the copy), two host
    buffers, each waited one step later -- the same bytes as reading every
    frame synchronously; an image other than the output delays the whole next
    frame and reads back the same too."""
    import torch

    sc = config2(present=(640, 360))
    sc.shift_every = 3
    runs = []
    for pipelined in (False, True):
        drv = FrameDriver(sc)
        ups = drv.initial_uploads()
        w = drv.world
        r = Renderer(sc.present[0], sc.present[1], sc.render_scale, node_capacity=w.node_capacity,
                     chunk_capacity=w.chunk_capacity, grid_capacity=w.grid_capacity, clip_levels=sc.clip_levels,
                     clip_res=sc.clip_res)
        try:
            r.upload_world(w, ups)
            pw, ph = sc.present
            iw, ih = r.internal
            bufs = [torch.empty((ph, pw, 4), dtype=torch.float32).pin_memory().numpy() for _ in range(2)]
            depth = [torch.empty((ih, iw), dtype=torch.float32).pin_memory().numpy() for _ in range(2)]
            outs, depths, prev = [], [], None
            for f in range(6):
                u, g, clip, cam = drv.step()
                if u:
                    r.apply_chunk_uploads(u)
                if g:
                    r.write_chunk_grid(w.grid)
                r.write_clipmap_updates(*clip)
                r.write_camera(cam)
                if pipelined:
                    r.encode_compute(sync=False)
                    t = r.read_image_async(A.IMG_OUTPUT, bufs[f % 2])
                    td = r.read_image_async(A.IMG_DEPTH, depth[f % 2])
                    if prev is not None:
                        r.read_image_wait(prev[0])
                        r.read_image_wait(prev[1])
                        outs.append(bufs[(f - 1) % 2].tobytes())
                        depths.append(depth[(f - 1) % 2].tobytes())
                    prev = (t, td)
                else:
                    r.encode_compute()
                    outs.append(r.read_image(A.IMG_OUTPUT).tobytes())
                    depths.append(r.read_image(A.IMG_DEPTH).tobytes())
            if pipelined:
                r.read_image_wait(prev[0])
                r.read_image_wait(prev[1])
                outs.append(bufs[5 % 2].tobytes())
                depths.append(depth[5 % 2].tobytes())
            runs.append((outs, depths))
        finally:
            r.close()
    assert runs[0][0] == runs[1][0]
    assert runs[0][1] == runs[1][1]
    assert len(set(runs[0][0])) > 1  # the frames differ


def test_views_rendered_in_one_launch_equal_views_rendered_alone():
    # vxe_view_render_batch_async: several views of different sizes and
    # cameras, every pass launched once for all of them, give each view the
    # frames it gets rendered alone -- over frames with histories feeding back
    # (and the histories' ping-pong) and on both lanes.
    from vxe.serve import make_sessions

    sc = config2(present=(320, 180))
    drv = FrameDriver(sc)
    ups = drv.initial_uploads()
    _, _, clip, cam = drv.step()
    w = drv.world
    r = Renderer(sc.present[0], sc.present[1], sc.render_scale, node_capacity=w.node_capacity,
                 chunk_capacity=w.chunk_capacity, grid_capacity=w.grid_capacity, clip_levels=sc.clip_levels,
                 clip_res=sc.clip_res)
    sessions = make_sessions(w, 5, seed=9, size_range=((96, 640), (64, 360)))
    together, alone = [], []
    try:
        r.upload_world(w, ups)
        r.write_clipmap_updates(*clip)
        r.write_camera(cam)
        together = [r.view(s.w, s.h, s.render_scale) for s in sessions]
        alone = [r.view(s.w, s.h, s.render_scale) for s in sessions]
        prev = [None] * len(sessions)
        for f in range(3):
            cams = []
            for i, s in enumerate(sessions):
                c = s.camera(w, f, prev[i])
                prev[i] = c.view_proj
                cams.append(c)
            r.render_views_async(f % 2, list(zip(together, cams)))
            for v, c in zip(alone, cams):
                v.render_async(1 - f % 2, c)
            for img in (A.IMG_OUTPUT, A.IMG_COLOR, A.IMG_DEPTH, A.IMG_PRIMARY_HIST_IN, A.IMG_GODRAY_IN):
                for i, (a, b) in enumerate(zip(together, alone)):
                    assert a.read_image(img).tobytes() == b.read_image(img).tobytes(), (f, img, i)
            r.batch_wait(0, block=True)
            r.batch_wait(1, block=True)
    finally:
        for v in together + alone:
            v.close()
        r.close()
