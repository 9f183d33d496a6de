"""Serving: continuous batching with several batches in flight; every request's
records are identical alone and in the mix (bit-exact)."""
import numpy as np
import pytest

from vxe import _abi as A
from vxe.renderer import Renderer
from vxe.scenes import FrameDriver, config2
from vxe.serve import _to_request, make_arrivals, serve

pytestmark = pytest.mark.gpu


def test_served_results_equal_results_alone():
    import torch

    sc = config2(present=(160, 96))
    drv = FrameDriver(sc)
    ups = drv.initial_uploads()
    _, _, clip, cam = drv.step()
    w = drv.world
    r = Renderer(160, 96, 1.0, node_capacity=w.node_capacity, chunk_capacity=w.chunk_capacity,
                 grid_capacity=w.grid_capacity, clip_levels=5, clip_res=256)
    try:
        r.upload_world(w, ups)
        r.write_clipmap_updates(*clip)
        r.write_camera(cam)
        reqs = make_arrivals(w, rate=3000.0, count=40, seed=5, vp_range=((48, 200), (32, 120)),
                             q_range=(200, 4000))
        rep = serve(r, w, reqs, torch, mem_budget=8 << 20, lanes=3, max_batch=8, keep_outputs=True)
        s = rep.summary()
        assert s["requests"] == 40 and s["batches"] > 1
        assert all(x.done > 0 for x in reqs)
        for q in reqs:
            mixed = q.out.cpu().numpy().view(A.HIT_DTYPE).copy()
            alone = _to_request(q, torch)
            torch.cuda.synchronize()
            r.submit_batch([alone], (8, 8), 2, A.BATCH_PERSISTENT)
            got = q.out.cpu().numpy().view(A.HIT_DTYPE)
            diff = np.nonzero(got != mixed)[0]
            assert diff.size == 0, (q.rid, q.kind, q.w, q.h, q.n, diff.size, diff[:4].tolist(),
                                    str(mixed[diff[0]]), str(got[diff[0]]))
    finally:
        r.close()


def test_served_session_frames_equal_frames_alone():
    # Session frames keep their histories resident between requests; each
    # served frame equals the same session's frame rendered alone in a fresh
    # view from the same camera sequence (bit-exact), while other sessions'
    # frames and query batches share the lanes.
    import torch

    from vxe.serve import make_sessions

    sc = config2(present=(160, 96))
    drv = FrameDriver(sc)
    ups = drv.initial_uploads()
    _, _, clip, cam = drv.step()
    w = drv.world
    r = Renderer(160, 96, 0.5, node_capacity=w.node_capacity, chunk_capacity=w.chunk_capacity,
                 grid_capacity=w.grid_capacity, clip_levels=5, clip_res=256)
    try:
        r.upload_world(w, ups)
        r.write_clipmap_updates(*clip)
        r.write_camera(cam)
        sessions = make_sessions(w, 4, seed=2, size_range=((64, 200), (48, 120)))
        reqs = make_arrivals(w, rate=2000.0, count=30, seed=4, q_range=(200, 3000), sessions=sessions)
        rep = serve(r, w, reqs, torch, mem_budget=256 << 20, lanes=3, max_batch=6, keep_outputs=True,
                    sessions=sessions)
        s = rep.summary()
        assert s["requests"] == 30 and s["view_evictions"] == 0 and s["batches"] > 1
        frames = [q for q in reqs if q.kind == "f"]
        assert len(frames) > 8
        for sid, sess in enumerate(make_sessions(w, 4, seed=2, size_range=((64, 200), (48, 120)))):
            mine = sorted((q for q in frames if q.session == sid), key=lambda q: q.frame)
            if not mine:
                continue
            v = r.view(sess.w, sess.h, sess.render_scale)
            try:
                prev = None
                for f, q in enumerate(mine):
                    cam_f = sess.camera(w, f, prev)
                    prev = cam_f.view_proj
                    v.render_async(0, cam_f)
                    r.batch_wait(0, block=True)
                    assert v.read_image(A.IMG_OUTPUT).tobytes() == q.out.tobytes(), (sid, f)
            finally:
                v.close()
    finally:
        r.close()
