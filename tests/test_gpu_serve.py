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
