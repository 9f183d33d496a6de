"""Batched launches: every schedule and tuning returns exactly the records of the
single-request paths (cold-frame hit records for viewports, vxe_trace_rays for queries)."""
import numpy as np
import pytest

from vxe import _abi as A
from vxe.batch import make_batch
from vxe.renderer import Renderer
from vxe.scenes import FrameDriver, config2

pytestmark = pytest.mark.gpu


# what the module's world fixture wrote besides the world: the clipmap (host
# mirror, uniform, resolution) and the context camera
_WRITTEN = {}


@pytest.fixture(scope="module")
def world_renderer():
    import torch

    sc = config2(present=(160, 96))
    drv = FrameDriver(sc)
    ups = drv.initial_uploads()
    _, _, clip, cam = drv.step()
    w = drv.world
    r = Renderer(sc.present[0], sc.present[1], 1.0, node_capacity=w.node_capacity, chunk_capacity=w.chunk_capacity,
                 grid_capacity=w.grid_capacity, clip_levels=sc.clip_levels, clip_res=sc.clip_res,
                 flags=A.FLAG_GODRAY_MACRO_ALIAS | A.FLAG_HIT_RECORDS)
    r.upload_world(w, ups)
    r.write_clipmap_updates(*clip)
    r.write_camera(cam)
    _WRITTEN.update(clip=(drv.clip, clip[0], sc.clip_res), camera=cam)
    yield torch, w, r
    r.close()


def _records(t):
    return t.cpu().numpy().view(A.HIT_DTYPE)


def test_batch_modes_and_tunings_agree_with_single_request_paths(world_renderer):
    torch, world, r = world_renderer
    b = make_batch(world, torch, seed=7, n_viewports=5, n_queries=6, vp_range=((40, 150), (30, 90)),
                   q_range=(500, 5000))
    base = None
    for mode in (A.BATCH_PLAIN, A.BATCH_PERSISTENT, A.BATCH_GRAPH):
        for tile, rpt in [((8, 8), 1), ((32, 1), 3), ((16, 8), 2)]:
            for o in b.outputs:
                o.fill_(0xCD)
            st = r.submit_batch(b.requests, tile, rpt, mode)
            assert st.rays == b.rays
            recs = [_records(o).copy() for o in b.outputs]
            if base is None:
                base = recs
            else:
                for x, y in zip(recs, base):
                    assert x.tobytes() == y.tobytes(), (mode, tile, rpt)
    # queries == vxe_trace_rays
    for k, req, rec, inp in zip(b.kinds, b.requests, base, _query_inputs(b)):
        if k == "q":
            o, d = inp
            ref = r.trace_rays(o, d, 120.0)
            assert rec.tobytes() == ref.tobytes()
            assert (rec["face"] != 255).mean() > 0.05


def _query_inputs(b):
    it = iter(b.inputs)
    out = []
    for k in b.kinds:
        if k == "q":
            o, d = next(it), next(it)
            out.append((o.cpu().numpy(), d.cpu().numpy()))
        else:
            out.append(None)
    return out


def test_viewport_requests_match_cold_frames(world_renderer):
    torch, world, r = world_renderer
    b = make_batch(world, torch, seed=11, n_viewports=3, n_queries=0, vp_range=((64, 160), (40, 96)))
    r.submit_batch(b.requests, (8, 4), 2, A.BATCH_PERSISTENT)
    for req, out in zip(b.requests, b.outputs):
        w, h = req.width, req.height
        r.resize_output(w, h)  # render_scale 1.0: internal = present; histories reset
        cam = req.camera
        r.write_camera(cam)
        r.encode_compute()
        want = r.read_image(A.IMG_HITS)
        got = _records(out)
        assert got.tobytes() == want.tobytes()


def test_config3_batch_sample_matches_oracle(world_renderer):
    # A sample of the config-3 mix (one viewport, four incoherent query
    # batches, seeded) traced in one persistent batch, checked against the
    # oracle directly: queries against its trace_rays, the viewport against
    # the hit records of its cold frame (no history hint).
    from oracle import oracle as O

    torch, world, r = world_renderer
    clipmap, clip_params, clip_res = _WRITTEN["clip"]
    b = make_batch(world, torch, seed=5, n_viewports=1, n_queries=4, vp_range=((200, 480), (120, 270)),
                   q_range=(2e3, 5e4))
    r.submit_batch(b.requests, (8, 4), 1, A.BATCH_PERSISTENT)
    for k, req, out, inp in zip(b.kinds, b.requests, b.outputs, _query_inputs(b)):
        got = _records(out)
        if k == "q":
            o, d = inp
            ref, _ = O.trace_rays(world, _WRITTEN["camera"], o, d, 120.0)
            assert got.tobytes() == ref.tobytes()
            assert (got["face"] != 255).mean() > 0.05
        else:
            w, h = req.width, req.height
            ora = O.OracleFrameRunner(world, (w, h), (w, h), clipmap.tex, clip_res)
            ora.render(req.camera, clip_params)
            assert got.tobytes() == ora.hits.tobytes()
            assert (got["face"] != 255).mean() > 0.3
