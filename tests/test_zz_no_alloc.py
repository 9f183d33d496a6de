"""The allocation-free entry point against the context path.

vxe_trace_primary_hits_noalloc serves callers that may not allocate device
memory themselves (an allocation-free frame loop, or an engine whose device
memory all comes from its own allocator).  It must return exactly the hit
records the regular context writes on a cold frame (first frame after
vxe_resize), bit for bit, and keep doing so on back-to-back calls that share
its fixed scratch array.  This file is named to run last.
"""
import ctypes as C

import numpy as np
import pytest

from vxe import _abi as A
from vxe.renderer import Renderer
from vxe.scenes import FrameDriver, features

pytestmark = pytest.mark.gpu


def _dev(arr, torch):
    return torch.from_numpy(np.ascontiguousarray(arr).view(np.uint8).reshape(-1)).cuda()


def test_noalloc_hits_equal_context_hits_on_two_calls():
    import torch

    sc = features(present=(120, 72))
    drv = FrameDriver(sc)
    ups = drv.initial_uploads()
    w = drv.world
    frames = [drv.step() for _ in range(3)]
    cams = [frames[0][3], frames[2][3]]
    clip_params = frames[2][2][0]  # layers in drv.clip.tex are the state after frame 2
    r = Renderer(sc.present[0], sc.present[1], sc.render_scale, node_capacity=w.node_capacity,
                 chunk_capacity=w.chunk_capacity, grid_capacity=w.grid_capacity, clip_levels=sc.clip_levels,
                 clip_res=sc.clip_res, flags=A.FLAG_GODRAY_MACRO_ALIAS | A.FLAG_HIT_RECORDS)
    bufs = {}
    try:
        r.upload_world(w, ups)
        levels, res = drv.clip.tex.shape[0], drv.clip.tex.shape[1]
        r.write_clipmap_updates(clip_params, [(l, 0, 0, res, res, drv.clip.tex[l]) for l in range(levels)])
        bufs = {k: _dev(v, torch) for k, v in dict(nodes=w.nodes, ropes=w.ropes, metas=w.metas, macro=w.macro,
                                                    colinfo=w.colinfo, grid=w.grid, clip=drv.clip.tex).items()}
        sv = A.SceneView(bufs["nodes"].data_ptr(), bufs["ropes"].data_ptr(), len(w.nodes), bufs["metas"].data_ptr(),
                         bufs["macro"].data_ptr(), bufs["colinfo"].data_ptr(), w.chunk_capacity, len(w.grid),
                         bufs["grid"].data_ptr(), bufs["clip"].data_ptr(), levels, res)
        iw, ih = sc.internal
        d_hits = torch.zeros(iw * ih * 32, dtype=torch.uint8, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        lib = A.lib()
        for cam in cams:  # two calls in a row through the same scratch
            r.resize_output(*sc.present)  # cold histories, like the entry point
            r.write_camera(cam)
            r.encode_compute()
            want = r.read_image(A.IMG_HITS)
            d_hits.fill_(0xAB)
            st = lib.vxe_trace_primary_hits_noalloc(C.byref(sv), C.byref(cam), C.byref(clip_params),
                                                    d_hits.data_ptr(), stream)
            assert st == A.VXE_OK, A.STATUS_NAMES.get(st, st)
            got = d_hits.cpu().numpy().view(A.HIT_DTYPE)
            assert (want["face"] != 255).mean() > 0.3
            assert got.tobytes() == want.tobytes()
        # sizes beyond the stated maximum are rejected before any launch
        big = A.CameraGpu()
        C.memmove(C.byref(big), C.byref(cams[0]), C.sizeof(big))
        big.render_present_px[0], big.render_present_px[1] = 4096, 2304
        st = lib.vxe_trace_primary_hits_noalloc(C.byref(sv), C.byref(big), C.byref(clip_params), d_hits.data_ptr(),
                                                stream)
        assert st == 2  # VXE_ERR_CAPACITY
        # a scene whose node records end after the first root, on the checked
        # build: every read past it is bounds checked (zero record, error
        # word) and reported; its next call clears its error word and is
        # exact again
        short = A.SceneView(*[getattr(sv, f) for f, _ in A.SceneView._fields_])
        short.node_count = 1
        chk = A.lib(checked=True)
        st = chk.vxe_trace_primary_hits_noalloc(C.byref(short), C.byref(cams[0]), C.byref(clip_params),
                                                d_hits.data_ptr(), stream)
        assert st == 6  # VXE_ERR_BOUNDS
        for l in (chk, lib):
            st = l.vxe_trace_primary_hits_noalloc(C.byref(sv), C.byref(cams[1]), C.byref(clip_params),
                                                  d_hits.data_ptr(), stream)
            assert st == A.VXE_OK
            assert d_hits.cpu().numpy().view(A.HIT_DTYPE).tobytes() == want.tobytes()
    finally:
        r.close()
        bufs.clear()
