"""Clipmap patch generation on the device: the texels vxe_clipmap_update_device
writes equal the CPU patches uploaded with vxe_write_clipmap, bit for bit,
over a camera path with scrolling strips, wrapped strips and full rebuilds."""
import numpy as np
import pytest

from vxe import scenes
from vxe.renderer import Renderer
from vxe.world import Clipmap

pytestmark = pytest.mark.gpu


def test_device_clipmap_equals_cpu_patches():
    sc = scenes.config5(present=(64, 36))
    levels, res = 6, 512
    cpu_clip = Clipmap(sc.spec, levels, res, 1.0)
    dev_clip = Clipmap(sc.spec, levels, res, 1.0)
    kw = dict(node_capacity=1 << 12, chunk_capacity=4, grid_capacity=4, clip_levels=levels, clip_res=res)
    a = Renderer(64, 36, 1.0, **kw)
    b = Renderer(64, 36, 1.0, **kw)
    try:
        # small steps (strips), a jump past half a level-0 window (wrapped
        # strips on coarse levels), a jump past every window (full rebuilds)
        path = [(100.0, 100.0), (100.4, 100.0), (103.7, 101.2), (140.0, 95.0), (141.0, 60.0), (2000.0, -500.0)]
        for x, z in path:
            params, patches = cpu_clip.update(x, z)
            a.write_clipmap_updates(params, patches)
            dev_clip.update_device(b, x, z)
            ta, tb = a.read_clipmap(), b.read_clipmap()
            assert np.array_equal(ta.view(np.uint32), tb.view(np.uint32)), (x, z)
            assert np.array_equal(ta, cpu_clip.tex)
    finally:
        a.close()
        b.close()
