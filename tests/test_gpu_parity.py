"""GPU parity: the CUDA passes against the CPU oracle, through the C ABI.

Bar: bit-exact (every float image equal element-wise, hit records identical).
"""
import numpy as np
import pytest

from parity import float_mismatch, run_parity
from vxe import _abi as A
from vxe import scenes
from vxe.scenes import FrameDriver

pytestmark = pytest.mark.gpu


def test_config1_single_chunk_frame_bit_exact():
    sc = scenes.config1()
    res = run_parity(sc, frames=1)
    assert res == [{}], res


def test_config1_temporal_frames_bit_exact():
    # Same camera, histories feeding back: exercises the hit-distance hint,
    # anchors, shadow reuse, local and composite TAA.
    sc = scenes.config1()
    sc.frames = 6
    res = run_parity(sc, frames=6)
    assert all(r == {} for r in res), res


def test_features_scene_all_shading_paths_bit_exact():
    sc = scenes.features()
    res = run_parity(sc, frames=4)
    assert all(r == {} for r in res), res


def test_features_scene_megakernel_schedule_bit_exact():
    # The one-kernel-per-pixel schedule must give the same images as the wavefront.
    sc = scenes.features()
    res = run_parity(sc, frames=3, extra_flags=A.FLAG_PRIMARY_MEGAKERNEL)
    assert all(r == {} for r in res), res


def test_frames_as_cuda_graph_bit_exact():
    # vxe_render_frame_graph: captured on the first frame, relaunched with new
    # arguments afterwards (camera, clipmap, ping-pong images) -- including a
    # grid shift with chunk uploads between frames.
    sc = scenes.config2(present=(320, 180))
    sc.shift_every = 2
    res = run_parity(sc, frames=4, graph=True)
    assert all(r == {} for r in res), res


def test_features_scene_without_grass_table_bit_exact():
    # Every grass march derives its blades itself (no per-frame cell table):
    # the same images as the table path and the oracle.
    sc = scenes.features()
    res = run_parity(sc, frames=2, extra_flags=A.FLAG_NO_GRASS_TABLE)
    assert all(r == {} for r in res), res


def test_features_scene_godray_alias_off_bit_exact():
    sc = scenes.features()
    res = run_parity(sc, frames=2, godray_alias=False)
    assert all(r == {} for r in res), res


def test_config2_world_with_grid_shift_bit_exact():
    # Full 16x4x16 world and 5-level clipmap at reduced resolution; a grid
    # shift (uploads + slot moves + grid rewrite) happens before frame 2.
    sc = scenes.config2(present=(320, 180))
    sc.shift_every = 2
    res = run_parity(sc, frames=3)
    assert all(r == {} for r in res), res


def test_queries_match_oracle():
    from oracle import oracle as O
    from parity import make_renderer

    sc = scenes.config2(present=(64, 36))
    drv = FrameDriver(sc)
    ups = drv.initial_uploads()
    _, _, clip, cam = drv.step()
    r = make_renderer(sc, drv.world)
    try:
        r.upload_world(drv.world, ups)
        r.write_camera(cam)
        rng = np.random.default_rng(5)
        lo, hi = drv.world.world_aabb_m()
        n = 20000
        o = rng.uniform(lo, hi, size=(n, 3)).astype(np.float32)
        d = rng.normal(size=(n, 3))
        d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
        g = r.trace_rays(o, d, 120.0)
        ref, _ = O.trace_rays(drv.world, cam, o, d, 120.0)
        assert (g["face"] != 255).mean() > 0.2
        for f in ("node", "face", "mat"):
            assert np.array_equal(g[f], ref[f]), f
        assert np.array_equal(g["voxel"], ref["voxel"])
        assert not float_mismatch(g["t"], ref["t"]).any()
    finally:
        r.close()


def test_detmath_device_equals_host():
    import ctypes as C

    from oracle import oracle as O

    rng = np.random.default_rng(0)
    x = np.concatenate([rng.uniform(-1e4, 1e4, 4000), rng.uniform(-10, 10, 4000), rng.uniform(0, 2, 2000),
                        np.array([0.0, -0.0, 1.0, np.pi, 1e-30, 88.0, -100.0, 3e5, np.inf, -np.inf, np.nan])])
    x = x.astype(np.float32)
    y = rng.uniform(-3, 100, x.size).astype(np.float32)
    y[:16] = np.array([0.0, -0.0, 0.0, np.nan, -0.0, 0.0, 1.0, -1.0, 0.5, 2.0, 8.0, 1.8, 5.0, 0.98, 96.0, 1.5])
    lib = A.lib()
    for which in range(6):
        xs = np.abs(x) if which == 3 else x
        dev = np.zeros_like(xs)
        st = lib.vxe_debug_detmath(which, xs.ctypes.data, y.ctypes.data, dev.ctypes.data, xs.size)
        assert st == 0
        host = O.detmath(which, xs, y)
        bad = float_mismatch(dev, host)
        # min/max: the sign of a zero result is compared too
        if which >= 4:
            bad |= (np.signbit(dev) != np.signbit(host)) & (dev == 0)
        assert not bad.any(), (which, xs[bad][:5], dev[bad][:5], host[bad][:5])


def test_upload_capacity_error_and_silent_skip():
    from parity import make_renderer

    sc = scenes.config1()
    drv = FrameDriver(sc)
    ups = drv.initial_uploads()
    r = make_renderer(sc, drv.world)
    try:
        bad = ups[0]
        bad.node_base = drv.world.node_capacity - 1
        bad.meta = bad.meta.copy()
        bad.meta[4] = bad.node_base
        with pytest.raises(A.VxeError) as ei:
            r.apply_chunk_uploads([bad])
        assert ei.value.status == 2
        r.set_flags(r.flags | A.FLAG_SILENT_CAPACITY_SKIP)
        r.apply_chunk_uploads([bad])  # skipped like the reference
    finally:
        r.close()


def test_config5_large_world_bit_exact():
    # The 32x8x32-chunk world (8192 slots, caves above 0.5) with its 6-level
    # 512^2 clipmap, at reduced resolution: bit-exact like the small worlds.
    sc = scenes.config5(present=(320, 180))
    res = run_parity(sc, frames=2)
    assert all(r == {} for r in res), res
