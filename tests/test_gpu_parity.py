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


# ---------------------------------------------------------------------------
# The bench's own configurations, at full size
# ---------------------------------------------------------------------------
def test_config2_1080p_streamed_frames_14_to_17_bit_exact():
    # The end-to-end workload at its size: 1920x1080 present / 960x540
    # internal, the context flags of the bench (godray alias only), path
    # frames 14..17 with the frame-16 grid shift and its chunk uploads (slot
    # moves, new chunks, grid rewrite) inside the run.
    sc = scenes.config2()
    res = run_parity(sc, frames=4, start_frame=14, flags=A.FLAG_GODRAY_MACRO_ALIAS)
    assert all(r == {} for r in res), res


def test_config2_1080p_resident_frames_15_16_bit_exact():
    # The device-resident workload the bench's `value` times: every chunk of
    # the path uploaded once, the frame-16 shift a grid-window rewrite.
    from parity import run_resident_parity

    res = run_resident_parity(scenes.config2(), frames=[15, 16])
    assert all(r == {} for r in res), res


def test_config5_4k_frames_bit_exact():
    # 32x8x32 chunks, 6-level 512^2 clipmap, 3840x2160 present / 1920x1080
    # internal: two frames with histories feeding back.
    sc = scenes.config5()
    res = run_parity(sc, frames=2, flags=A.FLAG_GODRAY_MACRO_ALIAS | A.FLAG_HIT_RECORDS)
    assert all(r == {} for r in res), res


@pytest.mark.parametrize("limits", [(64, 0), (0, 64), (1, 1)])
def test_probe_overflow_rewalk_bit_exact(limits):
    # Grass probes or slab tasks that do not fit the (capped) record buffers
    # send their pixels to k_primary_resolve's inline re-walk; the frames stay
    # bit-exact and the re-walk counter shows the path ran.
    sc = scenes.config2(present=(320, 180))
    stats = []

    def on_frame(g, o, bad, r, ora):
        stats.append(r.frame_stats())

    res = run_parity(sc, frames=2, setup=lambda r: r.set_record_limits(*limits), on_frame=on_frame)
    assert all(r == {} for r in res), res
    assert all(s["rewalk_pixels"] > 0 for s in stats), stats
    assert all(s["pending_pixels"] >= s["rewalk_pixels"] for s in stats), stats


def test_probe_records_fit_without_rewalk_on_bench_frame():
    # At the default buffer sizes the bench frame stores every probe and slab.
    sc = scenes.config2(present=(640, 360))
    stats = []
    res = run_parity(sc, frames=1, on_frame=lambda g, o, bad, r, ora: stats.append(r.frame_stats()))
    assert res == [{}], res
    s = stats[0]
    assert s["probes"] > 0 and s["slab_tasks"] > 0 and s["pending_pixels"] > 0, s
    assert s["voxel_pixels"] + s["far_pixels"] == 320 * 180, s


def test_no_chunks_draws_sky_like_the_reference():
    # With chunk_count 0 main_primary traces the heightfield but writes sky
    # (ray_main.wgsl:219-231): every depth is FOG_MAX_DIST.
    sc = scenes.config2(present=(160, 90))

    def empty(cam):
        cam.chunk_count = 0

    seen = []
    res = run_parity(sc, frames=2, cam_hook=empty, on_frame=lambda g, o, bad, r, ora: seen.append(g["depth"]))
    assert all(r == {} for r in res), res
    assert all(np.all(d == 120.0) for d in seen)


def test_profile_counts_match_oracle():
    # profile_counts (ray_main.wgsl:32-74) with cam.profile_flags & 1 over
    # temporal frames (hint-window and full traces, grass refinements,
    # heightfield and voxel shading, fresh and reused shadows).
    sc = scenes.features()
    counts = []

    def on(cam):
        cam.profile_flags = 1

    def on_frame(g, o, bad, r, ora):
        counts.append((r.read_primary_profile_counts_blocking().copy(), ora.profile.copy()))

    res = run_parity(sc, frames=3, cam_hook=on, on_frame=on_frame)
    assert all(r == {} for r in res), res
    for gpu, ref in counts:
        assert np.array_equal(gpu, ref), (gpu, ref)
    assert counts[-1][0][A.PROFILE_VOXEL] > 0 and counts[-1][0][A.PROFILE_SHADOW] > 0


def test_profile_counts_config2_wavefront_and_megakernel():
    # The same counts from the wavefront schedule (deferred probes, re-walks
    # under capped records) and the megakernel, on the config-2 world.
    for extra, limits in ((0, (0, 0)), (0, (16, 16)), (A.FLAG_PRIMARY_MEGAKERNEL, (0, 0))):
        sc = scenes.config2(present=(320, 180))
        counts = []

        def on(cam):
            cam.profile_flags = 1

        def on_frame(g, o, bad, r, ora):
            counts.append((r.read_primary_profile_counts_blocking().copy(), ora.profile.copy()))

        res = run_parity(sc, frames=2, cam_hook=on, on_frame=on_frame, extra_flags=extra,
                         setup=lambda r: r.set_record_limits(*limits))
        assert all(r == {} for r in res), res
        for gpu, ref in counts:
            assert np.array_equal(gpu, ref), (extra, limits, gpu, ref)


def test_profile_counts_stay_zero_with_flag_off_and_reset():
    sc = scenes.features()
    seen = []
    res = run_parity(sc, frames=1, on_frame=lambda g, o, bad, r, ora: seen.append(r.read_primary_profile_counts_blocking()))
    assert res == [{}]
    assert not seen[0].any()

    def on(cam):
        cam.profile_flags = 1

    def on_frame(g, o, bad, r, ora):
        assert r.read_primary_profile_counts_blocking().any()
        r.reset_primary_profile_counts()
        assert not r.read_primary_profile_counts_blocking().any()

    run_parity(sc, frames=1, cam_hook=on, on_frame=on_frame)


def test_corrupt_upload_sets_error_word_and_matches_oracle():
    # A chunk upload whose root points its children past the node arena
    # (child_base made on the host), rendered by the checked build
    # (libvxe_checked.so): every device read through it is bounds checked,
    # sets the node bit of the error word and returns a zero record, exactly
    # as the oracle's checked reads do (its oob counter); the images stay
    # finite and equal the oracle's.
    from oracle import oracle as O
    from parity import compare_frame, make_renderer, read_gpu_frame

    sc = scenes.config1()
    drv = FrameDriver(sc)
    ups = drv.initial_uploads()
    w = drv.world
    u = ups[0]
    base = u.node_base
    bad_child = w.node_capacity + 12345
    w.nodes[base]["child_base"] = bad_child  # host mirror the oracle reads
    nodes = u.data.nodes.copy()
    nodes[0]["child_base"] = bad_child
    u.data.nodes = nodes
    r = make_renderer(sc, w, checked=True)
    try:
        r.upload_world(w, ups)
        _, _, clip, cam = drv.step()
        params = drv.empty_clip()
        r.write_clipmap_updates(params, [])
        r.write_camera(cam)
        with pytest.raises(A.VxeError) as ei:
            r.encode_compute()  # synchronous: reports the error word
        assert ei.value.status == 6  # VXE_ERR_BOUNDS
        word = r.read_error_word()
        ora = O.OracleFrameRunner(w, sc.internal, sc.present, None, sc.clip_res)
        ora.render(cam, params)
        assert ora.primary_ctr.oob > 0
        assert word & 1, hex(word)  # node reads out of range
        g = read_gpu_frame(r)
        assert compare_frame(g, ora.outputs()) == {}
        assert np.isfinite(g["output"]).all() and np.isfinite(g["color"]).all()
    finally:
        r.close()


def test_budgeted_streaming_frames_bit_exact():
    # Host streaming through the reference's per-frame upload budget
    # (take_budgeted): at the grid shift the slot rewrites go first and the
    # entering chunks join the grid over the next frames as their uploads are
    # taken; every frame matches the oracle on the same grid.
    sc = scenes.config2(present=(320, 180))
    sc.shift_every = 2
    res = run_parity(sc, frames=4, budgeted=True)
    assert all(r == {} for r in res), res
    # the shift's uploads do not fit one frame's budget
    d = FrameDriver(sc, budgeted=True)
    d.initial_uploads()
    for _ in range(3):
        ups, _, _, _ = d.step()
    assert len(d.queue) > 0 and d.world.uploading


def test_corrupt_upload_clamped_build_stays_in_bounds():
    # The same corrupt chunk on the default build (clamped reads): the frame
    # completes with finite images and, on valid records elsewhere, the
    # unchanged results; nothing is reported.
    from parity import make_renderer

    sc = scenes.config1()
    drv = FrameDriver(sc)
    ups = drv.initial_uploads()
    u = ups[0]
    nodes = u.data.nodes.copy()
    nodes[0]["child_base"] = drv.world.node_capacity + 12345
    u.data.nodes = nodes
    r = make_renderer(sc, drv.world)
    try:
        r.upload_world(drv.world, ups)
        _, _, clip, cam = drv.step()
        r.write_clipmap_updates(drv.empty_clip(), [])
        r.write_camera(cam)
        r.encode_compute()
        assert r.read_error_word() == 0
        out = r.read_image(A.IMG_OUTPUT)
        assert np.isfinite(out).all()
    finally:
        r.close()
