"""The chunk builder on the device against the host builder (the C++ port of
svo/builder.rs:846-986 and builder_svo.rs / builder_ropes.rs): nodes, ropes,
macro words, colinfo words and counts byte for byte."""
import numpy as np
import pytest

from vxe import _abi as A
from vxe import scenes
from vxe.renderer import Renderer
from vxe.world import World, WorldSpec, build_chunk

pytestmark = pytest.mark.gpu

CARVE = WorldSpec(seed=12345, height_min=8, height_max=48, dirt_depth=3, carve_mod=50)
FEATURES = WorldSpec(seed=99, height_min=10, height_max=40, dirt_depth=3, cave_threshold=0.55, features=3)
PLAIN = WorldSpec(seed=7, height_min=20, height_max=100, dirt_depth=4, height_scale_vox=96.0, features=1)

# surface chunks, negative coordinates, an all-air chunk, all-solid chunks
# below the surface (the root collapses to one stone leaf without caves or
# carving), the surface crossing chunk boundaries in y
KEYS = [(0, 0, 0), (1, 0, -1), (-2, 0, 3), (5, 0, 5), (0, 3, 0), (0, -1, 0), (-3, -2, -4), (2, 1, 2), (7, 0, -6)]


def _renderer():
    return Renderer(64, 36, 1.0, node_capacity=1 << 16, chunk_capacity=16, grid_capacity=16, clip_levels=1,
                    clip_res=16)


def _compare(spec, keys, out):
    counts = out["counts"].cpu().numpy().view(np.uint32)
    macro = out["macro"].cpu().numpy().view(np.uint32)
    colinfo = out["colinfo"].cpu().numpy().view(np.uint32)
    for j, key in enumerate(keys):
        ref = build_chunk(spec, *key)
        n = len(ref.nodes)
        assert counts[j, 0] == n, (key, counts[j, 0], n)
        assert counts[j, 1] == ref.solid_voxels, key
        assert np.array_equal(macro[j], ref.macro), key
        assert np.array_equal(colinfo[j], ref.colinfo), key
        nodes = out["nodes"][j, :n].cpu().numpy().view(np.uint32).reshape(-1)
        ropes = out["ropes"][j, :n].cpu().numpy().view(np.uint32).reshape(-1)
        assert np.array_equal(nodes, ref.nodes.view(np.uint32).reshape(-1)), key
        assert np.array_equal(ropes, ref.ropes.view(np.uint32).reshape(-1)), key


@pytest.mark.parametrize("spec", [CARVE, FEATURES, PLAIN], ids=["carve", "caves_trees_lights", "plain_trees"])
def test_device_build_equals_host_builder(spec):
    import torch

    r = _renderer()
    try:
        coords = torch.tensor(KEYS, dtype=torch.int32, device="cuda:0")
        out = r.build_chunks(spec.params(), coords)
        _compare(spec, KEYS, out)
        counts = out["counts"].cpu().numpy()
        assert counts[:, 0].max() > 1000 and counts[:, 0].min() == 1  # full trees and collapsed roots
        t = r.build_timings()
        assert t["columns"] > 0 and t["svo"] > 0
    finally:
        r.close()


def test_device_build_config2_grid_and_world_prebuild():
    """Every chunk of the 16x4x16 config-2 grid in batches, through
    World.prebuild_device, against World.prebuild on the host builder."""
    import torch

    sc = scenes.config2(present=(64, 36))
    keys = [(x, y, z) for z in range(16) for y in range(4) for x in range(16)]
    r = _renderer()
    try:
        wd = World(sc.spec, sc.grid_origin, sc.grid_dims, sc.node_capacity)
        wd.prebuild_device(r, keys, batch=128)
        rng = np.random.default_rng(3)
        pick = [keys[i] for i in rng.choice(len(keys), 48, replace=False)]
        for key in pick:
            ref = build_chunk(sc.spec, *key)
            got = wd.cache[key]
            assert got.solid_voxels == ref.solid_voxels, key
            assert np.array_equal(got.nodes.view(np.uint32), ref.nodes.view(np.uint32)), key
            assert np.array_equal(got.ropes.view(np.uint32), ref.ropes.view(np.uint32)), key
            assert np.array_equal(got.macro, ref.macro) and np.array_equal(got.colinfo, ref.colinfo), key
        # the largest batch in one call
        coords = torch.tensor(keys[:A.BUILD_BATCH_MAX] if len(keys) >= A.BUILD_BATCH_MAX else keys,
                              dtype=torch.int32, device="cuda:0")
        out = r.build_chunks(sc.spec.params(), coords, node_cap=70000)
        counts = out["counts"].cpu().numpy().view(np.uint32)
        for j in rng.choice(len(coords), 8, replace=False):
            key = tuple(int(v) for v in coords[j].tolist())
            if counts[j, 0] <= 70000:
                _compare(sc.spec, [key], {k: v[j:j + 1] for k, v in out.items()})
    finally:
        r.close()


def test_node_cap_overflow_still_reports_counts():
    import torch

    r = _renderer()
    try:
        keys = [(0, 0, 0), (0, -1, 0)]
        coords = torch.tensor(keys, dtype=torch.int32, device="cuda:0")
        out = r.build_chunks(CARVE.params(), coords, node_cap=64)
        counts = out["counts"].cpu().numpy().view(np.uint32)
        ref0 = build_chunk(CARVE, *keys[0])
        assert counts[0, 0] == len(ref0.nodes) > 64
        assert counts[0, 1] == ref0.solid_voxels
        assert np.array_equal(out["colinfo"][0].cpu().numpy().view(np.uint32), ref0.colinfo)
        # a count-only call (cap 0) also gives the counts
        z = r.build_chunks(CARVE.params(), coords, node_cap=0)
        assert np.array_equal(z["counts"].cpu().numpy(), out["counts"].cpu().numpy())
    finally:
        r.close()


def test_resident_build_renders_like_host_upload():
    """World.populate_device (counting build, then the resident build into the
    context's arenas) against World.populate + upload of the host-built chunks:
    the same slots and arena ranges, and the same frame bit for bit."""
    from vxe.scenes import FrameDriver

    sc = scenes.config2(present=(640, 360))
    drv = FrameDriver(sc)
    ups = drv.initial_uploads()
    _, _, clip, cam = drv.step()
    w = drv.world
    kw = dict(node_capacity=w.node_capacity, chunk_capacity=w.chunk_capacity, grid_capacity=w.grid_capacity,
              clip_levels=sc.clip_levels, clip_res=sc.clip_res)
    ra = Renderer(sc.present[0], sc.present[1], sc.render_scale, **kw)
    rb = Renderer(sc.present[0], sc.present[1], sc.render_scale, **kw)
    try:
        ra.upload_world(w, ups)
        wb = World(sc.spec, sc.grid_origin, sc.grid_dims, sc.node_capacity)
        wb.populate_device(rb, batch=300)  # several resident builds
        assert wb.key_to_slot == w.key_to_slot and wb.alloc == w.alloc
        assert np.array_equal(wb.grid, w.grid)
        images = []
        for r in (ra, rb):
            r.write_clipmap_updates(*clip)
            r.write_camera(cam)
            r.encode_compute()
            images.append([r.read_image(i).tobytes() for i in (A.IMG_OUTPUT, A.IMG_COLOR, A.IMG_DEPTH)])
            assert r.read_error_word() == 0
        assert images[0] == images[1]
    finally:
        ra.close()
        rb.close()


def test_resident_build_reports_a_short_reservation():
    r = _renderer()
    try:
        wp = CARVE.params()
        key = (0, 0, 0)
        n = len(build_chunk(CARVE, *key).nodes)
        with pytest.raises(A.VxeError):  # two places on one slot
            r.build_resident(wp, [(key, 0, 0, n), ((1, 0, 0), 0, n, n)])
        r.build_resident(wp, [(key, 1, 0, n - 1)])
        assert r.read_error_word() & A.ERR_WORD_BUILD
        r.build_resident(wp, [(key, 1, 0, n)])
        assert r.read_error_word() == 0
    finally:
        r.close()


def test_device_build_random_worlds():
    """Random world parameters (cave thresholds, carving, heights, lattice
    spacing, features) and random chunks, byte for byte against the host
    builder; the cave thresholds exercise the exact threshold compare."""
    import torch

    rng = np.random.default_rng(2024)
    r = _renderer()
    try:
        for w in range(6):
            lo = int(rng.integers(-40, 60))
            spec = WorldSpec(seed=int(rng.integers(0, 2 ** 32 - 1)), height_min=lo,
                             height_max=lo + int(rng.integers(0, 120)), dirt_depth=int(rng.integers(0, 8)),
                             carve_mod=int(rng.choice([0, 0, 7, 50, 331])),
                             cave_threshold=float(rng.choice([2.0, rng.uniform(0.3, 0.95)])),
                             height_scale_vox=float(rng.choice([16.0, 48.0, 64.0, 100.0])),
                             features=int(rng.integers(0, 4)))
            keys = [(int(rng.integers(-30, 30)), int(rng.integers(-2, 3)), int(rng.integers(-30, 30)))
                    for _ in range(5)]
            coords = torch.tensor(keys, dtype=torch.int32, device="cuda:0")
            _compare(spec, keys, r.build_chunks(spec.params(), coords))
    finally:
        r.close()


def test_device_streaming_renders_like_host_streaming():
    """A world kept on the device (resident builds, device slot moves at each
    grid shift) against the host path (host builds, uploads of the moved and
    new chunks): the same slots and arena ranges after every shift and the
    same frames bit for bit, across three shifts (one back to the origin)."""
    sc = scenes.config2(present=(480, 270))
    sc.shift_every = 2
    kw = dict(node_capacity=sc.node_capacity, chunk_capacity=int(np.prod(sc.grid_dims)),
              grid_capacity=int(np.prod(sc.grid_dims)), clip_levels=sc.clip_levels, clip_res=sc.clip_res)
    from vxe.scenes import FrameDriver

    rh = Renderer(sc.present[0], sc.present[1], sc.render_scale, **kw)
    rd = Renderer(sc.present[0], sc.present[1], sc.render_scale, **kw)
    try:
        dh, dd = FrameDriver(sc), FrameDriver(sc, device_renderer=rd)
        rh.upload_world(dh.world, dh.initial_uploads())
        assert dd.initial_uploads() == []
        for f in range(6):
            if f == 5:  # back to the first origin on both sides
                rh.apply_chunk_uploads(dh.world.shift(-2, 0, 0))
                rh.write_chunk_grid(dh.world.grid)
                dd.world.shift_device(rd, -2, 0, 0)
            uh, gh, clip, cam = dh.step()
            ud, gd, clip_d, cam_d = dd.step()
            assert ud == [] and not gd
            if uh:
                rh.apply_chunk_uploads(uh)
            if gh:
                rh.write_chunk_grid(dh.world.grid)
            assert dd.world.key_to_slot == dh.world.key_to_slot and dd.world.alloc == dh.world.alloc
            assert np.array_equal(dd.world.grid, dh.world.grid)
            imgs = []
            for r, c, cm in ((rh, clip, cam), (rd, clip_d, cam_d)):
                r.write_clipmap_updates(*c)
                r.write_camera(cm)
                r.encode_compute()
                imgs.append([r.read_image(i).tobytes() for i in (A.IMG_OUTPUT, A.IMG_DEPTH)])
            assert imgs[0] == imgs[1], f
        assert rh.read_error_word() == 0 and rd.read_error_word() == 0
    finally:
        rh.close()
        rd.close()


def test_builder_and_slot_move_argument_checks():
    """Oversized batches, caps and out-of-range slots are refused before any
    launch, with the context still usable."""
    import torch

    r = _renderer()
    try:
        wp = CARVE.params()
        too_many = torch.zeros((A.BUILD_BATCH_MAX + 1, 3), dtype=torch.int32, device="cuda:0")
        with pytest.raises(A.VxeError):
            r.build_chunks(wp, too_many, node_cap=0)
        with pytest.raises(A.VxeError):
            r.build_chunks(wp, too_many[:1], node_cap=A.BUILD_NODE_CAP_MAX + 1)
        with pytest.raises(A.VxeError):  # slot outside the context's 16
            r.build_resident(wp, [((0, 0, 0), 16, 0, 10)])
        with pytest.raises(A.VxeError):  # nodes outside the arena
            r.build_resident(wp, [((0, 0, 0), 0, (1 << 16) - 5, 10)])
        with pytest.raises(A.VxeError):  # two places on the same arena nodes
            r.build_resident(wp, [((0, 0, 0), 0, 0, 10), ((1, 0, 0), 1, 5, 10)])
        with pytest.raises(A.VxeError):
            r.move_slots([(0, 16)])
        # still usable: a real build and a move
        key = (0, 0, 0)
        n = len(build_chunk(CARVE, *key).nodes)
        r.build_resident(wp, [(key, 2, 0, n)])
        r.move_slots([(2, 3)])
        assert r.read_error_word() == 0
    finally:
        r.close()
