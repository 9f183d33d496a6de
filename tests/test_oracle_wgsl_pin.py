"""Pins the oracle to the reference's own WGSL.

The reference's shaders are translated mechanically from its WGSL into C++ at
build time (oracle/wgsl_to_cpp.py -> oracle/_ref/libref_wgsl.so, over
oracle/wgsl_shim.h) and run beside the oracle, which restates them by hand
(oracle/vxe_oracle.cpp):
  * whole frames of the five compute passes (main_primary, main_local_taa,
    main_godray, main_composite, main_composite_taa) with the images and bind
    groups wired as the reference wires them, histories carried across
    frames: every image;
  * the cold primary voxel trace of every pixel (tile candidate lists in a
    one-lane emulation of the workgroup, the candidate loop);
  * the chunk walk of chunk_trace.wgsl with everything it calls (macro DDA,
    rope walk, leaf descent, anchors, grass probes, blade marches, leaves);
  * the clipmap heightfield march and the helpers that read the world (sun
    shadow march, godray integral, local-light gather, leaf query);
  * 54 pure shading helpers (sky, sun, clouds, fog, phase, tonemap,
    materials, wind, hashes, value noise, godray and light helpers).
With the same elementary functions on both sides (include/vxe/detmath.h),
every output must be identical bit for bit: a difference is a mis-reading in
the restatement.

The translated library is built only where the reference's sources are
present; elsewhere these tests are skipped.
"""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parents[1]
REF_LIB = REPO / "oracle" / "_ref" / "libref_wgsl.so"
ORACLE_LIB = REPO / "oracle" / "liboracle_vxe.so"

# the camera uniform the sky / fog / cloud helpers read: position and
# voxel_params = [voxel size, time_s, wind strength, fog density]
CAM_POS = np.array([12.5, 31.0, -7.25, 0.0], np.float32)
VOXEL_PARAMS = np.array([0.1, 7.3, 2.0, 0.002], np.float32)

FUNCS = ["hash_u32", "hash12", "hash31", "value_noise", "fbm", "hash1", "wind_field", "clamp_len", "grass_wind_xz",
         "grass_blade_params", "sdf_box", "phase_mie", "phase_blended", "sky_bg", "sky_sun", "sky_color",
         "fog_color_from_sky", "fog_inscatter", "fog_optical_depth_with_base", "apply_fog", "cloud_height01",
         "cloud_coverage_at_xz", "cloud_density", "cloud_light_transmittance", "cloud_sun_transmittance_fast",
         "cloud_density_godray", "cloud_sun_transmittance_godray", "tonemap_filmic_hable",
         "tonemap_filmic_white_scale", "bright_extract_hue", "intersect_aabb", "safe_inv", "ray_eps_vec",
         "macro_cell_size", "grass_lod_from_t", "hemi_ambient", "color_for_material", "apply_material_variation",
         "grass_wind_dir_xz", "grass_blade_slivers", "grass_blade_field", "grass_top_albedo", "base_albedo",
         "material_roughness", "material_f0", "material_emission", "approx_pow_0p75", "approx_pow_0p55",
         "exp_neg_fast", "godray_steps_for_tend", "godray_decompress", "godray_compress", "rot_about_axis",
         "sphere_dir_local"]


def load_libs():
    if not REF_LIB.exists():
        pytest.skip("the reference's WGSL was not translated here (no reference sources on this machine)")
    ref = C.CDLL(str(REF_LIB))
    ora = C.CDLL(str(ORACLE_LIB))
    fp = C.POINTER(C.c_float)
    ref.ref_wgsl_eval.argtypes = [C.c_char_p, fp, fp, C.c_uint]
    ref.ref_wgsl_widths.argtypes = [C.c_char_p, C.POINTER(C.c_uint), C.POINTER(C.c_uint)]
    ref.ref_wgsl_set_cam.argtypes = [fp, fp]
    ora.oracle_shading_eval.argtypes = [C.c_char_p, fp, fp, C.c_uint, fp, fp]
    ref.ref_wgsl_set_cam(CAM_POS.ctypes.data_as(fp), VOXEL_PARAMS.ctypes.data_as(fp))
    return ref, ora


def _dirs(rng, n, up_bias=0.0):
    d = rng.normal(size=(n, 3))
    d[:, 1] += up_bias
    return d / np.linalg.norm(d, axis=1, keepdims=True)


def gen_inputs(name: str, n: int, seed: int = 7) -> np.ndarray:
    """Seeded inputs in the ranges the frame passes these functions."""
    rng = np.random.default_rng(seed + sum(map(ord, name)))
    u = lambda lo, hi, k=1: rng.uniform(lo, hi, size=(n, k))
    sun = np.array([0.61237244, 0.5, 0.61237244])
    if name == "hash_u32":
        return rng.integers(0, 2**32, size=(n, 1), dtype=np.uint64).astype(np.uint32).view(np.float32)
    if name in ("hash12", "value_noise", "fbm"):
        x = u(-600, 600, 2)
    elif name in ("hash31", "hash1"):
        x = np.concatenate([np.floor(u(-200, 200, 3)), u(-200, 200, 3)])[:n]
    elif name == "wind_field":
        x = np.hstack([u(-100, 100), u(-2, 20), u(-100, 100), u(0, 120)])
    elif name == "clamp_len":
        x = np.hstack([u(-4, 4, 3), u(0.05, 3)])
    elif name == "grass_wind_xz":
        x = np.hstack([u(-100, 100), u(0, 12), u(-100, 100), u(0, 120), u(0, 3)])
    elif name == "grass_blade_params":
        ids = np.floor(u(-640, 640, 3)).astype(np.float32)
        i = rng.integers(0, 5, size=(n, 1)).astype(np.uint32).view(np.float32)
        return np.ascontiguousarray(np.hstack([ids, i]), np.float32)
    elif name == "sdf_box":
        x = np.hstack([u(-1, 1, 3), u(-0.5, 0.5, 3), u(0.01, 0.4, 3)])
    elif name in ("phase_mie", "phase_blended"):
        x = u(-1, 1)
    elif name in ("sky_bg", "sky_color"):
        x = _dirs(rng, n, 0.3)
    elif name == "sky_sun":  # half of the rays near the sun disc
        d = _dirs(rng, n)
        near = sun + 0.02 * rng.normal(size=(n, 3))
        d[: n // 2] = (near / np.linalg.norm(near, axis=1, keepdims=True))[: n // 2]
        x = d
    elif name in ("fog_color_from_sky", "fog_inscatter"):
        x = np.hstack([_dirs(rng, n), u(0, 2, 3)])
    elif name == "fog_optical_depth_with_base":
        d = _dirs(rng, n)
        d[: n // 8, 1] = rng.uniform(-5e-5, 5e-5, n // 8)  # the near-horizontal branch
        x = np.hstack([u(-0.01, 0.05), u(-50, 50), u(0, 60), u(-50, 50), d, u(0, 120)])
    elif name == "apply_fog":
        x = np.hstack([u(0, 3, 3), u(-50, 50), u(0, 60), u(-50, 50), _dirs(rng, n), u(0, 120), u(0, 2, 3)])
    elif name == "cloud_height01":
        x = u(150, 270)
    elif name == "cloud_coverage_at_xz":
        x = np.hstack([u(-3000, 3000, 2), u(0, 200)])
    elif name in ("cloud_density", "cloud_light_transmittance", "cloud_density_godray"):
        x = np.hstack([u(-3000, 3000), u(160, 260), u(-3000, 3000), u(0, 200)])
    elif name in ("cloud_sun_transmittance_fast", "cloud_sun_transmittance_godray"):
        x = np.hstack([u(-3000, 3000), u(0, 300), u(-3000, 3000), _dirs(rng, n, 2.0)])
    elif name == "tonemap_filmic_hable":
        x = u(0, 20, 3)
    elif name == "tonemap_filmic_white_scale":
        x = np.hstack([u(0, 20, 3), u(1, 12)])
    elif name == "bright_extract_hue":
        x = np.hstack([u(0, 10, 3), u(0, 2)])
    elif name == "intersect_aabb":  # boxes around and away from the origin, some axis-parallel rays
        d = _dirs(rng, n)
        d[: n // 8, 0] = 0.0
        lo = u(-2, 2, 3)
        x = np.hstack([u(-3, 3, 3), d, lo, lo + u(0.1, 2, 3)])
    elif name == "safe_inv":
        x = np.concatenate([u(-2, 2), u(-2e-8, 2e-8)])[:n]
    elif name == "ray_eps_vec":
        d = _dirs(rng, n)
        d[: n // 8, 1] = 0.0
        x = np.hstack([d, u(1e-5, 1e-2)])
    elif name in ("macro_cell_size", "grass_lod_from_t", "godray_steps_for_tend"):
        x = u(0, 130)
    elif name == "hemi_ambient":
        x = np.hstack([_dirs(rng, n), u(0, 2, 3)])
    elif name in ("color_for_material", "material_roughness", "material_f0", "material_emission"):
        return rng.integers(0, 8, size=(n, 1)).astype(np.uint32).view(np.float32)
    elif name == "apply_material_variation":
        m = rng.integers(0, 8, size=(n, 1)).astype(np.uint32).view(np.float32)
        return np.ascontiguousarray(np.hstack([u(0, 1, 3).astype(np.float32), m, u(-60, 60, 3).astype(np.float32)]))
    elif name == "grass_wind_dir_xz":
        x = np.hstack([u(-100, 100), u(0, 12), u(-100, 100), u(0, 120)])
    elif name == "grass_blade_slivers":
        x = np.hstack([u(-60, 60, 3), u(0, 120), u(0.5, 40), u(0, 1)])
    elif name == "grass_blade_field":
        x = np.hstack([u(-60, 60, 3), u(0, 120), u(0, 60)])
    elif name == "grass_top_albedo":
        x = np.hstack([u(0, 1, 3), u(-60, 60, 3), u(0, 60)])
    elif name == "base_albedo":
        m = rng.integers(0, 8, size=(n, 1)).astype(np.uint32).view(np.float32)
        return np.ascontiguousarray(np.hstack([m, u(-60, 60, 3).astype(np.float32), u(0, 120).astype(np.float32)]))
    elif name in ("approx_pow_0p75", "approx_pow_0p55", "exp_neg_fast"):
        x = u(-0.5, 3)
    elif name in ("godray_decompress", "godray_compress"):
        x = u(0, 4, 3)
    elif name == "rot_about_axis":
        x = np.hstack([u(-1, 1, 3), _dirs(rng, n), u(-7, 7)])
    elif name == "sphere_dir_local":
        cnt = rng.integers(1, 17, size=(n, 1))
        i = rng.integers(0, 16, size=(n, 1)) % cnt
        return np.ascontiguousarray(np.hstack([i, cnt]).astype(np.uint32).view(np.float32))
    else:
        raise KeyError(name)
    return np.ascontiguousarray(x, np.float32)


def _eval(lib, fn_name, name, x, out_w, extra=()):
    fp = C.POINTER(C.c_float)
    out = np.full((len(x), out_w), np.nan, np.float32)
    rc = getattr(lib, fn_name)(name.encode(), x.ctypes.data_as(fp), out.ctypes.data_as(fp), len(x), *extra)
    assert rc == 0, f"{fn_name} does not know {name}"
    return out


@pytest.mark.parametrize("name", FUNCS)
def test_oracle_shading_equals_translated_reference_wgsl(name):
    ref, ora = load_libs()
    iw, ow = C.c_uint(), C.c_uint()
    assert ref.ref_wgsl_widths(name.encode(), C.byref(iw), C.byref(ow)) == 0, f"{name} not translated"
    x = gen_inputs(name, 4096)
    assert x.shape[1] == iw.value
    fp = C.POINTER(C.c_float)
    want = _eval(ref, "ref_wgsl_eval", name, x, ow.value)
    got = _eval(ora, "oracle_shading_eval", name, x, ow.value,
                (CAM_POS.ctypes.data_as(fp), VOXEL_PARAMS.ctypes.data_as(fp)))
    diff = np.flatnonzero((want.view(np.uint32) != got.view(np.uint32)).any(axis=1))
    assert diff.size == 0, (f"{name}: {diff.size} of {len(x)} inputs differ, first input {x[diff[0]]}: "
                            f"reference {want[diff[0]]}, oracle {got[diff[0]]}")


def _walk_setup(scene_fn):
    """A world of `scene_fn`, the oracle scene over it, and the translated
    reference library bound to the same host arrays."""
    from oracle import oracle as O
    from vxe.scenes import FrameDriver

    ref, _ = load_libs()
    sc = scene_fn()
    drv = FrameDriver(sc)
    drv.initial_uploads()
    w = drv.world
    _, _, clip, cam = drv.step()
    clip_params = clip[0] if clip is not None else drv.empty_clip()  # config 1 has no clipmap
    runner = O.OracleFrameRunner(w, sc.internal, sc.present, drv.clip.tex if drv.clip is not None else None,
                                 sc.clip_res)
    ora_scene = runner.scene(cam, clip_params)
    runner._driver = drv  # the path's next frames (whole-frame test)
    keep = {}
    _set_ref_camera(ref, w, cam)
    lo = O.lib()
    lo.ora_trace_chunk.argtypes = [C.POINTER(O.OraScene), C.c_void_p, C.c_void_p, C.c_uint32]
    return ref, lo, ora_scene, w, cam, (runner, keep, clip_params)


def _set_ref_camera(ref, w, cam):
    """Binds the world's host arrays and copies `cam` into the translated
    reference's scene bindings."""
    u64 = C.c_uint64
    ref.ref_wgsl_set_scene(C.c_void_p(w.metas.ctypes.data), u64(w.metas.shape[0]), C.c_void_p(w.nodes.ctypes.data),
                           u64(len(w.nodes)), C.c_void_p(w.grid.ctypes.data), u64(len(w.grid)),
                           C.c_void_p(w.macro.ctypes.data), u64(len(w.macro)), C.c_void_p(w.ropes.ctypes.data),
                           u64(len(w.ropes)), C.c_void_p(w.colinfo.ctypes.data), u64(len(w.colinfo)),
                           C.c_void_p(C.addressof(cam)))


def _set_ref_clip(ref, runner, clip_params):
    """The clipmap uniform and texture layers of the oracle runner, for the
    translated reference (no layers: a clipmap with no texture)."""
    if runner.clip_tex is not None:
        runner._ref_tex = np.ascontiguousarray(runner.clip_tex, np.float32)
        t = runner._ref_tex
        ref.ref_wgsl_set_clip(C.c_void_p(C.addressof(clip_params)), t.ctypes.data_as(C.POINTER(C.c_float)),
                              C.c_int32(t.shape[1]), C.c_int32(t.shape[0]))
    else:
        ref.ref_wgsl_set_clip(C.c_void_p(C.addressof(clip_params)), None, C.c_int32(0), C.c_int32(0))


def _walk_rays(w, cam, n, rng):
    """Rays through random chunks: origins in and around the chunk, targets
    inside it, [t0, t1] the chunk box interval from t >= 0."""
    vs = float(cam.voxel_params[0])
    cs = cam.chunk_size * vs
    metas = w.metas.view(np.int32).reshape(-1, 12)
    slots = rng.integers(0, cam.chunk_count, n)
    org = metas[slots, :3].astype(np.float64) * vs
    ro = org + rng.uniform(-0.5, 1.5, (n, 3)) * cs
    rd = org + rng.uniform(0, 1, (n, 3)) * cs - ro
    rd /= np.linalg.norm(rd, axis=1, keepdims=True)
    ro, rd = ro.astype(np.float32), rd.astype(np.float32)
    inv = 1.0 / np.where(np.abs(rd) < 1e-8, 1e-8, rd.astype(np.float64))
    ta, tb = (org - ro) * inv, (org + cs - ro) * inv
    te = np.maximum(np.minimum(ta, tb).max(1), 0.0)
    tx = np.maximum(np.maximum(ta, tb).min(1), te)
    rays = np.zeros((n, 12), np.float32)
    rays[:, 0:3], rays[:, 3:6], rays[:, 6], rays[:, 7] = ro, rd, te, tx
    rays[:, 8] = slots.astype(np.uint32).view(np.float32)
    rays[:, 10] = np.full(n, 0xFFFFFFFF, np.uint32).view(np.float32)
    return rays


def _walk_both(ref, lo, ora_scene, rays):
    fp = C.POINTER(C.c_float)
    want = np.full((len(rays), 16), np.nan, np.float32)
    got = np.full((len(rays), 16), np.nan, np.float32)
    ref.ref_wgsl_trace_chunk(rays.ctypes.data_as(fp), want.ctypes.data_as(fp), len(rays))
    assert lo.ora_trace_chunk(C.byref(ora_scene), rays.ctypes.data, got.ctypes.data, len(rays)) == 0
    return want, got


@pytest.mark.parametrize("scene", ["features", "config1"])
def test_oracle_chunk_walk_equals_translated_reference_wgsl(scene):
    """The chunk walk (chunk_trace.wgsl trace_chunk_interval_stream_macro:
    macro DDA, rope walk, leaf descent, anchors, grass column probes and blade
    marches) of the oracle against the reference's own WGSL translated to
    C++, on random rays through every kind of chunk: hit, material, t,
    normal, chunk root, anchor, bit for bit."""
    from vxe import scenes

    fn = {"features": lambda: scenes.features(present=(64, 40)), "config1": scenes.config1}[scene]
    ref, lo, ora_scene, w, cam, _keep = _walk_setup(fn)
    rng = np.random.default_rng(11)
    rays = _walk_rays(w, cam, 20000, rng)
    want, got = _walk_both(ref, lo, ora_scene, rays)
    hits = want[:, 0].view(np.uint32) != 0
    assert 0.2 < hits.mean() < 0.98
    mats = set(want[hits, 1].view(np.uint32).tolist())
    assert {1, 2, 3} <= mats  # grass, dirt and stone hits at least
    diff = np.flatnonzero((want.view(np.uint32) != got.view(np.uint32)).any(axis=1))
    assert diff.size == 0, f"{diff.size} of {len(rays)} walks differ, first ray {rays[diff[0], :8]}"
    # the anchor path: the same rays again from half way along, seeded with
    # the anchor the first walk returned
    valid = want[:, 12].view(np.uint32) != 0
    assert valid.mean() > 0.2
    rays2 = rays.copy()
    rays2[:, 6] = 0.5 * (rays[:, 6] + rays[:, 7])
    rays2[:, 9] = valid.astype(np.uint32).view(np.float32)
    rays2[:, 10] = want[:, 13]
    want2, got2 = _walk_both(ref, lo, ora_scene, rays2)
    diff = np.flatnonzero((want2.view(np.uint32) != got2.view(np.uint32)).any(axis=1))
    assert diff.size == 0, f"{diff.size} anchored walks differ, first ray {rays2[diff[0], :11]}"


def test_oracle_scene_helpers_equal_translated_reference_wgsl():
    """The helpers that read the world, on the features world (caves, trees,
    light voxels, grass): the sun shadow march (shadows.wgsl
    sun_transmittance_geom_only), the godray in-scatter integral (godrays.wgsl
    godray_integrate_1, with its cloud and shadow samples), the local-light
    gather (light.wgsl gather_voxel_lights, its DDA to light voxels) and the
    leaf query (svo_query.wgsl query_leaf_world), bit for bit."""
    from vxe import scenes

    ref, lo, ora_scene, w, cam, _keep = _walk_setup(lambda: scenes.features(present=(64, 40)))
    lo.ora_scene_eval.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p, C.c_void_p, C.c_uint32]
    rng = np.random.default_rng(5)
    rays = _walk_rays(w, cam, 20000, rng)
    walk, _ = _walk_both(ref, lo, ora_scene, rays)
    hit = walk[:, 0].view(np.uint32) != 0
    hp = (rays[hit, :3] + rays[hit, 3:6] * walk[hit, 2:3]).astype(np.float32)
    nrm, rb = walk[hit, 3:6], walk[hit, 6:9]
    mats = walk[hit, 1].view(np.uint32)
    lights = hp[mats == 6]
    assert len(lights) > 0
    # half of the gather points are the surface points nearest a light voxel
    d = np.min(np.linalg.norm(hp[:, None, :] - lights[None, :64, :], axis=2), axis=1)
    near = np.argsort(d)[:3000]
    pick = np.concatenate([near, rng.choice(len(hp), 3000, replace=False)])
    vs = float(cam.voxel_params[0])
    cs = cam.chunk_size * vs
    metas = w.metas.view(np.int32).reshape(-1, 12)[: cam.chunk_count]
    lo3, hi3 = metas[:, :3].min(0) * vs, metas[:, :3].max(0) * vs + cs
    sun = np.array([0.61237244, 0.5, 0.61237244], np.float32)
    n = 6000
    cases = {
        "sun_transmittance_geom_only": np.hstack([np.vstack([hp[pick[:3000]] + nrm[pick[:3000]] * 0.01,
                                                              rng.uniform(lo3, hi3, (3000, 3))]), np.tile(sun, (n, 1))]),
        "godray_integrate_1": np.hstack([np.tile(np.array(cam.cam_pos[:3]), (n, 1)), _dirs(rng, n, 0.2),
                                         rng.uniform(0, 100, (n, 1)), rng.uniform(0, 1, (n, 2))]),
        "gather_voxel_lights": np.hstack([hp[pick], nrm[pick], rb[pick], np.zeros((n, 3))]),
        "query_leaf_world": rng.uniform(lo3, hi3, (n, 3)),
    }
    fp = C.POINTER(C.c_float)
    lit = 0
    for name, x in cases.items():
        x = np.ascontiguousarray(x, np.float32)
        iw, ow = C.c_uint(), C.c_uint()
        assert ref.ref_wgsl_widths(name.encode(), C.byref(iw), C.byref(ow)) == 0, name
        assert x.shape[1] == iw.value
        want = np.full((n, ow.value), np.nan, np.float32)
        got = np.full((n, ow.value), np.nan, np.float32)
        ref.ref_wgsl_eval(name.encode(), x.ctypes.data_as(fp), want.ctypes.data_as(fp), n)
        assert lo.ora_scene_eval(C.addressof(ora_scene), name.encode(), x.ctypes.data, got.ctypes.data, n) == 0
        diff = np.flatnonzero((want.view(np.uint32) != got.view(np.uint32)).any(axis=1))
        assert diff.size == 0, f"{name}: {diff.size} of {n} differ, first input {x[diff[0]]}"
        assert len(np.unique(want.view(np.uint32))) > 10, name
        if name == "gather_voxel_lights":
            lit = int((want != 0).any(axis=1).sum())
    assert lit > 50  # the gather found light voxels for enough of its points


def test_oracle_clipmap_march_equals_translated_reference_wgsl():
    """The clipmap heightfield (clipmap.wgsl: clip_trace_heightfield, its
    level samples, the toroidal texel offsets) on config 2's 5-level 256^2
    clipmap, bit for bit."""
    from vxe import scenes

    ref, lo, ora_scene, w, cam, keep = _walk_setup(lambda: scenes.config2(present=(64, 36)))
    runner, _, clip_params = keep
    tex = np.ascontiguousarray(runner.clip_tex, np.float32)
    ref.ref_wgsl_set_clip(C.c_void_p(C.addressof(clip_params)), tex.ctypes.data_as(C.POINTER(C.c_float)),
                          C.c_int32(tex.shape[1]), C.c_int32(tex.shape[0]))
    lo.ora_scene_eval.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p, C.c_void_p, C.c_uint32]
    rng = np.random.default_rng(3)
    n = 6000
    cp = np.array(cam.cam_pos[:3], np.float32)
    march = np.hstack([np.tile(cp, (n, 1)) + rng.uniform(-20, 20, (n, 3)) * [1, 0.2, 1], _dirs(rng, n, -0.4),
                       np.zeros((n, 1)), rng.uniform(20, 400, (n, 1))])
    levels = rng.integers(0, clip_params.levels, n).astype(np.uint32).view(np.float32)
    samples = np.hstack([cp[[0, 2]] + rng.uniform(-600, 600, (n, 2)), levels[:, None]])
    fp = C.POINTER(C.c_float)
    for name, x in (("clip_trace_heightfield", march), ("clip_height_at_level", samples),
                    ("clip_height_at_level_nearest", samples)):
        x = np.ascontiguousarray(x, np.float32)
        if name != "clip_trace_heightfield":
            x[:, 2] = levels
        iw, ow = C.c_uint(), C.c_uint()
        assert ref.ref_wgsl_widths(name.encode(), C.byref(iw), C.byref(ow)) == 0, name
        want = np.full((n, ow.value), np.nan, np.float32)
        got = np.full((n, ow.value), np.nan, np.float32)
        ref.ref_wgsl_eval(name.encode(), x.ctypes.data_as(fp), want.ctypes.data_as(fp), n)
        assert lo.ora_scene_eval(C.addressof(ora_scene), name.encode(), x.ctypes.data, got.ctypes.data, n) == 0
        diff = np.flatnonzero((want.view(np.uint32) != got.view(np.uint32)).any(axis=1))
        assert diff.size == 0, f"{name}: {diff.size} of {n} differ, first input {x[diff[0]]}"
        assert len(np.unique(want.view(np.uint32))) > 10, name  # nearest samples are whole voxel heights


@pytest.mark.parametrize("scene", ["features", "config2"])
def test_oracle_primary_trace_equals_translated_reference_wgsl(scene):
    """The cold primary voxel trace of every pixel of a frame: each 8x8
    tile's candidate list as main_primary's lane 0 builds it (chunk grid DDA
    of two tile rays, atomic appends, the sort by entry t) in a one-lane
    emulation of the workgroup, then each pixel's candidate loop
    (chunk_trace.wgsl trace_scene_voxels_candidates) with its chunk walks.
    In-grid flag, hit, material, t, normal, chunk root, exit t and anchor,
    bit for bit, and the same candidate count per tile."""
    from vxe import scenes

    fn = {"features": lambda: scenes.features(present=(128, 80)),
          "config2": lambda: scenes.config2(present=(640, 360))}[scene]
    ref, lo, ora_scene, w, cam, _keep = _walk_setup(fn)
    lo.ora_primary_tile.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p]
    ref.ref_wgsl_primary_tile.argtypes = [C.c_uint32, C.c_uint32, C.c_void_p]
    iw, ih = cam.render_present_px[0], cam.render_present_px[1]
    want = np.full((64, 16), np.nan, np.float32)
    got = np.full((64, 16), np.nan, np.float32)
    pixels = hits = 0
    for ty in range((ih + 7) // 8):
        for tx in range((iw + 7) // 8):
            cw = ref.ref_wgsl_primary_tile(tx, ty, want.ctypes.data)
            cg = lo.ora_primary_tile(C.addressof(ora_scene), tx, ty, got.ctypes.data)
            assert cw == cg, f"tile ({tx}, {ty}): {cw} candidates in the reference, {cg} in the oracle"
            bad = np.flatnonzero((want.view(np.uint32) != got.view(np.uint32)).any(axis=1))
            assert bad.size == 0, (f"tile ({tx}, {ty}) pixel {bad[0]}: reference {want[bad[0]]}, "
                                   f"oracle {got[bad[0]]}")
            pixels += 64
            hits += int((want[:, 1].view(np.uint32) != 0).sum())
    assert hits > 0.3 * pixels


def _frame_io(iw, ih, pw, ph):
    z = lambda *s: np.zeros(s, np.float32)
    stride = ((iw * 4 + 255) & ~255) // 4
    return [z(ih, iw, 4), z(ih, iw), z(ih, iw, 4), z(ih, iw, 4), z(ih, iw, 4), z(ih, iw), z(ih, stride),
            z(ih, iw, 4), z(ih, iw, 4), z(ih, iw, 4), z(ih, iw, 4), z(ph, pw, 4), z(ph, pw, 4), z(ph, pw, 4),
            z(ph, pw, 4)]


@pytest.mark.parametrize("scene,frames", [("features", 3), ("config1", 1), ("config2", 18), ("config5", 1)])
def test_oracle_frames_equal_translated_reference_wgsl(scene, frames):
    """Whole frames of the reference's own compute passes -- main_primary,
    main_local_taa, main_godray, main_composite, main_composite_taa, run per
    pixel in the order Renderer::encode_compute runs them, with the
    images and the godray pass's scene bind group wired as the reference
    wires them -- against the oracle's frames: every image bit for bit (color,
    depth, local, primary-hit history, shadow history, local TAA history,
    godray, pre-TAA composite, output, output history).  After each frame the
    histories feed the next one, as the reference's ping-pong and its shadow
    buffer -> texture copy do."""
    from vxe import scenes

    fn = {"features": lambda: scenes.features(present=(128, 80)), "config1": scenes.config1,
          "config2": lambda: scenes.config2(present=(320, 180)),
          "config5": lambda: scenes.config5(present=(320, 180))}[scene]
    ref, lo, ora_scene, w, cam, keep = _walk_setup(fn)
    runner, _, clip_params = keep
    drv_cam, drv_clip = cam, clip_params
    iw, ih, pw, ph = (cam.render_present_px[i] for i in range(4))
    io = _frame_io(iw, ih, pw, ph)
    ref.ref_wgsl_frame.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32]
    names = {0: "color", 1: "depth", 2: "local", 4: "primary_hist", 8: "local_hist", 10: "godray",
             11: "output_pre_taa", 13: "output", 14: "output_hist"}
    for f in range(frames):
        if f > 0:  # the next path frame on both sides
            _, _, clip, drv_cam = runner._driver.step()
            drv_clip = clip[0] if clip is not None else runner._driver.empty_clip()
            ora_scene = runner.scene(drv_cam, drv_clip)
            _set_ref_camera(ref, w, drv_cam)
        _set_ref_clip(ref, runner, drv_clip)
        ptrs = (C.c_void_p * 15)(*[a.ctypes.data for a in io])
        assert ref.ref_wgsl_frame(iw, ih, pw, ph, ptrs, 1 + f) == 0  # 1, 2, 3 host threads: the same images
        runner.render(drv_cam, drv_clip)
        o = runner.outputs()
        for k, nm in names.items():
            got = np.ascontiguousarray(o[nm]).reshape(-1).view(np.uint32)
            want = io[k].reshape(-1).view(np.uint32)
            bad = np.flatnonzero(want != got)
            assert bad.size == 0, f"frame {f} {nm}: {bad.size} of {want.size} values differ, first at {bad[0]}"
        bad = np.flatnonzero(io[6][:, :iw].reshape(-1).view(np.uint32) != o["shadow"].reshape(-1).view(np.uint32))
        assert bad.size == 0, f"frame {f} shadow: {bad.size} values differ"
        assert len(np.unique(io[13].view(np.uint32))) > 1000
        # histories for the next frame (the reference's ping-pong)
        io[3][:] = io[4]
        io[5][:] = io[6][:, :iw]
        io[7][:] = io[8]
        io[9][:] = io[10]
        io[12][:] = io[14]


@pytest.mark.parametrize("scene", ["features", "config2"])
def test_oracle_work_counters_equal_translated_reference_wgsl(scene):
    """The work counters the reference's main_primary keeps while
    cam.profile_flags & 1 (profile_counts: VOXEL, GRASS, HDR, FOG, SHADOW,
    ray_main.wgsl:32-74), over two frames on one host thread, against the
    oracle's counters of the same frames."""
    from vxe import scenes

    fn = {"features": lambda: scenes.features(present=(128, 80)),
          "config2": lambda: scenes.config2(present=(320, 180))}[scene]
    ref, lo, ora_scene, w, cam, keep = _walk_setup(fn)
    runner, _, clip_params = keep
    iw, ih, pw, ph = (cam.render_present_px[i] for i in range(4))
    io = _frame_io(iw, ih, pw, ph)
    ref.ref_wgsl_frame.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32]
    ref.ref_wgsl_take_profile.argtypes = [C.c_void_p]
    want = np.zeros(5, np.uint32)
    ref.ref_wgsl_take_profile(want.ctypes.data)  # cleared
    runner.profile[:] = 0
    drv_cam, drv_clip = cam, clip_params
    for f in range(2):
        if f > 0:
            _, _, clip, drv_cam = runner._driver.step()
            drv_clip = clip[0] if clip is not None else runner._driver.empty_clip()
        drv_cam.profile_flags = 1
        _set_ref_camera(ref, w, drv_cam)
        _set_ref_clip(ref, runner, drv_clip)
        ptrs = (C.c_void_p * 15)(*[a.ctypes.data for a in io])
        assert ref.ref_wgsl_frame(iw, ih, pw, ph, ptrs, 1) == 0
        runner.render(drv_cam, drv_clip)
        io[3][:] = io[4]
        io[5][:] = io[6][:, :iw]
        io[7][:] = io[8]
        io[9][:] = io[10]
        io[12][:] = io[14]
    ref.ref_wgsl_take_profile(want.ctypes.data)
    assert want[0] > 0 and want[4] > 0
    assert want.tolist() == runner.profile.tolist()
