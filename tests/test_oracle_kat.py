"""Known-answer checks of the oracle (CPU only).

The reference ships no tests or golden vectors.  Its shaders themselves are
run beside the oracle, translated to C++ (tests/test_oracle_wgsl_pin.py); the
checks here pin the oracle independently of them:
  * an independent FP64 Amanatides-Woo voxel DDA over the dense material grid
    (first solid voxel identical, t within 1e-5 relative),
  * determinism across thread counts,
  * a committed golden fixture (tests/golden/) that freezes the oracle's
    config-1 frame against accidental drift.
"""
import json
from pathlib import Path

import numpy as np

from oracle import oracle as O
from vxe import scenes
from vxe.scenes import FrameDriver
from vxe.world import chunk_materials

GOLDEN = Path(__file__).resolve().parent / "golden"


def fp64_first_voxel(mat, o, d, tmax):
    """Exact-ish first solid voxel of a 64^3 chunk at the origin (voxel 0.1 m)."""
    vs = 0.1
    o = np.asarray(o, dtype=np.float64) / vs
    d = np.asarray(d, dtype=np.float64)
    # clip to the chunk box [0, 64)^3
    t0, t1 = 0.0, tmax / vs
    for a in range(3):
        if abs(d[a]) < 1e-12:
            if o[a] < 0 or o[a] >= 64:
                return None
            continue
        ta, tb = (0 - o[a]) / d[a], (64 - o[a]) / d[a]
        t0, t1 = max(t0, min(ta, tb)), min(t1, max(ta, tb))
    if t0 > t1:
        return None
    p = o + d * (t0 + 1e-9)
    cell = np.clip(np.floor(p).astype(int), 0, 63)
    step = np.where(d > 0, 1, -1)
    nxt = cell + (d > 0)
    with np.errstate(divide="ignore", invalid="ignore"):
        tmaxv = np.where(np.abs(d) > 1e-12, (nxt - o) / d, np.inf)
        tdel = np.where(np.abs(d) > 1e-12, np.abs(1.0 / d), np.inf)
    t = t0
    while True:
        if mat[cell[1], cell[2], cell[0]] != 0:
            return t * vs, tuple(int(c) for c in cell)
        a = int(np.argmin(tmaxv))
        t = tmaxv[a]
        if t > t1:
            return None
        cell[a] += step[a]
        if cell[a] < 0 or cell[a] > 63:
            return None
        tmaxv[a] += tdel[a]


def test_query_traversal_matches_fp64_voxel_dda():
    sc = scenes.config1()
    drv = FrameDriver(sc)
    drv.initial_uploads()
    _, _, _, cam = drv.step()
    mat = chunk_materials(sc.spec, 0, 0, 0)
    rng = np.random.default_rng(11)
    n = 3000
    targets = rng.uniform(0.2, 6.2, size=(n, 3))
    origins = targets + rng.normal(size=(n, 3)) * 6.0
    d = targets - origins
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    o32, d32 = origins.astype(np.float32), d.astype(np.float32)
    hits, _ = O.trace_rays(drv.world, cam, o32, d32, 120.0, threads=4)
    disagree = []
    rel = []
    inside = 0
    for i in range(n):
        ref = fp64_first_voxel(mat, o32[i].astype(np.float64), d32[i].astype(np.float64), 120.0)
        h = hits[i]
        if ref is None:
            if h["face"] != 255:
                disagree.append(i)
            continue
        t, vox = ref
        if h["face"] == 255 or tuple(h["voxel"]) != vox:
            disagree.append(i)
        elif t == 0.0:
            # the origin lies inside a solid voxel: that voxel, at t = 0 up to
            # the traversal's entry nudge (eps_step = 1e-4 * voxel = 1e-5 m)
            inside += 1
            assert 0.0 <= float(h["t"]) <= 1.5e-5, (i, float(h["t"]))
        else:
            rel.append((abs(float(h["t"]) - t), t))
    # every ray: the same first solid voxel (or the same miss)
    assert not disagree, (len(disagree), disagree[:10])
    assert inside > 0 and len(rel) > n // 2
    # t tolerance: 1e-5 relative, floored at 1.5 x eps_step (1e-4 * voxel = 1e-5 m),
    # the reference's own nudge past every cell boundary (chunk_trace.wgsl:608,686).
    err = np.array([e for e, _ in rel])
    tt = np.array([t for _, t in rel])
    assert (err <= np.maximum(1e-5 * tt, 1.5e-5)).all(), err.max()
    assert np.median(err / tt) < 1e-6


def _render(threads):
    sc = scenes.features(present=(64, 40))
    drv = FrameDriver(sc)
    drv.initial_uploads()
    r = O.OracleFrameRunner(drv.world, sc.internal, sc.present, drv.clip.tex, sc.clip_res)
    for _ in range(2):
        _, _, clip, cam = drv.step()
        r.render(cam, clip[0], threads=threads)
    return {k: np.array(v, copy=True) for k, v in r.outputs().items()}


def test_oracle_is_deterministic_across_thread_counts():
    a, b = _render(1), _render(7)
    for k in a:
        if a[k].dtype.names:
            assert a[k].tobytes() == b[k].tobytes(), k
        else:
            assert np.array_equal(a[k], b[k], equal_nan=True), k


def test_golden_config1_frame():
    from golden.make_golden import config1_digest

    want = json.loads((GOLDEN / "config1_frame.json").read_text())
    got = config1_digest()
    assert got["hits_sha256"] == want["hits_sha256"]
    assert got["depth_sha256"] == want["depth_sha256"]
    assert got["output_sha256"] == want["output_sha256"]
    assert got["hit_counts"] == want["hit_counts"]
    assert np.allclose(got["samples"], want["samples"], rtol=0, atol=0)


def test_tile_lists_are_short_and_unique():
    sc = scenes.config2(present=(320, 180))
    drv = FrameDriver(sc)
    drv.initial_uploads()
    _, _, clip, cam = drv.step()
    counts, slots = O.tile_lists(drv.world, cam, clip[0], sc.internal)
    assert counts.max() <= 24 and counts.max() > 1
    for c, s in zip(counts, slots):
        live = s[:c]
        assert len(set(live.tolist())) == c
        assert (live < drv.world.chunk_count).all()
        assert (s[c:] == 0xFFFFFFFF).all()
