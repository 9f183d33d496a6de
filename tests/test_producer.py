"""Properties of the C++ producer (port of svo/builder*.rs) -- the reference has no tests,
so the builder is pinned by its structural invariants."""
import numpy as np
import pytest

from vxe import _abi as A
from vxe.world import WorldSpec, build_chunk, chunk_materials, ground_height

SPEC = WorldSpec(seed=12345, height_min=8, height_max=48, dirt_depth=3, carve_mod=50)
CAVES = WorldSpec(seed=99, height_min=10, height_max=40, dirt_depth=3, cave_threshold=0.55, features=3)


def key_decode(k):
    return k & 63, (k >> 6) & 63, (k >> 12) & 63, (k >> 18) & 7


def walk(nodes):
    """Yields (idx, x, y, z, size) for every node reachable from the root."""
    stack = [(0, 0, 0, 0, 64)]
    while stack:
        i, x, y, z, s = stack.pop()
        yield i, x, y, z, s
        n = nodes[i]
        if n["child_base"] == A.INVALID_U32:
            continue
        h = s // 2
        rank = 0
        for ci in range(8):
            if n["child_mask"] & (1 << ci):
                stack.append((int(n["child_base"]) + rank, x + (ci & 1) * h, y + ((ci >> 1) & 1) * h,
                              z + ((ci >> 2) & 1) * h, h))
                rank += 1


@pytest.mark.parametrize("spec,key", [(SPEC, (0, 0, 0)), (CAVES, (1, 0, -1))])
def test_keys_materials_and_leaves_match_dense_grid(spec, key):
    ch = build_chunk(spec, *key)
    mat = chunk_materials(spec, *key)  # [y, z, x]
    covered = np.zeros_like(mat, dtype=np.int32)
    for i, x, y, z, s in walk(ch.nodes):
        n = ch.nodes[i]
        kx, ky, kz, lvl = key_decode(int(n["key"]))
        assert 64 >> lvl == s and (kx * s, ky * s, kz * s) == (x, y, z), "pack_key round trip"
        if n["child_base"] == A.INVALID_U32:
            block = mat[y:y + s, z:z + s, x:x + s]
            assert (block == n["material"]).all(), "leaf material must cover its cube"
            covered[y:y + s, z:z + s, x:x + s] += 1
    # every solid voxel is inside exactly one leaf; implicit air everywhere else
    assert ((covered == 1) == (mat != 0)).all()


def test_macro_bits_are_or_of_solid_voxels():
    ch = build_chunk(CAVES, 0, 0, 0)
    mat = chunk_materials(CAVES, 0, 0, 0)
    bits = np.unpackbits(ch.macro.view(np.uint8), bitorder="little")
    for mz in range(8):
        for my in range(8):
            for mx in range(8):
                solid = (mat[my * 8:my * 8 + 8, mz * 8:mz * 8 + 8, mx * 8:mx * 8 + 8] != 0).any()
                assert bits[mx + 8 * (my + 8 * mz)] == solid


def test_colinfo_is_top_solid_voxel():
    ch = build_chunk(CAVES, 0, 0, 0)
    mat = chunk_materials(CAVES, 0, 0, 0)
    e16 = ch.colinfo.view(np.uint16)
    for lz in range(0, 64, 3):
        for lx in range(64):
            col = mat[:, lz, lx]
            ys = np.nonzero(col)[0]
            e = int(e16[lz * 64 + lx])
            if len(ys) == 0:
                assert e & 0xFF == 255
            else:
                assert e & 0xFF == ys[-1] and (e >> 8) == col[ys[-1]]


def test_ropes_point_beyond_the_face_to_not_smaller_cubes():
    """A rope target lies on the far side of the face, covers the face, and is not
    smaller than the source.  It is face-adjacent unless the sibling toward the
    face is implicit air: then builder_ropes.rs:106-127 falls back to the
    parent's neighbour descended one level, which skips the empty sibling."""
    ch = build_chunk(SPEC, 0, 0, 0)
    cube = {i: (x, y, z, s) for i, x, y, z, s in walk(ch.nodes)}
    faces = ["px", "nx", "py", "ny", "pz", "nz"]
    checked = adjacent = 0
    for i, (x, y, z, s) in cube.items():
        r = ch.ropes[i]
        for f, name in enumerate(faces):
            t = int(r[name])
            if t == A.INVALID_U32:
                continue
            tx, ty, tz, ts = cube[t]
            assert ts >= s
            axis, sign = f // 2, (1 if f % 2 == 0 else -1)
            lo = [x, y, z]
            tlo = [tx, ty, tz]
            if sign > 0:
                assert tlo[axis] >= lo[axis] + s
                adjacent += tlo[axis] == lo[axis] + s
            else:
                assert tlo[axis] + ts <= lo[axis]
                adjacent += tlo[axis] + ts == lo[axis]
            for a in range(3):
                if a != axis:
                    assert tlo[a] <= lo[a] and lo[a] + s <= tlo[a] + ts
            checked += 1
    assert checked > 1000 and adjacent > 0.9 * checked


def test_stone_collapse_and_uniform_collapse_happen():
    ch = build_chunk(WorldSpec(seed=1, height_min=40, height_max=48, dirt_depth=3), 0, 0, 0)
    leaves = ch.nodes[ch.nodes["child_base"] == A.INVALID_U32]
    lv = (leaves["key"] >> 18) & 7
    assert ((lv < 6) & (leaves["material"] == 3)).any(), "large stone leaves expected"


def test_ground_height_range():
    hs = [ground_height(SPEC, x, z) for x in range(0, 640, 7) for z in range(0, 640, 11)]
    assert min(hs) >= 8 and max(hs) <= 48 and max(hs) - min(hs) > 15


def test_empty_chunk_is_one_air_leaf():
    ch = build_chunk(SPEC, 0, 5, 0)
    assert len(ch.nodes) == 1 and ch.nodes[0]["child_base"] == A.INVALID_U32 and ch.nodes[0]["material"] == 0
    assert ch.macro_empty == 1
