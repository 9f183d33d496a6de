"""Host bookkeeping that defines what the passes read: slots, metas, arena, grid."""
import numpy as np
import pytest

from vxe import _abi as A
from vxe.world import NodeArena, World, WorldSpec, ChunkData

SPEC = WorldSpec(seed=5, height_min=8, height_max=20)


def fake_builder(key):
    n = 3 + (abs(hash(key)) % 5)
    nodes = np.zeros(n, dtype=A.NODE_DTYPE)
    nodes["child_base"] = A.INVALID_U32
    ropes = np.zeros(n, dtype=A.ROPES_DTYPE)
    macro = np.zeros(16, dtype=np.uint32)
    macro[0] = 1 if key[1] == 0 else 0
    return ChunkData(key, nodes, ropes, macro, np.zeros(2048, dtype=np.uint32))


def check_invariants(w: World):
    nx, ny, nz = w.grid_dims
    ox, oy, oz = w.grid_origin
    assert len(w.slot_to_key) == len(w.key_to_slot)
    spans = []
    for slot, key in enumerate(w.slot_to_key):
        assert w.key_to_slot[key] == slot
        m = w.metas[slot]
        assert tuple(m[0:3].view(np.int32)) == (key[0] * 64, key[1] * 64, key[2] * 64)
        base, n = w.alloc[key]
        assert m[4] == base and m[5] == n
        assert m[6] == slot * 16 and m[7] == slot * 2048
        assert m[8] == int(not w.chunk(key).macro.any())
        assert np.array_equal(w.nodes[base:base + n], w.chunk(key).nodes)
        assert np.array_equal(w.macro[slot * 16:slot * 16 + 16], w.chunk(key).macro)
        spans.append((base, base + n))
        ix, iy, iz = key[0] - ox, key[1] - oy, key[2] - oz
        assert w.grid[(iz * ny + iy) * nx + ix] == slot
    spans.sort()
    for (a0, a1), (b0, b1) in zip(spans, spans[1:]):
        assert a1 <= b0, "arena ranges overlap"
    assert (w.grid != A.INVALID_U32).sum() == len(w.slot_to_key)


def test_populate_and_shift_keep_slots_dense_and_grid_consistent():
    w = World(SPEC, (0, 0, 0), (4, 2, 3), node_capacity=4096, builder=fake_builder)
    ups = w.populate()
    assert len(ups) == 24 and w.chunk_count == 24
    check_invariants(w)
    for d in [(1, 0, 0), (1, 0, 0), (0, 0, -1), (-2, 0, 1)]:
        ups = w.shift(*d)
        check_invariants(w)
        assert len({u.slot for u in ups}) == len(ups)
        for u in ups:
            assert np.array_equal(u.meta, w.metas[u.slot])


def test_arena_first_fit_and_merge():
    a = NodeArena(100)
    x = a.alloc(30)
    y = a.alloc(30)
    z = a.alloc(30)
    assert (x, y, z) == (0, 30, 60) and a.alloc(20) is None
    a.release(30, 30)
    a.release(0, 30)
    assert a.free[0] == (0, 60)
    assert a.alloc(50) == 0


def test_arena_exhaustion_raises():
    w = World(SPEC, (0, 0, 0), (2, 1, 1), node_capacity=4, builder=fake_builder)
    with pytest.raises(MemoryError):
        w.populate()
