"""Host bookkeeping that defines what the passes read: slots, metas, arena, grid."""
import numpy as np
import pytest

from vxe import _abi as A
from vxe.world import ChunkData, NodeArena, Upload, World, WorldSpec

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


def test_arena_best_fit_and_full_coalescing():
    # streaming/node_arena.rs: the smallest range that fits (first of equals,
    # perfect fit ends the search), taken from its front; frees merge with
    # both neighbours.
    a = NodeArena(100)
    assert [a.alloc(30), a.alloc(30), a.alloc(30)] == [0, 30, 60]
    assert a.alloc(20) is None and a.alloc(0) == 0
    a.release(30, 30)
    assert a.free == [(30, 30), (90, 10)]
    assert a.alloc(10) == 90       # best fit (first fit would take 30)
    assert a.alloc(20) == 30       # front of the only range that fits
    assert a.free == [(50, 10)]
    a.release(0, 30)               # not adjacent to (50, 10)
    a.release(60, 30)              # merges forward into nothing, backward with (50, 10)
    assert a.free == [(0, 30), (50, 40)]
    a.release(30, 20)              # merges both ways
    assert a.free == [(0, 90)]
    a.release(90, 10)
    assert a.free == [(0, 100)]
    b = NodeArena(64)
    xs = [b.alloc(8) for _ in range(8)]
    for x in (8, 24, 40):
        b.release(x, 8)
    b.release(16, 8)               # joins 8..32
    assert b.free == [(8, 24), (40, 8)]
    assert b.alloc(8) == 40        # perfect fit beats the earlier, larger range


def test_arena_exhaustion_defers_the_chunk():
    # try_make_uploading (streaming/manager/slots.rs:201-221): no room and
    # nothing evictable (everything inside the active radius) defers the
    # build instead of failing.
    w = World(SPEC, (0, 0, 0), (2, 1, 1), node_capacity=4, builder=fake_builder)
    w.populate()
    assert w.deferred and all(k not in w.key_to_slot for k in w.deferred)
    assert w.evicted == []


def _evict_choice(keys, center, radius, protect):
    """slots.rs:478-507, restated: the largest dx^2 + dz^2 + 4 dy^2 (f32) outside
    the active x-z radius, first in slot order on ties."""
    best = None
    for k in keys:
        dx, dz = k[0] - center[0], k[2] - center[2]
        if k == protect or dx * dx + dz * dz <= radius * radius:
            continue
        d = np.float32(dx) * np.float32(dx) + np.float32(dz) * np.float32(dz) + \
            np.float32(4.0) * np.float32(k[1] - center[1]) ** 2
        if best is None or d > best[0]:
            best = (d, k)
    return None if best is None else best[1]


def test_arena_exhaustion_evicts_the_farthest_outside_the_active_radius():
    def sized(key):  # 10 nodes per chunk
        nodes = np.zeros(10, dtype=A.NODE_DTYPE)
        nodes["child_base"] = A.INVALID_U32
        return ChunkData(key, nodes, np.zeros(10, dtype=A.ROPES_DTYPE), np.ones(16, dtype=np.uint32),
                         np.zeros(2048, dtype=np.uint32))

    # 6x1x6 grid centred at (3, 0, 3); room for 30 of its 36 chunks
    w = World(SPEC, (0, 0, 0), (6, 1, 6), node_capacity=300, builder=sized, active_radius=2)
    assert w.center == (3, 0, 3)
    order = list(w.keys_in_grid())
    expect_evicted = []
    resident = []
    for k in order:
        if len(resident) == 30:
            victim = _evict_choice(resident, w.center, 2, k)
            expect_evicted.append(victim)
            i = resident.index(victim)  # the last slot moves into the hole
            resident[i] = resident[-1]
            resident.pop()
        resident.append(k)
    w.populate()
    assert w.evicted == expect_evicted
    assert not w.deferred
    assert w.slot_to_key == resident
    check_invariants(w)
    # the active area is never evicted
    assert all(not (abs(k[0] - 3) ** 2 + abs(k[2] - 3) ** 2 <= 4) for k in w.evicted)


def test_take_budgeted_order_and_budgets():
    # uploads.rs:138-238: slot rewrites first, then the active promotions
    # nearest first, then the rest; at most max_uploads per frame and the
    # byte budget (but always one upload).
    from vxe.world import UploadQueue

    def big(key):
        n = 400_000  # 19.2 MB of node + rope records
        nodes = np.zeros(n, dtype=A.NODE_DTYPE)
        return ChunkData(key, nodes, np.zeros(n, dtype=A.ROPES_DTYPE), np.ones(16, dtype=np.uint32),
                         np.zeros(2048, dtype=np.uint32))

    q = UploadQueue()
    w = World(SPEC, (0, 0, 0), (8, 1, 8), node_capacity=1 << 26, builder=big, active_radius=3, queue=q)
    assert w.populate() == []                 # the queue takes them
    assert len(q) == 64 and len(q.active) + len(q.other) == 64
    scores = [((u.key[0] - 4) ** 2 + (u.key[2] - 4) ** 2) for u in q.active]
    assert all(s <= 9 for s in scores)
    d1 = [abs(u.key[0] - 4) + abs(u.key[2] - 4) for u in q.active]
    assert d1 == sorted(d1)                   # nearest first (stable on ties)
    q.mark_slot_rewrite(5)
    q.mark_slot_rewrite(2)
    backlog = len(q)                          # 66
    max_bytes = min(max((64 << 20) + backlog * (256 << 10), 64 << 20), 128 << 20)
    first = q.take_budgeted(w)
    assert [u.slot for u in first[:2]] == [2, 5] and first[0].rewrite and first[1].rewrite
    assert first[0].nbytes == 48 + 64 + 8192
    promos = first[2:]
    per = 48 + 400_000 * 48 + 64 + 8192
    assert len(promos) == (max_bytes - 2 * (48 + 64 + 8192)) // per
    assert [u.key for u in promos] == [u.key for u in first[2:]]
    assert all(w.key_to_slot[u.key] == u.slot and u.meta[6] == u.slot * 16 for u in promos)
    total = 0
    while len(q):
        got = q.take_budgeted(w)
        assert got
        total += len(got)
    assert total + len(promos) == 64
    # rebucketing after a move uses the x-z square, keeping the queue order
    for key in list(w.key_to_slot)[:5]:
        q.enqueue(Upload(w.key_to_slot[key], w.metas[w.key_to_slot[key]].copy(), 0, w.chunk(key), key=key),
                  w.center, radius=3)
    q.rebucket((4, 0, 1), radius=3)
    assert all(abs(u.key[0] - 4) <= 3 and abs(u.key[2] - 1) <= 3 for u in q.active)
    assert all(not (abs(u.key[0] - 4) <= 3 and abs(u.key[2] - 1) <= 3) for u in q.other)
