"""Resident world bookkeeping: chunk builds, slots, node arena, chunk grid.

Mirrors the parts of the reference streaming manager that define the data the
passes read:
  * slots are dense in [0, chunk_count) and an unloaded slot is filled by
    moving the last slot into the hole (streaming/manager/slots.rs:163-766),
  * ChunkMetaGpu packing: origin = key * 64, macro_base = slot * 16,
    colinfo_base = slot * 2048, macro_empty = all macro words zero
    (slots.rs:231-250),
  * chunk grid index (iz * ny + iy) * nx + ix, INVALID for empty cells
    (streaming/manager/grid.rs:15-72).
  * the node arena: a best-fit free list over [0, node_capacity) with full
    coalescing (streaming/node_arena.rs:14-111); when it cannot place a
    chunk, up to EVICT_ATTEMPTS farthest chunks outside the active radius are
    unloaded first (slots.rs:203-223, 457-541), else the chunk is deferred,
  * the per-frame upload budget (UploadQueue.take_budgeted,
    streaming/manager/uploads.rs:138-238): slot rewrites first, then content
    rewrites, then the promotions of the active area nearest first.
Host mirrors of every device buffer are kept so a CPU checker can read
exactly what the device reads.
"""
from __future__ import annotations

import bisect
import ctypes as C
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import _abi as A


@dataclass
class WorldSpec:
    seed: int = 12345
    height_min: int = 8
    height_max: int = 48
    dirt_depth: int = 3
    carve_mod: int = 0          # 50 => 2 % of solid voxels carved
    cave_threshold: float = 2.0  # >= 1 disables caves
    height_scale_vox: float = 64.0
    features: int = 0           # bit0 trees, bit1 light voxels

    def params(self) -> A.WorldParams:
        return A.WorldParams(self.seed, self.height_min, self.height_max, self.dirt_depth, self.carve_mod,
                             self.cave_threshold, self.height_scale_vox, self.features)


@dataclass
class ChunkData:
    key: tuple
    nodes: np.ndarray      # NODE_DTYPE
    ropes: np.ndarray      # ROPES_DTYPE
    macro: np.ndarray      # (16,) u32
    colinfo: np.ndarray    # (2048,) u32
    solid_voxels: int = 0

    @property
    def macro_empty(self) -> int:
        return int(not self.macro.any())


def build_chunk(spec: WorldSpec, cx: int, cy: int, cz: int) -> ChunkData:
    """Runs the C++ port of the reference chunk builder (svo/builder.rs:846-986)."""
    lib = A.host_lib()
    wp = spec.params()
    out = A.BuiltChunk()
    st = lib.vxe_build_chunk(C.byref(wp), cx, cy, cz, C.byref(out))
    if st != A.VXE_OK:
        raise A.VxeError(st, "vxe_build_chunk")
    try:
        n = out.node_count
        nodes = np.ctypeslib.as_array(C.cast(out.nodes, C.POINTER(C.c_uint32)), shape=(n * 4,)).copy().view(A.NODE_DTYPE)
        ropes = np.ctypeslib.as_array(C.cast(out.ropes, C.POINTER(C.c_uint32)), shape=(n * 8,)).copy().view(A.ROPES_DTYPE)
        macro = np.array(out.macro_words, dtype=np.uint32)
        colinfo = np.array(out.colinfo_words, dtype=np.uint32)
        return ChunkData((cx, cy, cz), nodes, ropes, macro, colinfo, out.solid_voxels)
    finally:
        lib.vxe_free_chunk(C.byref(out))


def chunk_materials(spec: WorldSpec, cx: int, cy: int, cz: int) -> np.ndarray:
    m = np.zeros(64 * 64 * 64, dtype=np.uint8)
    st = A.host_lib().vxe_chunk_materials(C.byref(spec.params()), cx, cy, cz, m.ctypes.data)
    if st != A.VXE_OK:
        raise A.VxeError(st, "vxe_chunk_materials")
    return m.reshape(64, 64, 64)  # [y, z, x]


def ground_height(spec: WorldSpec, wx: int, wz: int) -> int:
    return int(A.host_lib().vxe_ground_height(C.byref(spec.params()), wx, wz))


EVICT_ATTEMPTS = 8                     # streaming/types.rs:15
MAX_UPLOADS_PER_FRAME = 64             # streaming/types.rs:25
MAX_UPLOAD_BYTES_PER_FRAME = 64 << 20  # streaming/types.rs:26
ACTIVE_RADIUS = 14                     # app/config.rs:7 (chunks, in x-z)


class NodeArena:
    """Free-list allocator over node indices (streaming/node_arena.rs:14-111).

    Free ranges are kept sorted by start.  alloc() is best-fit: the first of
    the smallest ranges that fit (a perfect fit ends the search), taken from
    its front.  release() inserts the range in order and merges it with both
    neighbours as far as they touch."""

    def __init__(self, capacity: int):
        self.capacity = capacity
        self.free = [(0, capacity)]  # sorted (start, length)

    def alloc(self, n: int):
        if n == 0:
            return 0
        best_i, best_len = None, 0xFFFFFFFF
        for i, (s, l) in enumerate(self.free):
            if l >= n and l < best_len:
                best_i, best_len = i, l
                if l == n:
                    break
        if best_i is None:
            return None
        s, l = self.free[best_i]
        if l == n:
            self.free.pop(best_i)
        else:
            self.free[best_i] = (s + n, l - n)
        return s

    def release(self, start: int, n: int) -> None:
        if n == 0:
            return
        i = bisect.bisect_left(self.free, (start,))
        self.free.insert(i, (start, n))
        while i > 0:  # merge backward
            (a0, al), (b0, bl) = self.free[i - 1], self.free[i]
            if a0 + al != b0:
                break
            self.free[i - 1] = (a0, al + bl)
            self.free.pop(i)
            i -= 1
        while i + 1 < len(self.free):  # merge forward
            (a0, al), (b0, bl) = self.free[i], self.free[i + 1]
            if a0 + al != b0:
                break
            self.free[i] = (a0, al + bl)
            self.free.pop(i + 1)


def in_active_xz(center, key, radius: int = ACTIVE_RADIUS) -> bool:
    """keep::in_active_xz (streaming/manager/keep.rs:31-36)."""
    dx, dz = key[0] - center[0], key[2] - center[2]
    return dx * dx + dz * dz <= radius * radius


def upload_dist_score(key, center) -> float:
    """uploads.rs:56-62: |dx| + |dz| + 2 |dy| in f32."""
    f = np.float32
    dx, dz, dy = f(key[0] - center[0]), f(key[2] - center[2]), f(key[1] - center[1])
    return float(abs(dx) + abs(dz) + f(2.0) * abs(dy))


def evict_score(key, center) -> float:
    """slots.rs:496-499: dx^2 + dz^2 + 4 dy^2 in f32."""
    f = np.float32
    dx, dz, dy = f(key[0] - center[0]), f(key[2] - center[2]), f(key[1] - center[1])
    return float(dx * dx + dz * dz + f(4.0) * dy * dy)


@dataclass
class Upload:
    slot: int
    meta: np.ndarray   # (12,) u32 view of one ChunkMetaGpu
    node_base: int
    data: ChunkData | None  # None => meta-only rewrite (slot move without new data)
    key: tuple | None = None
    rewrite: bool = False   # slot rewrite: meta + macro + colinfo words, no node records

    @property
    def nbytes(self) -> int:
        """upload_bytes (uploads.rs:46-54): meta, nodes, macro words, ropes, colinfo words."""
        if self.data is None:
            return 48
        n = 0 if self.rewrite else len(self.data.nodes)
        return 48 + n * 16 + 16 * 4 + n * 32 + 2048 * 4


class UploadQueue:
    """The streaming manager's upload queues and per-frame budget
    (streaming/manager/uploads.rs): slot rewrites (slots whose contents moved,
    newest first), content rewrites, promotions in the active area (sorted by
    distance to the centre) and the rest."""

    def __init__(self):
        self.slot_rewrite_q: deque = deque()
        self.slot_rewrite_set: set = set()
        self.rewrite: deque = deque()
        self.active: deque = deque()
        self.other: deque = deque()

    def __len__(self) -> int:
        return len(self.slot_rewrite_q) + len(self.rewrite) + len(self.active) + len(self.other)

    def mark_slot_rewrite(self, slot: int) -> None:
        """mark_slot_rewrite (uploads.rs:9-15)."""
        if slot not in self.slot_rewrite_set:
            self.slot_rewrite_set.add(slot)
            self.slot_rewrite_q.appendleft(slot)

    def enqueue(self, u: Upload, center, promote: bool = True, radius: int = ACTIVE_RADIUS) -> None:
        """enqueue (uploads.rs:64-90)."""
        if not promote:
            self.rewrite.appendleft(u)
            return
        if center is None:
            self.other.append(u)
            return
        if in_active_xz(center, u.key, radius):
            us = upload_dist_score(u.key, center)
            pos = next((i for i, e in enumerate(self.active) if upload_dist_score(e.key, center) > us),
                       len(self.active))
            self.active.insert(pos, u)
        else:
            self.other.append(u)

    def rebucket(self, center, radius: int = ACTIVE_RADIUS) -> None:
        """rebucket_for_center (uploads.rs:92-117).  Its test is the x-z
        square |dx|, |dz| <= radius (enqueue's is the disc), and it keeps the
        queues' order (active ones first) without sorting again."""
        def square(k):
            return abs(k[0] - center[0]) <= radius and abs(k[2] - center[2]) <= radius

        everything = list(self.active) + list(self.other)
        self.active = deque(u for u in everything if square(u.key))
        self.other = deque(u for u in everything if not square(u.key))

    def take_budgeted(self, world: "World") -> list:
        """take_budgeted (uploads.rs:138-238): this frame's uploads."""
        backlog = len(self)
        max_uploads = min(max(MAX_UPLOADS_PER_FRAME + backlog // 4, MAX_UPLOADS_PER_FRAME), 128)
        max_bytes = min(max(MAX_UPLOAD_BYTES_PER_FRAME + backlog * (256 << 10), MAX_UPLOAD_BYTES_PER_FRAME), 128 << 20)
        out, nbytes = [], 0
        # 0) slot rewrites first
        cap = min(256 + backlog, 2048)
        taken = 0
        while taken < cap and self.slot_rewrite_q:
            slot = self.slot_rewrite_q.popleft()
            self.slot_rewrite_set.discard(slot)
            u = world.slot_rewrite_upload(slot)
            if u is None:
                continue
            if nbytes + u.nbytes > max_bytes and out:  # at least one upload per frame
                self.slot_rewrite_set.add(slot)
                self.slot_rewrite_q.appendleft(slot)
                break
            nbytes += u.nbytes
            out.append(u)
            taken += 1
        # 1) content rewrites (capped), then active promotions, then the rest
        rewrite_cap = min(max(max_uploads // 2, 8), 64)
        rewrites = 0
        while True:
            if rewrites < rewrite_cap and self.rewrite:
                which, u = self.rewrite, self.rewrite.popleft()
                rewrites += 1
            elif self.active:
                which, u = self.active, self.active.popleft()
            elif self.other:
                which, u = self.other, self.other.popleft()
            else:
                break
            if len(out) >= max_uploads:
                which.append(u)
                break
            slot = world.key_to_slot.get(u.key)
            if slot is None:  # no longer resident
                continue
            u.slot = slot
            u.meta = u.meta.copy()
            u.meta[6] = slot * A.MACRO_WORDS_PER_CHUNK
            u.meta[7] = slot * A.COLINFO_WORDS_PER_CHUNK
            if nbytes + u.nbytes > max_bytes and out:
                which.append(u)
                break
            nbytes += u.nbytes
            out.append(u)
        return out


class World:
    """A resident grid of chunks around ``grid_origin`` with host mirrors."""

    def __init__(self, spec: WorldSpec, grid_origin, grid_dims, node_capacity: int, chunk_capacity: int | None = None,
                 builder=None, mirror: bool = True, active_radius: int = ACTIVE_RADIUS, queue: UploadQueue | None = None):
        """`mirror`: keep host copies of the node and rope arenas (what the
        CPU oracle and the host-side tests read); a streaming loop that only
        uploads can leave them out -- the chunk cache keeps each chunk's
        records for its uploads.  `active_radius`: chunks within it (x-z, of
        `center`) are never evicted.  `queue`: the uploads go through this
        per-frame budget (UploadQueue.take_budgeted) instead of being
        returned by populate() / shift()."""
        self.mirror = mirror
        self.active_radius = active_radius
        self.queue = queue
        self.evicted: list[tuple] = []   # keys unloaded to make room, in order
        self.deferred: list[tuple] = []  # keys that found no room (the reference re-queues their build)
        self._log: list = []             # uploads of add() / remove() since the last populate() / shift()
        self.uploading: set = set()      # with a queue: placed, not uploaded yet (not in the grid)
        self._device = False             # placing chunks built on the device (no host records)
        self._moves: list = []           # device slot moves made by evictions during a device placement
        self.spec = spec
        self.grid_origin = tuple(int(v) for v in grid_origin)
        self.grid_dims = tuple(int(v) for v in grid_dims)
        nx, ny, nz = self.grid_dims
        self.chunk_capacity = chunk_capacity or nx * ny * nz
        self.grid_capacity = nx * ny * nz
        self.arena = NodeArena(node_capacity)
        self.node_capacity = node_capacity
        self.nodes = np.zeros(node_capacity if mirror else 0, dtype=A.NODE_DTYPE)
        self.ropes = np.zeros(node_capacity if mirror else 0, dtype=A.ROPES_DTYPE)
        self.metas = np.zeros((self.chunk_capacity, 12), dtype=np.uint32)
        self.macro = np.zeros(self.chunk_capacity * A.MACRO_WORDS_PER_CHUNK, dtype=np.uint32)
        self.colinfo = np.zeros(self.chunk_capacity * A.COLINFO_WORDS_PER_CHUNK, dtype=np.uint32)
        self.grid = np.full(self.grid_capacity, A.INVALID_U32, dtype=np.uint32)
        self.slot_to_key: list[tuple] = []
        self.key_to_slot: dict[tuple, int] = {}
        self.alloc: dict[tuple, tuple] = {}  # key -> (node_base, node_count)
        self.cache: dict[tuple, ChunkData] = {}
        self.builder = builder or (lambda key: build_chunk(self.spec, *key))
        # the chunk the streaming is centred on (the camera's chunk in the reference)
        self.center = (self.grid_origin[0] + nx // 2, self.grid_origin[1] + ny // 2, self.grid_origin[2] + nz // 2)

    # -- data -----------------------------------------------------------------
    def chunk(self, key) -> ChunkData:
        if key not in self.cache:
            self.cache[key] = self.builder(key)
        return self.cache[key]

    @property
    def chunk_count(self) -> int:
        return len(self.slot_to_key)

    def keys_in_grid(self):
        ox, oy, oz = self.grid_origin
        nx, ny, nz = self.grid_dims
        for iz in range(nz):
            for iy in range(ny):
                for ix in range(nx):
                    yield (ox + ix, oy + iy, oz + iz)

    def _meta_for(self, slot: int, key, node_base: int, data: ChunkData) -> np.ndarray:
        m = np.zeros(12, dtype=np.uint32)
        org = np.array([key[0] * 64, key[1] * 64, key[2] * 64, 0], dtype=np.int32)
        m[0:4] = org.view(np.uint32)
        m[4] = node_base
        m[5] = len(data.nodes)
        m[6] = slot * A.MACRO_WORDS_PER_CHUNK
        m[7] = slot * A.COLINFO_WORDS_PER_CHUNK
        m[8] = data.macro_empty
        return m

    def _write_slot(self, slot: int, key, node_base: int, data: ChunkData) -> np.ndarray:
        n = len(data.nodes)
        if self.mirror:
            # plain word copies (a structured-array assignment copies field by field)
            self.nodes.view(np.uint32)[4 * node_base:4 * (node_base + n)] = data.nodes.view(np.uint32).reshape(-1)
            self.ropes.view(np.uint32)[8 * node_base:8 * (node_base + n)] = data.ropes.view(np.uint32).reshape(-1)
        self.macro[slot * 16:(slot + 1) * 16] = data.macro
        self.colinfo[slot * 2048:(slot + 1) * 2048] = data.colinfo
        meta = self._meta_for(slot, key, node_base, data)
        self.metas[slot] = meta
        return meta

    def _place(self, key, n: int):
        """Arena range for n nodes of `key` (try_make_uploading,
        slots.rs:201-221): best fit, else up to EVICT_ATTEMPTS farthest
        chunks unloaded first; None when there is still no room."""
        base = self.arena.alloc(n)
        if base is None:
            for _ in range(EVICT_ATTEMPTS):
                if not self.evict_one_farthest(protect=key):
                    break
                base = self.arena.alloc(n)
                if base is not None:
                    break
        if base is None:
            self.deferred.append(key)
        return base

    def evict_one_farthest(self, protect=None) -> bool:
        """evict_one_farthest (slots.rs:457-541): unloads the chunk farthest
        from `center` (dx^2 + dz^2 + 4 dy^2; the first in slot order on ties)
        among those outside the active radius, never `protect`.  The
        reference's second pass applies the same filter, so it finds
        nothing new: an active area that fills the arena defers builds."""
        best = None
        for k in self.slot_to_key:
            if k == protect or in_active_xz(self.center, k, self.active_radius):
                continue
            d = evict_score(k, self.center)
            if best is None or d > best[0]:
                best = (d, k)
        if best is None:
            return False
        k = best[1]
        self.evicted.append(k)
        if self._device:
            moved = self._unload(k)
            if moved is not None:
                self._moves.append(moved)
        else:
            self.remove(k)
        return True

    def add(self, key) -> Upload | None:
        """try_make_uploading (slots.rs:163-275): an arena range (evicting if
        needed) + the next dense slot.  None when the chunk was deferred."""
        data = self.chunk(key)
        n = len(data.nodes)
        base = self._place(key, n)
        if base is None:
            return None
        slot = len(self.slot_to_key)
        if slot >= self.chunk_capacity:
            raise MemoryError("chunk slots exhausted")
        self.slot_to_key.append(key)
        self.key_to_slot[key] = slot
        self.alloc[key] = (base, n)
        meta = self._write_slot(slot, key, base, data)
        u = Upload(slot, meta, base, data, key=key)
        self._log.append(u)
        if self.queue is not None:
            self.uploading.add(key)
            self.queue.enqueue(u, self.center, radius=self.active_radius)
        return u

    def _unload(self, key):
        """unload_chunk (slots.rs:277-363) for a resident chunk: frees its
        arena range; the last slot moves into its slot.  Returns the moved
        (from, to) slots or None."""
        slot = self.key_to_slot.pop(key)
        base, n = self.alloc.pop(key)
        self.arena.release(base, n)
        self.uploading.discard(key)
        last = len(self.slot_to_key) - 1
        moved = None
        if slot != last:
            mkey = self.slot_to_key[last]
            self.slot_to_key[slot] = mkey
            self.key_to_slot[mkey] = slot
            moved = (last, slot)
        self.slot_to_key.pop()
        return moved

    def remove(self, key) -> list[Upload]:
        """Unload: free arena, move the last slot into the hole (keeps slots dense)."""
        moved = self._unload(key)
        last = len(self.slot_to_key)
        ups = []
        if moved is not None:
            slot = moved[1]
            mkey = self.slot_to_key[slot]
            mbase, _ = self.alloc[mkey]
            data = self.chunk(mkey)
            # macro / colinfo live at slot-derived bases, so they move with the slot.
            meta = self._write_slot(slot, mkey, mbase, data)
            if self.queue is not None:
                self.queue.mark_slot_rewrite(slot)
            ups.append(Upload(slot, meta, mbase, data, key=mkey))
        self.metas[last] = 0
        self._log.extend(ups)
        return ups

    def mark_uploaded(self, uploads) -> bool:
        """The promotions among `uploads` completed (the caller applied them):
        those chunks join the grid (slots.rs:95-158).  Returns whether the
        grid changed."""
        done = [u.key for u in uploads if not u.rewrite and u.key in self.uploading]
        for k in done:
            self.uploading.discard(k)
        if done:
            self.rebuild_grid()
        return bool(done)

    def slot_rewrite_upload(self, slot: int) -> Upload | None:
        """make_slot_rewrite_upload (uploads.rs:17-43): the slot's current
        meta, macro and colinfo words (its nodes stay where they are)."""
        if slot >= len(self.slot_to_key):
            return None
        key = self.slot_to_key[slot]
        base, _ = self.alloc[key]
        return Upload(slot, self.metas[slot].copy(), base, self.chunk(key), key=key, rewrite=True)

    def rebuild_grid(self) -> np.ndarray:
        ox, oy, oz = self.grid_origin
        nx, ny, nz = self.grid_dims
        self.grid[:] = A.INVALID_U32
        for slot, (cx, cy, cz) in enumerate(self.slot_to_key):
            if (cx, cy, cz) in self.uploading:
                continue
            ix, iy, iz = cx - ox, cy - oy, cz - oz
            if 0 <= ix < nx and 0 <= iy < ny and 0 <= iz < nz:
                self.grid[(iz * ny + iy) * nx + ix] = slot
        return self.grid

    def prebuild(self, keys, threads: int | None = None) -> None:
        """Builds missing chunks on a thread pool (the C++ builder releases the GIL),
        like the reference's rayon build pool (streaming/build_pool.rs:19-25)."""
        import os
        from concurrent.futures import ThreadPoolExecutor

        todo = [k for k in keys if k not in self.cache]
        if len(todo) < 4:
            for k in todo:
                self.chunk(k)
            return
        with ThreadPoolExecutor(max_workers=threads or min(32, os.cpu_count() or 1)) as ex:
            for k, data in zip(todo, ex.map(self.builder, todo)):
                self.cache[k] = data

    def prebuild_device(self, renderer, keys, batch: int = 256) -> None:
        """Builds missing chunks on the device (Renderer.build_chunks) in batches
        and keeps the host copies the upload path reads; the results equal
        prebuild()'s byte for byte.  Per batch: a count-only build sizes the
        node buffers, the full build follows, the valid node and rope rows are
        compacted on the device and come back in one copy each."""
        import torch

        todo = [k for k in keys if k not in self.cache]
        wp = self.spec.params()
        for i in range(0, len(todo), batch):
            part = todo[i:i + batch]
            coords = torch.tensor(part, dtype=torch.int32, device=renderer.torch_device)
            cap = int(renderer.build_chunks(wp, coords, node_cap=0)["counts"][:, 0].max())
            out = renderer.build_chunks(wp, coords, node_cap=cap)
            cnt = out["counts"][:, 0]
            keep = torch.arange(cap, device=coords.device)[None, :] < cnt[:, None]
            nodes = out["nodes"][keep].cpu().numpy().view(np.uint32)
            ropes = out["ropes"][keep].cpu().numpy().view(np.uint32)
            counts = out["counts"].cpu().numpy().view(np.uint32)
            macro = out["macro"].cpu().numpy().view(np.uint32)
            colinfo = out["colinfo"].cpu().numpy().view(np.uint32)
            first = 0
            for j, key in enumerate(part):
                n = int(counts[j, 0])
                self.cache[key] = ChunkData(key, nodes[first:first + n].reshape(-1).view(A.NODE_DTYPE),
                                            ropes[first:first + n].reshape(-1).view(A.ROPES_DTYPE), macro[j],
                                            colinfo[j], int(counts[j, 1]))
                first += n

    def _add_device(self, renderer, keys, batch: int = 2048) -> None:
        """add() for `keys`, built on the device straight into `renderer`'s
        world: a counting build per batch gives the node counts, slots and
        arena ranges are taken exactly as add() takes them, the resident build
        writes nodes, ropes, macro / colinfo words and metas in place."""
        import torch

        wp = self.spec.params()
        for i in range(0, len(keys), batch):
            part = keys[i:i + batch]
            coords = torch.tensor(part, dtype=torch.int32, device=renderer.torch_device)
            counts = renderer.build_chunks(wp, coords, node_cap=0)["counts"].cpu().numpy().view(np.uint32)
            placed = []
            self._device = True
            try:
                for key, (n, _solid) in zip(part, counts.tolist()):
                    base = self._place(key, n)
                    if base is None:
                        continue
                    slot = len(self.slot_to_key)
                    if slot >= self.chunk_capacity:
                        raise MemoryError("chunk slots exhausted")
                    self.slot_to_key.append(key)
                    self.key_to_slot[key] = slot
                    self.alloc[key] = (base, n)
                    placed.append(key)
            finally:
                self._device = False
            # evictions moved slots (maybe slots of this batch, not built yet):
            # the moves first, then every placed chunk still resident at its final slot
            if self._moves:
                renderer.move_slots(self._moves)
                self._moves = []
            places = [(k, self.key_to_slot[k], *self.alloc[k]) for k in placed if k in self.key_to_slot]
            renderer.build_resident(wp, places)

    def populate_device(self, renderer, batch: int = 2048) -> None:
        """populate() with every chunk built on the device straight into
        `renderer`'s world (_add_device), then the grid.  No chunk data passes
        through the host, so this world's host mirrors (nodes, ropes, macro,
        colinfo, metas) stay empty for these chunks."""
        self._add_device(renderer, [k for k in self.keys_in_grid() if k not in self.key_to_slot], batch)
        self.rebuild_grid()
        renderer.write_chunk_grid(self.grid)

    def shift_device(self, renderer, dx: int, dy: int, dz: int) -> tuple:
        """shift() for a world kept on the device: chunks that left free their
        arena range and the last slot moves into each hole (vxe_move_slots, in
        the order remove() takes them), entering chunks are built resident
        (_add_device), then the grid -- the same slots, arena ranges and
        device records as shift() followed by the uploads it returns.  Returns
        (chunks built, slots moved)."""
        self.grid_origin = (self.grid_origin[0] + dx, self.grid_origin[1] + dy, self.grid_origin[2] + dz)
        self.center = (self.center[0] + dx, self.center[1] + dy, self.center[2] + dz)
        want = set(self.keys_in_grid())
        moves = []
        for k in [k for k in self.slot_to_key if k not in want]:
            moved = self._unload(k)
            if moved is not None:
                moves.append(moved)
        renderer.move_slots(moves)
        new = [k for k in self.keys_in_grid() if k not in self.key_to_slot]
        self._add_device(renderer, new)
        self.rebuild_grid()
        renderer.write_chunk_grid(self.grid)
        return len(new), len(moves)

    def _take_log(self) -> list[Upload]:
        """The uploads since the last batch, the last write of each slot
        (none when a queue takes them per frame)."""
        log, self._log = self._log, []
        if self.queue is not None:
            return []
        last = {}
        for u in log:
            last[u.slot] = u
        return [last[s] for s in sorted(last)]

    def populate(self) -> list[Upload]:
        self.prebuild(list(self.keys_in_grid()))
        for k in self.keys_in_grid():
            if k not in self.key_to_slot:
                self.add(k)
        self.rebuild_grid()
        return self._take_log()

    def shift(self, dx: int, dy: int, dz: int) -> list[Upload]:
        """Moves the grid origin (and the centre); unloads chunks that left
        and loads new ones.  Returns the slot writes (or [] with a queue)."""
        self.grid_origin = (self.grid_origin[0] + dx, self.grid_origin[1] + dy, self.grid_origin[2] + dz)
        self.center = (self.center[0] + dx, self.center[1] + dy, self.center[2] + dz)
        if self.queue is not None:
            self.queue.rebucket(self.center, self.active_radius)
        want = set(self.keys_in_grid())
        for k in [k for k in self.slot_to_key if k not in want]:
            self.remove(k)
        for k in self.keys_in_grid():
            if k not in self.key_to_slot:
                self.add(k)
        self.rebuild_grid()
        return self._take_log()

    @property
    def nodes_used(self) -> int:
        return sum(n for _, n in self.alloc.values())

    def world_aabb_m(self):
        ox, oy, oz = self.grid_origin
        nx, ny, nz = self.grid_dims
        lo = np.array([ox, oy, oz], dtype=np.float64) * 6.4
        return lo, lo + np.array([nx, ny, nz], dtype=np.float64) * 6.4


class Clipmap:
    """Toroidal clipmap state (C++ port of clipmap.rs:182-577)."""

    def __init__(self, spec: WorldSpec, levels: int, res: int = 256, base_cell_m: float = 1.0):
        self.levels, self.res = levels, res
        self._h = A.host_lib().vxe_clipmap_new(C.byref(spec.params()), levels, res, base_cell_m)
        if not self._h:
            raise A.VxeError(A.STATUS_NAMES and 1, "vxe_clipmap_new")
        self.tex = np.zeros((levels, res, res), dtype=np.float32)  # host mirror of the layers
        self.params = A.ClipmapGpu()

    def update(self, cam_x: float, cam_z: float):
        """Returns (params, [(level, x, y, w, h, data)]) and applies them to the host mirror."""
        params = A.ClipmapGpu()
        pp = C.POINTER(A.ClipPatch)()
        n = C.c_uint32()
        st = A.host_lib().vxe_clipmap_update(self._h, cam_x, cam_z, C.byref(params), C.byref(pp), C.byref(n))
        if st != A.VXE_OK:
            raise A.VxeError(st, "vxe_clipmap_update")
        patches = []
        for i in range(n.value):
            p = pp[i]
            data = np.ctypeslib.as_array(p.data, shape=(p.h * p.w,)).copy().reshape(p.h, p.w)
            self.tex[p.level, p.y:p.y + p.h, p.x:p.x + p.w] = data
            patches.append((p.level, p.x, p.y, p.w, p.h, data))
        self.params = params
        return params, patches

    def update_device(self, renderer, cam_x: float, cam_z: float):
        """The same update with the patch texels evaluated on the device straight
        into `renderer`'s clipmap (no host texels; the host mirror is not updated)."""
        st = renderer._lib.vxe_clipmap_update_device(renderer._ctx, self._h, cam_x, cam_z)
        if st != A.VXE_OK:
            raise A.VxeError(st, "vxe_clipmap_update_device", renderer._lib.vxe_last_error(renderer._ctx).decode())

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                A.host_lib().vxe_clipmap_free(h)
            except Exception:
                pass
            self._h = None


def build_camera(pos, yaw, pitch, present, internal, frame_index, time_s, world: World | None = None,
                 jitter=True, prev_view_proj=None, fovy_deg: float = 60.0) -> A.CameraGpu:
    """CameraGpu packing (app/app.rs:411-511)."""
    p = A.CameraParams()
    p.pos[:] = [float(v) for v in pos]
    p.yaw, p.pitch = float(yaw), float(pitch)
    p.fovy_rad = float(np.deg2rad(fovy_deg))
    p.z_near, p.z_far = 0.1, 1000.0
    p.present_w, p.present_h = present
    p.internal_w, p.internal_h = internal
    p.frame_index = frame_index
    p.jitter = 1 if jitter else 0
    p.time_s = float(time_s)
    if world is not None:
        p.chunk_count = world.chunk_count
        p.grid_origin_chunk[:] = list(world.grid_origin)
        p.grid_dims[:] = list(world.grid_dims)
    if prev_view_proj is not None:
        p.has_prev = 1
        C.memmove(C.byref(p.prev_view_proj), C.byref(prev_view_proj), C.sizeof(A.Mat4))
    cam = A.CameraGpu()
    st = A.host_lib().vxe_build_camera(C.byref(p), C.byref(cam))
    if st != A.VXE_OK:
        raise A.VxeError(st, "vxe_build_camera")
    return cam
