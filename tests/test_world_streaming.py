"""Host-side logic of the device-resident world (World.populate_device /
shift_device) against the host path (populate / shift): the same slots and
arena ranges, and slot moves that reproduce the host path's slot contents.
A fake renderer stands in for the device: its counting build uses the host
builder, and it applies placements and slot moves to per-slot keys the way
vxe_build_chunks_resident and vxe_move_slots move the device records."""
import numpy as np
import torch

from vxe.world import World, WorldSpec, build_chunk

SPEC = WorldSpec(seed=5, height_min=8, height_max=40, dirt_depth=3, carve_mod=50)


class FakeRenderer:
    torch_device = "cpu"

    def __init__(self, spec):
        self.spec = spec
        self.slots = {}      # slot -> (key, node_base, node_count) as the device would hold them
        self.grid = None
        self.calls = []

    def build_chunks(self, wp, coords, node_cap=None):
        assert node_cap == 0
        counts = [[len(build_chunk(self.spec, *map(int, c)).nodes), 0] for c in coords.tolist()]
        return {"counts": torch.tensor(counts, dtype=torch.int32)}

    def build_resident(self, wp, places):
        self.calls.append(("build", len(places)))
        for key, slot, base, n in places:
            self.slots[slot] = (tuple(key), base, n)

    def move_slots(self, moves):
        self.calls.append(("move", len(moves)))
        for f, t in moves:  # in order, like the kernel
            self.slots[t] = self.slots[f]

    def write_chunk_grid(self, grid):
        self.grid = grid.copy()


def test_device_streaming_bookkeeping_matches_host_path():
    dims = (6, 2, 5)
    host = World(SPEC, (0, 0, 0), dims, 1 << 22, chunk_capacity=int(np.prod(dims)))
    dev = World(SPEC, (0, 0, 0), dims, 1 << 22, chunk_capacity=int(np.prod(dims)))
    fake = FakeRenderer(SPEC)
    host.populate()
    dev.populate_device(fake, batch=7)  # several counting builds
    for step, d in enumerate([(1, 0, 0), (1, 0, 0), (0, 0, 1), (-2, 0, -1), (3, 0, 2)]):
        before = set(host.key_to_slot)
        host.shift(*d)
        entering = [k for k in host.key_to_slot if k not in before]
        leaving = before - set(host.key_to_slot)
        built, moved = dev.shift_device(fake, *d)
        assert built == len(entering) and moved <= len(leaving), step
        assert dev.key_to_slot == host.key_to_slot, step
        assert dev.alloc == host.alloc, step
        assert np.array_equal(fake.grid, host.grid), step
        # every live slot holds, on the device, the chunk the host path put there
        for slot, key in enumerate(host.slot_to_key):
            base, n = host.alloc[key]
            assert fake.slots[slot] == (key, base, n), (step, slot)
    assert any(c[0] == "move" and c[1] > 0 for c in fake.calls)
