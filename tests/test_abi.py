"""The C-ABI library loads and exports every symbol include/vxe/*.h declares (no GPU calls)."""
import ctypes as C
import re
from pathlib import Path

from vxe import _abi as A

HEADER = Path(__file__).resolve().parents[1] / "include" / "vxe" / "vxe.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(vxe_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported_and_bound():
    names = declared_functions()
    assert len(names) >= 30
    for checked in (False, True):  # libvxe.so and libvxe_checked.so
        lib = A.lib(checked)
        for n in names:
            assert hasattr(lib, n), f"{n} missing from {'libvxe_checked.so' if checked else 'libvxe.so'}"
            assert n in A.SIGNATURES, f"{n} has no ctypes signature"
    assert set(A.SIGNATURES) == set(names)


def test_struct_layouts_match_reference_pods():
    # render/gpu_types.rs: NodeGpu 16, NodeRopesGpu 32, ChunkMetaGpu 48, CameraGpu 464, ClipmapGpu 528
    assert C.sizeof(A.Node) == 16
    assert C.sizeof(A.NodeRopes) == 32
    assert C.sizeof(A.ChunkMeta) == 48
    assert C.sizeof(A.CameraGpu) == 464
    assert C.sizeof(A.ClipmapGpu) == 528
    assert A.CameraGpu.profile_flags.offset == 400
    assert A.CameraGpu._pad0.offset == 416
    assert A.CameraGpu.render_present_px.offset == 384
    assert A.ClipmapGpu.offset.offset == 16 + 16 * 16


def test_camera_packing_is_consistent():
    from vxe.world import build_camera
    import numpy as np

    cam = build_camera((1.0, 2.0, 3.0), 0.3, -0.2, (64, 32), (32, 16), frame_index=5, time_s=0.5, jitter=False)
    assert cam.chunk_size == 64 and cam.max_steps == 128 and cam.frame_index == 5
    assert list(cam.voxel_params) == [np.float32(0.1), np.float32(0.5), 2.0, np.float32(0.002)]
    assert list(cam.render_present_px) == [32, 16, 64, 32]
    # ray through the image centre is the forward vector (yaw, pitch)
    r00 = np.array(cam.ray00[:3], dtype=np.float64)
    dx = np.array(cam.ray_dx[:3], dtype=np.float64)
    dy = np.array(cam.ray_dy[:3], dtype=np.float64)
    c = r00 + 15.5 * dx + 7.5 * dy
    c /= np.linalg.norm(c)
    f = np.array([np.sin(0.3) * np.cos(-0.2), np.sin(-0.2), np.cos(0.3) * np.cos(-0.2)])
    assert np.allclose(c, f, atol=1e-5)


def test_noalloc_argument_checks_return_before_any_device_call():
    """vxe_trace_primary_hits_noalloc validates its arguments on the host
    before it touches the CUDA runtime, so these calls need no GPU.  Every
    call here fails exactly one check; the device pointers are placeholders
    that the host code never dereferences, so no call may pass validation."""
    fake = 0x1000  # a non-null placeholder for a device buffer
    base_sv = dict(nodes=fake, ropes=fake, node_count=8, metas=fake, macro_words=fake, colinfo_words=fake,
                   chunk_capacity=4, grid_cells=8, grid=fake, clip_tex=fake, clip_layers=2, clip_res=64)

    def call(sv=None, size=(64, 48), chunk_size=64, chunk_count=2, grid_dims=(2, 2, 2), levels=2, res=64,
             hits=fake, null_scene=False):
        v = A.SceneView(**{**base_sv, **(sv or {})})
        cam = A.CameraGpu()
        cam.chunk_size, cam.chunk_count = chunk_size, chunk_count
        cam.render_present_px[0], cam.render_present_px[1] = size
        for k in range(3):
            cam.grid_dims[k] = grid_dims[k]
        clip = A.ClipmapGpu()
        clip.levels, clip.res = levels, res
        return A.lib().vxe_trace_primary_hits_noalloc(None if null_scene else C.byref(v), C.byref(cam),
                                                      C.byref(clip), hits, None)

    INVALID, CAPACITY = 1, 2
    assert call(null_scene=True) == INVALID
    assert call(hits=None) == INVALID
    assert call(sv=dict(nodes=None)) == INVALID
    assert call(sv=dict(node_count=0)) == INVALID
    assert call(sv=dict(grid_cells=0)) == INVALID
    assert call(chunk_size=32) == INVALID  # the column words assume 64^3 chunks
    assert call(size=(0, 48)) == INVALID
    # 4096 x 2304 internal is 512 x 288 tiles of 8x8, beyond the fixed scratch
    assert 512 * 288 > A.NOALLOC_MAX_TILES
    assert call(size=(4096, 2304)) == CAPACITY
    assert call(grid_dims=(2, 2, 3)) == CAPACITY  # 12 grid cells > 8
    assert call(chunk_count=5) == CAPACITY  # more chunks than slots
    assert call(levels=3) == INVALID  # more clipmap levels than layers
    assert call(res=32) == INVALID  # resolution differs from the texture's
    assert call(sv=dict(clip_tex=None)) == INVALID  # levels but no texture
