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
    # vxe_trace_primary_hits_noalloc validates its arguments before touching
    # the device (these calls need no GPU; the pointers are never read).
    lib = A.lib()
    fake = 256
    sv = A.SceneView(fake, fake, 100, fake, fake, fake, 4, 8, fake, None, 0, 0)
    clip = A.ClipmapGpu()
    cam = A.CameraGpu()
    cam.chunk_size = 64
    cam.chunk_count = 2
    cam.render_present_px[0], cam.render_present_px[1] = 64, 32
    cam.grid_dims[0], cam.grid_dims[1], cam.grid_dims[2] = 2, 2, 2

    def call(s=sv, c=cam, cl=clip, hits=fake):
        return lib.vxe_trace_primary_hits_noalloc(C.byref(s), C.byref(c), C.byref(cl), hits, None)

    def variant(**kw):
        c = A.CameraGpu()
        C.memmove(C.byref(c), C.byref(cam), C.sizeof(c))
        for k, v in kw.items():
            if isinstance(v, tuple):
                getattr(c, k)[:len(v)] = list(v)
            else:
                setattr(c, k, v)
        return c

    assert call(hits=None) == 1                                   # no output buffer
    assert call(c=variant(chunk_size=32)) == 1                    # colinfo layout needs 64
    assert call(c=variant(render_present_px=(0, 32))) == 1        # empty image
    assert call(c=variant(render_present_px=(4096, 2304))) == 2   # beyond VXE_NOALLOC_MAX_TILES
    assert call(c=variant(grid_dims=(4, 2, 2))) == 2              # more cells than the grid holds
    assert call(c=variant(chunk_count=5)) == 2                    # more chunks than the metas hold
    lv = A.ClipmapGpu()
    lv.levels, lv.res = 2, 256
    assert call(cl=lv) == 1                                       # clipmap levels without a texture
    nul = A.SceneView(*[getattr(sv, f) for f, _ in A.SceneView._fields_])
    nul.nodes = None
    assert call(s=nul) == 1                                       # missing scene buffer
