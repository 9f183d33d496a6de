"""Builds the in-tree shared libraries.

* ``vxe/libvxe.so`` -- the product: sm_100a CUDA passes + C ABI + C++
  producers, compiled with ``-fmad=false -prec-div=true -prec-sqrt=true`` so
  every float operation is a single IEEE binary32 op; reads of the world's
  records at data-derived indices are clamped into their buffers.
* ``vxe/libvxe_checked.so`` -- the same with device bounds checks: an index
  outside its buffer reads a zero record and sets the context's error word.
* ``oracle/liboracle_vxe.so`` -- the CPU restatement used by tests and the
  CPU baseline (``-ffp-contract=off``, no fast math).
* ``oracle/libref_producer.so`` -- the host-side producers (chunk builder,
  camera packing, clipmap state: ``csrc/host/producer.cpp``) built by g++
  alone, so that the CPU timing of the reference path maps no CUDA library.

Both are rebuilt only when a source is newer than the library.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
REPO = PKG.parent
INCLUDE = REPO / "include"
CSRC = PKG / "csrc"
LIB = PKG / "vxe" / "libvxe.so"
LIB_CHECKED = PKG / "vxe" / "libvxe_checked.so"
ORACLE_SRC = REPO / "oracle" / "vxe_oracle.cpp"
ORACLE_LIB = REPO / "oracle" / "liboracle_vxe.so"
REF_PRODUCER_LIB = REPO / "oracle" / "libref_producer.so"
# The reference's pure shading helpers, translated from its WGSL where it lies
# (only in a checkout that has the reference; the GPU box does not) into a
# git-ignored library that pins the oracle (tests/test_oracle_wgsl_pin.py).
REF_SHADERS = Path("/root/reference/src/shaders")
REF_WGSL_DIR = REPO / "oracle" / "_ref"
REF_WGSL_LIB = REF_WGSL_DIR / "libref_wgsl.so"
BUILD_DIR = PKG / "_build"

ARCH = "-gencode=arch=compute_100a,code=sm_100a"
NVCC_FLAGS = [
    "-O3", "-std=c++17", ARCH, "-lineinfo",
    "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
    f"-I{INCLUDE}", f"-I{CSRC}",
]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall", f"-I{INCLUDE}"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libvxe.so")
    return cand


def _sources():
    cu = sorted(CSRC.glob("*.cu"))
    cpp = sorted((CSRC / "host").glob("*.cpp"))
    headers = sorted(CSRC.rglob("*.cuh")) + sorted(CSRC.rglob("*.h")) + sorted(INCLUDE.rglob("*.h"))
    return cu, cpp, headers


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(str(c) for c in cmd), flush=True)
    r = subprocess.run([str(c) for c in cmd], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed ({r.returncode}):\n{' '.join(map(str, cmd))}\n{r.stdout}\n{r.stderr}")
    return r


def build_lib(verbose: bool = False, force: bool = False, ptxas_verbose: bool = False, checked: bool = False) -> Path:
    target = LIB_CHECKED if checked else LIB
    cu, cpp, headers = _sources()
    if not force and not _stale(target, cu + cpp + headers + [Path(__file__)]):
        return target
    bdir = BUILD_DIR / ("checked" if checked else "fast")
    bdir.mkdir(parents=True, exist_ok=True)
    nvcc = _nvcc()
    objs = []
    for src in cu:
        obj = bdir / (src.stem + ".o")
        extra = ["-Xptxas", "-v"] if ptxas_verbose else []
        r = _run([nvcc, *NVCC_FLAGS, f"-DVXE_DEVICE_CHECKS={1 if checked else 0}", *extra, "-c", src, "-o", obj],
                 verbose)
        if ptxas_verbose:
            print(r.stderr)
        objs.append(obj)
    for src in cpp:
        obj = bdir / (src.stem + ".o")
        _run(["g++", *CXX_FLAGS, "-c", src, "-o", obj], verbose)
        objs.append(obj)
    tmp = target.with_suffix(".so.tmp")
    _run([nvcc, ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs], verbose)
    os.replace(tmp, target)
    return target


def build_oracle(verbose: bool = False, force: bool = False) -> Path:
    deps = [ORACLE_SRC, INCLUDE / "vxe" / "detmath.h", INCLUDE / "vxe" / "vxe.h"]
    if not force and not _stale(ORACLE_LIB, deps):
        return ORACLE_LIB
    tmp = ORACLE_LIB.with_suffix(".so.tmp")
    _run(["g++", *CXX_FLAGS, "-shared", "-o", tmp, ORACLE_SRC, "-lpthread"], verbose)
    os.replace(tmp, ORACLE_LIB)
    return ORACLE_LIB


def build_ref_producer(verbose: bool = False, force: bool = False) -> Path:
    src = CSRC / "host" / "producer.cpp"
    deps = [src, CSRC / "common" / "terrain_noise.h", INCLUDE / "vxe" / "vxe.h", INCLUDE / "vxe" / "detmath.h"]
    if not force and not _stale(REF_PRODUCER_LIB, deps):
        return REF_PRODUCER_LIB
    tmp = REF_PRODUCER_LIB.with_suffix(".so.tmp")
    _run(["g++", *CXX_FLAGS, "-shared", "-o", tmp, src, "-lpthread"], verbose)
    os.replace(tmp, REF_PRODUCER_LIB)
    return REF_PRODUCER_LIB


def build_ref_wgsl(verbose: bool = False, force: bool = False):
    """oracle/_ref/libref_wgsl.so from the reference's WGSL (oracle/wgsl_to_cpp.py); None without the reference."""
    if not REF_SHADERS.is_dir():
        return None
    translator = REPO / "oracle" / "wgsl_to_cpp.py"
    shim = REPO / "oracle" / "wgsl_shim.h"
    wgsl = sorted(REF_SHADERS.rglob("*.wgsl"))
    deps = [translator, shim, INCLUDE / "vxe" / "detmath.h", *wgsl]
    if not force and not _stale(REF_WGSL_LIB, deps):
        return REF_WGSL_LIB
    cpp = REF_WGSL_DIR / "ref_wgsl.cpp"
    _run([sys.executable, translator, REF_SHADERS, cpp], verbose)
    tmp = REF_WGSL_LIB.with_suffix(".so.tmp")
    # -O3: the reference arm of the bench times this library, so it gets the
    # faster build (still no FMA contraction or fast math: the pin is bit-exact)
    _run(["g++", *CXX_FLAGS, "-O3", f"-I{REPO / 'oracle'}", "-shared", "-o", tmp, cpp, "-lpthread"], verbose)
    os.replace(tmp, REF_WGSL_LIB)
    return REF_WGSL_LIB


def build_all(verbose: bool = False, force: bool = False) -> None:
    build_lib(verbose=verbose, force=force)
    build_lib(verbose=verbose, force=force, checked=True)
    build_oracle(verbose=verbose, force=force)
    build_ref_producer(verbose=verbose, force=force)
    build_ref_wgsl(verbose=verbose, force=force)


if __name__ == "__main__":
    build_all(verbose=True, force="--force" in sys.argv)
    if "--ptxas" in sys.argv:
        build_lib(verbose=True, force=True, ptxas_verbose=True)
