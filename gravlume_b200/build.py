"""In-tree build of libglc.so (sm_100a) with nvcc.

The library is the product: CUDA kernels plus the extern "C" boundary declared in include/glc.h.
It is built into gravlume_b200/_lib/ so that it ships with the source tree.
"""

from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB_DIR = PKG / "_lib"
LIB_PATH = LIB_DIR / "libglc.so"
# the nvcc flags and sources the library was last built with; a change of either rebuilds it
STAMP_PATH = LIB_DIR / "libglc.build"

SOURCES = ["glc_api.cu", "glc_static_scratch.cu", "glc_adjoint.cu", "glc_scene.cpp", "glc_flops.cpp"]
HEADERS = ["glc_geometry.cuh", "glc_dp54.cuh", "glc_tracer.cuh", "glc_kernels.cuh", "glc_certificate.cuh", "glc_escape_map.cuh", "glc_shadow.cuh", "glc_footprint.cuh",
           "glc_dual.cuh", "glc_adjoint.cuh", "glc_radiation.cuh", "glc_internal.h", "glc_context.h"]

# -prec-div=false / -prec-sqrt=false: binary32 division and square root by the approximate
# hardware sequences (a couple of ulp) rather than the correctly rounded ones, which the binary32
# stepping loop executes on every right-hand side (FP32 about 1.35x faster). Binary64 arithmetic
# and the directed-rounding intrinsics of the capture certificates are not affected; denormals are
# kept (no -ftz), so the certificates' upward-rounded bounds stay sound.
NVCC_FLAGS = [
    "-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
    "-prec-div=false", "-prec-sqrt=false",
    "-Xcompiler", "-fPIC", "-shared",
]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libglc")
    return cand


def _stamp() -> str:
    return " ".join(NVCC_FLAGS + SOURCES)


def _stale() -> bool:
    if not LIB_PATH.exists():
        return True
    if not STAMP_PATH.exists() or STAMP_PATH.read_text() != _stamp():
        return True
    t = LIB_PATH.stat().st_mtime
    deps = [CSRC / s for s in SOURCES + HEADERS] + [ROOT / "include" / "glc.h"]
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not _stale():
        return LIB_PATH
    LIB_DIR.mkdir(parents=True, exist_ok=True)
    tmp = LIB_PATH.with_suffix(".so.tmp")
    cmd = [nvcc(), *NVCC_FLAGS, *(["-Xptxas", "-v"] if verbose else []), "-o", str(tmp),
           *[str(CSRC / s) for s in SOURCES], "-lcudart"]
    subprocess.run(cmd, check=True, cwd=str(CSRC))
    os.replace(tmp, LIB_PATH)
    STAMP_PATH.write_text(_stamp())
    return LIB_PATH


if __name__ == "__main__":
    print(build(force=True, verbose=True))
