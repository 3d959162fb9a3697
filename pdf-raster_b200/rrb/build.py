"""Build the native library of the B200 AA-fill backend (librrb.so).

nvcc compiles the CUDA kernels for sm_100a only (`-gencode
arch=compute_100a,code=sm_100a`) together with the host-side C ABI, the
path builder and the scene generator into one shared library placed next to
this file, so it travels with the source tree. The CUDA runtime is linked
statically (nvcc's default), so the library loads on a machine without a GPU.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
ROOT = PKG_DIR.parent
CSRC = ROOT / "csrc"
INCLUDE = ROOT.parent / "include"
LIB = PKG_DIR / "librrb.so"

SOURCES = [CSRC / "rrb_backend.cu", CSRC / "rrb_static.cu", CSRC / "rrb_fills.cu", CSRC / "rrb_mlp.cu", CSRC / "rrb_features.cpp", CSRC / "rrb_encode.cpp", CSRC / "path_scene.cpp", CSRC / "rrb_server.cpp", CSRC / "rrb_stroke.cpp", CSRC / "rrb_clip.cu"]
DEPS = SOURCES + [CSRC / "rrb_kernels.cuh", CSRC / "rrb_device.cuh", CSRC / "rrb_hairline.cuh", CSRC / "rrb_stroke.h", INCLUDE / "rrb.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC,-O3,-ffp-contract=off",
    "-Xptxas", "-O3",
    "-shared",
]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build librrb.so")


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(p.stat().st_mtime > t for p in DEPS)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile librrb.so if any source is newer than it (or force)."""
    if not force and not needs_build():
        return LIB
    cmd = [nvcc_path(), *NVCC_FLAGS, "-I", str(INCLUDE), "-o", str(LIB), *map(str, SOURCES)]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    tmp = LIB.with_suffix(".so.tmp")
    cmd[cmd.index(str(LIB))] = str(tmp)
    subprocess.run(cmd, check=True, cwd=str(ROOT))
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
