"""Build the native library of the B200 AA-fill backend (librrb.so).

nvcc compiles the CUDA kernels for sm_100a only (`-gencode
arch=compute_100a,code=sm_100a`) together with the host-side C ABI and the
path builder into one shared library placed next to this file, so it travels
with the source tree. The CUDA runtime is linked statically (nvcc's default),
so the library loads on a machine without a GPU.

The seeded scene generator of the benchmark and the tests is a separate
host-only library, scenes/librrb_scenes.so (g++), so that a process which only
generates workloads never maps the backend.
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

SOURCES = [CSRC / "rrb_backend.cu", CSRC / "rrb_static.cu", CSRC / "rrb_fills.cu", CSRC / "rrb_mlp.cu", CSRC / "rrb_features.cpp", CSRC / "rrb_encode.cpp", CSRC / "path_builder.cpp", CSRC / "rrb_server.cpp", CSRC / "rrb_stroke.cpp", CSRC / "rrb_clip.cu"]
DEPS = SOURCES + [CSRC / "rrb_kernels.cuh", CSRC / "rrb_device.cuh", CSRC / "rrb_hairline.cuh", CSRC / "rrb_stroke.h",
                  CSRC / "path_builder.h", CSRC / "rrb_device_scope.h", INCLUDE / "rrb.h"]

SCENES_DIR = ROOT / "scenes"
SCENES_LIB = SCENES_DIR / "librrb_scenes.so"
SCENES_SOURCES = [SCENES_DIR / "scene_gen.cpp", CSRC / "path_builder.cpp"]
SCENES_DEPS = SCENES_SOURCES + [CSRC / "path_builder.h", INCLUDE / "rrb.h", INCLUDE / "rrb_scenes.h"]
# Same host floating-point rules as the backend build (no contraction), and
# symbols bound inside the library so the backend's rrb_path_* never interpose.
SCENES_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-shared", "-Wl,-Bsymbolic"]

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


def needs_build(lib: Path = LIB, deps=DEPS) -> bool:
    if not lib.exists():
        return True
    t = lib.stat().st_mtime
    return any(p.stat().st_mtime > t for p in deps)


def build_scenes(force: bool = False, verbose: bool = False) -> Path:
    """Compile scenes/librrb_scenes.so (host only) if needed."""
    if not force and not needs_build(SCENES_LIB, SCENES_DEPS):
        return SCENES_LIB
    tmp = SCENES_LIB.with_suffix(".so.tmp")
    cmd = [os.environ.get("CXX", "g++"), *SCENES_FLAGS, "-I", str(INCLUDE), "-o", str(tmp), *map(str, SCENES_SOURCES)]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True, cwd=str(ROOT))
    os.replace(tmp, SCENES_LIB)
    return SCENES_LIB


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile librrb.so (and the scene library) if any source is newer (or force)."""
    build_scenes(force, verbose)
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
