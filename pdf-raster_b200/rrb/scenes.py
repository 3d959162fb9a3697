"""The seeded synthetic workloads (include/rrb_scenes.h, librrb_scenes.so).

The generator lives in a host-only library of its own, so generating a scene
never maps the fill backend (librrb.so): the CPU baseline and the reference
arm of the benchmark build their inputs here and render with the oracle alone.

  kind 0  polygon page: 2,000 closed paths of 1-3 contours x 4-32 line/cubic
          segments on jittered circles, nonzero 70% / even-odd 30%, opaque;
  kind 1  glyph-dense text page: 150,000 quadratic glyphs on 60 baselines;
  kind 2  mixed pages of uneven size: {A4, Letter, A3} x {150, 300, 600} dpi,
          30% glyphs / 40% polygons / 30% axis-aligned rectangles, alpha
          32-255, log-normal path count per page (median 5,000, sigma 1.2).
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from ._abi import PathBatchParams

LIB_PATH = Path(__file__).resolve().parents[1] / "scenes" / "librrb_scenes.so"


class SceneParams(C.Structure):
    """rrb_scene_params; zero fields take each kind's defaults."""
    _fields_ = [
        ("kind", C.c_uint32),
        ("seed", C.c_uint64),
        ("n_pages", C.c_uint32),
        ("n_paths", C.c_uint32),
        ("page_w", C.c_uint32),
        ("page_h", C.c_uint32),
        ("page_scale", C.c_double),
        ("paths_scale", C.c_double),
        ("path_cap", C.c_uint32),
        ("reserved", C.c_uint32),
    ]


VP = C.c_void_p
SIGNATURES = {
    "rrb_scene_generate": (C.c_int, [C.POINTER(SceneParams), C.POINTER(VP)]),
    "rrb_scene_free": (None, [VP]),
    "rrb_scene_view": (None, [VP, C.POINTER(PathBatchParams)]),
    "rrb_scene_arena_bytes": (C.c_uint64, [VP]),
    "rrb_scene_counts": (None, [VP, C.POINTER(C.c_uint64)]),
}

_LIB = None


def use_library(path) -> None:
    """Generate scenes with another build of the same generator source (the
    CPU reference's copy under oracle/_build); call before the first scene."""
    global LIB_PATH
    path = Path(path).resolve()
    if _LIB is not None and path != LIB_PATH:
        raise RuntimeError(f"scene library already loaded from {LIB_PATH}")
    LIB_PATH = path


def lib() -> C.CDLL:
    """Load librrb_scenes.so (building it if needed) and declare its signatures."""
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            from . import build
            build.build_scenes()
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


class Scene:
    """A seeded synthetic workload (kind 0 polygons, 1 glyphs, 2 mixed pages).

    Arrays are numpy views of the generator's memory (valid while the Scene lives).
    """

    def __init__(self, kind: int, seed: int = 0, **kw):
        p = SceneParams(kind=kind, seed=seed)
        for k, v in kw.items():
            setattr(p, k, v)
        h = C.c_void_p()
        rc = lib().rrb_scene_generate(C.byref(p), C.byref(h))
        if rc:
            raise ValueError(f"scene generation failed (status {rc}): unknown kind {kind}")
        self._h = h.value
        self.view = PathBatchParams()
        lib().rrb_scene_view(self._h, C.byref(self.view))
        v = self.view
        self.n_paths = int(v.n_paths)
        self.n_pts = int(v.n_pts)
        self.n_pages = int(v.n_pages)
        asa = np.ctypeslib.as_array
        self.pts = asa(v.pts, shape=(self.n_pts * 2,)).reshape(self.n_pts, 2) if self.n_pts else np.zeros((0, 2))
        self.flags = asa(v.flags, shape=(self.n_pts,)) if self.n_pts else np.zeros(0, np.uint8)
        self.path_pt_off = asa(v.path_pt_off, shape=(self.n_paths + 1,))
        self.fill_rule = asa(v.fill_rule, shape=(self.n_paths,))
        self.gray = asa(v.gray, shape=(self.n_paths,))
        self.alpha = asa(v.alpha, shape=(self.n_paths,))
        self.path_page = asa(v.path_page, shape=(self.n_paths,))
        self.page_width = asa(v.page_width, shape=(self.n_pages,))
        self.page_height = asa(v.page_height, shape=(self.n_pages,))
        self.page_offset = asa(v.page_offset, shape=(self.n_pages,))
        self.arena_bytes = int(lib().rrb_scene_arena_bytes(self._h))
        cnt = (C.c_uint64 * 3)()
        lib().rrb_scene_counts(self._h, cnt)
        self.n_lines, self.n_cubics = int(cnt[0]), int(cnt[1])

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h and _LIB is not None:
            _LIB.rrb_scene_free(h)

    @property
    def pixels(self) -> int:
        return int(np.sum(self.page_width.astype(np.int64) * self.page_height.astype(np.int64)))

    def blank_arena(self, value: int = 255) -> np.ndarray:
        """Host page arena initialised to `value` (white pages)."""
        return np.full(self.arena_bytes, value, dtype=np.uint8)

    def page(self, arena: np.ndarray, i: int) -> np.ndarray:
        o, w, h = int(self.page_offset[i]), int(self.page_width[i]), int(self.page_height[i])
        return arena[o:o + w * h].reshape(h, w)
