"""ctypes binding of the CPU oracle (oracle/rr_oracle.{h,cpp}).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline / reference legs of bench.py, never by the product package.
`build()` compiles it with oracle/Makefile into oracle/_build/.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "librr_oracle.so"
# The workload generator built from the package's scene source into oracle/_build
# (oracle/Makefile), for the timed CPU reference: it then maps oracle/ libraries only.
SCENES_LIB_PATH = HERE / "_build" / "librr_scenes.so"

ROWMAP_DOCUMENTED = 0
ROWMAP_AS_SHIPPED = 1


class Seg(C.Structure):
    _fields_ = [("x0", C.c_double), ("y0", C.c_double), ("x1", C.c_double), ("y1", C.c_double),
                ("dxdy", C.c_double), ("dxdy_fp", C.c_int32), ("flags", C.c_uint32)]


class Intersect(C.Structure):
    _fields_ = [("x0", C.c_int32), ("x1", C.c_int32), ("count", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("paths", "segments", "aa_rows", "intersects", "unpinned_tie_rows",
                                          "nonterminating_rows")]

    def as_dict(self):
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


XF_HORIZ, XF_VERT, XF_FLIPPED = 1, 2, 4
PF_FIRST, PF_LAST, PF_CLOSED, PF_CURVE = 1, 2, 4, 8
IDENTITY = (1.0, 0.0, 0.0, 1.0, 0.0, 0.0)

_LIB = None

CAP_BUTT, CAP_ROUND, CAP_PROJECTING = 0, 1, 2
JOIN_MITER, JOIN_ROUND, JOIN_BEVEL = 0, 1, 2


class StrokeParams(C.Structure):
    """or_stroke_params: StrokeParams (stroke/mod.rs:29-48), stroke_adjust off."""
    _fields_ = [("line_width", C.c_double), ("miter_limit", C.c_double), ("dash_phase", C.c_double),
                ("dash", C.POINTER(C.c_double)), ("n_dash", C.c_int32), ("line_cap", C.c_int32),
                ("line_join", C.c_int32), ("stroke", C.c_int32)]


def build(arch: str | None = None) -> Path:
    """Compile the oracle if needed. `arch` overrides -march (default x86-64-v3, portable to any AVX2 host)."""
    srcs = [HERE / n for n in ("rr_oracle.cpp", "rr_oracle.h", "fill_oracle.cpp", "fill_oracle.h", "Makefile")]
    scene_srcs = [HERE.parent / "pdf-raster_b200" / "scenes" / "scene_gen.cpp",
                  HERE.parent / "pdf-raster_b200" / "csrc" / "path_builder.cpp",
                  HERE.parent / "pdf-raster_b200" / "csrc" / "path_builder.h",
                  HERE.parent / "include" / "rrb.h", HERE.parent / "include" / "rrb_scenes.h"]
    newest = max(p.stat().st_mtime for p in srcs + [q for q in scene_srcs if q.exists()])
    if all(x.exists() and x.stat().st_mtime >= newest for x in (LIB_PATH, SCENES_LIB_PATH)):
        return LIB_PATH
    env = dict(os.environ)
    cmd = ["make", "-C", str(HERE), f"ARCHFLAGS=-march={arch or 'x86-64-v3'}"]
    subprocess.run(cmd, check=True, env=env, stdout=subprocess.DEVNULL)
    return LIB_PATH


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        D, I32, U8, I64, VP = C.c_double, C.c_int32, C.c_uint8, C.c_int64, C.c_void_p
        sig = {
            "or_path_new": (VP, []), "or_path_free": (None, [VP]),
            "or_path_move_to": (C.c_int, [VP, D, D]), "or_path_line_to": (C.c_int, [VP, D, D]),
            "or_path_curve_to": (C.c_int, [VP, D, D, D, D, D, D]), "or_path_close": (C.c_int, [VP, C.c_int]),
            "or_path_len": (I64, [VP]), "or_path_pts": (C.POINTER(D), [VP]), "or_path_flags": (C.POINTER(U8), [VP]),
            "or_conic_to_cubic": (None, [D] * 6 + [C.POINTER(D)]),
            "or_transform": (None, [C.POINTER(D), D, D, C.POINTER(D)]),
            "or_flatten_curve": (I32, [C.POINTER(D), D, C.POINTER(D), I32]),
            "or_add_segment": (None, [D, D, D, D, C.POINTER(Seg)]),
            "or_xpath_new": (I64, [C.POINTER(D), C.POINTER(U8), I64, C.POINTER(D), D, C.c_int, C.POINTER(Seg), I64]),
            "or_xpath_aa_scale": (None, [C.POINTER(Seg), I64]),
            "or_scanner_new": (VP, [C.POINTER(Seg), I64, C.c_int, I32, I32, C.POINTER(Stats)]),
            "or_scanner_free": (None, [VP]),
            "or_scanner_bounds": (None, [VP, C.POINTER(I32)]),
            "or_scanner_row": (I64, [VP, I32, C.POINTER(Intersect), I64]),
            "or_scanner_test": (C.c_int, [VP, I32, I32]),
            "or_count_crossings": (None, [C.POINTER(Intersect), I64, I32, C.POINTER(I32)]),
            "or_add_intersection": (I64, [C.POINTER(Intersect), I64, I32, I32, I32]),
            "or_render_aa_line": (None, [VP, C.POINTER(U8), I64, I32, C.POINTER(I32), C.POINTER(Stats)]),
            "or_aabuf_set_span": (None, [C.POINTER(U8), I64, I64, I64, I64]),
            "or_aa_coverage_span": (None, [C.POINTER(U8), I64, I64, C.POINTER(U8), I64]),
            "or_aa_coverage_span_tier": (None, [C.POINTER(U8), I64, I64, C.POINTER(U8), I64, C.c_int]),
            "or_coverage_tier": (C.c_int, []),
            "or_aa_gamma": (C.POINTER(U8), []),
            "or_div255": (U8, [C.c_uint32]),
            "or_render_span_aa_gray": (None, [C.POINTER(U8), C.POINTER(U8), I64, U8, U8]),
            "or_composite_aa_rgb8_opaque": (None, [C.POINTER(U8), C.POINTER(U8), U8, C.POINTER(U8), I64]),
            "or_rgb_to_gray": (None, [C.POINTER(U8), C.POINTER(U8), I64]),
            "or_fill_path": (None, [C.POINTER(U8), I32, I32, C.POINTER(D), C.POINTER(U8), I64, C.POINTER(D), D,
                                    C.c_int, U8, U8, C.c_int, C.POINTER(Stats)]),
            "or_fill_path_clip_paths": (None, [C.POINTER(U8), I32, I32, C.POINTER(D), C.POINTER(U8), I64,
                                               C.POINTER(D), D, C.c_int, U8, U8, C.c_int, C.POINTER(D), I64,
                                               C.POINTER(C.POINTER(D)), C.POINTER(C.POINTER(U8)), C.POINTER(I64),
                                               C.POINTER(C.c_int), C.POINTER(Stats)]),
            "or_fill_path_clip_path": (None, [C.POINTER(U8), I32, I32, C.POINTER(D), C.POINTER(U8), I64, C.POINTER(D),
                                              D, C.c_int, U8, U8, C.c_int, C.POINTER(D), C.POINTER(D), C.POINTER(U8),
                                              I64, C.c_int, C.POINTER(Stats)]),
            "or_render_scene": (None, [C.POINTER(U8), C.POINTER(C.c_uint64), C.POINTER(C.c_uint32),
                                       C.POINTER(C.c_uint32), C.c_uint32, C.POINTER(D), C.POINTER(U8),
                                       C.POINTER(C.c_uint64), C.POINTER(U8), C.POINTER(U8), C.POINTER(U8),
                                       C.POINTER(C.c_uint32), C.c_uint64, C.POINTER(D), D, C.c_int, C.c_int,
                                       C.POINTER(Stats)]),
            "or_render_scene_rgb": (None, [C.POINTER(U8), C.POINTER(C.c_uint64), C.POINTER(C.c_uint32),
                                           C.POINTER(C.c_uint32), C.c_uint32, C.POINTER(D), C.POINTER(U8),
                                           C.POINTER(C.c_uint64), C.POINTER(U8), C.POINTER(U8), C.POINTER(U8),
                                           C.POINTER(C.c_uint32), C.c_uint64, C.POINTER(D), D, C.c_int, C.c_int,
                                           C.POINTER(Stats)]),
            "or_render_scene_ex": (None, [C.POINTER(U8), C.POINTER(C.c_uint64), C.POINTER(C.c_uint32),
                                          C.POINTER(C.c_uint32), C.c_uint32, C.POINTER(D), C.POINTER(U8),
                                          C.POINTER(C.c_uint64), C.POINTER(U8), C.POINTER(U8), C.POINTER(U8),
                                          C.POINTER(U8), C.POINTER(C.c_uint32), C.c_uint64, C.POINTER(D),
                                          C.POINTER(D), D, C.c_int, C.c_int, C.POINTER(Stats)]),
            "or_stroke_flatten": (C.c_int, [C.POINTER(D), C.POINTER(U8), I64, D, VP]),
            "or_stroke_dash": (C.c_int, [C.POINTER(D), C.POINTER(U8), I64, C.POINTER(D), I32, D, VP]),
            "or_stroke_outline": (C.c_int, [C.POINTER(D), C.POINTER(U8), I64, C.POINTER(StrokeParams), D, VP]),
            "or_render_scene_paint": (None, [C.POINTER(U8), C.POINTER(C.c_uint64), C.POINTER(C.c_uint32),
                                             C.POINTER(C.c_uint32), C.c_uint32, C.POINTER(D), C.POINTER(U8),
                                             C.POINTER(C.c_uint64), C.POINTER(U8), C.POINTER(U8), C.POINTER(U8),
                                             C.POINTER(U8), C.POINTER(C.c_uint32), C.c_uint64, C.POINTER(D),
                                             C.POINTER(StrokeParams), C.POINTER(D), D, C.c_int, C.c_int,
                                             C.POINTER(Stats)]),
            "or_aa_jitter": (None, [C.POINTER(C.c_float), C.POINTER(C.c_float)]),
            "or_aa_fill_cpu": (None, [C.POINTER(C.c_float), C.c_uint32, C.c_float, C.c_float, C.c_uint32,
                                      C.c_uint32, C.c_int, C.POINTER(U8)]),
            "or_build_tile_records": (I64, [C.POINTER(C.c_float), C.c_uint32, C.c_float, C.c_float, C.c_uint32,
                                            C.c_uint32, VP, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                            C.POINTER(C.c_uint32)]),
            "or_tile_fill": (None, [VP, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.c_uint32, C.c_uint32,
                                    C.c_uint32, C.c_int, C.POINTER(U8)]),
        }
        for n, (r, a) in sig.items():
            f = getattr(L, n)
            f.restype, f.argtypes = r, a
        _LIB = L
    return _LIB


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def _mat(m):
    return (C.c_double * 6)(*m)


# ---- A1/A2 --------------------------------------------------------------------
class OraclePath:
    """PathBuilder restatement; build() returns (pts[n,2], flags[n])."""

    def __init__(self):
        self.h = lib().or_path_new()

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_path_free(self.h)
            self.h = None

    def move_to(self, x, y):
        return lib().or_path_move_to(self.h, x, y)

    def line_to(self, x, y):
        return lib().or_path_line_to(self.h, x, y)

    def curve_to(self, *a):
        return lib().or_path_curve_to(self.h, *a)

    def close(self, force=False):
        return lib().or_path_close(self.h, int(force))

    def build(self):
        n = lib().or_path_len(self.h)
        if n == 0:
            return np.zeros((0, 2)), np.zeros(0, np.uint8)
        pts = np.ctypeslib.as_array(lib().or_path_pts(self.h), shape=(n * 2,)).reshape(n, 2).copy()
        return pts, np.ctypeslib.as_array(lib().or_path_flags(self.h), shape=(n,)).copy()


def conic_to_cubic(p0, pc, p3):
    o = (C.c_double * 4)()
    lib().or_conic_to_cubic(p0[0], p0[1], pc[0], pc[1], p3[0], p3[1], o)
    return (o[0], o[1]), (o[2], o[3])


# ---- A3-A6 -----------------------------------------------------------------------
def transform(m, x, y):
    o = (C.c_double * 2)()
    lib().or_transform(_mat(m), x, y, o)
    return o[0], o[1]


def flatten_curve(p0, p1, p2, p3, flatness_sq):
    cp = (C.c_double * 8)(*p0, *p1, *p2, *p3)
    out = np.zeros(2 * 1025, np.float64)
    n = lib().or_flatten_curve(cp, flatness_sq, _p(out, C.c_double), 1025)
    return out[: 2 * n].reshape(n, 2)


def add_segment(x0, y0, x1, y1) -> Seg:
    s = Seg()
    lib().or_add_segment(x0, y0, x1, y1, C.byref(s))
    return s


def xpath_new(pts, flags, matrix=IDENTITY, flatness=0.1, close=True, aa_scale=False):
    pts = np.ascontiguousarray(pts, np.float64).reshape(-1)
    flags = np.ascontiguousarray(flags, np.uint8)
    n = flags.size
    need = lib().or_xpath_new(_p(pts, C.c_double), _p(flags, C.c_uint8), n, _mat(matrix), flatness, int(close),
                              None, 0)
    segs = (Seg * max(1, need))()
    lib().or_xpath_new(_p(pts, C.c_double), _p(flags, C.c_uint8), n, _mat(matrix), flatness, int(close), segs, need)
    if aa_scale:
        lib().or_xpath_aa_scale(segs, need)
    return list(segs)[:need]


# ---- A7/A8 -----------------------------------------------------------------------
class Scanner:
    def __init__(self, segs, eo=False, clip_y_min=0, clip_y_max=1 << 20):
        arr = (Seg * max(1, len(segs)))(*segs)
        self.stats = Stats()
        self.h = lib().or_scanner_new(arr, len(segs), int(eo), clip_y_min, clip_y_max, C.byref(self.stats))

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_scanner_free(self.h)
            self.h = None

    def bounds(self):
        o = (C.c_int32 * 5)()
        lib().or_scanner_bounds(self.h, o)
        return dict(y_min=o[0], y_max=o[1], x_min=o[2], x_max=o[3], empty=bool(o[4]))

    def row(self, y):
        n = lib().or_scanner_row(self.h, y, None, 0)
        buf = (Intersect * max(1, n))()
        lib().or_scanner_row(self.h, y, buf, n)
        return [(b.x0, b.x1, b.count) for b in list(buf)[:n]]

    def test(self, x, y) -> bool:
        return bool(lib().or_scanner_test(self.h, x, y))

    def render_aa_line(self, aa_width, y):
        rb = (aa_width + 7) // 8
        buf = np.zeros(rb * 4, np.uint8)
        o = (C.c_int32 * 2)()
        st = Stats()
        lib().or_render_aa_line(self.h, _p(buf, C.c_uint8), aa_width, y, o, C.byref(st))
        return buf.reshape(4, rb), (o[0], o[1]), st


def count_crossings(row, x):
    arr = (Intersect * max(1, len(row)))(*[Intersect(*r) for r in row])
    o = (C.c_int32 * 2)()
    lib().or_count_crossings(arr, len(row), x, o)
    return o[0], bool(o[1])


def add_intersection(row, x0, x1, count):
    arr = (Intersect * (len(row) + 1))(*[Intersect(*r) for r in row])
    n = lib().or_add_intersection(arr, len(row), x0, x1, count)
    return [(a.x0, a.x1, a.count) for a in list(arr)[:n]]


def aabuf_set_span(buf, width, row, x0, x1):
    lib().or_aabuf_set_span(_p(buf, C.c_uint8), width, row, x0, x1)


# ---- A10-A12 -----------------------------------------------------------------------
def aa_coverage_span(rows4: np.ndarray, x0: int, n: int) -> np.ndarray:
    rows4 = np.ascontiguousarray(rows4, np.uint8)
    out = np.zeros(n, np.uint8)
    lib().or_aa_coverage_span(_p(rows4, C.c_uint8), rows4.shape[1], x0, _p(out, C.c_uint8), n)
    return out


def coverage_tier() -> int:
    """The coverage tier the oracle dispatches to on this host: 2 AVX-512 BITALG, 1 AVX2, 0 scalar."""
    return int(lib().or_coverage_tier())


def aa_coverage_span_tier(rows4: np.ndarray, x0: int, n: int, tier: int) -> np.ndarray:
    """aa_coverage_span through one tier (0 scalar, 1 AVX2, 2 AVX-512 BITALG; capped at the host's best)."""
    rows4 = np.ascontiguousarray(rows4, np.uint8)
    out = np.zeros(n, np.uint8)
    lib().or_aa_coverage_span_tier(_p(rows4, C.c_uint8), rows4.shape[1], x0, _p(out, C.c_uint8), n, tier)
    return out


def aa_gamma():
    g = lib().or_aa_gamma()
    return [g[i] for i in range(17)]


def div255(x: int) -> int:
    return int(lib().or_div255(x))


def render_span_aa_gray(dst: np.ndarray, shape: np.ndarray, a_input: int, gray: int):
    shape = np.ascontiguousarray(shape, np.uint8)
    lib().or_render_span_aa_gray(_p(dst, C.c_uint8), _p(shape, C.c_uint8), shape.size, a_input, gray)


def composite_aa_rgb8_opaque(dst: np.ndarray, src, a_input: int, shape: np.ndarray):
    s = np.asarray(src, np.uint8)
    shape = np.ascontiguousarray(shape, np.uint8)
    lib().or_composite_aa_rgb8_opaque(_p(dst, C.c_uint8), _p(s, C.c_uint8), a_input, _p(shape, C.c_uint8), shape.size)


def rgb_to_gray(rgb: np.ndarray) -> np.ndarray:
    rgb = np.ascontiguousarray(rgb, np.uint8)
    out = np.zeros(rgb.size // 3, np.uint8)
    lib().or_rgb_to_gray(_p(rgb, C.c_uint8), _p(out, C.c_uint8), out.size)
    return out


# ---- A9 + scenes -----------------------------------------------------------------
def fill_path(page: np.ndarray, pts, flags, eo=False, gray=0, alpha=255, rowmap=ROWMAP_DOCUMENTED, matrix=IDENTITY,
              flatness=0.1) -> dict:
    """fill_impl on a (H, W) u8 page in place; returns the oracle counters."""
    assert page.dtype == np.uint8 and page.flags["C_CONTIGUOUS"] and page.ndim == 2
    pts = np.ascontiguousarray(pts, np.float64).reshape(-1)
    flags = np.ascontiguousarray(flags, np.uint8)
    st = Stats()
    lib().or_fill_path(_p(page, C.c_uint8), page.shape[1], page.shape[0], _p(pts, C.c_double),
                       _p(flags, C.c_uint8), flags.size, _mat(matrix), flatness, int(eo), gray, alpha, rowmap,
                       C.byref(st))
    return st.as_dict()


def fill_path_clip_path(page: np.ndarray, pts, flags, clip_pts, clip_flags, clip_eo=False, eo=False, gray=0,
                        alpha=255, rowmap=ROWMAP_DOCUMENTED, clip_rect=None, matrix=IDENTITY, flatness=0.1) -> dict:
    """fill_impl on a (H, W) u8 page in place under the page clip, clip_to_rect(clip_rect) when given, and
    clip_to_path of (clip_pts, clip_flags) with rule clip_eo, as the renderer clips (XPath without aa_scale)."""
    assert page.dtype == np.uint8 and page.flags["C_CONTIGUOUS"] and page.ndim == 2
    pts = np.ascontiguousarray(pts, np.float64).reshape(-1)
    flags = np.ascontiguousarray(flags, np.uint8)
    cpts = np.ascontiguousarray(clip_pts, np.float64).reshape(-1)
    cfl = np.ascontiguousarray(clip_flags, np.uint8)
    rect = None if clip_rect is None else np.ascontiguousarray(clip_rect, np.float64).reshape(4)
    st = Stats()
    lib().or_fill_path_clip_path(_p(page, C.c_uint8), page.shape[1], page.shape[0], _p(pts, C.c_double),
                                 _p(flags, C.c_uint8), flags.size, _mat(matrix), flatness, int(eo), gray, alpha, rowmap,
                                 None if rect is None else _p(rect, C.c_double), _p(cpts, C.c_double),
                                 _p(cfl, C.c_uint8), cfl.size, int(clip_eo), C.byref(st))
    return st.as_dict()


def fill_path_clip_paths(page: np.ndarray, pts, flags, clips, eo=False, gray=0, alpha=255,
                         rowmap=ROWMAP_DOCUMENTED, clip_rect=None, matrix=IDENTITY, flatness=0.1) -> dict:
    """fill_path_clip_path under a stack of clip paths: clips = [(pts, flags, even_odd), ...], applied in order."""
    assert page.dtype == np.uint8 and page.flags["C_CONTIGUOUS"] and page.ndim == 2
    pts = np.ascontiguousarray(pts, np.float64).reshape(-1)
    flags = np.ascontiguousarray(flags, np.uint8)
    cp = [np.ascontiguousarray(c[0], np.float64).reshape(-1) for c in clips]
    cf = [np.ascontiguousarray(c[1], np.uint8) for c in clips]
    n = len(clips)
    pp = (C.POINTER(C.c_double) * max(1, n))(*[_p(a, C.c_double) for a in cp])
    fp = (C.POINTER(C.c_uint8) * max(1, n))(*[_p(a, C.c_uint8) for a in cf])
    ns = (C.c_int64 * max(1, n))(*[a.size for a in cf])
    eos = (C.c_int * max(1, n))(*[int(bool(c[2])) for c in clips])
    rect = None if clip_rect is None else np.ascontiguousarray(clip_rect, np.float64).reshape(4)
    st = Stats()
    lib().or_fill_path_clip_paths(_p(page, C.c_uint8), page.shape[1], page.shape[0], _p(pts, C.c_double),
                                  _p(flags, C.c_uint8), flags.size, _mat(matrix), flatness, int(eo), gray, alpha,
                                  rowmap, None if rect is None else _p(rect, C.c_double), n, pp, fp, ns, eos,
                                  C.byref(st))
    return st.as_dict()


def render_arrays(arena, page_offset, page_width, page_height, pts, flags, path_pt_off, fill_rule, gray, alpha,
                  path_page, rowmap=ROWMAP_DOCUMENTED, threads=1, matrix=IDENTITY, flatness=0.1) -> dict:
    """Render every path in order onto an arena of pages (in place)."""
    a = [np.ascontiguousarray(x, t) for x, t in (
        (page_offset, np.uint64), (page_width, np.uint32), (page_height, np.uint32),
        (np.reshape(pts, -1), np.float64), (flags, np.uint8), (path_pt_off, np.uint64), (fill_rule, np.uint8),
        (gray, np.uint8), (alpha, np.uint8), (path_page, np.uint32))]
    st = Stats()
    lib().or_render_scene(_p(arena, C.c_uint8), _p(a[0], C.c_uint64), _p(a[1], C.c_uint32), _p(a[2], C.c_uint32),
                          a[1].size, _p(a[3], C.c_double), _p(a[4], C.c_uint8), _p(a[5], C.c_uint64),
                          _p(a[6], C.c_uint8), _p(a[7], C.c_uint8), _p(a[8], C.c_uint8), _p(a[9], C.c_uint32),
                          a[6].size, _mat(matrix), flatness, rowmap, threads, C.byref(st))
    return st.as_dict()


def render_scene_rgb(scene, arena: np.ndarray, rgb: np.ndarray, rowmap=ROWMAP_DOCUMENTED, threads=1,
                     page_offset=None) -> dict:
    """The scene on Rgb8 pages (A12): `arena` holds 3 bytes per pixel at
    `page_offset` (default: 3 x the scene's), path p painted with rgb[p]."""
    po = np.ascontiguousarray(3 * scene.page_offset.astype(np.uint64) if page_offset is None else page_offset,
                              np.uint64)
    a = [np.ascontiguousarray(x, t) for x, t in (
        (scene.page_width, np.uint32), (scene.page_height, np.uint32), (np.reshape(scene.pts, -1), np.float64),
        (scene.flags, np.uint8), (scene.path_pt_off, np.uint64), (scene.fill_rule, np.uint8),
        (np.reshape(rgb, -1), np.uint8), (scene.alpha, np.uint8), (scene.path_page, np.uint32))]
    st = Stats()
    lib().or_render_scene_rgb(_p(arena, C.c_uint8), _p(po, C.c_uint64), _p(a[0], C.c_uint32), _p(a[1], C.c_uint32),
                              a[0].size, _p(a[2], C.c_double), _p(a[3], C.c_uint8), _p(a[4], C.c_uint64),
                              _p(a[5], C.c_uint8), _p(a[6], C.c_uint8), _p(a[7], C.c_uint8), _p(a[8], C.c_uint32),
                              a[5].size, _mat(IDENTITY), 0.1, rowmap, threads, C.byref(st))
    return st.as_dict()


def render_scene_ex(scene, arena: np.ndarray, rgb=None, clip=None, rowmap=ROWMAP_DOCUMENTED, threads=1,
                    page_offset=None) -> dict:
    """Gray pages (rgb None) or Rgb8 pages (rgb [n_paths, 3]); clip [n_paths, 4]
    device-space rectangles (x0, y0, x1, y1) or None. page_offset defaults to
    the scene's (x3 for Rgb8)."""
    bpp = 1 if rgb is None else 3
    po = np.ascontiguousarray(bpp * scene.page_offset.astype(np.uint64) if page_offset is None else page_offset,
                              np.uint64)
    a = [np.ascontiguousarray(x, t) for x, t in (
        (scene.page_width, np.uint32), (scene.page_height, np.uint32), (np.reshape(scene.pts, -1), np.float64),
        (scene.flags, np.uint8), (scene.path_pt_off, np.uint64), (scene.fill_rule, np.uint8),
        (scene.alpha, np.uint8), (scene.path_page, np.uint32))]
    gray = np.ascontiguousarray(getattr(scene, "gray", np.zeros(a[5].size, np.uint8)), np.uint8)
    rgbp = None if rgb is None else _p(np.ascontiguousarray(np.reshape(rgb, -1), np.uint8), C.c_uint8)
    keep = []
    clipp = None
    if clip is not None:
        c = np.ascontiguousarray(np.reshape(clip, -1), np.float64)
        keep.append(c)
        clipp = _p(c, C.c_double)
    if rgb is not None:
        keep.append(rgbp)
    st = Stats()
    lib().or_render_scene_ex(_p(arena, C.c_uint8), _p(po, C.c_uint64), _p(a[0], C.c_uint32), _p(a[1], C.c_uint32),
                             a[0].size, _p(a[2], C.c_double), _p(a[3], C.c_uint8), _p(a[4], C.c_uint64),
                             _p(a[5], C.c_uint8), _p(gray, C.c_uint8), rgbp, _p(a[6], C.c_uint8),
                             _p(a[7], C.c_uint32), a[5].size, clipp, _mat(IDENTITY), 0.1, rowmap, threads,
                             C.byref(st))
    return st.as_dict()


def render_scene(scene, arena: np.ndarray, rowmap=ROWMAP_DOCUMENTED, threads=1) -> dict:
    """Render an rrb.Scene (its numpy views) with the oracle into `arena` in place."""
    return render_arrays(arena, scene.page_offset, scene.page_width, scene.page_height, scene.pts, scene.flags,
                         scene.path_pt_off, scene.fill_rule, scene.gray, scene.alpha, scene.path_page,
                         rowmap=rowmap, threads=threads)


# ---- F1: the reference's GPU fill operators (fill.rs, tile_fill.cu) -------------
TILE_RECORD = np.dtype([("key", "<u4"), ("x_enter", "<f4"), ("dxdy", "<f4"), ("y0_tile", "<f4"),
                        ("y1_tile", "<f4"), ("sign", "<f4"), ("pad", "<u4"), ("pad2", "<u4")])


def aa_jitter():
    """The oracle's 64 sample offsets (x, y) as f32 arrays."""
    x, y = np.zeros(64, np.float32), np.zeros(64, np.float32)
    lib().or_aa_jitter(_p(x, C.c_float), _p(y, C.c_float))
    return x, y


def aa_fill_cpu(segs, x_min, y_min, width, height, eo=False):
    """aa_fill_cpu (fill.rs:346-398): u8 coverage [height, width] from f32 segs [n, 4]."""
    segs = np.ascontiguousarray(segs, np.float32).reshape(-1)
    out = np.zeros(width * height, np.uint8)
    lib().or_aa_fill_cpu(_p(segs, C.c_float), segs.size // 4, x_min, y_min, width, height, int(eo),
                         _p(out, C.c_uint8))
    return out.reshape(height, width)


def build_tile_records(segs, x_min, y_min, width, height):
    """build_tile_records (fill.rs:82-264) with a stable key sort: (records, starts, counts, grid_w)."""
    segs = np.ascontiguousarray(segs, np.float32).reshape(-1)
    gw = C.c_uint32()
    n = lib().or_build_tile_records(_p(segs, C.c_float), segs.size // 4, x_min, y_min, width, height, None, None,
                                    None, C.byref(gw))
    if n < 0:
        raise ValueError("raster too large for 16-bit tile keys")
    grid_w, grid_h = gw.value, (height + 15) // 16
    recs = np.zeros(max(n, 1), TILE_RECORD)
    starts = np.zeros(grid_w * grid_h, np.uint32)
    counts = np.zeros(grid_w * grid_h, np.uint32)
    lib().or_build_tile_records(_p(segs, C.c_float), segs.size // 4, x_min, y_min, width, height,
                                recs.ctypes.data, _p(starts, C.c_uint32), _p(counts, C.c_uint32), C.byref(gw))
    return recs[:n], starts, counts, grid_w


def tile_fill(records, starts, counts, grid_w, width, height, eo=False):
    """tile_fill (tile_fill.cu:132-177), IEEE f32 as written: u8 coverage [height, width]."""
    records = np.ascontiguousarray(records, TILE_RECORD)
    if records.size == 0:
        records = np.zeros(1, TILE_RECORD)
    starts = np.ascontiguousarray(starts, np.uint32)
    counts = np.ascontiguousarray(counts, np.uint32)
    out = np.zeros(width * height, np.uint8)
    lib().or_tile_fill(records.ctypes.data, _p(starts, C.c_uint32), _p(counts, C.c_uint32), grid_w, width, height,
                       int(eo), _p(out, C.c_uint8))
    return out.reshape(height, width)


# ---- F2: strokes ------------------------------------------------------------------
def stroke_params(strokes, keep):
    """StrokeParams array from a list of dicts (None = fill): keys line_width,
    line_cap, line_join, miter_limit (10), dash (sequence), dash_phase (0)."""
    arr = (StrokeParams * max(1, len(strokes)))()
    for i, d in enumerate(strokes):
        if d is None:
            continue
        dash = np.ascontiguousarray(d.get("dash", ()), np.float64)
        keep.append(dash)
        arr[i].line_width = float(d["line_width"])
        arr[i].miter_limit = float(d.get("miter_limit", 10.0))
        arr[i].dash_phase = float(d.get("dash_phase", 0.0))
        arr[i].dash = _p(dash, C.c_double) if dash.size else None
        arr[i].n_dash = int(dash.size)
        arr[i].line_cap = int(d.get("line_cap", CAP_BUTT))
        arr[i].line_join = int(d.get("line_join", JOIN_MITER))
        arr[i].stroke = 1
    return arr


def _path_arrays(pts, flags):
    p = np.ascontiguousarray(np.reshape(pts, -1), np.float64)
    f = np.ascontiguousarray(flags, np.uint8)
    return p, f


def _take(h):
    o = OraclePath.__new__(OraclePath)
    o.h = h
    return o.build()


def stroke_flatten(pts, flags, flatness=0.1):
    """flatten_path (stroke/path.rs:40-86): (pts[n,2], flags[n])."""
    p, f = _path_arrays(pts, flags)
    h = lib().or_path_new()
    lib().or_stroke_flatten(_p(p, C.c_double), _p(f, C.c_uint8), f.size, flatness, h)
    return _take(h)


def stroke_dash(pts, flags, dash, phase=0.0):
    """make_dashed_path (stroke/path.rs:107-220) of an already flat path."""
    p, f = _path_arrays(pts, flags)
    d = np.ascontiguousarray(dash, np.float64)
    h = lib().or_path_new()
    lib().or_stroke_dash(_p(p, C.c_double), _p(f, C.c_uint8), f.size, _p(d, C.c_double), d.size, phase, h)
    return _take(h)


def stroke_outline(pts, flags, flatness=0.1, **stroke):
    """What stroke() draws: (kind, pts, flags); kind 0 nothing, 1 the outline
    make_stroke_path builds (filled nonzero), 2 a hairline polyline."""
    p, f = _path_arrays(pts, flags)
    keep = []
    sp = stroke_params([stroke], keep)
    h = lib().or_path_new()
    kind = lib().or_stroke_outline(_p(p, C.c_double), _p(f, C.c_uint8), f.size, sp, flatness, h)
    pts2, fl2 = _take(h)
    return kind, pts2, fl2


def render_scene_paint(scene, arena: np.ndarray, strokes, rgb=None, clip=None, rowmap=ROWMAP_DOCUMENTED, threads=1,
                       page_offset=None, flatness=0.1) -> dict:
    """render_scene_ex where path p is stroked with strokes[p] (a dict as in
    stroke_params) or filled when strokes[p] is None."""
    bpp = 1 if rgb is None else 3
    po = np.ascontiguousarray(bpp * scene.page_offset.astype(np.uint64) if page_offset is None else page_offset,
                              np.uint64)
    a = [np.ascontiguousarray(x, t) for x, t in (
        (scene.page_width, np.uint32), (scene.page_height, np.uint32), (np.reshape(scene.pts, -1), np.float64),
        (scene.flags, np.uint8), (scene.path_pt_off, np.uint64), (scene.fill_rule, np.uint8),
        (scene.alpha, np.uint8), (scene.path_page, np.uint32))]
    gray = np.ascontiguousarray(getattr(scene, "gray", np.zeros(a[5].size, np.uint8)), np.uint8)
    keep = []
    sp = stroke_params(list(strokes), keep)
    rgbp = None
    if rgb is not None:
        r = np.ascontiguousarray(np.reshape(rgb, -1), np.uint8)
        keep.append(r)
        rgbp = _p(r, C.c_uint8)
    clipp = None
    if clip is not None:
        c = np.ascontiguousarray(np.reshape(clip, -1), np.float64)
        keep.append(c)
        clipp = _p(c, C.c_double)
    st = Stats()
    lib().or_render_scene_paint(_p(arena, C.c_uint8), _p(po, C.c_uint64), _p(a[0], C.c_uint32),
                                _p(a[1], C.c_uint32), a[0].size, _p(a[2], C.c_double), _p(a[3], C.c_uint8),
                                _p(a[4], C.c_uint64), _p(a[5], C.c_uint8), _p(gray, C.c_uint8), rgbp,
                                _p(a[6], C.c_uint8), _p(a[7], C.c_uint32), a[5].size, clipp, sp, _mat(IDENTITY),
                                flatness, rowmap, threads, C.byref(st))
    return st.as_dict()
