"""Non-rectangular clip paths (F3) in the oracle: Clip::clip_to_path
(crates/raster/src/clip.rs:141-176), detect_rect (:322-359) and clip_aa_line
(:246-254), with the clip's XPath built as the renderer builds it
(pdf_interp/src/renderer/page/mod.rs:1003-1009: close_subpaths, no aa_scale).

clip_aa_line lets every clip scanner's render_aa_line clear the AA buffer and
draw its own coverage, so a fill under a clip path paints the clip path's
coverage, in the fill's paint, on the fill's rows; and without aa_scale that
coverage is the clip path at a quarter of its size. These tests pin that
reading on the CPU: it is the parity definition a device version must meet.
"""

import numpy as np
import pytest

W, H = 64, 48


def _poly(points, closed=True):
    pts = [tuple(p) for p in points]
    fl = [1] + [0] * (len(pts) - 1)
    if closed:
        if pts[0] != pts[-1]:
            pts.append(pts[0])
            fl.append(0)
        fl[0] |= 4
        fl[-1] |= 4
    fl[-1] |= 2
    return np.array(pts, float), np.array(fl, np.uint8)


def _random_poly(rng, n, lo, hi):
    c = rng.uniform(lo, hi)
    ang = np.sort(rng.uniform(0, 2 * np.pi, n))
    r = rng.uniform(3, 30, n)
    return _poly(np.stack([c[0] + r * np.cos(ang), c[1] + r * np.sin(ang)], 1))


def _random_curvy(rng, n, lo, hi):
    """A closed path of n cubic segments around a random centre."""
    c = rng.uniform(lo, hi)
    ang = np.sort(rng.uniform(0, 2 * np.pi, n))
    r = rng.uniform(5, 30, n)
    v = np.stack([c[0] + r * np.cos(ang), c[1] + r * np.sin(ang)], 1)
    pts, fl = [v[0]], [1]
    for k in range(n):
        a, b = v[k], v[(k + 1) % n]
        pts += [a + rng.normal(0, 8, 2), b + rng.normal(0, 8, 2), b]
        fl += [8, 8, 0]
    fl[0] |= 4
    fl[-1] |= 4 | 2
    return np.array(pts, float), np.array(fl, np.uint8)


def _rows_of(oracle, pts, fl, eo, rowmap):
    """Pixel rows the fill driver draws for a path under the page clip."""
    segs = oracle.xpath_new(pts, fl, close=True, aa_scale=True)
    b = oracle.Scanner(segs, eo, 0, 4 * H - 1).bounds()
    if b["empty"]:
        return set()
    if rowmap == oracle.ROWMAP_DOCUMENTED:
        return set(range(b["y_min"] // 4, b["y_max"] // 4 + 1))
    return {a // 4 for a in range(b["y_min"], b["y_max"] + 1) if a % 4 == 3}


class _OnePath:
    def __init__(self, pts, fl, gray):
        self.pts, self.flags = pts, fl
        self.path_pt_off = np.array([0, len(fl)], np.uint64)
        self.fill_rule = np.zeros(1, np.uint8)
        self.gray = np.array([gray], np.uint8)
        self.alpha = np.array([255], np.uint8)
        self.path_page = np.zeros(1, np.uint32)
        self.page_width, self.page_height = np.array([W], np.uint32), np.array([H], np.uint32)
        self.page_offset = np.zeros(1, np.uint64)


def test_rectangle_clip_path_is_the_rectangle_clip(oracle):
    """A clip path of two horizontal and two vertical segments reduces to
    clip_to_rect: the same page as the rectangle clip of render_scene_ex."""
    rng = np.random.default_rng(1)
    for i in range(40):
        pts, fl = _random_poly(rng, 7, [10, 10], [54, 38])
        x0, y0 = rng.uniform(0, 30, 2)
        x1, y1 = x0 + rng.uniform(2, 30), y0 + rng.uniform(2, 20)
        got = np.full((H, W), 255, np.uint8)
        oracle.fill_path_clip_path(got, pts, fl, *_poly([(x0, y0), (x1, y0), (x1, y1), (x0, y1)]), gray=30)
        exp = np.full(W * H, 255, np.uint8)
        oracle.render_scene_ex(_OnePath(pts, fl, 30), exp, clip=np.array([[x0, y0, x1, y1]]))
        assert np.array_equal(got, exp.reshape(H, W)), i


def test_empty_clip_path_paints_nothing(oracle):
    pts, fl = _poly([(5, 5), (40, 8), (30, 40)])
    page = np.full((H, W), 255, np.uint8)
    oracle.fill_path_clip_path(page, pts, fl, np.array([[10.0, 10.0]]), np.array([3], np.uint8))
    assert (page == 255).all()


@pytest.mark.parametrize("clip_eo", [False, True])
def test_clip_path_paints_the_quarter_size_clip_on_the_fill_rows(oracle, clip_eo):
    """Documented row map: the page is the fill of the clip path at a quarter of
    its size (its points and flatness divided by 4, both exact), kept on the
    pixel rows the fill path's own loop visits."""
    rng = np.random.default_rng(2)
    for i in range(60):
        pts, fl = _random_poly(rng, int(rng.integers(3, 9)), [8, 8], [56, 40])
        if i % 3 == 0:  # a clip path of cubics
            cpts, cfl = _random_curvy(rng, int(rng.integers(2, 6)), [30, 30], [200, 150])
        else:
            cpts, cfl = _random_poly(rng, int(rng.integers(3, 9)), [20, 20], [200, 150])
        got = np.full((H, W), 255, np.uint8)
        oracle.fill_path_clip_path(got, pts, fl, cpts, cfl, clip_eo=clip_eo, gray=20, alpha=200)
        quarter = np.full((H, W), 255, np.uint8)
        oracle.fill_path(quarter, cpts / 4.0, cfl, eo=clip_eo, gray=20, alpha=200, flatness=0.1 / 4.0)
        exp = np.full((H, W), 255, np.uint8)
        rows = sorted(_rows_of(oracle, pts, fl, False, oracle.ROWMAP_DOCUMENTED))
        rows = [y for y in rows if 0 <= y < H]
        exp[rows] = quarter[rows]
        assert np.array_equal(got, exp), i


@pytest.mark.parametrize("rowmap", ["documented", "as_shipped"])
def test_clip_path_output_depends_on_the_fill_rows_only(oracle, rowmap):
    """Two fills with the same AA row range (a wide and a narrow box, both
    inside the page) give the same page under the same clip path."""
    rm = oracle.ROWMAP_DOCUMENTED if rowmap == "documented" else oracle.ROWMAP_AS_SHIPPED
    rng = np.random.default_rng(3)
    compared = 0
    for i in range(40):
        y0, y1 = sorted(rng.uniform(1, 46, 2))
        if y1 - y0 < 1:
            y1 = y0 + 1
        wide = _poly([(1, y0), (62, y0), (62, y1), (1, y1)])
        narrow = _poly([(30, y0), (30.5, y0 + 0.5), (31, y1), (29.5, y1 - 0.25)])
        cpts, cfl = _random_poly(rng, int(rng.integers(3, 9)), [20, 20], [200, 150])
        a = np.full((H, W), 255, np.uint8)
        b = np.full((H, W), 255, np.uint8)
        oracle.fill_path_clip_path(a, *wide, cpts, cfl, rowmap=rm, gray=0)
        oracle.fill_path_clip_path(b, *narrow, cpts, cfl, rowmap=rm, gray=0)
        if _rows_of(oracle, *wide, False, rm) == _rows_of(oracle, *narrow, False, rm):
            assert np.array_equal(a, b), i
            compared += 1
    assert compared >= 30


def test_clip_path_stacks(oracle):
    """A stack of clip paths (successive W): each scanner overwrites the AA
    lines, so the last non-rectangular clip path is drawn; rectangle clip
    paths narrow the rectangle wherever they stand; an empty path lets
    nothing through."""
    rng = np.random.default_rng(4)
    for i in range(30):
        pts, fl = _random_poly(rng, int(rng.integers(3, 9)), [8, 8], [56, 40])
        ca = _random_poly(rng, 6, [20, 20], [200, 150]) + (bool(i % 2),)
        cb = _random_curvy(rng, 3, [30, 30], [200, 150]) + (False,)
        x0, y0 = rng.uniform(0, 30, 2)
        rect = (x0, y0, x0 + rng.uniform(5, 30), y0 + rng.uniform(5, 20))
        rp = _poly([(rect[0], rect[1]), (rect[2], rect[1]), (rect[2], rect[3]), (rect[0], rect[3])]) + (False,)
        ref = np.full((H, W), 255, np.uint8)
        oracle.fill_path_clip_path(ref, pts, fl, cb[0], cb[1], clip_eo=cb[2], gray=9, clip_rect=rect)
        for stack in ([ca, rp, cb], [rp, ca, cb], [ca, cb, rp]):
            got = np.full((H, W), 255, np.uint8)
            oracle.fill_path_clip_paths(got, pts, fl, stack, gray=9)
            assert np.array_equal(got, ref), (i, len(stack))
        empty = (np.zeros((0, 2)), np.zeros(0, np.uint8), False)
        got = np.full((H, W), 255, np.uint8)
        oracle.fill_path_clip_paths(got, pts, fl, [ca, empty, cb], gray=9)
        assert (got == 255).all()
