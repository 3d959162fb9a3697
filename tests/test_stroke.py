"""Strokes (F2): the reference's stroke() — flatten_path, make_dashed_path,
make_stroke_path (crates/raster/src/stroke/path.rs) filled nonzero with AA, or
stroke_narrow's hairline spans for line width 0 (stroke/mod.rs:95-256).

CPU: the oracle against the reference's own stroke tests (stroke/mod.rs:310-443)
and hand-derived answers; the product's host outline builder
(rrb_stroke_outline) against the oracle's, point for point, on seeded paths
over every cap, join, dash and width. GPU: rrb_record_stroke_batch through
the C ABI against the oracle, byte for byte.
"""

import numpy as np
import pytest

BUTT, ROUND, PROJ = 0, 1, 2
MITER, RJOIN, BEVEL = 0, 1, 2


def _path(*subpaths, closed=()):
    """Points and PathBuilder flags of line subpaths (closed ones get the
    closing lineTo and CLOSED marks as PathBuilder::close adds them)."""
    pts, fl = [], []
    for k, sp in enumerate(subpaths):
        start = len(fl)
        for i, p in enumerate(sp):
            pts.append(p)
            fl.append(1 if i == 0 else 0)
        if k in closed:
            if tuple(sp[0]) != tuple(sp[-1]):
                pts.append(sp[0])
                fl.append(0)
            fl[start] |= 4
            fl[-1] |= 4
        fl[-1] |= 2
    return np.array(pts, float), np.array(fl, np.uint8)


# ---- the reference's tests (stroke/mod.rs:310-443) on the oracle ---------------------

def test_make_stroke_path_non_degenerate(oracle):
    pts, fl = _path([(0, 0), (10, 0)])
    kind, out, _ = oracle.stroke_outline(pts, fl, flatness=1.0, line_width=2.0)
    assert kind == 1 and len(out) >= 4


def test_make_dashed_path_respects_dash_array(oracle):
    pts, fl = _path([(0, 0), (20, 0)])
    out, ofl = oracle.stroke_dash(pts, fl, [4.0, 2.0])
    assert len(out) and (out[:, 0] >= -1e-9).all() and (out[:, 0] <= 20 + 1e-9).all()
    assert np.count_nonzero(ofl & 1) >= 2


def test_zero_dash_is_empty(oracle):
    pts, fl = _path([(0, 0), (10, 0)])
    out, _ = oracle.stroke_dash(pts, fl, [0.0])
    assert len(out) == 0


def test_flatten_path_removes_curves(oracle):
    pts = np.array([(0, 0), (1, 2), (3, 4), (4, 0)], float)
    fl = np.array([1, 8, 8, 2], np.uint8)
    out, ofl = oracle.stroke_flatten(pts, fl, 1.0)
    assert not (ofl & 8).any() and len(out) >= 2


def test_stroke_narrow_draws_diagonal(oracle):
    # (1,1)-(8,8) hairline on a 16x16 page: some diagonal pixel is painted.
    pts, fl = _path([(1, 1), (8, 8)])
    page = _render_one(oracle, pts, fl, 16, 16, dict(line_width=0.0), gray=0)
    assert any(page[i, i] == 0 for i in range(1, 9))


# ---- hand-derived answers ------------------------------------------------------------

class _One:
    def __init__(self, pts, fl, w, h, gray, alpha):
        self.pts, self.flags = pts, fl
        self.path_pt_off = np.array([0, len(fl)], np.uint64)
        self.fill_rule = np.zeros(1, np.uint8)
        self.gray = np.array([gray], np.uint8)
        self.alpha = np.array([alpha], np.uint8)
        self.path_page = np.zeros(1, np.uint32)
        self.page_width, self.page_height = np.array([w], np.uint32), np.array([h], np.uint32)
        self.page_offset = np.zeros(1, np.uint64)


def _render_one(oracle, pts, fl, w, h, stroke, gray=0, alpha=255, clip=None):
    page = np.full(w * h, 255, np.uint8)
    oracle.render_scene_paint(_One(pts, fl, w, h, gray, alpha), page, [stroke], clip=clip)
    return page.reshape(h, w)


def _fill_rect(oracle, x0, y0, x1, y1, w, h):
    page = np.full((h, w), 255, np.uint8)
    pts, fl = _path([(x0, y1), (x0, y0), (x1, y0), (x1, y1)], closed=(0,))
    oracle.fill_path(page, pts, fl)
    return page


def test_butt_and_projecting_caps_are_their_rectangles(oracle):
    # A horizontal stroke of width 2 is the fill of its rectangle: butt caps
    # end at the endpoints, projecting caps w/2 beyond them. (Splash's AA
    # scanner includes an edge's closing AA row and column, so the pixels are
    # the rectangle fill's, not whole pixels.)
    pts, fl = _path([(2, 5), (12, 5)])
    butt = _render_one(oracle, pts, fl, 16, 10, dict(line_width=2.0, line_cap=BUTT))
    assert np.array_equal(butt, _fill_rect(oracle, 2, 4, 12, 6, 16, 10))
    assert (butt[5, 2:12] == 0).all() and (butt[:4] == 255).all() and (butt[7:] == 255).all()
    proj = _render_one(oracle, pts, fl, 16, 10, dict(line_width=2.0, line_cap=PROJ))
    assert np.array_equal(proj, _fill_rect(oracle, 1, 4, 13, 6, 16, 10))


def test_joins(oracle):
    pts, fl = _path([(0, 0), (10, 0), (10, 10)])
    k, mit, _ = oracle.stroke_outline(pts, fl, line_width=2.0, line_join=MITER, miter_limit=10.0)
    assert any(np.array_equal(p, [11.0, -1.0]) for p in mit)  # the miter apex of the right angle
    k, bev, _ = oracle.stroke_outline(pts, fl, line_width=2.0, line_join=BEVEL)
    assert not any(np.array_equal(p, [11.0, -1.0]) for p in bev) and len(bev) == len(mit) - 1
    # Limit below sqrt(2): the right-angle miter (ratio sqrt 2) becomes a bevel.
    k, lim, _ = oracle.stroke_outline(pts, fl, line_width=2.0, line_join=MITER, miter_limit=1.4)
    assert len(lim) == len(bev)
    k, rnd, rfl = oracle.stroke_outline(pts, fl, line_width=2.0, line_join=RJOIN)
    assert (rfl & 8).any()


def test_dash_phase(oracle):
    pts, fl = _path([(0, 0), (20, 0)])
    out, ofl = oracle.stroke_dash(pts, fl, [4.0, 2.0], 5.0)
    # Phase 5 lands 1 into the gap: dashes [1,5], [7,11], [13,17], [19,20].
    starts = out[(ofl & 1) != 0][:, 0]
    assert np.allclose(starts, [1, 7, 13, 19])


def test_hairline_spans(oracle):
    pts, fl = _path([(0.5, 3.5), (10.5, 3.5)])
    page = _render_one(oracle, pts, fl, 16, 8, dict(line_width=0.0), gray=40)
    exp = np.full((8, 16), 255, np.uint8)
    exp[3, 0:11] = 40
    assert np.array_equal(page, exp)
    # Translucent: one blend per pixel, div255((255 - a) * d + a * g).
    page = _render_one(oracle, pts, fl, 16, 8, dict(line_width=0.0), gray=0, alpha=128)
    assert page[3, 5] == oracle.div255((255 - 128) * 255)


def test_zero_length_round_cap_is_a_circle(oracle):
    pts, fl = _path([(5, 5), (5, 5)])
    k, out, ofl = oracle.stroke_outline(pts, fl, line_width=4.0, line_cap=ROUND)
    assert k == 1 and np.count_nonzero(ofl & 8) == 8  # four cubic quarter arcs
    k, out, _ = oracle.stroke_outline(pts, fl, line_width=4.0, line_cap=BUTT)
    assert k == 0 and len(out) == 0


# ---- seeded paths: the product's host outline builder against the oracle -------------

def random_stroke_path(rng, w=200.0, h=150.0):
    """Points and flags of 1-3 subpaths of lines and cubics, some closed, some
    with repeated points, as PathBuilder makes them."""
    pts, fl = [], []
    for _ in range(int(rng.integers(1, 4))):
        start = len(fl)
        cur = rng.uniform([0, 0], [w, h])
        pts.append(cur)
        fl.append(1)
        for _ in range(int(rng.integers(1, 7))):
            r = rng.random()
            if r < 0.15:
                nxt = cur.copy()  # coincident point
            else:
                nxt = np.clip(cur + rng.normal(0, 30, 2), [-20, -20], [w + 20, h + 20])
            if rng.random() < 0.3:
                c1 = cur + rng.normal(0, 20, 2)
                c2 = nxt + rng.normal(0, 20, 2)
                pts += [c1, c2, nxt]
                fl += [8, 8, 0]
            else:
                pts.append(nxt)
                fl.append(0)
            cur = nxt
        if rng.random() < 0.4:
            if not np.array_equal(pts[start], pts[-1]):
                pts.append(pts[start].copy())
                fl.append(0)
            fl[start] |= 4
            fl[-1] |= 4
        fl[-1] |= 2
    return np.array(pts, float), np.array(fl, np.uint8)


def random_stroke(rng):
    d = dict(line_width=float(rng.choice([0.0, 0.3, 1.0, 2.5, 7.0])), line_cap=int(rng.integers(0, 3)),
             line_join=int(rng.integers(0, 3)), miter_limit=float(rng.choice([1.2, 2.0, 10.0])))
    if rng.random() < 0.3:
        dashes = [[3.0, 2.0], [5.0, 1.0, 1.0, 1.0], [0.0, 4.0], [7.5]]
        d["dash"] = dashes[int(rng.integers(0, len(dashes)))]
        d["dash_phase"] = float(rng.uniform(-10, 10))
    return d


def test_host_outline_matches_oracle(oracle, rrb_lib):
    rng = np.random.default_rng(11)
    kinds = set()
    for i in range(1500):
        pts, fl = random_stroke_path(rng)
        st = random_stroke(rng)
        flat = float(rng.choice([0.1, 0.5]))
        a = rrb_lib.stroke_outline(pts, fl, flatness=flat, **st)
        b = oracle.stroke_outline(pts, fl, flatness=flat, **st)
        assert a[0] == b[0], (i, st)
        assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2]), (i, st)
        kinds.add(a[0])
    assert kinds == {1, 2} or kinds == {0, 1, 2}


def test_host_outline_round_join_chains_match_oracle(oracle, rrb_lib):
    """Long chains of round joins, where the builder reuses each segment's
    length and join angle for the next join: smooth curves turning one way,
    zigzags turning both ways, collinear vertices (no join drawn) between
    turns, and closed subpaths whose last join turns into the first segment."""
    rng = np.random.default_rng(23)
    cases = []
    for _ in range(60):  # curves flattened into many short segments
        c = rng.uniform(20, 180, 2)
        pts, fl = [c], [1]
        for _ in range(int(rng.integers(1, 5))):
            pts += [c + rng.normal(0, 40, 2), c + rng.normal(0, 40, 2), c + rng.normal(0, 60, 2)]
            fl += [8, 8, 0]
            c = pts[-1]
        fl[-1] |= 2
        cases.append((np.array(pts, float), np.array(fl, np.uint8)))
    for _ in range(60):  # zigzags with collinear runs, some closed
        n = int(rng.integers(4, 40))
        xs = np.cumsum(rng.uniform(1, 15, n))
        ys = rng.choice([-6.0, 0.0, 0.0, 6.0], n) + 50
        sub = [tuple(p) for p in np.stack([xs, ys], 1)]
        cases.append(_path(sub, closed=(0,) if rng.random() < 0.4 else ()))
    for pts, fl in cases:
        for w in (0.5, 2.0, 9.0):
            st = dict(line_width=w, line_join=RJOIN, line_cap=int(rng.integers(0, 3)))
            a = rrb_lib.stroke_outline(pts, fl, flatness=0.1, **st)
            b = oracle.stroke_outline(pts, fl, flatness=0.1, **st)
            assert a[0] == b[0] == 1
            assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])


def test_host_outline_rejects_bad_params(rrb_lib):
    pts, fl = _path([(0, 0), (10, 0)])
    for bad in (dict(line_width=-1.0), dict(line_width=float("nan")), dict(line_width=1.0, line_cap=3),
                dict(line_width=1.0, dash=[1.0, -2.0])):
        with pytest.raises(rrb_lib.BackendError):
            rrb_lib.stroke_outline(pts, fl, **bad)


# ---- GPU: rrb_record_stroke_batch against the oracle ------------------------------

class StrokeScene:
    """Seeded paint batch over n_pages pages: paths (sorted by page) with a
    stroke dict or None (fill) each."""

    def __init__(self, seed, n_paths=240, n_pages=1, w=220, h=170):
        rng = np.random.default_rng(seed)
        pts, fls, off, strokes = [], [], [0], []
        for _ in range(n_paths):
            p, f = random_stroke_path(rng, w, h)
            pts.append(p)
            fls.append(f)
            off.append(off[-1] + len(f))
            strokes.append(None if rng.random() < 0.15 else random_stroke(rng))
        self.pts = np.concatenate(pts)
        self.flags = np.concatenate(fls)
        self.path_pt_off = np.array(off, np.uint64)
        self.fill_rule = rng.integers(0, 2, n_paths).astype(np.uint8)
        self.gray = rng.integers(0, 256, n_paths).astype(np.uint8)
        self.alpha = np.where(rng.random(n_paths) < 0.5, 255, rng.integers(32, 256, n_paths)).astype(np.uint8)
        self.path_page = np.sort(rng.integers(0, n_pages, n_paths)).astype(np.uint32)
        self.page_width = np.full(n_pages, w, np.uint32)
        self.page_height = np.full(n_pages, h, np.uint32)
        self.page_offset = (np.arange(n_pages) * w * h).astype(np.uint64)
        self.arena_bytes = n_pages * w * h
        self.strokes = strokes
        self.n_paths = n_paths


def _gpu_paint(backend, rrb_lib, sc, rgb=None, clip=None, rowmap=0, tile=(64, 16)):
    bpp = 1 if rgb is None else 3
    pages = backend.alloc_device(bpp * sc.arena_bytes)
    keep = []
    p = rrb_lib.batch_params(sc.pts, sc.flags, sc.path_pt_off, sc.fill_rule, sc.gray, sc.alpha, sc.path_page,
                             sc.page_width, sc.page_height, bpp * sc.page_offset, pages, rowmap=rowmap, keep=keep)
    try:
        backend.set_tuning(*tile)
        backend.begin_page()
        try:
            backend.record_fill_buffer(pages, 255)
            backend.record_stroke_batch(p, sc.strokes, rgb, clip)
        finally:
            backend.wait_page(backend.submit_page())
        got = np.empty(bpp * sc.arena_bytes, np.uint8)
        backend.wait_download(backend.download_async(pages, got))
        return got
    finally:
        backend.set_tuning(64, 16, auto_tile=True)
        backend.free_device(pages)


@pytest.mark.gpu
@pytest.mark.parametrize("rowmap", [0, 1])
@pytest.mark.parametrize("tile", [(16, 16), (32, 32), (64, 16), (128, 16), (128, 32)])
def test_stroke_batch_matches_oracle(backend, oracle, rrb_lib, rowmap, tile):
    sc = StrokeScene(5, n_paths=300, n_pages=2)
    exp = np.full(sc.arena_bytes, 255, np.uint8)
    oracle.render_scene_paint(sc, exp, sc.strokes, rowmap=rowmap)
    got = _gpu_paint(backend, rrb_lib, sc, rowmap=rowmap, tile=tile)
    d = np.nonzero(got != exp)[0]
    assert d.size == 0, f"{d.size} bytes differ, first at {d[:5]}"


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [6, 7])
def test_stroke_batch_rgb_and_clip(backend, oracle, rrb_lib, seed):
    sc = StrokeScene(seed, n_paths=200, n_pages=1)
    rng = np.random.default_rng(seed)
    rgb = rng.integers(0, 256, (sc.n_paths, 3), dtype=np.uint8)
    clip = np.tile([20.5, 15.25, 180.75, 140.5], (sc.n_paths, 1))
    clip[::3] = (-5, -5, 400, 400)
    exp = np.full(3 * sc.arena_bytes, 255, np.uint8)
    oracle.render_scene_paint(sc, exp, sc.strokes, rgb=rgb, clip=clip)
    got = _gpu_paint(backend, rrb_lib, sc, rgb=rgb, clip=clip)
    d = np.nonzero(got != exp)[0]
    assert d.size == 0, f"{d.size} bytes differ, first at {d[:5]}"
    exp = np.full(sc.arena_bytes, 255, np.uint8)
    oracle.render_scene_paint(sc, exp, sc.strokes, clip=clip)
    got = _gpu_paint(backend, rrb_lib, sc, clip=clip)
    assert np.array_equal(got, exp)


@pytest.mark.gpu
def test_hairlines_only_and_bad_params(backend, oracle, rrb_lib):
    sc = StrokeScene(8, n_paths=150)
    sc.strokes = [dict(line_width=0.0, dash=[2.0, 1.0]) if i % 2 else dict(line_width=0.0)
                  for i in range(sc.n_paths)]
    exp = np.full(sc.arena_bytes, 255, np.uint8)
    oracle.render_scene_paint(sc, exp, sc.strokes)
    assert np.array_equal(_gpu_paint(backend, rrb_lib, sc), exp)
    sc.strokes[3] = dict(line_width=-2.0)
    with pytest.raises(rrb_lib.BackendError) as e:
        _gpu_paint(backend, rrb_lib, sc)
    assert e.value.status == 4


@pytest.mark.gpu
@pytest.mark.parametrize("rgb_pages", [False, True])
def test_stroke_page_matches_oracle(backend, oracle, rrb_lib, rgb_pages):
    """The benchmark's stroke page generator at Letter @150 dpi: rules, boxes,
    polylines, curves, dashes and fills interleaved in one batch."""
    from rrb.strokes import StrokePage

    sp = StrokePage(3, n_paths=2500, w=1275, h=1650)
    rgb = np.random.default_rng(4).integers(0, 256, (sp.n_paths, 3), dtype=np.uint8) if rgb_pages else None
    bpp = 3 if rgb_pages else 1
    exp = np.full(bpp * sp.arena_bytes, 255, np.uint8)
    oracle.render_scene_paint(sp, exp, sp.strokes, rgb=rgb)
    got = _gpu_paint(backend, rrb_lib, sp, rgb=rgb)
    d = np.nonzero(got != exp)[0]
    assert d.size == 0, f"{d.size} bytes differ, first at {d[:5]}"
