"""F3 clip paths through the product: rrb_lower_clip_paths lowers a batch with
a clip path per fill onto the rectangle-clipped batch of
rrb_record_path_batch_ex (a fill under a clip path paints the clip path at a
quarter of its size, in its paint and the clip's rule, on its pixel rows:
Clip::clip_aa_line, crates/raster/src/clip.rs:246-254, with the clip's XPath
built without aa_scale, pdf_interp/src/renderer/page/mod.rs:1003-1009).

CPU: the lowered batch rendered by the oracle's rectangle-clip renderer equals
the oracle's literal clip-path fill (or_fill_path_clip_path), path after path
on one page (documented row map: the oracle's batch renderer has no visited-
row override). GPU: the device's page for the same batch, through the C ABI,
under both row maps — under the shipped one a clip path draws the clip
scanner's rows 16y+12 .. 16y+15 on the pixel rows its fill's loop visits.
"""

from types import SimpleNamespace

import numpy as np
import pytest

W, H = 72, 56


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


def _random_poly(rng, n, lo, hi, rmax=30):
    c = rng.uniform(lo, hi)
    ang = np.sort(rng.uniform(0, 2 * np.pi, n))
    r = rng.uniform(3, rmax, n)
    return _poly(np.stack([c[0] + r * np.cos(ang), c[1] + r * np.sin(ang)], 1))


def _random_curvy(rng, n, lo, hi):
    c = rng.uniform(lo, hi)
    ang = np.sort(rng.uniform(0, 2 * np.pi, n))
    r = rng.uniform(5, 40, n)
    v = np.stack([c[0] + r * np.cos(ang), c[1] + r * np.sin(ang)], 1)
    pts, fl = [v[0]], [1]
    for k in range(n):
        a, b = v[k], v[(k + 1) % n]
        pts += [a + rng.normal(0, 10, 2), b + rng.normal(0, 10, 2), b]
        fl += [8, 8, 0]
    fl[0] |= 4
    fl[-1] |= 4 | 2
    return np.array(pts, float), np.array(fl, np.uint8)


class _Scene:
    def __init__(self, paths, rule, gray, alpha):
        self.pts = np.concatenate([p for p, _ in paths]).reshape(-1, 2)
        self.flags = np.concatenate([f for _, f in paths])
        self.path_pt_off = np.cumsum([0] + [len(f) for _, f in paths]).astype(np.uint64)
        self.fill_rule = np.asarray(rule, np.uint8)
        self.gray = np.asarray(gray, np.uint8)
        self.alpha = np.asarray(alpha, np.uint8)
        self.path_page = np.zeros(len(paths), np.uint32)
        self.page_width, self.page_height = np.array([W], np.uint32), np.array([H], np.uint32)
        self.page_offset = np.zeros(1, np.uint64)
        self.n_paths = len(paths)


def _batch(rng, n_paths):
    """Paths, paint, clip rectangles and clip paths of one seeded batch."""
    paths, rule, gray, alpha, rects, clips = [], [], [], [], [], []
    for i in range(n_paths):
        paths.append(_random_poly(rng, int(rng.integers(3, 9)), [6, 6], [66, 50]))
        rule.append(int(rng.random() < 0.3))
        gray.append(int(rng.integers(0, 256)))
        alpha.append(int(rng.choice([255, int(rng.integers(40, 255))])))
        kind = i % 6
        rect = None
        if kind in (1, 3):
            x0, y0 = rng.uniform(-5, 50, 2)
            rect = [x0, y0, x0 + rng.uniform(3, 40), y0 + rng.uniform(3, 30)]
        rects.append(rect if rect is not None else [-1e9, -1e9, 1e9, 1e9])
        if kind in (2, 3):
            cp = _random_poly(rng, int(rng.integers(3, 9)), [20, 20], [260, 200], rmax=90)
        elif kind == 4:
            cp = _random_curvy(rng, int(rng.integers(2, 5)), [40, 40], [240, 180])
        elif kind == 5:  # a rectangle: detect_rect makes it a rectangle clip
            x0, y0 = rng.uniform(0, 50, 2)
            w = rng.uniform(4, 30)
            cp = _poly([(x0, y0), (x0 + w, y0), (x0 + w, y0 + 15), (x0, y0 + 15)])
        else:
            cp = None
        clips.append(None if cp is None else (cp[0], cp[1], bool(rng.random() < 0.5)))
    return paths, rule, gray, alpha, np.array(rects, float), clips


def _batch_stacks(rng, n_paths):
    """Clip stacks (lists of clip paths) and clip rectangles off the page."""
    paths, rule, gray, alpha, rects, clips = [], [], [], [], [], []
    empty = (np.zeros((0, 2)), np.zeros(0, np.uint8), False)
    for i in range(n_paths):
        paths.append(_random_poly(rng, int(rng.integers(3, 9)), [6, 6], [66, 50]))
        rule.append(int(rng.random() < 0.3))
        gray.append(int(rng.integers(0, 256)))
        alpha.append(int(rng.choice([255, int(rng.integers(40, 255))])))
        a = _random_poly(rng, 6, [20, 20], [260, 200], rmax=90) + (bool(rng.random() < 0.5),)
        b = _random_curvy(rng, 3, [40, 40], [240, 180]) + (bool(rng.random() < 0.5),)
        x0, y0 = rng.uniform(0, 50, 2)
        r = _poly([(x0, y0), (x0 + 25, y0), (x0 + 25, y0 + 18), (x0, y0 + 18)]) + (False,)
        kind = i % 6
        clips.append([[a, b], [r, a], [a, r], [a, empty, b], [r], None][kind])
        rects.append([-30.0, 5.0, -2.0, 40.0] if i % 7 == 3 else [-1e9, -1e9, 1e9, 1e9])
    return paths, rule, gray, alpha, np.array(rects, float), clips


def _expected(oracle, paths, rule, gray, alpha, rects, clips, rowmap=0):
    page = np.full((H, W), 255, np.uint8)
    for i, (p, f) in enumerate(paths):
        r = rects[i]
        if isinstance(clips[i], list):
            oracle.fill_path_clip_paths(page, p, f, clips[i], eo=bool(rule[i]), gray=gray[i], alpha=alpha[i],
                                        clip_rect=r, rowmap=rowmap)
        elif clips[i] is not None:
            cp, cf, ceo = clips[i]
            oracle.fill_path_clip_path(page, p, f, cp, cf, clip_eo=ceo, eo=bool(rule[i]), gray=gray[i],
                                       alpha=alpha[i], clip_rect=r, rowmap=rowmap)
        else:
            flat = page.reshape(-1)
            oracle.render_scene_ex(_Scene([(p, f)], [rule[i]], [gray[i]], [alpha[i]]), flat, clip=r.reshape(1, 4),
                                   rowmap=rowmap)
    return page


def _params(rrb_lib, paths, rule, gray, alpha, keep, pages=None):
    s = _Scene(paths, rule, gray, alpha)
    return rrb_lib.batch_params(s.pts, s.flags, s.path_pt_off, s.fill_rule, s.gray, s.alpha, s.path_page,
                                s.page_width, s.page_height, s.page_offset, pages, keep=keep), s


@pytest.mark.parametrize("seed", [0, 1, 2, 3, 10, 11, 12])
def test_lowered_batch_paints_the_oracle_clip(oracle, rrb_lib, seed):
    rng = np.random.default_rng(seed)
    paths, rule, gray, alpha, rects, clips = (_batch if seed < 10 else _batch_stacks)(rng, 18)
    keep = []
    params, s = _params(rrb_lib, paths, rule, gray, alpha, keep)
    low = rrb_lib.lower_clip_paths(params, clips, rects)
    src = low["src_path"]
    lowered = SimpleNamespace(pts=low["pts"], flags=low["flags"], path_pt_off=low["path_pt_off"],
                              fill_rule=low["fill_rule"], gray=s.gray[src], alpha=s.alpha[src],
                              path_page=np.zeros(len(src), np.uint32), page_width=s.page_width,
                              page_height=s.page_height, page_offset=s.page_offset)
    got = np.full(W * H, 255, np.uint8)
    oracle.render_scene_ex(lowered, got, clip=low["clip_rects"])
    exp = _expected(oracle, paths, rule, gray, alpha, rects, clips)
    assert np.array_equal(got.reshape(H, W), exp)
    assert (exp != 255).any()


def test_disjoint_rectangles_paint_nothing(oracle, rrb_lib):
    """A clip rectangle and a rectangle clip path that do not meet leave an
    inverted rectangle, which is empty; the lowering drops the fill (the
    device would read the inverted corners as a rectangle)."""
    p, f = _poly([(2, 2), (60, 4), (50, 50), (3, 40)])
    rect_path = _poly([(20, 5), (40, 5), (40, 30), (20, 30)]) + (False,)
    keep = []
    params, _ = _params(rrb_lib, [(p, f)], [0], [0], [255], keep)
    low = rrb_lib.lower_clip_paths(params, [rect_path], np.array([[0.0, 0.0, 10.0, 56.0]]))
    assert len(low["src_path"]) == 0
    page = np.full((H, W), 255, np.uint8)
    oracle.fill_path_clip_paths(page, p, f, [rect_path], clip_rect=[0.0, 0.0, 10.0, 56.0])
    assert (page == 255).all()


def test_lowering_needs_identity_and_a_known_row_map(rrb_lib):
    p, f = _poly([(1, 1), (20, 3), (9, 18)])
    keep = []
    params, _ = _params(rrb_lib, [(p, f)], [0], [0], [255], keep)
    params.matrix[0] = 2.0
    with pytest.raises(rrb_lib.BackendError):
        rrb_lib.lower_clip_paths(params, [(p, f, False)])
    params.matrix[0] = 1.0
    params.rowmap = 2
    with pytest.raises(rrb_lib.BackendError):
        rrb_lib.lower_clip_paths(params, [(p, f, False)])
    params.rowmap = rrb_lib.RRB_ROWMAP_DOCUMENTED
    params.path_page[0] = 3  # no such page
    with pytest.raises(rrb_lib.BackendError):
        rrb_lib.lower_clip_paths(params, [(p, f, False)])
    params.path_page[0] = 0
    params.pts = None  # points missing
    with pytest.raises(rrb_lib.BackendError):
        rrb_lib.lower_clip_paths(params, [(p, f, False)])


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_clip_paths_on_the_device_match_oracle(backend, oracle, rrb_lib, seed):
    rng = np.random.default_rng(seed)
    paths, rule, gray, alpha, rects, clips = _batch(rng, 18)
    exp = _expected(oracle, paths, rule, gray, alpha, rects, clips)
    pages = backend.alloc_device(W * H)
    keep = []
    params, _ = _params(rrb_lib, paths, rule, gray, alpha, keep, pages)
    try:
        backend.begin_page()
        try:
            backend.record_fill_buffer(pages, 255)
            backend.record_path_batch_clip_paths(params, clips, rects)
        finally:
            backend.wait_page(backend.submit_page())
        got = np.empty(W * H, np.uint8)
        backend.wait_download(backend.download_async(pages, got))
    finally:
        backend.free_device(pages)
    assert np.array_equal(got.reshape(H, W), exp)


def test_shipped_lowering_visits_the_fills_rows(oracle, rrb_lib):
    """Under the shipped row map a lowered clip path keeps the clip scanner's
    rows as its clip and gets the fill's visited rows: the pixel rows y whose
    AA row 4y+3 lies in the fill's scanner range; paths without a clip path
    keep their own rows (INT32_MIN)."""
    rng = np.random.default_rng(5)
    paths, rule, gray, alpha, rects, clips = _batch(rng, 12)
    keep = []
    params, s = _params(rrb_lib, paths, rule, gray, alpha, keep)
    params.rowmap = rrb_lib.RRB_ROWMAP_AS_SHIPPED
    low = rrb_lib.lower_clip_paths(params, clips, rects)
    own = np.iinfo(np.int32).min
    checked = 0
    for k, i in enumerate(low["src_path"]):
        v0, v1 = (int(v) for v in low["visit_rows"][k])
        if i % 6 not in (2, 3, 4):  # no clip path, or a rectangle one (detect_rect)
            assert v0 == own
            continue
        r = rects[i]
        y_lo = int(np.floor(max(0.0, min(r[1], r[3]))))
        y_hi = int(np.ceil(min(float(H), max(r[1], r[3])))) - 1
        sc = oracle.Scanner(oracle.xpath_new(paths[i][0], paths[i][1], aa_scale=True), bool(rule[i]), 4 * y_lo,
                            4 * (y_hi + 1) - 1)
        b = sc.bounds()
        assert v0 == b["y_min"] >> 2 and v1 == (b["y_max"] - 3) // 4, (i, v0, v1, b)
        checked += 1
    assert checked >= 4


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [0, 1, 10, 11])
def test_clip_paths_on_the_device_match_oracle_as_shipped(backend, oracle, rrb_lib, seed):
    rng = np.random.default_rng(seed)
    paths, rule, gray, alpha, rects, clips = (_batch if seed < 10 else _batch_stacks)(rng, 18)
    exp = _expected(oracle, paths, rule, gray, alpha, rects, clips, rowmap=1)
    pages = backend.alloc_device(W * H)
    keep = []
    params, _ = _params(rrb_lib, paths, rule, gray, alpha, keep, pages)
    params.rowmap = rrb_lib.RRB_ROWMAP_AS_SHIPPED
    try:
        backend.begin_page()
        try:
            backend.record_fill_buffer(pages, 255)
            backend.record_path_batch_clip_paths(params, clips, rects)
        finally:
            backend.wait_page(backend.submit_page())
        got = np.empty(W * H, np.uint8)
        backend.wait_download(backend.download_async(pages, got))
    finally:
        backend.free_device(pages)
    assert np.array_equal(got.reshape(H, W), exp)
    assert (exp != 255).any()
