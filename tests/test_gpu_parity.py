"""GPU parity: the B200 path through the C ABI against the CPU oracle, bit for bit.

Every comparison is exact (np.array_equal on u8 pages): coverage, winding and
div255 compositing are integer work, and the FP64 flattening follows the
reference's operation order, so any differing pixel is a bug.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROWMAPS = [0, 1]


def _oracle_arena(oracle, scene, rowmap, init=255, threads=8):
    a = scene.blank_arena(init)
    st = oracle.render_scene(scene, a, rowmap=rowmap, threads=threads)
    return a, st


def _gpu_arena(backend, scene, rowmap, init=255):
    a = scene.blank_arena(init)
    backend.render_scene(scene, a, rowmap=rowmap)
    return a


def _diff(a, b):
    d = np.nonzero(a != b)[0]
    return f"{d.size} differing bytes, first at {d[:5]}" if d.size else "equal"


# ---- single paths through rrb_record_path_fill --------------------------------------

def _paths(rrb):
    """Hand-made paths covering the edge cases of the scanline rules."""
    out = {}

    def mk(name, ops):
        b = rrb.PathBuilder()
        for op, *a in ops:
            getattr(b, op)(*a)
        out[name] = b.build()

    mk("triangle", [("move_to", 3.2, 2.7), ("line_to", 40.9, 5.1), ("line_to", 20.4, 37.3), ("close",)])
    mk("rect_frac", [("move_to", 5.3, 4.8), ("line_to", 50.55, 4.8), ("line_to", 50.55, 30.1), ("line_to", 5.3, 30.1),
                     ("close",)])
    mk("rect_int", [("move_to", 8, 8), ("line_to", 24, 8), ("line_to", 24, 20), ("line_to", 8, 20), ("close",)])
    mk("curves", [("move_to", 10, 30), ("curve_to", 10, 0, 60, 0, 60, 30), ("curve_to", 60, 55, 10, 55, 10, 30),
                  ("close",)])
    mk("donut", [("move_to", 5, 5), ("line_to", 55, 5), ("line_to", 55, 45), ("line_to", 5, 45), ("close",),
                 ("move_to", 15, 15), ("line_to", 45, 15), ("line_to", 45, 35), ("line_to", 15, 35), ("close",)])
    mk("star", [("move_to", 30, 2), ("line_to", 47, 52), ("line_to", 3, 20), ("line_to", 57, 20), ("line_to", 13, 52),
                ("close",)])
    mk("offpage", [("move_to", -40, -30), ("line_to", -5, -30), ("line_to", -5, -2), ("close",)])
    mk("partial", [("move_to", -20.5, 10.25), ("line_to", 30.75, -12.5), ("line_to", 120.2, 70.6), ("close",)])
    mk("beyond", [("move_to", 70, 10), ("line_to", 200, 10), ("line_to", 200, 90), ("close",)])
    mk("sliver", [("move_to", 10.1, 3), ("line_to", 10.3, 3), ("line_to", 10.3, 50), ("line_to", 10.1, 50),
                  ("close",)])
    mk("horiz_line", [("move_to", 3, 10.5), ("line_to", 50, 10.5), ("close",)])
    mk("point", [("move_to", 7, 7), ("close",)])
    mk("quirk", [("move_to", 5, 5), ("line_to", 30, 5), ("curve_to", 30, 20, 15, 30, 5, 5), ("close",),
                 ("move_to", 35, 35), ("line_to", 55, 35), ("line_to", 55, 55), ("close",)])
    mk("conics", [("move_to", 10, 20), ("conic_to", 30, -5, 50, 20), ("conic_to", 30, 45, 10, 20), ("close",)])
    mk("overlap_winding", [("move_to", 5, 5), ("line_to", 40, 5), ("line_to", 40, 40), ("line_to", 5, 40), ("close",),
                           ("move_to", 20, 20), ("line_to", 55, 20), ("line_to", 55, 55), ("line_to", 20, 55),
                           ("close",)])
    mk("huge", [("move_to", -1e7, -1e7), ("line_to", 1e7, -3e6), ("line_to", 2e6, 1e7), ("close",)])
    # A comb: one contour with 40 teeth, so AA rows carry ~80 merged entries
    # (exercises the rows whose list does not fit in shared memory).
    ops = [("move_to", 2.0, 2.0)]
    x = 2.0
    for i in range(40):
        ops += [("line_to", x + 0.7, 2.0), ("line_to", x + 0.7, 50.0), ("line_to", x + 1.3, 50.0),
                ("line_to", x + 1.3, 2.0)]
        x += 1.45
    ops += [("line_to", x, 2.0), ("line_to", x, 58.0), ("line_to", 2.0, 58.0), ("close",)]
    mk("comb", ops)
    return out


@pytest.fixture(scope="module")
def paths(rrb_lib):
    return _paths(rrb_lib)


@pytest.mark.parametrize("rowmap", ROWMAPS)
@pytest.mark.parametrize("rule", [0, 1])
def test_single_paths(backend, oracle, rrb_lib, paths, rowmap, rule):
    W, H = 97, 61
    rng = np.random.default_rng(5)
    init = rng.integers(0, 256, (H, W), dtype=np.uint8)
    buf = backend.alloc_device(W * H)
    try:
        for i, (name, (pts, fl)) in enumerate(sorted(paths.items())):
            gray, alpha = int(rng.integers(0, 256)), int(rng.choice([255, 200, 37]))
            exp = init.copy()
            oracle.fill_path(exp, pts, fl, eo=bool(rule), gray=gray, alpha=alpha, rowmap=rowmap)
            backend.upload_async(buf, init)
            backend.begin_page()
            backend.record_path_fill(pts, fl, buf, W, H, fill_rule=rule, gray=gray, alpha=alpha, rowmap=rowmap)
            f = backend.submit_page()
            backend.wait_page(f)
            got = np.empty_like(init)
            backend.wait_download(backend.download_async(buf, got))
            assert np.array_equal(got, exp), f"{name}: {_diff(got.ravel(), exp.ravel())}"
    finally:
        backend.free_device(buf)


def test_comb_takes_the_slow_row_path(backend, rrb_lib, paths):
    pts, fl = paths["comb"]
    W, H = 97, 61
    buf = backend.alloc_device(W * H)
    try:
        backend.begin_page()
        backend.record_path_fill(pts, fl, buf, W, H)
        backend.wait_page(backend.submit_page())
        assert backend.last_batch_stats()["row_overflows"] > 0
    finally:
        backend.free_device(buf)


# ---- scenes through rrb_record_path_batch -------------------------------------------

SMALL = {
    "polygons": dict(kind=0, seed=3, n_paths=300, page_w=640, page_h=480),
    "glyphs": dict(kind=1, seed=4, n_paths=4000, page_w=800, page_h=600),
    "mixed": dict(kind=2, seed=5, n_pages=6, page_scale=0.15, paths_scale=0.03),
}


@pytest.mark.parametrize("rowmap", ROWMAPS)
@pytest.mark.parametrize("name", list(SMALL))
def test_small_scenes(backend, oracle, rrb_lib, name, rowmap):
    s = rrb_lib.Scene(**SMALL[name])
    exp, _ = _oracle_arena(oracle, s, rowmap)
    got = _gpu_arena(backend, s, rowmap)
    assert np.array_equal(got, exp), _diff(got, exp)


@pytest.mark.parametrize("tile", [(16, 16), (32, 32), (64, 16), (128, 16), (128, 32)])
def test_tile_shapes_agree(backend, oracle, rrb_lib, tile):
    s = rrb_lib.Scene(kind=2, seed=9, n_pages=3, page_scale=0.12, paths_scale=0.04)
    exp, _ = _oracle_arena(oracle, s, 0)
    backend.set_tuning(*tile)
    try:
        got = _gpu_arena(backend, s, 0)
    finally:
        backend.set_tuning(64, 16, auto_tile=True)
    assert np.array_equal(got, exp), _diff(got, exp)


def test_plain_per_path_equals_batched(backend, rrb_lib):
    """The plain form (one record_path_fill per path) and the batch give the same page."""
    s = rrb_lib.Scene(kind=0, seed=21, n_paths=60, page_w=320, page_h=240)
    batched = _gpu_arena(backend, s, 0)
    W, H = int(s.page_width[0]), int(s.page_height[0])
    buf = backend.alloc_device(W * H)
    try:
        backend.upload_async(buf, np.full(W * H, 255, np.uint8))
        backend.begin_page()
        for p in range(s.n_paths):
            a, b = int(s.path_pt_off[p]), int(s.path_pt_off[p + 1])
            backend.record_path_fill(s.pts[a:b], s.flags[a:b], buf, W, H, fill_rule=int(s.fill_rule[p]),
                                     gray=int(s.gray[p]), alpha=int(s.alpha[p]))
        backend.wait_page(backend.submit_page())
        plain = np.empty(W * H, np.uint8)
        backend.wait_download(backend.download_async(buf, plain))
    finally:
        backend.free_device(buf)
    assert np.array_equal(plain, batched[: W * H])


def test_resident_batch_rerenders_identically(backend, oracle, rrb_lib):
    s = rrb_lib.Scene(kind=1, seed=8, n_paths=2500, page_w=640, page_h=400)
    exp, _ = _oracle_arena(oracle, s, 0)
    pages = backend.alloc_device(s.arena_bytes)
    s.view.pages = None
    batch = backend.batch_upload(s.view)
    try:
        for _ in range(3):
            backend.begin_page()
            backend.record_fill_buffer(pages, 255)
            batch.record(pages)
            backend.wait_page(backend.submit_page())
            got = np.empty(s.arena_bytes, np.uint8)
            backend.wait_download(backend.download_async(pages, got))
            assert np.array_equal(got, exp), _diff(got, exp)
    finally:
        batch.free()
        backend.free_device(pages)


# ---- full-size workloads --------------------------------------------------------------

@pytest.mark.parametrize("rowmap", ROWMAPS)
def test_full_polygon_page(backend, oracle, rrb_lib, rowmap):
    """2,000 paths on a Letter page at 300 dpi, seed 0."""
    s = rrb_lib.Scene(kind=0, seed=0)
    exp, st = _oracle_arena(oracle, s, rowmap)
    got = _gpu_arena(backend, s, rowmap)
    assert np.array_equal(got, exp), _diff(got, exp)
    assert backend.last_batch_stats()["segments"] == st["segments"]


def test_full_glyph_page(backend, oracle, rrb_lib):
    """150,000 glyphs on one Letter page at 300 dpi, seed 0."""
    s = rrb_lib.Scene(kind=1, seed=0)
    exp, st = _oracle_arena(oracle, s, 0)
    got = _gpu_arena(backend, s, 0)
    assert np.array_equal(got, exp), _diff(got, exp)
    stats = backend.last_batch_stats()
    assert stats["segments"] == st["segments"] and stats["aa_rows"] == st["aa_rows"]


# ---- state machine and memory budget (GpuBackend contract) ---------------------------

def test_record_outside_page_is_a_state_error(backend, rrb_lib, paths):
    pts, fl = paths["triangle"]
    buf = backend.alloc_device(64 * 64)
    try:
        with pytest.raises(rrb_lib.BackendError) as e:
            backend.record_path_fill(pts, fl, buf, 64, 64)
        assert e.value.kind == "StateError"
    finally:
        backend.free_device(buf)


def test_zero_size_alloc_and_bounds(backend, rrb_lib):
    with pytest.raises(rrb_lib.BackendError) as e:
        backend.alloc_device(0)
    assert e.value.kind == "ZeroSizeAlloc"
    buf = backend.alloc_device(16)
    try:
        with pytest.raises(rrb_lib.BackendError) as e:
            backend.upload_async(buf, np.zeros(32, np.uint8))
        assert e.value.kind == "InvariantViolation"
    finally:
        backend.free_device(buf)


def test_memory_budget_is_enforced(rrb_lib):
    with rrb_lib.B200Backend(0, mem_budget=1 << 20) as b:
        x = b.alloc_device(1 << 19)
        with pytest.raises(rrb_lib.BackendError) as e:
            b.alloc_device(1 << 20)
        assert e.value.kind == "OutOfMemory"
        assert b.detect_vram_budget().used_bytes >= 1 << 19
        b.free_device(x)


# ---- overdraw: rectilinear runs, full-tile layers, opaque occlusion, waves ----------

def _stacked_rects(rrb, W, H, n, seed):
    """Rectangles covering most of the page (some opaque, most translucent) with
    polygons in between: full-tile layer runs, occluding opaque layers, and
    rectangle edges inside tiles."""
    rng = np.random.default_rng(seed)
    pts, flags, off, rule, gray, alpha = [], [], [0], [], [], []
    for i in range(n):
        b = rrb.PathBuilder()
        if i % 5 == 3:
            cx, cy, r = rng.uniform(0, W), rng.uniform(0, H), rng.uniform(5, 40)
            b.move_to(cx + r, cy)
            for k in range(1, 9):
                t = 2 * np.pi * k / 9
                b.curve_to(cx + r * np.cos(t - 0.3), cy + r * np.sin(t - 0.3), cx + r * np.cos(t - 0.1),
                           cy + r * np.sin(t - 0.1), cx + r * np.cos(t), cy + r * np.sin(t))
            b.close()
        else:
            x0, y0 = rng.uniform(-10, W * 0.3), rng.uniform(-10, H * 0.3)
            x1, y1 = rng.uniform(W * 0.6, W + 10), rng.uniform(H * 0.6, H + 10)
            if i % 7 == 1:  # counter-clockwise and integral
                x0, y0, x1, y1 = float(int(x0)), float(int(y0)), float(int(x1)), float(int(y1))
                b.move_to(x0, y0)
                b.line_to(x0, y1)
                b.line_to(x1, y1)
                b.line_to(x1, y0)
            else:
                b.move_to(x0, y0)
                b.line_to(x1, y0)
                b.line_to(x1, y1)
                b.line_to(x0, y1)
            b.close()
        p, f = b.build()
        pts.append(p)
        flags.append(f)
        off.append(off[-1] + len(f))
        rule.append(i % 2)
        gray.append(int(rng.integers(0, 256)))
        alpha.append(255 if i % 11 == 5 else int(rng.integers(32, 255)))
    return (np.concatenate(pts), np.concatenate(flags), np.array(off, np.uint64), np.array(rule, np.uint8),
            np.array(gray, np.uint8), np.array(alpha, np.uint8))


@pytest.mark.parametrize("rowmap", ROWMAPS)
@pytest.mark.parametrize("tile", [(16, 16), (32, 32), (64, 16), (128, 16), (128, 32)])
def test_stacked_rectangles(backend, oracle, rrb_lib, rowmap, tile):
    W, H = 211, 157
    pts, flags, off, rule, gray, alpha = _stacked_rects(rrb_lib, W, H, 60, seed=7)
    n = len(rule)
    init = np.random.default_rng(1).integers(0, 256, W * H, dtype=np.uint8)
    exp = init.copy()
    oracle.render_arrays(exp, [0], [W], [H], pts, flags, off, rule, gray, alpha, np.zeros(n, np.uint32), rowmap=rowmap)
    buf = backend.alloc_device(W * H)
    keep = []
    backend.set_tuning(*tile)
    try:
        p = rrb_lib.batch_params(pts, flags, off, rule, gray, alpha, np.zeros(n, np.uint32), [W], [H], [0], buf,
                                 rowmap=rowmap, keep=keep)
        got = init.copy()
        backend.render_pages_host(p, got)
    finally:
        backend.set_tuning(64, 16, auto_tile=True)
        backend.free_device(buf)
    assert np.array_equal(got, exp), _diff(got, exp)


def test_waves_match_oracle(backend, oracle, rrb_lib):
    """Pages processed in several memory waves give the same pages."""
    s = rrb_lib.Scene(kind=2, seed=13, n_pages=7, page_scale=0.12, paths_scale=0.03)
    exp, _ = _oracle_arena(oracle, s, 0)
    backend.set_tuning(wave_points=max(1000, s.n_pts // 5))
    try:
        got = _gpu_arena(backend, s, 0)
    finally:
        backend.set_tuning(wave_points=0)
    assert np.array_equal(got, exp), _diff(got, exp)


def _page_subscene(s, pages):
    """Arrays of the paths of `pages` of scene `s`, with their own page arena."""
    sel = np.isin(s.path_page, pages)
    idx = np.nonzero(sel)[0]
    pts, flags, off = [], [], [0]
    for p in idx:
        a, b = int(s.path_pt_off[p]), int(s.path_pt_off[p + 1])
        pts.append(s.pts[a:b])
        flags.append(s.flags[a:b])
        off.append(off[-1] + b - a)
    remap = {pg: i for i, pg in enumerate(pages)}
    w = np.array([s.page_width[pg] for pg in pages], np.uint32)
    h = np.array([s.page_height[pg] for pg in pages], np.uint32)
    po = np.concatenate([[0], np.cumsum(w.astype(np.uint64) * h)[:-1]]).astype(np.uint64)
    return dict(pts=np.concatenate(pts), flags=np.concatenate(flags), path_pt_off=np.array(off, np.uint64),
                fill_rule=s.fill_rule[idx], gray=s.gray[idx], alpha=s.alpha[idx],
                path_page=np.array([remap[int(x)] for x in s.path_page[idx]], np.uint32),
                page_width=w, page_height=h, page_offset=po, arena=int(np.sum(w.astype(np.uint64) * h)))


def test_full_mixed_pages(backend, oracle, rrb_lib):
    """64 mixed pages (1.17 Gpx, 662k paths) in one batch: the two smallest pages
    against the oracle byte for byte, and the whole arena identical when the
    batch is split into waves."""
    s = rrb_lib.Scene(kind=2, seed=0)
    got = _gpu_arena(backend, s, 0)
    sizes = s.page_width.astype(np.int64) * s.page_height
    small = [int(i) for i in np.argsort(sizes, kind="stable")[:2]]
    sub = _page_subscene(s, small)
    exp = np.full(sub["arena"], 255, np.uint8)
    oracle.render_arrays(exp, sub["page_offset"], sub["page_width"], sub["page_height"], sub["pts"], sub["flags"],
                         sub["path_pt_off"], sub["fill_rule"], sub["gray"], sub["alpha"], sub["path_page"], threads=2)
    for i, pg in enumerate(small):
        o, n = int(s.page_offset[pg]), int(sizes[pg])
        oo = int(sub["page_offset"][i])
        assert np.array_equal(got[o:o + n], exp[oo:oo + n]), f"page {pg}: {_diff(got[o:o + n], exp[oo:oo + n])}"
    backend.set_tuning(wave_points=s.n_pts // 6)
    try:
        waved = _gpu_arena(backend, s, 0)
    finally:
        backend.set_tuning(wave_points=0)
    assert np.array_equal(waved, got), _diff(waved, got)
