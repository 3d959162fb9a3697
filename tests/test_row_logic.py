"""Device logic of the fill path on the CPU. flatten_curve (flatten.rs:109-215),
make_edge + edge_entry (add_segment, aa_scale and fill_intersections,
xpath.rs:283-402, scanner/mod.rs:511-587), walk_row (render_aa_line,
scanner/mod.rs:393-467) and sweep_cells (the 4x4 coverage of draw_aa_line,
fill/mod.rs:344-401, from spans) are __host__ __device__ functions;
tests/row_logic_shim.cu calls the same source on the host. Each is checked
against the oracle on seeded inputs: flattened points bit for bit, every AA
row's merged and sorted entries, every AA row's spans against the oracle's
AaBuf bits, and every pixel row's cells against its 0..16 coverage. The
hairline span functions (stroke_narrow / draw_narrow_span,
stroke/mod.rs:95-256) are checked by the pages they paint.
"""

import ctypes as C
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
SHIM = ROOT / "tests" / "row_logic_shim.cu"


@pytest.fixture(scope="module")
def shim(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(nvcc).exists():
        pytest.skip("nvcc not found")
    out = tmp_path_factory.mktemp("row_logic") / "librow_logic.so"
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17", "-shared",
                    "-Xcompiler", "-fPIC,-ffp-contract=off", "-I", str(ROOT / "include"), "-o", str(out), str(SHIM)],
                   check=True, cwd=str(ROOT))
    lib = C.CDLL(str(out))
    i32p = C.POINTER(C.c_int32)
    lib.rl_walk_row.argtypes = [i32p, i32p, i32p, C.c_int, C.c_int, C.c_int32, C.c_int32, C.c_int32, i32p, i32p,
                                C.POINTER(C.c_uint32)]
    lib.rl_walk_row.restype = C.c_int
    lib.rl_sweep_cells.argtypes = [i32p, i32p, i32p, C.c_int, C.POINTER(C.c_uint32)]
    lib.rl_sweep_cells.restype = C.c_int
    dp = C.POINTER(C.c_double)
    lib.rl_flatten_curve.argtypes = [dp, C.c_double, dp, C.c_int]
    lib.rl_flatten_curve.restype = C.c_int
    lib.rl_flatten_curve_lanes.argtypes = [dp, C.c_double, dp, C.c_int, dp, C.POINTER(C.c_int)]
    lib.rl_flatten_curve_lanes.restype = C.c_int
    lib.rl_make_edges.argtypes = [dp, C.c_int, C.c_int32, C.c_int32, i32p]
    lib.rl_make_edges.restype = None
    lib.rl_row_entries.argtypes = [i32p, C.c_int, C.c_int32, i32p]
    lib.rl_row_entries.restype = C.c_int
    lib.rl_hairline_spans.argtypes = [dp, C.c_uint32, C.c_uint32, dp, i32p]
    lib.rl_hairline_spans.restype = C.c_int
    lib.rl_recti_spans.argtypes = [i32p, C.c_int, C.c_int, C.c_int32, C.c_int32, C.c_int32, C.c_int32, i32p, i32p,
                                   C.POINTER(C.c_uint32)]
    lib.rl_recti_spans.restype = C.c_int
    lib.rl_recti_box.argtypes = [i32p, C.c_int, C.c_int, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, i32p]
    lib.rl_recti_box.restype = C.c_int
    lib.rl_xpath_segments.argtypes = [dp, C.POINTER(C.c_uint8), C.c_uint64, dp, C.c_double, dp, C.c_int64]
    lib.rl_xpath_segments.restype = C.c_int64
    return lib


def _i32(a):
    return np.ascontiguousarray(a, np.int32)


def walk(shim, row, eo, aa_width):
    """Spans (x0, x1 exclusive) of one AA row's sorted entries, and whether it ran out."""
    n = len(row)
    x0 = _i32([r[0] for r in row] or [0])
    x1 = _i32([r[1] for r in row] or [0])
    cn = _i32([r[2] for r in row] or [0])
    s0 = np.zeros(max(1, n), np.int32)
    s1 = np.zeros(max(1, n), np.int32)
    nt = C.c_uint32()
    p = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
    ns = shim.rl_walk_row(p(x0), p(x1), p(cn), n, int(eo), aa_width, 0, aa_width, p(s0), p(s1), C.byref(nt))
    return list(zip(s0[:ns].tolist(), s1[:ns].tolist())), nt.value


def sweep(shim, spans4):
    """Cells of one pixel row from its four AA rows' spans, expanded to coverage per pixel."""
    stride = max(1, max(len(s) for s in spans4))
    x0 = np.zeros(4 * stride, np.int32)
    x1 = np.zeros(4 * stride, np.int32)
    for k, sp in enumerate(spans4):
        for i, (a, b) in enumerate(sp):
            x0[k * stride + i], x1[k * stride + i] = a, b
    n4 = _i32([len(s) for s in spans4])
    cells = np.zeros(4 * max(1, int(n4.sum())), np.uint32)
    p = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
    nc = shim.rl_sweep_cells(p(n4), p(x0), p(x1), stride, cells.ctypes.data_as(C.POINTER(C.c_uint32)))
    assert nc <= 4 * int(n4.sum())
    return cells[:nc]


def coverage_of(cells, width):
    cov = np.zeros(width, np.int32)
    last = -1
    for c in cells.tolist():
        x0, ln, cv = c & 0x3FFF, ((c >> 14) & 0x3FFF) + 1, (c >> 28) + 1
        assert x0 > last, "cells sorted and disjoint"
        last = x0 + ln - 1
        cov[x0:min(width, x0 + ln)] = cv
    return cov


def random_path(rng, w, h, closed=True):
    """1-3 subpaths of lines and cubics, vertices partly outside the page;
    closed=False leaves every subpath open (no return to its first point)."""
    pts, fl = [], []
    for _ in range(int(rng.integers(1, 4))):
        start = len(fl)
        cur = rng.uniform([-5, -5], [w + 5, h + 5])
        pts.append(cur)
        fl.append(1)
        for _ in range(int(rng.integers(2, 9))):
            nxt = rng.uniform([-8, -8], [w + 8, h + 8])
            if rng.random() < 0.35:
                pts += [cur + rng.normal(0, 12, 2), nxt + rng.normal(0, 12, 2), nxt]
                fl += [8, 8, 0]
            else:
                pts.append(nxt)
                fl.append(0)
            cur = nxt
        if closed:
            if not np.array_equal(pts[start], pts[-1]):
                pts.append(np.array(pts[start], float))
                fl.append(0)
            fl[start] |= 4
            fl[-1] |= 4
        fl[-1] |= 2
    return np.array(pts, float), np.array(fl, np.uint8)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_walk_and_sweep_match_oracle(oracle, shim, seed):
    rng = np.random.default_rng(seed)
    W, H = 48, 40
    aw = 4 * W
    rows_checked = ran_out = 0
    for i in range(40):
        # Open paths without the implicit close leave rows whose winding never returns to 0.
        close = i % 5 != 4
        pts, fl = random_path(rng, W, H, closed=close)
        eo = bool(i % 3 == 0)
        segs = oracle.xpath_new(pts, fl, flatness=0.25, close=close, aa_scale=True)
        sc = oracle.Scanner(segs, eo, 0, 4 * H - 1)
        for y in range(H):
            bits, _, st = sc.render_aa_line(aw, y)
            spans4, nt_sum = [], 0
            for k in range(4):
                spans, nt = walk(shim, sc.row(4 * y + k), eo, aw)
                line = np.zeros(aw, bool)
                for a, b in spans:
                    assert 0 <= a < b <= aw
                    line[a:b] = True
                assert np.array_equal(np.packbits(line), bits[k]), (i, y, k)
                spans4.append(spans)
                nt_sum += nt
            assert nt_sum == st.nonterminating_rows
            ran_out += nt_sum
            want = oracle.aa_coverage_span(bits, 0, W).astype(np.int32)
            assert np.array_equal(coverage_of(sweep(shim, spans4), W), want), (i, y)
            rows_checked += 1
    assert rows_checked == 40 * H
    if seed == 0:
        assert ran_out > 0  # the open paths exercised the unclosed-span arm


def test_sweep_cell_edges(oracle, shim):
    """Spans ending on pixel boundaries, one-column spans, spans covering a
    whole pixel in one sub-row only, and empty sub-rows."""
    cases = [
        [[(0, 4)], [(0, 4)], [(0, 4)], [(0, 4)]],
        [[(3, 5)], [], [(4, 8)], [(7, 8)]],
        [[(1, 2), (5, 6), (9, 10)], [(0, 12)], [], [(2, 3)]],
        [[(0, 40)], [(0, 40)], [(0, 40)], [(0, 39)]],
        [[], [], [], []],
    ]
    W = 12
    for spans4 in cases:
        bits = np.zeros((4, (4 * W + 7) // 8), np.uint8)
        for k, sp in enumerate(spans4):
            line = np.zeros(4 * W, bool)
            for a, b in sp:
                line[a:b] = True
            bits[k] = np.packbits(line)
        want = oracle.aa_coverage_span(bits, 0, W).astype(np.int32)
        assert np.array_equal(coverage_of(sweep(shim, spans4), W), want), spans4


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def test_flatten_curve_matches_oracle(oracle, shim):
    """The same points, bit for bit, for ordinary, tiny, huge (beyond f64::MAX/2,
    the midpoint's other branches) and degenerate cubics."""
    rng = np.random.default_rng(5)
    out = np.zeros(2 * 1025, np.float64)
    for i in range(3000):
        scale = [1e-3, 1.0, 40.0, 3000.0, 1e308][i % 5]
        c = np.clip(rng.normal(0, 1, 8), -1.5, 1.5) * scale
        if i % 7 == 0:
            c[2:4] = c[0:2]  # a control point on the start
        if i % 11 == 0:
            c[:] = c[0]  # all four points equal
        fsq = [0.01, 0.25, 1.0][i % 3]
        n = shim.rl_flatten_curve(_dp(np.ascontiguousarray(c)), fsq, _dp(out), 1025)
        want = oracle.flatten_curve(c[0:2], c[2:4], c[4:6], c[6:8], fsq)
        assert n == len(want), i
        assert np.array_equal(out[: 2 * n].view(np.uint64), np.ascontiguousarray(want).reshape(-1).view(np.uint64)), i


def test_flatten_split_over_lanes_matches_oracle(oracle, shim):
    """A curve split over the 32 lanes of a warp (the depth-5 subtrees of the
    subdivision, how k_seg_count_big / k_seg_write_big flatten curves of more
    than 32 segments) yields flatten_curve's points bit for bit, and each
    lane's first start point is the previous lane's last endpoint (or the
    curve's start)."""
    rng = np.random.default_rng(17)
    out = np.zeros(2 * 1025, np.float64)
    starts = np.zeros(64, np.float64)
    counts = (C.c_int * 32)()
    seen_big = 0
    for i in range(3000):
        scale = [1e-3, 1.0, 40.0, 3000.0, 1e308, 1e5][i % 6]
        c = np.clip(rng.normal(0, 1, 8), -1.5, 1.5) * scale
        if i % 7 == 0:
            c[2:4] = c[0:2]
        if i % 13 == 0:
            c[:] = c[0]
        fsq = [0.01, 0.25, 1.0, 1e-6][i % 4]
        n = shim.rl_flatten_curve_lanes(_dp(np.ascontiguousarray(c)), fsq, _dp(out), 1025, _dp(starts), counts)
        want = np.ascontiguousarray(oracle.flatten_curve(c[0:2], c[2:4], c[4:6], c[6:8], fsq)).reshape(-1)
        assert n == len(want) // 2, i
        assert np.array_equal(out[: 2 * n].view(np.uint64), want.view(np.uint64)), i
        k, prev = 0, c[0:2]
        for lane in range(32):
            if counts[lane]:
                assert np.array_equal(starts[2 * lane: 2 * lane + 2].view(np.uint64), np.asarray(prev).view(np.uint64))
                k += counts[lane]
                prev = want[2 * k - 2: 2 * k]
        seen_big += n > 32
    assert seen_big > 300


def _sat_inc(v):
    return v if v == 2**31 - 1 else v + 1


@pytest.mark.parametrize("seed", [3, 4])
def test_row_entries_match_scanner(oracle, shim, seed):
    """Per AA row: the entries of make_edge + edge_entry, merged in segment
    order with the last entry written (write_intersect) and stably sorted, are
    the oracle scanner's row."""
    rng = np.random.default_rng(seed)
    W, H = 48, 40
    for i in range(30):
        pts, fl = random_path(rng, W, H)
        segs = oracle.xpath_new(pts, fl, flatness=0.25, close=True)
        # Segments in walk order: add_segment stored flipped ones (OR_XF_FLIPPED = 4) with y0 <= y1.
        ends = np.array([(s.x1, s.y1, s.x0, s.y0) if s.flags & 4 else (s.x0, s.y0, s.x1, s.y1) for s in segs],
                        np.float64).reshape(-1)
        edges = np.zeros(8 * max(1, len(segs)), np.int32)
        shim.rl_make_edges(_dp(ends), len(segs), 0, 4 * H - 1, _ip(edges))
        scaled = oracle.xpath_new(pts, fl, flatness=0.25, close=True, aa_scale=True)
        sc = oracle.Scanner(scaled, bool(i % 2), 0, 4 * H - 1)
        buf = np.zeros(4 * max(1, len(segs)), np.int32)
        for r in range(4 * H):
            k = shim.rl_row_entries(_ip(edges), len(segs), r, _ip(buf))
            row = []
            for j in range(k):
                lo, hi, c = (int(v) for v in buf[4 * j + 1: 4 * j + 4])
                if row and _sat_inc(row[-1][1]) >= lo and row[-1][0] <= _sat_inc(hi):
                    a, b, cc = row[-1]
                    row[-1] = (min(a, lo), max(b, hi), (cc + c + 2**31) % 2**32 - 2**31)
                else:
                    row.append((lo, hi, c))
            row.sort(key=lambda e: e[0])  # stable, as the device's insertion sort
            assert row == [tuple(e) for e in sc.row(r)], (i, r)


class _OnePath:
    def __init__(self, pts, w, h):
        self.pts = np.asarray(pts, np.float64)
        self.flags = np.array([1, 2], np.uint8)
        self.path_pt_off = np.array([0, 2], np.uint64)
        self.fill_rule = np.zeros(1, np.uint8)
        self.gray = np.zeros(1, np.uint8)
        self.alpha = np.full(1, 255, np.uint8)
        self.path_page = np.zeros(1, np.uint32)
        self.page_width, self.page_height = np.array([w], np.uint32), np.array([h], np.uint32)
        self.page_offset = np.zeros(1, np.uint64)


def test_hairline_spans_match_oracle(oracle, shim):
    """One-segment hairlines (sloped, flat, vertical, short, partly or wholly
    off the page, with and without a clip rectangle): the spans of hl_segment
    and hl_row_span paint the oracle's page."""
    rng = np.random.default_rng(9)
    W, H = 40, 30
    out = np.zeros(3 * 4096, np.int32)
    for i in range(2000):
        p = rng.uniform([-12, -12], [W + 12, H + 12], (2, 2))
        if i % 6 == 1:
            p[1, 1] = p[0, 1]  # flat
        if i % 6 == 2:
            p[1, 0] = p[0, 0]  # vertical
        if i % 6 == 3:
            p[1] = p[0] + rng.normal(0, 0.7, 2)  # short
        rect = None
        if i % 3 == 0:
            a, b = rng.uniform([-5, -5], [W + 5, H + 5], (2, 2))
            rect = np.array([a[0], a[1], b[0], b[1]], np.float64)
        want = np.full(W * H, 255, np.uint8)
        oracle.render_scene_paint(_OnePath(p, W, H), want, [dict(line_width=0.0)],
                                  clip=None if rect is None else rect.reshape(1, 4))
        seg = np.ascontiguousarray(p.reshape(-1))
        k = shim.rl_hairline_spans(_dp(seg), W, H, None if rect is None else _dp(rect), _ip(out))
        got = np.full((H, W), 255, np.uint8)
        for j in range(k):
            y, a, b = (int(v) for v in out[3 * j: 3 * j + 3])
            assert 0 <= y < H and 0 <= a <= b < W, (i, y, a, b)
            got[y, a: b + 1] = 0
        assert np.array_equal(got, want.reshape(H, W)), i


def test_recti_row_spans_match_oracle(oracle, shim):
    """Rectilinear paths (1-4 rectangles with fractional corners, some
    overlapping or reversed, nonzero and even-odd): recti_row_spans sets every
    AA row's bits as render_aa_line does."""
    rng = np.random.default_rng(13)
    W, H = 40, 32
    aw = 4 * W
    s0 = np.zeros(64, np.int32)
    s1 = np.zeros(64, np.int32)
    nt = C.c_uint32()
    for i in range(150):
        subs = []
        for _ in range(int(rng.integers(1, 5))):
            x0, y0 = rng.uniform([-6, -6], [W + 2, H + 2])
            x1, y1 = x0 + rng.uniform(0.3, 25), y0 + rng.uniform(0.3, 20)
            corners = [(x0, y0), (x1, y0), (x1, y1), (x0, y1)]
            if rng.random() < 0.4:
                corners = corners[::-1]  # the other winding direction
            subs.append(corners)
        pts, fl = _path_closed(subs)
        eo = bool(i % 2)
        segs = oracle.xpath_new(pts, fl, flatness=0.25, close=True)
        assert len(segs) <= 32
        ends = np.array([(s.x1, s.y1, s.x0, s.y0) if s.flags & 4 else (s.x0, s.y0, s.x1, s.y1) for s in segs],
                        np.float64).reshape(-1)
        edges = np.zeros(8 * max(1, len(segs)), np.int32)
        shim.rl_make_edges(_dp(ends), len(segs), 0, 4 * H - 1, _ip(edges))
        sc = oracle.Scanner(oracle.xpath_new(pts, fl, flatness=0.25, close=True, aa_scale=True), eo, 0, 4 * H - 1)
        for y in range(H):
            bits, _, _ = sc.render_aa_line(aw, y)
            for k in range(4):
                ns = shim.rl_recti_spans(_ip(edges), len(segs), int(eo), 4 * y + k, aw, 0, aw, _ip(s0), _ip(s1),
                                         C.byref(nt))
                line = np.zeros(aw, bool)
                for a, b in zip(s0[:ns].tolist(), s1[:ns].tolist()):
                    line[a:b] = True
                assert np.array_equal(np.packbits(line), bits[k]), (i, y, k)


def test_box_coverage_matches_oracle(oracle, shim):
    """Rectangles (fractional corners, partly off the page, either winding,
    both rules) and other rectilinear paths: whenever the box test
    (recti_events + recti_box) accepts a path, the composite's closed form
    cx * cy reproduces every pixel the oracle paints, under both row maps;
    single on-page rectangles are always accepted, and paths whose rows differ
    are refused."""
    rng = np.random.default_rng(29)
    W, H = 48, 40
    aw = 4 * W
    gamma = oracle.aa_gamma()
    inv = {255 - int(g): k for k, g in enumerate(gamma)}  # page value after one opaque black layer -> coverage
    out = np.zeros(4, np.int32)
    boxes = refused = 0
    for i in range(300):
        kind = i % 3
        subs = []
        x0, y0 = rng.uniform([-8, -8], [W + 2, H + 2])
        x1, y1 = x0 + rng.uniform(0.2, 30), y0 + rng.uniform(0.2, 26)
        subs.append([(x0, y0), (x1, y0), (x1, y1), (x0, y1)])
        if kind == 1:  # a second rectangle beside or below: an L, a stack or two disjoint boxes
            a0, b0 = rng.uniform([-4, -4], [W, H])
            a1, b1 = a0 + rng.uniform(0.5, 20), b0 + rng.uniform(0.5, 15)
            if rng.random() < 0.3:
                a0, a1 = x0, x1  # stacked on the same columns: still one box where the two touch or overlap
            subs.append([(a0, b0), (a1, b0), (a1, b1), (a0, b1)])
        if kind == 2 and rng.random() < 0.5:
            subs[0] = subs[0][::-1]
        pts, fl = _path_closed(subs)
        eo = bool(rng.integers(0, 2))
        segs = oracle.xpath_new(pts, fl, flatness=0.1, close=True)
        ends = np.array([(s.x1, s.y1, s.x0, s.y0) if s.flags & 4 else (s.x0, s.y0, s.x1, s.y1) for s in segs],
                        np.float64).reshape(-1)
        edges = np.zeros(8 * max(1, len(segs)), np.int32)
        shim.rl_make_edges(_dp(ends), len(segs), 0, 4 * H - 1, _ip(edges))
        e = edges.reshape(-1, 8)[: len(segs)]
        live = e[(e[:, 2] & 16) == 0]
        if not len(live) or np.any((live[:, 2] & 3) == 2):
            continue  # no rows on the page, or a sloped edge (not a rectilinear path)
        ay0, ay1 = int(live[:, 0].min()), int(live[:, 1].max())
        is_box = shim.rl_recti_box(_ip(edges), len(segs), int(eo), ay0, ay1, aw, 0, aw, _ip(out))
        on_page = kind != 1 and 0 <= x0 and x1 <= W and 0 <= y0 and y1 <= H
        # Edges in adjacent AA columns (or rows) merge into one zero-count entry
        # that paints nothing, so only rectangles at least two AA units across
        # must be boxes.
        if on_page and np.floor(4 * x1) - np.floor(4 * x0) >= 2 and np.floor(4 * y1) - np.floor(4 * y0) >= 2:
            assert is_box, (i, subs)
        for rowmap in (0, 1):
            page = np.full((H, W), 255, np.uint8)
            oracle.fill_path(page, pts, fl, eo=eo, gray=0, alpha=255, rowmap=rowmap)
            cov = np.vectorize(inv.get)(page)
            if is_box:
                s0, s1, r0, r1 = (int(v) for v in out)
                assert ay0 <= r0 <= r1 <= ay1
                xs = 4 * np.arange(W)
                cx = np.clip(np.minimum(xs + 4, s1) - np.maximum(xs, s0), 0, None)
                ys = 16 * np.arange(H) + 12 if rowmap else 4 * np.arange(H)
                cy = np.clip(np.minimum(ys + 4, r1 + 1) - np.maximum(ys, r0), 0, None)
                if rowmap:  # the shipped loop visits pixel row y only when AA row 4y+3 is in the scanner's range
                    vis = 4 * np.arange(H) + 3
                    cy[(vis < ay0) | (vis > ay1)] = 0
                assert np.array_equal(cov, np.outer(cy, cx)), (i, rowmap, subs)
        boxes += bool(is_box)
        refused += not is_box
    assert boxes > 150 and refused > 20


def _path_closed(subpaths):
    pts, fl = [], []
    for sp in subpaths:
        start = len(fl)
        for j, p in enumerate(sp):
            pts.append(p)
            fl.append(1 if j == 0 else 0)
        pts.append(sp[0])
        fl.append(0)
        fl[start] |= 4
        fl[-1] |= 4 | 2
    return np.array(pts, float), np.array(fl, np.uint8)


def test_host_xpath_walk_matches_oracle(oracle, shim):
    """The clip-path lowering's host walk (k_walk + k_seg_write restated) gives
    XPath::new's segments bit for bit: lines, cubics, subpaths that close by
    a segment or within 1e-10, a curve end marked LAST (the walk runs on into
    the next subpath), transforms and flatness."""
    rng = np.random.default_rng(17)
    out = np.zeros(4 * 20000, np.float64)
    for i in range(400):
        pts, fl = random_path(rng, 60, 50, closed=i % 4 != 3)
        if i % 9 == 0 and (fl & 8).any():
            j = int(np.nonzero(fl & 8)[0][-1]) + 1  # the end point after the last control pair
            if j < len(fl):
                fl = fl.copy()
                fl[j] |= 2
        if i % 11 == 0:
            pts = pts.copy()
            pts[-1] = pts[0] + rng.choice([0.0, 3e-11, -5e-11, 2e-10], 2)
        m = (1.0, 0.0, 0.0, 1.0, 0.0, 0.0) if i % 3 else tuple(rng.normal(0, 1, 6))
        flat = float(rng.choice([0.1, 0.3, 1.0]))
        p = np.ascontiguousarray(pts, np.float64).reshape(-1)
        f = np.ascontiguousarray(fl, np.uint8)
        mm = np.array(m, np.float64)
        n = shim.rl_xpath_segments(_dp(p), f.ctypes.data_as(C.POINTER(C.c_uint8)), f.size, _dp(mm), flat, _dp(out),
                                   20000)
        want = oracle.xpath_new(pts, fl, matrix=m, flatness=flat, close=True)
        assert n == len(want), i
        # add_segment stores flipped segments with y0 <= y1 (OR_XF_FLIPPED = 4): compare in walk order.
        exp = np.array([(s.x1, s.y1, s.x0, s.y0) if s.flags & 4 else (s.x0, s.y0, s.x1, s.y1) for s in want],
                       np.float64).reshape(-1)
        assert np.array_equal(out[: 4 * n].view(np.uint64), exp.view(np.uint64)), i
