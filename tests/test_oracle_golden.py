"""Pin the CPU oracle against every known answer the reference holds for the path.

Each test names the reference unit test it restates (file:line within
pthomasfournet/pdf-raster). The reference is Rust and cannot run here, so
these vectors are read from its test sources; together with the hand-derived
rectangle coverage below they pin the restatement that the GPU path is then
compared against bit for bit.
"""

import math
from fractions import Fraction

import numpy as np
import pytest


@pytest.fixture(scope="module")
def O(oracle):
    return oracle


# ---- xpath.rs tests (crates/raster/src/xpath.rs:506-680) -----------------------------

def test_horizontal_segment_not_flipped(O):  # xpath.rs:506-518
    s = O.add_segment(0.0, 5.0, 10.0, 5.0)
    assert s.flags & O.XF_HORIZ and not s.flags & O.XF_FLIPPED
    assert s.y0 == 5.0 and s.y1 == 5.0


def test_downward_segment_flipped(O):  # xpath.rs:520-531
    s = O.add_segment(0.0, 10.0, 0.0, 0.0)
    assert s.flags & O.XF_FLIPPED and s.y0 <= s.y1


def test_aa_scale_multiplies_coords(O):  # xpath.rs:533-550
    b = O.OraclePath()
    b.move_to(1.0, 0.0)
    b.line_to(3.0, 2.0)
    pts, fl = b.build()
    segs = O.xpath_new(pts, fl, close=False, aa_scale=True)
    s = segs[0]
    assert (s.x0, s.y0, s.x1, s.y1) == (4.0, 0.0, 12.0, 8.0)
    assert s.dxdy == 1.0  # (3-1)/(2-0): unchanged by the scale


def test_vertical_segment_dxdy_zero(O):  # xpath.rs:552-562
    s = O.add_segment(5.0, 0.0, 5.0, 10.0)
    assert s.flags & O.XF_VERT and s.dxdy == 0.0


def test_triangle_from_path(O):  # xpath.rs:565-576
    b = O.OraclePath()
    b.move_to(0.0, 0.0)
    b.line_to(4.0, 0.0)
    b.line_to(2.0, 4.0)
    assert b.close(False) == 0
    pts, fl = b.build()
    assert len(O.xpath_new(pts, fl, flatness=1.0, close=False)) == 3


def test_degenerate_point_segment(O):  # xpath.rs:580-592
    s = O.add_segment(3.0, 7.0, 3.0, 7.0)
    assert s.flags & O.XF_HORIZ and s.flags & O.XF_VERT and not s.flags & O.XF_FLIPPED
    assert s.dxdy == 0.0 and math.copysign(1, s.dxdy) == 1


def test_sloped_segment_dxdy(O):  # xpath.rs:595-609
    s = O.add_segment(2.0, 1.0, 6.0, 5.0)
    assert s.flags == 0 and s.dxdy == 1.0


def test_flipped_sloped_segment_dxdy_consistent(O):  # xpath.rs:613-630
    s = O.add_segment(6.0, 5.0, 2.0, 1.0)
    assert s.flags & O.XF_FLIPPED and s.y0 <= s.y1 and s.dxdy == 1.0


@pytest.mark.parametrize("seg,fp", [((0.0, 0.0, 4.0, 4.0), 65536), ((0.0, 0.0, 2.0, 4.0), 32768),
                                    ((0.0, 2.0, 5.0, 2.0), 0), ((3.0, 0.0, 3.0, 5.0), 0)])
def test_dxdy_fp(O, seg, fp):  # xpath.rs:633-680
    assert O.add_segment(*seg).dxdy_fp == fp


def test_dxdy_fp_rounds_half_away_and_saturates(O):
    # (dxdy * 65536).round() as i32 with saturation (xpath.rs:376-391).
    assert O.add_segment(0.0, 0.0, 1.0, 131072.0).dxdy_fp == 1  # 0.5 -> 1
    assert O.add_segment(0.0, 0.0, -1.0, 131072.0).dxdy_fp == -1  # -0.5 -> -1
    assert O.add_segment(0.0, 0.0, 1e9, 1.0).dxdy_fp == 2**31 - 1
    assert O.add_segment(0.0, 0.0, -1e9, 1.0).dxdy_fp == -(2**31)


# ---- flatten.rs tests (crates/raster/src/path/flatten.rs:225-303) ----------------------

def test_flat_curve_emits_one_segment(O):  # flatten.rs:225-248
    out = O.flatten_curve((0, 0), (1, 0), (2, 0), (3, 0), 0.1)
    assert len(out) >= 1 and np.all(np.abs(out[:, 1]) < 1e-10)
    assert abs(out[-1, 0] - 3.0) < 1e-10


def test_endpoints_match_cubic(O):  # flatten.rs:250-266
    k = 0.55228475  # BEZIER_CIRCLE (types.rs:45)
    out = O.flatten_curve((0, 0), (0, k), (1 - k, 1), (1, 1), 0.01 * 0.01)
    assert abs(out[-1, 0] - 1.0) < 1e-10 and abs(out[-1, 1] - 1.0) < 1e-10


def test_does_not_exceed_max_curve_splits(O):  # flatten.rs:268-282
    out = O.flatten_curve((0, 0), (1e8, -1e8), (-1e8, 1e8), (0, 0), 0.25)
    assert len(out) <= 1024


def test_curve_to_line_is_two_points(O):  # flatten.rs:284-303
    o = (5.0, 7.0)
    out = O.flatten_curve(o, o, o, o, np.finfo(np.float64).eps)
    assert out.shape == (1, 2) and tuple(out[0]) == o


def test_flatten_last_point_is_p3_exactly(O):
    # The endpoint slot is written once at set-up, so the last point is p3 bit for bit.
    p3 = (123.456789, -987.654321)
    out = O.flatten_curve((0.1, 0.2), (50.3, 900.7), (-30.0, 5.5), p3, 0.01)
    assert tuple(out[-1]) == p3 and len(out) > 1


# ---- scanner tests (crates/raster/src/scanner/mod.rs:696-793) --------------------------

def _triangle(O, close=True):
    b = O.OraclePath()
    b.move_to(0.0, 0.0)
    b.line_to(4.0, 0.0)
    b.line_to(2.0, 4.0)
    b.close(False)
    pts, fl = b.build()
    return O.xpath_new(pts, fl, flatness=1.0, close=close)


def test_empty_on_no_segs(O):  # scanner/mod.rs:711-716
    assert O.Scanner([], False, 0, 10).bounds()["empty"]


def test_triangle_has_rows(O):  # scanner/mod.rs:718-724
    b = O.Scanner(_triangle(O), False, 0, 4).bounds()
    assert not b["empty"] and b["y_min"] <= b["y_max"]


def test_horizontal_segment_count_zero(O):  # scanner/mod.rs:726-732
    assert O.add_intersection([], 0, 5, 0)[0][2] == 0


def test_inside_outside_triangle(O):  # scanner/mod.rs:734-748
    sc = O.Scanner(_triangle(O), False, 0, 4)
    assert sc.test(2, 1)
    assert not sc.test(10, 2) and not sc.test(2, 5)


def test_row_out_of_range_returns_empty(O):  # scanner/mod.rs:750-761
    sc = O.Scanner(_triangle(O), False, 0, 4)
    b = sc.bounds()
    for y in (b["y_min"] - 1, b["y_max"] + 1, -(2**31), 2**31 - 1):
        assert sc.row(y) == []


def test_add_intersection_merge_adjacent(O):  # scanner/mod.rs:763-773
    row = O.add_intersection([], 0, 3, -1)
    row = O.add_intersection(row, 4, 7, 1)
    assert row == [(0, 7, 0)]


def test_add_intersection_disjoint(O):  # scanner/mod.rs:775-782
    row = O.add_intersection([], 0, 2, -1)
    assert len(O.add_intersection(row, 5, 7, -1)) == 2


def test_count_crossings(O):  # scanner/mod.rs:784-793 (and the next test)
    assert O.count_crossings([(2, 5, -1)], 3) == (0, True)
    assert O.count_crossings([(2, 5, -1)], 6) == (-1, False)


# ---- AaBuf + render_aa_line (bitmap.rs:462-573, scanner/mod.rs:393-467) ---------------

def test_aabuf_set_span_msb_first(O):
    buf = np.zeros(4 * 2, np.uint8)
    O.aabuf_set_span(buf, 16, 0, 3, 11)  # bits 3..10 of row 0
    assert buf[0] == 0b00011111 and buf[1] == 0b11100000
    O.aabuf_set_span(buf, 16, 1, 8, 16)  # byte-aligned right edge
    assert buf[2] == 0 and buf[3] == 0xFF
    O.aabuf_set_span(buf, 16, 2, 5, 5)  # empty
    assert buf[4] == 0 and buf[5] == 0


def test_render_aa_line_nonzero_vs_evenodd(O):
    # Two nested squares wound the same way: NZ fills the hole, EO does not.
    b = O.OraclePath()
    for (x0, y0, x1, y1) in ((0, 0, 8, 8), (2, 2, 6, 6)):
        b.move_to(x0, y0)
        b.line_to(x1, y0)
        b.line_to(x1, y1)
        b.line_to(x0, y1)
        b.close(False)
    pts, fl = b.build()
    segs = O.xpath_new(pts, fl, close=True, aa_scale=True)
    nz = O.Scanner(segs, False, 0, 63)
    eo = O.Scanner(segs, True, 0, 63)
    bn, (x0n, x1n), _ = nz.render_aa_line(64, 4)  # pixel row 4: AA rows 16..19
    be, (x0e, x1e), _ = eo.render_aa_line(64, 4)
    # Vertical edges enter as entries [floor(x), floor(x)] and a span ends at the
    # closing entry's x1 + 1, so the right edge's floor column is covered.
    assert (x0n, x1n) == (0, 8) and (x0e, x1e) == (0, 8)
    cov_n = O.aa_coverage_span(bn, 0, 16)
    cov_e = O.aa_coverage_span(be, 0, 16)
    assert list(cov_n[:9]) == [16] * 8 + [4]
    # EO: spans [0, 9) and [24, 33) in AA columns.
    assert list(cov_e[:9]) == [16, 16, 4, 0, 0, 0, 16, 16, 4]


# ---- fill/mod.rs AA_GAMMA (fill/mod.rs:515-538) -----------------------------------

def test_aa_gamma_table(O):
    g = O.aa_gamma()
    assert g == [0, 4, 11, 21, 32, 45, 59, 74, 90, 108, 126, 145, 166, 187, 209, 231, 255]
    assert g == [int(math.floor((i / 16) ** 1.5 * 255 + 0.5)) for i in range(17)]


# ---- aa_coverage.rs tests (crates/raster/src/simd/aa_coverage.rs:570-665) ---------

def _rows(r):
    return np.array(r, np.uint8)


def test_coverage_all_zero_all_ones(O):
    assert list(O.aa_coverage_span(_rows([[0] * 4] * 4), 0, 8)) == [0] * 8
    assert list(O.aa_coverage_span(_rows([[0xFF] * 4] * 4), 0, 8)) == [16] * 8


def test_coverage_single_pixel_even_odd(O):
    assert list(O.aa_coverage_span(_rows([[0xF0, 0, 0, 0]] + [[0] * 4] * 3), 0, 2)) == [4, 0]
    assert list(O.aa_coverage_span(_rows([[0x0F, 0, 0, 0]] + [[0] * 4] * 3), 0, 2)) == [0, 4]


def test_coverage_x0_offset(O):
    r = _rows([[0, 0xA0, 0, 0], [0, 0x50, 0, 0], [0] * 4, [0] * 4])
    assert O.aa_coverage_span(r, 2, 1)[0] == 4


@pytest.mark.parametrize("x0,n", [(1, 10), (0, 300)])
def test_coverage_matches_popcount(O, x0, n):
    # dispatch_test_rows (aa_coverage.rs:553-563): rows i*mul+add (u8 wrapping) and !i.
    rb = (x0 + n + 1) // 2
    i = np.arange(rb, dtype=np.uint16)
    rows = np.stack([((i * m + a) & 0xFF) for m, a in ((0x37, 0), (0x53, 0), (0x17, 0))] + [(~i) & 0xFF]).astype(np.uint8)
    got = O.aa_coverage_span(rows, x0, n)
    x = np.arange(x0, x0 + n)
    nib = np.where(x % 2 == 0, rows[:, x // 2] >> 4, rows[:, x // 2] & 0xF)
    exp = np.vectorize(lambda v: bin(int(v)).count("1"))(nib).sum(axis=0)
    assert np.array_equal(got, exp)


@pytest.mark.parametrize("tier", [1, 2])
def test_coverage_simd_tier_matches_scalar(O, tier):
    # avx2_coverage_matches_scalar / avx512_coverage_matches_scalar (aa_coverage.rs:684-717):
    # TIER_TEST_N = 300 pixels of the dispatch test rows, the SIMD tier against the scalar
    # loop; plus every even and odd x0 up to 8 and spans that end inside, on and past a chunk.
    if O.coverage_tier() < tier:
        pytest.skip(f"host lacks coverage tier {tier}")
    rng = np.random.default_rng(tier)
    for x0, n in [(0, 300)] + [(x, k) for x in range(9) for k in (1, 63, 64, 127, 128, 129, 255, 256, 257, 700)]:
        rb = (x0 + n + 1) // 2
        i = np.arange(rb, dtype=np.uint16)
        rows = np.stack([((i * m + a) & 0xFF) for m, a in ((0x37, 0), (0x53, 0), (0x17, 0))] +
                        [(~i) & 0xFF]).astype(np.uint8)
        for r in (rows, rng.integers(0, 256, rows.shape, dtype=np.uint8)):
            assert np.array_equal(O.aa_coverage_span_tier(r, x0, n, tier), O.aa_coverage_span_tier(r, x0, n, 0)), \
                (tier, x0, n)


def test_coverage_dispatch_uses_the_hosts_best_tier(O):
    # dispatch_coverage (aa_coverage.rs:497-514): AVX-512 BITALG when present, else AVX2.
    flags = open("/proc/cpuinfo").read().split("flags")[1].split("\n")[0].split()
    want = 2 if {"avx512_bitalg", "avx512bw"} <= set(flags) else (1 if "avx2" in flags else 0)
    assert O.coverage_tier() == want


# ---- div255 (crates/color/src/convert.rs:316-345) -------------------------------------

def test_div255_exhaustive(O):
    for x in range(0, 65536):
        got = O.div255(x)
        assert abs(got - min(round(x / 255.0), 255)) <= 1


def test_div255_products_and_formula(O):
    for a in range(256):
        for b in range(0, 256, 5):
            v = O.div255(a * b)
            assert abs(v - round(a * b / 255)) <= 1
            x = a * b
            assert v == min((x + (x >> 8) + 0x80) >> 8, 255)


# ---- AA pipe (crates/raster/src/pipe/aa.rs:234-612; simd/composite.rs tests) -----

def test_gray_pipe_full_and_zero_coverage(O):
    dst = np.array([10, 200, 77], np.uint8)
    O.render_span_aa_gray(dst, np.array([255, 255, 255], np.uint8), 255, 42)
    assert list(dst) == [42, 42, 42]  # full coverage writes src
    dst = np.array([10, 200, 77], np.uint8)
    O.render_span_aa_gray(dst, np.zeros(3, np.uint8), 255, 42)
    assert list(dst) == [10, 200, 77]  # zero coverage leaves dst


def test_gray_pipe_half_coverage(O):
    dst = np.zeros(1, np.uint8)
    O.render_span_aa_gray(dst, np.array([128], np.uint8), 255, 255)
    assert 125 <= dst[0] <= 131  # half_coverage_blends_correctly (pipe/aa.rs)
    dst = np.zeros(1, np.uint8)
    O.render_span_aa_gray(dst, np.array([128], np.uint8), 255, 200)
    assert 95 <= dst[0] <= 105  # no_alpha_plane_uses_opaque_dst


def test_rgb_fast_path_pinned_bytes(O):  # identity_transfer_takes_fast_path_with_pinned_bytes
    color = (200, 100, 50)
    shape = (np.arange(17, dtype=np.uint16) * 17 & 0xFF).astype(np.uint8)
    dst = (np.arange(51, dtype=np.uint16) * 13 & 0xFF).astype(np.uint8)
    exp = dst.astype(np.int64).copy()
    for i, sh in enumerate(shape):
        a = (255 * int(sh) + 255) >> 8
        for j, sc in enumerate(color):
            exp[3 * i + j] = ((255 - a) * exp[3 * i + j] + a * sc + 255) >> 8
    O.composite_aa_rgb8_opaque(dst, color, 255, shape)
    assert list(dst) == list(exp)


def test_rgb_opaque_full_zero_half(O):  # simd/composite.rs tests
    d = np.full(12, 10, np.uint8)
    O.composite_aa_rgb8_opaque(d, (200, 100, 50), 255, np.full(4, 255, np.uint8))
    assert list(d) == [200, 100, 50] * 4
    orig = (np.arange(12) * 10).astype(np.uint8)
    d = orig.copy()
    O.composite_aa_rgb8_opaque(d, (200, 100, 50), 255, np.zeros(4, np.uint8))
    assert list(d) == list(orig)
    d = np.zeros(3, np.uint8)
    O.composite_aa_rgb8_opaque(d, (255, 255, 255), 255, np.array([128], np.uint8))
    assert 125 <= d[0] <= 131


def test_rgb_to_gray_bt709(O):  # pdf_raster/src/render.rs:1306-1324
    rgb = np.array([255, 255, 255, 0, 0, 0, 255, 0, 0, 0, 255, 0, 0, 0, 255, 10, 20, 30], np.uint8)
    exp = [(2126 * r + 7152 * g + 722 * b + 5000) // 10000 for r, g, b in rgb.reshape(-1, 3).astype(int)]
    assert list(O.rgb_to_gray(rgb)) == exp == [255, 0, 54, 182, 18, 19]


# ---- path construction (path/mod.rs:310-448, font/outline.rs:106-112) -------------

def test_close_adds_line_only_when_open(O):
    b = O.OraclePath()
    b.move_to(0, 0)
    b.line_to(5, 0)
    b.line_to(0, 0)
    b.close(False)  # first == last: no closing line
    pts, fl = b.build()
    assert len(pts) == 3 and fl[0] & O.PF_CLOSED and fl[2] & O.PF_CLOSED
    b = O.OraclePath()
    b.move_to(0, 0)
    b.line_to(5, 0)
    b.close(False)
    pts, fl = b.build()
    assert len(pts) == 3 and tuple(pts[2]) == (0.0, 0.0)
    b = O.OraclePath()
    assert b.line_to(1, 1) == 1  # NoCurPt
    b.move_to(0, 0)
    assert b.move_to(1, 1) == 2  # BogusPath


def _fma(a, b, c):
    # Exact a*b+c rounded once (int/int true division rounds correctly).
    f = Fraction(a) * Fraction(b) + Fraction(c)
    return f.numerator / f.denominator


def test_conic_to_cubic_is_fma_form(O):
    p0, pc, p3 = (0.1, 0.7), (3.3, -2.9), (10.01, 4.5)
    c1, c2 = O.conic_to_cubic(p0, pc, p3)
    assert c1[0] == _fma(p0[0], 1 / 3, pc[0] * (2 / 3))
    assert c1[1] == _fma(p0[1], 1 / 3, pc[1] * (2 / 3))
    assert c2[0] == _fma(pc[0], 2 / 3, p3[0] * (1 / 3))
    assert c2[1] == _fma(pc[1], 2 / 3, p3[1] * (1 / 3))


def test_walk_quirk_curve_end_runs_into_next_subpath(O):
    # A subpath ending on a curve is not terminated by LAST (xpath.rs:210-234):
    # the walk adds a line to the next subpath's first point and the final
    # closing segment returns to the FIRST subpath's start.
    b = O.OraclePath()
    b.move_to(0, 0)
    b.line_to(10, 0)
    b.curve_to(10, 5, 5, 10, 0, 0)  # ends where it started
    b.close(False)  # first == last: nothing appended
    b.move_to(20, 20)
    b.line_to(30, 20)
    b.line_to(30, 30)
    b.close(False)
    pts, fl = b.build()
    segs = O.xpath_new(pts, fl, flatness=100.0, close=True)
    ends = [(s.x0, s.y0, s.x1, s.y1) for s in segs]
    # one bridge segment (0,0)->(20,20) and a final close (20,20)->(0,0)
    assert any({(a, b), (c, d)} == {(0.0, 0.0), (20.0, 20.0)} for a, b, c, d in ends[:-1])
    a, b_, c, d = ends[-1]
    assert {(a, b_), (c, d)} == {(20.0, 20.0), (0.0, 0.0)}


# ---- hand-derived rectangle coverage (restatement cross-check iii) ---------------

def _rect_coverage(W, H, xa, ya, xb, yb):
    """Coverage 0..16 per pixel of move(xa,ya) line(xb,ya) line(xb,yb) line(xa,yb) close.

    Walking the scanner rules by hand: AA rows strictly between floor(4ya) and
    floor(4yb) are painted over AA columns [floor(4xa), floor(4xb)]; the two
    boundary rows carry entries whose counts cancel and paint nothing.
    """
    R0, R1 = math.floor(4 * ya), math.floor(4 * yb)
    C0, C1 = math.floor(4 * xa), math.floor(4 * xb) + 1
    cov = np.zeros((H, W), np.int64)
    for y in range(H):
        rows = sum(1 for r in range(4 * y, 4 * y + 4) if R0 < r < R1)
        for x in range(W):
            cols = max(0, min(C1, 4 * x + 4, 4 * W) - max(C0, 4 * x, 0))
            cov[y, x] = rows * cols
    return cov


@pytest.mark.parametrize("rect", [(2.3, 1.6, 9.85, 7.1), (0.0, 0.0, 5.0, 5.0), (-3.2, 2.26, 4.6, 11.9),
                                  (10.05, 0.4, 17.93, 3.6)])
def test_rectangles_match_hand_rule(O, rect):
    W, H = 16, 10
    xa, ya, xb, yb = rect
    b = O.OraclePath()
    b.move_to(xa, ya)
    b.line_to(xb, ya)
    b.line_to(xb, yb)
    b.line_to(xa, yb)
    b.close(False)
    pts, fl = b.build()
    page = np.full((H, W), 255, np.uint8)
    O.fill_path(page, pts, fl, gray=0, alpha=255)
    g = np.array(O.aa_gamma())
    exp = 255 - g[_rect_coverage(W, H, *rect)]
    assert np.array_equal(page, exp.astype(np.uint8))


def test_shipped_rowmap_draws_row_4y_plus_3(O):
    # ROWMAP_AS_SHIPPED: pixel row y shows pixel row 4y+3's coverage.
    W, H = 16, 40
    b = O.OraclePath()
    b.move_to(1.25, 0.0)
    b.line_to(14.5, 0.0)
    b.line_to(14.5, 40.0)
    b.line_to(1.25, 40.0)
    b.close(False)
    pts, fl = b.build()
    doc = np.full((H, W), 255, np.uint8)
    shp = np.full((H, W), 255, np.uint8)
    O.fill_path(doc, pts, fl, rowmap=O.ROWMAP_DOCUMENTED)
    O.fill_path(shp, pts, fl, rowmap=O.ROWMAP_AS_SHIPPED)
    for y in range(H):
        src = 4 * y + 3
        if src < H and 4 * src + 3 < 4 * 40 - 1:
            assert np.array_equal(shp[y], doc[src]), y
    assert np.all(shp[12:] == 255)  # rows past (y_max-12)/16 are never drawn
