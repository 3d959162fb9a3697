"""The product renderer's RGB page form (A12): paths composited onto Rgb8
pages with composite_aa_rgb8_opaque, then BT.709 luma to Gray8.

CPU: the oracle's composite and luma against the reference's unit tests
(crates/raster/src/simd/composite.rs tests). GPU: rrb_record_path_batch_rgb and
rrb_record_rgb_to_gray through the C ABI against the oracle, byte for byte.
"""

import numpy as np
import pytest


def test_rgb_composite_known_answers(oracle):
    # composite.rs:125-208.
    src = np.array([200, 100, 50], np.uint8)
    dst = np.full(12, 10, np.uint8)
    oracle.composite_aa_rgb8_opaque(dst, src, 255, np.full(4, 255, np.uint8))
    assert dst.reshape(4, 3).tolist() == [[200, 100, 50]] * 4
    orig = (np.arange(12) * 10).astype(np.uint8)
    dst = orig.copy()
    oracle.composite_aa_rgb8_opaque(dst, src, 255, np.zeros(4, np.uint8))
    assert np.array_equal(dst, orig)
    dst = np.zeros(3, np.uint8)
    oracle.composite_aa_rgb8_opaque(dst, np.array([255, 255, 255], np.uint8), 255, np.array([128], np.uint8))
    assert 125 <= dst[0] <= 131
    # The 37-pixel span against the scalar formula of the same test.
    count, a_in = 37, 200
    shape = (np.arange(count) * 7 % 256).astype(np.uint8)
    init = (np.arange(count * 3) * 3 % 256).astype(np.uint8)
    s = np.array([100, 150, 200], np.uint32)
    a_src = (a_in * shape.astype(np.uint32) + 255) >> 8
    exp = ((255 - a_src)[:, None] * init.reshape(-1, 3).astype(np.uint32) + a_src[:, None] * s + 255) >> 8
    got = init.copy()
    oracle.composite_aa_rgb8_opaque(got, s.astype(np.uint8), a_in, shape)
    assert np.array_equal(got.reshape(-1, 3), exp.astype(np.uint8))


def test_luma_known_answers(oracle):
    rgb = np.array([[0, 0, 0], [255, 255, 255], [255, 0, 0], [0, 255, 0], [0, 0, 255], [10, 200, 30]], np.uint8)
    gray = oracle.rgb_to_gray(rgb.reshape(-1))
    assert gray.tolist() == [(2126 * r + 7152 * g + 722 * b + 5000) // 10000 for r, g, b in rgb.astype(int)]
    assert gray[1] == 255


def _rgb_of(scene, seed):
    rng = np.random.default_rng(seed)
    return rng.integers(0, 256, (scene.n_paths, 3), dtype=np.uint8)


SCENES = {
    "mixed": dict(kind=2, seed=21, n_pages=4, page_scale=0.12, paths_scale=0.02),
    "polygons": dict(kind=0, seed=22, n_paths=400, page_w=600, page_h=420),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(SCENES))
@pytest.mark.parametrize("rowmap", [0, 1])
def test_rgb_pages_match_oracle(backend, oracle, rrb_lib, name, rowmap):
    scene = rrb_lib.Scene(**SCENES[name])
    rgb = _rgb_of(scene, 5)
    exp = np.full(3 * scene.arena_bytes, 255, np.uint8)
    oracle.render_scene_rgb(scene, exp, rgb, rowmap=rowmap)
    pages = backend.alloc_device(3 * scene.arena_bytes)
    keep = []
    p = rrb_lib.batch_params(scene.pts, scene.flags, scene.path_pt_off, scene.fill_rule, scene.gray, scene.alpha,
                             scene.path_page, scene.page_width, scene.page_height,
                             3 * scene.page_offset.astype(np.uint64), pages, rowmap=rowmap, keep=keep)
    try:
        for tile in rrb_lib.TILE_SHAPES:
            backend.set_tuning(*tile)
            backend.begin_page()
            backend.record_fill_buffer(pages, 255)
            backend.record_path_batch_rgb(p, rgb)
            backend.wait_page(backend.submit_page())
            got = np.empty(3 * scene.arena_bytes, np.uint8)
            backend.wait_download(backend.download_async(pages, got))
            d = np.nonzero(got != exp)[0]
            assert d.size == 0, f"{name} tile {tile}: {d.size} bytes differ, first at {d[:5]}"
    finally:
        backend.set_tuning(64, 16, auto_tile=True)
        backend.free_device(pages)


@pytest.mark.gpu
def test_rgb_full_tile_layers_and_luma(backend, oracle, rrb_lib):
    """Stacked page-covering rectangles (full-tile layers folded into per-channel
    maps, opaque ones occluding what lies under them), then luma on the device."""
    W, H = 300, 200
    b = []
    rng = np.random.default_rng(3)
    for i in range(7):
        pb = rrb_lib.PathBuilder()
        x0, y0 = -5 + i, -3 + 0.5 * i
        pb.move_to(x0, y0)
        pb.line_to(W + 7, y0)
        pb.line_to(W + 7, H + 9)
        pb.line_to(x0, H + 9)
        pb.close()
        b.append(pb.build())
    pts = np.concatenate([x[0] for x in b])
    flags = np.concatenate([x[1] for x in b])
    off = np.cumsum([0] + [len(x[1]) for x in b]).astype(np.uint64)
    n = len(b)
    alpha = np.array([255, 90, 200, 255, 40, 128, 250], np.uint8)
    rgb = rng.integers(0, 256, (n, 3), dtype=np.uint8)
    zeros = np.zeros(n, np.uint8)

    class S:
        pass

    sc = S()
    sc.pts, sc.flags, sc.path_pt_off, sc.fill_rule, sc.alpha = pts, flags, off, zeros, alpha
    sc.path_page = np.zeros(n, np.uint32)
    sc.page_width, sc.page_height = np.array([W], np.uint32), np.array([H], np.uint32)
    sc.page_offset = np.zeros(1, np.uint64)
    exp = np.full(3 * W * H, 255, np.uint8)
    oracle.render_scene_rgb(sc, exp, rgb)
    pages = backend.alloc_device(3 * W * H)
    gray = backend.alloc_device(W * H)
    keep = []
    p = rrb_lib.batch_params(pts, flags, off, zeros, zeros, alpha, sc.path_page, sc.page_width, sc.page_height,
                             sc.page_offset, pages, keep=keep)
    try:
        for tile in rrb_lib.TILE_SHAPES:
            backend.set_tuning(*tile)
            backend.begin_page()
            backend.record_fill_buffer(pages, 255)
            backend.record_path_batch_rgb(p, rgb)
            backend.record_rgb_to_gray(pages, gray, W * H)
            backend.wait_page(backend.submit_page())
            got = np.empty(3 * W * H, np.uint8)
            backend.wait_download(backend.download_async(pages, got))
            assert np.array_equal(got, exp), tile
            g = np.empty(W * H, np.uint8)
            backend.wait_download(backend.download_async(gray, g))
            assert np.array_equal(g, oracle.rgb_to_gray(exp))
    finally:
        backend.set_tuning(64, 16, auto_tile=True)
        backend.free_device(pages)
        backend.free_device(gray)


def test_netpbm_output_matches_the_reference_format(rrb_lib):
    # pgm.rs / ppm.rs tests: "P5\n3 2\n255\n" + 6 bytes; P6 with 3 bytes per pixel.
    g = np.full((2, 3), 128, np.uint8)
    out = rrb_lib.encode_netpbm(g)
    assert out == b"P5\n3 2\n255\n" + bytes([128] * 6)
    rgb = np.arange(2 * 3 * 3, dtype=np.uint8).reshape(2, 3, 3)
    out = rrb_lib.encode_netpbm(rgb)
    assert out == b"P6\n3 2\n255\n" + rgb.tobytes()
    assert rrb_lib.encode_netpbm(np.zeros((0, 5), np.uint8)) == b"P5\n5 0\n255\n"
