"""Rectangular clips (F3): each path clipped to a device-space rectangle as
Clip::clip_to_rect does on the page clip (the reference's treatment of a
rectangular W/W* clip path, crates/raster/src/clip.rs:116-140).

CPU: the oracle's clip is the page clip when the rectangle covers the page and
confines painting to the rectangle's integer bounds. GPU:
rrb_record_path_batch_ex through the C ABI against the oracle, byte for byte,
gray and Rgb8 pages, both row maps, every tile shape.
"""

import numpy as np
import pytest


def _clips(n, w, h, seed):
    rng = np.random.default_rng(seed)
    c = np.empty((n, 4))
    for i in range(n):
        kind = i % 6
        if kind == 0:    # covers the page: the same as no clip
            c[i] = (-50.0, -20.0, w + 30.0, h + 40.0)
        elif kind == 1:  # empty (zero width)
            c[i] = (w / 3, 0.0, w / 3, h)
        elif kind == 2:  # outside the page
            c[i] = (w + 5.0, h + 5.0, w + 90.0, h + 60.0)
        elif kind == 3:  # corners given in the other order, fractional
            x0, x1 = sorted(rng.uniform(-10, w + 10, 2))
            y0, y1 = sorted(rng.uniform(-10, h + 10, 2))
            c[i] = (x1 + 0.37, y1 + 0.61, x0 - 0.25, y0 - 0.5)
        else:            # a random rectangle on the page
            x0, x1 = sorted(rng.uniform(0, w, 2))
            y0, y1 = sorted(rng.uniform(0, h, 2))
            c[i] = (x0, y0, x1, y1)
    return c


def test_oracle_clip_bounds(oracle, rrb_lib):
    s = rrb_lib.Scene(0, 5, n_paths=60, page_w=300, page_h=200)
    ref = s.blank_arena()
    oracle.render_scene(s, ref)
    page_cover = s.blank_arena()
    oracle.render_scene_ex(s, page_cover, clip=np.tile([-10, -10, 1e6, 1e6], (s.n_paths, 1)))
    assert np.array_equal(ref, page_cover)
    box = s.blank_arena()
    oracle.render_scene_ex(s, box, clip=np.tile([50.5, 40.25, 200.75, 150.5], (s.n_paths, 1)))
    pg = s.page(box, 0)
    # x_min_i = 50, x_max_i = ceil(200.75) - 1 = 200; y_min_i = 40, y_max_i = ceil(150.5) - 1 = 150.
    assert not (pg[:40] != 255).any() and not (pg[151:] != 255).any()
    assert not (pg[:, :50] != 255).any() and not (pg[:, 201:] != 255).any()
    inner = pg[40:151, 50:201]
    assert (inner != 255).any() and np.array_equal(inner, s.page(ref, 0)[40:151, 50:201])


SCENES = {
    "polygons": dict(kind=0, seed=31, n_paths=300, page_w=520, page_h=380),
    "mixed": dict(kind=2, seed=32, n_pages=3, page_scale=0.1, paths_scale=0.02),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(SCENES))
@pytest.mark.parametrize("rowmap", [0, 1])
@pytest.mark.parametrize("rgb_pages", [False, True])
def test_clipped_batches_match_oracle(backend, oracle, rrb_lib, name, rowmap, rgb_pages):
    s = rrb_lib.Scene(**SCENES[name])
    w, h = int(s.page_width.max()), int(s.page_height.max())
    clip = _clips(s.n_paths, w, h, 7)
    bpp = 3 if rgb_pages else 1
    rgb = np.random.default_rng(2).integers(0, 256, (s.n_paths, 3), dtype=np.uint8) if rgb_pages else None
    exp = np.full(bpp * s.arena_bytes, 255, np.uint8)
    oracle.render_scene_ex(s, exp, rgb=rgb, clip=clip, rowmap=rowmap)
    pages = backend.alloc_device(bpp * s.arena_bytes)
    keep = []
    p = rrb_lib.batch_params(s.pts, s.flags, s.path_pt_off, s.fill_rule, s.gray, s.alpha, s.path_page,
                             s.page_width, s.page_height, bpp * s.page_offset.astype(np.uint64), pages,
                             rowmap=rowmap, keep=keep)
    try:
        for tile in rrb_lib.TILE_SHAPES:
            backend.set_tuning(*tile)
            backend.begin_page()
            backend.record_fill_buffer(pages, 255)
            backend.record_path_batch_ex(p, rgb, clip)
            backend.wait_page(backend.submit_page())
            got = np.empty(bpp * s.arena_bytes, np.uint8)
            backend.wait_download(backend.download_async(pages, got))
            d = np.nonzero(got != exp)[0]
            assert d.size == 0, f"{name} tile {tile}: {d.size} bytes differ, first at {d[:5]}"
    finally:
        backend.set_tuning(64, 16, auto_tile=True)
        backend.free_device(pages)


@pytest.mark.gpu
def test_clip_rectangles_must_be_finite(backend, rrb_lib):
    s = rrb_lib.Scene(0, 3, n_paths=4, page_w=64, page_h=64)
    pages = backend.alloc_device(s.arena_bytes)
    keep = []
    p = rrb_lib.batch_params(s.pts, s.flags, s.path_pt_off, s.fill_rule, s.gray, s.alpha, s.path_page,
                             s.page_width, s.page_height, s.page_offset, pages, keep=keep)
    clip = np.tile([0.0, 0.0, 10.0, np.nan], (4, 1))
    try:
        backend.begin_page()
        with pytest.raises(rrb_lib.BackendError) as e:
            backend.record_path_batch_ex(p, None, clip)
        assert e.value.status == 4
    finally:
        backend.wait_page(backend.submit_page())
        backend.free_device(pages)
