"""Resident batches replayed without waiting on the stream.

A device-resident batch renders the same inputs every time, so after a render
has found each wave's sizes on the device (path pieces, edges, row groups,
cells, overflow rows), later renders with the same tile shape, row-stage
shape and row map take them from the batch and launch every stage without
reading anything back; each wave's counters go to page-locked memory and are
read after one wait at the end of the render. These tests render a batch
that runs in several waves until the replays start, and check that every
render gives the oracle's pages, that the replays keep the statistics of the
renders that read their sizes back, and that a replay waits on the stream
once.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _render(backend, batch, pages, n):
    backend.begin_page()
    backend.record_fill_buffer(pages, 255)
    batch.record(pages)
    backend.wait_page(backend.submit_page())
    got = np.empty(n, np.uint8)
    backend.wait_download(backend.download_async(pages, got))
    return got, backend.last_batch_stats()


@pytest.mark.parametrize("tile", [(64, 16), (128, 16), (128, 32), (32, 32)])
def test_replays_keep_pixels_and_stats_and_wait_once(backend, oracle, rrb_lib, tile):
    s = rrb_lib.Scene(kind=2, seed=23, n_pages=6, page_scale=0.25, paths_scale=0.1)
    exp = s.blank_arena()
    oracle.render_scene(s, exp, threads=4)
    pages = backend.alloc_device(s.arena_bytes)
    backend.set_tuning(*tile, wave_points=max(1, s.n_pts // 3))  # several waves of pages
    s.view.pages = None
    batch = backend.batch_upload(s.view)
    try:
        stats = []
        for k in range(10):  # row-shape trials, the chosen shape's first render, then replays
            got, st = _render(backend, batch, pages, s.arena_bytes)
            d = np.nonzero(got != exp)[0]
            assert d.size == 0, f"render {k}: {d.size} bytes differ, first at {d[:5]}"
            stats.append(st)
        last = stats[-1]
        # The last render that read its sizes back ran the row shape the batch
        # settled on (the replays' shape), so its statistics are the reference.
        first = [st for st in stats if st["host_syncs"] > 1][-1]
        assert last["waves"] >= 2
        assert last["host_syncs"] == 1, last  # one wait for the whole render
        assert first["host_syncs"] >= 3 * first["waves"]
        for key in ("paths", "pieces", "segments", "aa_rows", "spans", "row_overflows", "tiles", "tile_pairs",
                    "nonterminating_rows", "kernel_launches", "row_groups", "waves"):
            assert last[key] == first[key], key
    finally:
        batch.free()
        backend.set_tuning(64, 16, wave_points=0, auto_tile=True)
        backend.free_device(pages)


def test_new_inputs_are_not_replayed(backend, oracle, rrb_lib):
    """Sizes belong to the inputs they were found for: uploading another
    batch, or rendering through rrb_record_path_batch, reads sizes back."""
    a = rrb_lib.Scene(kind=0, seed=31, n_paths=200, page_w=500, page_h=400)
    b = rrb_lib.Scene(kind=0, seed=32, n_paths=260, page_w=500, page_h=400)
    pages = backend.alloc_device(a.arena_bytes)
    try:
        for sc in (a, b, a):
            exp = sc.blank_arena()
            oracle.render_scene(sc, exp)
            got = sc.blank_arena()
            backend.render_scene(sc, got, pages=pages)
            assert np.array_equal(got, exp)
            assert backend.last_batch_stats()["host_syncs"] >= 3
    finally:
        backend.free_device(pages)


def test_automatic_tile_trials_keep_pixels(backend, oracle, rrb_lib):
    """With automatic tiles a resident batch renders once with each of 64x16,
    128x16 and 128x32 (row shape 0), then with the other row-stage shapes on the
    fastest of those tiles, then keeps the fastest pair and
    replays it: every render, trials included, gives the oracle's pages."""
    s = rrb_lib.Scene(kind=2, seed=29, n_pages=3, page_scale=0.3, paths_scale=0.1)
    exp = s.blank_arena()
    oracle.render_scene(s, exp, threads=4)
    pages = backend.alloc_device(s.arena_bytes)
    backend.set_tuning(64, 16, auto_tile=True)
    assert backend.get_tuning().auto_tile == 1
    s.view.pages = None
    batch = backend.batch_upload(s.view)
    try:
        seen = set()
        for k in range(20):
            got, st = _render(backend, batch, pages, s.arena_bytes)
            assert np.array_equal(got, exp), f"render {k} ({st['tile_w']}x{st['tile_h']}, rows {st['row_shape']})"
            seen.add((st["tile_w"], st["tile_h"], st["row_shape"]))
            if st["trials_left"] == 0 and st["host_syncs"] == 1:
                break
        assert {(64, 16, 0), (128, 16, 0), (128, 32, 0)} <= seen
        assert {rs for *_, rs in seen} == {0, 1, 2, 3, 4}  # every row-stage shape ran
        assert st["trials_left"] == 0 and st["host_syncs"] == 1  # settled and replaying
        assert (st["tile_w"], st["tile_h"]) in {(64, 16), (128, 16), (128, 32)}
        # A batch uploaded per call on this context then takes the settled tile shape.
        settled = (st["tile_w"], st["tile_h"])
        keep = []
        p = rrb_lib.batch_params(s.pts, s.flags, s.path_pt_off, s.fill_rule, s.gray, s.alpha, s.path_page,
                                 s.page_width, s.page_height, s.page_offset, pages, keep=keep)
        backend.begin_page()
        backend.record_fill_buffer(pages, 255)
        backend.record_path_batch(p)
        backend.wait_page(backend.submit_page())
        st2 = backend.last_batch_stats()
        assert (st2["tile_w"], st2["tile_h"]) == settled
        got = np.empty(s.arena_bytes, np.uint8)
        backend.wait_download(backend.download_async(pages, got))
        assert np.array_equal(got, exp)
    finally:
        batch.free()
        backend.set_tuning(64, 16, auto_tile=True)
        backend.free_device(pages)


def test_explicit_tile_turns_automatic_tiles_off(backend):
    backend.set_tuning(32, 32)
    try:
        t = backend.get_tuning()
        assert (t.tile_w, t.tile_h, t.auto_tile) == (32, 32, 2)
        backend.set_tuning(auto_tile=True)
        assert backend.get_tuning().auto_tile == 1
    finally:
        backend.set_tuning(64, 16, auto_tile=True)
