"""Row-stage shapes: a device-resident batch renders once with each shape of
the row kernel (list entries per AA row x warps per block x edge groups
staged per warp: 12 x 8 x 2, 16 x 4 x 2, 12 x 8 x 1, 8 x 16 x 2, 16 x 4 x 1,
i.e. 512, 256, 256, 1024 and 128 edges staged per block) and then keeps the
fastest. Every render must give the oracle's pages byte for byte, whichever
shape ran."""

import numpy as np
import pytest


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(kind=0, seed=41, n_paths=600, page_w=900, page_h=700),
                                dict(kind=1, seed=42, n_paths=3000, page_w=1200, page_h=900)])
def test_resident_renders_match_oracle_under_every_shape(backend, oracle, rrb_lib, kw):
    s = rrb_lib.Scene(**kw)
    exp = s.blank_arena()
    oracle.render_scene(s, exp, threads=4)
    pages = backend.alloc_device(s.arena_bytes)
    batch = backend.batch_upload(s.view)
    try:
        seen = set()
        for k in range(12):  # the tile trials, the row-shape trials, then the fastest shape
            backend.begin_page()
            backend.record_fill_buffer(pages, 255)
            batch.record(pages)
            backend.wait_page(backend.submit_page())
            seen.add(backend.last_batch_stats()["row_shape"])
            got = np.empty(s.arena_bytes, np.uint8)
            backend.wait_download(backend.download_async(pages, got))
            d = np.nonzero(got != exp)[0]
            assert d.size == 0, f"render {k}: {d.size} bytes differ, first at {d[:5]}"
        assert seen == {0, 1, 2, 3, 4}
    finally:
        batch.free()
        backend.free_device(pages)
