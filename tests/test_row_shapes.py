"""Row-stage shapes: a device-resident batch renders once with each shape of
the row kernel (12 list entries per AA row with 8 warps per block, 16 entries
with 4 warps) and then keeps the faster. Every render must give the oracle's
pages byte for byte, whichever shape ran."""

import numpy as np
import pytest


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(kind=0, seed=41, n_paths=600, page_w=900, page_h=700),
                                dict(kind=1, seed=42, n_paths=3000, page_w=1200, page_h=900)])
def test_resident_renders_match_oracle_under_both_shapes(backend, oracle, rrb_lib, kw):
    s = rrb_lib.Scene(**kw)
    exp = s.blank_arena()
    oracle.render_scene(s, exp, threads=4)
    pages = backend.alloc_device(s.arena_bytes)
    batch = backend.batch_upload(s.view)
    try:
        for k in range(5):  # shape 0, shape 1, then the faster one, three times
            backend.begin_page()
            backend.record_fill_buffer(pages, 255)
            batch.record(pages)
            backend.wait_page(backend.submit_page())
            got = np.empty(s.arena_bytes, np.uint8)
            backend.wait_download(backend.download_async(pages, got))
            d = np.nonzero(got != exp)[0]
            assert d.size == 0, f"render {k}: {d.size} bytes differ, first at {d[:5]}"
    finally:
        batch.free()
        backend.free_device(pages)
