"""Streamed batches: a host batch in page-locked memory of at least 4 Mi
points is rendered in ranges of consecutive paths, each range's points copied
on a second stream while the ranges before it render (rrb_record_path_batch,
rrb_render_pages_host). Rendering path ranges one after another composites
each page in path order, so the pages equal the oracle's byte for byte."""

import numpy as np
import pytest


def _pinned(backend, arr, bufs):
    arr = np.ascontiguousarray(arr)
    buf = backend.alloc_host_pinned(max(1, arr.nbytes))
    bufs.append(buf)
    v = buf.array()[: arr.nbytes].view(arr.dtype)
    v[:] = arr.reshape(-1)
    return v


SCENES = {
    "glyphs_one_page": dict(kind=1, seed=3, n_paths=20000),
    "mixed_8_pages": dict(kind=2, seed=5, n_pages=8, page_scale=0.15, paths_scale=0.8),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(SCENES))
def test_streamed_batch_matches_oracle(backend, oracle, rrb_lib, name):
    s = rrb_lib.Scene(**SCENES[name])
    assert s.n_pts >= 4 << 20
    exp = s.blank_arena()
    oracle.render_scene(s, exp, threads=8)
    bufs = []
    pages = backend.alloc_device(s.arena_bytes)
    try:
        h = {k: _pinned(backend, getattr(s, k), bufs) for k in ("pts", "flags", "path_pt_off", "fill_rule", "gray",
                                                                   "alpha", "path_page", "page_width", "page_height",
                                                                   "page_offset")}
        keep = []
        p = rrb_lib.batch_params(h["pts"], h["flags"], h["path_pt_off"], h["fill_rule"], h["gray"], h["alpha"],
                                 h["path_page"], h["page_width"], h["page_height"], h["page_offset"], pages, keep=keep)
        host = _pinned(backend, s.blank_arena(), bufs)
        backend.render_pages_host(p, host)
        assert backend.last_batch_stats()["waves"] > 1  # the ranges of the streamed path
        d = np.nonzero(np.asarray(host) != exp)[0]
        assert d.size == 0, f"{d.size} bytes differ, first at {d[:5]}"
        # The same batch from pageable memory (one upload, then the render) agrees.
        keep2 = []
        q = rrb_lib.batch_params(s.pts, s.flags, s.path_pt_off, s.fill_rule, s.gray, s.alpha, s.path_page,
                                 s.page_width, s.page_height, s.page_offset, pages, keep=keep2)
        host2 = s.blank_arena()
        backend.render_pages_host(q, host2)
        assert np.array_equal(host2, exp)
        # Pages filled on the device (init 255) instead of uploaded: the host
        # buffer's old page content is ignored, streamed and from pageable
        # memory (arena bytes outside every page are not written back).
        def pages_equal(got):
            return all(np.array_equal(got[o:o + w * h], exp[o:o + w * h])
                       for o, w, h in zip(s.page_offset.tolist(), s.page_width.tolist(), s.page_height.tolist()))

        host[:] = 7
        backend.render_pages_host(p, host, init=255)
        assert backend.last_batch_stats()["waves"] > 1
        assert pages_equal(np.asarray(host))
        host2[:] = 7
        backend.render_pages_host(q, host2, init=255)
        assert pages_equal(host2)
    finally:
        backend.free_device(pages)
        for b in bufs:
            backend.free_host_pinned(b)
