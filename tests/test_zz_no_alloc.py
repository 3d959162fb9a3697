"""rrb_record_path_fill_static through the C ABI: the same pixels as
rrb_record_path_fill on consecutive calls and as the CPU oracle, no device
allocation, and every documented limit (points, edges, crossings per AA row,
coverage cells) rejected with the page untouched.

Collected last on purpose: it must hold both in a fresh process (the first
call sets up the static scratch array) and after every other test.
"""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W, H = 211, 157


def _builder_path(rrb, ops):
    b = rrb.PathBuilder()
    for op, *a in ops:
        getattr(b, op)(*a)
    return b.build()


def _comb(rrb, teeth):
    ops = [("move_to", 2.0, 2.0)]
    x = 2.0
    for _ in range(teeth):
        ops += [("line_to", x + 0.7, 2.0), ("line_to", x + 0.7, 50.0), ("line_to", x + 1.3, 50.0),
                ("line_to", x + 1.3, 2.0)]
        x += 1.45
    ops += [("line_to", x, 2.0), ("line_to", x, 58.0), ("line_to", 2.0, 58.0), ("close",)]
    return _builder_path(rrb, ops)


def _cases(rrb):
    """(name, pts, flags, rule, gray, alpha, rowmap) in call order."""
    out = [
        ("curves", _builder_path(rrb, [("move_to", 10, 30), ("curve_to", 10, 0, 160, 0, 160, 90),
                                       ("curve_to", 160, 150, 10, 150, 10, 30), ("close",)]), 0, 20, 255, 0),
        ("rect", _builder_path(rrb, [("move_to", 5.3, 4.8), ("line_to", 150.55, 4.8), ("line_to", 150.55, 130.1),
                                     ("line_to", 5.3, 130.1), ("close",)]), 0, 90, 200, 0),
        ("partial", _builder_path(rrb, [("move_to", -20.5, 10.25), ("line_to", 130.75, -12.5),
                                        ("line_to", 320.2, 170.6), ("close",)]), 1, 200, 128, 1),
        ("comb40", _comb(rrb, 40), 1, 0, 255, 0),
        ("donut", _builder_path(rrb, [("move_to", 5, 5), ("line_to", 155, 5), ("line_to", 155, 145),
                                      ("line_to", 5, 145), ("close",), ("move_to", 35, 35), ("line_to", 125, 35),
                                      ("line_to", 125, 105), ("line_to", 35, 105), ("close",)]), 1, 60, 255, 1),
    ]
    # Generated glyph and polygon outlines, scaled onto the page.
    for kind, seed, take in ((1, 7, 6), (0, 9, 6)):
        s = rrb.Scene(kind, seed, n_paths=64, page_w=W, page_h=H)
        for i in range(take):
            a, b = int(s.path_pt_off[i]), int(s.path_pt_off[i + 1])
            out.append((f"scene{kind}_{i}", (s.pts[a:b].copy(), s.flags[a:b].copy()), int(s.fill_rule[i]),
                        int(s.gray[i]), int(s.alpha[i]), i & 1))
    return [(n, p[0], p[1], r, g, al, rm) for n, p, r, g, al, rm in out]


def _render(backend, buf, fn, pts, fl, rule, gray, alpha, rowmap):
    backend.begin_page()
    try:
        fn(pts, fl, buf, W, H, fill_rule=rule, gray=gray, alpha=alpha, rowmap=rowmap)
    finally:
        backend.wait_page(backend.submit_page())
    got = np.empty(W * H, np.uint8)
    backend.wait_download(backend.download_async(buf, got))
    return got


@pytest.fixture(scope="module")
def pages(rrb_lib):
    be = rrb_lib.B200Backend(0)
    init = np.random.default_rng(3).integers(0, 256, W * H, dtype=np.uint8)
    a, b = be.alloc_device(W * H), be.alloc_device(W * H)
    be.upload_async(a, init)
    be.upload_async(b, init)
    yield be, a, b, init
    be.free_device(a)
    be.free_device(b)
    be.close()


def test_static_fill_matches_record_path_fill_on_consecutive_calls(rrb_lib, pages):
    be, a, b, init = pages
    cases = _cases(rrb_lib)
    # The paths are composited one after another onto the same two pages, so
    # every call also checks that nothing of the previous call's use of the
    # shared scratch array leaks into the next.
    for name, pts, fl, rule, gray, alpha, rowmap in cases:
        ref = _render(be, a, be.record_path_fill, pts, fl, rule, gray, alpha, rowmap)
        got = _render(be, b, be.record_path_fill_static, pts, fl, rule, gray, alpha, rowmap)
        d = np.nonzero(ref != got)[0]
        assert d.size == 0, f"{name}: {d.size} pixels differ, first at {d[:5]}"
    assert not np.array_equal(ref, init)


def test_static_fill_matches_the_oracle(rrb_lib, oracle, pages):
    """The static entry point against the CPU oracle directly: every case
    composited in order onto a fresh copy of the same initial page."""
    be, _, b, init = pages
    be.upload_async(b, init)
    exp = init.copy().reshape(H, W)
    for name, pts, fl, rule, gray, alpha, rowmap in _cases(rrb_lib):
        got = _render(be, b, be.record_path_fill_static, pts, fl, rule, gray, alpha, rowmap)
        oracle.fill_path(exp, pts, fl, eo=bool(rule), gray=gray, alpha=alpha, rowmap=rowmap)
        d = np.nonzero(got != exp.reshape(-1))[0]
        assert d.size == 0, f"{name}: {d.size} pixels differ from the oracle, first at {d[:5]}"


def test_static_fill_twice_in_a_row_matches(rrb_lib, pages):
    be, a, b, _ = pages
    name, pts, fl, rule, gray, alpha, rowmap = _cases(rrb_lib)[0]
    for _ in range(2):
        ref = _render(be, a, be.record_path_fill, pts, fl, rule, gray, alpha, rowmap)
        got = _render(be, b, be.record_path_fill_static, pts, fl, rule, gray, alpha, rowmap)
        assert np.array_equal(ref, got)


def test_static_fill_allocates_nothing(rrb_lib, pages):
    import torch

    be, _, b, _ = pages
    cases = _cases(rrb_lib)
    _render(be, b, be.record_path_fill_static, *cases[0][1:])  # set-up done, modules loaded
    used0 = be.detect_vram_budget().used_bytes
    free0 = torch.cuda.mem_get_info(0)[0]
    for name, pts, fl, rule, gray, alpha, rowmap in cases[:6]:
        _render(be, b, be.record_path_fill_static, pts, fl, rule, gray, alpha, rowmap)
    assert be.detect_vram_budget().used_bytes == used0
    assert torch.cuda.mem_get_info(0)[0] == free0


def test_static_fill_limits_leave_the_page_untouched(rrb_lib, pages):
    be, _, b, _ = pages
    before = np.empty(W * H, np.uint8)
    be.wait_download(be.download_async(b, before))
    # More merged crossings on an AA row than the per-row limit (a comb of 80 teeth: ~160).
    pts, fl = _comb(rrb_lib, 80)
    with pytest.raises(rrb_lib.BackendError) as e:
        _render(be, b, be.record_path_fill_static, pts, fl, 0, 0, 255, 0)
    assert e.value.status == 3 and "crossings" in str(e.value)
    # More points than the array holds.
    n = rrb_lib._abi.RRB_STATIC_MAX_POINTS + 1
    pts = np.zeros((n, 2))
    fl = np.zeros(n, np.uint8)
    fl[0] = 1
    with pytest.raises(rrb_lib.BackendError) as e:
        _render(be, b, be.record_path_fill_static, pts, fl, 0, 0, 255, 0)
    assert e.value.status == 3 and "at most" in str(e.value)
    after = np.empty(W * H, np.uint8)
    be.wait_download(be.download_async(b, after))
    assert np.array_equal(before, after)
    # The entry point still works after a rejection.
    name, pts, fl, rule, gray, alpha, rowmap = _cases(rrb_lib)[1]
    _render(be, b, be.record_path_fill_static, pts, fl, rule, gray, alpha, rowmap)


def test_static_fill_edge_limit_leaves_the_page_untouched(rrb_lib, pages):
    """A path of 300 huge cubics flattens to 1,024 edges each, past
    RRB_STATIC_MAX_EDGES (262,144): rejected after the count, page untouched."""
    be, _, b, _ = pages
    before = np.empty(W * H, np.uint8)
    be.wait_download(be.download_async(b, before))
    ops = [("move_to", 10.0, 10.0)]
    for k in range(300):
        s = 1e6 * (1 + (k % 3))
        ops.append(("curve_to", -s, s, s, -s, 10.0 + k % 7, 10.0 + k % 5))
    ops.append(("close",))
    pts, fl = _builder_path(rrb_lib, ops)
    with pytest.raises(rrb_lib.BackendError) as e:
        _render(be, b, be.record_path_fill_static, pts, fl, 0, 0, 255, 0)
    assert e.value.status == 3 and "edges" in str(e.value)
    after = np.empty(W * H, np.uint8)
    be.wait_download(be.download_async(b, after))
    assert np.array_equal(before, after)


def test_static_fill_cell_limit_leaves_the_page_untouched(rrb_lib, pages):
    """A comb of 60 teeth (122 merged crossings per AA row, under the row
    limit) on a page 60,000 rows tall needs more coverage cells than
    RRB_STATIC_MAX_CELLS: found on the device, the blend is skipped, the page
    keeps its bytes and the call reports the cell limit."""
    be = pages[0]
    w2, h2 = W, 60000  # about 120 cells per pixel row: some 7 M cells
    ops = [("move_to", 2.0, 2.0)]
    x = 2.0
    for _ in range(60):
        ops += [("line_to", x + 0.7, 2.0), ("line_to", x + 0.7, h2 - 8.0), ("line_to", x + 1.3, h2 - 8.0),
                ("line_to", x + 1.3, 2.0)]
        x += 1.45
    ops += [("line_to", x, 2.0), ("line_to", x, h2 - 2.0), ("line_to", 2.0, h2 - 2.0), ("close",)]
    pts, fl = _builder_path(rrb_lib, ops)
    buf = be.alloc_device(w2 * h2)
    try:
        init = np.random.default_rng(8).integers(0, 256, w2 * h2, dtype=np.uint8)
        be.upload_async(buf, init)
        be.begin_page()
        try:
            with pytest.raises(rrb_lib.BackendError) as e:
                be.record_path_fill_static(pts, fl, buf, w2, h2, fill_rule=1, gray=0, alpha=255, rowmap=0)
        finally:
            be.wait_page(be.submit_page())
        assert e.value.status == 3 and "coverage cells" in str(e.value)
        after = np.empty(w2 * h2, np.uint8)
        be.wait_download(be.download_async(buf, after))
        assert np.array_equal(init, after)
    finally:
        be.free_device(buf)


def test_static_fill_outside_a_page_is_a_state_error(rrb_lib, pages):
    be, _, b, _ = pages
    p = be._fill_params(*_cases(rrb_lib)[0][1:3], b, W, H, 0, 0, 255, 0, rrb_lib.IDENTITY, 0.1, 0)
    assert rrb_lib.lib().rrb_record_path_fill_static(be._h, C.byref(p)) == 9
