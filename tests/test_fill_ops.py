"""The reference's coverage operators (record_aa_fill / record_tile_fill).

CPU: the oracle restatement (oracle/fill_oracle.cpp) against the reference's
own unit tests (crates/gpu/src/fill.rs tests, crates/gpu/src/lib.rs
gpu_vs_cpu) and the sample-offset table extracted from the reference source
(tests/golden/aa_fill_jitter.json). GPU: rrb_record_aa_fill,
rrb_record_tile_fill and rrb_record_tile_fill_segs through the C ABI against
the oracle, byte for byte.
"""

import json
from pathlib import Path

import numpy as np
import pytest

HERE = Path(__file__).resolve().parent


def rect(x0, y0, x1, y1):
    return [x0, y0, x1, y0, x1, y0, x1, y1, x1, y1, x0, y1, x0, y1, x0, y0]


# ---- CPU: the oracle against the reference's known answers -------------------------

def test_jitter_tables_match_the_reference_source(oracle, rrb_lib):
    fx = json.loads((HERE / "golden" / "aa_fill_jitter.json").read_text())
    want_x = np.array([float(v) for v in fx["x"]], np.float32)
    want_y = np.array([float(v) for v in fx["y"]], np.float32)
    for x, y in (oracle.aa_jitter(), rrb_lib.aa_fill_jitter()):
        assert np.array_equal(x.view(np.uint32), want_x.view(np.uint32))
        assert np.array_equal(y.view(np.uint32), want_y.view(np.uint32))


def test_aa_fill_cpu_known_answers(oracle):
    # fill.rs:472-530 and lib.rs gpu_vs_cpu (1x1 windows).
    assert oracle.aa_fill_cpu(rect(-100, -100, 100, 100), 0, 0, 1, 1)[0, 0] == 255
    assert oracle.aa_fill_cpu(rect(0, 0, 10, 10), 200, 200, 1, 1)[0, 0] == 0
    assert not oracle.aa_fill_cpu([], 0, 0, 4, 4).any()
    donut = rect(-10, -10, 10, 10) + rect(-5, -5, 5, 5)
    assert oracle.aa_fill_cpu(donut, -0.5, -0.5, 1, 1, eo=True)[0, 0] == 0
    assert oracle.aa_fill_cpu(donut, -0.5, -0.5, 1, 1, eo=False)[0, 0] == 255
    half = oracle.aa_fill_cpu(rect(-100, -100, 0.5, 100), 0, 0, 1, 1)[0, 0]
    assert 0 < half < 255
    tri = oracle.aa_fill_cpu([0, 0, 8, 0, 8, 0, 0, 8, 0, 8, 0, 0], 0, 0, 8, 8)
    assert tri[0, 0] == 255 and tri[7, 7] == 0


def test_build_tile_records_known_answers(oracle):
    # fill.rs:532-591.
    recs, starts, counts, gw = oracle.build_tile_records([], 0, 0, 32, 32)
    assert len(recs) == 0 and gw == 2 and not starts.any() and not counts.any()
    recs, *_ = oracle.build_tile_records([8, 0, 8, 17], 0, 0, 64, 64)
    assert len(recs) == 2
    recs, *_ = oracle.build_tile_records([0, 0, 32, 32], 0, 0, 128, 128)
    assert len(recs) >= 2
    recs, starts, counts, gw = oracle.build_tile_records([24, 0, 24, 8, 8, 16, 8, 24], 0, 0, 80, 80)
    assert gw == 5 and np.all(np.diff(recs["key"].astype(np.int64)) >= 0)
    assert counts[1] == 1 and counts[gw] == 1
    recs, starts, counts, gw = oracle.build_tile_records([4, 0, 60, 63], 0, 0, 64, 64)
    assert counts.sum() == len(recs)
    assert np.array_equal(starts[:-1] + counts[:-1], starts[1:])


def test_tile_fill_oracle_within_one_tile(oracle):
    # tile_fill.cu accumulates only the records of the pixel's own tile (no
    # backdrop from tiles to the left), so a shape is filled exactly when all
    # of its edges lie in one tile row segment of the pixel's tile.
    recs, starts, counts, gw = oracle.build_tile_records(rect(2.5, 3, 12.25, 13.5), 0, 0, 16, 16)
    cov = oracle.tile_fill(recs, starts, counts, gw, 16, 16)
    assert (cov[3:13, 3:12] == 255).all() and not cov[:2].any() and not cov[14:].any() and not cov[:, 13:].any()
    assert cov[5, 2] == 0 and cov[3, 5] == 255 and cov[13, 5] == 127  # vertical edges step at the pixel centre
    segs = rect(1, 1, 15, 15) + rect(5, 5, 11, 11)
    recs, starts, counts, gw = oracle.build_tile_records(segs, 0, 0, 16, 16)
    eo = oracle.tile_fill(recs, starts, counts, gw, 16, 16, eo=True)
    nz = oracle.tile_fill(recs, starts, counts, gw, 16, 16, eo=False)
    assert (nz[5:11, 5:11] == 255).all() and (nz[2:4, 2:14] == 255).all()
    # Even-odd folds the fractional part of |area| (tile_fill.cu:161-167): a
    # whole winding of 1 or 2 becomes 0; only fractional pixels keep coverage.
    assert not eo[5:11, 5:11].any() and not eo[2:4, 2:14].any()
    # Across a tile boundary the left tile sees only the left edge.
    recs, starts, counts, gw = oracle.build_tile_records(rect(4, 4, 28, 20), 0, 0, 32, 32)
    cov = oracle.tile_fill(recs, starts, counts, gw, 32, 32)
    assert (cov[4:16, 2:4] == 255).all() and not cov[4:16, 4:16].any() and (cov[4:16, 16:28] == 255).all()


# ---- GPU: the operators through the C ABI --------------------------------------------

def _outline_segs(oracle, rrb, kind, seed, n_paths, w, h):
    """f32 segments of generated outlines, flattened by the oracle (flatness 0.1)."""
    s = rrb.Scene(kind, seed, n_paths=n_paths, page_w=w, page_h=h)
    out = []
    for i in range(s.n_paths):
        a, b = int(s.path_pt_off[i]), int(s.path_pt_off[i + 1])
        for g in oracle.xpath_new(s.pts[a:b], s.flags[a:b]):
            if g.flags & 0x04:  # stored flipped: the path runs from (x1,y1) to (x0,y0)
                out.append((g.x1, g.y1, g.x0, g.y0))
            else:
                out.append((g.x0, g.y0, g.x1, g.y1))
    return np.asarray(out, np.float32).reshape(-1, 4)


def _cases(oracle, rrb):
    rng = np.random.default_rng(11)
    cases = {}
    # Star polygons with fractional vertices, partly off the coverage window.
    for i, (w, h) in enumerate([(1, 1), (7, 5), (64, 40), (600, 37), (97, 300)]):
        k = 5 + 2 * i
        ang = np.arange(k) * 2 * np.pi * (k // 2) / k
        cx, cy, r = w / 2 + 0.3, h / 2 - 0.2, 0.6 * max(w, h)
        pts = np.stack([cx + r * np.cos(ang), cy + r * np.sin(ang)], 1)
        segs = np.concatenate([pts, np.roll(pts, -1, 0)], 1).astype(np.float32)
        cases[f"star{k}_{w}x{h}"] = (segs, w, h)
    cases["glyphs"] = (_outline_segs(oracle, rrb, 1, 3, 8, 96, 64), 96, 64)
    cases["polygons"] = (_outline_segs(oracle, rrb, 0, 4, 2, 160, 100), 160, 100)
    # Degenerate and non-finite segments mixed into a square.
    bad = np.array([[3, 3, 9, 3], [5, 5, 5, 5], [np.nan, 1, 4, 9], [1, np.nan, 4, 9], [np.inf, 2, 7, 8],
                    [2, -np.inf, 7, 8], [1e30, 0, -1e30, 12], [2, 2, 2.0000001, 11]], np.float32)
    cases["degenerate"] = (np.concatenate([np.asarray(rect(2.5, 1.25, 13.75, 10.5), np.float32).reshape(-1, 4),
                                           bad]), 16, 12)
    # A comb whose sample lines cross ~160 edges (the per-line list overflows).
    teeth = []
    for t in range(80):
        x = 1.0 + 1.5 * t
        teeth += [[x, 1, x, 30], [x + 0.6, 30, x + 0.6, 1]]
    cases["comb"] = (np.asarray(teeth, np.float32), 128, 32)
    # Many segments in one band (more than a band keeps in shared memory).
    ys = rng.uniform(0, 8, (3000, 2)).astype(np.float32)
    xs = rng.uniform(0, 256, (3000, 2)).astype(np.float32)
    many = np.stack([xs[:, 0], ys[:, 0], xs[:, 1], ys[:, 1]], 1)
    cases["many"] = (many, 256, 16)
    return cases


@pytest.fixture(scope="module")
def fill_cases(oracle, rrb_lib):
    return _cases(oracle, rrb_lib)


def _run(backend, fn):
    backend.begin_page()
    try:
        fn()
    finally:
        backend.wait_page(backend.submit_page())


def _dev(backend, arr):
    arr = np.ascontiguousarray(arr)
    buf = backend.alloc_device(max(16, arr.nbytes))
    if arr.nbytes:
        backend.upload_async(buf, arr.view(np.uint8).reshape(-1))
    return buf


@pytest.mark.gpu
@pytest.mark.parametrize("rule", [0, 1])
def test_aa_fill_matches_aa_fill_cpu(backend, oracle, fill_cases, rule):
    for name, (segs, w, h) in fill_cases.items():
        exp = oracle.aa_fill_cpu(segs, 0.0, 0.0, w, h, eo=bool(rule))
        sb, cb = _dev(backend, segs), backend.alloc_device(w * h)
        try:
            backend.upload_async(cb, np.full(w * h, 77, np.uint8))  # every byte is overwritten
            _run(backend, lambda: backend.record_aa_fill(sb, len(segs), cb, w, h, rule))
            got = np.empty(w * h, np.uint8)
            backend.wait_download(backend.download_async(cb, got))
            d = np.nonzero(got != exp.ravel())[0]
            assert d.size == 0, f"{name}: {d.size} bytes differ, first at {d[:5]}"
        finally:
            backend.free_device(sb)
            backend.free_device(cb)


@pytest.mark.gpu
def test_aa_fill_without_segments_is_zero(backend):
    cb = backend.alloc_device(40 * 30)
    sb = backend.alloc_device(16)
    try:
        backend.upload_async(cb, np.full(1200, 9, np.uint8))
        _run(backend, lambda: backend.record_aa_fill(sb, 0, cb, 40, 30, 0))
        got = np.empty(1200, np.uint8)
        backend.wait_download(backend.download_async(cb, got))
        assert not got.any()
    finally:
        backend.free_device(cb)
        backend.free_device(sb)


@pytest.mark.gpu
@pytest.mark.parametrize("rule", [0, 1])
def test_tile_fill_matches_oracle(backend, oracle, fill_cases, rule):
    for name, (segs, w, h) in fill_cases.items():
        recs, starts, counts, gw = oracle.build_tile_records(segs, 0.0, 0.0, w, h)
        exp = oracle.tile_fill(recs, starts, counts, gw, w, h, eo=bool(rule))
        bufs = [_dev(backend, recs if len(recs) else np.zeros(1, oracle.TILE_RECORD)), _dev(backend, starts),
                _dev(backend, counts)]
        cb = backend.alloc_device(w * h)
        try:
            _run(backend, lambda: backend.record_tile_fill(*bufs, cb, w, h, rule))
            got = np.empty(w * h, np.uint8)
            backend.wait_download(backend.download_async(cb, got))
            d = np.nonzero(got != exp.ravel())[0]
            assert d.size == 0, f"{name}: {d.size} bytes differ, first at {d[:5]}"
        finally:
            for b in bufs + [cb]:
                backend.free_device(b)


@pytest.mark.gpu
@pytest.mark.parametrize("rule", [0, 1])
def test_tile_fill_from_segments_matches_oracle(backend, oracle, fill_cases, rule):
    for name, (segs, w, h) in fill_cases.items():
        recs, starts, counts, gw = oracle.build_tile_records(segs, 0.0, 0.0, w, h)
        exp = oracle.tile_fill(recs, starts, counts, gw, w, h, eo=bool(rule))
        sb, cb = _dev(backend, segs), backend.alloc_device(w * h)
        try:
            out = {}
            _run(backend, lambda: out.setdefault("n", backend.record_tile_fill_segs(sb, len(segs), cb, w, h, rule)))
            assert out["n"] == len(recs), name
            got = np.empty(w * h, np.uint8)
            backend.wait_download(backend.download_async(cb, got))
            d = np.nonzero(got != exp.ravel())[0]
            assert d.size == 0, f"{name}: {d.size} bytes differ, first at {d[:5]}"
        finally:
            backend.free_device(sb)
            backend.free_device(cb)


@pytest.mark.gpu
def test_tile_fill_range_past_the_records_is_an_empty_tile(backend, oracle):
    segs = np.asarray(rect(2, 2, 30, 30), np.float32).reshape(-1, 4)
    recs, starts, counts, gw = oracle.build_tile_records(segs, 0.0, 0.0, 32, 32)
    counts = counts.copy()
    counts[3] = len(recs) + 5  # tile (1, 1) claims records that do not exist
    bufs = [_dev(backend, recs), _dev(backend, starts), _dev(backend, counts)]
    cb = backend.alloc_device(32 * 32)
    try:
        _run(backend, lambda: backend.record_tile_fill(*bufs, cb, 32, 32, 0))
        got = np.empty((32, 32), np.uint8)
        backend.wait_download(backend.download_async(cb, got.reshape(-1)))
        exp = oracle.tile_fill(recs, starts, np.where(np.arange(4) == 3, 0, counts), gw, 32, 32)
        assert np.array_equal(got, exp) and not got[16:, 16:].any()
    finally:
        for b in bufs + [cb]:
            backend.free_device(b)


@pytest.mark.gpu
def test_fill_ops_outside_a_page_are_state_errors(backend, rrb_lib):
    sb, cb = backend.alloc_device(64), backend.alloc_device(64)
    try:
        with pytest.raises(rrb_lib.BackendError) as e:
            backend.record_aa_fill(sb, 1, cb, 8, 8, 0)
        assert e.value.status == 9
    finally:
        backend.free_device(sb)
        backend.free_device(cb)
