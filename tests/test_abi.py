"""CPU checks of the C ABI: the library loads, exports every declared symbol,
struct layouts agree with the C compiler, host-side logic matches the oracle,
and malformed batches are rejected without a device (the FakeBackend pattern
of crates/gpu/src/backend/params.rs:978-1075).
"""

import ctypes as C
import re
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "rrb.h"
SCENES_HEADER = ROOT / "include" / "rrb_scenes.h"


def declared_functions(header=HEADER):
    text = re.sub(r"/\*.*?\*/", "", header.read_text(), flags=re.S)
    return sorted(set(re.findall(r"^[A-Za-z_][\w\s\*]*?\b(rrb_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol(rrb_lib):
    lib = rrb_lib.lib()
    names = declared_functions()
    assert len(names) >= 45
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    from rrb import _abi
    assert sorted(_abi.SIGNATURES) == names  # every declaration has a ctypes binding


def test_scene_library_exports_its_header_and_is_separate(rrb_lib):
    """librrb_scenes.so exports rrb_scenes.h; the backend library does not
    carry the generator, and generating a scene maps no backend library."""
    from rrb import scenes
    names = declared_functions(SCENES_HEADER)
    assert names == sorted(scenes.SIGNATURES)
    lib = scenes.lib()
    assert all(hasattr(lib, n) for n in names)
    assert not any(hasattr(rrb_lib.lib(), n) for n in names)
    code = ("import sys; sys.path.insert(0, %r); from rrb.scenes import Scene; s = Scene(2, 1, n_pages=1, "
            "page_scale=0.05, paths_scale=0.01); print(s.n_paths); "
            "print(any('librrb.so' in l for l in open('/proc/self/maps')))" % str(ROOT / "pdf-raster_b200"))
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, check=True).stdout.split()
    assert int(out[0]) > 0 and out[1] == "False"


def test_version_and_status_names(rrb_lib):
    lib = rrb_lib.lib()
    assert b"sm_100a" in lib.rrb_version()
    assert lib.rrb_status_name(0) == b"ok"
    assert lib.rrb_status_name(4) == b"InvariantViolation"


STRUCTS = {
    "rrb_path_fill_params": ("PathFillParams", ["pts", "flags", "n_pts", "matrix", "flatness", "fill_rule", "gray",
                                                "alpha", "rowmap", "page", "page_offset", "width", "height"]),
    "rrb_path_batch_params": ("PathBatchParams", ["pts", "flags", "n_pts", "path_pt_off", "fill_rule", "gray",
                                                  "alpha", "path_page", "n_paths", "page_width", "page_height",
                                                  "page_offset", "n_pages", "pages", "matrix", "flatness", "rowmap"]),
    "rrb_vram_budget": ("VramBudget", ["total_bytes", "free_bytes", "budget_bytes", "used_bytes"]),
    "rrb_tuning": ("Tuning", ["tile_w", "tile_h", "rows_per_chunk", "wave_points", "auto_tile", "reserved"]),
    "rrb_batch_stats": ("BatchStats", ["paths", "pieces", "segments", "aa_rows", "spans", "row_overflows", "tiles",
                                       "tile_pairs", "nonterminating_rows", "kernel_launches", "scratch_grows",
                                       "waves", "host_ns", "row_groups", "host_syncs", "tile_w", "tile_h",
                                       "row_shape", "trials_left"]),
    "rrb_stage_time": ("StageTime", ["name", "ms", "launches"]),
    "rrb_server_config": ("ServerConfig", ["device", "workers", "mem_budget_bytes", "max_batch_pages", "tile_w",
                                           "tile_h", "predict_threads", "reserved"]),
    "rrb_request_result": ("RequestResult", ["status", "latency_ns", "queue_ns"]),
    "rrb_server_stats_t": ("ServerStats", ["completed", "batches", "batched_requests", "queued", "in_use_bytes",
                                           "peak_in_use_bytes", "tile_batches", "prep_ns", "render_ns", "download_ns"]),
    "rrb_server_cost_model": ("ServerCostModel", ["params", "x_mean", "x_std", "y_mean", "y_std", "table", "policy"]),
    "rrb_aa_fill_params": ("AaFillParams", ["segs", "n_segs", "coverage", "width", "height", "fill_rule"]),
    "rrb_tile_record": ("TileRecord", ["key", "x_enter", "dxdy", "y0_tile", "y1_tile", "sign", "pad", "pad2"]),
    "rrb_tile_fill_params": ("TileFillParams", ["records", "tile_starts", "tile_counts", "coverage", "width",
                                                "height", "fill_rule"]),
    "rrb_scan_params": ("ScanParams", ["data", "block_sums", "len_elems", "phase"]),
    "rrb_stroke_params": ("StrokeParams", ["line_width", "miter_limit", "dash_phase", "dash", "n_dash", "line_cap",
                                           "line_join", "stroke", "reserved"]),
    "rrb_scene_params": ("scenes.SceneParams", ["kind", "seed", "n_pages", "n_paths", "page_w", "page_h",
                                                "page_scale", "paths_scale", "path_cap", "reserved"]),
}


def test_struct_layouts_match_c_compiler(rrb_lib, tmp_path):
    from rrb import _abi
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', f'#include "{SCENES_HEADER}"',
             "int main(void){"]
    for cname, (_, fields) in STRUCTS.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in fields:
            lines.append(f'printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-o", str(exe), str(src)], check=True)
    out = dict(l.rsplit(" ", 1) for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                         check=True).stdout.splitlines())
    from rrb import scenes
    for cname, (pyname, fields) in STRUCTS.items():
        st = getattr(scenes, pyname.split(".")[1]) if pyname.startswith("scenes.") else getattr(_abi, pyname)
        assert C.sizeof(st) == int(out[f"{cname} size"]), cname
        for f in fields:
            assert getattr(st, f).offset == int(out[f"{cname}.{f}"]), (cname, f)


def _random_ops(rng, n):
    ops = []
    for _ in range(n):
        k = rng.integers(0, 5)
        if k == 0:
            ops.append(("move_to", tuple(rng.uniform(-50, 50, 2))))
        elif k == 1:
            ops.append(("line_to", tuple(rng.uniform(-50, 50, 2))))
        elif k == 2:
            ops.append(("curve_to", tuple(rng.uniform(-50, 50, 6))))
        elif k == 3:
            ops.append(("close", (bool(rng.integers(0, 2)),)))
        else:
            ops.append(("line_to_first", ()))
    return ops


def test_path_builder_matches_oracle(rrb_lib, oracle):
    rng = np.random.default_rng(7)
    for trial in range(30):
        a, b = rrb_lib.PathBuilder(), oracle.OraclePath()
        first = None
        for op, args in _random_ops(rng, 40):
            if op == "line_to_first":
                if first is None:
                    continue
                op, args = "line_to", first
            if op == "move_to":
                first = args
            ra = rb = 0
            try:
                getattr(a, op)(*args)
            except ValueError as e:
                ra = {"NoCurPt": 1, "BogusPath": 2}[str(e)]
            rb = getattr(b, op)(*args)
            assert ra == rb, (trial, op)
        pa, fa = a.build()
        pb, fb = b.build()
        assert np.array_equal(pa, pb) and np.array_equal(fa, fb)


def test_conic_to_cubic_matches_oracle(rrb_lib, oracle):
    rng = np.random.default_rng(3)
    for _ in range(200):
        p = rng.uniform(-1e4, 1e4, 6)
        assert rrb_lib.conic_to_cubic(p[0:2], p[2:4], p[4:6]) == oracle.conic_to_cubic(p[0:2], p[2:4], p[4:6])


def test_scene_generator_is_seeded(rrb_lib):
    a = rrb_lib.Scene(0, seed=11, n_paths=50, page_w=300, page_h=200)
    b = rrb_lib.Scene(0, seed=11, n_paths=50, page_w=300, page_h=200)
    c = rrb_lib.Scene(0, seed=12, n_paths=50, page_w=300, page_h=200)
    assert np.array_equal(a.pts, b.pts) and np.array_equal(a.flags, b.flags)
    assert not np.array_equal(a.pts[:10], c.pts[:10])
    assert a.n_paths == 50 and a.path_pt_off[-1] == a.n_pts
    g = rrb_lib.Scene(1, seed=0, n_paths=600, page_w=400, page_h=300)
    assert set(np.unique(g.gray)) == {0} and set(np.unique(g.alpha)) == {255}
    assert g.n_lines == 0 and g.n_cubics > 600 * 12  # quadratics elevated to cubics
    m = rrb_lib.Scene(2, seed=0, n_pages=5, page_scale=0.1, paths_scale=0.01)
    assert m.n_pages == 5 and np.all(np.diff(m.path_page.astype(np.int64)) >= 0)
    assert m.alpha.min() >= 32
    with pytest.raises(ValueError):
        rrb_lib.Scene(9)


def _valid_batch(rrb_lib, keep):
    s = rrb_lib.Scene(0, seed=1, n_paths=5, page_w=64, page_h=48)
    keep.append(s)
    return rrb_lib.batch_params(s.pts, s.flags, s.path_pt_off, s.fill_rule, s.gray, s.alpha, s.path_page,
                                s.page_width, s.page_height, s.page_offset, None, keep=keep), s.arena_bytes


def _validate(rrb_lib, p, n):
    msg = C.create_string_buffer(256)
    rc = rrb_lib.lib().rrb_validate_path_batch(C.byref(p), n, msg, 256)
    return rc, msg.value.decode()


@pytest.mark.parametrize("mutate,needle", [
    (lambda p, k: setattr(p, "rowmap", 2), "rowmap"),
    (lambda p, k: setattr(p, "flatness", float("nan")), "flatness"),
    (lambda p, k: p.matrix.__setitem__(0, float("inf")), "matrix"),
    (lambda p, k: setattr(p, "n_pts", p.n_pts - 1), "path_pt_off"),
    (lambda p, k: p.page_width.__setitem__(0, 0), "page width"),
    (lambda p, k: p.page_width.__setitem__(0, 20000), "page width"),
    (lambda p, k: p.fill_rule.__setitem__(2, 7), "fill_rule"),
    (lambda p, k: p.path_page.__setitem__(1, 3), "path_page"),
    (lambda p, k: setattr(p, "pts", None), "null array"),
])
def test_validation_rejects_malformed_batches(rrb_lib, mutate, needle):
    keep = []
    p, n = _valid_batch(rrb_lib, keep)
    assert _validate(rrb_lib, p, n) == (0, "")
    mutate(p, keep)
    rc, msg = _validate(rrb_lib, p, n)
    assert rc == 4 and needle in msg


def test_validation_rejects_short_page_buffer(rrb_lib):
    keep = []
    p, n = _valid_batch(rrb_lib, keep)
    rc, msg = _validate(rrb_lib, p, n - 1)
    assert rc == 4 and "page buffer" in msg


def test_validation_rejects_a_page_offset_that_would_wrap(rrb_lib):
    """page_offset + page bytes computed in 64 bits must not wrap around and
    pass: an offset of 2^64 - 11 is past any buffer."""
    keep = []
    p, n = _valid_batch(rrb_lib, keep)
    off = np.array([np.iinfo(np.uint64).max - 10], np.uint64)
    keep.append(off)
    p.page_offset = off.ctypes.data_as(C.POINTER(C.c_uint64))
    rc, msg = _validate(rrb_lib, p, n)
    assert rc == 4 and "page buffer" in msg


def test_no_device_fails_loudly(rrb_lib):
    """Without a CUDA device the backend raises; it never renders on the CPU."""
    try:
        b = rrb_lib.B200Backend(0)
    except rrb_lib.BackendError as e:
        assert e.kind == "DeviceError"
        return
    b.close()  # a device is present: nothing to check here
