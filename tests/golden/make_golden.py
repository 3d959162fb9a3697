"""Generate the golden fixtures in this directory (run from the repository root).

    python tests/golden/make_golden.py

Each fixture holds the inputs of one render (either the seeded scene
parameters plus a SHA-256 of the generated arrays, or the full arrays for the
hand-made edge-case paths), the expected page bytes produced by the CPU
oracle (oracle/, the restatement of the reference CPU scanline rasterizer),
and the oracle's counters. tests/test_golden.py checks on the CPU that the
oracle and the generator still reproduce them, and on the GPU that the B200
path does, byte for byte.
"""

from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path[:0] = [str(ROOT / "pdf-raster_b200"), str(ROOT / "oracle")]

SCENES = {
    "polygons_320x240": dict(kind=0, seed=3, n_paths=300, page_w=320, page_h=240),
    "glyphs_400x300": dict(kind=1, seed=4, n_paths=1200, page_w=400, page_h=300),
    "mixed_3pages": dict(kind=2, seed=5, n_pages=3, page_scale=0.08, paths_scale=0.01),
}


def scene_hash(s) -> str:
    h = hashlib.sha256()
    for a in (s.pts, s.flags, s.path_pt_off, s.fill_rule, s.gray, s.alpha, s.path_page, s.page_width, s.page_height,
              s.page_offset):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def handmade_paths():
    """Edge cases of the scanline rules, built through the product's PathBuilder."""
    import rrb

    def mk(ops):
        b = rrb.PathBuilder()
        for op, *a in ops:
            getattr(b, op)(*a)
        return b.build()

    paths = [
        mk([("move_to", 3.2, 2.7), ("line_to", 40.9, 5.1), ("line_to", 20.4, 37.3), ("close",)]),
        mk([("move_to", 5.3, 4.8), ("line_to", 50.55, 4.8), ("line_to", 50.55, 30.1), ("line_to", 5.3, 30.1),
            ("close",)]),
        mk([("move_to", 10, 30), ("curve_to", 10, 0, 60, 0, 60, 30), ("curve_to", 60, 55, 10, 55, 10, 30), ("close",)]),
        mk([("move_to", 30, 2), ("line_to", 47, 52), ("line_to", 3, 20), ("line_to", 57, 20), ("line_to", 13, 52),
            ("close",)]),
        mk([("move_to", -20.5, 10.25), ("line_to", 30.75, -12.5), ("line_to", 120.2, 70.6), ("close",)]),
        mk([("move_to", 5, 5), ("line_to", 30, 5), ("curve_to", 30, 20, 15, 30, 5, 5), ("close",),
            ("move_to", 35, 35), ("line_to", 55, 35), ("line_to", 55, 55), ("close",)]),
        mk([("move_to", 10.1, 3), ("line_to", 10.3, 3), ("line_to", 10.3, 50), ("line_to", 10.1, 50), ("close",)]),
        mk([("move_to", 10, 20), ("conic_to", 30, -5, 50, 20), ("conic_to", 30, 45, 10, 20), ("close",)]),
    ]
    ops = [("move_to", 2.0, 2.0)]
    x = 2.0
    for _ in range(40):
        ops += [("line_to", x + 0.7, 2.0), ("line_to", x + 0.7, 50.0), ("line_to", x + 1.3, 50.0),
                ("line_to", x + 1.3, 2.0)]
        x += 1.45
    ops += [("line_to", x, 2.0), ("line_to", x, 58.0), ("line_to", 2.0, 58.0), ("close",)]
    paths.append(mk(ops))
    return paths


def main():
    import rr_oracle
    import rrb

    rr_oracle.build()
    manifest = {}
    for name, params in SCENES.items():
        s = rrb.Scene(**params)
        for rowmap in (0, 1):
            arena = s.blank_arena()
            st = rr_oracle.render_scene(s, arena, rowmap=rowmap)
            key = f"{name}_rowmap{rowmap}"
            np.savez_compressed(HERE / f"{key}.npz", expected=arena)
            manifest[key] = dict(params=params, rowmap=rowmap, input_sha256=scene_hash(s),
                                 expected_sha256=hashlib.sha256(arena.tobytes()).hexdigest(), oracle=st)
    # Hand-made paths: full inputs, one page of 97x61 with a seeded random background.
    paths = handmade_paths()
    rng = np.random.default_rng(12)
    W, H = 97, 61
    init = rng.integers(0, 256, W * H, dtype=np.uint8)
    pts = np.concatenate([p for p, _ in paths])
    flags = np.concatenate([f for _, f in paths])
    off = np.cumsum([0] + [len(f) for _, f in paths]).astype(np.uint64)
    n = len(paths)
    rule = (np.arange(n) % 2).astype(np.uint8)
    gray = rng.integers(0, 256, n, dtype=np.uint8)
    alpha = np.array([255, 200, 37, 255, 128, 255, 90, 255, 255][:n], np.uint8)
    for rowmap in (0, 1):
        arena = init.copy()
        st = rr_oracle.render_arrays(arena, [0], [W], [H], pts, flags, off, rule, gray, alpha, np.zeros(n, np.uint32),
                                     rowmap=rowmap)
        key = f"handmade_rowmap{rowmap}"
        np.savez_compressed(HERE / f"{key}.npz", expected=arena, init=init, pts=pts, flags=flags, path_pt_off=off,
                            fill_rule=rule, gray=gray, alpha=alpha)
        manifest[key] = dict(params=dict(width=W, height=H), rowmap=rowmap,
                             expected_sha256=hashlib.sha256(arena.tobytes()).hexdigest(), oracle=st)
    (HERE / "manifest.json").write_text(json.dumps(manifest, indent=1, sort_keys=True) + "\n")
    print(f"wrote {len(manifest)} fixtures")


if __name__ == "__main__":
    main()
