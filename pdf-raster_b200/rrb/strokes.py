"""Seeded stroke-heavy pages: the vector paint of forms, tables and charts.

A page mixes table rules (hairlines and 1-3 px lines), boxes, chart
polylines with every cap and join, stroked curves, dashed separators and a
few filled shapes, in paint order. Used by the benchmark's stroke workload
and the stroke parity tests; the reference publishes no stroke dataset.
"""

from __future__ import annotations

import numpy as np

from . import RRB_CAP_BUTT, RRB_CAP_PROJECTING, RRB_CAP_ROUND, RRB_JOIN_BEVEL, RRB_JOIN_MITER, RRB_JOIN_ROUND

DESCRIPTION = ("stroke page: {n} paths on one {w}x{h} u8 page (Letter @300 dpi) in paint order — 35% table rules "
               "(hairline / 1-3 px, butt), 20% boxes (hairline / 1-2 px, miter), 20% chart polylines (0.5-6 px, "
               "every cap and join), 10% stroked curves (1-4 px, round), 10% dashed rules, 5% filled shapes; gray "
               "0-200, 10% translucent")


class StrokePage:
    """Arrays of a paint batch (the rrb.Scene attribute names) plus one
    stroke dict (or None for a fill) per path."""

    def __init__(self, seed: int = 0, n_paths: int = 20000, w: int = 2550, h: int = 3300):
        rng = np.random.default_rng(seed)
        pts, fls, strokes = [], [], []
        off = [0]

        def add(p, f, st):
            pts.append(np.asarray(p, float))
            fls.append(np.asarray(f, np.uint8))
            off.append(off[-1] + len(f))
            strokes.append(st)

        for _ in range(n_paths):
            r = rng.random()
            if r < 0.35:  # table rule
                x, y = rng.uniform(0, w), rng.uniform(0, h)
                ln = rng.uniform(20, 900)
                p = [(x, y), (x + ln, y)] if rng.random() < 0.6 else [(x, y), (x, y + ln)]
                add(p, [1, 2], dict(line_width=float(rng.choice([0.0, 0.0, 1.0, 2.0, 3.0])), line_cap=RRB_CAP_BUTT))
            elif r < 0.55:  # box
                x, y = rng.uniform(0, w - 40), rng.uniform(0, h - 40)
                bw, bh = rng.uniform(10, 600), rng.uniform(8, 300)
                add([(x, y), (x + bw, y), (x + bw, y + bh), (x, y + bh), (x, y)], [5, 0, 0, 0, 6],
                    dict(line_width=float(rng.choice([0.0, 1.0, 2.0])), line_join=RRB_JOIN_MITER))
            elif r < 0.75:  # chart polyline
                n = int(rng.integers(3, 13))
                x0, y0 = rng.uniform(0, w - 400), rng.uniform(100, h - 100)
                xs = x0 + np.cumsum(rng.uniform(5, 60, n))
                ys = y0 + np.cumsum(rng.normal(0, 25, n))
                add(np.stack([xs, ys], 1), [1] + [0] * (n - 2) + [2],
                    dict(line_width=float(rng.choice([0.5, 1.5, 3.0, 6.0])),
                         line_cap=int(rng.choice([RRB_CAP_BUTT, RRB_CAP_ROUND, RRB_CAP_PROJECTING])),
                         line_join=int(rng.choice([RRB_JOIN_MITER, RRB_JOIN_ROUND, RRB_JOIN_BEVEL])),
                         miter_limit=float(rng.choice([2.0, 10.0]))))
            elif r < 0.85:  # stroked curve
                k = int(rng.integers(1, 5))
                c = rng.uniform([0, 0], [w, h])
                p, f = [c], [1]
                for _ in range(k):
                    p += [c + rng.normal(0, 60, 2), c + rng.normal(0, 60, 2), c + rng.normal(0, 80, 2)]
                    f += [8, 8, 0]
                    c = p[-1]
                f[-1] = 2
                add(p, f, dict(line_width=float(rng.choice([1.0, 2.0, 4.0])), line_cap=RRB_CAP_ROUND,
                               line_join=RRB_JOIN_ROUND))
            elif r < 0.95:  # dashed rule
                x, y = rng.uniform(0, w), rng.uniform(0, h)
                ln = rng.uniform(50, 1200)
                dashes = ([6.0, 3.0], [2.0, 2.0], [10.0, 4.0, 2.0, 4.0])
                add([(x, y), (x + ln, y + rng.normal(0, 5))], [1, 2],
                    dict(line_width=float(rng.choice([0.0, 1.0, 2.0])), dash=dashes[int(rng.integers(0, 3))],
                         dash_phase=float(rng.uniform(0, 10))))
            else:  # filled shape
                c = rng.uniform([0, 0], [w, h])
                n = int(rng.integers(3, 8))
                ang = np.sort(rng.uniform(0, 2 * np.pi, n))
                rad = rng.uniform(5, 80)
                p = np.stack([c[0] + rad * np.cos(ang), c[1] + rad * np.sin(ang)], 1)
                add(np.vstack([p, p[:1]]), [5] + [0] * (n - 1) + [6], None)
        self.pts = np.concatenate(pts).reshape(-1, 2)
        self.flags = np.concatenate(fls)
        self.path_pt_off = np.array(off, np.uint64)
        self.n_paths = n_paths
        self.n_pts = int(self.flags.size)
        self.fill_rule = np.zeros(n_paths, np.uint8)
        self.gray = rng.integers(0, 201, n_paths).astype(np.uint8)
        self.alpha = np.where(rng.random(n_paths) < 0.1, rng.integers(64, 255, n_paths), 255).astype(np.uint8)
        self.path_page = np.zeros(n_paths, np.uint32)
        self.page_width = np.array([w], np.uint32)
        self.page_height = np.array([h], np.uint32)
        self.page_offset = np.zeros(1, np.uint64)
        self.n_pages = 1
        self.arena_bytes = w * h
        self.strokes = strokes
        self.description = DESCRIPTION.format(n=n_paths, w=w, h=h)

    @property
    def pixels(self) -> int:
        return int(self.page_width[0]) * int(self.page_height[0])

    def blank_arena(self, value: int = 255) -> np.ndarray:
        return np.full(self.arena_bytes, value, np.uint8)
