"""Pin whole-batch parity by page digests (run from the repository root).

    python tests/golden/make_batch_digests.py mixed   [--workers N]
    python tests/golden/make_batch_digests.py serving [--workers N] [--requests 128]

`mixed`   renders every page of the 64-page mixed batch (the seeded
          generator's kind 2, seed 0: {A4, Letter, A3} x {150, 300, 600} dpi,
          30% glyphs / 40% polygons / 30% rectangles, alpha 32-255) with the
          CPU oracle and writes one SHA-256 per page to mixed_batch_digests.json.
`serving` renders the pages that serving requests 0..R-1 ask for. Each request
          is one page of the same generator seeded by its request id
          (kind 2, seed = id, one page), and its digest goes to
          serving_request_digests.json.

The oracle (oracle/, the C++ restatement of the reference CPU scanline
rasterizer) renders each page alone on one thread. Pages run in a process pool
(spawned, largest first). Each record also holds a SHA-256 of the page's
generated inputs, so generator drift is told apart from a rendering change,
and the oracle's counters: rows with more than 20 merged entries and tied x0
(whose order the reference leaves to its unstable sort) and rows whose winding
never returns to zero. Partial results are kept in <out>.partial.json, so an
interrupted run resumes where it stopped.
"""

from __future__ import annotations

import argparse
import hashlib
import json
import multiprocessing as mp
import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
MIXED = dict(kind=2, seed=0)


def _paths(root: Path):
    for p in (root / "pdf-raster_b200", root / "oracle"):
        if str(p) not in sys.path:
            sys.path.insert(0, str(p))


def input_digest(s) -> str:
    """SHA-256 of one page's generated inputs (a SceneShard or a one-page Scene)."""
    h = hashlib.sha256()
    for a in (s.pts, s.flags, s.path_pt_off, s.fill_rule, s.gray, s.alpha, s.page_width, s.page_height):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def page_digest(arena: np.ndarray, offset: int, width: int, height: int) -> str:
    return hashlib.sha256(np.ascontiguousarray(arena[offset:offset + width * height]).tobytes()).hexdigest()


def request_scene(rrb, request_id: int):
    """The one page serving request `request_id` renders."""
    return rrb.Scene(kind=2, seed=int(request_id), n_pages=1)


_STATE = {}


def _init(root: str):
    _paths(Path(root))
    import rr_oracle
    import rrb

    rr_oracle.build()
    _STATE["rrb"], _STATE["oracle"] = rrb, rr_oracle


def _mixed_page(pg: int) -> dict:
    rrb, orc = _STATE["rrb"], _STATE["oracle"]
    if "mixed" not in _STATE:
        _STATE["mixed"] = rrb.Scene(**MIXED)
    from rrb.shard import SceneShard

    sub = SceneShard(_STATE["mixed"], pages=(pg, pg + 1))
    return _render("page", pg, sub, orc)


def _request_page(rid: int) -> dict:
    rrb, orc = _STATE["rrb"], _STATE["oracle"]
    return _render("request", rid, request_scene(rrb, rid), orc)


def _render(key: str, idx: int, s, orc) -> dict:
    arena = s.blank_arena()
    t = time.perf_counter()
    st = orc.render_scene(s, arena)
    secs = time.perf_counter() - t
    w, h = int(s.page_width[0]), int(s.page_height[0])
    return {key: idx, "width": w, "height": h, "paths": int(s.n_paths), "points": int(s.n_pts),
            "input_sha256": input_digest(s), "page_sha256": page_digest(arena, int(s.page_offset[0]), w, h),
            "oracle_s": round(secs, 2), "unpinned_tie_rows": st["unpinned_tie_rows"],
            "nonterminating_rows": st["nonterminating_rows"]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["mixed", "serving"])
    ap.add_argument("--workers", type=int, default=max(1, (os.cpu_count() or 2) - 1))
    ap.add_argument("--requests", type=int, default=128)
    ap.add_argument("--root", default=str(ROOT), help="tree whose built libraries render (default: this one)")
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    _paths(Path(args.root))
    import rrb

    if args.what == "mixed":
        out = Path(args.out or HERE / "mixed_batch_digests.json")
        sc = rrb.Scene(**MIXED)
        from rrb.shard import SceneShard

        cost = []
        for pg in range(sc.n_pages):
            sub = SceneShard(sc, pages=(pg, pg + 1))
            cost.append(sub.n_paths * sub.pixels)
        items, key, fn = list(range(sc.n_pages)), "page", _mixed_page
        header = {"scene": {"generator": "rrb_scene_generate", **MIXED}, "pages": sc.n_pages}
        del sc
    else:
        out = Path(args.out or HERE / "serving_request_digests.json")
        cost = []
        for r in range(args.requests):
            s = request_scene(rrb, r)
            cost.append(s.n_paths * s.pixels)
        items, key, fn = list(range(args.requests)), "request", _request_page
        header = {"scene": {"generator": "rrb_scene_generate", "kind": 2, "seed": "request id", "n_pages": 1},
                  "requests": args.requests}
    partial = out.with_suffix(".partial.json")
    done = {}
    if partial.exists():
        for rec in json.loads(partial.read_text()):
            done[rec[key]] = rec
    todo = sorted((i for i in items if i not in done), key=lambda i: -cost[i])
    print(f"{len(done)} done, {len(todo)} to render on {args.workers} workers", flush=True)
    ctx = mp.get_context("spawn")
    t0 = time.time()
    with ctx.Pool(args.workers, initializer=_init, initargs=(args.root,)) as pool:
        for rec in pool.imap_unordered(fn, todo):
            done[rec[key]] = rec
            partial.write_text(json.dumps(sorted(done.values(), key=lambda r: r[key])))
            print(f"[{time.time() - t0:7.0f}s] {key} {rec[key]}: {rec['paths']} paths, {rec['oracle_s']} s, "
                  f"ties {rec['unpinned_tie_rows']}", flush=True)
    recs = [done[i] for i in items]
    doc = {"about": "SHA-256 of each page rendered by the CPU oracle (documented row map, one thread per page); "
                    "made by tests/golden/make_batch_digests.py", **header,
           "oracle_seconds_total": round(sum(r["oracle_s"] for r in recs), 1), "records": recs}
    out.write_text(json.dumps(doc, indent=1) + "\n")
    partial.unlink(missing_ok=True)
    print("wrote", out)


if __name__ == "__main__":
    main()
