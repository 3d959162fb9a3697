"""Multi-GPU layout of page rendering: one process per GPU, pages sharded.

Pages are independent units (every path belongs to exactly one page and
composites only onto it), so N ranks split a batch's pages between them and
render their shard with no exchange on the data path. torch.distributed is
used only around the data path: a barrier before timing and a max-over-ranks
reduction of each rank's device time (the slowest rank sets the job's time).
"""

from __future__ import annotations

import numpy as np


def page_shard(n_pages: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous page range [begin, end) of `rank`; ranks get sizes that differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(n_pages, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def shard_arrays(scene, rank: int, world: int) -> dict:
    """The arrays of `scene` (rrb.Scene) restricted to this rank's pages,
    re-based to start at point 0, path 0, page 0 and arena byte 0."""
    return range_arrays(scene, *page_shard(scene.n_pages, rank, world))


def range_arrays(scene, p0: int, p1: int) -> dict:
    """The arrays of `scene` restricted to pages [p0, p1), re-based as in shard_arrays."""
    if not 0 <= p0 <= p1 <= scene.n_pages:
        raise ValueError("page range out of bounds")
    sel = np.nonzero((scene.path_page >= p0) & (scene.path_page < p1))[0]
    if sel.size:
        a, b = int(scene.path_pt_off[sel[0]]), int(scene.path_pt_off[sel[-1] + 1])
        off = scene.path_pt_off[sel[0]:sel[-1] + 2] - a
    else:
        a = b = 0
        off = np.zeros(1, np.uint64)
    page_off = scene.page_offset[p0:p1].astype(np.uint64)
    base = int(page_off[0]) if p1 > p0 else 0
    ends = page_off + scene.page_width[p0:p1].astype(np.uint64) * scene.page_height[p0:p1].astype(np.uint64)
    return {
        "pts": scene.pts[a:b], "flags": scene.flags[a:b], "path_pt_off": off.astype(np.uint64),
        "fill_rule": scene.fill_rule[sel], "gray": scene.gray[sel], "alpha": scene.alpha[sel],
        "path_page": (scene.path_page[sel] - p0).astype(np.uint32),
        "page_width": scene.page_width[p0:p1], "page_height": scene.page_height[p0:p1],
        "page_offset": page_off - base, "arena_bytes": int(ends.max() - base) if p1 > p0 else 0,
        "pages": (p0, p1), "arena_base": base,
    }


def max_over_ranks(value: float, dist=None) -> float:
    """The largest `value` of all ranks (the job's time), or `value` without a process group."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class SceneShard:
    """This rank's pages of an rrb.Scene (or the pages `pages` = [p0, p1)), with
    the Scene attributes a renderer uses (arrays, counts, `view` batch
    parameters, blank_arena); arena_base is the first page's byte offset in the
    whole scene's arena."""

    def __init__(self, scene, rank: int = 0, world: int = 1, pages: tuple[int, int] | None = None):
        from . import batch_params

        sh = range_arrays(scene, *pages) if pages is not None else shard_arrays(scene, rank, world)
        self._scene = scene  # the arrays below can be views of the scene's memory: keep it alive
        self.arena_base = int(sh["arena_base"])
        self.pages_range = sh["pages"]
        for k in ("pts", "flags", "path_pt_off", "fill_rule", "gray", "alpha", "path_page", "page_width",
                  "page_height", "page_offset"):
            setattr(self, k, np.ascontiguousarray(sh[k]))
        self.n_pages = int(self.page_width.size)
        self.n_paths = int(self.fill_rule.size)
        self.n_pts = int(self.flags.size)
        self.arena_bytes = int(sh["arena_bytes"])
        self.n_cubics = int(np.count_nonzero(self.flags & 0x08)) // 2
        self.n_lines = max(0, self.n_pts - 3 * self.n_cubics - int(np.count_nonzero(self.flags & 0x01)))
        self._keep = []
        self.view = batch_params(self.pts, self.flags, self.path_pt_off, self.fill_rule, self.gray, self.alpha,
                                 self.path_page, self.page_width, self.page_height, self.page_offset, None,
                                 keep=self._keep)

    @property
    def pixels(self) -> int:
        return int(np.sum(self.page_width.astype(np.int64) * self.page_height.astype(np.int64)))

    def blank_arena(self, value: int = 255) -> np.ndarray:
        return np.full(self.arena_bytes, value, dtype=np.uint8)
