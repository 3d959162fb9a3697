"""rrb — B200-native anti-aliased path fill behind the reference's GpuBackend surface.

`B200Backend` mirrors the reference trait `GpuBackend`
(crates/gpu/src/backend/mod.rs:216-503): alloc_device / alloc_device_zeroed /
free_device / upload_async / download_async / begin_page / record_* /
submit_page / wait_page / detect_vram_budget, with status codes mapped to
`BackendError`-named exceptions. Every call goes through the C ABI of
librrb.so (include/rrb.h); there is no CPU fallback: without the library, or
without a CUDA device, calls raise.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._abi import (RRB_CAP_BUTT, RRB_CAP_PROJECTING, RRB_CAP_ROUND, RRB_FILL_EVEN_ODD,  # noqa: F401
                   RRB_FILL_NONZERO, RRB_JOIN_BEVEL, RRB_JOIN_MITER, RRB_JOIN_ROUND, RRB_ROWMAP_AS_SHIPPED,
                   RRB_ROWMAP_DOCUMENTED, BatchStats, ClipPath, PathBatchParams, PathFillParams, RequestResult,
                   ServerConfig, ServerStats, StageTime, StrokeParams, Tuning, VramBudget)

__all__ = ["B200Backend", "BackendError", "DeviceBuffer", "PinnedBuffer", "Scene", "PathBuilder", "Server", "lib",
           "conic_to_cubic", "RRB_FILL_NONZERO", "RRB_FILL_EVEN_ODD", "RRB_ROWMAP_DOCUMENTED",
           "RRB_ROWMAP_AS_SHIPPED"]

IDENTITY = (1.0, 0.0, 0.0, 1.0, 0.0, 0.0)


def lib() -> C.CDLL:
    return _abi.load()


class BackendError(RuntimeError):
    """A non-zero rrb status; `.kind` is the BackendError variant name."""

    def __init__(self, status: int, message: str):
        self.status = status
        self.kind = lib().rrb_status_name(status).decode()
        super().__init__(f"{self.kind}: {message}")


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


@dataclass
class DeviceBuffer:
    handle: int
    size: int

    @property
    def ptr(self) -> int:
        return lib().rrb_device_ptr(self.handle) or 0


@dataclass
class PinnedBuffer:
    handle: int
    size: int

    def array(self) -> np.ndarray:
        p = lib().rrb_host_ptr(self.handle)
        return np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint8)), shape=(self.size,))


class PathBuilder:
    """PathBuilder::{move_to,line_to,curve_to,close} (crates/raster/src/path/mod.rs:310-448)."""

    ERRORS = {1: "NoCurPt", 2: "BogusPath"}

    def __init__(self):
        self._h = lib().rrb_path_new()

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            lib().rrb_path_free(h)

    def _chk(self, rc: int):
        if rc:
            raise ValueError(self.ERRORS.get(rc, str(rc)))

    def move_to(self, x, y):
        self._chk(lib().rrb_path_move_to(self._h, x, y))

    def line_to(self, x, y):
        self._chk(lib().rrb_path_line_to(self._h, x, y))

    def curve_to(self, x1, y1, x2, y2, x3, y3):
        self._chk(lib().rrb_path_curve_to(self._h, x1, y1, x2, y2, x3, y3))

    def conic_to(self, xc, yc, x3, y3):
        self._chk(lib().rrb_path_conic_to(self._h, xc, yc, x3, y3))

    def close(self, force: bool = False):
        self._chk(lib().rrb_path_close(self._h, int(force)))

    def build(self):
        """Return copies of (pts[n,2] f64, flags[n] u8)."""
        n = lib().rrb_path_len(self._h)
        if n == 0:
            return np.zeros((0, 2)), np.zeros(0, np.uint8)
        pts = np.ctypeslib.as_array(lib().rrb_path_pts(self._h), shape=(n * 2,)).reshape(n, 2).copy()
        fl = np.ctypeslib.as_array(lib().rrb_path_flags(self._h), shape=(n,)).copy()
        return pts, fl


def conic_to_cubic(p0, pc, p3):
    out = (C.c_double * 4)()
    lib().rrb_conic_to_cubic(p0[0], p0[1], pc[0], pc[1], p3[0], p3[1], out)
    return (out[0], out[1]), (out[2], out[3])


from .scenes import Scene  # noqa: E402  (the seeded workloads; librrb_scenes.so)


def batch_params(pts, flags, path_pt_off, fill_rule, gray, alpha, path_page, page_width, page_height,
                 page_offset, pages: DeviceBuffer | None, matrix=IDENTITY, flatness=0.1,
                 rowmap=RRB_ROWMAP_DOCUMENTED, keep=None) -> PathBatchParams:
    """Build a PathBatchParams over numpy arrays (kept alive through `keep`)."""
    arrs = dict(
        pts=np.ascontiguousarray(pts, np.float64).reshape(-1),
        flags=np.ascontiguousarray(flags, np.uint8),
        path_pt_off=np.ascontiguousarray(path_pt_off, np.uint64),
        fill_rule=np.ascontiguousarray(fill_rule, np.uint8),
        gray=np.ascontiguousarray(gray, np.uint8),
        alpha=np.ascontiguousarray(alpha, np.uint8),
        path_page=np.ascontiguousarray(path_page, np.uint32),
        page_width=np.ascontiguousarray(page_width, np.uint32),
        page_height=np.ascontiguousarray(page_height, np.uint32),
        page_offset=np.ascontiguousarray(page_offset, np.uint64),
    )
    if keep is not None:
        keep.extend(arrs.values())
    p = PathBatchParams()
    p.pts = _ptr(arrs["pts"], C.c_double)
    p.flags = _ptr(arrs["flags"], C.c_uint8)
    p.n_pts = arrs["flags"].size
    p.path_pt_off = _ptr(arrs["path_pt_off"], C.c_uint64)
    p.fill_rule = _ptr(arrs["fill_rule"], C.c_uint8)
    p.gray = _ptr(arrs["gray"], C.c_uint8)
    p.alpha = _ptr(arrs["alpha"], C.c_uint8)
    p.path_page = _ptr(arrs["path_page"], C.c_uint32)
    p.n_paths = arrs["fill_rule"].size
    p.page_width = _ptr(arrs["page_width"], C.c_uint32)
    p.page_height = _ptr(arrs["page_height"], C.c_uint32)
    p.page_offset = _ptr(arrs["page_offset"], C.c_uint64)
    p.n_pages = arrs["page_width"].size
    p.pages = pages.handle if pages is not None else None
    for i in range(6):
        p.matrix[i] = matrix[i]
    p.flatness = flatness
    p.rowmap = rowmap
    return p


class B200Backend:
    """The B200 backend: one device, one stream (GpuBackend, mod.rs:216-503)."""

    def __init__(self, device: int = 0, mem_budget: int = 0):
        h = C.c_void_p()
        rc = lib().rrb_init(device, mem_budget, C.byref(h))
        if rc:
            raise BackendError(rc, f"rrb_init(device={device}) failed")
        self._h = h.value

    def close(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            lib().rrb_destroy(h)

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> int:
        return self._h

    def _chk(self, rc: int):
        if rc:
            raise BackendError(rc, lib().rrb_last_error_message(self._h).decode())

    # ---- memory
    def alloc_device(self, size: int) -> DeviceBuffer:
        h = C.c_void_p()
        self._chk(lib().rrb_alloc_device(self._h, size, C.byref(h)))
        return DeviceBuffer(h.value, size)

    def alloc_device_zeroed(self, size: int) -> DeviceBuffer:
        h = C.c_void_p()
        self._chk(lib().rrb_alloc_device_zeroed(self._h, size, C.byref(h)))
        return DeviceBuffer(h.value, size)

    def device_buffer_len(self, buf: DeviceBuffer) -> int:
        return int(lib().rrb_device_buffer_len(buf.handle))

    def free_device(self, buf: DeviceBuffer):
        self._chk(lib().rrb_free_device(self._h, buf.handle))

    def alloc_host_pinned(self, size: int) -> PinnedBuffer:
        h = C.c_void_p()
        self._chk(lib().rrb_alloc_host_pinned(self._h, size, C.byref(h)))
        return PinnedBuffer(h.value, size)

    def free_host_pinned(self, buf: PinnedBuffer):
        self._chk(lib().rrb_free_host_pinned(self._h, buf.handle))

    # ---- transfers
    def upload_async(self, dst: DeviceBuffer, src: np.ndarray, offset: int = 0) -> int:
        src = np.ascontiguousarray(src)
        f = C.c_uint64()
        self._chk(lib().rrb_upload_async(self._h, dst.handle, offset, src.ctypes.data, src.nbytes, C.byref(f)))
        return f.value

    def download_async(self, src: DeviceBuffer, dst: np.ndarray, offset: int = 0) -> int:
        assert dst.flags["C_CONTIGUOUS"]
        f = C.c_uint64()
        self._chk(lib().rrb_download_async(self._h, src.handle, offset, dst.ctypes.data, dst.nbytes, C.byref(f)))
        return f.value

    def wait_download(self, fence: int):
        self._chk(lib().rrb_wait_download(self._h, fence))

    def submit_transfer(self) -> int:
        f = C.c_uint64()
        self._chk(lib().rrb_submit_transfer(self._h, C.byref(f)))
        return f.value

    def wait_transfer(self, fence: int, timeout_ns: int = 0):
        self._chk(lib().rrb_wait_transfer(self._h, fence, timeout_ns))

    def detect_vram_budget(self) -> VramBudget:
        b = VramBudget()
        self._chk(lib().rrb_detect_vram_budget(self._h, C.byref(b)))
        return b

    # ---- page state machine
    def begin_page(self):
        self._chk(lib().rrb_begin_page(self._h))

    def record_zero_buffer(self, buf: DeviceBuffer):
        self._chk(lib().rrb_record_zero_buffer(self._h, buf.handle))

    def submit_page(self) -> int:
        f = C.c_uint64()
        self._chk(lib().rrb_submit_page(self._h, C.byref(f)))
        return f.value

    def wait_page(self, fence: int, timeout_ns: int = 0):
        self._chk(lib().rrb_wait_page(self._h, fence, timeout_ns))

    def record_path_fill(self, pts, flags, page: DeviceBuffer, width: int, height: int, *, fill_rule=0,
                         gray=0, alpha=255, rowmap=RRB_ROWMAP_DOCUMENTED, matrix=IDENTITY, flatness=0.1,
                         page_offset=0):
        pts = np.ascontiguousarray(pts, np.float64).reshape(-1)
        flags = np.ascontiguousarray(flags, np.uint8)
        p = PathFillParams()
        p.pts = _ptr(pts, C.c_double)
        p.flags = _ptr(flags, C.c_uint8)
        p.n_pts = flags.size
        for i in range(6):
            p.matrix[i] = matrix[i]
        p.flatness = flatness
        p.fill_rule, p.gray, p.alpha, p.rowmap = fill_rule, gray, alpha, rowmap
        p.page = page.handle
        p.page_offset = page_offset
        p.width, p.height = width, height
        self._chk(lib().rrb_record_path_fill(self._h, C.byref(p)))

    def record_path_fill_static(self, pts, flags, page: DeviceBuffer, width: int, height: int, *, fill_rule=0,
                                gray=0, alpha=255, rowmap=RRB_ROWMAP_DOCUMENTED, matrix=IDENTITY, flatness=0.1,
                                page_offset=0):
        """record_path_fill without device allocation (rrb_record_path_fill_static)."""
        self._chk(lib().rrb_record_path_fill_static(
            self._h, C.byref(self._fill_params(pts, flags, page, width, height, fill_rule, gray, alpha, rowmap,
                                               matrix, flatness, page_offset))))

    @staticmethod
    def _fill_params(pts, flags, page, width, height, fill_rule, gray, alpha, rowmap, matrix, flatness,
                     page_offset) -> PathFillParams:
        pts = np.ascontiguousarray(pts, np.float64).reshape(-1)
        flags = np.ascontiguousarray(flags, np.uint8)
        p = PathFillParams()
        p._keep = (pts, flags)
        p.pts = _ptr(pts, C.c_double)
        p.flags = _ptr(flags, C.c_uint8)
        p.n_pts = flags.size
        for i in range(6):
            p.matrix[i] = matrix[i]
        p.flatness = flatness
        p.fill_rule, p.gray, p.alpha, p.rowmap = fill_rule, gray, alpha, rowmap
        p.page = page.handle
        p.page_offset = page_offset
        p.width, p.height = width, height
        return p

    # ---- the reference's coverage operators (record_aa_fill / record_tile_fill)
    def record_aa_fill(self, segs: DeviceBuffer, n_segs: int, coverage: DeviceBuffer, width: int, height: int,
                       fill_rule: int = 0):
        p = _abi.AaFillParams(segs=segs.handle, n_segs=n_segs, coverage=coverage.handle, width=width,
                              height=height, fill_rule=fill_rule)
        self._chk(lib().rrb_record_aa_fill(self._h, C.byref(p)))

    def record_tile_fill(self, records: DeviceBuffer, tile_starts: DeviceBuffer, tile_counts: DeviceBuffer,
                         coverage: DeviceBuffer, width: int, height: int, fill_rule: int = 0):
        p = _abi.TileFillParams(records=records.handle, tile_starts=tile_starts.handle,
                                tile_counts=tile_counts.handle, coverage=coverage.handle, width=width,
                                height=height, fill_rule=fill_rule)
        self._chk(lib().rrb_record_tile_fill(self._h, C.byref(p)))

    def record_tile_fill_segs(self, segs: DeviceBuffer, n_segs: int, coverage: DeviceBuffer, width: int,
                              height: int, fill_rule: int = 0) -> int:
        """tile_fill with the records built on the device; returns the record count."""
        p = _abi.AaFillParams(segs=segs.handle, n_segs=n_segs, coverage=coverage.handle, width=width,
                              height=height, fill_rule=fill_rule)
        n = C.c_uint64()
        self._chk(lib().rrb_record_tile_fill_segs(self._h, C.byref(p), C.byref(n)))
        return int(n.value)

    def record_scan(self, data: DeviceBuffer, block_sums: DeviceBuffer, len_elems: int, phase: int):
        """GpuBackend::record_scan: one phase (0 per-tile, 1 block sums, 2 scatter) of the in-place
        exclusive u32 scan; call 0, 1, 2 in order inside begin_page/submit_page."""
        p = _abi.ScanParams(data=data.handle, block_sums=block_sums.handle, len_elems=len_elems, phase=phase)
        self._chk(lib().rrb_record_scan(self._h, C.byref(p)))

    def record_path_batch_rgb(self, params: PathBatchParams, path_rgb: np.ndarray):
        """Rgb8 pages (3 bytes per pixel): path p painted with path_rgb[p] = (r, g, b)."""
        rgb = np.ascontiguousarray(path_rgb, np.uint8).reshape(-1)
        self._chk(lib().rrb_record_path_batch_rgb(self._h, C.byref(params), _ptr(rgb, C.c_uint8)))

    def record_path_batch_ex(self, params: PathBatchParams, path_rgb: np.ndarray | None = None,
                             clip_rects: np.ndarray | None = None, visit_rows: np.ndarray | None = None):
        """Gray or (path_rgb) Rgb8 pages; clip_rects [n_paths, 4] device-space (x0, y0, x1, y1) or None;
        visit_rows [n_paths, 2] pixel rows the shipped row map's loop visits per path (INT32_MIN: its own),
        or None (rrb_record_path_batch_visit)."""
        rgb = None if path_rgb is None else np.ascontiguousarray(path_rgb, np.uint8).reshape(-1)
        clip = None if clip_rects is None else np.ascontiguousarray(clip_rects, np.float64).reshape(-1)
        if visit_rows is None:
            self._chk(lib().rrb_record_path_batch_ex(self._h, C.byref(params),
                                                     None if rgb is None else _ptr(rgb, C.c_uint8),
                                                     None if clip is None else _ptr(clip, C.c_double)))
            return
        vis = np.ascontiguousarray(visit_rows, np.int32).reshape(-1)
        self._chk(lib().rrb_record_path_batch_visit(self._h, C.byref(params),
                                                    None if rgb is None else _ptr(rgb, C.c_uint8),
                                                    None if clip is None else _ptr(clip, C.c_double),
                                                    _ptr(vis, C.c_int32)))

    def record_path_batch_clip_paths(self, params: PathBatchParams, clip_paths, clip_rects: np.ndarray | None = None,
                                     path_rgb: np.ndarray | None = None):
        """The batch with clip paths per fill (clip_paths[p] = None, (pts, flags, even_odd) or a list of them)
        and optional clip rectangles: rrb_lower_clip_paths, then rrb_record_path_batch_ex on the lowered batch."""
        low = lower_clip_paths(params, clip_paths, clip_rects)
        n = int(params.n_paths)
        asa = np.ctypeslib.as_array
        src = low["src_path"]
        gray = asa(params.gray, shape=(max(1, n),))[:n][src]
        alpha = asa(params.alpha, shape=(max(1, n),))[:n][src]
        page = asa(params.path_page, shape=(max(1, n),))[:n][src]
        keep = []
        npg = int(params.n_pages)
        lowered = batch_params(low["pts"], low["flags"], low["path_pt_off"], low["fill_rule"], gray, alpha, page,
                               asa(params.page_width, shape=(npg,)).copy(), asa(params.page_height, shape=(npg,)).copy(),
                               asa(params.page_offset, shape=(npg,)).copy(), None, flatness=params.flatness,
                               rowmap=params.rowmap, keep=keep)
        lowered.pages = params.pages
        rgb = None if path_rgb is None else np.ascontiguousarray(path_rgb, np.uint8).reshape(-1, 3)[src]
        self.record_path_batch_ex(lowered, rgb, low["clip_rects"], low["visit_rows"])

    def record_stroke_batch(self, params: PathBatchParams, strokes, path_rgb: np.ndarray | None = None,
                            clip_rects: np.ndarray | None = None):
        """Paint the batch in path order: path p stroked with strokes[p] (a
        dict: line_width, line_cap, line_join, miter_limit, dash, dash_phase)
        or filled when strokes[p] is None; or strokes = an array made once by
        stroke_params (kept alive by the caller). path_rgb / clip_rects as in
        record_path_batch_ex."""
        keep = []
        # A prebuilt array (stroke_params(...)) is passed as it is; a list of dicts is converted.
        sp = strokes if isinstance(strokes, C.Array) else stroke_params(strokes, keep)
        rgb = None if path_rgb is None else np.ascontiguousarray(path_rgb, np.uint8).reshape(-1)
        clip = None if clip_rects is None else np.ascontiguousarray(clip_rects, np.float64).reshape(-1)
        self._chk(lib().rrb_record_stroke_batch(self._h, C.byref(params), sp,
                                                None if rgb is None else _ptr(rgb, C.c_uint8),
                                                None if clip is None else _ptr(clip, C.c_double)))

    def record_rgb_to_gray(self, rgb: DeviceBuffer, gray: DeviceBuffer, n_px: int, rgb_offset: int = 0,
                           gray_offset: int = 0):
        self._chk(lib().rrb_record_rgb_to_gray(self._h, rgb.handle, rgb_offset, gray.handle, gray_offset, n_px))

    def record_path_batch(self, params: PathBatchParams):
        self._chk(lib().rrb_record_path_batch(self._h, C.byref(params)))

    def render_pages_host(self, params: PathBatchParams, host_pages: np.ndarray, init: int | None = None):
        """Render onto host pages in one call: their content goes up, the pages come back. With
        init (0..255) the pages start as that byte, filled on the device (no page upload)."""
        assert host_pages.dtype == np.uint8 and host_pages.flags["C_CONTIGUOUS"]
        if init is None:
            self._chk(lib().rrb_render_pages_host(self._h, C.byref(params), host_pages.ctypes.data,
                                                  host_pages.nbytes))
        else:
            self._chk(lib().rrb_render_pages_host_init(self._h, C.byref(params), host_pages.ctypes.data,
                                                       host_pages.nbytes, int(init)))

    def record_fill_buffer(self, buf: DeviceBuffer, value: int, offset: int = 0, length: int | None = None):
        n = buf.size - offset if length is None else length
        self._chk(lib().rrb_record_fill_buffer(self._h, buf.handle, offset, n, value))

    # ---- device-resident batches
    def batch_upload(self, params: PathBatchParams) -> "ResidentBatch":
        h = C.c_void_p()
        self._chk(lib().rrb_batch_upload(self._h, C.byref(params), C.byref(h)))
        return ResidentBatch(self, h.value)

    def record_batch(self, batch: "ResidentBatch", pages: DeviceBuffer, rowmap: int = RRB_ROWMAP_DOCUMENTED):
        self._chk(lib().rrb_record_batch(self._h, batch.handle, pages.handle, rowmap))

    # ---- profiling
    @property
    def stream(self) -> int:
        """cudaStream_t of this backend (every call is ordered on it)."""
        return int(lib().rrb_stream(self._h) or 0)

    def set_profiling(self, enable: bool = True):
        self._chk(lib().rrb_set_profiling(self._h, int(enable)))

    def stage_times(self) -> dict:
        buf = (StageTime * 32)()
        n = C.c_int()
        self._chk(lib().rrb_last_stage_times(self._h, buf, 32, C.byref(n)))
        return {buf[i].name.decode(): (float(buf[i].ms), int(buf[i].launches)) for i in range(min(n.value, 32))}

    # ---- tuning / stats
    def set_tuning(self, tile_w: int = 0, tile_h: int = 0, wave_points: int | None = None,
                   auto_tile: bool | None = None):
        """Tile shape (16x16 / 32x32 / 64x16 / 128x16 / 128x32) and, if given, path points per page wave
        (0 = default). auto_tile: resident batches choose 64x16, 128x16 or 128x32 by trial (a given tile
        shape turns it off unless auto_tile is passed)."""
        auto = 0 if auto_tile is None else (1 if auto_tile else 2)
        t = Tuning(tile_w=tile_w, tile_h=tile_h, wave_points=0xFFFFFFFF if wave_points is None else wave_points,
                   auto_tile=auto)
        self._chk(lib().rrb_set_tuning(self._h, C.byref(t)))

    def get_tuning(self) -> Tuning:
        t = Tuning()
        self._chk(lib().rrb_get_tuning(self._h, C.byref(t)))
        return t

    def last_batch_stats(self) -> dict:
        s = BatchStats()
        self._chk(lib().rrb_last_batch_stats(self._h, C.byref(s)))
        return {n: int(getattr(s, n)) for n, _ in BatchStats._fields_}

    # ---- convenience: render a Scene into a host arena, end to end
    def render_scene(self, scene: Scene, host_arena: np.ndarray, pages: DeviceBuffer | None = None,
                     rowmap=RRB_ROWMAP_DOCUMENTED):
        """Upload `host_arena`, render every path of `scene` into it on the device, download it."""
        own = pages is None
        if own:
            pages = self.alloc_device(max(1, scene.arena_bytes))
        scene.view.pages = pages.handle
        scene.view.rowmap = rowmap
        try:
            self.render_pages_host(scene.view, host_arena)
        finally:
            scene.view.pages = None
            if own:
                self.free_device(pages)


class ResidentBatch:
    """A path batch whose inputs stay in device memory (rrb_batch_upload)."""

    def __init__(self, backend: B200Backend, handle: int):
        self.backend, self.handle = backend, handle

    def record(self, pages: DeviceBuffer, rowmap: int = RRB_ROWMAP_DOCUMENTED):
        self.backend.record_batch(self, pages, rowmap)

    def free(self):
        h, self.handle = self.handle, None
        if h and self.backend.handle:
            self.backend._chk(lib().rrb_batch_free(self.backend.handle, h))


class Server:
    """Continuous-batching page-render server (rrb_server_*)."""

    def __init__(self, device: int = 0, workers: int = 2, mem_budget: int = 0, max_batch_pages: int = 64,
                 tile: tuple[int, int] = (0, 0), predict_threads: int = 0):
        cfg = ServerConfig(device=device, workers=workers, mem_budget_bytes=mem_budget,
                           max_batch_pages=max_batch_pages, tile_w=tile[0], tile_h=tile[1],
                           predict_threads=predict_threads)
        h = C.c_void_p()
        rc = lib().rrb_server_create(C.byref(cfg), C.byref(h))
        if rc:
            raise BackendError(rc, "rrb_server_create failed")
        self._h = h.value
        self._keep = {}

    def submit(self, params: PathBatchParams, host_pages: np.ndarray, init: int = 255, keep=None) -> int:
        """Queue a render; `params`' arrays and `host_pages` must live until wait()."""
        t = C.c_uint64()
        rc = lib().rrb_server_submit(self._h, C.byref(params), host_pages.ctypes.data, host_pages.nbytes, init,
                                     C.byref(t))
        if rc:
            raise BackendError(rc, "rrb_server_submit rejected the request")
        self._keep[t.value] = (params, host_pages, keep)
        return t.value

    def wait(self, ticket: int, timeout_ns: int = 0) -> dict:
        r = RequestResult()
        rc = lib().rrb_server_wait(self._h, ticket, timeout_ns, C.byref(r))
        self._keep.pop(ticket, None)
        if rc:
            raise BackendError(rc, f"request {ticket} failed")
        return {"latency_ns": int(r.latency_ns), "queue_ns": int(r.queue_ns)}

    def stats(self) -> dict:
        s = ServerStats()
        lib().rrb_server_stats(self._h, C.byref(s))
        out = {n: int(getattr(s, n)) for n, _ in ServerStats._fields_ if n != "tile_batches"}
        out["tile_batches"] = [int(v) for v in s.tile_batches]
        return out

    def set_cost_model(self, model=None, table=None, shortest_first=True, tile_by_model=True):
        """Scheduler policy from a trained rrb.autotune.CostModel (or only its table)."""
        keep = []

        def f32(a):
            a = np.ascontiguousarray(a, np.float32)
            keep.append(a)
            return _ptr(a, C.c_float)

        m = _abi.ServerCostModel()
        if model is not None:
            m.params, m.x_mean, m.x_std = f32(model.params), f32(model.x_mean), f32(model.x_std)
            m.y_mean, m.y_std = model.y_mean, model.y_std
            table = model.table if table is None else table
        if table is not None:
            t = np.ascontiguousarray(table, np.int32)
            keep.append(t)
            m.table = _ptr(t, C.c_int32)
        m.policy = (_abi.RRB_SCHED_SHORTEST_FIRST if shortest_first else 0) | \
                   (_abi.RRB_SCHED_TILE_BY_MODEL if tile_by_model else 0)
        rc = lib().rrb_server_set_cost_model(self._h, C.byref(m))
        if rc:
            raise BackendError(rc, "rrb_server_set_cost_model failed")

    def close(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            lib().rrb_server_destroy(h)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        self.close()


def stroke_params(strokes, keep: list) -> "C.Array":
    """StrokeParams array, one per path, from dicts (None: fill the path)."""
    arr = (StrokeParams * max(1, len(strokes)))()
    for i, d in enumerate(strokes):
        if d is None:
            continue
        dash = np.ascontiguousarray(d.get("dash", ()), np.float64)
        keep.append(dash)
        arr[i].line_width = float(d["line_width"])
        arr[i].miter_limit = float(d.get("miter_limit", 10.0))
        arr[i].dash_phase = float(d.get("dash_phase", 0.0))
        arr[i].dash = _ptr(dash, C.c_double) if dash.size else None
        arr[i].n_dash = int(dash.size)
        arr[i].line_cap = int(d.get("line_cap", RRB_CAP_BUTT))
        arr[i].line_join = int(d.get("line_join", RRB_JOIN_MITER))
        arr[i].stroke = 1
    return arr


def lower_clip_paths(params: PathBatchParams, clip_paths, clip_rects=None) -> dict:
    """rrb_lower_clip_paths (host): the batch with clip_paths[p] = None, (pts, flags, even_odd), or a list of
    them (a stack applied in order) per path and optional clip_rects [n_paths, 4], as a rectangle-clipped
    batch: dict of pts [n, 2], flags, path_pt_off, fill_rule, src_path (the input path of each lowered path),
    clip_rects [m, 4] and visit_rows [m, 2] (the pixel rows the shipped row map's loop visits; INT32_MIN: the
    path's own)."""
    n = int(params.n_paths)
    keep = []
    cps = None

    def fill(entry, c):
        pts, fl, eo = c
        a = np.ascontiguousarray(pts, np.float64).reshape(-1)
        f = np.ascontiguousarray(fl, np.uint8)
        keep.extend((a, f))
        entry.pts = _ptr(a, C.c_double) if f.size else None
        entry.flags = _ptr(f, C.c_uint8) if f.size else None
        entry.n_pts = f.size
        entry.even_odd = int(bool(eo))

    if clip_paths is not None:
        cps = (ClipPath * max(1, n))()
        for i, c in enumerate(clip_paths):
            if c is None:
                continue
            stack = list(c) if isinstance(c, list) else [c]
            fill(cps[i], stack[0])
            if len(stack) > 1:
                rest = (ClipPath * (len(stack) - 1))()
                keep.append(rest)
                for j, cj in enumerate(stack[1:]):
                    fill(rest[j], cj)
                prev = cps[i]
                for j in range(len(stack) - 1):
                    prev.next = C.pointer(rest[j])
                    prev = rest[j]
    rect = None if clip_rects is None else np.ascontiguousarray(clip_rects, np.float64).reshape(-1)
    rp = None if rect is None else _ptr(rect, C.c_double)
    npt, npa = C.c_uint64(), C.c_uint64()
    rc = lib().rrb_lower_clip_paths(C.byref(params), rp, cps, None, None, 0, None, None, None, None, None, 0,
                                    C.byref(npt), C.byref(npa))
    if rc:
        raise BackendError(rc, "rrb_lower_clip_paths")
    m, k = npt.value, npa.value
    pts = np.zeros(2 * max(1, m), np.float64)
    fl = np.zeros(max(1, m), np.uint8)
    off = np.zeros(k + 1, np.uint64)
    src = np.zeros(max(1, k), np.uint64)
    rule = np.zeros(max(1, k), np.uint8)
    rects = np.zeros(4 * max(1, k), np.float64)
    visit = np.zeros(2 * max(1, k), np.int32)
    rc = lib().rrb_lower_clip_paths(C.byref(params), rp, cps, _ptr(pts, C.c_double), _ptr(fl, C.c_uint8), m,
                                    _ptr(off, C.c_uint64), _ptr(src, C.c_uint64), _ptr(rule, C.c_uint8),
                                    _ptr(rects, C.c_double), _ptr(visit, C.c_int32), k + 1, C.byref(npt),
                                    C.byref(npa))
    if rc:
        raise BackendError(rc, "rrb_lower_clip_paths")
    return dict(pts=pts[: 2 * m].reshape(m, 2), flags=fl[:m], path_pt_off=off, fill_rule=rule[:k],
                src_path=src[:k].astype(np.int64), clip_rects=rects[: 4 * k].reshape(k, 4),
                visit_rows=visit[: 2 * k].reshape(k, 2))


def stroke_outline(pts, flags, flatness: float = 0.1, **stroke):
    """What rrb_record_stroke_batch draws for one path (host): (kind, pts[n, 2],
    flags[n]); kind 0 nothing, 1 an outline filled nonzero, 2 a hairline polyline."""
    p = np.ascontiguousarray(np.reshape(pts, -1), np.float64)
    f = np.ascontiguousarray(flags, np.uint8)
    keep = []
    sp = stroke_params([stroke], keep)
    n, kind = C.c_uint64(), C.c_int()
    rc = lib().rrb_stroke_outline(_ptr(p, C.c_double), _ptr(f, C.c_uint8), f.size, sp, flatness, None, None, 0,
                                  C.byref(n), C.byref(kind))
    if rc:
        raise BackendError(rc, "rrb_stroke_outline")
    xy = np.empty(2 * n.value, np.float64)
    fl = np.empty(n.value, np.uint8)
    if n.value:
        rc = lib().rrb_stroke_outline(_ptr(p, C.c_double), _ptr(f, C.c_uint8), f.size, sp, flatness,
                                      _ptr(xy, C.c_double), _ptr(fl, C.c_uint8), n.value, C.byref(n), C.byref(kind))
        if rc:
            raise BackendError(rc, "rrb_stroke_outline")
    return kind.value, xy.reshape(-1, 2), fl


def encode_netpbm(page: np.ndarray) -> bytes:
    """P5 (a [h, w] Gray8 page) or P6 (a [h, w, 3] Rgb8 page) bytes (rrb_encode_netpbm)."""
    page = np.ascontiguousarray(page, np.uint8)
    h, w = page.shape[:2]
    ch = 1 if page.ndim == 2 else page.shape[2]
    n = C.c_size_t()
    rc = lib().rrb_encode_netpbm(page.ctypes.data, w, h, ch, None, 0, C.byref(n))
    if rc:
        raise BackendError(rc, "rrb_encode_netpbm")
    out = np.empty(n.value, np.uint8)
    rc = lib().rrb_encode_netpbm(page.ctypes.data, w, h, ch, out.ctypes.data, out.size, C.byref(n))
    if rc:
        raise BackendError(rc, "rrb_encode_netpbm")
    return out.tobytes()


TILE_SHAPES = ((16, 16), (32, 32), (64, 16))


def page_features(params: PathBatchParams, page: int, tile: tuple[int, int]) -> np.ndarray:
    """The cost model's 24 features of one page for one tile shape (rrb_page_features)."""
    out = np.zeros(_abi.RRB_MLP_IN, np.float32)
    rc = lib().rrb_page_features(C.byref(params), page, tile[0], tile[1], _ptr(out, C.c_float))
    if rc:
        raise BackendError(rc, "rrb_page_features")
    return out


def page_features_all(params: PathBatchParams, page: int) -> np.ndarray:
    """[3, 24] features of one page for the tile shapes of TILE_SHAPES (rrb_page_features_all)."""
    out = np.zeros((3, _abi.RRB_MLP_IN), np.float32)
    rc = lib().rrb_page_features_all(C.byref(params), page, _ptr(out, C.c_float))
    if rc:
        raise BackendError(rc, "rrb_page_features_all")
    return out


def aa_fill_jitter() -> tuple[np.ndarray, np.ndarray]:
    """The 64 (x, y) sample offsets of rrb_record_aa_fill."""
    x, y = np.zeros(64, np.float32), np.zeros(64, np.float32)
    lib().rrb_aa_fill_jitter(_ptr(x, C.c_float), _ptr(y, C.c_float))
    return x, y


class MLP:
    """The cost model's network on the device (rrb_mlp_*): 24 -> 64 -> 64 -> 1."""

    N_PARAMS = _abi.RRB_MLP_PARAMS
    N_IN = _abi.RRB_MLP_IN

    def __init__(self, device: int = 0, seed: int = 0):
        h = C.c_void_p()
        rc = lib().rrb_mlp_create(device, seed, C.byref(h))
        if rc:
            raise BackendError(rc, "rrb_mlp_create failed")
        self._h = h.value

    def close(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            lib().rrb_mlp_destroy(h)

    def __del__(self):
        self.close()

    @staticmethod
    def _f32(a, shape=None):
        a = np.ascontiguousarray(a, np.float32)
        if shape is not None:
            a = a.reshape(shape)
        return a

    def params(self) -> np.ndarray:
        out = np.empty(self.N_PARAMS, np.float32)
        rc = lib().rrb_mlp_get_params(self._h, _ptr(out, C.c_float))
        if rc:
            raise BackendError(rc, "get_params")
        return out

    def set_params(self, w):
        w = self._f32(w)
        assert w.size == self.N_PARAMS
        rc = lib().rrb_mlp_set_params(self._h, _ptr(w, C.c_float))
        if rc:
            raise BackendError(rc, "set_params")

    def loss_grad(self, X, y):
        X, y = self._f32(X, (-1, self.N_IN)), self._f32(y)
        g = np.empty(self.N_PARAMS, np.float32)
        loss = C.c_float()
        rc = lib().rrb_mlp_loss_grad(self._h, _ptr(X, C.c_float), _ptr(y, C.c_float), len(y), _ptr(g, C.c_float),
                                     C.byref(loss))
        if rc:
            raise BackendError(rc, "loss_grad")
        return float(loss.value), g

    def train(self, X, y, epochs=30, batch=4096, lr=1e-3, seed=0) -> float:
        X, y = self._f32(X, (-1, self.N_IN)), self._f32(y)
        loss = C.c_float()
        rc = lib().rrb_mlp_train(self._h, _ptr(X, C.c_float), _ptr(y, C.c_float), len(y), epochs, batch, lr, seed,
                                 C.byref(loss))
        if rc:
            raise BackendError(rc, "train")
        return float(loss.value)

    @staticmethod
    def predict_host(params, X) -> np.ndarray:
        """rrb_mlp_predict_host: the same forward pass on the host (same bits)."""
        params = np.ascontiguousarray(params, np.float32)
        X = np.ascontiguousarray(X, np.float32).reshape(-1, MLP.N_IN)
        out = np.empty(len(X), np.float32)
        rc = lib().rrb_mlp_predict_host(_ptr(params, C.c_float), _ptr(X, C.c_float), len(X), _ptr(out, C.c_float))
        if rc:
            raise BackendError(rc, "predict_host")
        return out

    def predict(self, X) -> np.ndarray:
        X = self._f32(X, (-1, self.N_IN))
        out = np.empty(len(X), np.float32)
        rc = lib().rrb_mlp_predict(self._h, _ptr(X, C.c_float), len(X), _ptr(out, C.c_float))
        if rc:
            raise BackendError(rc, "predict")
        return out
