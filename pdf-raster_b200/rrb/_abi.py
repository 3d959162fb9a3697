"""ctypes declarations of the C ABI in include/rrb.h.

Struct layouts here must match the header field for field; tests check the
sizes against offsets computed by the C compiler through rrb_abi_sizes-free
means (ctypes alignment rules equal the C ABI rules on x86-64).
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "librrb.so"

# status codes (include/rrb.h)
RRB_OK = 0
RRB_ERR_ZERO_SIZE_ALLOC = 1
RRB_ERR_UNALIGNED_FILL = 2
RRB_ERR_POOL_EXHAUSTED = 3
RRB_ERR_INVARIANT = 4
RRB_ERR_OTHER = 5
RRB_ERR_TIMEOUT = 6
RRB_ERR_DEVICE = 7
RRB_ERR_OUT_OF_MEMORY = 8
RRB_ERR_STATE = 9

RRB_FILL_NONZERO = 0
RRB_FILL_EVEN_ODD = 1
RRB_ROWMAP_DOCUMENTED = 0
RRB_ROWMAP_AS_SHIPPED = 1
RRB_STATIC_SCRATCH_BYTES = 32 << 20
RRB_STATIC_MAX_POINTS = 1 << 16
RRB_STATIC_MAX_EDGES = 1 << 18
RRB_STATIC_MAX_ROW_CROSSINGS = 128
RRB_STATIC_MAX_CELLS = 2801024
RRB_MLP_IN = 24
RRB_SCHED_SHORTEST_FIRST = 1
RRB_SCHED_TILE_BY_MODEL = 2
RRB_MLP_HIDDEN = 64
RRB_MLP_PARAMS = 64 * 24 + 64 + 64 * 64 + 64 + 64 + 1


class VramBudget(C.Structure):
    _fields_ = [("total_bytes", C.c_uint64), ("free_bytes", C.c_uint64),
                ("budget_bytes", C.c_uint64), ("used_bytes", C.c_uint64)]


class PathFillParams(C.Structure):
    _fields_ = [
        ("pts", C.POINTER(C.c_double)),
        ("flags", C.POINTER(C.c_uint8)),
        ("n_pts", C.c_uint32),
        ("matrix", C.c_double * 6),
        ("flatness", C.c_double),
        ("fill_rule", C.c_uint8),
        ("gray", C.c_uint8),
        ("alpha", C.c_uint8),
        ("rowmap", C.c_uint8),
        ("page", C.c_void_p),
        ("page_offset", C.c_uint64),
        ("width", C.c_uint32),
        ("height", C.c_uint32),
    ]


class AaFillParams(C.Structure):
    _fields_ = [("segs", C.c_void_p), ("n_segs", C.c_uint32), ("coverage", C.c_void_p), ("width", C.c_uint32),
                ("height", C.c_uint32), ("fill_rule", C.c_uint8)]


class TileRecord(C.Structure):
    _fields_ = [("key", C.c_uint32), ("x_enter", C.c_float), ("dxdy", C.c_float), ("y0_tile", C.c_float),
                ("y1_tile", C.c_float), ("sign", C.c_float), ("pad", C.c_uint32), ("pad2", C.c_uint32)]


class TileFillParams(C.Structure):
    _fields_ = [("records", C.c_void_p), ("tile_starts", C.c_void_p), ("tile_counts", C.c_void_p), ("coverage", C.c_void_p),
                ("width", C.c_uint32), ("height", C.c_uint32), ("fill_rule", C.c_uint8)]


class ScanParams(C.Structure):
    _fields_ = [("data", C.c_void_p), ("block_sums", C.c_void_p), ("len_elems", C.c_uint32), ("phase", C.c_uint32)]


class PathBatchParams(C.Structure):
    _fields_ = [
        ("pts", C.POINTER(C.c_double)),
        ("flags", C.POINTER(C.c_uint8)),
        ("n_pts", C.c_uint64),
        ("path_pt_off", C.POINTER(C.c_uint64)),
        ("fill_rule", C.POINTER(C.c_uint8)),
        ("gray", C.POINTER(C.c_uint8)),
        ("alpha", C.POINTER(C.c_uint8)),
        ("path_page", C.POINTER(C.c_uint32)),
        ("n_paths", C.c_uint64),
        ("page_width", C.POINTER(C.c_uint32)),
        ("page_height", C.POINTER(C.c_uint32)),
        ("page_offset", C.POINTER(C.c_uint64)),
        ("n_pages", C.c_uint32),
        ("pages", C.c_void_p),
        ("matrix", C.c_double * 6),
        ("flatness", C.c_double),
        ("rowmap", C.c_uint8),
    ]


class Tuning(C.Structure):
    _fields_ = [("tile_w", C.c_uint32), ("tile_h", C.c_uint32), ("rows_per_chunk", C.c_uint32),
                ("wave_points", C.c_uint32), ("auto_tile", C.c_uint32), ("reserved", C.c_uint32 * 3)]


class BatchStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in (
        "paths", "pieces", "segments", "aa_rows", "spans", "row_overflows", "tiles", "tile_pairs",
        "nonterminating_rows", "kernel_launches", "scratch_grows", "waves", "host_ns", "row_groups", "host_syncs",
        "tile_w", "tile_h", "row_shape", "trials_left")]


class StageTime(C.Structure):
    _fields_ = [("name", C.c_char * 24), ("ms", C.c_float), ("launches", C.c_uint32)]


class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int), ("workers", C.c_uint32), ("mem_budget_bytes", C.c_uint64),
                ("max_batch_pages", C.c_uint32), ("tile_w", C.c_uint32), ("tile_h", C.c_uint32),
                ("predict_threads", C.c_uint32),
                ("reserved", C.c_uint32 * 2)]


class RequestResult(C.Structure):
    _fields_ = [("status", C.c_int), ("latency_ns", C.c_uint64), ("queue_ns", C.c_uint64)]


class ServerStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("completed", "batches", "batched_requests", "queued", "in_use_bytes",
                                          "peak_in_use_bytes")] + [("tile_batches", C.c_uint64 * 3)] + [
        (n, C.c_uint64) for n in ("prep_ns", "render_ns", "download_ns")]


class ServerCostModel(C.Structure):
    _fields_ = [("params", C.POINTER(C.c_float)), ("x_mean", C.POINTER(C.c_float)), ("x_std", C.POINTER(C.c_float)),
                ("y_mean", C.c_float), ("y_std", C.c_float), ("table", C.POINTER(C.c_int32)), ("policy", C.c_uint32)]


RRB_CAP_BUTT, RRB_CAP_ROUND, RRB_CAP_PROJECTING = 0, 1, 2
RRB_JOIN_MITER, RRB_JOIN_ROUND, RRB_JOIN_BEVEL = 0, 1, 2


class StrokeParams(C.Structure):
    _fields_ = [("line_width", C.c_double), ("miter_limit", C.c_double), ("dash_phase", C.c_double),
                ("dash", C.POINTER(C.c_double)), ("n_dash", C.c_uint32), ("line_cap", C.c_uint8),
                ("line_join", C.c_uint8), ("stroke", C.c_uint8), ("reserved", C.c_uint8)]


class ClipPath(C.Structure):
    pass


ClipPath._fields_ = [("pts", C.POINTER(C.c_double)), ("flags", C.POINTER(C.c_uint8)), ("n_pts", C.c_uint64),
                     ("even_odd", C.c_uint8), ("reserved", C.c_uint8 * 7), ("next", C.POINTER(ClipPath))]


# Every exported symbol of include/rrb.h with its signature: (restype, argtypes).
VP = C.c_void_p
SIGNATURES = {
    "rrb_init": (C.c_int, [C.c_int, C.c_uint64, C.POINTER(VP)]),
    "rrb_destroy": (C.c_int, [VP]),
    "rrb_last_error_message": (C.c_char_p, [VP]),
    "rrb_status_name": (C.c_char_p, [C.c_int]),
    "rrb_version": (C.c_char_p, []),
    "rrb_alloc_device": (C.c_int, [VP, C.c_size_t, C.POINTER(VP)]),
    "rrb_alloc_device_zeroed": (C.c_int, [VP, C.c_size_t, C.POINTER(VP)]),
    "rrb_device_buffer_len": (C.c_size_t, [VP]),
    "rrb_device_ptr": (VP, [VP]),
    "rrb_free_device": (C.c_int, [VP, VP]),
    "rrb_alloc_host_pinned": (C.c_int, [VP, C.c_size_t, C.POINTER(VP)]),
    "rrb_host_ptr": (VP, [VP]),
    "rrb_free_host_pinned": (C.c_int, [VP, VP]),
    "rrb_upload_async": (C.c_int, [VP, VP, C.c_size_t, VP, C.c_size_t, C.POINTER(C.c_uint64)]),
    "rrb_download_async": (C.c_int, [VP, VP, C.c_size_t, VP, C.c_size_t, C.POINTER(C.c_uint64)]),
    "rrb_wait_download": (C.c_int, [VP, C.c_uint64]),
    "rrb_submit_transfer": (C.c_int, [VP, C.POINTER(C.c_uint64)]),
    "rrb_wait_transfer": (C.c_int, [VP, C.c_uint64, C.c_uint64]),
    "rrb_detect_vram_budget": (C.c_int, [VP, C.POINTER(VramBudget)]),
    "rrb_begin_page": (C.c_int, [VP]),
    "rrb_record_zero_buffer": (C.c_int, [VP, VP]),
    "rrb_submit_page": (C.c_int, [VP, C.POINTER(C.c_uint64)]),
    "rrb_wait_page": (C.c_int, [VP, C.c_uint64, C.c_uint64]),
    "rrb_record_path_fill": (C.c_int, [VP, C.POINTER(PathFillParams)]),
    "rrb_record_path_fill_static": (C.c_int, [VP, C.POINTER(PathFillParams)]),
    "rrb_lower_clip_paths": (C.c_int, [C.POINTER(PathBatchParams), C.POINTER(C.c_double), C.POINTER(ClipPath),
                                       C.POINTER(C.c_double), C.POINTER(C.c_uint8), C.c_uint64,
                                       C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint8),
                                       C.POINTER(C.c_double), C.POINTER(C.c_int32), C.c_uint64, C.POINTER(C.c_uint64),
                                       C.POINTER(C.c_uint64)]),
    "rrb_record_path_batch_ex": (C.c_int, [VP, C.POINTER(PathBatchParams), C.POINTER(C.c_uint8),
                                           C.POINTER(C.c_double)]),
    "rrb_record_path_batch_visit": (C.c_int, [VP, C.POINTER(PathBatchParams), C.POINTER(C.c_uint8),
                                              C.POINTER(C.c_double), C.POINTER(C.c_int32)]),
    "rrb_record_path_batch_rgb": (C.c_int, [VP, C.POINTER(PathBatchParams), C.POINTER(C.c_uint8)]),
    "rrb_record_stroke_batch": (C.c_int, [VP, C.POINTER(PathBatchParams), C.POINTER(StrokeParams),
                                          C.POINTER(C.c_uint8), C.POINTER(C.c_double)]),
    "rrb_stroke_outline": (C.c_int, [C.POINTER(C.c_double), C.POINTER(C.c_uint8), C.c_uint64,
                                     C.POINTER(StrokeParams), C.c_double, C.POINTER(C.c_double),
                                     C.POINTER(C.c_uint8), C.c_uint64, C.POINTER(C.c_uint64),
                                     C.POINTER(C.c_int)]),
    "rrb_record_rgb_to_gray": (C.c_int, [VP, VP, C.c_size_t, VP, C.c_size_t, C.c_uint64]),
    "rrb_record_aa_fill": (C.c_int, [VP, C.POINTER(AaFillParams)]),
    "rrb_aa_fill_jitter": (None, [C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "rrb_record_tile_fill": (C.c_int, [VP, C.POINTER(TileFillParams)]),
    "rrb_record_tile_fill_segs": (C.c_int, [VP, C.POINTER(AaFillParams), C.POINTER(C.c_uint64)]),
    "rrb_record_scan": (C.c_int, [VP, C.POINTER(ScanParams)]),
    "rrb_record_path_batch": (C.c_int, [VP, C.POINTER(PathBatchParams)]),
    "rrb_set_tuning": (C.c_int, [VP, C.POINTER(Tuning)]),
    "rrb_get_tuning": (C.c_int, [VP, C.POINTER(Tuning)]),
    "rrb_last_batch_stats": (C.c_int, [VP, C.POINTER(BatchStats)]),
    "rrb_batch_upload": (C.c_int, [VP, C.POINTER(PathBatchParams), C.POINTER(VP)]),
    "rrb_record_batch": (C.c_int, [VP, VP, VP, C.c_int]),
    "rrb_batch_free": (C.c_int, [VP, VP]),
    "rrb_record_fill_buffer": (C.c_int, [VP, VP, C.c_size_t, C.c_size_t, C.c_uint8]),
    "rrb_set_profiling": (C.c_int, [VP, C.c_int]),
    "rrb_stream": (VP, [VP]),
    "rrb_last_stage_times": (C.c_int, [VP, C.POINTER(StageTime), C.c_int, C.POINTER(C.c_int)]),
    "rrb_validate_path_batch": (C.c_int, [C.POINTER(PathBatchParams), C.c_size_t, C.c_char_p, C.c_size_t]),
    "rrb_render_pages_host": (C.c_int, [VP, C.POINTER(PathBatchParams), VP, C.c_size_t]),
    "rrb_render_pages_host_init": (C.c_int, [VP, C.POINTER(PathBatchParams), VP, C.c_size_t, C.c_int]),
    "rrb_server_create": (C.c_int, [C.POINTER(ServerConfig), C.POINTER(VP)]),
    "rrb_server_submit": (C.c_int, [VP, C.POINTER(PathBatchParams), VP, C.c_size_t, C.c_uint8,
                                    C.POINTER(C.c_uint64)]),
    "rrb_server_wait": (C.c_int, [VP, C.c_uint64, C.c_uint64, C.POINTER(RequestResult)]),
    "rrb_server_stats": (C.c_int, [VP, C.POINTER(ServerStats)]),
    "rrb_server_set_cost_model": (C.c_int, [VP, C.POINTER(ServerCostModel)]),
    "rrb_server_destroy": (C.c_int, [VP]),
    "rrb_encode_netpbm": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p, C.c_size_t,
                                    C.POINTER(C.c_size_t)]),
    "rrb_page_features_all": (C.c_int, [C.POINTER(PathBatchParams), C.c_uint32, C.POINTER(C.c_float)]),
    "rrb_page_features": (C.c_int, [C.POINTER(PathBatchParams), C.c_uint32, C.c_uint32, C.c_uint32,
                                    C.POINTER(C.c_float)]),
    "rrb_mlp_create": (C.c_int, [C.c_int, C.c_uint64, C.POINTER(VP)]),
    "rrb_mlp_destroy": (C.c_int, [VP]),
    "rrb_mlp_set_params": (C.c_int, [VP, C.POINTER(C.c_float)]),
    "rrb_mlp_get_params": (C.c_int, [VP, C.POINTER(C.c_float)]),
    "rrb_mlp_loss_grad": (C.c_int, [VP, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_uint32,
                                    C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "rrb_mlp_train": (C.c_int, [VP, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_uint32, C.c_uint32, C.c_uint32,
                                C.c_float, C.c_uint64, C.POINTER(C.c_float)]),
    "rrb_mlp_predict_host": (C.c_int, [C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_uint32,
                                       C.POINTER(C.c_float)]),
    "rrb_mlp_predict": (C.c_int, [VP, C.POINTER(C.c_float), C.c_uint32, C.POINTER(C.c_float)]),
    "rrb_path_new": (VP, []),
    "rrb_path_free": (None, [VP]),
    "rrb_path_clear": (None, [VP]),
    "rrb_path_move_to": (C.c_int, [VP, C.c_double, C.c_double]),
    "rrb_path_line_to": (C.c_int, [VP, C.c_double, C.c_double]),
    "rrb_path_curve_to": (C.c_int, [VP] + [C.c_double] * 6),
    "rrb_path_conic_to": (C.c_int, [VP] + [C.c_double] * 4),
    "rrb_path_close": (C.c_int, [VP, C.c_int]),
    "rrb_path_len": (C.c_uint64, [VP]),
    "rrb_path_pts": (C.POINTER(C.c_double), [VP]),
    "rrb_path_flags": (C.POINTER(C.c_uint8), [VP]),
    "rrb_conic_to_cubic": (None, [C.c_double] * 6 + [C.POINTER(C.c_double)]),
}

_LIB = None


def load() -> C.CDLL:
    """Load librrb.so (raising if it was not built) and declare every signature."""
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python pdf-raster_b200/rrb/build.py` "
                "(the AA fill has no CPU fallback)")
        lib = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB
