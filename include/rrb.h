/*
 * rrb.h — C ABI of the B200 anti-aliased fill backend ("rrb").
 *
 * This is the drop-in boundary beside the reference's CUDA / Vulkan / CPU
 * backends: every entry point mirrors one method of the reference trait
 * `GpuBackend` (crates/gpu/src/backend/mod.rs:216-503) or one of its
 * parameter structs (crates/gpu/src/backend/params.rs), with plain pointers,
 * sizes and an int status instead of Rust types, so a Rust
 * `impl GpuBackend for B200Backend` can bind these symbols one to one.
 *
 * Status codes mirror `BackendError` (mod.rs:35-72) plus a timeout and a
 * device error. The text of the last failure is available from
 * rrb_last_error_message(ctx).
 *
 * Pixels written by rrb_record_path_fill / rrb_record_path_batch are bit-exact
 * with the reference CPU scanline rasterizer (crates/raster fill_impl with
 * vector_antialias = true, Gray8 page, div255 source-over).
 */
#ifndef RRB_H
#define RRB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (BackendError, crates/gpu/src/backend/mod.rs:35-72) ---- */
#define RRB_OK 0
#define RRB_ERR_ZERO_SIZE_ALLOC 1     /* BackendError::ZeroSizeAlloc */
#define RRB_ERR_UNALIGNED_FILL 2      /* BackendError::UnalignedFill */
#define RRB_ERR_POOL_EXHAUSTED 3      /* BackendError::DescriptorPoolExhausted */
#define RRB_ERR_INVARIANT 4           /* BackendError::InvariantViolation (validate()) */
#define RRB_ERR_OTHER 5               /* BackendError::Other */
#define RRB_ERR_TIMEOUT 6             /* wait_page / wait_transfer exceeded timeout_ns */
#define RRB_ERR_DEVICE 7              /* CUDA runtime / kernel error */
#define RRB_ERR_OUT_OF_MEMORY 8       /* allocation beyond the device memory budget */
#define RRB_ERR_STATE 9               /* begin/record/submit called out of order */

/* Fill rules (AaFillParams::fill_rule, params.rs:90-103). */
#define RRB_FILL_NONZERO 0
#define RRB_FILL_EVEN_ODD 1

/* Row map of the AA driver loop (crates/raster/src/fill/mod.rs:176-203). */
#define RRB_ROWMAP_DOCUMENTED 0 /* pixel row y <- AA rows 4y..4y+3 (module docs, Splash) */
#define RRB_ROWMAP_AS_SHIPPED 1 /* the literal loop: pixel row y <- AA rows 16y+12..16y+15 */

/* PathFlags (crates/raster/src/path/mod.rs:70-79). */
#define RRB_PATH_FIRST 0x01u
#define RRB_PATH_LAST 0x02u
#define RRB_PATH_CLOSED 0x04u
#define RRB_PATH_CURVE 0x08u

typedef struct rrb_ctx rrb_ctx;       /* one backend = one device + one stream */
typedef struct rrb_buf rrb_buf;       /* opaque device buffer (GpuBackend::DeviceBuffer) */
typedef struct rrb_host_buf rrb_host_buf; /* opaque pinned host buffer (GpuBackend::HostBuffer) */
typedef uint64_t rrb_fence;           /* GpuBackend::PageFence; 0 is never a valid fence */

/* VramBudget (crates/gpu/src/backend/mod.rs, detect_vram_budget). */
typedef struct {
    uint64_t total_bytes;
    uint64_t free_bytes;
    uint64_t budget_bytes; /* the limit passed to rrb_init (0 = whole device) */
    uint64_t used_bytes;   /* bytes this backend holds now */
} rrb_vram_budget;

/* ---- lifetime ----------------------------------------------------------- */
/* CudaBackend::new equivalent: bind `device`, create the stream, cap this
 * backend's device allocations at mem_budget_bytes (0 = no cap). */
int rrb_init(int device, uint64_t mem_budget_bytes, rrb_ctx** out);
int rrb_destroy(rrb_ctx* ctx);
const char* rrb_last_error_message(const rrb_ctx* ctx);
const char* rrb_status_name(int status);
/* Library build identifier (kernel arch, version). */
const char* rrb_version(void);

/* ---- memory: GpuBackend::{alloc_device, alloc_device_zeroed, device_buffer_len,
 *      free_device, alloc_host_pinned, free_host_pinned} (mod.rs:235-295) ---- */
int rrb_alloc_device(rrb_ctx* ctx, size_t size, rrb_buf** out);
int rrb_alloc_device_zeroed(rrb_ctx* ctx, size_t size, rrb_buf** out);
size_t rrb_device_buffer_len(const rrb_buf* buf);
/* Raw device address of a buffer (for interop with other CUDA code). */
void* rrb_device_ptr(const rrb_buf* buf);
int rrb_free_device(rrb_ctx* ctx, rrb_buf* buf);
int rrb_alloc_host_pinned(rrb_ctx* ctx, size_t size, rrb_host_buf** out);
void* rrb_host_ptr(const rrb_host_buf* buf);
int rrb_free_host_pinned(rrb_ctx* ctx, rrb_host_buf* buf);

/* ---- transfers: GpuBackend::{upload_async, download_async, wait_download,
 *      submit_transfer, wait_transfer} (mod.rs:405-480) ---- */
int rrb_upload_async(rrb_ctx* ctx, const rrb_buf* dst, size_t dst_offset, const void* src,
                     size_t len, rrb_fence* out_fence);
int rrb_download_async(rrb_ctx* ctx, const rrb_buf* src, size_t src_offset, void* dst, size_t len,
                       rrb_fence* out_fence);
int rrb_wait_download(rrb_ctx* ctx, rrb_fence fence);
int rrb_submit_transfer(rrb_ctx* ctx, rrb_fence* out_fence);
int rrb_wait_transfer(rrb_ctx* ctx, rrb_fence fence, uint64_t timeout_ns);
int rrb_detect_vram_budget(rrb_ctx* ctx, rrb_vram_budget* out);

/* ---- per-page state machine: begin_page -> record_* -> submit_page ->
 *      wait_page (mod.rs:195-204, 306, 400-405) ---- */
int rrb_begin_page(rrb_ctx* ctx);
/* GpuBackend::record_zero_buffer (mod.rs:378-395). */
int rrb_record_zero_buffer(rrb_ctx* ctx, const rrb_buf* buf);
int rrb_submit_page(rrb_ctx* ctx, rrb_fence* out_fence);
/* Blocks until the fence completes or timeout_ns elapses (0 = no limit). */
int rrb_wait_page(rrb_ctx* ctx, rrb_fence fence, uint64_t timeout_ns);

/* ---- the anti-aliased path fill ------------------------------------------
 * A page is a device-resident u8 Gray8 bitmap of width*height bytes, row
 * stride `width`, no alpha plane (the renderer's page: pdf_interp
 * renderer/page/mod.rs:479-480 filled with 255).
 *
 * One path (replaces raster::fill / raster::eo_fill, crates/raster/src/fill/
 * mod.rs:55-104, called from PageRenderer::fill_path, crates/pdf_interp/src/
 * renderer/page/mod.rs:1061-1138, with DEVICE_MATRIX, page clip and
 * vector_antialias = true). `pts` holds n_pts (x,y) f64 pairs and `flags`
 * n_pts PathFlags bytes, both HOST memory, exactly as Path::{pts,flags}. The
 * path is flattened in FP64 and rasterised on the device; nothing comes back
 * to the host. */
typedef struct {
    const double* pts;     /* host, [n_pts*2] */
    const uint8_t* flags;  /* host, [n_pts]   */
    uint32_t n_pts;
    double matrix[6];      /* XPath::new matrix; identity in the renderer */
    double flatness;       /* max(gs.flatness, 0.1) in the renderer */
    uint8_t fill_rule;     /* RRB_FILL_NONZERO / RRB_FILL_EVEN_ODD */
    uint8_t gray;          /* solid source gray */
    uint8_t alpha;         /* PipeState::a_input (fill_alpha * 255) */
    uint8_t rowmap;        /* RRB_ROWMAP_* */
    const rrb_buf* page;   /* device Gray8 page */
    uint64_t page_offset;  /* byte offset of the page inside `page` */
    uint32_t width, height;
} rrb_path_fill_params;
int rrb_record_path_fill(rrb_ctx* ctx, const rrb_path_fill_params* p);

/* rrb_record_path_fill_static: the same fill, with the same parameters and
 * the same pixels as rrb_record_path_fill, that allocates no device memory.
 * It has no counterpart in the reference.
 *
 * For callers that cannot allocate device memory while they draw: cudaMalloc
 * and cudaFree synchronise the whole device, which stalls every other stream
 * of a busy serving GPU, and a process whose device memory was handed out up
 * front (an external pool, an admission budget already granted) must not hit
 * an out-of-memory error in the middle of a page. Every intermediate lives
 * in one array of RRB_STATIC_SCRATCH_BYTES that the library reserves in
 * device memory when its module loads; the array is not counted in the
 * context's memory budget and the context's own buffers are not touched.
 *
 * Limits (beyond them: RRB_ERR_POOL_EXHAUSTED with the limit in
 * rrb_last_error_message, and the page untouched): at most
 * RRB_STATIC_MAX_POINTS points, flattening to at most RRB_STATIC_MAX_EDGES
 * edges, at most RRB_STATIC_MAX_ROW_CROSSINGS merged crossings on any AA
 * row, and at most RRB_STATIC_MAX_CELLS coverage cells. Larger paths go
 * through rrb_record_path_fill.
 *
 * The first call on a device does the set-up: it looks up the array's
 * device address (which loads the module holding it). Make that first call
 * before any stream capture begins. All calls in a process share the one
 * array per device; calls that overlapped on the device would race on it,
 * so each call holds a process-wide lock until its own device work has
 * finished and concurrent callers run one after another. Like
 * rrb_record_path_fill it must come between rrb_begin_page and
 * rrb_submit_page, runs on the context's stream and has finished when it
 * returns: between its stages it waits on that stream to read sizes back
 * from the device (up to four times per call). It does not update
 * rrb_last_batch_stats. As every entry point, it makes the context's device
 * current for the call and then restores the calling thread's current
 * context (a thread that had none keeps the context's device current). */
#define RRB_STATIC_SCRATCH_BYTES (32u << 20)
#define RRB_STATIC_MAX_POINTS (1u << 16)
#define RRB_STATIC_MAX_EDGES (1u << 18)
#define RRB_STATIC_MAX_ROW_CROSSINGS 128
#define RRB_STATIC_MAX_CELLS 2801024u
int rrb_record_path_fill_static(rrb_ctx* ctx, const rrb_path_fill_params* p);

/* ---- the reference's coverage operators (record_aa_fill / record_tile_fill) ----
 * Same parameter layouts as AaFillParams / TileFillParams
 * (crates/gpu/src/backend/params.rs:90-103,170-185) and the same contract:
 * device buffers in, a u8 coverage buffer of width x height written (every
 * byte), no compositing, queued on the context's stream inside
 * begin_page/submit_page. fill_rule: 0 nonzero, anything else even-odd. */
typedef struct {
    const rrb_buf* segs;      /* device f32 [n_segs][4] = {x0, y0, x1, y1}, coverage-local pixels, 16-B aligned */
    uint32_t n_segs;
    const rrb_buf* coverage;  /* device u8 [height][width] */
    uint32_t width, height;
    uint8_t fill_rule;
} rrb_aa_fill_params;
/* 64 Halton(2,3) samples per pixel, coverage = (hits * 255 + 32) >> 6;
 * bit-identical to aa_fill_cpu (crates/gpu/src/fill.rs:346-421). */
int rrb_record_aa_fill(rrb_ctx* ctx, const rrb_aa_fill_params* p);
/* The 64 sample offsets (x, y in [0,1)) the operator uses. */
void rrb_aa_fill_jitter(float* x64, float* y64);

/* TileRecord (crates/gpu/src/fill.rs:12-39; tile_fill.cu), 32 bytes. */
typedef struct {
    uint32_t key;       /* (tile_y << 16) | tile_x */
    float x_enter;      /* tile-local x at y0_tile */
    float dxdy;
    float y0_tile, y1_tile;
    float sign;         /* +1 / -1 */
    uint32_t pad, pad2;
} rrb_tile_record;
typedef struct {
    const rrb_buf* records;      /* device rrb_tile_record[], sorted by key */
    const rrb_buf* tile_starts;  /* device u32 [grid_w * grid_h], grid_w = ceil(width / 16) */
    const rrb_buf* tile_counts;  /* device u32 [grid_w * grid_h] */
    const rrb_buf* coverage;     /* device u8 [height][width] */
    uint32_t width, height;
    uint8_t fill_rule;
} rrb_tile_fill_params;
/* Analytic signed-area coverage per 16x16 tile (tile_fill.cu:60-177), every
 * operation in IEEE f32 as written. A tile whose record range runs past the
 * records buffer is filled as empty. */
int rrb_record_tile_fill(rrb_ctx* ctx, const rrb_tile_fill_params* p);
/* tile_fill from segments: the tile records are built on the device
 * (build_tile_records, crates/gpu/src/fill.rs:82-264, with a stable key
 * sort) and kept in the context's scratch. Synchronises once, to size the
 * records; *n_records (optional) receives their count. */
int rrb_record_tile_fill_segs(rrb_ctx* ctx, const rrb_aa_fill_params* p, uint64_t* n_records);

/* GpuBackend::record_scan (crates/gpu/src/backend/mod.rs:340-353; ScanParams
 * and ScanPhase, params.rs:207-372): one phase of the three-phase exclusive
 * scan of len_elems u32 in place (u32 sums wrap). Tiles of 1,024 elements
 * (SCAN_WORKGROUP_SIZE 512 threads x 2): phase 0 scans each tile and writes
 * its total to block_sums[tile]; phase 1 scans block_sums (at most 1,024
 * tiles, SCAN_MAX_BLOCKS); phase 2 adds block_sums[tile] to every element of
 * its tile. Call the three in order inside begin_page/submit_page. The same
 * invariants as ScanParams::validate: len_elems > 0, data holds len_elems
 * u32, block_sums holds ceil(len_elems / 1024) u32, and that count is at
 * most 1,024; else RRB_ERR_INVARIANT. */
#define RRB_SCAN_WORKGROUP_SIZE 512u
#define RRB_SCAN_MAX_BLOCKS 1024u
#define RRB_SCAN_PER_WORKGROUP 0u
#define RRB_SCAN_BLOCK_SUMS 1u
#define RRB_SCAN_SCATTER_BLOCK_SUMS 2u
typedef struct {
    const rrb_buf* data;        /* device u32 [len_elems], scanned in place */
    const rrb_buf* block_sums;  /* device u32 [ceil(len_elems / 1024)] */
    uint32_t len_elems;
    uint32_t phase;             /* RRB_SCAN_* */
} rrb_scan_params;
int rrb_record_scan(rrb_ctx* ctx, const rrb_scan_params* p);

/* Many paths over many pages in one submission (the batched form). All
 * arrays are HOST memory; the backend uploads them and renders every path,
 * in index order per page, into device pages. Paths on different pages are
 * independent; paths on one page composite in index order. */
typedef struct {
    const double* pts;          /* [n_pts*2] */
    const uint8_t* flags;       /* [n_pts] */
    uint64_t n_pts;
    const uint64_t* path_pt_off;/* [n_paths+1], offsets into pts/flags */
    const uint8_t* fill_rule;   /* [n_paths] */
    const uint8_t* gray;        /* [n_paths] */
    const uint8_t* alpha;       /* [n_paths] */
    const uint32_t* path_page;  /* [n_paths] page index */
    uint64_t n_paths;
    const uint32_t* page_width; /* [n_pages] */
    const uint32_t* page_height;/* [n_pages] */
    const uint64_t* page_offset;/* [n_pages] byte offset of each page in `pages` */
    uint32_t n_pages;
    const rrb_buf* pages;       /* device arena holding every page */
    double matrix[6];
    double flatness;
    uint8_t rowmap;
} rrb_path_batch_params;
int rrb_record_path_batch(rrb_ctx* ctx, const rrb_path_batch_params* p);

/* The product renderer's RGB page form (the A12 variant: the page is Rgb8 and
 * each path composites with composite_aa_rgb8_opaque, crates/raster/src/simd/
 * composite.rs:56+, a_src = (alpha * shape + 255) >> 8 and per channel
 * ((255 - a_src) * dst + a_src * src + 255) >> 8). Pages are 3 bytes per
 * pixel (row stride 3 * width, page_offset in bytes); path p is painted with
 * path_rgb[3p..3p+2] (host); the gray array is not read. Coverage, order and
 * every other rule are those of rrb_record_path_batch. */
int rrb_record_path_batch_rgb(rrb_ctx* ctx, const rrb_path_batch_params* p, const uint8_t* path_rgb);
/* The general batch: path_rgb != NULL selects Rgb8 pages as above; with
 * clip_rects != NULL path p is clipped to the device-space rectangle
 * clip_rects[4p..4p+3] = (x0, y0, x1, y1) (host doubles, any corner order):
 * the path's clip is its page intersected with the rectangle, with the integer
 * bounds floor(x_min) .. ceil(x_max) - 1 of Clip::clip_to_rect
 * (crates/raster/src/clip.rs:116-125,266-271) — the reference's treatment of a
 * rectangular W/W* clip path (detect_rect, clip.rs:130-140). */
int rrb_record_path_batch_ex(rrb_ctx* ctx, const rrb_path_batch_params* p, const uint8_t* path_rgb,
                             const double* clip_rects);
/* rrb_record_path_batch_ex with, under RRB_ROWMAP_AS_SHIPPED, the pixel rows
 * the shipped driver loop visits given per path: visit_rows[2p..2p+1] =
 * [v0, v1] (host int32; NULL: each path's own, the rows y whose AA row 4y+3
 * lies in its scanner range, fill/mod.rs:176-203). Path p then draws pixel
 * rows v0 .. v1 from its AA rows 16y+12 .. 16y+15. This is how a clip path
 * paints on its fill's rows (rrb_lower_clip_paths); the documented row map
 * ignores visit_rows. No counterpart in the reference, which clips inside
 * fill_impl. */
int rrb_record_path_batch_visit(rrb_ctx* ctx, const rrb_path_batch_params* p, const uint8_t* path_rgb,
                                const double* clip_rects, const int32_t* visit_rows);
/* ---- clip paths (W / W* on a path that is not an axis-aligned rectangle) ----
 * A fill's clip paths: points and PathBuilder flags in user space (the batch
 * matrix applies), applied in order from the first through `next` as
 * successive Clip::clip_to_path calls. An entry without points and without a
 * `next` means no clip path; an entry without points in a stack is an empty
 * path, which lets nothing through (clip.rs:142-148). */
typedef struct rrb_clip_path_s {
    const double* pts;
    const uint8_t* flags;
    uint64_t n_pts;
    uint8_t even_odd;     /* W* */
    uint8_t reserved[7];
    const struct rrb_clip_path_s* next;
} rrb_clip_path;
/* Host only; no counterpart in the reference, which clips inside fill_impl.
 * Lowers a batch whose path i is clipped to its page, clip_rects[4i..4i+3]
 * (when clip_rects != NULL) and the clip paths of clip_paths[i] (when
 * clip_paths != NULL) onto a batch for rrb_record_path_batch_ex with clip
 * rectangles. The pixels are the reference's: Clip::clip_aa_line
 * (crates/raster/src/clip.rs:246-254) lets the clip path's scanner draw its
 * own coverage into the fill's AA lines, and the renderer builds the clip's
 * XPath without aa_scale (crates/pdf_interp/src/renderer/page/mod.rs:
 * 1003-1009), so a clipped fill paints the clip path at a quarter of its
 * size, in the fill's paint and the clip's rule, on the fill's pixel rows
 * (nothing when the fill's box lies outside the clip rectangle); a clip path
 * that detect_rect (clip.rs:322-359) finds to be a rectangle clips as that
 * rectangle; of a stack, the last other clip path is drawn (each clip
 * scanner overwrites the AA lines in turn) within the intersection of the
 * rectangles. Lowered path k comes from input path out_src_path[k] (its gray,
 * alpha, page and colour), has fill rule out_rule[k] and clip rectangle
 * out_clip_rects[4k..4k+3], and visits pixel rows out_visit_rows[2k..2k+1]
 * under the as-shipped row map (see rrb_record_path_batch_visit); its points
 * are out_pts / out_flags from out_path_pt_off[k] to out_path_pt_off[k + 1].
 * Under RRB_ROWMAP_DOCUMENTED a clipped fill draws one render_aa_line per
 * pixel row of the fill, so the lowered path is clipped to the fill's rows;
 * under RRB_ROWMAP_AS_SHIPPED the loop visits the pixel rows y whose AA row
 * 4y+3 lies in the fill's scanner range and shows the clip scanner's rows
 * 16y+12 .. 16y+15, so the lowered path keeps the clip scanner's rows and
 * gets the fill's visited rows. Any output may be NULL; *n_pts_out and
 * *n_paths_out always receive the sizes, and RRB_ERR_POOL_EXHAUSTED says an
 * output was too small. Needs the identity matrix (the renderer's
 * DEVICE_MATRIX). */
int rrb_lower_clip_paths(const rrb_path_batch_params* p, const double* clip_rects, const rrb_clip_path* clip_paths,
                         double* out_pts, uint8_t* out_flags, uint64_t pts_cap, uint64_t* out_path_pt_off,
                         uint64_t* out_src_path, uint8_t* out_rule, double* out_clip_rects, int32_t* out_visit_rows,
                         uint64_t paths_cap, uint64_t* n_pts_out, uint64_t* n_paths_out);

/* ---- strokes (crates/raster/src/stroke/mod.rs:58-283, stroke/path.rs) ----
 * StrokeParams (stroke/mod.rs:29-48) of one path. The flatness is the batch's
 * (the reference's renderer passes max(gs.flatness, 0.1) for both), and
 * stroke adjustment is off as the reference's renderer always has it
 * (crates/pdf_interp/src/renderer/page/mod.rs:1217-1227). */
#define RRB_CAP_BUTT 0
#define RRB_CAP_ROUND 1
#define RRB_CAP_PROJECTING 2
#define RRB_JOIN_MITER 0
#define RRB_JOIN_ROUND 1
#define RRB_JOIN_BEVEL 2
typedef struct {
    double line_width;    /* user space; 0 draws a hairline (stroke_narrow), > 0 an outline (stroke_wide) */
    double miter_limit;
    double dash_phase;
    const double* dash;   /* host, n_dash entries >= 0; n_dash 0: solid */
    uint32_t n_dash;
    uint8_t line_cap;     /* RRB_CAP_* */
    uint8_t line_join;    /* RRB_JOIN_* */
    uint8_t stroke;       /* 0: the path is filled with its fill rule instead */
    uint8_t reserved;
} rrb_stroke_params;
/* Paint a batch in path order, path p stroked when stroke[p].stroke, else
 * filled as by rrb_record_path_batch_ex (path_rgb / clip_rects as there; for
 * Rgb8 hairlines with alpha < 255 the blend is render_span's general arm,
 * c = div255((255 - a) * dst + a * src), pipe/general.rs:261-312). stroke()
 * per path: flatten_path, make_dashed_path when a dash array is set, then
 * make_stroke_path's outline filled nonzero with AA (line_width > 0) or
 * stroke_narrow's one-pixel spans (line_width 0). Outlines are built on the
 * host (their round joins call libm atan2 / cos / sin and every segment libm
 * hypot, whose last bits set the pixels), all filling and compositing on the
 * device. Replaces the per-path raster::stroke call of PageRenderer::stroke_path
 * (crates/pdf_interp/src/renderer/page/mod.rs:1201-1246). */
int rrb_record_stroke_batch(rrb_ctx* ctx, const rrb_path_batch_params* p, const rrb_stroke_params* stroke,
                            const uint8_t* path_rgb, const double* clip_rects);
/* What rrb_record_stroke_batch draws for one path, on the host: *kind 0
 * nothing, 1 the outline (filled nonzero), 2 the polyline of a hairline.
 * Writes at most cap points to out_pts[2*cap] / out_flags[cap] (either may be
 * NULL to ask for the size) and the full count to *out_n. */
int rrb_stroke_outline(const double* pts, const uint8_t* flags, uint64_t n_pts, const rrb_stroke_params* stroke,
                       double flatness, double* out_pts, uint8_t* out_flags, uint64_t cap, uint64_t* out_n,
                       int* kind);

/* rgb_to_gray (crates/pdf_raster/src/render.rs:1306-1324) on the device:
 * gray[i] = (2126 r + 7152 g + 722 b + 5000) / 10000 for n_px pixels. */
int rrb_record_rgb_to_gray(rrb_ctx* ctx, const rrb_buf* rgb, size_t rgb_offset, const rrb_buf* gray,
                           size_t gray_offset, uint64_t n_px);

/* Device-resident batches: the inputs of a path batch are validated and
 * uploaded once, then rendered any number of times into device pages with no
 * further host-to-device traffic (the serving loop keeps them resident).
 * rrb_record_path_batch is rrb_batch_upload + rrb_record_batch on a
 * context-owned batch. */
typedef struct rrb_batch rrb_batch;
int rrb_batch_upload(rrb_ctx* ctx, const rrb_path_batch_params* p, rrb_batch** out);
int rrb_record_batch(rrb_ctx* ctx, rrb_batch* batch, const rrb_buf* pages, int rowmap);
int rrb_batch_free(rrb_ctx* ctx, rrb_batch* batch);

/* Fill `len` bytes of `buf` at `off` with `value` inside the current page
 * (record_zero_buffer generalised: pages start white, 255). */
int rrb_record_fill_buffer(rrb_ctx* ctx, const rrb_buf* buf, size_t off, size_t len, uint8_t value);

/* Per-stage device time of the last batch, measured with CUDA events on the
 * backend's stream while profiling is enabled. */
typedef struct {
    char name[24];
    float ms;
    uint32_t launches;
} rrb_stage_time;
int rrb_set_profiling(rrb_ctx* ctx, int enable);
/* The cudaStream_t every call of this context is ordered on (for callers
 * that time or order their own work against the backend). */
void* rrb_stream(rrb_ctx* ctx);
int rrb_last_stage_times(rrb_ctx* ctx, rrb_stage_time* out, int cap, int* n);

/* Host-side validation of a batch without a device (the params validate()
 * step, crates/gpu/src/backend/params.rs:57,334; FakeBackend pattern,
 * params.rs:978-1075). pages_len is the byte size of the page arena. The
 * first violated invariant is written to msg. */
int rrb_validate_path_batch(const rrb_path_batch_params* p, size_t pages_len, char* msg, size_t msg_len);

/* Per-batch tuning knobs (tile shape etc.); 0 fields keep the current
 * values. Tile shapes accepted: 16x16, 32x32, 64x16, 128x16, 128x32.
 * auto_tile: 1 = a device-resident batch (rrb_record_batch) chooses its tile
 * shape by trial: its first renders run 64x16, 128x16 and 128x32 with row-stage
 * shape 0, then the other row-stage shapes with the fastest of those tiles, and
 * it keeps the fastest pair (by CUDA events; renders that grew scratch are
 * repeated). 2 = every batch uses tile_w x tile_h (resident batches still try
 * every row-stage shape). With 1, batches that are not
 * resident use the tile shape the context's last resident batch settled on
 * (64x16 before any, and again after each rrb_set_tuning). The default is 1.
 * Giving a tile shape without auto_tile sets 2. */
typedef struct {
    uint32_t tile_w, tile_h;
    uint32_t rows_per_chunk;    /* AA rows per row-kernel work item: 32 */
    uint32_t wave_points;       /* path points per wave of pages (0 = default, 40 Mi) */
    uint32_t auto_tile;         /* 0 = keep, 1 = on, 2 = off */
    uint32_t reserved[3];
} rrb_tuning;
int rrb_set_tuning(rrb_ctx* ctx, const rrb_tuning* t);
int rrb_get_tuning(rrb_ctx* ctx, rrb_tuning* t);

/* Counters of the last recorded batch (filled after the page fence). */
typedef struct {
    uint64_t paths, pieces, segments;       /* input paths, walk pieces, flattened segments */
    uint64_t aa_rows, spans, row_overflows; /* AA rows built, spans emitted, rows on the slow path */
    uint64_t tiles, tile_pairs;             /* tiles with work, (tile, path) pairs */
    uint64_t nonterminating_rows;           /* rows whose winding never returns to 0 */
    uint64_t kernel_launches;               /* kernels launched by the last record call */
    uint64_t scratch_grows;                 /* scratch buffers the call had to (re)allocate */
    uint64_t waves;                         /* page groups the batch was rendered in */
    uint64_t host_ns;                       /* host time of the call before its first kernel: validation,
                                               stroke outlines, staging and enqueued uploads */
    uint64_t row_groups;                    /* pixel-row index entries written by the row stage */
    uint64_t host_syncs;                    /* times the call waited on its stream for a device-side size */
    uint64_t tile_w, tile_h;                /* tile shape of the render */
    uint64_t row_shape;                     /* row-stage shape (entries per AA row x warps x edge groups per
                                               warp): 0 = 12x8x2, 1 = 16x4x2, 2 = 12x8x1, 3 = 8x16x2,
                                               4 = 16x4x1 */
    uint64_t trials_left;                   /* resident batches: tuning trials still to run (0: settled) */
} rrb_batch_stats;
int rrb_last_batch_stats(rrb_ctx* ctx, rrb_batch_stats* out);

/* Host-side convenience for a user holding host pages: uploads the pages,
 * records the batch, downloads the pages and waits (one call, end to end). */
int rrb_render_pages_host(rrb_ctx* ctx, const rrb_path_batch_params* p, uint8_t* host_pages,
                          size_t host_pages_len);
/* The same for pages that start blank: the device fills its pages with
 * init_value (0..255) instead of uploading host_pages, then renders and
 * downloads them into host_pages (the renderer's fresh pages, e.g. white
 * 255, without a host fill or a page upload). */
int rrb_render_pages_host_init(rrb_ctx* ctx, const rrb_path_batch_params* p, uint8_t* host_pages,
                               size_t host_pages_len, int init_value);

/* ---- serving: continuous batching of page renders --------------------------
 * Worker threads, each with its own context and stream, form batches from the
 * request queue in arrival order at every batch boundary, admitting requests
 * while the estimated device bytes of all in-flight batches stay within
 * mem_budget_bytes (a single request larger than the budget still runs when
 * nothing else is in flight). Requests arriving while batches run join the
 * next batch that has room. A request's arrays must stay valid until
 * rrb_server_wait returns for it; its pages start at init_value and come
 * back into host_pages (layout of its page_offset). */
typedef struct rrb_server rrb_server;
typedef struct {
    int device;
    uint32_t workers;          /* contexts (streams) rendering concurrently; 0 = 2 */
    uint64_t mem_budget_bytes; /* admission cap on in-flight device bytes; 0 = none */
    uint32_t max_batch_pages;  /* pages per batch; 0 = 64 */
    uint32_t tile_w, tile_h;   /* 0 = default tile */
    uint32_t predict_threads;  /* host threads computing cost-model predictions; 0 = 4 */
    uint32_t reserved[2];
} rrb_server_config;
typedef struct {
    int status;
    uint64_t latency_ns; /* submit -> pages on the host */
    uint64_t queue_ns;   /* submit -> its batch started */
} rrb_request_result;
typedef struct {
    uint64_t completed, batches, batched_requests, queued, in_use_bytes, peak_in_use_bytes;
    uint64_t tile_batches[3]; /* batches rendered with 16x16, 32x32, 64x16 tiles */
    uint64_t prep_ns;         /* workers' time concatenating requests into batches */
    uint64_t render_ns;       /* ... uploading and rendering batches (until the pages are done) */
    uint64_t download_ns;     /* ... copying pages back to the requests' buffers */
} rrb_server_stats_t;
int rrb_server_create(const rrb_server_config* cfg, rrb_server** out);
int rrb_server_submit(rrb_server* s, const rrb_path_batch_params* p, uint8_t* host_pages, size_t host_pages_len,
                      uint8_t init_value, uint64_t* ticket);
int rrb_server_wait(rrb_server* s, uint64_t ticket, uint64_t timeout_ns, rrb_request_result* res);
int rrb_server_stats(rrb_server* s, rrb_server_stats_t* out);
int rrb_server_destroy(rrb_server* s);

/* The scheduler's cost model (trained by rrb.autotune): the MLP of the
 * rrb_mlp_* section predicts log device ms of each queued page for each tile
 * shape from rrb_page_features, normalised by x_mean / x_std, and
 * ms = exp(y * y_std + y_mean). With RRB_SCHED_SHORTEST_FIRST, batches admit
 * queued requests by predicted time, shortest first (arrival order
 * otherwise); with RRB_SCHED_TILE_BY_MODEL each batch renders with the tile
 * shape of least predicted total time — from the autotuner table (16
 * entries, index page-size bin * 4 + edge-density bin, value 0..2 in the
 * order 16x16, 32x32, 64x16) when params is NULL, and 64x16 when both are
 * NULL. Features and predictions (rrb_page_features_all, rrb_mlp_predict_host:
 * host work only) are computed by predict_threads host threads between submit
 * and the queue, so submitting stays cheap. Set the model before submitting
 * requests. */
#define RRB_SCHED_SHORTEST_FIRST 1u
#define RRB_SCHED_TILE_BY_MODEL 2u
typedef struct {
    const float* params;   /* RRB_MLP_PARAMS floats, or NULL */
    const float* x_mean;   /* RRB_MLP_IN floats (with params) */
    const float* x_std;
    float y_mean, y_std;
    const int32_t* table;  /* [16], or NULL */
    uint32_t policy;       /* RRB_SCHED_* bits */
} rrb_server_cost_model;
int rrb_server_set_cost_model(rrb_server* s, const rrb_server_cost_model* m);

/* ---- learned cost model -----------------------------------------------------
 * FP32 MLP RRB_MLP_IN -> 64 -> 64 -> 1 (ReLU) predicting log render time of a
 * page for a tile shape from page features, trained on the device by its own
 * forward / backward / Adam kernels (MSE loss). Parameters, in order:
 * W1[64][24], b1[64], W2[64][64], b2[64], W3[64], b3. It never touches pixels. */
#define RRB_MLP_IN 24
#define RRB_MLP_HIDDEN 64
#define RRB_MLP_PARAMS (64 * 24 + 64 + 64 * 64 + 64 + 64 + 1)
typedef struct rrb_mlp rrb_mlp;
int rrb_mlp_create(int device, uint64_t seed, rrb_mlp** out);  /* He-normal initialisation */
int rrb_mlp_destroy(rrb_mlp* m);
int rrb_mlp_set_params(rrb_mlp* m, const float* params);       /* also resets Adam state */
int rrb_mlp_get_params(rrb_mlp* m, float* params);
/* One forward/backward over n samples without updating: mean loss and its gradient. */
int rrb_mlp_loss_grad(rrb_mlp* m, const float* X, const float* y, uint32_t n, float* grad_out, float* loss_out);
/* Adam over shuffled minibatches of `batch` (0 = full batch); host arrays X[n][24], y[n]. */
int rrb_mlp_train(rrb_mlp* m, const float* X, const float* y, uint32_t n, uint32_t epochs, uint32_t batch,
                  float lr, uint64_t seed, float* final_loss);
int rrb_mlp_predict(rrb_mlp* m, const float* X, uint32_t n, float* out);
/* The forward pass on the host from a parameter vector: the same operations in
 * the same order as the device kernel, so the same bits as rrb_mlp_predict. */
int rrb_mlp_predict_host(const float* params, const float* X, uint32_t n, float* out);

/* ---- page output (crates/encode pgm.rs / ppm.rs) -----------------------------
 * Netpbm bytes of a page already on the host: channels 1 writes P5 (Gray8),
 * 3 writes P6 (Rgb8); header "P5\n{w} {h}\n255\n" then the pixel rows.
 * *out_len receives the byte count; out == NULL only queries it. */
int rrb_encode_netpbm(const uint8_t* pixels, uint32_t width, uint32_t height, uint32_t channels, uint8_t* out,
                      size_t out_cap, size_t* out_len);

/* ---- cost-model features ------------------------------------------------------
 * RRB_MLP_IN floats describing page `page` of a batch for composite tile
 * shape tile_w x tile_h (16x16, 32x32 or 64x16), computed on the host from
 * the batch's arrays in one pass (no device work):
 *   0 log1p(pixels)            1 log1p(paths)          2 log1p(points)
 *   3 line / (line + curve)    4 log1p(curves)         5 log1p(est. flattened edges)
 *   6 log1p(mean segment len)  7 log1p(sum path-box area / page area)
 *   8 log1p(mean path-box area) 9 even-odd fraction    10 alpha < 255 fraction
 *  11 rectilinear fraction     12 fraction of tiles under some path box
 *  13-20 fraction of tiles whose path-box count is 0, 1-3, 4-15, 16-63, 64-255, 256-1023,
 *        1024-4095, >= 4096
 *  21-23 tile shape one-hot (16x16, 32x32, 64x16) */
int rrb_page_features(const rrb_path_batch_params* p, uint32_t page, uint32_t tile_w, uint32_t tile_h,
                      float* out);
/* The features of all three tile shapes in one pass: out[3][RRB_MLP_IN], rows
 * 16x16, 32x32, 64x16. */
int rrb_page_features_all(const rrb_path_batch_params* p, uint32_t page, float* out);

/* ---- path construction on the host (A1, A2) --------------------------------
 * PathBuilder::{move_to, line_to, curve_to, close} (crates/raster/src/path/
 * mod.rs:310-448) and conic_to_cubic (crates/font/src/outline.rs:106-112). */
typedef struct rrb_path rrb_path;
rrb_path* rrb_path_new(void);
void rrb_path_free(rrb_path* p);
void rrb_path_clear(rrb_path* p);
int rrb_path_move_to(rrb_path* p, double x, double y);       /* 0, or 1 NoCurPt / 2 BogusPath */
int rrb_path_line_to(rrb_path* p, double x, double y);
int rrb_path_curve_to(rrb_path* p, double x1, double y1, double x2, double y2, double x3, double y3);
int rrb_path_conic_to(rrb_path* p, double xc, double yc, double x3, double y3);
int rrb_path_close(rrb_path* p, int force);
uint64_t rrb_path_len(const rrb_path* p);
const double* rrb_path_pts(const rrb_path* p);
const uint8_t* rrb_path_flags(const rrb_path* p);
void rrb_conic_to_cubic(double p0x, double p0y, double pcx, double pcy, double p3x, double p3y,
                        double out[4]);

#ifdef __cplusplus
}
#endif
#endif /* RRB_H */
