/*
 * rr_oracle.h — CPU oracle for the rasterrocket anti-aliased fill path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the parity checker: a literal
 * C++ restatement of the reference CPU scanline rasterizer (crates/raster,
 * crates/color, crates/font of pthomasfournet/pdf-raster). Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline / reference legs may
 * load it. The product path (pdf-raster_b200/) never links or calls it.
 *
 * Every function cites the reference file:line it follows. The reference is
 * Rust and cannot be compiled in this environment (no cargo/rustc), so this
 * restatement is the parity definition; it is pinned against every unit-test
 * vector the reference holds for the path (tests/test_oracle_golden.py).
 *
 * Build: oracle/Makefile (g++ -O3 -ffp-contract=off; std::fma wherever the
 * reference calls f64::mul_add, plain IEEE +,-,*,/ elsewhere).
 */
#ifndef RR_ORACLE_H
#define RR_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* PathFlags (crates/raster/src/path/mod.rs:70-79). */
#define OR_PF_FIRST 0x01u
#define OR_PF_LAST 0x02u
#define OR_PF_CLOSED 0x04u
#define OR_PF_CURVE 0x08u

/* XPathFlags (crates/raster/src/xpath.rs:49-60). */
#define OR_XF_HORIZ 0x01u
#define OR_XF_VERT 0x02u
#define OR_XF_FLIPPED 0x04u

/* Row map of the AA driver loop (crates/raster/src/fill/mod.rs:176-203). */
#define OR_ROWMAP_DOCUMENTED 0 /* pixel row y <- AA rows 4y..4y+3 */
#define OR_ROWMAP_AS_SHIPPED 1 /* literal loop: pixel row y <- AA rows 16y+12..16y+15 */

/* Page compositing mode. */
#define OR_COMPOSITE_GRAY8 0 /* render_span_aa_inner None arm, exact div255 (pipe/aa.rs:192-208) */

/* XPathSeg (crates/raster/src/xpath.rs:70-107). */
typedef struct {
    double x0, y0, x1, y1, dxdy;
    int32_t dxdy_fp;
    uint32_t flags;
} or_seg;

/* Intersect (crates/raster/src/scanner/mod.rs:74-85). */
typedef struct {
    int32_t x0, x1, count;
} or_intersect;

/* Counters for the cases where the reference's own output is not pinned. */
typedef struct {
    uint64_t paths;             /* fill calls */
    uint64_t segments;          /* flattened XPath segments */
    uint64_t aa_rows;           /* scanner AA rows built */
    uint64_t intersects;        /* compacted Intersect entries */
    uint64_t unpinned_tie_rows; /* rows > 20 entries with tied x0 that ipnsort may permute */
    uint64_t nonterminating_rows; /* render_aa_line rows whose winding never returns to 0 */
} or_stats;

/* ---- path construction (A1, A2) ---------------------------------------- */
/* PathBuilder::{move_to,line_to,curve_to,close} (path/mod.rs:310-448) on a
 * caller-owned growable arrays object. */
typedef struct or_path or_path;
or_path* or_path_new(void);
void or_path_free(or_path* p);
int or_path_move_to(or_path* p, double x, double y);                 /* 0 ok, 1 NoCurPt, 2 BogusPath */
int or_path_line_to(or_path* p, double x, double y);
int or_path_curve_to(or_path* p, double x1, double y1, double x2, double y2, double x3, double y3);
int or_path_close(or_path* p, int force);
int64_t or_path_len(const or_path* p);
const double* or_path_pts(const or_path* p);   /* [len*2] */
const uint8_t* or_path_flags(const or_path* p); /* [len] */
/* conic_to_cubic (crates/font/src/outline.rs:106-112): out = {x1,y1,x2,y2}. */
void or_conic_to_cubic(double p0x, double p0y, double pcx, double pcy, double p3x, double p3y,
                       double out[4]);

/* ---- A3-A6: XPath ----------------------------------------------------- */
void or_transform(const double m[6], double x, double y, double out[2]);
/* flatten_curve (path/flatten.rs:109-215): p = {x0,y0,x1,y1,x2,y2,x3,y3};
 * writes up to cap points (x,y interleaved); returns the point count. */
int32_t or_flatten_curve(const double p[8], double flatness_sq, double* out_xy, int32_t cap);
void or_add_segment(double x0, double y0, double x1, double y1, or_seg* out);
/* XPath::new (xpath.rs:162-260). Returns the segment count; writes at most cap. */
int64_t or_xpath_new(const double* pts, const uint8_t* flags, int64_t n_pts, const double m[6],
                     double flatness, int close_subpaths, or_seg* out, int64_t cap);
void or_xpath_aa_scale(or_seg* segs, int64_t n);

/* ---- A7: XPathScanner ---------------------------------------------------
 * Build a scanner (scanner/mod.rs:131-248). Returns an opaque handle. */
typedef struct or_scanner or_scanner;
or_scanner* or_scanner_new(const or_seg* segs, int64_t n, int eo, int32_t clip_y_min,
                           int32_t clip_y_max, or_stats* st);
void or_scanner_free(or_scanner* s);
/* y_min, y_max, x_min, x_max, is_empty. */
void or_scanner_bounds(const or_scanner* s, int32_t out[5]);
/* Number of intersects of row y and a copy of them (up to cap). */
int64_t or_scanner_row(const or_scanner* s, int32_t y, or_intersect* out, int64_t cap);
int or_scanner_test(const or_scanner* s, int32_t x, int32_t y);
/* count_crossings (scanner/mod.rs:327-340) on an explicit row. */
void or_count_crossings(const or_intersect* row, int64_t n, int32_t x, int32_t out[2]);
/* add_intersection (scanner/mod.rs:654-672) applied to a row vector. */
int64_t or_add_intersection(or_intersect* row, int64_t n, int32_t x0, int32_t x1, int32_t count);

/* ---- A8: render_aa_line + AaBuf -----------------------------------------
 * aa_buf is 4 rows x ceil(aa_width/8) bytes, MSB-first (bitmap.rs:462-573).
 * Returns x0, x1 as out[0], out[1]. */
void or_render_aa_line(const or_scanner* s, uint8_t* aa_buf, int64_t aa_width, int32_t y,
                       int32_t out[2], or_stats* st);
void or_aabuf_set_span(uint8_t* aa_buf, int64_t aa_width, int64_t row, int64_t x0, int64_t x1);

/* ---- A10, A11: coverage, gamma, compositing ---------------------------- */
/* The coverage tier dispatch picks on this host (2 AVX-512 BITALG, 1 AVX2,
 * 0 scalar), and one tier run explicitly (scalar-vs-SIMD agreement). */
int or_coverage_tier(void);
void or_aa_coverage_span_tier(const uint8_t* aa_buf, int64_t row_bytes, int64_t x0, uint8_t* shape, int64_t n,
                              int tier);
void or_aa_coverage_span(const uint8_t* aa_buf, int64_t row_bytes, int64_t x0, uint8_t* shape,
                         int64_t n);
const uint8_t* or_aa_gamma(void);
uint8_t or_div255(uint32_t x);
void or_render_span_aa_gray(uint8_t* dst, const uint8_t* shape, int64_t n, uint8_t a_input,
                            uint8_t gray);
/* A12 product variant: composite_aa_rgb8_opaque (simd/composite.rs:56+) and
 * rgb_to_gray (crates/pdf_raster/src/render.rs:1306-1324). */
void or_composite_aa_rgb8_opaque(uint8_t* dst_rgb, const uint8_t src[3], uint8_t a_input,
                                 const uint8_t* shape, int64_t n);
void or_rgb_to_gray(const uint8_t* rgb, uint8_t* gray, int64_t n_px);

/* ---- A9: fill driver ------------------------------------------------------
 * fill_impl (fill/mod.rs:110-244) for one solid path on a Gray8 page with the
 * page clip Clip::new(0,0,W,H,true) and vector_antialias = true. */
void or_fill_path(uint8_t* page, int32_t width, int32_t height, const double* pts,
                  const uint8_t* flags, int64_t n_pts, const double m[6], double flatness, int eo,
                  uint8_t gray, uint8_t alpha, int rowmap, or_stats* st);
/* fill_impl under a clip made by Clip::new(0, 0, W, H), clip_to_rect(clip_rect)
 * when given, then clip_to_path of the clip path (clip.rs:141-176, its XPath
 * built as the renderer builds it: close_subpaths, no aa_scale,
 * pdf_interp/src/renderer/page/mod.rs:1003-1009) with rule clip_eo. */
void or_fill_path_clip_path(uint8_t* page, int32_t width, int32_t height, const double* pts, const uint8_t* flags,
                            int64_t n_pts, const double m[6], double flatness, int eo, uint8_t gray, uint8_t alpha,
                            int rowmap, const double* clip_rect, const double* clip_pts, const uint8_t* clip_flags,
                            int64_t clip_n, int clip_eo, or_stats* st);
/* The same under a stack of clip paths, clip_to_path applied in order
 * (clip_pts[k] / clip_flags[k] / clip_n[k] / clip_eo[k]). */
void or_fill_path_clip_paths(uint8_t* page, int32_t width, int32_t height, const double* pts, const uint8_t* flags,
                             int64_t n_pts, const double m[6], double flatness, int eo, uint8_t gray, uint8_t alpha,
                             int rowmap, const double* clip_rect, int64_t n_clips, const double* const* clip_pts,
                             const uint8_t* const* clip_flags, const int64_t* clip_n, const int* clip_eo,
                             or_stats* st);

/* The same fill onto an Rgb8 page (3 bytes per pixel, row stride 3 * width)
 * with a solid RGB source, through composite_aa_rgb8_opaque (A12). */
void or_fill_path_rgb(uint8_t* page_rgb, int32_t width, int32_t height, const double* pts, const uint8_t* flags,
                      int64_t n_pts, const double m[6], double flatness, int eo, const uint8_t rgb[3], uint8_t alpha,
                      int rowmap, or_stats* st);

/* Render a whole scene: paths [0, n_paths) in order onto their pages.
 * path_pt_off[n_paths+1] indexes pts/flags; pages live in one arena at
 * page_off[p] with page_w[p] x page_h[p]. Pages are independent and are
 * rendered on up to n_threads host threads (one page per worker, as rayon). */
void or_render_scene(uint8_t* arena, const uint64_t* page_off, const uint32_t* page_w,
                     const uint32_t* page_h, uint32_t n_pages, const double* pts,
                     const uint8_t* flags, const uint64_t* path_pt_off, const uint8_t* rule,
                     const uint8_t* gray, const uint8_t* alpha, const uint32_t* path_page,
                     uint64_t n_paths, const double m[6], double flatness, int rowmap,
                     int n_threads, or_stats* st);
/* The scene on Rgb8 pages (page_off in bytes, 3 bytes per pixel), path p
 * painted with rgb[3p..3p+2]. */
void or_render_scene_rgb(uint8_t* arena, const uint64_t* page_off, const uint32_t* page_w, const uint32_t* page_h,
                         uint32_t n_pages, const double* pts, const uint8_t* flags, const uint64_t* path_pt_off,
                         const uint8_t* rule, const uint8_t* rgb, const uint8_t* alpha, const uint32_t* path_page,
                         uint64_t n_paths, const double m[6], double flatness, int rowmap, int n_threads,
                         or_stats* st);

/* The general form: gray pages (rgb == NULL) or Rgb8 pages (rgb[3p..]); with
 * clip != NULL path p is clipped to the device-space rectangle
 * clip[4p..4p+3] = (x0, y0, x1, y1) as Clip::clip_to_rect does on the page clip
 * (clip.rs:116-125: the clip becomes page ∩ rect, integer bounds floor/ceil). */
void or_render_scene_ex(uint8_t* arena, const uint64_t* page_off, const uint32_t* page_w, const uint32_t* page_h,
                        uint32_t n_pages, const double* pts, const uint8_t* flags, const uint64_t* path_pt_off,
                        const uint8_t* rule, const uint8_t* gray, const uint8_t* rgb, const uint8_t* alpha,
                        const uint32_t* path_page, uint64_t n_paths, const double* clip, const double m[6],
                        double flatness, int rowmap, int n_threads, or_stats* st);

/* ---- F2: strokes (stroke/mod.rs:58-283, stroke/path.rs:40-745) -------- */
#define OR_CAP_BUTT 0
#define OR_CAP_ROUND 1
#define OR_CAP_PROJECTING 2
#define OR_JOIN_MITER 0
#define OR_JOIN_ROUND 1
#define OR_JOIN_BEVEL 2

/* StrokeParams (stroke/mod.rs:29-48) with stroke_adjust = false and the
 * scene's flatness; stroke == 0 makes the path an ordinary fill. */
typedef struct {
    double line_width, miter_limit, dash_phase;
    const double* dash;
    int32_t n_dash;
    int32_t line_cap, line_join;
    int32_t stroke;
} or_stroke_params;

/* flatten_path (stroke/path.rs:40-86) and make_dashed_path (:107-220) into out. */
int or_stroke_flatten(const double* pts, const uint8_t* flags, int64_t n, double flatness, or_path* out);
int or_stroke_dash(const double* pts, const uint8_t* flags, int64_t n, const double* dash, int32_t n_dash,
                   double phase, or_path* out);
/* What stroke() draws for one path: 0 nothing (no points); 1 out = make_stroke_path's
 * outline (filled nonzero); 2 out = the flattened (dashed) polyline of a
 * hairline (line_width 0, drawn by stroke_narrow). */
int or_stroke_outline(const double* pts, const uint8_t* flags, int64_t n, const or_stroke_params* sp,
                      double flatness, or_path* out);
/* or_render_scene_ex where path p is stroked when stroke && stroke[p].stroke. */
void or_render_scene_paint(uint8_t* arena, const uint64_t* page_off, const uint32_t* page_w, const uint32_t* page_h,
                           uint32_t n_pages, const double* pts, const uint8_t* flags, const uint64_t* path_pt_off,
                           const uint8_t* rule, const uint8_t* gray, const uint8_t* rgb, const uint8_t* alpha,
                           const uint32_t* path_page, uint64_t n_paths, const double* clip,
                           const or_stroke_params* stroke, const double m[6], double flatness, int rowmap,
                           int n_threads, or_stats* st);

#ifdef __cplusplus
}
#endif
#endif
