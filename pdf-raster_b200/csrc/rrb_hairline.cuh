// rrb_hairline.cuh — hairline strokes (line width 0) on the device:
// stroke_narrow (crates/raster/src/stroke/mod.rs:95-170) and
// draw_narrow_span (:204-256).
//
// A hairline path draws, segment by segment, one span of whole pixels per
// pixel row the segment crosses, each composited with render_span without a
// shape (full coverage). Spans of one segment never share a row, but spans of
// different segments do, and there the pixel is blended once per segment. So
// every segment is its own layer: a rectilinear pseudo-path whose "runs" are
// its pixel rows, each with one coverage-16 cell, composited in segment order
// by the same tile compositor as fills (k_super_bin + k_composite).
//
// Segments arrive as two-point paths of the batch with the internal fill rule
// RULE_HAIRLINE (the host walks the flattened and dashed polyline as
// XPath::new with close_subpaths = false does, xpath.rs:162-260), so they
// interleave with fills and stroke outlines in one render, in path order.
#pragma once

#include "rrb_kernels.cuh"

namespace rrb {

// The clip of stroke_narrow: Clip::new(0, 0, W, H) intersected with the
// path's rectangle (clip.rs:73-88,116-125,266-271), float and integer bounds.
struct HlClip {
    double x_min, y_min, x_max, y_max;
    int32_t x_min_i, y_min_i, x_max_i, y_max_i;
};

__host__ __device__ __forceinline__ HlClip hl_clip(uint32_t W, uint32_t H, const double* __restrict__ rect) {
    HlClip c{0.0, 0.0, static_cast<double>(W), static_cast<double>(H), 0, 0, 0, 0};
    if (rect) {
        c.x_min = fmax(c.x_min, fmin(rect[0], rect[2]));
        c.x_max = fmin(c.x_max, fmax(rect[0], rect[2]));
        c.y_min = fmax(c.y_min, fmin(rect[1], rect[3]));
        c.y_max = fmin(c.y_max, fmax(rect[1], rect[3]));
    }
    c.x_min_i = splash_floor(c.x_min);
    c.y_min_i = splash_floor(c.y_min);
    c.x_max_i = sat_i32_of_integral(ceil(c.x_max)) - 1;
    c.y_max_i = sat_i32_of_integral(ceil(c.y_max)) - 1;
    return c;
}

__host__ __device__ __forceinline__ int32_t wrap_add(int32_t a, int32_t b) {
    return static_cast<int32_t>(static_cast<uint32_t>(a) + static_cast<uint32_t>(b));
}

// One hairline segment as stroke_narrow sees it: endpoints oriented y0 <= y1,
// the rows it draws, and whether test_rect found it wholly inside the clip.
struct HlSeg {
    double sx0, sy0, dxdy;
    int32_t cy0, cx0, cy1, cx1;  // sloped: rows [cy0, cy1] with end columns; flat: row cy0, columns [cx0, cx1]
    int32_t r0, r1;              // rows that reach the page (r0 > r1: none)
    bool flat, inside, ltr;
};

__host__ __device__ __forceinline__ HlSeg hl_segment(const double* __restrict__ pts, const double* __restrict__ m,
                                                     uint64_t pt, uint32_t W, uint32_t H, const HlClip& clip) {
    HlSeg g{};
    // add_segment (xpath.rs:324-402) on the transformed endpoints.
    double ax, ay, bx, by;
    transform(m, pts[2 * pt], pts[2 * pt + 1], ax, ay);
    transform(m, pts[2 * pt + 2], pts[2 * pt + 3], bx, by);
    double x0 = ax, y0 = ay, x1 = bx, y1 = by, dxdy = 0.0;
    if (bits_of(ay) != bits_of(by)) {
        const bool vert = bits_of(ax) == bits_of(bx);
        dxdy = vert ? 0.0 : ddiv(dsub(bx, ax), dsub(by, ay));
        if (ay > by) {
            x0 = bx;
            y0 = by;
            x1 = ax;
            y1 = ay;
        }
    }
    // stroke_narrow: orient so that y0 <= y1.
    double sx0 = x0, sy0 = y0, sx1 = x1, sy1 = y1;
    if (!(y0 <= y1)) {
        sx0 = x1;
        sy0 = y1;
        sx1 = x0;
        sy1 = y0;
    }
    const int32_t iy0 = splash_floor(sy0), iy1 = splash_floor(sy1);
    const int32_t ix0 = splash_floor(sx0), ix1 = splash_floor(sx1);
    const int32_t xl = min(ix0, ix1), xr = max(ix0, ix1);
    // Clip::test_rect (clip.rs:196-215); right + 1 / bottom + 1 wrap as i32.
    const double r1 = static_cast<double>(wrap_add(xr, 1)), b1 = static_cast<double>(wrap_add(iy1, 1));
    g.r0 = 1;
    g.r1 = 0;
    if (r1 <= clip.x_min || static_cast<double>(xl) >= clip.x_max || b1 <= clip.y_min ||
        static_cast<double>(iy0) >= clip.y_max)
        return g;
    g.inside = static_cast<double>(xl) >= clip.x_min && r1 <= clip.x_max && static_cast<double>(iy0) >= clip.y_min &&
               b1 <= clip.y_max;
    g.sx0 = sx0;
    g.sy0 = sy0;
    g.dxdy = dxdy;
    if (iy0 == iy1) {
        g.flat = true;
        g.cy0 = g.cy1 = iy0;
        g.cx0 = xl;
        g.cx1 = xr;
    } else {
        g.cy0 = iy0;
        g.cx0 = ix0;
        g.cy1 = iy1;
        g.cx1 = ix1;
        if (g.cy0 < clip.y_min_i) {
            g.cy0 = clip.y_min_i;
            g.cx0 = splash_floor(dfma(dsub(clip.y_min, sy0), dxdy, sx0));
        }
        if (g.cy1 > clip.y_max_i) {
            g.cy1 = clip.y_max_i;
            g.cx1 = splash_floor(dfma(dsub(clip.y_max, sy0), dxdy, sx0));
        }
        g.ltr = g.cx0 <= g.cx1;
    }
    // draw_narrow_span draws rows inside the page, and for a clip that is not
    // wholly inside only rows where Clip::test can pass.
    int64_t lo = g.cy0 > 0 ? g.cy0 : 0, hi = g.cy1 < static_cast<int64_t>(H) - 1 ? g.cy1 : static_cast<int64_t>(H) - 1;
    if (!g.inside) {
        if (clip.y_min_i > lo) lo = clip.y_min_i;
        if (clip.y_max_i < hi) hi = clip.y_max_i;
    }
    if (lo <= hi) {
        g.r0 = static_cast<int32_t>(lo);
        g.r1 = static_cast<int32_t>(hi);
    }
    (void)W;
    return g;
}

// The clamped span of row y (cy0 <= y <= cy1) as draw_narrow_span paints it;
// x0 > x1 when nothing is painted.
__host__ __device__ __forceinline__ int2 hl_row_span(const HlSeg& g, int32_t y, uint32_t W, const HlClip& clip) {
    int32_t a, b;
    if (g.flat) {
        a = g.cx0;
        b = g.cx1;
    } else {
        // xa = the previous row's xb: (y - 1) + 1 - sy0 as the reference's loop computes it.
        const int32_t xa = y == g.cy0 ? g.cx0
                                      : splash_floor(dfma(dsub(dadd(static_cast<double>(y - 1), 1.0), g.sy0), g.dxdy, g.sx0));
        const int32_t xb = y < g.cy1 ? splash_floor(dfma(dsub(dadd(static_cast<double>(y), 1.0), g.sy0), g.dxdy, g.sx0))
                                     : (g.ltr ? wrap_add(g.cx1, 1) : wrap_add(g.cx1, -1));
        if (g.ltr) {
            a = xa;
            b = xa == xb ? xa : wrap_add(xb, -1);
        } else if (xa == xb) {
            a = b = xa;
        } else {
            a = wrap_add(xb, 1);
            b = xa;
        }
    }
    if (g.inside) return make_int2(max(a, 0), min(b, static_cast<int32_t>(W) - 1));
    return make_int2(max(a, clip.x_min_i), min(b, clip.x_max_i));
}

// Pass 1, thread per path; hairline segments only (rule RULE_HAIRLINE): the
// rows drawn (one run each) into run_count, and the layer's PathInfo. Its
// columns are a bound here (the end columns +-2, in the clip): every span lies
// between the floors of the segment's x at its rows, which differ from the
// end columns by at most one; k_hl_write narrows them to the spans.
__global__ void k_hl_count(const double* __restrict__ pts, const uint64_t* __restrict__ path_pt_off,
                           const uint8_t* __restrict__ rule, const double* __restrict__ mtx,
                           const uint32_t* __restrict__ path_page, const uint32_t* __restrict__ page_w,
                           const uint32_t* __restrict__ page_h, const double* __restrict__ clip_rect,
                           const uint8_t* __restrict__ gray, const uint8_t* __restrict__ alpha, uint32_t n_paths,
                           int rowmap, PathInfo* __restrict__ info, uint32_t* __restrict__ run_count,
                           BatchCounters* __restrict__ ctr) {
    __shared__ double m[6];
    if (threadIdx.x < 6) m[threadIdx.x] = mtx[threadIdx.x];
    __syncthreads();
    unsigned long long total = 0;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n_paths; p += gridDim.x * blockDim.x) {
        if (rule[p] != RULE_HAIRLINE) continue;
        const uint32_t pg = path_page[p], W = page_w[pg], H = page_h[pg];
        const HlClip clip = hl_clip(W, H, clip_rect ? clip_rect + 4 * p : nullptr);
        const HlSeg g = hl_segment(pts, m, path_pt_off[p], W, H, clip);
        PathInfo P{};
        P.px0 = 1;
        P.px1 = 0;
        P.bx0 = P.by0 = 1;
        P.bx1 = P.by1 = 0;
        P.e_begin = P.e_end = 0;
        P.page = pg;
        P.paint = static_cast<uint32_t>(gray[p]) | (static_cast<uint32_t>(alpha[p]) << 8) | PI_RECTI | PI_SOLID;
        uint32_t n = 0;
        if (g.r0 <= g.r1) {
            n = static_cast<uint32_t>(g.r1 - g.r0 + 1);
            P.py0 = g.r0;
            P.py1 = g.r1;
            // Row groups as the compositor looks them up: pixel row y is group
            // y, or 4y + 3 under the as-shipped row map.
            const int32_t g0 = rowmap ? 4 * g.r0 + 3 : g.r0, g1 = rowmap ? 4 * g.r1 + 3 : g.r1;
            P.y0 = 4 * g0;
            P.y1 = 4 * g1 + 3;
            const int32_t lo = g.inside ? 0 : clip.x_min_i, hi = g.inside ? static_cast<int32_t>(W) - 1 : clip.x_max_i;
            const int64_t a = static_cast<int64_t>(min(g.cx0, g.cx1)) - 2, b = static_cast<int64_t>(max(g.cx0, g.cx1)) + 2;
            P.px0 = static_cast<int32_t>(a > lo ? a : lo);
            P.px1 = static_cast<int32_t>(b < hi ? b : hi);
        } else {
            P.py0 = P.y0 = 1;
            P.py1 = P.y1 = 0;
        }
        info[p] = P;
        run_count[p] = n;
        total += n;
    }
    // The 64-bit total, so the host can refuse a batch whose run count would
    // overflow the 32-bit offsets before any run is written. Every lane of
    // every warp reaches this point (blocks are whole warps).
    for (int o = 16; o; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
    if ((threadIdx.x & 31) == 0 && total) atomicAdd(&ctr->hl_rows, total);
}

// Pass 2, warp per path; hairline segments only: run r of the layer =
// (group, group, its cell, 0 or 1 cells), the cell = the row's span at
// coverage 16 (cells taken from the batch's cell cursor), and the layer's
// columns narrowed to its spans.
__global__ void k_hl_write(const double* __restrict__ pts, const uint64_t* __restrict__ path_pt_off,
                           const uint8_t* __restrict__ rule, const double* __restrict__ mtx,
                           const uint32_t* __restrict__ path_page, const uint32_t* __restrict__ page_w,
                           const uint32_t* __restrict__ page_h, const double* __restrict__ clip_rect,
                           uint32_t n_paths, int rowmap, const uint32_t* __restrict__ run_off,
                           PathInfo* __restrict__ info, int4* __restrict__ runs, uint32_t* __restrict__ cells,
                           uint32_t cell_cap, BatchCounters* __restrict__ ctr) {
    __shared__ double m[6];
    if (threadIdx.x < 6) m[threadIdx.x] = mtx[threadIdx.x];
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t p = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); p < n_paths; p += warps) {
        if (rule[p] != RULE_HAIRLINE) continue;
        const uint32_t pg = path_page[p], W = page_w[pg], H = page_h[pg];
        const HlClip clip = hl_clip(W, H, clip_rect ? clip_rect + 4 * p : nullptr);
        const HlSeg g = hl_segment(pts, m, path_pt_off[p], W, H, clip);
        const uint32_t base = run_off[p];
        const uint32_t n = g.r0 <= g.r1 ? static_cast<uint32_t>(g.r1 - g.r0 + 1) : 0u;
        uint32_t c0 = 0;
        if (lane == 0 && n) c0 = atomicAdd(&ctr->cell_cursor, n);
        c0 = __shfl_sync(0xffffffffu, c0, 0);
        const bool fits = static_cast<uint64_t>(c0) + n <= cell_cap;
        if (!fits && lane == 0) atomicOr(&ctr->err, ERR_SPAN_CAP);
        int32_t lo = INT32_MAX, hi = INT32_MIN;
        for (uint32_t k = lane; k < n && fits; k += 32) {
            const int32_t y = g.r0 + static_cast<int32_t>(k);
            const int2 sp = hl_row_span(g, y, W, clip);
            const int32_t grp = rowmap ? 4 * y + 3 : y;
            const bool any = sp.x <= sp.y;
            runs[base + k] = make_int4(grp, grp, static_cast<int32_t>(c0 + k), any ? 1 : 0);
            if (any) {
                cells[c0 + k] = static_cast<uint32_t>(sp.x) | (static_cast<uint32_t>(sp.y - sp.x) << 14) | (15u << 28);
                lo = min(lo, sp.x);
                hi = max(hi, sp.y);
            }
        }
        for (int o = 16; o; o >>= 1) {
            lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        if (lane == 0) {
            info[p].px0 = lo <= hi ? lo : 1;
            info[p].px1 = lo <= hi ? hi : 0;
            info[p].run_off = base;
            info[p].run_cnt = fits ? n : 0u;
        }
    }
}

}  // namespace rrb
