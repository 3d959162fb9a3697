// Host entry points over device functions of the fill path, for the CPU
// tests (tests/test_row_logic.py): flatten_curve, make_edge and edge_entry
// (segment set-up and per-row entries), walk_row (the winding walk of one AA
// row into spans), sweep_cells (four AA rows' spans into a pixel row's
// coverage cells), recti_row_spans (rectilinear paths), the hairline spans
// (hl_clip, hl_segment, hl_row_span) and the host XPath walk of the clip-path
// lowering (rrb_clip.cu, included here for its internal functions). All are __host__ __device__; the kernels run the same
// source on the GPU. Build with -ffp-contract=off for the host so that no
// multiply-add is fused where the device's explicit rounding keeps them apart.
#include <cstdint>
#include <cstring>

#include "../pdf-raster_b200/csrc/rrb_hairline.cuh"
#include "../pdf-raster_b200/csrc/rrb_clip.cu"

namespace {

struct RowIn {
    const int32_t *x0s, *x1s, *counts;
    __host__ __device__ void operator()(int i, int32_t& a, int32_t& b, int32_t& c) const {
        a = x0s[i];
        b = x1s[i];
        c = counts[i];
    }
};

struct SpanOut {
    int32_t *x0, *x1;
    __host__ __device__ void operator()(int k, int32_t a, int32_t b) const {
        x0[k] = a;
        x1[k] = b;
    }
};

struct Bounds {
    const int32_t *x0, *x1;
    int stride;
    __host__ __device__ int32_t operator()(int k, int i, bool end) const {
        return end ? x1[k * stride + i] : x0[k * stride + i];
    }
};

struct CellOut {
    uint32_t* cells;
    __host__ __device__ void operator()(int q, uint32_t c) const { cells[q] = c; }
};

}  // namespace

extern "C" int rl_walk_row(const int32_t* x0s, const int32_t* x1s, const int32_t* counts, int n, int eo,
                           int32_t aa_width, int32_t lo, int32_t hi, int32_t* span_x0, int32_t* span_x1,
                           uint32_t* nonterminating) {
    uint32_t nt = 0;
    const int ns = rrb::walk_row(n, eo ? 1 : ~0, aa_width, lo, hi, RowIn{x0s, x1s, counts}, SpanOut{span_x0, span_x1},
                                 nt);
    *nonterminating = nt;
    return ns;
}

// n4[k] spans of sub-row k at span_x0/x1[k * stride + i]; cells[] receives
// x0 | (len - 1) << 14 | (cov - 1) << 28 per cell, at most 4 * (n4 sum).
extern "C" int rl_sweep_cells(const int32_t* n4, const int32_t* span_x0, const int32_t* span_x1, int stride,
                              uint32_t* cells) {
    const int n[4] = {n4[0], n4[1], n4[2], n4[3]};
    return rrb::sweep_cells(n, Bounds{span_x0, span_x1, stride}, CellOut{cells});
}

// flatten_curve (the device's flattening of one cubic): writes up to cap
// points (x, y) of the subdivision and returns their count.
namespace {
struct PointsOut {
    double* out;
    int cap;
    int* n;
    __host__ __device__ void operator()(double x, double y) const {
        if (*n < cap) {
            out[2 * *n] = x;
            out[2 * *n + 1] = y;
        }
        ++*n;
    }
};
}  // namespace

extern "C" int rl_flatten_curve(const double* c, double flat_sq, double* out, int cap) {
    int n = 0;
    rrb::flatten_curve(c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7], flat_sq, PointsOut{out, cap, &n});
    return n;
}

// A curve flattened the way k_seg_count_big / k_seg_write_big split it over
// a warp: lanes 0..31 in turn (curve_lane_flatten), their leaves' endpoints
// concatenated; starts[l] receives lane l's first start point and counts[l]
// its number of leaves. Returns the total.
extern "C" int rl_flatten_curve_lanes(const double* c, double flat_sq, double* out, int cap, double* starts,
                                      int* counts) {
    int n = 0;
    const rrb::CurveNode root{c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7]};
    const bool in_range = rrb::curve_in_range(c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7]);
    for (int lane = 0; lane < 32; ++lane) {
        PointsOut emit{out, cap, &n};
        double sx, sy;
        counts[lane] = in_range ? rrb::curve_lane_flatten<true>(root, lane, flat_sq, sx, sy, emit)
                                : rrb::curve_lane_flatten<false>(root, lane, flat_sq, sx, sy, emit);
        starts[2 * lane] = sx;
        starts[2 * lane + 1] = sy;
    }
    return n;
}

// make_edge of each segment (x0, y0, x1, y1 in device space, as the walk
// produces them) clipped to AA rows [clip_lo, clip_hi]: 8 int32 per edge.
extern "C" void rl_make_edges(const double* segs, int n, int32_t clip_lo, int32_t clip_hi, int32_t* out) {
    for (int i = 0; i < n; ++i) {
        const rrb::Edge e = rrb::make_edge(segs[4 * i], segs[4 * i + 1], segs[4 * i + 2], segs[4 * i + 3], clip_lo,
                                           clip_hi);
        std::memcpy(out + 8 * i, &e, sizeof e);
    }
}

// edge_entry of every edge that covers AA row r, in edge order: (edge index,
// lo, hi, count) per entry; returns the entry count.
extern "C" int rl_row_entries(const int32_t* edges, int n, int32_t r, int32_t* out) {
    int k = 0;
    for (int i = 0; i < n; ++i) {
        rrb::Edge e;
        std::memcpy(&e, edges + 8 * i, sizeof e);
        if ((e.flags & rrb::EF_EMPTY) || r < e.row0 || r > e.row1) continue;
        int32_t lo, hi, c;
        rrb::edge_entry(e, r, lo, hi, c);
        out[4 * k] = i;
        out[4 * k + 1] = lo;
        out[4 * k + 2] = hi;
        out[4 * k + 3] = c;
        ++k;
    }
    return k;
}

// The pixel spans one hairline segment (x0, y0) -> (x1, y1) paints on a W x H
// page, clipped to rect (x_min, y_min, x_max, y_max; null: the page): (row,
// first, last) per painted row; returns the count.
extern "C" int rl_hairline_spans(const double* seg, uint32_t W, uint32_t H, const double* rect, int32_t* out) {
    const double m[6] = {1.0, 0.0, 0.0, 1.0, 0.0, 0.0};
    const rrb::HlClip clip = rrb::hl_clip(W, H, rect);
    const rrb::HlSeg g = rrb::hl_segment(seg, m, 0, W, H, clip);
    int k = 0;
    for (int32_t y = g.r0; y <= g.r1; ++y) {
        const int2 sp = rrb::hl_row_span(g, y, W, clip);
        if (sp.x > sp.y) continue;
        out[3 * k] = y;
        out[3 * k + 1] = sp.x;
        out[3 * k + 2] = sp.y;
        ++k;
    }
    return k;
}

// recti_row_spans (the row stage of rectilinear paths) over n edges of one
// path with fill rule eo: AA row r's spans clipped to [lo, hi); returns the count.
extern "C" int rl_recti_spans(const int32_t* edges, int n, int eo, int32_t r, int32_t aa_width, int32_t lo,
                              int32_t hi, int32_t* span_x0, int32_t* span_x1, uint32_t* nonterminating) {
    rrb::PathInfo P{};
    P.e_begin = 0;
    P.e_end = static_cast<uint32_t>(n);
    P.paint = eo ? (1u << 16) : 0u;
    uint32_t nt = 0;
    const int ns = rrb::recti_row_spans(P, reinterpret_cast<const rrb::Edge*>(edges), r, aa_width, lo, hi, span_x0,
                                        span_x1, nt);
    *nonterminating = nt;
    return ns;
}

// The box test of rectilinear paths (recti_events + recti_box, PI_BOX) over n
// edges whose AA rows span [y0, y1]: 1, the span [out[0], out[1]) of AA
// columns and the painted AA rows [out[2], out[3]] when every painted AA row
// holds that one span, else 0.
extern "C" int rl_recti_box(const int32_t* edges, int n, int eo, int32_t y0, int32_t y1, int32_t aa_width,
                            int32_t lo, int32_t hi, int32_t* out) {
    rrb::PathInfo P{};
    P.e_begin = 0;
    P.e_end = static_cast<uint32_t>(n);
    P.paint = eo ? (1u << 16) : 0u;
    P.y0 = y0;
    P.y1 = y1;
    const rrb::Edge* e = reinterpret_cast<const rrb::Edge*>(edges);
    int32_t ev[rrb::RECTI_MAX_EVENTS];
    const int nev = rrb::recti_events(P, e, ev);
    return rrb::recti_box(P, e, ev, nev, aa_width, lo, hi, out[0], out[1], out[2], out[3]) ? 1 : 0;
}

// The clip-path lowering's XPath walk (xpath_segments in rrb_clip.cu): up to
// cap segments (x0, y0, x1, y1) in device space; returns the count.
extern "C" int64_t rl_xpath_segments(const double* pts, const uint8_t* flags, uint64_t n, const double* m,
                                     double flatness, double* out, int64_t cap) {
    std::vector<Seg> segs;
    std::vector<size_t> starts;
    xpath_segments(pts, flags, n, m, rrb::dmul(flatness, flatness), segs, starts);
    for (size_t k = 0; k < segs.size() && static_cast<int64_t>(k) < cap; ++k) {
        out[4 * k] = segs[k].x0;
        out[4 * k + 1] = segs[k].y0;
        out[4 * k + 2] = segs[k].x1;
        out[4 * k + 3] = segs[k].y1;
    }
    return static_cast<int64_t>(segs.size());
}
