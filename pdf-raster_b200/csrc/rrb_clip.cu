// rrb_clip.cu — non-rectangular clip paths (W / W* on a path that is not an
// axis-aligned rectangle), lowered on the host onto the rectangle-clipped
// batch that the device already renders.
//
// What the reference paints. Clip::clip_to_path (crates/raster/src/clip.rs:
// 141-176) pushes a scanner of the clip path's XPath, which the renderer
// builds with close_subpaths and without aa_scale (pdf_interp/src/renderer/
// page/mod.rs:1003-1009). fill_impl (raster/src/fill/mod.rs:110-244) then
// calls Clip::clip_aa_line for every AA line of the fill (clip.rs:246-254),
// and each clip scanner's render_aa_line clears the AA buffer and draws its
// own coverage (scanner/mod.rs:393-394) before the line is composited. So,
// unless the fill's box lies wholly outside the clip rectangle (test_rect,
// clip.rs:196-216), the page receives the clip path's coverage in the fill's
// paint on the pixel rows of the fill's loop; and because the clip's XPath is
// not scaled by AA_SIZE, that coverage is the clip path at a quarter of its
// size. The fill path's own coverage never reaches the page.
//
// The lowering. Per clipped fill, the clip path's XPath segments (walked and
// flattened here exactly as k_walk and k_seg_write do) become a polyline whose
// points are divided by 4 (exact); the device's make_edge multiplies them back
// by 4, so its edges are the clip scanner's segments and its AA rows are the
// clip scanner's rows. That polyline is filled with the clip's rule and the
// fill's paint, within the clip's columns. Which pixel rows it draws depends
// on the row map:
// - documented (one render_aa_line per pixel row y of the fill): the fill's
//   pixel rows, each showing the clip scanner's rows 4y .. 4y+3; the lowered
//   path is clipped to the fill's rows;
// - as shipped (fill/mod.rs:176-203: the loop runs over the fill's AA rows
//   and draws pixel row y = aa_y / 4 at aa_y % 4 == 3 after the clip scanner
//   rendered "row" aa_y, i.e. its rows 16y+12 .. 16y+15): the rows y with
//   4y+3 in the fill's scanner range, each showing the clip scanner's rows
//   16y+12 .. 16y+15 inside that scanner's own range (the clip rectangle's
//   rows when clip_to_path built it, clip.rs:152-171). The lowered path keeps
//   those rows as its clip and gets the fill's visited rows as visit rows
//   (rrb_record_path_batch_visit).
// A clip path that detect_rect (clip.rs:322-359) reduces to a rectangle
// becomes a rectangle clip of the fill itself.
// Of a stack of clip paths the last one that is not a rectangle is drawn:
// every scanner renders the same AA line in turn. The batch matrix must be
// the identity, as the renderer's DEVICE_MATRIX is (page/mod.rs:177).

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/rrb.h"
#include "rrb_device.cuh"

namespace {

using namespace rrb;

struct Seg {
    double x0, y0, x1, y1;
};

// Appends the segments of a flattened curve, from its start point on
// (flatten_curve is __host__ __device__; this emitter only runs on the host).
struct Chain {
    std::vector<Seg>* out;
    double cx, cy;
    __host__ __device__ void operator()(double fx, double fy) {
#ifndef __CUDA_ARCH__
        out->push_back(Seg{cx, cy, fx, fy});
#endif
        cx = fx;
        cy = fy;
    }
};

// XPath::new (xpath.rs:162-260) with close_subpaths, as k_walk (pieces) and
// k_seg_write (their segments) compute it: segments in walk order, in device
// space, and the index in `out` where each walk-subpath's segments begin.
void xpath_segments(const double* pts, const uint8_t* flags, uint64_t n, const double m[6], double flat_sq,
                    std::vector<Seg>& out, std::vector<size_t>& starts) {
    auto tp = [&](uint64_t i, double& x, double& y) { transform(m, pts[2 * i], pts[2 * i + 1], x, y); };
    uint64_t i = 0;
    while (i < n) {
        if (!(flags[i] & PF_FIRST)) {
            ++i;
            continue;
        }
        starts.push_back(out.size());
        const uint64_t sp = i;
        uint64_t cur = i;
        ++i;
        while (i < n) {
            const uint8_t f = flags[i];
            if (f & PF_CURVE) {
                if (i + 2 >= n) break;
                double x0, y0, x1, y1, x2, y2, x3, y3;
                tp(cur, x0, y0);
                tp(i, x1, y1);
                tp(i + 1, x2, y2);
                tp(i + 2, x3, y3);
                flatten_curve(x0, y0, x1, y1, x2, y2, x3, y3, flat_sq, Chain{&out, x0, y0});
                cur = i + 2;
                i += 3;
            } else {
                double ax, ay, bx, by;
                tp(cur, ax, ay);
                tp(i, bx, by);
                out.push_back(Seg{ax, ay, bx, by});
                cur = i;
                ++i;
                if (f & PF_LAST) break;
            }
        }
        double sx, sy, cx, cy;
        tp(sp, sx, sy);
        tp(cur, cx, cy);
        if (fabs(rrb::dsub(cx, sx)) > 1e-10 || fabs(rrb::dsub(cy, sy)) > 1e-10) out.push_back(Seg{cx, cy, sx, sy});
    }
}

// f64::min / f64::max: a NaN operand yields the other operand.
double rmin(double a, double b) { return std::fmin(a, b); }
double rmax(double a, double b) { return std::fmax(a, b); }

// The clip rectangle: Clip::new(0, 0, W, H) and clip_to_rect (clip.rs:73-88,
// 116-127, 266-271), float bounds and their integer bounds.
struct Rect {
    double x_min, y_min, x_max, y_max;
    int32_t x_min_i, y_min_i, x_max_i, y_max_i;
    void recompute() {
        x_min_i = splash_floor(x_min);
        y_min_i = splash_floor(y_min);
        x_max_i = sat_i32_of_integral(std::ceil(x_max)) - 1;
        y_max_i = sat_i32_of_integral(std::ceil(y_max)) - 1;
    }
    void clip_to(double a0, double b0, double a1, double b1) {
        x_min = rmax(x_min, rmin(a0, a1));
        x_max = rmin(x_max, rmax(a0, a1));
        y_min = rmax(y_min, rmin(b0, b1));
        y_max = rmin(y_max, rmax(b0, b1));
        recompute();
    }
};

bool same_bits(double a, double b) { return bits_of(a) == bits_of(b); }

// detect_rect (clip.rs:322-359) on XPath segments: add_segment marks HORIZ
// when the y bits agree (and VERT too when the x bits agree), else VERT when
// the x bits agree (xpath.rs:324-402).
bool detect_rect(const std::vector<Seg>& segs, double& x0, double& y0, double& x1, double& y1) {
    if (segs.size() != 4) return false;
    int verts = 0, horizs = 0;
    for (const Seg& s : segs) {
        const bool h = same_bits(s.y0, s.y1), v = same_bits(s.x0, s.x1);
        horizs += h;
        verts += v;
    }
    if (verts != 2 || horizs != 2) return false;
    x0 = INFINITY;
    x1 = -INFINITY;
    y0 = INFINITY;
    y1 = -INFINITY;
    for (const Seg& s : segs) {
        if (same_bits(s.x0, s.x1)) {
            x0 = rmin(rmin(x0, s.x0), s.x1);
            x1 = rmax(rmax(x1, s.x0), s.x1);
        }
        if (same_bits(s.y0, s.y1)) {
            y0 = rmin(rmin(y0, s.y0), s.y1);
            y1 = rmax(rmax(y1, s.y0), s.y1);
        }
    }
    return true;
}

// XPathScanner::new's box (scanner/mod.rs:131-248) of the fill's AA-scaled
// segments within AA rows [clip_lo, clip_hi]; false when the scanner is empty.
bool scanner_box(const std::vector<Seg>& segs, int32_t clip_lo, int32_t clip_hi, int32_t& x_min, int32_t& x_max,
                 int32_t& y_min, int32_t& y_max) {
    if (segs.empty() || clip_lo > clip_hi) return false;
    double xa = INFINITY, xb = -INFINITY, ya = INFINITY, yb = -INFINITY;
    for (const Seg& s0 : segs) {
        const Seg s{rrb::dmul(s0.x0, 4.0), rrb::dmul(s0.y0, 4.0), rrb::dmul(s0.x1, 4.0), rrb::dmul(s0.y1, 4.0)};
        if (std::isnan(s.x0) || std::isnan(s.y0) || std::isnan(s.x1) || std::isnan(s.y1)) continue;
        const double sy_min = rmin(s.y0, s.y1), sy_max = rmax(s.y0, s.y1);
        if (sy_min >= static_cast<double>(clip_hi) + 1.0 || sy_max < static_cast<double>(clip_lo)) continue;
        xa = rmin(rmin(xa, s.x0), s.x1);
        xb = rmax(rmax(xb, s.x0), s.x1);
        ya = rmin(ya, sy_min);
        yb = rmax(yb, sy_max);
    }
    if (xa > xb) return false;
    x_min = splash_floor(xa);
    x_max = splash_floor(xb);
    y_min = max(splash_floor(ya), clip_lo);
    y_max = min(splash_floor(yb), clip_hi);
    return y_min <= y_max;
}

// Visit rows meaning "the path's own" (rrb_record_path_batch_visit).
constexpr int32_t kOwnRows = INT32_MIN;

struct Out {
    double* pts;
    uint8_t* flags;
    uint64_t pts_cap;
    uint64_t* path_pt_off;
    uint64_t* src_path;
    uint8_t* rule;
    double* clip_rects;
    int32_t* visit_rows;
    uint64_t paths_cap;
    uint64_t n_pts = 0, n_paths = 0;

    void point(double x, double y, uint8_t f) {
        if (pts && n_pts < pts_cap) {
            pts[2 * n_pts] = x;
            pts[2 * n_pts + 1] = y;
        }
        if (flags && n_pts < pts_cap) flags[n_pts] = f;
        ++n_pts;
    }
    // visit v0 = kOwnRows: the path's own visited rows.
    void path(uint64_t src, uint8_t r, const Rect& c, double y0, double y1, uint64_t first_pt,
              int32_t v0 = kOwnRows, int32_t v1 = kOwnRows) {
        if (n_paths < paths_cap) {
            if (path_pt_off) path_pt_off[n_paths] = first_pt;
            if (src_path) src_path[n_paths] = src;
            if (rule) rule[n_paths] = r;
            if (clip_rects) {
                double* q = clip_rects + 4 * n_paths;
                q[0] = c.x_min;
                q[1] = y0;
                q[2] = c.x_max;
                q[3] = y1;
            }
            if (visit_rows) {
                visit_rows[2 * n_paths] = v0;
                visit_rows[2 * n_paths + 1] = v1;
            }
        }
        ++n_paths;
    }
};

}  // namespace

extern "C" int rrb_lower_clip_paths(const rrb_path_batch_params* p, const double* clip_rects,
                                    const rrb_clip_path* clip_paths, double* out_pts, uint8_t* out_flags,
                                    uint64_t pts_cap, uint64_t* out_path_pt_off, uint64_t* out_src_path,
                                    uint8_t* out_rule, double* out_clip_rects, int32_t* out_visit_rows,
                                    uint64_t paths_cap, uint64_t* n_pts_out, uint64_t* n_paths_out) {
    if (!p || !n_pts_out || !n_paths_out || (p->n_paths && (!p->path_pt_off || !p->fill_rule || !p->path_page)) ||
        (p->n_pts && (!p->pts || !p->flags)) || (p->n_pages && (!p->page_width || !p->page_height)))
        return RRB_ERR_INVARIANT;
    static const double kIdentity[6] = {1.0, 0.0, 0.0, 1.0, 0.0, 0.0};
    for (int k = 0; k < 6; ++k)
        if (!same_bits(p->matrix[k], kIdentity[k])) return RRB_ERR_INVARIANT;
    if (p->rowmap > RRB_ROWMAP_AS_SHIPPED) return RRB_ERR_INVARIANT;
    const bool shipped = p->rowmap == RRB_ROWMAP_AS_SHIPPED;
    const double flat_sq = rrb::dmul(p->flatness, p->flatness);
    Out o{out_pts, out_flags, pts_cap, out_path_pt_off, out_src_path, out_rule, out_clip_rects, out_visit_rows,
          paths_cap};
    std::vector<Seg> segs;
    std::vector<size_t> starts;
    for (uint64_t i = 0; i < p->n_paths; ++i) {
        const uint64_t a = p->path_pt_off[i], b = p->path_pt_off[i + 1];
        if (b < a || b > p->n_pts) return RRB_ERR_INVARIANT;
        const uint32_t pg = p->path_page[i];
        if (pg >= p->n_pages) return RRB_ERR_INVARIANT;
        Rect c{0.0, 0.0, static_cast<double>(p->page_width[pg]), static_cast<double>(p->page_height[pg]), 0, 0, 0, 0};
        c.recompute();
        if (clip_rects) {
            const double* r = clip_rects + 4 * i;
            c.clip_to(r[0], r[1], r[2], r[3]);
        }
        const rrb_clip_path* head = clip_paths ? clip_paths + i : nullptr;
        const bool has_clip = head && (head->n_pts > 0 || head->next);
        // The stack in order: empty paths empty the clip, rectangles narrow it,
        // and the last other clip path is the one whose coverage is drawn.
        bool have_path = false, emptied = false, eo_last = false;
        Rect c_scan = c;  // the clip rectangle when the drawn clip path's scanner was built
        segs.clear();
        starts.clear();
        int depth = 0;
        for (const rrb_clip_path* e = has_clip ? head : nullptr; e; e = e->next) {
            if (++depth > 4096) return RRB_ERR_INVARIANT;  // a cycle
            if (e->n_pts && (!e->pts || !e->flags)) return RRB_ERR_INVARIANT;
            std::vector<Seg> es;
            std::vector<size_t> est;
            if (e->n_pts) xpath_segments(e->pts, e->flags, e->n_pts, p->matrix, flat_sq, es, est);
            if (es.empty()) {
                emptied = true;  // clip.rs:142-148
                continue;
            }
            double rx0, ry0, rx1, ry1;
            if (detect_rect(es, rx0, ry0, rx1, ry1)) {
                c.clip_to(rx0, ry0, rx1, ry1);
                continue;
            }
            segs.swap(es);
            starts.swap(est);
            eo_last = e->even_odd != 0;
            have_path = true;
            c_scan = c;
        }
        // A clip with no integer column or row paints nothing (test_rect is
        // AllOutside, or the clamped span is empty). The device would read an
        // inverted rectangle as its normalised corners, so such paths are
        // dropped; an inverted one with a column left (floor(x_min) ==
        // ceil(x_max) - 1) normalises to the same integer bounds.
        if (emptied || c.x_min_i > c.x_max_i || c.y_min_i > c.y_max_i) continue;
        if (!have_path) {
            const uint64_t first = o.n_pts;
            for (uint64_t k = a; k < b; ++k) o.point(p->pts[2 * k], p->pts[2 * k + 1], p->flags[k]);
            o.path(i, p->fill_rule[i], c, c.y_min, c.y_max, first);
            continue;
        }
        // The fill's box and rows, and test_rect against the clip rectangle.
        std::vector<Seg> fsegs;
        std::vector<size_t> fstarts;
        xpath_segments(p->pts + 2 * a, p->flags + a, b - a, p->matrix, flat_sq, fsegs, fstarts);
        const int32_t clip_lo = c.y_min_i * 4, clip_hi = (c.y_max_i + 1) * 4 - 1;
        int32_t sx0, sx1, sy0, sy1;
        if (!scanner_box(fsegs, clip_lo, clip_hi, sx0, sx1, sy0, sy1)) continue;
        const int32_t left = sx0 / 4, right = sx1 / 4, top = sy0 / 4, bottom = sy1 / 4;
        if (static_cast<double>(right + 1) <= c.x_min || static_cast<double>(left) >= c.x_max ||
            static_cast<double>(bottom + 1) <= c.y_min || static_cast<double>(top) >= c.y_max)
            continue;  // AllOutside: fill_impl returns
        // The clip path's walk-subpaths, a quarter of their size.
        const uint64_t first = o.n_pts;
        for (size_t s = 0; s < starts.size(); ++s) {
            const size_t e0 = starts[s], e1 = s + 1 < starts.size() ? starts[s + 1] : segs.size();
            if (e0 == e1) continue;
            o.point(rrb::dmul(segs[e0].x0, 0.25), rrb::dmul(segs[e0].y0, 0.25), PF_FIRST);
            for (size_t e = e0; e < e1; ++e)
                o.point(rrb::dmul(segs[e].x1, 0.25), rrb::dmul(segs[e].y1, 0.25), e + 1 == e1 ? PF_LAST : 0);
        }
        if (shipped) {
            // The clip scanner's rows; the fill's visited pixel rows: 4y + 3 in [sy0, sy1].
            o.path(i, eo_last ? 1 : 0, c, c_scan.y_min, c_scan.y_max, first, sy0 >> 2, floor_div(sy1 - 3, 4));
        } else {
            // Rows top..bottom of the fill's loop (clamped to the page by the device).
            o.path(i, eo_last ? 1 : 0, c, static_cast<double>(top), static_cast<double>(bottom) + 1.0, first);
        }
    }
    if (out_path_pt_off && o.n_paths < paths_cap) out_path_pt_off[o.n_paths] = o.n_pts;
    *n_pts_out = o.n_pts;
    *n_paths_out = o.n_paths;
    return (o.n_pts > pts_cap && out_pts) || (o.n_paths > paths_cap && out_path_pt_off) ? RRB_ERR_POOL_EXHAUSTED
                                                                                         : RRB_OK;
}
