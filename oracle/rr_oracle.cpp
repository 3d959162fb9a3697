// rr_oracle.cpp — CPU oracle (test infrastructure only; see rr_oracle.h).
//
// Literal restatement of the reference CPU scanline anti-aliased fill path of
// pthomasfournet/pdf-raster. Citations are file:line within that project.
// Compile with -ffp-contract=off: Rust never contracts a*b+c, so every fused
// multiply-add below is an explicit std::fma where the reference writes
// f64::mul_add, and every other operation is a single IEEE-754 op.

#include "rr_oracle.h"

#include <immintrin.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

namespace {

constexpr int32_t AA_SIZE = 4;             // crates/raster/src/types.rs:27
constexpr int32_t MAX_CURVE_SPLITS = 1024; // crates/raster/src/types.rs:36

// AA_GAMMA (crates/raster/src/fill/mod.rs:46-48).
const uint8_t AA_GAMMA[17] = {0, 4, 11, 21, 32, 45, 59, 74, 90, 108, 126, 145, 166, 187, 209, 231, 255};

// saturate_f64_to_i32 (crates/color/src/convert.rs:221-240): non-finite -> MAX
// for +inf, MIN otherwise; `x as i64` saturates; then i32::try_from saturates.
inline int32_t saturate_f64_to_i32(double x) {
    if (!std::isfinite(x)) return x == std::numeric_limits<double>::infinity() ? INT32_MAX : INT32_MIN;
    int64_t v;
    if (x >= 9223372036854775807.0) v = INT64_MAX;
    else if (x <= -9223372036854775808.0) v = INT64_MIN;
    else v = static_cast<int64_t>(x);
    if (v > INT32_MAX) return INT32_MAX;
    if (v < INT32_MIN) return INT32_MIN;
    return static_cast<int32_t>(v);
}

// splash_floor (crates/color/src/convert.rs:262-265).
inline int32_t splash_floor(double x) { return saturate_f64_to_i32(std::floor(x)); }
// splash_ceil (crates/color/src/convert.rs:283-286).
inline int32_t splash_ceil(double x) { return saturate_f64_to_i32(std::ceil(x)); }

// fp_from_f64 (crates/raster/src/scanner/mod.rs:51-66): truncating 16.16
// conversion with saturation; `NaN as i32` is 0 in Rust.
inline int32_t fp_from_f64(double x) {
    double fp = x * 65536.0;
    if (fp >= 2147483647.0) return INT32_MAX;
    if (fp <= -2147483648.0) return INT32_MIN;
    if (std::isnan(fp)) return 0;
    return static_cast<int32_t>(fp);
}

// Rust f64::min / f64::max ignore a NaN operand, like C fmin/fmax.
inline double rmin(double a, double b) { return std::fmin(a, b); }
inline double rmax(double a, double b) { return std::fmax(a, b); }
// Rust f64::clamp (std): x<min -> min; x>max -> max.
inline double rclamp(double x, double lo, double hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}
inline int32_t sat_add_i32(int32_t a, int32_t b) {
    int64_t s = static_cast<int64_t>(a) + b;
    if (s > INT32_MAX) return INT32_MAX;
    if (s < INT32_MIN) return INT32_MIN;
    return static_cast<int32_t>(s);
}
inline uint64_t bits(double x) {
    uint64_t u;
    std::memcpy(&u, &x, 8);
    return u;
}
// f64::midpoint for operands with |a|,|b| <= f64::MAX/2 (all page coordinates).
inline double midpoint(double a, double b) {
    const double HI = std::numeric_limits<double>::max() / 2.0;
    const double LO = std::numeric_limits<double>::min() * 2.0;
    double aa = std::fabs(a), ab = std::fabs(b);
    if (aa <= HI && ab <= HI) return (a + b) / 2.0;
    if (aa < LO) return a + (b / 2.0);
    if (ab < LO) return (a / 2.0) + b;
    return (a / 2.0) + (b / 2.0);
}

}  // namespace

// ============================================================================
// A1: Path + PathBuilder (crates/raster/src/path/mod.rs:174-448)
// ============================================================================
struct or_path {
    std::vector<double> pts;  // x,y interleaved
    std::vector<uint8_t> flags;
    size_t cur_subpath = 0;
    size_t len() const { return flags.size(); }
    bool no_current_point() const { return cur_subpath == len(); }          // mod.rs:206-208
    bool one_point_subpath() const { return len() != 0 && cur_subpath == len() - 1; }  // :220-222
};

extern "C" {

or_path* or_path_new(void) { return new or_path(); }
void or_path_free(or_path* p) { delete p; }

// PathBuilder::move_to (path/mod.rs:330-339).
int or_path_move_to(or_path* p, double x, double y) {
    if (p->one_point_subpath()) return 2;  // BogusPath
    size_t len = p->len();
    p->pts.push_back(x);
    p->pts.push_back(y);
    p->flags.push_back(OR_PF_FIRST | OR_PF_LAST);
    p->cur_subpath = len;
    return 0;
}

// PathBuilder::line_to (path/mod.rs:354-364).
int or_path_line_to(or_path* p, double x, double y) {
    if (p->no_current_point()) return 1;  // NoCurPt
    p->flags.back() &= static_cast<uint8_t>(~OR_PF_LAST);
    p->pts.push_back(x);
    p->pts.push_back(y);
    p->flags.push_back(OR_PF_LAST);
    return 0;
}

// PathBuilder::curve_to (path/mod.rs:383-406).
int or_path_curve_to(or_path* p, double x1, double y1, double x2, double y2, double x3, double y3) {
    if (p->no_current_point()) return 1;
    p->flags.back() &= static_cast<uint8_t>(~OR_PF_LAST);
    p->pts.push_back(x1); p->pts.push_back(y1); p->flags.push_back(OR_PF_CURVE);
    p->pts.push_back(x2); p->pts.push_back(y2); p->flags.push_back(OR_PF_CURVE);
    p->pts.push_back(x3); p->pts.push_back(y3); p->flags.push_back(OR_PF_LAST);
    return 0;
}

// PathBuilder::close (path/mod.rs:409-448): the closing lineTo(first) is added
// only when force, or when the subpath has >= 2 points and first != last
// (PathPoint PartialEq, i.e. f64 ==).
int or_path_close(or_path* p, int force) {
    if (p->no_current_point()) return 1;
    size_t sp = p->cur_subpath;
    size_t last_idx = p->len() - 1;
    double fx = p->pts[2 * sp], fy = p->pts[2 * sp + 1];
    double lx = p->pts[2 * last_idx], ly = p->pts[2 * last_idx + 1];
    bool differ = !(fx == lx && fy == ly);
    if (force || (sp != last_idx && differ)) {
        int rc = or_path_line_to(p, fx, fy);
        if (rc) return rc;
    }
    size_t new_last = p->len() - 1;
    p->flags[sp] |= OR_PF_CLOSED;
    p->flags[new_last] |= OR_PF_CLOSED;
    p->cur_subpath = p->len();
    return 0;
}

int64_t or_path_len(const or_path* p) { return static_cast<int64_t>(p->len()); }
const double* or_path_pts(const or_path* p) { return p->pts.data(); }
const uint8_t* or_path_flags(const or_path* p) { return p->flags.data(); }

// A2: conic_to_cubic (crates/font/src/outline.rs:106-112).
void or_conic_to_cubic(double p0x, double p0y, double pcx, double pcy, double p3x, double p3y,
                       double out[4]) {
    out[0] = std::fma(p0x, 1.0 / 3.0, pcx * (2.0 / 3.0));
    out[1] = std::fma(p0y, 1.0 / 3.0, pcy * (2.0 / 3.0));
    out[2] = std::fma(pcx, 2.0 / 3.0, p3x * (1.0 / 3.0));
    out[3] = std::fma(pcy, 2.0 / 3.0, p3y * (1.0 / 3.0));
}

// ============================================================================
// A3: transform (crates/raster/src/xpath.rs:421-426)
// ============================================================================
void or_transform(const double m[6], double x, double y, double out[2]) {
    out[0] = std::fma(x, m[0], std::fma(y, m[2], m[4]));
    out[1] = std::fma(x, m[1], std::fma(y, m[3], m[5]));
}

// ============================================================================
// A5: flatten_curve (crates/raster/src/path/flatten.rs:109-215), with the
// explicit cx/cy/c_next slot arrays of CurveData (flatten.rs:54-82).
// ============================================================================
int32_t or_flatten_curve(const double p[8], double flatness_sq, double* out_xy, int32_t cap) {
    const int32_t n = MAX_CURVE_SPLITS + 1;
    static thread_local std::vector<double> cx(n * 3), cy(n * 3);
    static thread_local std::vector<int32_t> c_next(n);
    const int32_t max = MAX_CURVE_SPLITS;
    cx[0] = p[0]; cy[0] = p[1];
    cx[1] = p[2]; cy[1] = p[3];
    cx[2] = p[4]; cy[2] = p[5];
    cx[max * 3] = p[6]; cy[max * 3] = p[7];
    c_next[0] = max;
    int32_t count = 0;
    int32_t pp1 = 0;
    while (pp1 < max) {
        int32_t pp2 = c_next[pp1];
        double xl0 = cx[pp1 * 3], yl0 = cy[pp1 * 3];
        double xx1 = cx[pp1 * 3 + 1], yy1 = cy[pp1 * 3 + 1];
        double xx2 = cx[pp1 * 3 + 2], yy2 = cy[pp1 * 3 + 2];
        double xr3 = cx[pp2 * 3], yr3 = cy[pp2 * 3];
        double mx = midpoint(xl0, xr3);
        double my = midpoint(yl0, yr3);
        double dx1 = xx1 - mx, dy1 = yy1 - my;
        double dx2 = xx2 - mx, dy2 = yy2 - my;
        double d1 = std::fma(dx1, dx1, dy1 * dy1);
        double d2 = std::fma(dx2, dx2, dy2 * dy2);
        if (pp2 - pp1 == 1 || (d1 <= flatness_sq && d2 <= flatness_sq)) {
            if (count < cap) {
                out_xy[2 * count] = xr3;
                out_xy[2 * count + 1] = yr3;
            }
            ++count;
            pp1 = pp2;
        } else {
            double xl1 = midpoint(xl0, xx1), yl1 = midpoint(yl0, yy1);
            double xh = midpoint(xx1, xx2), yh = midpoint(yy1, yy2);
            double xl2 = midpoint(xl1, xh), yl2 = midpoint(yl1, yh);
            double xr2 = midpoint(xx2, xr3), yr2 = midpoint(yy2, yr3);
            double xr1 = midpoint(xh, xr2), yr1 = midpoint(yh, yr2);
            double xr0 = midpoint(xl2, xr1), yr0 = midpoint(yl2, yr1);
            int32_t pp3 = (pp1 + pp2) / 2;  // i32::midpoint of non-negatives
            cx[pp1 * 3 + 1] = xl1; cy[pp1 * 3 + 1] = yl1;
            cx[pp1 * 3 + 2] = xl2; cy[pp1 * 3 + 2] = yl2;
            c_next[pp1] = pp3;
            cx[pp3 * 3] = xr0; cy[pp3 * 3] = yr0;
            cx[pp3 * 3 + 1] = xr1; cy[pp3 * 3 + 1] = yr1;
            cx[pp3 * 3 + 2] = xr2; cy[pp3 * 3 + 2] = yr2;
            c_next[pp3] = pp2;
        }
    }
    return count;
}

// ============================================================================
// A4: add_segment (crates/raster/src/xpath.rs:324-402)
// ============================================================================
void or_add_segment(double x0, double y0, double x1, double y1, or_seg* out) {
    uint32_t flags = 0;
    if (bits(y0) == bits(y1)) {
        flags |= OR_XF_HORIZ;
        if (bits(x0) == bits(x1)) flags |= OR_XF_VERT;
        *out = or_seg{x0, y0, x1, y1, 0.0, 0, flags};
        return;
    }
    if (bits(x0) == bits(x1)) flags |= OR_XF_VERT;
    double dxdy = (flags & OR_XF_VERT) ? 0.0 : (x1 - x0) / (y1 - y0);
    if (y0 > y1) {
        std::swap(x0, x1);
        std::swap(y0, y1);
        flags |= OR_XF_FLIPPED;
    }
    int32_t dxdy_fp;
    double fp = dxdy * 65536.0;
    if (fp >= 2147483647.0) dxdy_fp = INT32_MAX;
    else if (fp <= -2147483648.0) dxdy_fp = INT32_MIN;
    else if (std::isnan(fp)) dxdy_fp = 0;
    else dxdy_fp = static_cast<int32_t>(std::round(fp));  // f64::round: half away from zero
    *out = or_seg{x0, y0, x1, y1, dxdy, dxdy_fp, flags};
}

// ============================================================================
// A4: XPath::new walk (crates/raster/src/xpath.rs:162-260). Stroke-adjust
// hints are empty for fills (build_adjusts on no hints is a no-op).
// ============================================================================
int64_t or_xpath_new(const double* pts, const uint8_t* flags, int64_t n, const double m[6],
                     double flatness, int close_subpaths, or_seg* out, int64_t cap) {
    double flatness_sq = flatness * flatness;
    std::vector<double> t(2 * n);
    for (int64_t i = 0; i < n; ++i) or_transform(m, pts[2 * i], pts[2 * i + 1], &t[2 * i]);
    int64_t ns = 0;
    auto add = [&](double ax, double ay, double bx, double by) {
        if (ns < cap) or_add_segment(ax, ay, bx, by, &out[ns]);
        ++ns;
    };
    std::vector<double> flat(2 * (MAX_CURVE_SPLITS + 1));
    int64_t i = 0;
    while (i < n) {
        if (flags[i] & OR_PF_FIRST) {
            double sp_x = t[2 * i], sp_y = t[2 * i + 1];
            double cur_x = sp_x, cur_y = sp_y;
            ++i;
            while (i < n) {
                if (flags[i] & OR_PF_CURVE) {
                    if (i + 2 >= n) break;
                    double cp[8] = {cur_x, cur_y, t[2 * i], t[2 * i + 1], t[2 * i + 2], t[2 * i + 3],
                                    t[2 * i + 4], t[2 * i + 5]};
                    int32_t k = or_flatten_curve(cp, flatness_sq, flat.data(), MAX_CURVE_SPLITS + 1);
                    for (int32_t j = 0; j < k; ++j) {
                        add(cur_x, cur_y, flat[2 * j], flat[2 * j + 1]);
                        cur_x = flat[2 * j];
                        cur_y = flat[2 * j + 1];
                    }
                    // Quirk: the curve branch does not test LAST (xpath.rs:210-234).
                    i += 3;
                } else {
                    double nx = t[2 * i], ny = t[2 * i + 1];
                    add(cur_x, cur_y, nx, ny);
                    cur_x = nx;
                    cur_y = ny;
                    bool is_last = (flags[i] & OR_PF_LAST) != 0;
                    ++i;
                    if (is_last) break;
                }
            }
            if (close_subpaths && (std::fabs(cur_x - sp_x) > 1e-10 || std::fabs(cur_y - sp_y) > 1e-10))
                add(cur_x, cur_y, sp_x, sp_y);
        } else {
            ++i;
        }
    }
    return ns;
}

// A6: XPath::aa_scale (crates/raster/src/xpath.rs:283-303).
void or_xpath_aa_scale(or_seg* segs, int64_t n) {
    const double s = static_cast<double>(AA_SIZE);
    for (int64_t i = 0; i < n; ++i) {
        segs[i].x0 *= s;
        segs[i].y0 *= s;
        segs[i].x1 *= s;
        segs[i].y1 *= s;
    }
}

}  // extern "C"

// ============================================================================
// A7: XPathScanner (crates/raster/src/scanner/mod.rs:131-248, 476-642)
// ============================================================================
struct or_scanner {
    bool eo = false;
    int32_t x_min = 1, x_max = 0, y_min = 0, y_max = -1;
    std::vector<uint32_t> row_start;
    std::vector<or_intersect> inters;
    bool is_empty() const { return x_min > x_max || y_min > y_max; }
    // XPathScanner::row (scanner/mod.rs:296-318).
    const or_intersect* row(int32_t y, int64_t* n) const {
        if (y < y_min || y > y_max) {
            *n = 0;
            return nullptr;
        }
        size_t i = static_cast<size_t>(static_cast<int64_t>(y) - y_min);
        size_t s = row_start[i], e = row_start[i + 1];
        *n = static_cast<int64_t>(e - s);
        return inters.data() + s;
    }
};

namespace {

// write_intersect (scanner/mod.rs:600-642): merge with the last entry written
// to this row when the spans touch or overlap, else append.
inline void write_intersect(int32_t row, int32_t y_min, const std::vector<uint32_t>& row_start,
                            std::vector<uint32_t>& cursors, std::vector<or_intersect>& it,
                            int32_t x0, int32_t x1, int32_t count) {
    int32_t lo = std::min(x0, x1), hi = std::max(x0, x1);
    size_t idx = static_cast<size_t>(row - y_min);
    size_t base = row_start[idx];
    size_t cur = cursors[idx];
    if (cur > 0) {
        or_intersect& last = it[base + cur - 1];
        if (sat_add_i32(last.x1, 1) >= lo && last.x0 <= sat_add_i32(hi, 1)) {
            last.count = static_cast<int32_t>(static_cast<uint32_t>(last.count) + static_cast<uint32_t>(count));
            last.x0 = std::min(last.x0, lo);
            last.x1 = std::max(last.x1, hi);
            return;
        }
    }
    it[base + cur] = or_intersect{lo, hi, count};
    cursors[idx] += 1;
}

// count_intersections (scanner/mod.rs:476-499).
void count_intersections(const or_seg* segs, int64_t n, int32_t y_min, int32_t y_max,
                         std::vector<uint32_t>& counts) {
    for (int64_t k = 0; k < n; ++k) {
        const or_seg& s = segs[k];
        if (std::isnan(s.x0) || std::isnan(s.y0)) continue;
        double sy_min = rmin(s.y0, s.y1), sy_max = rmax(s.y0, s.y1);
        int32_t row_y0 = std::max(splash_floor(sy_min), y_min);
        int32_t row_y1 = std::min(splash_floor(sy_max), y_max);
        if (s.flags & OR_XF_HORIZ) {
            int32_t row = splash_floor(sy_min);
            if (row >= y_min && row <= y_max) {
                uint32_t& c = counts[static_cast<size_t>(row - y_min)];
                if (c != UINT32_MAX) ++c;
            }
        } else {
            for (int64_t row = row_y0; row <= row_y1; ++row) {
                uint32_t& c = counts[static_cast<size_t>(row - y_min)];
                if (c != UINT32_MAX) ++c;
            }
        }
    }
}

// fill_intersections (scanner/mod.rs:511-587).
void fill_intersections(const or_seg* segs, int64_t n, int32_t y_min, int32_t y_max,
                        const std::vector<uint32_t>& row_start, std::vector<uint32_t>& cursors,
                        std::vector<or_intersect>& it) {
    for (int64_t k = 0; k < n; ++k) {
        const or_seg& s = segs[k];
        if (std::isnan(s.x0) || std::isnan(s.y0)) continue;
        double sy_min = rmin(s.y0, s.y1), sy_max = rmax(s.y0, s.y1);
        int32_t row_y0 = std::max(splash_floor(sy_min), y_min);
        int32_t row_y1 = std::min(splash_floor(sy_max), y_max);
        if (s.flags & OR_XF_HORIZ) {
            int32_t row = splash_floor(sy_min);
            if (row >= y_min && row <= y_max) {
                int32_t x0 = splash_floor(rmin(s.x0, s.x1));
                int32_t x1 = splash_floor(rmax(s.x0, s.x1));
                write_intersect(row, y_min, row_start, cursors, it, x0, x1, 0);
            }
        } else if (s.flags & OR_XF_VERT) {
            int32_t count = (s.flags & OR_XF_FLIPPED) ? 1 : -1;
            int32_t x = splash_floor(s.x0);
            for (int64_t row = row_y0; row <= row_y1; ++row) {
                int32_t c = sy_min < static_cast<double>(row) ? count : 0;
                write_intersect(static_cast<int32_t>(row), y_min, row_start, cursors, it, x, x, c);
            }
        } else {
            int32_t count = (s.flags & OR_XF_FLIPPED) ? 1 : -1;
            double x_base = std::fma(s.y0, -s.dxdy, s.x0);
            double sx_min = rmin(s.x0, s.x1), sx_max = rmax(s.x0, s.x1);
            int32_t fp_min = fp_from_f64(sx_min), fp_max = fp_from_f64(sx_max);
            double xx_init = static_cast<double>(row_y0) > s.y0
                                 ? std::fma(static_cast<double>(row_y0), s.dxdy, x_base)
                                 : s.x0;
            int32_t px0 = splash_floor(rclamp(xx_init, sx_min, sx_max));
            int32_t xx1_fp = fp_from_f64(std::fma(static_cast<double>(row_y0) + 1.0, s.dxdy, x_base));
            for (int64_t row = row_y0; row <= row_y1; ++row) {
                int32_t c1 = std::min(std::max(xx1_fp, fp_min), fp_max);
                int32_t px1 = c1 >> 16;  // arithmetic shift = floor
                int32_t c = sy_min < static_cast<double>(row) ? count : 0;
                write_intersect(static_cast<int32_t>(row), y_min, row_start, cursors, it, px0, px1, c);
                px0 = px1;
                xx1_fp = sat_add_i32(xx1_fp, s.dxdy_fp);
            }
        }
    }
}

// Per-row sort_unstable_by_key(|ix| ix.x0) (scanner/mod.rs:230). Rust std
// sorts slices of <= 20 elements by insertion sort (stable). Longer slices go
// through ipnsort: an existing non-descending run is left as is and a strictly
// descending run is reversed (both tie-free or stable); anything else reaches
// quicksort, whose order among equal keys is unspecified. That last case is
// sorted stably here and counted as unpinned when it has equal keys on
// differing entries.
void sort_row(or_intersect* v, size_t n, or_stats* st) {
    if (n < 2) return;
    if (n <= 20) {
        for (size_t i = 1; i < n; ++i) {
            or_intersect t = v[i];
            size_t j = i;
            while (j > 0 && t.x0 < v[j - 1].x0) {
                v[j] = v[j - 1];
                --j;
            }
            v[j] = t;
        }
        return;
    }
    bool desc = v[1].x0 < v[0].x0;
    size_t run = 2;
    if (desc) {
        while (run < n && v[run].x0 < v[run - 1].x0) ++run;
    } else {
        while (run < n && !(v[run].x0 < v[run - 1].x0)) ++run;
    }
    if (run == n) {
        if (desc) std::reverse(v, v + n);
        return;
    }
    std::stable_sort(v, v + n, [](const or_intersect& a, const or_intersect& b) { return a.x0 < b.x0; });
    if (st) {
        for (size_t i = 1; i < n; ++i) {
            if (v[i].x0 == v[i - 1].x0 && (v[i].x1 != v[i - 1].x1 || v[i].count != v[i - 1].count)) {
                st->unpinned_tie_rows++;
                break;
            }
        }
    }
}

}  // namespace

extern "C" {

// XPathScanner::new (scanner/mod.rs:131-248).
or_scanner* or_scanner_new(const or_seg* segs, int64_t n, int eo, int32_t clip_y_min,
                           int32_t clip_y_max, or_stats* st) {
    or_scanner* sc = new or_scanner();
    sc->eo = eo != 0;
    if (n == 0 || clip_y_min > clip_y_max) return sc;
    double x_min_fp = std::numeric_limits<double>::infinity();
    double x_max_fp = -std::numeric_limits<double>::infinity();
    double y_min_fp = std::numeric_limits<double>::infinity();
    double y_max_fp = -std::numeric_limits<double>::infinity();
    for (int64_t k = 0; k < n; ++k) {
        const or_seg& s = segs[k];
        if (std::isnan(s.x0) || std::isnan(s.y0) || std::isnan(s.x1) || std::isnan(s.y1)) continue;
        double sy_min = rmin(s.y0, s.y1), sy_max = rmax(s.y0, s.y1);
        if (sy_min >= static_cast<double>(clip_y_max) + 1.0 || sy_max < static_cast<double>(clip_y_min))
            continue;
        x_min_fp = rmin(rmin(x_min_fp, s.x0), s.x1);
        x_max_fp = rmax(rmax(x_max_fp, s.x0), s.x1);
        y_min_fp = rmin(y_min_fp, sy_min);
        y_max_fp = rmax(y_max_fp, sy_max);
    }
    if (x_min_fp > x_max_fp) return sc;
    int32_t x_min = splash_floor(x_min_fp), x_max = splash_floor(x_max_fp);
    int32_t y_min = std::max(splash_floor(y_min_fp), clip_y_min);
    int32_t y_max = std::min(splash_floor(y_max_fp), clip_y_max);
    if (y_min > y_max) return sc;
    size_t n_rows = static_cast<size_t>(static_cast<int64_t>(y_max) - y_min + 1);
    std::vector<uint32_t> counts(n_rows, 0);
    count_intersections(segs, n, y_min, y_max, counts);
    std::vector<uint32_t> alloc_start(n_rows + 1);
    uint64_t total = 0;
    for (size_t i = 0; i < n_rows; ++i) {
        alloc_start[i] = static_cast<uint32_t>(total);
        total += counts[i];
    }
    alloc_start[n_rows] = static_cast<uint32_t>(total);
    std::vector<or_intersect> it(total, or_intersect{0, 0, 0});
    std::fill(counts.begin(), counts.end(), 0u);
    fill_intersections(segs, n, y_min, y_max, alloc_start, counts, it);
    sc->row_start.resize(n_rows + 1);
    size_t write_pos = 0;
    for (size_t i = 0; i < n_rows; ++i) {
        sc->row_start[i] = static_cast<uint32_t>(write_pos);
        size_t rb = alloc_start[i], nw = counts[i];
        sort_row(it.data() + rb, nw, st);
        std::memmove(it.data() + write_pos, it.data() + rb, nw * sizeof(or_intersect));
        write_pos += nw;
    }
    sc->row_start[n_rows] = static_cast<uint32_t>(write_pos);
    it.resize(write_pos);
    sc->inters = std::move(it);
    sc->x_min = x_min;
    sc->x_max = x_max;
    sc->y_min = y_min;
    sc->y_max = y_max;
    if (st) {
        st->aa_rows += n_rows;
        st->intersects += write_pos;
    }
    return sc;
}

void or_scanner_free(or_scanner* s) { delete s; }

void or_scanner_bounds(const or_scanner* s, int32_t out[5]) {
    out[0] = s->y_min;
    out[1] = s->y_max;
    out[2] = s->x_min;
    out[3] = s->x_max;
    out[4] = s->is_empty() ? 1 : 0;
}

int64_t or_scanner_row(const or_scanner* s, int32_t y, or_intersect* out, int64_t cap) {
    int64_t n;
    const or_intersect* r = s->row(y, &n);
    for (int64_t i = 0; i < n && i < cap; ++i) out[i] = r[i];
    return n;
}

// count_crossings (scanner/mod.rs:327-340).
void or_count_crossings(const or_intersect* row, int64_t n, int32_t x, int32_t out[2]) {
    int32_t count = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (row[i].x0 > x) break;
        if (x <= row[i].x1) {
            out[0] = count;
            out[1] = 1;
            return;
        }
        count = static_cast<int32_t>(static_cast<uint32_t>(count) + static_cast<uint32_t>(row[i].count));
    }
    out[0] = count;
    out[1] = 0;
}

// XPathScanner::test (scanner/mod.rs:343-349).
int or_scanner_test(const or_scanner* s, int32_t x, int32_t y) {
    int64_t n;
    const or_intersect* r = s->row(y, &n);
    int32_t mask = s->eo ? 1 : ~0;
    int32_t out[2];
    or_count_crossings(r, n, x, out);
    return (out[1] || (out[0] & mask) != 0) ? 1 : 0;
}

// add_intersection (scanner/mod.rs:654-672).
int64_t or_add_intersection(or_intersect* row, int64_t n, int32_t x0, int32_t x1, int32_t count) {
    int32_t lo = std::min(x0, x1), hi = std::max(x0, x1);
    if (n == 0) {
        row[0] = or_intersect{lo, hi, count};
        return 1;
    }
    or_intersect& last = row[n - 1];
    if (sat_add_i32(last.x1, 1) < lo || last.x0 > sat_add_i32(hi, 1)) {
        row[n] = or_intersect{lo, hi, count};
        return n + 1;
    }
    last.count = static_cast<int32_t>(static_cast<uint32_t>(last.count) + static_cast<uint32_t>(count));
    last.x0 = std::min(last.x0, lo);
    last.x1 = std::max(last.x1, hi);
    return n;
}

// AaBuf::set_span (crates/raster/src/bitmap.rs:535-573).
void or_aabuf_set_span(uint8_t* buf, int64_t width, int64_t row, int64_t x0, int64_t x1) {
    x0 = std::min(x0, width);
    x1 = std::min(x1, width);
    if (x0 >= x1) return;
    int64_t rb = (width + 7) / 8;
    uint8_t* base = buf + row * rb;
    int64_t b0 = x0 >> 3, b1 = (x1 - 1) >> 3;
    uint8_t right_mask = (x1 & 7) == 0 ? 0xff : static_cast<uint8_t>(~(0xffu >> (x1 & 7)));
    if (b0 == b1) {
        base[b0] |= static_cast<uint8_t>((0xffu >> (x0 & 7)) & right_mask);
    } else {
        base[b0] |= static_cast<uint8_t>(0xffu >> (x0 & 7));
        for (int64_t b = b0 + 1; b < b1; ++b) base[b] = 0xff;
        base[b1] |= right_mask;
    }
}

// XPathScanner::render_aa_line (scanner/mod.rs:393-467). One guard is added:
// when a row's winding count never returns to zero the reference loops
// forever after painting [xx, aa_width); here the walk stops after that paint
// and the row is counted in st->nonterminating_rows.
void or_render_aa_line(const or_scanner* s, uint8_t* aa_buf, int64_t aa_width, int32_t y,
                       int32_t out[2], or_stats* st) {
    int64_t rb = (aa_width + 7) / 8;
    std::memset(aa_buf, 0, static_cast<size_t>(rb * AA_SIZE));
    int32_t aw = aa_width > INT32_MAX ? INT32_MAX : static_cast<int32_t>(aa_width);
    int32_t xx_min = aw, xx_max = -1;
    int32_t mask = s->eo ? 1 : ~0;
    for (int32_t yy = 0; yy < AA_SIZE; ++yy) {
        int64_t scan_y64 = static_cast<int64_t>(y) * AA_SIZE + yy;
        int64_t nrow = 0;
        const or_intersect* row = nullptr;
        if (scan_y64 >= INT32_MIN && scan_y64 <= INT32_MAX) row = s->row(static_cast<int32_t>(scan_y64), &nrow);
        int32_t count = 0;
        int64_t i = 0;
        int32_t xx = 0;
        while (i < nrow || (count & mask) != 0) {
            if ((count & mask) == 0) {
                if (i >= nrow) break;
                xx = row[i].x0;
                count = static_cast<int32_t>(static_cast<uint32_t>(count) + static_cast<uint32_t>(row[i].count));
                ++i;
                continue;
            }
            int32_t span_x1;
            bool ran_out = false;
            for (;;) {
                if (i >= nrow) {
                    span_x1 = aw;
                    ran_out = true;
                    break;
                }
                count = static_cast<int32_t>(static_cast<uint32_t>(count) + static_cast<uint32_t>(row[i].count));
                int32_t end = static_cast<int32_t>(static_cast<uint32_t>(row[i].x1) + 1u);
                ++i;
                if ((count & mask) == 0) {
                    span_x1 = end;
                    break;
                }
            }
            int64_t bx0 = std::max(xx, 0);
            int64_t bx1 = std::max(std::min(span_x1, aw), 0);
            if (bx0 < bx1) {
                or_aabuf_set_span(aa_buf, aa_width, yy, bx0, bx1);
                if (bx0 < xx_min) xx_min = static_cast<int32_t>(bx0);
                if (bx1 > xx_max) xx_max = static_cast<int32_t>(bx1);
            }
            xx = span_x1;
            if (ran_out) {
                if (st) st->nonterminating_rows++;
                break;
            }
        }
    }
    if (xx_min > xx_max) {
        out[0] = 0;
        out[1] = -1;
        return;
    }
    out[0] = xx_min / AA_SIZE;
    out[1] = (xx_max - 1) / AA_SIZE;
}

// aa_coverage_span (crates/raster/src/simd/aa_coverage.rs:490-514): the
// coverage count 0..16 of output pixels x0 .. x0+n-1 from the four AaBuf
// sub-rows (row_bytes apart). Pixel x is nibble x & 1 of byte x >> 1 of each
// row (even pixel = high nibble). The reference dispatches on the host CPU:
// an odd x0 goes to the scalar loop; otherwise the AVX-512 BITALG tier when
// avx512bitalg and avx512bw are present, else the AVX2 tier, else scalar.
// All tiers count the same bits; the SIMD ones take whole chunks of row bytes
// (64 for AVX-512, 32 for AVX2: coverage_chunk_params, :84-93) and leave the
// rest of the span to the scalar loop, as the reference does.
namespace {

// aa_coverage_span_scalar (:51-69).
void coverage_scalar(const uint8_t* aa_buf, int64_t row_bytes, int64_t x0, uint8_t* shape, int64_t n) {
    for (int64_t i = 0; i < n; ++i) {
        int64_t x = x0 + i;
        int64_t bi = x >> 1;
        bool odd = (x & 1) != 0;
        int c = 0;
        for (int r = 0; r < 4; ++r) {
            uint8_t b = aa_buf[r * row_bytes + bi];
            uint8_t nib = odd ? (b & 0x0f) : (b >> 4);
            c += __builtin_popcount(nib);
        }
        shape[i] = static_cast<uint8_t>(c);
    }
}

// Writes even pixel 2k <- hi[k], odd pixel 2k+1 <- lo[k] for the first
// min(2 * bytes, n) pixels of a chunk.
inline void interleave(const uint8_t* hi, const uint8_t* lo, int bytes, uint8_t* shape, int64_t n) {
    for (int k = 0; k < bytes; ++k) {
        if (2 * k < n) shape[2 * k] = hi[k];
        if (2 * k + 1 < n) shape[2 * k + 1] = lo[k];
    }
}

// AVX2 tier (:310-380): a 16-entry nibble-popcount table looked up with a
// byte shuffle, 32 row bytes (64 pixels) per step.
__attribute__((target("avx2"))) void coverage_avx2(const uint8_t* aa_buf, int64_t row_bytes, int64_t x0,
                                                    uint8_t* shape, int64_t n) {
    const int64_t b0 = x0 >> 1, chunks = ((n + 1) / 2) / 32;
    const __m256i table = _mm256_setr_epi8(0, 1, 1, 2, 1, 2, 2, 3, 1, 2, 2, 3, 2, 3, 3, 4,
                                           0, 1, 1, 2, 1, 2, 2, 3, 1, 2, 2, 3, 2, 3, 3, 4);
    const __m256i low4 = _mm256_set1_epi8(0x0f);
    alignas(32) uint8_t hi[32], lo[32];
    for (int64_t c = 0; c < chunks; ++c) {
        __m256i acc_hi = _mm256_setzero_si256(), acc_lo = _mm256_setzero_si256();
        for (int r = 0; r < 4; ++r) {
            const __m256i v = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(aa_buf + r * row_bytes + b0 + 32 * c));
            acc_hi = _mm256_add_epi8(acc_hi, _mm256_shuffle_epi8(table, _mm256_and_si256(_mm256_srli_epi16(v, 4), low4)));
            acc_lo = _mm256_add_epi8(acc_lo, _mm256_shuffle_epi8(table, _mm256_and_si256(v, low4)));
        }
        _mm256_store_si256(reinterpret_cast<__m256i*>(hi), acc_hi);
        _mm256_store_si256(reinterpret_cast<__m256i*>(lo), acc_lo);
        interleave(hi, lo, 32, shape + 64 * c, n - 64 * c);
    }
    if (64 * chunks < n) coverage_scalar(aa_buf, row_bytes, x0 + 64 * chunks, shape + 64 * chunks, n - 64 * chunks);
}

// AVX-512 BITALG tier (:403-471): a per-byte popcount of each isolated
// nibble, 64 row bytes (128 pixels) per step.
__attribute__((target("avx512f,avx512bw,avx512bitalg"))) void coverage_avx512(const uint8_t* aa_buf,
                                                                              int64_t row_bytes, int64_t x0,
                                                                              uint8_t* shape, int64_t n) {
    const int64_t b0 = x0 >> 1, chunks = ((n + 1) / 2) / 64;
    const __m512i low4 = _mm512_set1_epi8(0x0f);
    alignas(64) uint8_t hi[64], lo[64];
    for (int64_t c = 0; c < chunks; ++c) {
        __m512i acc_hi = _mm512_setzero_si512(), acc_lo = _mm512_setzero_si512();
        for (int r = 0; r < 4; ++r) {
            const __m512i v = _mm512_loadu_si512(aa_buf + r * row_bytes + b0 + 64 * c);
            acc_hi = _mm512_add_epi8(acc_hi, _mm512_popcnt_epi8(_mm512_and_si512(_mm512_srli_epi16(v, 4), low4)));
            acc_lo = _mm512_add_epi8(acc_lo, _mm512_popcnt_epi8(_mm512_and_si512(v, low4)));
        }
        _mm512_store_si512(hi, acc_hi);
        _mm512_store_si512(lo, acc_lo);
        interleave(hi, lo, 64, shape + 128 * c, n - 128 * c);
    }
    if (128 * chunks < n) coverage_scalar(aa_buf, row_bytes, x0 + 128 * chunks, shape + 128 * chunks, n - 128 * chunks);
}

int detect_tier() {
    __builtin_cpu_init();
    if (__builtin_cpu_supports("avx512bitalg") && __builtin_cpu_supports("avx512bw")) return 2;
    if (__builtin_cpu_supports("avx2")) return 1;
    return 0;
}

const int g_tier = detect_tier();

}  // namespace

// The tier dispatch uses on this host: 2 AVX-512 BITALG, 1 AVX2, 0 scalar.
int or_coverage_tier(void) { return g_tier; }

// One tier explicitly (for the scalar-vs-SIMD agreement check); a tier the
// host lacks falls back to the best one it has. Odd x0 is always scalar.
void or_aa_coverage_span_tier(const uint8_t* aa_buf, int64_t row_bytes, int64_t x0, uint8_t* shape, int64_t n,
                              int tier) {
    if (n <= 0) return;
    if (tier > g_tier) tier = g_tier;
    if ((x0 & 1) || tier == 0) coverage_scalar(aa_buf, row_bytes, x0, shape, n);
    else if (tier == 2) coverage_avx512(aa_buf, row_bytes, x0, shape, n);
    else coverage_avx2(aa_buf, row_bytes, x0, shape, n);
}

void or_aa_coverage_span(const uint8_t* aa_buf, int64_t row_bytes, int64_t x0, uint8_t* shape,
                         int64_t n) {
    or_aa_coverage_span_tier(aa_buf, row_bytes, x0, shape, n, g_tier);
}

const uint8_t* or_aa_gamma(void) { return AA_GAMMA; }

// div255 (crates/color/src/convert.rs:50-58).
uint8_t or_div255(uint32_t x) {
    uint32_t s = (x + (x >> 8) + 0x80) >> 8;
    return static_cast<uint8_t>(s > 255 ? 255 : s);
}

// render_span_aa_inner, no alpha plane, one component (pipe/aa.rs:192-208).
void or_render_span_aa_gray(uint8_t* dst, const uint8_t* shape, int64_t n, uint8_t a_input,
                            uint8_t gray) {
    uint32_t ai = a_input;
    for (int64_t i = 0; i < n; ++i) {
        uint32_t a_src = or_div255(ai * shape[i]);
        dst[i] = or_div255((255u - a_src) * dst[i] + a_src * gray);
    }
}

// composite_aa_rgb8_opaque (crates/raster/src/simd/composite.rs:30-32,56+).
void or_composite_aa_rgb8_opaque(uint8_t* dst, const uint8_t src[3], uint8_t a_input,
                                 const uint8_t* shape, int64_t n) {
    auto d = [](uint32_t v) { return static_cast<uint32_t>((v + 255u) >> 8); };
    for (int64_t k = 0; k < n; ++k) {
        uint32_t a_src = d(uint32_t(a_input) * shape[k]);
        uint32_t inv = 255u - a_src;
        for (int c = 0; c < 3; ++c) dst[3 * k + c] = static_cast<uint8_t>(d(inv * dst[3 * k + c] + a_src * src[c]));
    }
}

// rgb_to_gray (crates/pdf_raster/src/render.rs:1306-1324).
void or_rgb_to_gray(const uint8_t* rgb, uint8_t* gray, int64_t n) {
    for (int64_t i = 0; i < n; ++i) {
        uint32_t r = rgb[3 * i], g = rgb[3 * i + 1], b = rgb[3 * i + 2];
        gray[i] = static_cast<uint8_t>((2126u * r + 7152u * g + 722u * b + 5000u) / 10000u);
    }
}

// fill_impl (crates/raster/src/fill/mod.rs:110-244), vector_antialias = true,
// page clip Clip::new(0, 0, W, H, true) (clip.rs:73-88, recompute_int_bounds
// :266-271), Gray8 page without alpha plane, identity transfer, solid source.
}  // extern "C"

namespace {

// fill_impl for one path; `span(y, x0, shape, n)` composites a gamma-mapped
// shape span onto pixel row y (the page's pixel format lives in `span`).
// The clip of a fill: Clip::new(0, 0, W, H) and, with `rect`, clip_to_rect
// (clip.rs:73-88,116-125,266-271): float bounds and their integer bounds.
struct ClipRect {
    double x_min, y_min, x_max, y_max;
    int32_t x_min_i, y_min_i, x_max_i, y_max_i;
};

ClipRect make_clip(int32_t width, int32_t height, const double* rect) {
    ClipRect c{0.0, 0.0, static_cast<double>(width), static_cast<double>(height), 0, 0, 0, 0};
    if (rect) {
        c.x_min = std::max(c.x_min, std::min(rect[0], rect[2]));
        c.x_max = std::min(c.x_max, std::max(rect[0], rect[2]));
        c.y_min = std::max(c.y_min, std::min(rect[1], rect[3]));
        c.y_max = std::min(c.y_max, std::max(rect[1], rect[3]));
    }
    c.x_min_i = splash_floor(c.x_min);
    c.y_min_i = splash_floor(c.y_min);
    c.x_max_i = splash_ceil(c.x_max) - 1;
    c.y_max_i = splash_ceil(c.y_max) - 1;
    return c;
}

// Clip::recompute_int_bounds (clip.rs:266-271).
void recompute_int_bounds(ClipRect& c) {
    c.x_min_i = splash_floor(c.x_min);
    c.y_min_i = splash_floor(c.y_min);
    c.x_max_i = splash_ceil(c.x_max) - 1;
    c.y_max_i = splash_ceil(c.y_max) - 1;
}

// detect_rect (clip.rs:322-359): exactly four segments, two carrying VERT and
// two carrying HORIZ (a zero-length segment carries both), give the box of
// the vertical segments' x and the horizontal segments' y.
bool detect_rect(const std::vector<or_seg>& segs, double& x0, double& y0, double& x1, double& y1) {
    if (segs.size() != 4) return false;
    int verts = 0, horizs = 0;
    for (const or_seg& g : segs) {
        if (g.flags & OR_XF_VERT) ++verts;
        if (g.flags & OR_XF_HORIZ) ++horizs;
    }
    if (verts != 2 || horizs != 2) return false;
    x0 = INFINITY;
    x1 = -INFINITY;
    y0 = INFINITY;
    y1 = -INFINITY;
    for (const or_seg& g : segs) {
        if (g.flags & OR_XF_VERT) {
            x0 = std::fmin(std::fmin(x0, g.x0), g.x1);  // f64::min ignores a NaN operand, as fmin does
            x1 = std::fmax(std::fmax(x1, g.x0), g.x1);
        }
        if (g.flags & OR_XF_HORIZ) {
            y0 = std::fmin(std::fmin(y0, g.y0), g.y1);
            y1 = std::fmax(std::fmax(y1, g.y0), g.y1);
        }
    }
    return true;
}

// A clip region: the rectangle and the path-clip scanners pushed by
// clip_to_path (clip.rs:141-176).
struct ClipState {
    ClipRect r;
    std::vector<or_scanner*> scanners;
    ClipState() = default;
    ClipState(const ClipState&) = delete;
    ClipState& operator=(const ClipState&) = delete;
    ~ClipState() {
        for (or_scanner* sc : scanners) or_scanner_free(sc);
    }
};

// Clip::clip_to_path (clip.rs:141-176) with the renderer's XPath: built with
// close_subpaths = true and without aa_scale (pdf_interp/src/renderer/page/
// mod.rs:1003-1009). An empty path empties the clip; a detected rectangle
// becomes clip_to_rect (clip.rs:119-127); otherwise a scanner over AA rows
// [4 y_min_i, 4 (y_max_i + 1) - 1] is pushed.
void clip_to_path(ClipState& cs, const double* pts, const uint8_t* flags, int64_t n, const double m[6],
                  double flatness, int eo, or_stats* st) {
    const int64_t need = or_xpath_new(pts, flags, n, m, flatness, 1, nullptr, 0);
    std::vector<or_seg> segs(static_cast<size_t>(need));
    if (need) or_xpath_new(pts, flags, n, m, flatness, 1, segs.data(), need);
    ClipRect& c = cs.r;
    if (segs.empty()) {
        c.x_max = c.x_min - 1.0;
        c.y_max = c.y_min - 1.0;
        recompute_int_bounds(c);
        return;
    }
    double rx0, ry0, rx1, ry1;
    if (detect_rect(segs, rx0, ry0, rx1, ry1)) {
        c.x_min = std::fmax(c.x_min, std::fmin(rx0, rx1));
        c.x_max = std::fmin(c.x_max, std::fmax(rx0, rx1));
        c.y_min = std::fmax(c.y_min, std::fmin(ry0, ry1));
        c.y_max = std::fmin(c.y_max, std::fmax(ry0, ry1));
        recompute_int_bounds(c);
        return;
    }
    const int32_t y_lo = c.y_min_i * AA_SIZE, y_hi = (c.y_max_i + 1) * AA_SIZE - 1;
    cs.scanners.push_back(or_scanner_new(segs.data(), need, eo, y_lo, y_hi, st));
}

// clip_state: when given, the clip (rectangle and path scanners) instead of
// the page and clip_rect. With path scanners the fill is never AllInside
// (clip.rs:210-216) and clip_aa_line lets every scanner render the AA rows
// of the same row argument into the buffer (clip.rs:246-254).
template <typename Span>
void fill_path_impl(int32_t width, int32_t height, const double* pts, const uint8_t* flags, int64_t n_pts,
                    const double m[6], double flatness, int eo, int rowmap, or_stats* st, Span span,
                    const double* clip_rect = nullptr, const ClipState* clip_state = nullptr) {
    if (n_pts == 0) return;
    if (st) st->paths++;
    // XPath::new with close_subpaths = true, then aa_scale.
    int64_t need = or_xpath_new(pts, flags, n_pts, m, flatness, 1, nullptr, 0);
    std::vector<or_seg> segs(static_cast<size_t>(need));
    or_xpath_new(pts, flags, n_pts, m, flatness, 1, segs.data(), need);
    or_xpath_aa_scale(segs.data(), need);
    if (st) st->segments += static_cast<uint64_t>(need);
    // Clip integer bounds (the page, or the page and a clip rectangle).
    const ClipRect cr = clip_state ? clip_state->r : make_clip(width, height, clip_rect);
    const bool has_paths = clip_state && !clip_state->scanners.empty();
    int32_t clip_x_min_i = cr.x_min_i, clip_y_min_i = cr.y_min_i;
    int32_t clip_x_max_i = cr.x_max_i;
    int32_t clip_y_max_i = cr.y_max_i;
    int32_t y_lo = clip_y_min_i * AA_SIZE;
    int32_t y_hi = (clip_y_max_i + 1) * AA_SIZE - 1;
    or_scanner* sc = or_scanner_new(segs.data(), need, eo, y_lo, y_hi, st);
    if (sc->is_empty() || width == 0) {
        delete sc;
        return;
    }
    // Clip::test_rect (clip.rs:196-215) against the page rectangle.
    int32_t left = sc->x_min / AA_SIZE, top = sc->y_min / AA_SIZE;
    int32_t right = sc->x_max / AA_SIZE, bottom = sc->y_max / AA_SIZE;
    double cx_min = cr.x_min, cx_max = cr.x_max, cy_min = cr.y_min, cy_max = cr.y_max;
    bool all_outside = static_cast<double>(right + 1) <= cx_min || static_cast<double>(left) >= cx_max ||
                       static_cast<double>(bottom + 1) <= cy_min || static_cast<double>(top) >= cy_max;
    if (all_outside) {
        delete sc;
        return;
    }
    bool all_inside = static_cast<double>(left) >= cx_min && static_cast<double>(right + 1) <= cx_max &&
                      static_cast<double>(top) >= cy_min && static_cast<double>(bottom + 1) <= cy_max && !has_paths;
    int64_t aa_width = static_cast<int64_t>(width) * AA_SIZE;
    int64_t rb = (aa_width + 7) / 8;
    std::vector<uint8_t> aa_buf(static_cast<size_t>(rb * AA_SIZE), 0);
    std::vector<uint8_t> shape(static_cast<size_t>(width));
    auto draw = [&](int32_t x0, int32_t x1, int32_t y) {
        // draw_aa_line (fill/mod.rs:344-401).
        int64_t cnt = static_cast<int64_t>(x1) - x0 + 1;
        or_aa_coverage_span(aa_buf.data(), rb, x0, shape.data(), cnt);
        bool any = false;
        for (int64_t i = 0; i < cnt; ++i) {
            if (shape[i]) {
                shape[i] = AA_GAMMA[shape[i]];
                any = true;
            }
        }
        if (!any) return;
        span(y, x0, shape.data(), cnt);
    };
    auto clip_aa_line = [&](int32_t row_arg, int32_t* x0, int32_t* x1) {
        // Clip::clip_aa_line (clip.rs:246-254): each path-clip scanner's
        // render_aa_line clears the buffer and draws its own coverage.
        if (has_paths) {
            int32_t cx[2];
            for (const or_scanner* cs : clip_state->scanners) {
                or_render_aa_line(cs, aa_buf.data(), aa_width, row_arg, cx, st);
                *x0 = cx[0];
                *x1 = cx[1];
            }
        }
        *x0 = std::max(*x0, clip_x_min_i);
        *x1 = std::min(*x1, clip_x_max_i);
    };
    int32_t xr[2];
    if (rowmap == OR_ROWMAP_AS_SHIPPED) {
        // Literal loop (fill/mod.rs:176-204): render_aa_line is handed the AA
        // row index as its device-row argument.
        for (int32_t aa_y = sc->y_min; aa_y <= sc->y_max; ++aa_y) {
            int32_t y = aa_y / AA_SIZE;
            int32_t aa_row = aa_y % AA_SIZE;
            or_render_aa_line(sc, aa_buf.data(), aa_width, aa_y, xr, st);
            if (!all_inside) clip_aa_line(aa_y, &xr[0], &xr[1]);
            if (aa_row == AA_SIZE - 1) {
                if (xr[0] <= xr[1] && y >= 0 && y < height) draw(xr[0], xr[1], y);
                std::fill(aa_buf.begin(), aa_buf.end(), 0);
            }
        }
    } else {
        // Documented form (fill/mod.rs:12-17): one render_aa_line per pixel row.
        int32_t y0 = sc->y_min / AA_SIZE, y1 = sc->y_max / AA_SIZE;
        for (int32_t y = y0; y <= y1; ++y) {
            or_render_aa_line(sc, aa_buf.data(), aa_width, y, xr, st);
            if (!all_inside) clip_aa_line(y, &xr[0], &xr[1]);
            if (xr[0] <= xr[1] && y >= 0 && y < height) draw(xr[0], xr[1], y);
        }
    }
    delete sc;
}

// ============================================================================
// F2: strokes (crates/raster/src/stroke/mod.rs:58-283, stroke/path.rs:40-745).
// stroke(): flatten_path -> make_dashed_path (dash array set) -> line width
// 0: stroke_narrow (hairline spans, no AA) / else stroke_wide (outline of
// make_stroke_path filled nonzero with AA). Stroke adjustment is not restated:
// the reference's renderer always passes stroke_adjust = false
// (pdf_interp/src/renderer/page/mod.rs:1217-1227), so no hints are made.
// ============================================================================

constexpr double BEZIER_CIRCLE = 0.55228475;              // types.rs:45
constexpr double BEZIER_CIRCLE2 = 0.5 * BEZIER_CIRCLE;    // stroke/path.rs:16
constexpr double MITER_NEARLY_STRAIGHT = 0.9999;          // stroke/path.rs:22
constexpr double PI_F64 = 3.141592653589793;              // std::f64::consts::PI

// splash_dist (stroke/path.rs:741-745): f64::hypot, i.e. libm hypot.
inline double splash_dist(double x0, double y0, double x1, double y1) { return std::hypot(x1 - x0, y1 - y0); }

struct PathView {
    const double* pts;
    const uint8_t* flags;
    size_t n;
    double x(size_t i) const { return pts[2 * i]; }
    double y(size_t i) const { return pts[2 * i + 1]; }
    bool first(size_t i) const { return flags[i] & OR_PF_FIRST; }
    bool last(size_t i) const { return flags[i] & OR_PF_LAST; }
    bool closed(size_t i) const { return flags[i] & OR_PF_CLOSED; }
    bool curve(size_t i) const { return flags[i] & OR_PF_CURVE; }
};

PathView view_of(const or_path& p) { return PathView{p.pts.data(), p.flags.data(), p.len()}; }

// flatten_path (stroke/path.rs:40-86): curves flattened in user space against
// flatness^2; builder errors are ignored as the reference ignores them.
void flatten_path(const PathView& path, double flatness, or_path* out) {
    const double flatness_sq = flatness * flatness;
    std::vector<double> flat(2 * (MAX_CURVE_SPLITS + 1));
    size_t i = 0;
    while (i < path.n) {
        if (path.first(i)) {
            or_path_move_to(out, path.x(i), path.y(i));
            i += 1;
        } else if (path.curve(i)) {
            if (i == 0 || i + 2 >= path.n) break;  // the reference indexes out of bounds here
            const double cp[8] = {path.x(i - 1), path.y(i - 1), path.x(i), path.y(i),
                                  path.x(i + 1), path.y(i + 1), path.x(i + 2), path.y(i + 2)};
            const int32_t k = or_flatten_curve(cp, flatness_sq, flat.data(), MAX_CURVE_SPLITS + 1);
            for (int32_t j = 0; j < k; ++j) or_path_line_to(out, flat[2 * j], flat[2 * j + 1]);
            i += 3;
            if (path.closed(i - 1)) or_path_close(out, 0);
        } else {
            or_path_line_to(out, path.x(i), path.y(i));
            i += 1;
            if (path.closed(i - 1)) or_path_close(out, 0);
        }
    }
}

// make_dashed_path (stroke/path.rs:107-220).
void make_dashed_path(const PathView& path, const double* line_dash, size_t n_dash, double line_dash_phase,
                      or_path* out) {
    double line_dash_total = 0.0;
    for (size_t k = 0; k < n_dash; ++k) line_dash_total += line_dash[k];
    if (n_dash == 0 || line_dash_total < std::numeric_limits<double>::epsilon()) return;
    double phase = line_dash_phase;
    {
        const int32_t periods = splash_floor(phase / line_dash_total);
        phase -= static_cast<double>(periods) * line_dash_total;
    }
    bool dash_start_on = true;
    size_t dash_start_idx = 0;
    if (phase > 0.0) {
        while (dash_start_idx < n_dash && phase >= line_dash[dash_start_idx]) {
            dash_start_on = !dash_start_on;
            phase -= line_dash[dash_start_idx];
            dash_start_idx += 1;
        }
        if (dash_start_idx == n_dash) return;
    }
    size_t i = 0;
    while (i < path.n) {
        size_t j = i;
        while (j < (path.n > 0 ? path.n - 1 : 0) && !path.last(j)) j += 1;
        bool dash_on = dash_start_on;
        size_t dash_idx = dash_start_idx;
        double dash_dist = line_dash[dash_idx] - phase;
        bool new_path = true;
        for (size_t k = i; k < j; ++k) {
            const double x0 = path.x(k), y0 = path.y(k);
            const double x1 = path.x(k + 1), y1 = path.y(k + 1);
            double seg_len = splash_dist(x0, y0, x1, y1);
            double xa = x0, ya = y0;
            while (seg_len > 0.0) {
                if (dash_dist >= seg_len) {
                    if (dash_on) {
                        if (new_path) {
                            or_path_move_to(out, xa, ya);
                            new_path = false;
                        }
                        or_path_line_to(out, x1, y1);
                    }
                    dash_dist -= seg_len;
                    seg_len = 0.0;
                } else {
                    const double xb = xa + (dash_dist / seg_len) * (x1 - xa);
                    const double yb = ya + (dash_dist / seg_len) * (y1 - ya);
                    if (dash_on) {
                        if (new_path) {
                            or_path_move_to(out, xa, ya);
                            new_path = false;
                        }
                        or_path_line_to(out, xb, yb);
                    }
                    xa = xb;
                    ya = yb;
                    seg_len -= dash_dist;
                    dash_dist = 0.0;
                }
                if (dash_dist <= 0.0) {
                    dash_on = !dash_on;
                    dash_idx += 1;
                    if (dash_idx == n_dash) dash_idx = 0;
                    dash_dist = line_dash[dash_idx];
                    new_path = true;
                }
            }
        }
        i = j + 1;
    }
    if (out->len() == 0 && path.n > 0) {
        bool all_same = true;
        for (size_t k = 0; k + 1 < path.n; ++k)
            if (!(path.x(k) == path.x(k + 1) && path.y(k) == path.y(k + 1))) all_same = false;
        if (all_same) {
            or_path_move_to(out, path.x(0), path.y(0));
            or_path_line_to(out, path.x(0), path.y(0));
        }
    }
}

// advance_past_coincident (stroke/path.rs:723-733).
size_t advance_past_coincident(const PathView& path, size_t start) {
    size_t i = start;
    while (!path.last(i) && i + 1 < path.n && path.x(i + 1) == path.x(i) && path.y(i + 1) == path.y(i)) i += 1;
    return i;
}

// make_stroke_path (stroke/path.rs:250-706) without stroke-adjust hints.
void make_stroke_path(const PathView& path, double w, const or_stroke_params& sp, or_path* out) {
    if (path.n == 0) return;
    size_t subpath_start0 = 0, subpath_start1 = 0;
    bool closed = false;
    size_t i0 = 0;
    size_t i1 = advance_past_coincident(path, i0);
    while (i1 < path.n) {
        const bool first = path.first(i0);
        if (first) {
            subpath_start0 = i0;
            subpath_start1 = i1;
            closed = path.closed(i0);
        }
        (void)subpath_start0;
        const size_t j0 = i1 + 1;
        const size_t j1 = j0 < path.n ? advance_past_coincident(path, j0) : j0;
        if (path.last(i1)) {
            if (first && sp.line_cap == OR_CAP_ROUND) {
                const double cx = path.x(i0), cy = path.y(i0);
                const double r = 0.5 * w;
                const double bc2w = BEZIER_CIRCLE2 * w;
                or_path_move_to(out, cx + r, cy);
                or_path_curve_to(out, cx + r, cy + bc2w, cx + bc2w, cy + r, cx, cy + r);
                or_path_curve_to(out, cx - bc2w, cy + r, cx - r, cy + bc2w, cx - r, cy);
                or_path_curve_to(out, cx - r, cy - bc2w, cx - bc2w, cy - r, cx, cy - r);
                or_path_curve_to(out, cx + bc2w, cy - r, cx + r, cy - bc2w, cx + r, cy);
                or_path_close(out, 0);
            }
            i0 = j0;
            i1 = j1;
            continue;
        }
        const bool last = path.last(j1);
        const size_t k0 = last ? subpath_start1 + 1 : j1 + 1;
        const double seg_dist = splash_dist(path.x(i1), path.y(i1), path.x(j0), path.y(j0));
        if (seg_dist == 0.0) {
            i0 = j0;
            i1 = j1;
            continue;
        }
        const double d = 1.0 / seg_dist;
        const double dx = d * (path.x(j0) - path.x(i1));
        const double dy = d * (path.y(j0) - path.y(i1));
        const double wdx = 0.5 * w * dx;
        const double wdy = 0.5 * w * dy;
        const double ix = path.x(i0), iy = path.y(i0);
        if (or_path_move_to(out, ix - wdy, iy + wdx) != 0) break;
        if (first && !closed) {
            switch (sp.line_cap) {
                case OR_CAP_BUTT:
                    or_path_line_to(out, ix + wdy, iy - wdx);
                    break;
                case OR_CAP_ROUND:
                    or_path_curve_to(out, ix - wdy - BEZIER_CIRCLE * wdx, iy + wdx - BEZIER_CIRCLE * wdy,
                                     ix - wdx - BEZIER_CIRCLE * wdy, iy - wdy + BEZIER_CIRCLE * wdx, ix - wdx,
                                     iy - wdy);
                    or_path_curve_to(out, ix - wdx + BEZIER_CIRCLE * wdy, iy - wdy - BEZIER_CIRCLE * wdx,
                                     ix + wdy - BEZIER_CIRCLE * wdx, iy - wdx - BEZIER_CIRCLE * wdy, ix + wdy,
                                     iy - wdx);
                    break;
                default:  // projecting
                    or_path_line_to(out, ix - wdx - wdy, iy + wdx - wdy);
                    or_path_line_to(out, ix - wdx + wdy, iy - wdx - wdy);
                    or_path_line_to(out, ix + wdy, iy - wdx);
                    break;
            }
        } else {
            or_path_line_to(out, ix + wdy, iy - wdx);
        }
        const double jx = path.x(j0), jy = path.y(j0);
        or_path_line_to(out, jx + wdy, jy - wdx);
        if (last && !closed) {
            switch (sp.line_cap) {
                case OR_CAP_BUTT:
                    or_path_line_to(out, jx - wdy, jy + wdx);
                    break;
                case OR_CAP_ROUND:
                    or_path_curve_to(out, jx + wdy + BEZIER_CIRCLE * wdx, jy - wdx + BEZIER_CIRCLE * wdy,
                                     jx + wdx + BEZIER_CIRCLE * wdy, jy + wdy - BEZIER_CIRCLE * wdx, jx + wdx,
                                     jy + wdy);
                    or_path_curve_to(out, jx + wdx - BEZIER_CIRCLE * wdy, jy + wdy + BEZIER_CIRCLE * wdx,
                                     jx - wdy + BEZIER_CIRCLE * wdx, jy + wdx + BEZIER_CIRCLE * wdy, jx - wdy,
                                     jy + wdx);
                    break;
                default:
                    or_path_line_to(out, jx + wdy + wdx, jy - wdx + wdy);
                    or_path_line_to(out, jx - wdy + wdx, jy + wdx + wdy);
                    or_path_line_to(out, jx - wdy, jy + wdx);
                    break;
            }
        } else {
            or_path_line_to(out, jx - wdy, jy + wdx);
        }
        or_path_close(out, 0);  // close(stroke_adjust = false)
        if (!last || closed) {
            const double dn = 1.0 / splash_dist(path.x(j1), path.y(j1), path.x(k0), path.y(k0));
            const double dx_next = dn * (path.x(k0) - path.x(j1));
            const double dy_next = dn * (path.y(k0) - path.y(j1));
            const double wdx_next = 0.5 * w * dx_next;
            const double wdy_next = 0.5 * w * dy_next;
            const double crossprod = dx * dy_next - dy * dx_next;
            const double dotprod = -(dx * dx_next + dy * dy_next);
            const bool has_angle = crossprod != 0.0 || dx * dx_next < 0.0 || dy * dy_next < 0.0;
            double miter, m;
            if (dotprod > MITER_NEARLY_STRAIGHT) {
                miter = (sp.miter_limit + 1.0) * (sp.miter_limit + 1.0);
                m = 0.0;
            } else {
                miter = std::fmax(2.0 / (1.0 - dotprod), 1.0);
                m = std::sqrt(miter - 1.0);
            }
            if (has_angle && sp.line_join == OR_JOIN_ROUND) {
                if (crossprod < 0.0) {
                    double angle = std::atan2(dx, -dy);
                    const double angle_next = std::atan2(dx_next, -dy_next);
                    if (angle < angle_next) angle = angle + 2.0 * PI_F64;
                    const double d_angle = (angle - angle_next) / PI_F64;
                    if (d_angle < 0.501) {
                        const double kappa = d_angle * BEZIER_CIRCLE * w;
                        const double cx1 = jx - wdy + kappa * dx, cy1 = jy + wdx + kappa * dy;
                        const double cx2 = jx - wdy_next - kappa * dx_next, cy2 = jy + wdx_next - kappa * dy_next;
                        or_path_move_to(out, jx, jy);
                        or_path_line_to(out, jx - wdy_next, jy + wdx_next);
                        or_path_curve_to(out, cx2, cy2, cx1, cy1, jx - wdy, jy + wdx);
                    } else {
                        const double d_join = splash_dist(-wdy, wdx, -wdy_next, wdx_next);
                        if (d_join > 0.0) {
                            const double dx_join = (-wdy_next + wdy) / d_join;
                            const double dy_join = (wdx_next - wdx) / d_join;
                            const double xc = jx + 0.5 * w * std::cos(0.5 * (angle + angle_next));
                            const double yc = jy + 0.5 * w * std::sin(0.5 * (angle + angle_next));
                            const double kappa = d_angle * BEZIER_CIRCLE2 * w;
                            const double cx1 = jx - wdy + kappa * dx, cy1 = jy + wdx + kappa * dy;
                            const double cx2 = xc - kappa * dx_join, cy2 = yc - kappa * dy_join;
                            const double cx3 = xc + kappa * dx_join, cy3 = yc + kappa * dy_join;
                            const double cx4 = jx - wdy_next - kappa * dx_next, cy4 = jy + wdx_next - kappa * dy_next;
                            or_path_move_to(out, jx, jy);
                            or_path_line_to(out, jx - wdy_next, jy + wdx_next);
                            or_path_curve_to(out, cx4, cy4, cx3, cy3, xc, yc);
                            or_path_curve_to(out, cx2, cy2, cx1, cy1, jx - wdy, jy + wdx);
                        }
                    }
                } else {
                    const double angle = std::atan2(-dx, dy);
                    double angle_next = std::atan2(-dx_next, dy_next);
                    if (angle_next < angle) angle_next = angle_next + 2.0 * PI_F64;
                    const double d_angle = (angle_next - angle) / PI_F64;
                    if (d_angle < 0.501) {
                        const double kappa = d_angle * BEZIER_CIRCLE * w;
                        const double cx1 = jx + wdy + kappa * dx, cy1 = jy - wdx + kappa * dy;
                        const double cx2 = jx + wdy_next - kappa * dx_next, cy2 = jy - wdx_next - kappa * dy_next;
                        or_path_move_to(out, jx, jy);
                        or_path_line_to(out, jx + wdy, jy - wdx);
                        or_path_curve_to(out, cx1, cy1, cx2, cy2, jx + wdy_next, jy - wdx_next);
                    } else {
                        const double d_join = splash_dist(wdy, -wdx, wdy_next, -wdx_next);
                        if (d_join > 0.0) {
                            const double dx_join = (wdy_next - wdy) / d_join;
                            const double dy_join = (-wdx_next + wdx) / d_join;
                            const double xc = jx + 0.5 * w * std::cos(0.5 * (angle + angle_next));
                            const double yc = jy + 0.5 * w * std::sin(0.5 * (angle + angle_next));
                            const double kappa = d_angle * BEZIER_CIRCLE2 * w;
                            const double cx1 = jx + wdy + kappa * dx, cy1 = jy - wdx + kappa * dy;
                            const double cx2 = xc - kappa * dx_join, cy2 = yc - kappa * dy_join;
                            const double cx3 = xc + kappa * dx_join, cy3 = yc + kappa * dy_join;
                            const double cx4 = jx + wdy_next - kappa * dx_next, cy4 = jy - wdx_next - kappa * dy_next;
                            or_path_move_to(out, jx, jy);
                            or_path_line_to(out, jx + wdy, jy - wdx);
                            or_path_curve_to(out, cx1, cy1, cx2, cy2, xc, yc);
                            or_path_curve_to(out, cx3, cy3, cx4, cy4, jx + wdy_next, jy - wdx_next);
                        }
                    }
                }
            } else if (has_angle) {
                or_path_move_to(out, jx, jy);
                if (crossprod < 0.0) {
                    or_path_line_to(out, jx - wdy_next, jy + wdx_next);
                    if (sp.line_join == OR_JOIN_MITER && std::sqrt(miter) <= sp.miter_limit)
                        or_path_line_to(out, jx - wdy + wdx * m, jy + wdx + wdy * m);
                    or_path_line_to(out, jx - wdy, jy + wdx);
                } else {
                    or_path_line_to(out, jx + wdy, jy - wdx);
                    if (sp.line_join == OR_JOIN_MITER && std::sqrt(miter) <= sp.miter_limit)
                        or_path_line_to(out, jx + wdy + wdx * m, jy - wdx + wdy * m);
                    or_path_line_to(out, jx + wdy_next, jy - wdx_next);
                }
            }
            or_path_close(out, 0);
        }
        i0 = j0;
        i1 = j1;
    }
}

// The path stroke() fills or draws: flattened, then dashed when a dash array
// is set (stroke/mod.rs:67-78). Returns false when nothing is to be drawn.
bool stroke_polyline(const PathView& in, const or_stroke_params& sp, double flatness, or_path* out) {
    if (in.n == 0) return false;
    or_path flat;
    flatten_path(in, flatness, &flat);
    if (sp.n_dash > 0) {
        make_dashed_path(view_of(flat), sp.dash, static_cast<size_t>(sp.n_dash), sp.dash_phase, out);
        return out->len() != 0;
    }
    *out = flat;
    return true;
}

// stroke_narrow (stroke/mod.rs:95-170) + draw_narrow_span (:204-256): spans
// (y, x0, x1) handed to `span` already clamped and clipped. The clip is the
// page, or the page and a clip rectangle (rect clips have no path scanners, so
// Clip::test inside the integer bounds is true).
template <typename SpanFn>
void stroke_narrow_impl(int32_t width, int32_t height, const or_path& path, const double m[6], double flatness,
                        const double* clip_rect, SpanFn span) {
    const int64_t need = or_xpath_new(path.pts.data(), path.flags.data(), static_cast<int64_t>(path.len()), m,
                                      flatness, 0, nullptr, 0);
    std::vector<or_seg> segs(static_cast<size_t>(need));
    or_xpath_new(path.pts.data(), path.flags.data(), static_cast<int64_t>(path.len()), m, flatness, 0, segs.data(),
                 need);
    const ClipRect clip = make_clip(width, height, clip_rect);
    auto draw = [&](int32_t x0, int32_t x1, int32_t y, bool all_inside) {
        if (y < 0 || y >= height) return;
        int32_t sx0, sx1;
        if (all_inside) {
            sx0 = std::max(x0, 0);
            sx1 = std::min(x1, width - 1);
        } else {
            sx0 = std::max(x0, clip.x_min_i);
            sx1 = std::min(x1, clip.x_max_i);
        }
        if (sx0 > sx1) return;
        if (!all_inside && (y < clip.y_min_i || y > clip.y_max_i)) return;  // Clip::test fails on every pixel
        span(y, sx0, sx1);
    };
    for (const or_seg& seg : segs) {
        double sx0, sy0, sx1, sy1;
        if (seg.y0 <= seg.y1) {
            sx0 = seg.x0; sy0 = seg.y0; sx1 = seg.x1; sy1 = seg.y1;
        } else {
            sx0 = seg.x1; sy0 = seg.y1; sx1 = seg.x0; sy1 = seg.y0;
        }
        const int32_t y0 = splash_floor(sy0), y1 = splash_floor(sy1);
        const int32_t x0 = splash_floor(sx0), x1 = splash_floor(sx1);
        const int32_t xl = std::min(x0, x1), xr = std::max(x0, x1);
        // Clip::test_rect (clip.rs:196-215), right + 1 / bottom + 1 in i32 as the reference computes them.
        const double r1 = static_cast<double>(static_cast<int32_t>(static_cast<uint32_t>(xr) + 1u));
        const double b1 = static_cast<double>(static_cast<int32_t>(static_cast<uint32_t>(y1) + 1u));
        if (r1 <= clip.x_min || static_cast<double>(xl) >= clip.x_max || b1 <= clip.y_min ||
            static_cast<double>(y0) >= clip.y_max)
            continue;
        const bool all_inside = static_cast<double>(xl) >= clip.x_min && r1 <= clip.x_max &&
                                static_cast<double>(y0) >= clip.y_min && b1 <= clip.y_max;
        if (y0 == y1) {
            draw(xl, xr, y0, all_inside);
            continue;
        }
        const double dxdy = seg.dxdy;
        int32_t cy0 = y0, cx0 = x0, cy1 = y1, cx1 = x1;
        if (cy0 < clip.y_min_i) {
            cy0 = clip.y_min_i;
            cx0 = splash_floor(std::fma(clip.y_min - sy0, dxdy, sx0));
        }
        if (cy1 > clip.y_max_i) {
            cy1 = clip.y_max_i;
            cx1 = splash_floor(std::fma(clip.y_max - sy0, dxdy, sx0));
        }
        int32_t xa = cx0;
        const bool left_to_right = cx0 <= cx1;
        for (int32_t y = cy0; y <= cy1; ++y) {
            int32_t xb;
            if (y < cy1) xb = splash_floor(std::fma(static_cast<double>(y) + 1.0 - sy0, dxdy, sx0));
            else xb = left_to_right ? cx1 + 1 : cx1 - 1;
            int32_t a, b;
            if (left_to_right) {
                a = xa;
                b = xa == xb ? xa : xb - 1;
            } else if (xa == xb) {
                a = b = xa;
            } else {
                a = xb + 1;
                b = xa;
            }
            draw(a, b, y, all_inside);
            xa = xb;
        }
    }
}

// One painting operator of a scene: a fill (rule as given) or a stroke.
template <typename AaSpan, typename SolidSpan>
void paint_path(int32_t W, int32_t H, const double* pts, const uint8_t* flags, int64_t n, const double m[6],
                double flatness, int eo, int rowmap, or_stats* st, const or_stroke_params* sp, const double* clip,
                AaSpan aa_span, SolidSpan solid_span) {
    if (!sp || !sp->stroke) {
        fill_path_impl(W, H, pts, flags, n, m, flatness, eo, rowmap, st, aa_span, clip);
        return;
    }
    or_path poly;
    if (!stroke_polyline(PathView{pts, flags, static_cast<size_t>(n)}, *sp, flatness, &poly)) return;
    if (sp->line_width == 0.0) {
        stroke_narrow_impl(W, H, poly, m, flatness, clip, solid_span);
        return;
    }
    or_path outline;
    make_stroke_path(view_of(poly), sp->line_width, *sp, &outline);
    fill_path_impl(W, H, outline.pts.data(), outline.flags.data(), static_cast<int64_t>(outline.len()), m, flatness,
                   0, rowmap, st, aa_span, clip);
}

// Pages of a scene on up to n_threads workers; rgb == nullptr: Gray8 pages
// and gray[] sources, else Rgb8 pages (3 bytes per pixel) and rgb[3 * p].
void render_scene_impl(uint8_t* arena, const uint64_t* page_off, const uint32_t* page_w,
                       const uint32_t* page_h, uint32_t n_pages, const double* pts,
                       const uint8_t* flags, const uint64_t* path_pt_off, const uint8_t* rule,
                       const uint8_t* gray, const uint8_t* rgb, const uint8_t* alpha, const uint32_t* path_page,
                       uint64_t n_paths, const double m[6], double flatness, int rowmap,
                       int n_threads, or_stats* st, const double* clip = nullptr,
                       const or_stroke_params* sp = nullptr);

}  // namespace

extern "C" {

void or_fill_path(uint8_t* page, int32_t width, int32_t height, const double* pts,
                  const uint8_t* flags, int64_t n_pts, const double m[6], double flatness, int eo,
                  uint8_t gray, uint8_t alpha, int rowmap, or_stats* st) {
    fill_path_impl(width, height, pts, flags, n_pts, m, flatness, eo, rowmap, st,
                   [&](int32_t y, int32_t x0, const uint8_t* shape, int64_t n) {
                       or_render_span_aa_gray(page + static_cast<int64_t>(y) * width + x0, shape, n, alpha, gray);
                   });
}

void or_fill_path_clip_paths(uint8_t* page, int32_t width, int32_t height, const double* pts, const uint8_t* flags,
                             int64_t n_pts, const double m[6], double flatness, int eo, uint8_t gray, uint8_t alpha,
                             int rowmap, const double* clip_rect, int64_t n_clips, const double* const* clip_pts,
                             const uint8_t* const* clip_flags, const int64_t* clip_n, const int* clip_eo,
                             or_stats* st) {
    ClipState cs;
    cs.r = make_clip(width, height, clip_rect);
    for (int64_t k = 0; k < n_clips; ++k) clip_to_path(cs, clip_pts[k], clip_flags[k], clip_n[k], m, flatness, clip_eo[k], st);
    fill_path_impl(width, height, pts, flags, n_pts, m, flatness, eo, rowmap, st,
                   [&](int32_t y, int32_t x0, const uint8_t* shape, int64_t n) {
                       or_render_span_aa_gray(page + static_cast<int64_t>(y) * width + x0, shape, n, alpha, gray);
                   },
                   nullptr, &cs);
}

void or_fill_path_clip_path(uint8_t* page, int32_t width, int32_t height, const double* pts, const uint8_t* flags,
                            int64_t n_pts, const double m[6], double flatness, int eo, uint8_t gray, uint8_t alpha,
                            int rowmap, const double* clip_rect, const double* clip_pts, const uint8_t* clip_flags,
                            int64_t clip_n, int clip_eo, or_stats* st) {
    or_fill_path_clip_paths(page, width, height, pts, flags, n_pts, m, flatness, eo, gray, alpha, rowmap, clip_rect, 1,
                            &clip_pts, &clip_flags, &clip_n, &clip_eo, st);
}

void or_fill_path_rgb(uint8_t* page_rgb, int32_t width, int32_t height, const double* pts, const uint8_t* flags,
                      int64_t n_pts, const double m[6], double flatness, int eo, const uint8_t rgb[3], uint8_t alpha,
                      int rowmap, or_stats* st) {
    fill_path_impl(width, height, pts, flags, n_pts, m, flatness, eo, rowmap, st,
                   [&](int32_t y, int32_t x0, const uint8_t* shape, int64_t n) {
                       or_composite_aa_rgb8_opaque(page_rgb + 3 * (static_cast<int64_t>(y) * width + x0), rgb, alpha,
                                                   shape, n);
                   });
}

void or_render_scene(uint8_t* arena, const uint64_t* page_off, const uint32_t* page_w,
                     const uint32_t* page_h, uint32_t n_pages, const double* pts,
                     const uint8_t* flags, const uint64_t* path_pt_off, const uint8_t* rule,
                     const uint8_t* gray, const uint8_t* alpha, const uint32_t* path_page,
                     uint64_t n_paths, const double m[6], double flatness, int rowmap,
                     int n_threads, or_stats* st) {
    render_scene_impl(arena, page_off, page_w, page_h, n_pages, pts, flags, path_pt_off, rule, gray, nullptr, alpha,
                      path_page, n_paths, m, flatness, rowmap, n_threads, st);
}

void or_render_scene_ex(uint8_t* arena, const uint64_t* page_off, const uint32_t* page_w, const uint32_t* page_h,
                        uint32_t n_pages, const double* pts, const uint8_t* flags, const uint64_t* path_pt_off,
                        const uint8_t* rule, const uint8_t* gray, const uint8_t* rgb, const uint8_t* alpha,
                        const uint32_t* path_page, uint64_t n_paths, const double* clip, const double m[6],
                        double flatness, int rowmap, int n_threads, or_stats* st) {
    render_scene_impl(arena, page_off, page_w, page_h, n_pages, pts, flags, path_pt_off, rule, gray, rgb, alpha,
                      path_page, n_paths, m, flatness, rowmap, n_threads, st, clip);
}

void or_render_scene_paint(uint8_t* arena, const uint64_t* page_off, const uint32_t* page_w, const uint32_t* page_h,
                           uint32_t n_pages, const double* pts, const uint8_t* flags, const uint64_t* path_pt_off,
                           const uint8_t* rule, const uint8_t* gray, const uint8_t* rgb, const uint8_t* alpha,
                           const uint32_t* path_page, uint64_t n_paths, const double* clip,
                           const or_stroke_params* stroke, const double m[6], double flatness, int rowmap,
                           int n_threads, or_stats* st) {
    render_scene_impl(arena, page_off, page_w, page_h, n_pages, pts, flags, path_pt_off, rule, gray, rgb, alpha,
                      path_page, n_paths, m, flatness, rowmap, n_threads, st, clip, stroke);
}

int or_stroke_outline(const double* pts, const uint8_t* flags, int64_t n, const or_stroke_params* sp,
                      double flatness, or_path* out) {
    or_path poly;
    if (!sp || !stroke_polyline(PathView{pts, flags, static_cast<size_t>(n)}, *sp, flatness, &poly)) return 0;
    if (sp->line_width == 0.0) {
        *out = poly;
        return 2;
    }
    make_stroke_path(view_of(poly), sp->line_width, *sp, out);
    return out->len() ? 1 : 0;
}

int or_stroke_flatten(const double* pts, const uint8_t* flags, int64_t n, double flatness, or_path* out) {
    flatten_path(PathView{pts, flags, static_cast<size_t>(n)}, flatness, out);
    return 0;
}

int or_stroke_dash(const double* pts, const uint8_t* flags, int64_t n, const double* dash, int32_t n_dash,
                   double phase, or_path* out) {
    make_dashed_path(PathView{pts, flags, static_cast<size_t>(n)}, dash, static_cast<size_t>(std::max(n_dash, 0)),
                     phase, out);
    return 0;
}

void or_render_scene_rgb(uint8_t* arena, const uint64_t* page_off, const uint32_t* page_w, const uint32_t* page_h,
                         uint32_t n_pages, const double* pts, const uint8_t* flags, const uint64_t* path_pt_off,
                         const uint8_t* rule, const uint8_t* rgb, const uint8_t* alpha, const uint32_t* path_page,
                         uint64_t n_paths, const double m[6], double flatness, int rowmap, int n_threads,
                         or_stats* st) {
    render_scene_impl(arena, page_off, page_w, page_h, n_pages, pts, flags, path_pt_off, rule, nullptr, rgb, alpha,
                      path_page, n_paths, m, flatness, rowmap, n_threads, st);
}

}  // extern "C"

namespace {

void render_scene_impl(uint8_t* arena, const uint64_t* page_off, const uint32_t* page_w,
                       const uint32_t* page_h, uint32_t n_pages, const double* pts,
                       const uint8_t* flags, const uint64_t* path_pt_off, const uint8_t* rule,
                       const uint8_t* gray, const uint8_t* rgb, const uint8_t* alpha, const uint32_t* path_page,
                       uint64_t n_paths, const double m[6], double flatness, int rowmap,
                       int n_threads, or_stats* st, const double* clip, const or_stroke_params* sp) {
    // Paths of each page, in scene order.
    std::vector<std::vector<uint64_t>> per_page(n_pages);
    for (uint64_t p = 0; p < n_paths; ++p)
        if (path_page[p] < n_pages) per_page[path_page[p]].push_back(p);
    std::atomic<uint32_t> next{0};
    std::vector<or_stats> stats(static_cast<size_t>(std::max(n_threads, 1)));
    auto worker = [&](int t) {
        or_stats& ls = stats[static_cast<size_t>(t)];
        std::memset(&ls, 0, sizeof ls);
        for (;;) {
            uint32_t pg = next.fetch_add(1);
            if (pg >= n_pages) break;
            uint8_t* page = arena + page_off[pg];
            for (uint64_t p : per_page[pg]) {
                uint64_t a = path_pt_off[p], b = path_pt_off[p + 1];
                const int32_t W = static_cast<int32_t>(page_w[pg]), H = static_cast<int32_t>(page_h[pg]);
                const double* cp = clip ? clip + 4 * p : nullptr;
                const or_stroke_params* psp = sp ? sp + p : nullptr;
                const uint8_t a_in = alpha[p];
                if (rgb) {
                    const uint8_t* src = rgb + 3 * p;
                    paint_path(W, H, pts + 2 * a, flags + a, static_cast<int64_t>(b - a), m, flatness, rule[p] != 0,
                               rowmap, &ls, psp, cp,
                               [&](int32_t y, int32_t x0, const uint8_t* shape, int64_t n) {
                                   or_composite_aa_rgb8_opaque(page + 3 * (static_cast<int64_t>(y) * W + x0), src, a_in,
                                                               shape, n);
                               },
                               [&](int32_t y, int32_t x0, int32_t x1) {
                                   // render_span without shape: simple copy at alpha 255, else
                                   // the general arm's div255 per channel (pipe/general.rs:261-312).
                                   uint8_t* d = page + 3 * (static_cast<int64_t>(y) * W + x0);
                                   for (int64_t i = 0; i < 3 * (static_cast<int64_t>(x1) - x0 + 1); ++i)
                                       d[i] = or_div255((255u - a_in) * d[i] + a_in * src[i % 3]);
                               });
                } else {
                    const uint8_t g = gray[p];
                    paint_path(W, H, pts + 2 * a, flags + a, static_cast<int64_t>(b - a), m, flatness, rule[p] != 0,
                               rowmap, &ls, psp, cp,
                               [&](int32_t y, int32_t x0, const uint8_t* shape, int64_t n) {
                                   or_render_span_aa_gray(page + static_cast<int64_t>(y) * W + x0, shape, n, a_in, g);
                               },
                               [&](int32_t y, int32_t x0, int32_t x1) {
                                   uint8_t* d = page + static_cast<int64_t>(y) * W;
                                   for (int32_t x = x0; x <= x1; ++x) d[x] = or_div255((255u - a_in) * d[x] + a_in * g);
                               });
                }
            }
        }
    };
    int nt = std::max(1, std::min<int>(n_threads, static_cast<int>(n_pages)));
    if (nt == 1) {
        worker(0);
    } else {
        std::vector<std::thread> th;
        for (int t = 0; t < nt; ++t) th.emplace_back(worker, t);
        for (auto& x : th) x.join();
    }
    if (st) {
        for (int t = 0; t < nt; ++t) {
            st->paths += stats[t].paths;
            st->segments += stats[t].segments;
            st->aa_rows += stats[t].aa_rows;
            st->intersects += stats[t].intersects;
            st->unpinned_tie_rows += stats[t].unpinned_tie_rows;
            st->nonterminating_rows += stats[t].nonterminating_rows;
        }
    }
}

}  // namespace
