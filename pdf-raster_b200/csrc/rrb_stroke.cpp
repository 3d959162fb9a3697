// rrb_stroke.cpp — stroke outlines on the host (the reference's stroke(),
// crates/raster/src/stroke/mod.rs:58-89 and stroke/path.rs:40-745).
//
// A stroke becomes geometry the device pipeline already renders: an outline
// path filled nonzero with AA (line width > 0, stroke_wide) or the polyline
// whose one-pixel spans stroke_narrow draws (line width 0). The outline is
// built here on the host because its points come from libm: every segment's
// length is f64::hypot and round joins use atan2 / cos / sin, and the last
// bit of each feeds the fill. Calling the same libm functions as the
// reference's Rust (which binds the platform libm) gives the same points;
// CUDA's device versions differ from them in the last place.
//
// Paths are independent, so a batch's paths are stroked in parallel: worker
// threads take chunks of consecutive paths, each writes its chunk's geometry
// into its own buffers (reused across paths, no per-path allocation), and the
// chunks are concatenated in path order.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <string>
#include <thread>
#include <vector>

#include "../../include/rrb.h"
#include "rrb_stroke.h"

namespace {

constexpr int kMaxSplits = 1024;                 // MAX_CURVE_SPLITS (types.rs:36)
constexpr double kBezierCircle = 0.55228475;     // BEZIER_CIRCLE (types.rs:45)
constexpr double kBezierCircle2 = 0.5 * kBezierCircle;
constexpr double kMiterNearlyStraight = 0.9999;  // stroke/path.rs:22
constexpr double kPi = 3.141592653589793;        // std::f64::consts::PI

// f64 -> i32 as splash_floor (color/src/convert.rs:221-240): floor, then
// saturate (NaN -> i32::MIN through the non-finite arm).
int32_t floor_i32(double x) {
    const double f = std::floor(x);
    if (!(f >= -2147483648.0)) return f > 0 ? INT32_MAX : INT32_MIN;
    if (f >= 2147483647.0) return INT32_MAX;
    return static_cast<int32_t>(f);
}

double seg_len(double x0, double y0, double x1, double y1) { return std::hypot(x1 - x0, y1 - y0); }

// Point list with PathBuilder's rules (path/mod.rs:310-448): move_to fails on
// a one-point subpath, line_to / curve_to / close fail without a current
// point, close appends lineTo(first) unless the subpath is one point or
// already ends on its first point, and marks both ends CLOSED.
struct Sink {
    std::vector<double>* xy;
    std::vector<uint8_t>* fl;
    size_t base = 0;   // this path's first point in xy / fl
    size_t start = 0;  // current subpath's first point (relative); == size(): no current point

    size_t size() const { return fl->size() - base; }
    bool no_point() const { return start == size(); }
    void push(double x, double y, uint8_t f) {
        xy->push_back(x);
        xy->push_back(y);
        fl->push_back(f);
    }
    bool move(double x, double y) {
        if (size() != 0 && start == size() - 1) return false;
        start = size();
        push(x, y, RRB_PATH_FIRST | RRB_PATH_LAST);
        return true;
    }
    bool line(double x, double y) {
        if (no_point()) return false;
        fl->back() &= static_cast<uint8_t>(~RRB_PATH_LAST);
        push(x, y, RRB_PATH_LAST);
        return true;
    }
    bool curve(double x1, double y1, double x2, double y2, double x3, double y3) {
        if (no_point()) return false;
        fl->back() &= static_cast<uint8_t>(~RRB_PATH_LAST);
        push(x1, y1, RRB_PATH_CURVE);
        push(x2, y2, RRB_PATH_CURVE);
        push(x3, y3, RRB_PATH_LAST);
        return true;
    }
    bool close() {
        if (no_point()) return false;
        const size_t s = base + start, e = fl->size() - 1;
        const double fx = (*xy)[2 * s], fy = (*xy)[2 * s + 1];
        if (s != e && !((*xy)[2 * e] == fx && (*xy)[2 * e + 1] == fy)) line(fx, fy);
        (*fl)[s] |= RRB_PATH_CLOSED;
        fl->back() |= RRB_PATH_CLOSED;
        start = size();
        return true;
    }
};

struct Pts {
    const double* xy;
    const uint8_t* fl;
    size_t n;
    double x(size_t i) const { return xy[2 * i]; }
    double y(size_t i) const { return xy[2 * i + 1]; }
    bool has(size_t i, uint8_t f) const { return (fl[i] & f) != 0; }
};

// flatten_curve (path/flatten.rs:109-215): the reference's subdivision on the
// interval [0, kMaxSplits], kept as a stack of pending right halves instead of
// slot arrays (each half is (start, c1, c2, interval end); its end point is
// the start of the half below it, or p3). Same midpoints in the same order.
double mid(double a, double b) {
    // f64::midpoint: (a + b) / 2 when both magnitudes are at most f64::MAX / 2.
    const double hi = 8.98846567431157854e+307, lo = 2.0 * std::numeric_limits<double>::min();
    const double aa = std::fabs(a), ab = std::fabs(b);
    if (aa <= hi && ab <= hi) return (a + b) / 2.0;
    if (aa < lo) return a + (b / 2.0);
    if (ab < lo) return (a / 2.0) + b;
    return (a / 2.0) + (b / 2.0);
}

template <typename Emit>
void flatten_curve(const double c[8], double flat_sq, Emit emit) {
    struct Half {
        double x0, y0, x1, y1, x2, y2;
        int end;
    };
    Half stack[11];
    int top = 0;
    double ax = c[0], ay = c[1], bx = c[2], by = c[3], cx = c[4], cy = c[5];
    int lo = 0;
    while (lo < kMaxSplits) {
        const int hi = top ? stack[top - 1].end : kMaxSplits;
        const double ex = top ? stack[top - 1].x0 : c[6], ey = top ? stack[top - 1].y0 : c[7];
        const double mx = mid(ax, ex), my = mid(ay, ey);
        const double d1x = bx - mx, d1y = by - my, d2x = cx - mx, d2y = cy - my;
        const double d1 = std::fma(d1x, d1x, d1y * d1y), d2 = std::fma(d2x, d2x, d2y * d2y);
        if (hi - lo == 1 || (d1 <= flat_sq && d2 <= flat_sq)) {
            emit(ex, ey);
            lo = hi;
            if (top) {
                --top;
                ax = stack[top].x0;
                ay = stack[top].y0;
                bx = stack[top].x1;
                by = stack[top].y1;
                cx = stack[top].x2;
                cy = stack[top].y2;
            }
        } else {
            const double l1x = mid(ax, bx), l1y = mid(ay, by);
            const double hx = mid(bx, cx), hy = mid(by, cy);
            const double l2x = mid(l1x, hx), l2y = mid(l1y, hy);
            const double r2x = mid(cx, ex), r2y = mid(cy, ey);
            const double r1x = mid(hx, r2x), r1y = mid(hy, r2y);
            const double r0x = mid(l2x, r1x), r0y = mid(l2y, r1y);
            // The half [ (lo+hi)/2, hi ] waits; the loop continues on [lo, (lo+hi)/2].
            stack[top++] = Half{r0x, r0y, r1x, r1y, r2x, r2y, (lo + hi) / 2};
            bx = l1x;
            by = l1y;
            cx = l2x;
            cy = l2y;
        }
    }
}

// flatten_path (stroke/path.rs:40-86): curves flattened in user space
// against flatness^2; builder refusals are dropped as the reference drops them.
void flatten_path(const Pts& in, double flatness, Sink& out) {
    const double flat_sq = flatness * flatness;
    size_t i = 0;
    while (i < in.n) {
        if (in.has(i, RRB_PATH_FIRST)) {
            out.move(in.x(i), in.y(i));
            ++i;
            continue;
        }
        if (in.has(i, RRB_PATH_CURVE)) {
            if (i == 0 || i + 2 >= in.n) break;  // malformed curve: the reference would index out of range
            const double c[8] = {in.x(i - 1), in.y(i - 1), in.x(i), in.y(i), in.x(i + 1), in.y(i + 1), in.x(i + 2),
                                 in.y(i + 2)};
            flatten_curve(c, flat_sq, [&](double x, double y) { out.line(x, y); });
            i += 3;
        } else {
            out.line(in.x(i), in.y(i));
            ++i;
        }
        if (in.has(i - 1, RRB_PATH_CLOSED)) out.close();
    }
}

// make_dashed_path (stroke/path.rs:107-220).
void dash_path(const Pts& in, const double* dash, size_t nd, double phase0, Sink& out) {
    double total = 0.0;
    for (size_t k = 0; k < nd; ++k) total += dash[k];
    if (nd == 0 || total < std::numeric_limits<double>::epsilon()) return;
    double phase = phase0;
    phase -= static_cast<double>(floor_i32(phase / total)) * total;
    bool on0 = true;
    size_t idx0 = 0;
    if (phase > 0.0) {
        while (idx0 < nd && phase >= dash[idx0]) {
            on0 = !on0;
            phase -= dash[idx0];
            ++idx0;
        }
        if (idx0 == nd) return;
    }
    const size_t mark = out.size();
    size_t i = 0;
    while (i < in.n) {
        size_t j = i;
        while (j + 1 < in.n && !in.has(j, RRB_PATH_LAST)) ++j;
        bool on = on0;
        size_t idx = idx0;
        double left = dash[idx] - phase;  // distance to the end of the current dash entry
        bool open = true;                 // the next "on" piece starts a new subpath
        for (size_t k = i; k < j; ++k) {
            const double x1 = in.x(k + 1), y1 = in.y(k + 1);
            double xa = in.x(k), ya = in.y(k);
            double len = seg_len(xa, ya, x1, y1);
            while (len > 0.0) {
                if (left >= len) {
                    if (on) {
                        if (open) out.move(xa, ya);
                        open = false;
                        out.line(x1, y1);
                    }
                    left -= len;
                    len = 0.0;
                } else {
                    const double xb = xa + (left / len) * (x1 - xa);
                    const double yb = ya + (left / len) * (y1 - ya);
                    if (on) {
                        if (open) out.move(xa, ya);
                        open = false;
                        out.line(xb, yb);
                    }
                    xa = xb;
                    ya = yb;
                    len -= left;
                    left = 0.0;
                }
                if (left <= 0.0) {
                    on = !on;
                    idx = idx + 1 == nd ? 0 : idx + 1;
                    left = dash[idx];
                    open = true;
                }
            }
        }
        i = j + 1;
    }
    if (out.size() == mark && in.n > 0) {
        // Nothing drawn and every point the same: a zero-length dash keeps the caps (Acrobat).
        bool same = true;
        for (size_t k = 0; k + 1 < in.n && same; ++k) same = in.x(k) == in.x(k + 1) && in.y(k) == in.y(k + 1);
        if (same) {
            out.move(in.x(0), in.y(0));
            out.line(in.x(0), in.y(0));
        }
    }
}

// advance_past_coincident (stroke/path.rs:723-733).
size_t skip_same(const Pts& p, size_t i) {
    while (!p.has(i, RRB_PATH_LAST) && i + 1 < p.n && p.x(i + 1) == p.x(i) && p.y(i + 1) == p.y(i)) ++i;
    return i;
}

// Round join arcs (stroke/path.rs:461-584) at vertex (jx, jy) between the
// segment with unit direction (dx, dy) and the next one (nx, ny). The join
// takes each direction's angle as atan2(x, -y) on a left turn (kind 1) or
// atan2(-x, y) otherwise (kind 0). a_kind / a_val: the current segment's
// angle when the previous join already took it in this join's kind (-1:
// none); an_kind / an_val receive the next segment's, for the next join.
void round_join(Sink& out, double jx, double jy, double w, double dx, double dy, double wdx, double wdy, double nx,
                double ny, double wnx, double wny, double cross, int a_kind, double a_val, int& an_kind,
                double& an_val) {
    if (cross < 0.0) {
        double a = a_kind == 1 ? a_val : std::atan2(dx, -dy);
        const double an = std::atan2(nx, -ny);
        an_kind = 1;
        an_val = an;
        if (a < an) a = a + 2.0 * kPi;
        const double da = (a - an) / kPi;
        if (da < 0.501) {
            const double kappa = da * kBezierCircle * w;
            out.move(jx, jy);
            out.line(jx - wny, jy + wnx);
            out.curve(jx - wny - kappa * nx, jy + wnx - kappa * ny, jx - wdy + kappa * dx, jy + wdx + kappa * dy,
                      jx - wdy, jy + wdx);
            return;
        }
        const double dj = seg_len(-wdy, wdx, -wny, wnx);
        if (!(dj > 0.0)) return;
        const double djx = (-wny + wdy) / dj, djy = (wnx - wdx) / dj;
        const double xc = jx + 0.5 * w * std::cos(0.5 * (a + an));
        const double yc = jy + 0.5 * w * std::sin(0.5 * (a + an));
        const double kappa = da * kBezierCircle2 * w;
        out.move(jx, jy);
        out.line(jx - wny, jy + wnx);
        out.curve(jx - wny - kappa * nx, jy + wnx - kappa * ny, xc + kappa * djx, yc + kappa * djy, xc, yc);
        out.curve(xc - kappa * djx, yc - kappa * djy, jx - wdy + kappa * dx, jy + wdx + kappa * dy, jx - wdy,
                  jy + wdx);
        return;
    }
    const double a = a_kind == 0 ? a_val : std::atan2(-dx, dy);
    double an = std::atan2(-nx, ny);
    an_kind = 0;
    an_val = an;
    if (an < a) an = an + 2.0 * kPi;
    const double da = (an - a) / kPi;
    if (da < 0.501) {
        const double kappa = da * kBezierCircle * w;
        out.move(jx, jy);
        out.line(jx + wdy, jy - wdx);
        out.curve(jx + wdy + kappa * dx, jy - wdx + kappa * dy, jx + wny - kappa * nx, jy - wnx - kappa * ny,
                  jx + wny, jy - wnx);
        return;
    }
    const double dj = seg_len(wdy, -wdx, wny, -wnx);
    if (!(dj > 0.0)) return;
    const double djx = (wny - wdy) / dj, djy = (-wnx + wdx) / dj;
    const double xc = jx + 0.5 * w * std::cos(0.5 * (a + an));
    const double yc = jy + 0.5 * w * std::sin(0.5 * (a + an));
    const double kappa = da * kBezierCircle2 * w;
    out.move(jx, jy);
    out.line(jx + wdy, jy - wdx);
    out.curve(jx + wdy + kappa * dx, jy - wdx + kappa * dy, xc - kappa * djx, yc - kappa * djy, xc, yc);
    out.curve(xc + kappa * djx, yc + kappa * djy, jx + wny - kappa * nx, jy - wnx - kappa * ny, jx + wny, jy - wnx);
}

// Start cap at (x, y) (stroke/path.rs:354-383): from the left side
// (x - wdy, y + wdx), already moved to, round to the right side (x + wdy, y - wdx).
void start_cap(Sink& out, int kind, double x, double y, double wdx, double wdy) {
    if (kind == RRB_CAP_ROUND) {
        out.curve(x - wdy - kBezierCircle * wdx, y + wdx - kBezierCircle * wdy, x - wdx - kBezierCircle * wdy,
                  y - wdy + kBezierCircle * wdx, x - wdx, y - wdy);
        out.curve(x - wdx + kBezierCircle * wdy, y - wdy - kBezierCircle * wdx, x + wdy - kBezierCircle * wdx,
                  y - wdx - kBezierCircle * wdy, x + wdy, y - wdx);
    } else if (kind == RRB_CAP_PROJECTING) {
        out.line(x - wdx - wdy, y + wdx - wdy);
        out.line(x - wdx + wdy, y - wdx - wdy);
        out.line(x + wdy, y - wdx);
    } else {
        out.line(x + wdy, y - wdx);
    }
}

// End cap at (x, y) (stroke/path.rs:394-422): from the right side back to the
// left side (x - wdy, y + wdx). The sums are written in the reference's order
// (floating-point addition does not reassociate).
void end_cap(Sink& out, int kind, double x, double y, double wdx, double wdy) {
    if (kind == RRB_CAP_ROUND) {
        out.curve(x + wdy + kBezierCircle * wdx, y - wdx + kBezierCircle * wdy, x + wdx + kBezierCircle * wdy,
                  y + wdy - kBezierCircle * wdx, x + wdx, y + wdy);
        out.curve(x + wdx - kBezierCircle * wdy, y + wdy + kBezierCircle * wdx, x - wdy + kBezierCircle * wdx,
                  y + wdx + kBezierCircle * wdy, x - wdy, y + wdx);
    } else if (kind == RRB_CAP_PROJECTING) {
        out.line(x + wdy + wdx, y - wdx + wdy);
        out.line(x - wdy + wdx, y + wdx + wdy);
        out.line(x - wdy, y + wdx);
    } else {
        out.line(x - wdy, y + wdx);
    }
}

// make_stroke_path (stroke/path.rs:250-706), without stroke-adjust hints.
// Every segment becomes a closed quadrilateral (with its caps at open
// subpath ends), every interior vertex (and the closing vertex of a closed
// subpath) a closed join piece; the nonzero fill of their union is the stroke.
void outline_path(const Pts& p, double w, const rrb_stroke_params& sp, Sink& out) {
    if (p.n == 0) return;
    // The segment a join turns into is the next iteration's segment: its
    // length (hypot) and, after a round join, its angle (atan2) are kept,
    // keyed by the segment's end-point indices, so a reuse is the same libm
    // call on the same points.
    struct {
        size_t a = SIZE_MAX, b = SIZE_MAX;
        double len = 0.0;
        int ang_kind = -1;
        double ang = 0.0;
    } next;
    size_t sub1 = 0;
    bool closed = false;
    size_t i0 = 0, i1 = skip_same(p, 0);
    while (i1 < p.n) {
        const bool first = p.has(i0, RRB_PATH_FIRST);
        if (first) {
            sub1 = i1;
            closed = p.has(i0, RRB_PATH_CLOSED);
        }
        const size_t j0 = i1 + 1;
        const size_t j1 = j0 < p.n ? skip_same(p, j0) : j0;
        if (p.has(i1, RRB_PATH_LAST)) {
            // Zero-length subpath: only a round cap draws (a circle).
            if (first && sp.line_cap == RRB_CAP_ROUND) {
                const double cx = p.x(i0), cy = p.y(i0), r = 0.5 * w, k = kBezierCircle2 * w;
                out.move(cx + r, cy);
                out.curve(cx + r, cy + k, cx + k, cy + r, cx, cy + r);
                out.curve(cx - k, cy + r, cx - r, cy + k, cx - r, cy);
                out.curve(cx - r, cy - k, cx - k, cy - r, cx, cy - r);
                out.curve(cx + k, cy - r, cx + r, cy - k, cx + r, cy);
                out.close();
            }
            i0 = j0;
            i1 = j1;
            continue;
        }
        const bool last = p.has(j1, RRB_PATH_LAST);
        const size_t k0 = last ? sub1 + 1 : j1 + 1;
        const bool known = next.a == i1 && next.b == j0;
        const double len = known ? next.len : seg_len(p.x(i1), p.y(i1), p.x(j0), p.y(j0));
        if (len == 0.0) {
            i0 = j0;
            i1 = j1;
            continue;
        }
        const double inv = 1.0 / len;
        const double dx = inv * (p.x(j0) - p.x(i1)), dy = inv * (p.y(j0) - p.y(i1));
        const double wdx = 0.5 * w * dx, wdy = 0.5 * w * dy;
        const double ix = p.x(i0), iy = p.y(i0), jx = p.x(j0), jy = p.y(j0);
        if (!out.move(ix - wdy, iy + wdx)) break;
        if (first && !closed) start_cap(out, sp.line_cap, ix, iy, wdx, wdy);
        else out.line(ix + wdy, iy - wdx);
        out.line(jx + wdy, jy - wdx);
        if (last && !closed) end_cap(out, sp.line_cap, jx, jy, wdx, wdy);
        else out.line(jx - wdy, jy + wdx);
        out.close();
        if (!last || closed) {
            const double nlen = seg_len(p.x(j1), p.y(j1), p.x(k0), p.y(k0));
            const double inv_n = 1.0 / nlen;
            int an_kind = -1;
            double an_val = 0.0;
            const double nx = inv_n * (p.x(k0) - p.x(j1)), ny = inv_n * (p.y(k0) - p.y(j1));
            const double wnx = 0.5 * w * nx, wny = 0.5 * w * ny;
            const double cross = dx * ny - dy * nx;
            const double dot = -(dx * nx + dy * ny);
            const bool angle = cross != 0.0 || dx * nx < 0.0 || dy * ny < 0.0;
            double miter = (sp.miter_limit + 1.0) * (sp.miter_limit + 1.0), m = 0.0;
            if (!(dot > kMiterNearlyStraight)) {
                miter = std::fmax(2.0 / (1.0 - dot), 1.0);
                m = std::sqrt(miter - 1.0);
            }
            if (angle && sp.line_join == RRB_JOIN_ROUND) {
                round_join(out, jx, jy, w, dx, dy, wdx, wdy, nx, ny, wnx, wny, cross, known ? next.ang_kind : -1,
                           next.ang, an_kind, an_val);
            } else if (angle) {
                const bool apex = sp.line_join == RRB_JOIN_MITER && std::sqrt(miter) <= sp.miter_limit;
                out.move(jx, jy);
                if (cross < 0.0) {
                    out.line(jx - wny, jy + wnx);
                    if (apex) out.line(jx - wdy + wdx * m, jy + wdx + wdy * m);
                    out.line(jx - wdy, jy + wdx);
                } else {
                    out.line(jx + wdy, jy - wdx);
                    if (apex) out.line(jx + wdy + wdx * m, jy - wdx + wdy * m);
                    out.line(jx + wny, jy - wnx);
                }
            }
            out.close();
            next.a = j1;
            next.b = k0;
            next.len = nlen;
            next.ang_kind = an_kind;
            next.ang = an_val;
        }
        i0 = j0;
        i1 = j1;
    }
}

// Scratch of one worker: the flattened and the dashed polyline of the path
// in hand, reused from path to path.
struct Scratch {
    std::vector<double> xy1, xy2;
    std::vector<uint8_t> fl1, fl2;
};

// What stroke() draws for one path, appended to (xy, fl): returns
// RRB_STROKE_NOTHING, RRB_STROKE_OUTLINE or RRB_STROKE_HAIRLINE.
int stroke_one(const Pts& in, const rrb_stroke_params& sp, double flatness, Scratch& s, std::vector<double>& xy,
               std::vector<uint8_t>& fl) {
    if (in.n == 0) return rrb_stroke::NOTHING;
    s.xy1.clear();
    s.fl1.clear();
    Sink flat{&s.xy1, &s.fl1};
    flatten_path(in, flatness, flat);
    Pts poly{s.xy1.data(), s.fl1.data(), s.fl1.size()};
    if (sp.n_dash > 0) {
        s.xy2.clear();
        s.fl2.clear();
        Sink dashed{&s.xy2, &s.fl2};
        dash_path(poly, sp.dash, sp.n_dash, sp.dash_phase, dashed);
        if (s.fl2.empty()) return rrb_stroke::NOTHING;
        poly = Pts{s.xy2.data(), s.fl2.data(), s.fl2.size()};
    }
    if (sp.line_width == 0.0) {
        xy.insert(xy.end(), poly.xy, poly.xy + 2 * poly.n);
        fl.insert(fl.end(), poly.fl, poly.fl + poly.n);
        return rrb_stroke::HAIRLINE;
    }
    Sink out{&xy, &fl, fl.size(), 0};
    outline_path(poly, sp.line_width, sp, out);
    return rrb_stroke::OUTLINE;
}

}  // namespace

namespace rrb_stroke {

int check_params(const rrb_stroke_params& sp, std::string& msg) {
    if (!sp.stroke) return RRB_OK;
    if (!(std::isfinite(sp.line_width) && sp.line_width >= 0.0)) return msg = "line_width must be finite and >= 0", RRB_ERR_INVARIANT;
    if (!std::isfinite(sp.miter_limit)) return msg = "miter_limit must be finite", RRB_ERR_INVARIANT;
    if (sp.line_cap > RRB_CAP_PROJECTING || sp.line_join > RRB_JOIN_BEVEL)
        return msg = "line_cap / line_join out of range", RRB_ERR_INVARIANT;
    if (sp.n_dash) {
        if (!sp.dash) return msg = "dash array is null", RRB_ERR_INVARIANT;
        if (!std::isfinite(sp.dash_phase)) return msg = "dash_phase must be finite", RRB_ERR_INVARIANT;
        for (uint32_t k = 0; k < sp.n_dash; ++k)
            if (!(std::isfinite(sp.dash[k]) && sp.dash[k] >= 0.0))
                return msg = "dash entries must be finite and >= 0", RRB_ERR_INVARIANT;
    }
    return RRB_OK;
}

namespace {

// Runs fn(worker) on up to `want` threads (the calling thread is one).
template <typename Fn>
void parallel(unsigned want, Fn fn) {
    if (want <= 1) {
        fn();
        return;
    }
    std::vector<std::thread> th;
    th.reserve(want - 1);
    for (unsigned t = 1; t < want; ++t) th.emplace_back(fn);
    fn();
    for (auto& t : th) t.join();
}

// Hairline segments of a polyline, walked as XPath::new walks a path without
// curves and without closing (xpath.rs:162-260): from each FIRST point
// through the points up to the next LAST. emit(a, b) gets point indices.
template <typename Emit>
uint32_t hairline_segments(const uint8_t* fl, uint64_t n, Emit emit) {
    uint32_t k = 0;
    uint64_t j = 0;
    while (j < n) {
        if (!(fl[j] & RRB_PATH_FIRST)) {
            ++j;
            continue;
        }
        uint64_t cur = j++;
        while (j < n) {
            emit(cur, j);
            ++k;
            cur = j;
            const bool last = fl[j] & RRB_PATH_LAST;
            ++j;
            if (last) break;
        }
    }
    return k;
}

}  // namespace

int build(const rrb_path_batch_params* p, const rrb_stroke_params* sp, const uint8_t* path_rgb,
          const double* clip_rects, HostAlloc& alloc, PaintBatch& out, std::string& msg) {
    const uint64_t n = p->n_paths;
    out.n_paths = out.n_pts = 0;
    for (uint64_t i = 0; i < n; ++i) {
        const int rc = check_params(sp[i], msg);
        if (rc) return rc;
    }
    constexpr uint64_t kChunk = 64;
    const uint64_t n_chunks = (n + kChunk - 1) / kChunk;
    if (out.chunks.size() < n_chunks) out.chunks.resize(n_chunks);
    const double flatness = std::max(p->flatness, 0.0);
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned nt = static_cast<unsigned>(std::min<uint64_t>(std::min(hw, 32u), n_chunks));
    // Pass 1: stroke each chunk's paths into its own buffers; count the
    // output paths and points.
    std::atomic<uint64_t> next{0};
    parallel(nt, [&]() {
        Scratch s;
        for (;;) {
            const uint64_t c = next.fetch_add(1);
            if (c >= n_chunks) return;
            Chunk& ch = out.chunks[c];
            const uint64_t b = c * kChunk, e = std::min(n, b + kChunk);
            ch.xy.clear();
            ch.fl.clear();
            ch.kind.assign(e - b, NOTHING);
            ch.len.assign(e - b, 0);
            ch.segs.assign(e - b, 0);
            ch.out_paths = ch.out_pts = 0;
            for (uint64_t i = b; i < e; ++i) {
                const uint64_t a0 = p->path_pt_off[i], a1 = p->path_pt_off[i + 1];
                const size_t k = i - b;
                if (!sp[i].stroke) {
                    ch.kind[k] = a1 > a0 ? FILL : NOTHING;
                    if (a1 > a0) {
                        ch.out_paths += 1;
                        ch.out_pts += a1 - a0;
                    }
                    continue;
                }
                const size_t before = ch.fl.size();
                int kind = stroke_one(Pts{p->pts + 2 * a0, p->flags + a0, static_cast<size_t>(a1 - a0)}, sp[i],
                                      flatness, s, ch.xy, ch.fl);
                ch.len[k] = ch.fl.size() - before;
                if (ch.len[k] == 0) kind = NOTHING;
                ch.kind[k] = static_cast<uint8_t>(kind);
                if (kind == OUTLINE) {
                    ch.out_paths += 1;
                    ch.out_pts += ch.len[k];
                } else if (kind == HAIRLINE) {
                    ch.segs[k] = hairline_segments(ch.fl.data() + before, ch.len[k], [](uint64_t, uint64_t) {});
                    ch.out_paths += ch.segs[k];
                    ch.out_pts += 2ull * ch.segs[k];
                }
            }
        }
    });
    // Offsets of each chunk's output.
    std::vector<uint64_t> path_at(n_chunks + 1, 0), pt_at(n_chunks + 1, 0);
    for (uint64_t c = 0; c < n_chunks; ++c) {
        path_at[c + 1] = path_at[c] + out.chunks[c].out_paths;
        pt_at[c + 1] = pt_at[c] + out.chunks[c].out_pts;
    }
    const uint64_t np = path_at[n_chunks], npt = pt_at[n_chunks];
    if (npt >= (1ull << 30) || np >= (1ull << 31))
        return msg = "painted geometry exceeds 2^30 points or 2^31 paths", RRB_ERR_POOL_EXHAUSTED;
    out.n_paths = np;
    out.n_pts = npt;
    if (np == 0) return RRB_OK;
    out.pts.reserve(alloc, 2 * npt);
    out.flags.reserve(alloc, npt);
    out.off.reserve(alloc, np + 1);
    out.rule.reserve(alloc, np);
    out.gray.reserve(alloc, np);
    out.alpha.reserve(alloc, np);
    out.page.reserve(alloc, np);
    if (path_rgb) out.rgb.reserve(alloc, 3 * np);
    if (clip_rects) out.clip.reserve(alloc, 4 * np);
    if (!out.pts.p || !out.flags.p || !out.off.p || !out.rule.p || !out.gray.p || !out.alpha.p || !out.page.p ||
        (path_rgb && !out.rgb.p) || (clip_rects && !out.clip.p))
        return msg = "out of host memory for the paint batch", RRB_ERR_OUT_OF_MEMORY;
    out.off.p[np] = npt;
    // Pass 2: every chunk writes its output paths at its offsets.
    next = 0;
    parallel(nt, [&]() {
        for (;;) {
            const uint64_t c = next.fetch_add(1);
            if (c >= n_chunks) return;
            const Chunk& ch = out.chunks[c];
            uint64_t q = path_at[c], at = pt_at[c], g = 0;  // output path, output point, chunk geometry point
            const uint64_t b = c * kChunk, e = std::min(n, b + kChunk);
            auto meta = [&](uint64_t i, uint8_t rule) {
                out.off.p[q] = at;
                out.rule.p[q] = rule;
                out.gray.p[q] = p->gray[i];
                out.alpha.p[q] = p->alpha[i];
                out.page.p[q] = p->path_page[i];
                if (path_rgb) std::memcpy(out.rgb.p + 3 * q, path_rgb + 3 * i, 3);
                if (clip_rects) std::memcpy(out.clip.p + 4 * q, clip_rects + 4 * i, 4 * sizeof(double));
                ++q;
            };
            for (uint64_t i = b; i < e; ++i) {
                const size_t k = i - b;
                switch (ch.kind[k]) {
                    case FILL: {
                        const uint64_t a0 = p->path_pt_off[i], m = p->path_pt_off[i + 1] - a0;
                        meta(i, p->fill_rule[i]);
                        std::memcpy(out.pts.p + 2 * at, p->pts + 2 * a0, 2 * m * sizeof(double));
                        std::memcpy(out.flags.p + at, p->flags + a0, m);
                        at += m;
                        break;
                    }
                    case OUTLINE:
                        meta(i, 0);
                        std::memcpy(out.pts.p + 2 * at, ch.xy.data() + 2 * g, 2 * ch.len[k] * sizeof(double));
                        std::memcpy(out.flags.p + at, ch.fl.data() + g, ch.len[k]);
                        at += ch.len[k];
                        break;
                    case HAIRLINE: {
                        const double* xy = ch.xy.data() + 2 * g;
                        hairline_segments(ch.fl.data() + g, ch.len[k], [&](uint64_t a, uint64_t bb) {
                            meta(i, kRuleHairline);
                            double* o = out.pts.p + 2 * at;
                            o[0] = xy[2 * a];
                            o[1] = xy[2 * a + 1];
                            o[2] = xy[2 * bb];
                            o[3] = xy[2 * bb + 1];
                            out.flags.p[at] = RRB_PATH_FIRST;
                            out.flags.p[at + 1] = RRB_PATH_LAST;
                            at += 2;
                        });
                        break;
                    }
                    default:
                        break;
                }
                g += ch.len[k];
            }
        }
    });
    return RRB_OK;
}

}  // namespace rrb_stroke

extern "C" int rrb_stroke_outline(const double* pts, const uint8_t* flags, uint64_t n_pts,
                                  const rrb_stroke_params* stroke, double flatness, double* out_pts,
                                  uint8_t* out_flags, uint64_t cap, uint64_t* out_n, int* kind) {
    if (!stroke || !out_n || !kind || (n_pts && (!pts || !flags))) return RRB_ERR_INVARIANT;
    std::string msg;
    rrb_stroke_params sp = *stroke;
    sp.stroke = 1;
    if (const int rc = rrb_stroke::check_params(sp, msg)) return rc;
    Scratch s;
    std::vector<double> xy;
    std::vector<uint8_t> fl;
    *kind = stroke_one(Pts{pts, flags, static_cast<size_t>(n_pts)}, sp, std::max(flatness, 0.0), s, xy, fl);
    if (fl.empty()) *kind = rrb_stroke::NOTHING;
    *out_n = fl.size();
    const uint64_t k = std::min<uint64_t>(cap, fl.size());
    if (out_pts && k) std::memcpy(out_pts, xy.data(), 2 * k * sizeof(double));
    if (out_flags && k) std::memcpy(out_flags, fl.data(), k);
    return RRB_OK;
}
