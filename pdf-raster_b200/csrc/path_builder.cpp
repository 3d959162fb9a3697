// path_builder.cpp — host-side path construction.
//
// rrb_path_* restates PathBuilder (crates/raster/src/path/mod.rs:310-448):
// same flags, same close(false) rule (a closing lineTo(first) only when the
// subpath has >= 2 points and first != last), so the device sees exactly the
// Path::{pts, flags} arrays the reference renderer would hand to fill().
// Quadratic segments enter through conic_to_cubic
// (crates/font/src/outline.rs:106-112) as the reference's font outline
// decoder does.

#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/rrb.h"
#include "path_builder.h"


extern "C" {

rrb_path* rrb_path_new(void) { return new rrb_path(); }
void rrb_path_free(rrb_path* p) { delete p; }
void rrb_path_clear(rrb_path* p) {
    p->pts.clear();
    p->flags.clear();
    p->cur_subpath = 0;
}

// PathBuilder::move_to: BogusPath when a one-point subpath is active.
int rrb_path_move_to(rrb_path* p, double x, double y) {
    if (p->one_point_subpath()) return 2;
    size_t len = p->len();
    p->pts.push_back(x);
    p->pts.push_back(y);
    p->flags.push_back(RRB_PATH_FIRST | RRB_PATH_LAST);
    p->cur_subpath = len;
    return 0;
}

// PathBuilder::line_to: clears LAST on the previous endpoint.
int rrb_path_line_to(rrb_path* p, double x, double y) {
    if (p->no_current_point()) return 1;
    p->flags.back() &= static_cast<uint8_t>(~RRB_PATH_LAST);
    p->pts.push_back(x);
    p->pts.push_back(y);
    p->flags.push_back(RRB_PATH_LAST);
    return 0;
}

// PathBuilder::curve_to: two CURVE control points then the LAST endpoint.
int rrb_path_curve_to(rrb_path* p, double x1, double y1, double x2, double y2, double x3, double y3) {
    if (p->no_current_point()) return 1;
    p->flags.back() &= static_cast<uint8_t>(~RRB_PATH_LAST);
    const double q[6] = {x1, y1, x2, y2, x3, y3};
    const uint8_t f[3] = {RRB_PATH_CURVE, RRB_PATH_CURVE, RRB_PATH_LAST};
    for (int k = 0; k < 3; ++k) {
        p->pts.push_back(q[2 * k]);
        p->pts.push_back(q[2 * k + 1]);
        p->flags.push_back(f[k]);
    }
    return 0;
}

void rrb_conic_to_cubic(double p0x, double p0y, double pcx, double pcy, double p3x, double p3y,
                        double out[4]) {
    out[0] = std::fma(p0x, 1.0 / 3.0, pcx * (2.0 / 3.0));
    out[1] = std::fma(p0y, 1.0 / 3.0, pcy * (2.0 / 3.0));
    out[2] = std::fma(pcx, 2.0 / 3.0, p3x * (1.0 / 3.0));
    out[3] = std::fma(pcy, 2.0 / 3.0, p3y * (1.0 / 3.0));
}

// Quadratic segment from the current point: degree-elevated to a cubic.
int rrb_path_conic_to(rrb_path* p, double xc, double yc, double x3, double y3) {
    if (p->no_current_point()) return 1;
    double c[4];
    size_t n = p->len();
    rrb_conic_to_cubic(p->pts[2 * (n - 1)], p->pts[2 * (n - 1) + 1], xc, yc, x3, y3, c);
    return rrb_path_curve_to(p, c[0], c[1], c[2], c[3], x3, y3);
}

// PathBuilder::close.
int rrb_path_close(rrb_path* p, int force) {
    if (p->no_current_point()) return 1;
    size_t sp = p->cur_subpath, last = p->len() - 1;
    double fx = p->pts[2 * sp], fy = p->pts[2 * sp + 1];
    double lx = p->pts[2 * last], ly = p->pts[2 * last + 1];
    bool differ = !(fx == lx && fy == ly);
    if (force || (sp != last && differ)) {
        int rc = rrb_path_line_to(p, fx, fy);
        if (rc) return rc;
    }
    p->flags[sp] |= RRB_PATH_CLOSED;
    p->flags[p->len() - 1] |= RRB_PATH_CLOSED;
    p->cur_subpath = p->len();
    return 0;
}

uint64_t rrb_path_len(const rrb_path* p) { return p->len(); }
const double* rrb_path_pts(const rrb_path* p) { return p->pts.data(); }
const uint8_t* rrb_path_flags(const rrb_path* p) { return p->flags.data(); }

}  // extern "C"

