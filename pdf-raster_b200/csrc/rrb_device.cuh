// rrb_device.cuh — device-side arithmetic of the AA fill path.
//
// Every FP64 operation that the reference performs as a single IEEE op is
// written with an explicit round-to-nearest intrinsic (__dadd_rn, __dmul_rn,
// ...) so nvcc cannot contract it into an FMA; every f64::mul_add of the
// reference is __fma_rn. That keeps flattening and segment set-up bit-exact
// with the reference CPU rasterizer independently of -fmad.
//
// The functions are __host__ __device__: compiled for the host (the CPU
// tests do, with -ffp-contract=off) the same operations are plain IEEE
// double operations and std::fma, which round the same way.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

namespace rrb {

constexpr int AA = 4;                     // AA_SIZE (crates/raster/src/types.rs:27)
constexpr int MAX_CURVE_SPLITS = 1024;    // types.rs:36
constexpr int FLATTEN_STACK = 10;         // log2(MAX_CURVE_SPLITS) pending right halves

// PathFlags (crates/raster/src/path/mod.rs:70-79).
constexpr uint8_t PF_FIRST = 0x01, PF_LAST = 0x02, PF_CLOSED = 0x04, PF_CURVE = 0x08;

// Edge kinds of the int32 edge record.
constexpr int EK_HORIZ = 0, EK_VERT = 1, EK_SLOPED = 2;
constexpr int EF_KIND_MASK = 3, EF_POSITIVE = 4, EF_FIRST_ZERO = 8, EF_EMPTY = 16;

#ifdef __CUDA_ARCH__
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double dfma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ unsigned long long bits_of(double x) { return __double_as_longlong(x); }
__device__ __forceinline__ bool is_pos_inf(double x) { return x == __longlong_as_double(0x7ff0000000000000LL); }
__device__ __forceinline__ int32_t trunc_i32(double x) { return __double2int_rz(x); }
#else
inline double dadd(double a, double b) { return a + b; }
inline double dsub(double a, double b) { return a - b; }
inline double dmul(double a, double b) { return a * b; }
inline double ddiv(double a, double b) { return a / b; }
inline double dfma(double a, double b, double c) { return std::fma(a, b, c); }
inline unsigned long long bits_of(double x) {
    unsigned long long b;
    std::memcpy(&b, &x, sizeof b);
    return b;
}
inline bool is_pos_inf(double x) { return x == HUGE_VAL; }
inline int32_t trunc_i32(double x) { return static_cast<int32_t>(x); }  // |x| < 2^31 at every call
#endif

// f64::midpoint (Rust std): (a+b)/2 when both |a|,|b| <= f64::MAX/2. x/2
// and x*0.5 are the same correctly rounded value of the same real number, so
// the halving is a multiplication.
__host__ __device__ __forceinline__ double midpoint(double a, double b) {
    const double HI = 8.98846567431157854e+307;   // f64::MAX / 2
    const double LO = 4.45014771701440277e-308;   // f64::MIN_POSITIVE * 2
    double aa = fabs(a), ab = fabs(b);
    if (aa <= HI && ab <= HI) return dmul(dadd(a, b), 0.5);
    if (aa < LO) return dadd(a, dmul(b, 0.5));
    if (ab < LO) return dadd(dmul(a, 0.5), b);
    return dadd(dmul(a, 0.5), dmul(b, 0.5));
}

// saturate_f64_to_i32 / splash_floor (crates/color/src/convert.rs:221-265).
__host__ __device__ __forceinline__ int32_t sat_i32_of_integral(double x) {
    if (!isfinite(x)) return is_pos_inf(x) ? INT32_MAX : INT32_MIN;
    if (x >= 2147483647.0) return INT32_MAX;
    if (x <= -2147483648.0) return INT32_MIN;
    return static_cast<int32_t>(x);
}
__host__ __device__ __forceinline__ int32_t splash_floor(double x) { return sat_i32_of_integral(floor(x)); }

// fp_from_f64 (crates/raster/src/scanner/mod.rs:51-66): truncating 16.16.
__host__ __device__ __forceinline__ int32_t fp_from_f64(double x) {
    double fp = dmul(x, 65536.0);
    if (fp >= 2147483647.0) return INT32_MAX;
    if (fp <= -2147483648.0) return INT32_MIN;
    if (isnan(fp)) return 0;
    return trunc_i32(fp);
}

__host__ __device__ __forceinline__ int32_t sat_i64_to_i32(long long v) {
    return v > INT32_MAX ? INT32_MAX : (v < INT32_MIN ? INT32_MIN : static_cast<int32_t>(v));
}

// transform (crates/raster/src/xpath.rs:421-426).
__host__ __device__ __forceinline__ void transform(const double* m, double x, double y, double& ox, double& oy) {
    ox = dfma(x, m[0], dfma(y, m[2], m[4]));
    oy = dfma(x, m[1], dfma(y, m[3], m[5]));
}

// The int32 edge record: everything fill_intersections (scanner/mod.rs:511-587)
// derives from one AA-scaled XPathSeg, so the row stage needs no FP64.
//   row0,row1  clipped AA row range (EF_EMPTY when none)
//   flags      kind | EF_POSITIVE (FLIPPED: count +1, else -1) | EF_FIRST_ZERO
//              (row0 is not strictly below seg_y_min: count 0 on row0)
//   a          HORIZ: floor(min x); VERT: floor(x0); SLOPED: px0 of row0
//   b          HORIZ: floor(max x); SLOPED: xx1_fp of row0 (16.16)
//   dfp        SLOPED: dxdy_fp; cmin/cmax: SLOPED 16.16 clamp bounds
struct __align__(16) Edge {
    int32_t row0, row1, flags, a, b, dfp, cmin, cmax;
};

// add_segment (xpath.rs:324-402) + aa_scale (xpath.rs:283-303) + the
// per-segment set-up of count/fill_intersections, clipped to AA rows
// [clip_lo, clip_hi].
__host__ __device__ __forceinline__ Edge make_edge(double x0, double y0, double x1, double y1, int32_t clip_lo,
                                                   int32_t clip_hi) {
    Edge e;
    e.dfp = 0;
    e.cmin = 0;
    e.cmax = 0;
    e.b = 0;
    unsigned long long by0 = bits_of(y0), by1 = bits_of(y1);
    unsigned long long bx0 = bits_of(x0), bx1 = bits_of(x1);
    if (by0 == by1) {
        // HORIZ: never flipped, dxdy = 0; aa_scale then multiplies by 4.
        double sx0 = dmul(x0, 4.0), sx1 = dmul(x1, 4.0), sy = dmul(y0, 4.0);
        e.flags = EK_HORIZ;
        if (isnan(sx0) || isnan(sy)) {
            e.flags |= EF_EMPTY;
            e.row0 = 1;
            e.row1 = 0;
            e.a = 0;
            return e;
        }
        int32_t row = splash_floor(sy);
        if (row >= clip_lo && row <= clip_hi) {
            e.row0 = row;
            e.row1 = row;
        } else {
            e.flags |= EF_EMPTY;
            e.row0 = 1;
            e.row1 = 0;
        }
        e.a = splash_floor(fmin(sx0, sx1));
        e.b = splash_floor(fmax(sx0, sx1));
        return e;
    }
    bool vert = bx0 == bx1;
    double dxdy = vert ? 0.0 : ddiv(dsub(x1, x0), dsub(y1, y0));
    bool flipped = false;
    if (y0 > y1) {
        double t = x0; x0 = x1; x1 = t;
        t = y0; y0 = y1; y1 = t;
        flipped = true;
    }
    int32_t dxdy_fp;
    {
        double fp = dmul(dxdy, 65536.0);
        if (fp >= 2147483647.0) dxdy_fp = INT32_MAX;
        else if (fp <= -2147483648.0) dxdy_fp = INT32_MIN;
        else if (isnan(fp)) dxdy_fp = 0;
        else dxdy_fp = static_cast<int32_t>(round(fp));
    }
    x0 = dmul(x0, 4.0);
    y0 = dmul(y0, 4.0);
    x1 = dmul(x1, 4.0);
    y1 = dmul(y1, 4.0);
    e.flags = (vert ? EK_VERT : EK_SLOPED) | (flipped ? EF_POSITIVE : 0);
    if (isnan(x0) || isnan(y0)) {
        e.flags |= EF_EMPTY;
        e.row0 = 1;
        e.row1 = 0;
        e.a = 0;
        return e;
    }
    double sy_min = fmin(y0, y1), sy_max = fmax(y0, y1);
    int32_t r0 = max(splash_floor(sy_min), clip_lo);
    int32_t r1 = min(splash_floor(sy_max), clip_hi);
    e.row0 = r0;
    e.row1 = r1;
    if (r0 > r1) e.flags |= EF_EMPTY;
    if (!(sy_min < static_cast<double>(r0))) e.flags |= EF_FIRST_ZERO;
    if (vert) {
        e.a = splash_floor(x0);
        return e;
    }
    double x_base = dfma(y0, -dxdy, x0);
    double sxmin = fmin(x0, x1), sxmax = fmax(x0, x1);
    e.cmin = fp_from_f64(sxmin);
    e.cmax = fp_from_f64(sxmax);
    double r0d = static_cast<double>(r0);
    double xx_init = r0d > y0 ? dfma(r0d, dxdy, x_base) : x0;
    double xc = xx_init;
    if (xc < sxmin) xc = sxmin;
    if (xc > sxmax) xc = sxmax;
    e.a = splash_floor(xc);
    e.b = fp_from_f64(dfma(dadd(r0d, 1.0), dxdy, x_base));
    e.dfp = dxdy_fp;
    return e;
}

// Floor of a / b for b > 0.
__host__ __device__ __forceinline__ int32_t floor_div(int32_t a, int32_t b) {
    return a >= 0 ? a / b : -((-a + b - 1) / b);
}

// Intersect entry of edge `e` on AA row r (row0 <= r <= row1): the closed form
// of fill_intersections' stepping. The saturating accumulator
// xx1_fp += dxdy_fp is monotone, so after k steps it equals the exact sum
// clamped to the i32 range.
__host__ __device__ __forceinline__ void edge_entry(const Edge& e, int32_t r, int32_t& lo, int32_t& hi, int32_t& c) {
    int kind = e.flags & EF_KIND_MASK;
    if (kind == EK_HORIZ) {
        lo = e.a;
        hi = e.b;
        c = 0;
        return;
    }
    c = ((e.flags & EF_FIRST_ZERO) && r == e.row0) ? 0 : ((e.flags & EF_POSITIVE) ? 1 : -1);
    if (kind == EK_VERT) {
        lo = e.a;
        hi = e.a;
        return;
    }
    long long k = static_cast<long long>(r) - e.row0;
    // The exact sums after k and k - 1 steps (|k * dfp| < 2^62: no overflow).
    const long long s1 = static_cast<long long>(e.b) + k * e.dfp;
    int32_t x1v = sat_i64_to_i32(s1);
    int32_t px1 = min(max(x1v, e.cmin), e.cmax) >> 16;
    int32_t px0;
    if (k == 0) {
        px0 = e.a;
    } else {
        int32_t x0v = sat_i64_to_i32(s1 - e.dfp);
        px0 = min(max(x0v, e.cmin), e.cmax) >> 16;
    }
    lo = min(px0, px1);
    hi = max(px0, px1);
}

// AA column range [lo, hi] of the entries an edge can produce.
__host__ __device__ __forceinline__ void edge_xrange(const Edge& e, int32_t& lo, int32_t& hi) {
    int kind = e.flags & EF_KIND_MASK;
    if (kind == EK_HORIZ) {
        lo = e.a;
        hi = e.b;
    } else if (kind == EK_VERT) {
        lo = e.a;
        hi = e.a;
    } else {
        lo = min(e.a, e.cmin >> 16);
        hi = max(e.a, e.cmax >> 16);
    }
}

// flatten_curve (crates/raster/src/path/flatten.rs:109-215) with the slot
// arrays replaced by the chain of pending right halves: slot p's data is
// (start, c1, c2) and its endpoint is the start of the next pending slot (or
// p3 when that is slot MAX_CURVE_SPLITS). Splitting [pp1,pp2] pushes slot
// pp3 = (pp1+pp2)/2; emitting pops. Interval lengths halve per push, so at
// most log2(1024) = 10 halves are pending. Same operations in the same
// order as the reference, hence the same points.
// (a+b)/2 for operands known to be within +-f64::MAX/2 (midpoint's first branch).
__host__ __device__ __forceinline__ double midpoint_in_range(double a, double b) { return dmul(dadd(a, b), 0.5); }

template <bool IN_RANGE, typename Emit>
__host__ __device__ __forceinline__ int flatten_range_impl(double c0x, double c0y, double c1x, double c1y, double c2x,
                                                           double c2y, double r3x, double r3y, int pp_lo, int pp_hi,
                                                           double flat_sq, int limit, Emit& emit);

// Every point the subdivision computes is a midpoint of two earlier points,
// i.e. a convex combination of the four control points, so when all control
// coordinates lie within +-f64::MAX/2 every midpoint call takes the (a+b)/2
// branch: the check is made once per curve and the loop runs branch-free.
__host__ __device__ __forceinline__ bool curve_in_range(double p0x, double p0y, double p1x, double p1y, double p2x,
                                                        double p2y, double p3x, double p3y) {
    const double HI = 8.98846567431157854e+307;
    const double m = fmax(fmax(fmax(fabs(p0x), fabs(p0y)), fmax(fabs(p1x), fabs(p1y))),
                          fmax(fmax(fabs(p2x), fabs(p2y)), fmax(fabs(p3x), fabs(p3y))));
    return m <= HI;
}

template <typename Emit>
__host__ __device__ __forceinline__ int flatten_curve(double p0x, double p0y, double p1x, double p1y, double p2x,
                                                      double p2y, double p3x, double p3y, double flat_sq,
                                                      Emit emit) {
    if (curve_in_range(p0x, p0y, p1x, p1y, p2x, p2y, p3x, p3y))
        return flatten_range_impl<true>(p0x, p0y, p1x, p1y, p2x, p2y, p3x, p3y, 0, MAX_CURVE_SPLITS, flat_sq, 0, emit);
    return flatten_range_impl<false>(p0x, p0y, p1x, p1y, p2x, p2y, p3x, p3y, 0, MAX_CURVE_SPLITS, flat_sq, 0, emit);
}

// The segment count of a curve, or limit + 1 as soon as it exceeds limit.
__host__ __device__ __forceinline__ int flatten_count_capped(double p0x, double p0y, double p1x, double p1y,
                                                             double p2x, double p2y, double p3x, double p3y,
                                                             double flat_sq, int limit) {
    auto none = [](double, double) {};
    if (curve_in_range(p0x, p0y, p1x, p1y, p2x, p2y, p3x, p3y))
        return flatten_range_impl<true>(p0x, p0y, p1x, p1y, p2x, p2y, p3x, p3y, 0, MAX_CURVE_SPLITS, flat_sq, limit,
                                        none);
    return flatten_range_impl<false>(p0x, p0y, p1x, p1y, p2x, p2y, p3x, p3y, 0, MAX_CURVE_SPLITS, flat_sq, limit,
                                     none);
}

// One node of the subdivision: the piece of the curve between two slots,
// start point c0, control points c1, c2 and endpoint r3.
struct CurveNode {
    double c0x, c0y, c1x, c1y, c2x, c2y, r3x, r3y;
};

// flatten_curve's leaf test of a node: its chord midpoint against both
// control points.
template <bool IN_RANGE>
__host__ __device__ __forceinline__ bool node_is_flat(const CurveNode& n, double flat_sq) {
    auto mid = [](double a, double b) { return IN_RANGE ? midpoint_in_range(a, b) : midpoint(a, b); };
    const double mx = mid(n.c0x, n.r3x), my = mid(n.c0y, n.r3y);
    const double dx1 = dsub(n.c1x, mx), dy1 = dsub(n.c1y, my);
    const double dx2 = dsub(n.c2x, mx), dy2 = dsub(n.c2y, my);
    const double d1 = dfma(dx1, dx1, dmul(dy1, dy1));
    const double d2 = dfma(dx2, dx2, dmul(dy2, dy2));
    return d1 <= flat_sq && d2 <= flat_sq;
}

// flatten_curve's split of a node into its two halves.
template <bool IN_RANGE>
__host__ __device__ __forceinline__ void node_split(const CurveNode& n, CurveNode& left, CurveNode& right) {
    auto mid = [](double a, double b) { return IN_RANGE ? midpoint_in_range(a, b) : midpoint(a, b); };
    const double xl1 = mid(n.c0x, n.c1x), yl1 = mid(n.c0y, n.c1y);
    const double xh = mid(n.c1x, n.c2x), yh = mid(n.c1y, n.c2y);
    const double xl2 = mid(xl1, xh), yl2 = mid(yl1, yh);
    const double xr2 = mid(n.c2x, n.r3x), yr2 = mid(n.c2y, n.r3y);
    const double xr1 = mid(xh, xr2), yr1 = mid(yh, yr2);
    const double xr0 = mid(xl2, xr1), yr0 = mid(yl2, yr1);
    left = CurveNode{n.c0x, n.c0y, xl1, yl1, xl2, yl2, xr0, yr0};
    right = CurveNode{xr0, yr0, xr1, yr1, xr2, yr2, n.r3x, n.r3y};
}

// The subdivision restricted to the node over slots [pp_lo, pp_hi) with start
// c0, controls c1, c2 and endpoint r3: emits the endpoint of every leaf in
// order and returns their number (flatten_curve is the whole curve, slots
// [0, 1024)). limit > 0: stops once more than limit leaves are found,
// returning limit + 1.
template <bool IN_RANGE, typename Emit>
__host__ __device__ __forceinline__ int flatten_range_impl(double c0x, double c0y, double c1x, double c1y, double c2x,
                                                           double c2y, double r3x, double r3y, int pp_lo, int pp_hi,
                                                           double flat_sq, int limit, Emit& emit) {
    double sx[FLATTEN_STACK][6];
    int sidx[FLATTEN_STACK];
    int top = 0;
    int pp1 = pp_lo;
    int count = 0;
    while (pp1 < pp_hi) {
        int pp2;
        CurveNode n;
        if (top > 0) {
            pp2 = sidx[top - 1];
            n = CurveNode{c0x, c0y, c1x, c1y, c2x, c2y, sx[top - 1][0], sx[top - 1][1]};
        } else {
            pp2 = pp_hi;
            n = CurveNode{c0x, c0y, c1x, c1y, c2x, c2y, r3x, r3y};
        }
        if (pp2 - pp1 == 1 || node_is_flat<IN_RANGE>(n, flat_sq)) {
            emit(n.r3x, n.r3y);
            ++count;
            if (limit > 0 && count > limit) return count;
            pp1 = pp2;
            if (top > 0) {
                --top;
                c0x = sx[top][0];
                c0y = sx[top][1];
                c1x = sx[top][2];
                c1y = sx[top][3];
                c2x = sx[top][4];
                c2y = sx[top][5];
            }
        } else {
            CurveNode l, r;
            node_split<IN_RANGE>(n, l, r);
            const int pp3 = (pp1 + pp2) >> 1;
            // pp2 - pp1 >= 2 here, so fewer than FLATTEN_STACK halves are pending.
            sx[top][0] = r.c0x;
            sx[top][1] = r.c0y;
            sx[top][2] = r.c1x;
            sx[top][3] = r.c1y;
            sx[top][4] = r.c2x;
            sx[top][5] = r.c2y;
            sidx[top] = pp3;
            ++top;
            c1x = l.c1x;
            c1y = l.c1y;
            c2x = l.c2x;
            c2y = l.c2y;
        }
    }
    return count;
}

// A curve split among the 32 lanes of a warp: lane l takes the subtree of
// slots [32 l, 32 l + 32), the node the sequential subdivision reaches after
// five halvings. Each lane walks down from the root with node_is_flat and
// node_split, so the node it reaches (and every point below it) is computed
// by the same operations on the same values as in flatten_curve. If an
// ancestor is a leaf, the lane whose subtree starts at that leaf's first slot
// emits it (mode 1: the segment c0 -> r3 of `node`) and the others emit
// nothing (mode 2); otherwise (mode 0) the lane flattens `node` over its
// slots with flatten_range_impl. In lane order the leaves are the curve's
// leaves in order.
constexpr int CURVE_LANE_DEPTH = 5;
constexpr int CURVE_LANE_SLOTS = MAX_CURVE_SPLITS >> CURVE_LANE_DEPTH;  // 32

template <bool IN_RANGE>
__host__ __device__ __forceinline__ int curve_lane_node(const CurveNode& root, int lane, double flat_sq,
                                                        CurveNode& node) {
    node = root;
    int lo = 0, hi = MAX_CURVE_SPLITS;
    const int target = lane * CURVE_LANE_SLOTS;
    for (int d = 0; d < CURVE_LANE_DEPTH; ++d) {
        if (node_is_flat<IN_RANGE>(node, flat_sq)) return target == lo ? 1 : 2;  // hi - lo >= 64 here
        CurveNode l, r;
        node_split<IN_RANGE>(node, l, r);
        const int mid = (lo + hi) >> 1;
        if (target < mid) {
            node = l;
            hi = mid;
        } else {
            node = r;
            lo = mid;
        }
    }
    return 0;
}

// The leaves of lane `lane` of a curve (see curve_lane_node): emits their
// endpoints and returns their number; c0 receives the lane's first start point.
template <bool IN_RANGE, typename Emit>
__host__ __device__ __forceinline__ int curve_lane_flatten(const CurveNode& root, int lane, double flat_sq,
                                                           double& c0x, double& c0y, Emit& emit) {
    CurveNode n;
    const int mode = curve_lane_node<IN_RANGE>(root, lane, flat_sq, n);
    c0x = n.c0x;
    c0y = n.c0y;
    if (mode == 2) return 0;
    if (mode == 1) {
        emit(n.r3x, n.r3y);
        return 1;
    }
    const int lo = lane * CURVE_LANE_SLOTS;
    return flatten_range_impl<IN_RANGE>(n.c0x, n.c0y, n.c1x, n.c1y, n.c2x, n.c2y, n.r3x, n.r3y, lo,
                                        lo + CURVE_LANE_SLOTS, flat_sq, 0, emit);
}

// div255 (crates/color/src/convert.rs:50-58).
__host__ __device__ __forceinline__ uint32_t div255(uint32_t x) {
    uint32_t s = (x + (x >> 8) + 0x80u) >> 8;
    return s > 255u ? 255u : s;
}

}  // namespace rrb
