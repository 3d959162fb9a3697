// rrb_kernels.cuh — the AA fill pipeline kernels.
//
// Stage map onto the reference CPU path (crates/raster):
//   k_walk          XPath::new subpath walk (xpath.rs:162-260), incl. the
//                   curve-branch LAST quirk and the 1e-10 closing test
//   k_seg_count     flatten_curve pass 1 (path/flatten.rs:109-215): counts
//   k_seg_write     flatten_curve pass 2 + add_segment + aa_scale + the
//                   per-segment set-up of fill_intersections -> Edge records
//   k_path_bbox     XPathScanner::new bounding box (scanner/mod.rs:131-180)
//   k_super_*       per-page tile binning: ordered path lists per supertile
//   k_rows          fill_intersections + write_intersect merge + per-row sort
//                   + render_aa_line winding walk (scanner/mod.rs:393-642),
//                   one warp per 32 AA rows of one path
//   k_rows_slow     the same for rows whose merged list exceeds shared memory
//   k_composite     draw_aa_line coverage + AA_GAMMA + render_span_aa div255
//                   source-over (fill/mod.rs:344-401, pipe/aa.rs:192-208),
//                   one CTA per page tile, paths in index order
#pragma once

#include <cstddef>
#include <cstdint>

#include "rrb_device.cuh"

namespace rrb {

// Piece slots: one per input point. kind in bits 30-31 of .y.
constexpr uint32_t PK_NONE = 0, PK_LINE = 1, PK_CURVE = 2, PK_CLOSE = 3;

// 64 bytes, 16-byte aligned; the pixel rectangle leads so it loads as one int4.
struct __align__(16) PathInfo {
    int32_t px0, px1;        // pixel columns touched (px0 > px1: none)
    int32_t py0, py1;        // pixel rows touched under the row map
    int32_t y0, y1;          // AA rows [y0, y1] (y0 > y1: no rows)
    uint32_t e_begin, e_end; // edge range
    uint32_t paint;          // gray | alpha << 8 | rule << 16 | PI_RECTI
    uint32_t page;
    uint32_t run_off, run_cnt; // rectilinear paths: pixel-row runs of identical coverage
    int32_t bx0, bx1, by0, by1; // solid box: pixels with coverage 16 (bx0 > bx1: none)
};

constexpr uint32_t PI_RECTI = 1u << 17;  // all edges horizontal or vertical, at most RECTI_MAX_EDGES
// Spans drawn without a shape (hairline strokes): on Rgb8 pages they blend
// with render_span's general arm c = div255((255 - a) * dst + a * src)
// (pipe/general.rs:261-312) instead of the AA fast path; on Gray8 pages the
// two agree (a_src = div255(a * 255) = a).
constexpr uint32_t PI_SOLID = 1u << 19;
// A rectilinear path whose every AA row in [y0, y1] holds the same single
// span [S0, S1) of AA columns (an axis-aligned rectangle): the coverage of
// pixel (x, y) is cx * cy, cx = |[4x, 4x+4) n [S0, S1)| and cy = the number
// of the pixel row's AA rows inside [y0, y1] — draw_aa_line's nibble popcount
// summed over four identical sub-rows. Such a path keeps S0 in run_off, S1 in
// run_cnt and the AA rows it paints in [y0, y1] (set by k_recti), and has no
// runs or cells: the composite evaluates its coverage directly.
constexpr uint32_t PI_BOX = 1u << 20;
constexpr uint32_t RECTI_MAX_EDGES = 32;

// Error / status word bits shared by all kernels of a batch.
constexpr uint32_t ERR_EDGE_CAP = 1, ERR_ROW_CAP = 2, ERR_SPAN_CAP = 4, ERR_OVF_CAP = 8,
                   ERR_SCRATCH_CAP = 16, ERR_SUPER_CAP = 32;

// Device counters of a batch.
struct BatchCounters {
    uint32_t err;
    uint32_t cell_cursor;
    uint32_t ovf_count;
    uint32_t scratch_cursor;
    uint32_t nonterminating;
    uint32_t ovf2_count;
    uint32_t tile_cursor;  // k_composite's work queue: the next tile to take
    uint32_t big_curves;   // curves flattened by a warp each (k_seg_count's big_list)
    unsigned long long raw_entries;  // sum over edges of the rows they cover
    unsigned long long aa_rows;      // sum over paths of y1 - y0 + 1
    unsigned long long hl_rows;      // hairline segments: pixel rows drawn (one run and one cell each)
};

// Internal fill-rule value of a hairline segment: a two-point path drawn as
// stroke_narrow's one-pixel spans, not filled (see rrb_hairline.cuh).
constexpr uint8_t RULE_HAIRLINE = 2;

// Clip of path p in AA units: columns [x, y) and rows [z, w] — the page, or
// the page and a clip rectangle (Clip::clip_to_rect) when path_clip is given.
__device__ __forceinline__ int4 path_clip_of(const int4* __restrict__ path_clip, uint32_t p, int32_t aa_width,
                                             int32_t aa_height) {
    return path_clip ? path_clip[p] : make_int4(0, aa_width, 0, aa_height - 1);
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// ---------------------------------------------------------------------------
// XPath::new walk, one thread per path. Pieces are written at the path's
// point slots [off, off+n); unused slots get PK_NONE. Point indices are global.
// ---------------------------------------------------------------------------
__global__ void k_walk(const double* __restrict__ pts, const uint8_t* __restrict__ flags,
                       const uint64_t* __restrict__ path_pt_off, uint32_t n_paths,
                       const double* __restrict__ mtx, const uint32_t* __restrict__ path_page,
                       const uint32_t* __restrict__ page_h, uint2* __restrict__ pieces,
                       uint32_t* __restrict__ path_pieces, const uint8_t* __restrict__ rule,
                       uint32_t long_min = 0xffffffffu) {
    __shared__ double m[6];
    if (threadIdx.x < 6) m[threadIdx.x] = mtx[threadIdx.x];
    __syncthreads();
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n_paths; p += gridDim.x * blockDim.x) {
        uint32_t off = static_cast<uint32_t>(path_pt_off[p]);
        uint32_t n = static_cast<uint32_t>(path_pt_off[p + 1]) - off;
        if (n >= long_min) continue;  // walked by k_walk_long
        uint32_t slot = off;
        uint32_t i = 0;
        if (rule && rule[p] == RULE_HAIRLINE) n = 0;  // hairline segments have no fill edges
        while (i < n) {
            if (flags[off + i] & PF_FIRST) {
                uint32_t sp = i, cur = i;
                ++i;
                while (i < n) {
                    uint8_t f = flags[off + i];
                    if (f & PF_CURVE) {
                        if (i + 2 >= n) break;
                        pieces[slot++] = make_uint2(off + cur, (PK_CURVE << 30) | (off + i));
                        cur = i + 2;
                        i += 3;
                    } else {
                        pieces[slot++] = make_uint2(off + cur, (PK_LINE << 30) | (off + i));
                        cur = i;
                        ++i;
                        if (f & PF_LAST) break;
                    }
                }
                double sx, sy, cx, cy;
                transform(m, pts[2 * (off + sp)], pts[2 * (off + sp) + 1], sx, sy);
                transform(m, pts[2 * (off + cur)], pts[2 * (off + cur) + 1], cx, cy);
                if (fabs(dsub(cx, sx)) > 1e-10 || fabs(dsub(cy, sy)) > 1e-10)
                    pieces[slot++] = make_uint2(off + cur, (PK_CLOSE << 30) | (off + sp));
            } else {
                ++i;
            }
        }
        path_pieces[p] = slot - off;
    }
}

// The same walk for paths of at least long_min points, one warp per path.
// A serial walk of a long path (stroke outlines have thousands of points)
// keeps one lane busy while its warp's other paths are done, and its lanes
// diverge at every subpath end. Here each point's part in the walk is read
// from its neighbours' flags, which is exact when the path is well formed:
// it starts with FIRST; CURVE points come in pairs after a non-CURVE point
// and before a non-CURVE end point; no FIRST point is a control or end point;
// no two consecutive points are FIRST; and a point after which the walk
// breaks (an inner line point with LAST) is followed by a FIRST point. Then
// the walk examines every point but control and end points of curves:
//   start (FIRST, and the first point or just after a break): no piece;
//   first control point of a curve: CURVE piece from the point before;
//   any other examined point: LINE piece from the point before, and a break
//   when it has LAST (the end point of a curve is never tested for LAST,
//   xpath.rs:210-234);
// and the closing test of a walk-subpath runs at each break and at the last
// point, against the latest start. The warp scans 32 points at a time for
// the latest start and the piece slots. A path that is not well formed is
// walked serially by lane 0.
__global__ void k_walk_long(const double* __restrict__ pts, const uint8_t* __restrict__ flags,
                            const uint64_t* __restrict__ path_pt_off, uint32_t n_paths,
                            const double* __restrict__ mtx, uint2* __restrict__ pieces,
                            uint32_t* __restrict__ path_pieces, const uint8_t* __restrict__ rule,
                            uint32_t long_min) {
    __shared__ double m[6];
    if (threadIdx.x < 6) m[threadIdx.x] = mtx[threadIdx.x];
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < n_paths; p += warps) {
        const uint32_t off = static_cast<uint32_t>(path_pt_off[p]);
        const uint32_t n = static_cast<uint32_t>(path_pt_off[p + 1]) - off;
        if (n < long_min) continue;
        if (rule && rule[p] == RULE_HAIRLINE) {
            if (lane == 0) path_pieces[p] = 0;
            continue;
        }
        const uint8_t* F = flags + off;
        auto fl = [&](int64_t i) -> uint32_t { return (i >= 0 && i < static_cast<int64_t>(n)) ? F[i] : 0u; };
        // Well-formedness, 32 points at a time.
        bool ok = true;
        for (uint32_t b = 0; b < n && ok; b += 32) {
            const int64_t i = static_cast<int64_t>(b) + lane;
            bool good = true;
            if (i < static_cast<int64_t>(n)) {
                const uint32_t f0 = fl(i), fm1 = fl(i - 1), fm2 = fl(i - 2), fp1 = fl(i + 1), fp2 = fl(i + 2);
                const bool curve = f0 & PF_CURVE, pc = fm1 & PF_CURVE;
                const bool ctrl1 = curve && !pc, ctrl2 = curve && pc, endpt = !curve && pc;
                const bool lin = !curve && !endpt;
                const bool prev_lin = i >= 1 && !pc && !(fm2 & PF_CURVE);
                const bool start = (f0 & PF_FIRST) && (i == 0 || (prev_lin && (fm1 & PF_LAST)));
                if (i == 0 && !(f0 & PF_FIRST)) good = false;
                if ((f0 & PF_FIRST) && (curve || endpt)) good = false;
                if (ctrl1 && !(i >= 1 && i + 2 < static_cast<int64_t>(n) && (fp1 & PF_CURVE) && !(fp2 & PF_CURVE)))
                    good = false;
                if (ctrl2 && !(i >= 2 && !(fm2 & PF_CURVE))) good = false;
                if ((f0 & PF_FIRST) && (fm1 & PF_FIRST) && i >= 1) good = false;
                if (lin && !start && (f0 & PF_LAST) && i + 1 < static_cast<int64_t>(n) && !(fp1 & PF_FIRST))
                    good = false;
            }
            ok = __all_sync(0xffffffffu, good);
        }
        if (!ok) {
            // Serial walk of a path that is not well formed (the k_walk loop).
            if (lane == 0) {
                uint32_t slot = off, i = 0;
                while (i < n) {
                    if (F[i] & PF_FIRST) {
                        uint32_t sp = i, cur = i;
                        ++i;
                        while (i < n) {
                            const uint8_t f = F[i];
                            if (f & PF_CURVE) {
                                if (i + 2 >= n) break;
                                pieces[slot++] = make_uint2(off + cur, (PK_CURVE << 30) | (off + i));
                                cur = i + 2;
                                i += 3;
                            } else {
                                pieces[slot++] = make_uint2(off + cur, (PK_LINE << 30) | (off + i));
                                cur = i;
                                ++i;
                                if (f & PF_LAST) break;
                            }
                        }
                        double sx, sy, cx, cy;
                        transform(m, pts[2 * (off + sp)], pts[2 * (off + sp) + 1], sx, sy);
                        transform(m, pts[2 * (off + cur)], pts[2 * (off + cur) + 1], cx, cy);
                        if (fabs(dsub(cx, sx)) > 1e-10 || fabs(dsub(cy, sy)) > 1e-10)
                            pieces[slot++] = make_uint2(off + cur, (PK_CLOSE << 30) | (off + sp));
                    } else {
                        ++i;
                    }
                }
                path_pieces[p] = slot - off;
            }
            continue;
        }
        uint32_t slot_base = off;
        int64_t last_start = -1;
        for (uint32_t b = 0; b < n; b += 32) {
            const int64_t i = static_cast<int64_t>(b) + lane;
            const bool valid = i < static_cast<int64_t>(n);
            bool piece = false, is_curve = false, close_ev = false, start = false;
            if (valid) {
                const uint32_t f0 = fl(i), fm1 = fl(i - 1), fm2 = fl(i - 2);
                const bool curve = f0 & PF_CURVE, pc = fm1 & PF_CURVE;
                const bool ctrl1 = curve && !pc, endpt = !curve && pc;
                const bool lin = !curve && !endpt;
                const bool prev_lin = i >= 1 && !pc && !(fm2 & PF_CURVE);
                start = (f0 & PF_FIRST) && (i == 0 || (prev_lin && (fm1 & PF_LAST)));
                is_curve = ctrl1;
                piece = ctrl1 || (lin && !start);
                const bool brk = lin && !start && (f0 & PF_LAST);
                close_ev = brk || (i == static_cast<int64_t>(n) - 1);
            }
            // The latest start at or before each point.
            int64_t sp = start ? i : -1;
            for (int o = 1; o < 32; o <<= 1) {
                const int64_t t = __shfl_up_sync(0xffffffffu, sp, o);
                if (static_cast<int>(lane) >= o) sp = max(sp, t);
            }
            sp = max(sp, last_start);
            bool close = false;
            if (close_ev && sp >= 0) {
                double sx, sy, cx, cy;
                transform(m, pts[2 * (off + sp)], pts[2 * (off + sp) + 1], sx, sy);
                transform(m, pts[2 * (off + i)], pts[2 * (off + i) + 1], cx, cy);
                close = fabs(dsub(cx, sx)) > 1e-10 || fabs(dsub(cy, sy)) > 1e-10;
            }
            const uint32_t cnt = (piece ? 1u : 0u) + (close ? 1u : 0u);
            uint32_t incl = cnt;
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                if (static_cast<int>(lane) >= o) incl += t;
            }
            uint32_t at = slot_base + incl - cnt;
            if (piece)
                pieces[at++] = make_uint2(off + static_cast<uint32_t>(i - 1),
                                          ((is_curve ? PK_CURVE : PK_LINE) << 30) | (off + static_cast<uint32_t>(i)));
            if (close)
                pieces[at] = make_uint2(off + static_cast<uint32_t>(i), (PK_CLOSE << 30) | (off + static_cast<uint32_t>(sp)));
            slot_base += __shfl_sync(0xffffffffu, incl, 31);
            last_start = __shfl_sync(0xffffffffu, sp, 31);
        }
        if (lane == 0) path_pieces[p] = slot_base - off;
    }
}

// Pack each path's pieces (the first path_pieces[p] slots of its point range)
// densely at piece_off[p], with the AA-row clip of the path (its page, or the
// page and its clip rectangle; the lower bound is only stored with a clip).
__global__ void k_compact_pieces(const uint64_t* __restrict__ path_pt_off, const uint32_t* __restrict__ piece_off,
                                 uint32_t n_paths, const uint32_t* __restrict__ path_page,
                                 const uint32_t* __restrict__ page_h, const uint2* __restrict__ slots,
                                 uint2* __restrict__ pieces, uint32_t* __restrict__ piece_clip,
                                 const int4* __restrict__ path_clip, uint32_t* __restrict__ piece_clip_lo) {
    // One warp per path: its lanes copy the pieces (long stroke outlines have
    // thousands) in coalesced strides.
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < n_paths; p += warps) {
        const uint32_t src = static_cast<uint32_t>(path_pt_off[p]);
        const uint32_t dst = piece_off[p], n = piece_off[p + 1] - dst;
        uint32_t clip_hi = 4u * page_h[path_page[p]] - 1u, clip_lo = 0;
        if (path_clip) {
            const int4 cl = path_clip[p];
            clip_lo = static_cast<uint32_t>(cl.z);
            clip_hi = static_cast<uint32_t>(cl.w);
        }
        for (uint32_t k = lane; k < n; k += 32) {
            pieces[dst + k] = slots[src + k];
            piece_clip[dst + k] = clip_hi;
            if (piece_clip_lo) piece_clip_lo[dst + k] = clip_lo;
        }
    }
}

__device__ __forceinline__ void load_tpt(const double* pts, const double* m, uint32_t i, double& x, double& y) {
    transform(m, pts[2 * i], pts[2 * i + 1], x, y);
}

// Curves of more than this many segments are flattened by a warp each
// (k_seg_count_big / k_seg_write_big): thread-per-curve work is that long.
constexpr int CURVE_BIG = 32;

// Segments per piece slot. SPLIT: a curve with more than CURVE_BIG segments
// is counted 0 here and appended to big_list (big-curve count in
// ctr->big_curves) for k_seg_count_big.
// Register budgets (CTAs per SM the compiler must fit; 0: its own choice)
// of the thread-per-piece flatten kernels (128 threads) and k_path_bbox (256).
#ifndef RRB_SEG_CTAS
#define RRB_SEG_CTAS 0
#endif
#ifndef RRB_BBOX_CTAS
#define RRB_BBOX_CTAS 0
#endif
#if RRB_SEG_CTAS > 0
#define RRB_SEG_BOUNDS __launch_bounds__(128, RRB_SEG_CTAS)
#else
#define RRB_SEG_BOUNDS
#endif
#if RRB_BBOX_CTAS > 0
#define RRB_BBOX_BOUNDS __launch_bounds__(256, RRB_BBOX_CTAS)
#else
#define RRB_BBOX_BOUNDS
#endif

template <bool SPLIT>
__global__ void RRB_SEG_BOUNDS k_seg_count(const double* __restrict__ pts, const uint2* __restrict__ pieces, uint32_t n_slots,
                            const double* __restrict__ mtx, double flat_sq, uint32_t* __restrict__ counts,
                            uint32_t* __restrict__ big_list, BatchCounters* __restrict__ ctr) {
    __shared__ double m[6];
    if (threadIdx.x < 6) m[threadIdx.x] = mtx[threadIdx.x];
    __syncthreads();
    // Whole warps step together (blockDim is a multiple of 32), so the ballot
    // below sees all 32 lanes.
    for (uint32_t s0 = blockIdx.x * blockDim.x; s0 < n_slots; s0 += gridDim.x * blockDim.x) {
        const uint32_t s = s0 + threadIdx.x;
        const uint2 pc = s < n_slots ? pieces[s] : make_uint2(0u, 0u);
        uint32_t kind = pc.y >> 30;
        uint32_t c = 0;
        bool big = false;
        if (kind == PK_LINE || kind == PK_CLOSE) {
            c = 1;
        } else if (kind == PK_CURVE) {
            uint32_t i = pc.y & 0x3fffffffu;
            double x0, y0, x1, y1, x2, y2, x3, y3;
            load_tpt(pts, m, pc.x, x0, y0);
            load_tpt(pts, m, i, x1, y1);
            load_tpt(pts, m, i + 1, x2, y2);
            load_tpt(pts, m, i + 2, x3, y3);
            if (SPLIT) {
                c = static_cast<uint32_t>(flatten_count_capped(x0, y0, x1, y1, x2, y2, x3, y3, flat_sq, CURVE_BIG));
                big = c > static_cast<uint32_t>(CURVE_BIG);
                if (big) c = 0;
            } else {
                c = flatten_curve(x0, y0, x1, y1, x2, y2, x3, y3, flat_sq, [](double, double) {});
            }
        }
        if (s < n_slots) counts[s] = c;
        if (SPLIT) {
            const uint32_t bm = __ballot_sync(0xffffffffu, big);
            if (bm) {
                const int lead = __ffs(bm) - 1;
                uint32_t base = 0;
                if (static_cast<int>(threadIdx.x & 31) == lead) base = atomicAdd(&ctr->big_curves, __popc(bm));
                base = __shfl_sync(0xffffffffu, base, lead);
                if (big) big_list[base + __popc(bm & lanemask_lt())] = s;
            }
        }
    }
}

__device__ __forceinline__ CurveNode load_curve(const double* pts, const double* m, const uint2 pc) {
    const uint32_t i = pc.y & 0x3fffffffu;
    CurveNode r;
    load_tpt(pts, m, pc.x, r.c0x, r.c0y);
    load_tpt(pts, m, i, r.c1x, r.c1y);
    load_tpt(pts, m, i + 1, r.c2x, r.c2y);
    load_tpt(pts, m, i + 2, r.r3x, r.r3y);
    return r;
}

__device__ __forceinline__ bool curve_root_in_range(const CurveNode& r) {
    return curve_in_range(r.c0x, r.c0y, r.c1x, r.c1y, r.c2x, r.c2y, r.r3x, r.r3y);
}

// One warp per big curve (k_seg_count's big_list): each lane counts the
// leaves of its subtree (curve_lane_flatten); the sum is the curve's count.
constexpr int CURVE_LANES = 32;  // lanes per big curve; each lane's count is at most CURVE_LANE_SLOTS

// The big-curve kernels run 128-thread CTAs; RRB_BIG_CURVE_CTAS > 0 asks the
// compiler to fit that many per SM (a register budget). 8 (64 registers)
// took the mixed batch's flatten + records from 15.9 to 14.8 ms against the
// unbounded 96 registers; 6 (80 registers) gave 15.4.
#ifndef RRB_BIG_CURVE_CTAS
#define RRB_BIG_CURVE_CTAS 8
#endif
#if RRB_BIG_CURVE_CTAS > 0
#define RRB_BIG_CURVE_BOUNDS __launch_bounds__(128, RRB_BIG_CURVE_CTAS)
#else
#define RRB_BIG_CURVE_BOUNDS
#endif

__global__ void RRB_BIG_CURVE_BOUNDS k_seg_count_big(const double* __restrict__ pts, const uint2* __restrict__ pieces,
                                const double* __restrict__ mtx, double flat_sq, const uint32_t* __restrict__ big_list,
                                const BatchCounters* __restrict__ ctr, uint32_t* __restrict__ counts,
                                uint8_t* __restrict__ lane_cnt, uint32_t lane_cap) {
    __shared__ double m[6];
    if (threadIdx.x < 6) m[threadIdx.x] = mtx[threadIdx.x];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const uint32_t n_big = ctr->big_curves;
    const uint32_t warp_g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t q = warp_g; q < n_big; q += nwarps) {
        const uint32_t s = big_list[q];
        const CurveNode root = load_curve(pts, m, pieces[s]);
        auto none = [](double, double) {};
        double cx, cy;
        int c = curve_root_in_range(root) ? curve_lane_flatten<true>(root, lane, flat_sq, cx, cy, none)
                                          : curve_lane_flatten<false>(root, lane, flat_sq, cx, cy, none);
        if (q < lane_cap) lane_cnt[static_cast<uint64_t>(q) * CURVE_LANES + lane] = static_cast<uint8_t>(c);
        for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if (lane == 0) counts[s] = static_cast<uint32_t>(c);
    }
}

// Edge records per piece slot, at edge_off[slot]. SPLIT: curves with more
// than CURVE_BIG segments are left to k_seg_write_big.
template <bool SPLIT>
__global__ void RRB_SEG_BOUNDS k_seg_write(const double* __restrict__ pts, const uint2* __restrict__ pieces, uint32_t n_slots,
                            const double* __restrict__ mtx, double flat_sq, const uint32_t* __restrict__ edge_off,
                            uint32_t edge_cap, Edge* __restrict__ edges,
                            const uint32_t* __restrict__ slot_clip_hi, const uint32_t* __restrict__ slot_clip_lo) {
    __shared__ double m[6];
    if (threadIdx.x < 6) m[threadIdx.x] = mtx[threadIdx.x];
    __syncthreads();
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n_slots; s += gridDim.x * blockDim.x) {
        uint2 pc = pieces[s];
        uint32_t kind = pc.y >> 30;
        if (kind == PK_NONE) continue;
        uint32_t base = edge_off[s];
        if (SPLIT && kind == PK_CURVE && edge_off[s + 1] - base > static_cast<uint32_t>(CURVE_BIG)) continue;
        int32_t chi = static_cast<int32_t>(slot_clip_hi[s]);
        const int32_t clo = slot_clip_lo ? static_cast<int32_t>(slot_clip_lo[s]) : 0;
        uint32_t j = pc.y & 0x3fffffffu;
        double x0, y0;
        load_tpt(pts, m, pc.x, x0, y0);
        if (kind == PK_LINE || kind == PK_CLOSE) {
            double x1, y1;
            load_tpt(pts, m, j, x1, y1);
            if (base < edge_cap) edges[base] = make_edge(x0, y0, x1, y1, clo, chi);
        } else {
            double x1, y1, x2, y2, x3, y3;
            load_tpt(pts, m, j, x1, y1);
            load_tpt(pts, m, j + 1, x2, y2);
            load_tpt(pts, m, j + 2, x3, y3);
            double cx = x0, cy = y0;
            uint32_t k = base;
            flatten_curve(x0, y0, x1, y1, x2, y2, x3, y3, flat_sq, [&](double fx, double fy) {
                if (k < edge_cap) edges[k] = make_edge(cx, cy, fx, fy, clo, chi);
                ++k;
                cx = fx;
                cy = fy;
            });
        }
    }
}

// One warp per big curve: each lane's count of its subtree's leaves (kept by
// k_seg_count_big for the first lane_cap curves, counted again for the
// rest), an exclusive scan over the lanes places them, and each lane writes
// the edge records of its leaves from its subtree's start point on.
__global__ void RRB_BIG_CURVE_BOUNDS k_seg_write_big(const double* __restrict__ pts, const uint2* __restrict__ pieces,
                                const double* __restrict__ mtx, double flat_sq, const uint32_t* __restrict__ big_list,
                                const BatchCounters* __restrict__ ctr, const uint32_t* __restrict__ edge_off,
                                uint32_t edge_cap, Edge* __restrict__ edges,
                                const uint32_t* __restrict__ slot_clip_hi, const uint32_t* __restrict__ slot_clip_lo,
                                const uint8_t* __restrict__ lane_cnt, uint32_t lane_cap) {
    __shared__ double m[6];
    if (threadIdx.x < 6) m[threadIdx.x] = mtx[threadIdx.x];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const uint32_t n_big = ctr->big_curves;
    const uint32_t warp_g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t q = warp_g; q < n_big; q += nwarps) {
        const uint32_t s = big_list[q];
        const CurveNode root = load_curve(pts, m, pieces[s]);
        const bool in_range = curve_root_in_range(root);
        const int32_t chi = static_cast<int32_t>(slot_clip_hi[s]);
        const int32_t clo = slot_clip_lo ? static_cast<int32_t>(slot_clip_lo[s]) : 0;
        auto none = [](double, double) {};
        double cx = 0.0, cy = 0.0;
        int mine;
        if (q < lane_cap) mine = lane_cnt[static_cast<uint64_t>(q) * CURVE_LANES + lane];
        else mine = in_range ? curve_lane_flatten<true>(root, lane, flat_sq, cx, cy, none)
                             : curve_lane_flatten<false>(root, lane, flat_sq, cx, cy, none);
        int incl = mine;
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        uint32_t k = edge_off[s] + static_cast<uint32_t>(incl - mine);
        auto emit = [&](double fx, double fy) {
            if (k < edge_cap) edges[k] = make_edge(cx, cy, fx, fy, clo, chi);
            ++k;
            cx = fx;
            cy = fy;
        };
        if (mine) {
            // The flatten sets (cx, cy) to the lane's start point before its
            // first leaf is emitted.
            if (in_range) curve_lane_flatten<true>(root, lane, flat_sq, cx, cy, emit);
            else curve_lane_flatten<false>(root, lane, flat_sq, cx, cy, emit);
        }
    }
}

// Per-path offsets and page indices of a wave (a run of pages of a larger
// batch), rebased to the wave's first point and first page.
__global__ void k_rebase_paths(const uint64_t* __restrict__ off_in, uint64_t* __restrict__ off_out, uint64_t pt_base,
                               const uint32_t* __restrict__ page_in, uint32_t* __restrict__ page_out, uint32_t pg_base,
                               uint32_t n_paths) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= n_paths; i += gridDim.x * blockDim.x) {
        off_out[i] = off_in[i] - pt_base;
        if (i < n_paths) page_out[i] = page_in[i] - pg_base;
    }
}

// ---------------------------------------------------------------------------
// Device-wide exclusive scan of u32 (three phases, host-known n).
// out[i] = sum(in[0..i)), out[n] = total. in and out may alias.
// ---------------------------------------------------------------------------
constexpr int SCAN_THREADS = 512;
constexpr int SCAN_MAX_BLOCKS = 1024;

__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* sh, uint32_t& total) {
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[warp] = x;
    __syncthreads();
    int nw = blockDim.x >> 5;
    if (warp == 0) {
        uint32_t w = lane < nw ? sh[lane] : 0u;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < nw) sh[lane] = w;
    }
    __syncthreads();
    uint32_t wp = warp ? sh[warp - 1] : 0u;
    total = sh[nw - 1];
    __syncthreads();
    return wp + x - v;
}

__global__ void k_scan_reduce(const uint32_t* __restrict__ in, uint32_t n, uint32_t per_block,
                              uint32_t* __restrict__ block_sums) {
    __shared__ uint32_t sh[32];
    uint32_t b0 = blockIdx.x * per_block;
    uint32_t b1 = min(n, b0 + per_block);
    uint32_t acc = 0;
    for (uint32_t i = b0 + threadIdx.x; i < b1; i += blockDim.x) acc += in[i];
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
        block_sums[blockIdx.x] = t;
    }
}

__global__ void k_scan_blocks(uint32_t* __restrict__ block_sums, uint32_t nb) {
    __shared__ uint32_t sh[32];
    uint32_t v = threadIdx.x < nb ? block_sums[threadIdx.x] : 0u;
    uint32_t total;
    uint32_t ex = block_excl_scan(v, sh, total);
    if (threadIdx.x < nb) block_sums[threadIdx.x] = ex;
    if (threadIdx.x == 0) block_sums[SCAN_MAX_BLOCKS] = total;
}

__global__ void k_scan_down(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint32_t n,
                            uint32_t per_block, const uint32_t* __restrict__ block_sums) {
    __shared__ uint32_t sh[32];
    uint32_t b0 = blockIdx.x * per_block;
    uint32_t b1 = min(n, b0 + per_block);
    uint32_t carry = block_sums[blockIdx.x];
    for (uint32_t t0 = b0; t0 < b1; t0 += blockDim.x) {
        uint32_t i = t0 + threadIdx.x;
        uint32_t v = i < b1 ? in[i] : 0u;
        uint32_t total;
        uint32_t ex = block_excl_scan(v, sh, total);
        if (i < b1) out[i] = carry + ex;
        carry += total;
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = block_sums[SCAN_MAX_BLOCKS];
}

// ---------------------------------------------------------------------------
// Path bounding box (XPathScanner::new, scanner/mod.rs:131-180): one warp per
// path reduces its edges to the AA row range and AA column range, then maps
// them to the pixel rectangle the row map can touch. path_visit (optional,
// read under the as-shipped row map only) gives per path the pixel rows the
// shipped driver loop visits when they come from another path's AA range.
// ---------------------------------------------------------------------------
__global__ void RRB_BBOX_BOUNDS k_path_bbox(const uint32_t* __restrict__ piece_off, const uint32_t* __restrict__ edge_off,
                            const Edge* __restrict__ edges, uint32_t n_paths, const uint8_t* __restrict__ rule,
                            const uint8_t* __restrict__ gray, const uint8_t* __restrict__ alpha,
                            const uint32_t* __restrict__ path_page, const uint32_t* __restrict__ page_w,
                            const uint32_t* __restrict__ page_h, int rowmap, PathInfo* __restrict__ info,
                            uint32_t* __restrict__ path_groups, uint32_t* __restrict__ path_chunks,
                            int chunk_rows, BatchCounters* __restrict__ ctr, int32_t* __restrict__ gmin,
                            int32_t* __restrict__ gmax, const int4* __restrict__ path_clip,
                            const int2* __restrict__ path_visit) {
    int lane = threadIdx.x & 31;
    uint32_t warp_g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t p = warp_g; p < n_paths; p += nwarps) {
        uint32_t eb = edge_off[piece_off[p]], ee = edge_off[piece_off[p + 1]];
        int32_t y0 = INT32_MAX, y1 = INT32_MIN, xl = INT32_MAX, xh = INT32_MIN;
        unsigned long long raw = 0;
        bool axis_only = true;
        // Aligned groups of 32 edges: one group per iteration, its row range
        // merged into gmin/gmax (atomically: a group can straddle two paths).
        for (uint32_t base4 = eb & ~31u; base4 < ee; base4 += 128) {
          // Four groups' loads in flight before any is reduced.
          Edge e4[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
              const uint32_t j = base4 + 32 * u + lane;
              if (j >= eb && j < ee) e4[u] = edges[j];
              else e4[u].flags = EF_EMPTY;
          }
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const uint32_t base = base4 + 32 * u;
            if (base >= ee) break;
            int32_t g0 = INT32_MAX, g1 = INT32_MIN;
            {
                const Edge e = e4[u];
                if (!(e.flags & EF_EMPTY)) {
                    int32_t lo, hi;
                    edge_xrange(e, lo, hi);
                    raw += static_cast<unsigned long long>(e.row1 - e.row0 + 1);
                    y0 = min(y0, e.row0);
                    y1 = max(y1, e.row1);
                    xl = min(xl, lo);
                    xh = max(xh, hi);
                    g0 = e.row0;
                    g1 = e.row1;
                }
            }
            for (int o = 16; o; o >>= 1) {
                g0 = min(g0, __shfl_xor_sync(0xffffffffu, g0, o));
                g1 = max(g1, __shfl_xor_sync(0xffffffffu, g1, o));
            }
            axis_only &= __all_sync(0xffffffffu, (e4[u].flags & EF_EMPTY) ||
                                                     (e4[u].flags & EF_KIND_MASK) != EK_SLOPED);
            if (lane == 0 && g0 <= g1) {
                atomicMin(&gmin[base >> 5], g0);
                atomicMax(&gmax[base >> 5], g1);
            }
          }
        }
        for (int o = 16; o; o >>= 1) {
            y0 = min(y0, __shfl_xor_sync(0xffffffffu, y0, o));
            y1 = max(y1, __shfl_xor_sync(0xffffffffu, y1, o));
            xl = min(xl, __shfl_xor_sync(0xffffffffu, xl, o));
            xh = max(xh, __shfl_xor_sync(0xffffffffu, xh, o));
            raw += __shfl_xor_sync(0xffffffffu, raw, o);
        }
        if (lane == 0) {
            if (raw) atomicAdd(&ctr->raw_entries, raw);
            if (y0 <= y1) atomicAdd(&ctr->aa_rows, static_cast<unsigned long long>(y1 - y0 + 1));
            uint32_t pg = path_page[p];
            int32_t W = static_cast<int32_t>(page_w[pg]), H = static_cast<int32_t>(page_h[pg]);
            PathInfo pi;
            pi.e_begin = eb;
            pi.e_end = ee;
            pi.paint = uint32_t(gray[p]) | (uint32_t(alpha[p]) << 8) | (uint32_t(rule[p] ? 1 : 0) << 16);
            pi.page = pg;
            pi.run_off = pi.run_cnt = 0;
            pi.bx0 = 1;
            pi.bx1 = 0;
            pi.by0 = 1;
            pi.by1 = 0;
            const bool recti = axis_only && y0 <= y1 && ee - eb <= RECTI_MAX_EDGES;
            if (recti) pi.paint |= PI_RECTI;
            uint32_t rows = 0, groups = 0;
            if (y0 <= y1) {
                pi.y0 = y0;
                pi.y1 = y1;
                rows = static_cast<uint32_t>(y1 - (y0 & ~3) + 1);     // rows of the 4-aligned chunks
                groups = static_cast<uint32_t>((y1 >> 2) - (y0 >> 2) + 1);
                // Pixel columns: spans cover AA columns [max(x0, lo), min(x1+1, hi)).
                const int4 clp = path_clip_of(path_clip, p, 4 * W, 4 * H);
                int32_t cl = max(xl, clp.x), ch = min(xh, clp.y - 1);
                pi.px0 = cl >> 2;
                pi.px1 = ch >> 2;
                if (xh < clp.x || xl >= clp.y || clp.x >= clp.y) {
                    pi.px0 = 1;
                    pi.px1 = 0;
                }
                // Pixel rows under the row map.
                if (rowmap == 0) {
                    pi.py0 = y0 >> 2;
                    pi.py1 = y1 >> 2;
                } else {
                    pi.py0 = y0 >> 2;
                    int32_t t = y1 - 12;
                    pi.py1 = t >= 0 ? (t >> 4) : -1;
                    // The shipped loop visits the pixel rows of another path's AA
                    // range (a clip path drawn on its fill's rows): those rows,
                    // up to the last one with content of this path.
                    if (path_visit && path_visit[p].x != INT32_MIN) {  // INT32_MIN: the path's own rows
                        pi.py0 = path_visit[p].x;
                        pi.py1 = min(pi.py1, path_visit[p].y);
                    }
                }
                pi.py0 = max(pi.py0, 0);
                pi.py1 = min(pi.py1, H - 1);
            } else {
                pi.y0 = 1;
                pi.y1 = 0;
                pi.px0 = 1;
                pi.px1 = 0;
                pi.py0 = 1;
                pi.py1 = 0;
            }
            info[p] = pi;
            // Rectilinear paths skip the row stage: k_recti builds their row runs.
            path_groups[p] = recti ? 0u : groups;
            path_chunks[p] = recti ? 0u : (rows + chunk_rows - 1) / chunk_rows;
        }
    }
}

// ---------------------------------------------------------------------------
// Supertile binning: for each supertile of a page, the ordered list of paths
// of that page whose pixel rectangle overlaps it. One warp per supertile
// ballots over 32 paths at a time, so list order is path order.
// ---------------------------------------------------------------------------
struct PageGeom {
    uint32_t w, h;
    uint32_t path_begin, path_end;
    uint32_t tile_base, ntx;       // tiles of this page start at tile_base, ntx per row
    uint32_t super_base, nsx;      // supertiles start at super_base, nsx per row
    uint32_t work_base, nblk;      // binning work items: (supertile, block of BIN_BLOCK paths)
    uint64_t offset;               // page byte offset in the arena
};

constexpr uint32_t BIN_BLOCK = 2048;  // paths per binning work item

__device__ __forceinline__ uint32_t find_page_by(const PageGeom* pg, uint32_t n_pages, uint32_t idx, bool super) {
    uint32_t lo = 0, hi = n_pages;  // last page with base <= idx
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        uint32_t b = super ? pg[mid].super_base : pg[mid].tile_base;
        if (b <= idx) lo = mid;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ uint32_t find_page_work(const PageGeom* pg, uint32_t n_pages, uint32_t q) {
    uint32_t lo = 0, hi = n_pages;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (pg[mid].work_base <= q) lo = mid;
        else hi = mid;
    }
    return lo;
}

// One warp per work item (supertile s, block b of the page's paths): the
// paths of block b that overlap s, in path order. Work items of one
// supertile are consecutive, so after an exclusive scan of the counts the
// supertile's list is the contiguous range [off(s,0), off(s,nblk)).
// The writing pass also records in super_start[s] one past the list position
// of the last opaque path whose solid box holds the whole supertile (clipped
// to the page): compositing of every tile of s can start there, since that
// layer sets each of its pixels to the path's colour (super_start zeroed
// beforehand; 0 = no such path).
template <bool WRITE>
__global__ void k_super_bin(const PathInfo* __restrict__ info, const PageGeom* __restrict__ pages, uint32_t n_pages,
                            uint32_t n_work, int stw, int sth, uint32_t* __restrict__ work_count,
                            const uint32_t* __restrict__ work_off, uint32_t* __restrict__ super_list,
                            uint32_t* __restrict__ super_start) {
    int lane = threadIdx.x & 31;
    uint32_t warp_g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t q = warp_g; q < n_work; q += nwarps) {
        uint32_t pg = find_page_work(pages, n_pages, q);
        PageGeom G = pages[pg];
        uint32_t local = q - G.work_base;
        uint32_t sl = local / G.nblk, blk = local % G.nblk;
        int32_t sx = static_cast<int32_t>(sl % G.nsx), sy = static_cast<int32_t>(sl / G.nsx);
        int32_t x0 = sx * stw, x1 = x0 + stw - 1, y0 = sy * sth, y1 = y0 + sth - 1;
        uint32_t pb = G.path_begin + blk * BIN_BLOCK;
        uint32_t pe = min(G.path_end, pb + BIN_BLOCK);
        uint32_t cnt = 0;
        uint32_t base = WRITE ? work_off[q] : 0u;
        const int32_t cx1 = min(x1, static_cast<int32_t>(G.w) - 1), cy1 = min(y1, static_cast<int32_t>(G.h) - 1);
        uint32_t opaque_end = 0;  // one past the list position of the last opaque full layer seen
        for (uint32_t j = pb; j < pe; j += 32) {
            uint32_t qq = j + lane;
            bool hit = false;
            if (qq < pe) {
                static_assert(sizeof(PathInfo) % 16 == 0 && offsetof(PathInfo, px0) == 0, "int4 load of the rectangle");
                const int4 r = *reinterpret_cast<const int4*>(&info[qq]);  // px0, px1, py0, py1
                hit = r.x <= r.y && r.z <= r.w && r.x <= x1 && r.y >= x0 && r.z <= y1 && r.w >= y0;
            }
            uint32_t m = __ballot_sync(0xffffffffu, hit);
            if (WRITE && hit) {
                const uint32_t pos = base + cnt + __popc(m & lanemask_lt());
                super_list[pos] = qq;
                static_assert(offsetof(PathInfo, paint) == 32 && offsetof(PathInfo, bx0) == 48, "int4 loads");
                const uint32_t paint = reinterpret_cast<const uint4*>(&info[qq])[2].x;
                if (((paint >> 8) & 0xffu) == 255u) {
                    const int4 b = reinterpret_cast<const int4*>(&info[qq])[3];  // bx0, bx1, by0, by1
                    if (b.x <= x0 && b.y >= cx1 && b.z <= y0 && b.w >= cy1) opaque_end = max(opaque_end, pos + 1);
                }
            }
            cnt += __popc(m);
        }
        if (!WRITE && lane == 0) work_count[q] = cnt;
        if (WRITE) {
            for (int o = 16; o; o >>= 1) opaque_end = max(opaque_end, __shfl_xor_sync(0xffffffffu, opaque_end, o));
            if (lane == 0 && opaque_end) atomicMax(&super_start[G.super_base + sl], opaque_end);
        }
    }
}

// ---------------------------------------------------------------------------
// Row stage: one warp per chunk of 32 consecutive AA rows of one path; lane =
// row. The path's edges are visited in order, 32 at a time: a ballot selects
// those overlapping the chunk and the set bits are walked in ascending order,
// so each row sees its entries in segment order and the write_intersect merge
// (merge only with the last entry written to the row) is reproduced exactly.
// The merged list lives in shared memory (KCAP entries per row); rows that
// overflow go to k_rows_slow.
// ---------------------------------------------------------------------------
constexpr int ROWS_WARPS = 8;

// 32x32 bit-matrix transpose across a warp: on entry bit j of lane i is
// A[i][j]; on exit bit j of lane i is A[j][i]. Five butterfly stages, each
// swapping the off-diagonal s x s blocks with the partner lane i ^ s.
__device__ __forceinline__ uint32_t warp_transpose32(uint32_t x, int lane) {
    const uint32_t LOW[5] = {0x0000FFFFu, 0x00FF00FFu, 0x0F0F0F0Fu, 0x33333333u, 0x55555555u};
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const int s = 16 >> k;
        const uint32_t lo = LOW[k];
        const uint32_t p = __shfl_xor_sync(0xffffffffu, x, s);
        x = (lane & s) ? ((x & ~lo) | ((p & ~lo) >> s)) : ((x & lo) | ((p & lo) << s));
    }
    return x;
}

__host__ __device__ __forceinline__ int32_t sat_inc(int32_t v) { return v == INT32_MAX ? v : v + 1; }

// Winding walk of render_aa_line (scanner/mod.rs:393-467) for one AA row over
// its sorted entries, emitting the union of the covered spans clamped to the
// clip's AA columns [lo, hi) (the page: [0, aa_width); an unclosed span ends
// at aa_width as in the reference) in place over the entry arrays. Returns the
// span count.
template <typename Get, typename Put>
__host__ __device__ __forceinline__ int walk_row(int n, int32_t mask, int32_t aa_width, int32_t lo, int32_t hi,
                                                 Get get, Put put, uint32_t& nonterm) {
    int32_t count = 0, xx = 0;
    int i = 0, ns = 0;
    bool have = false;
    int32_t cs = 0, ce = 0;
    while (i < n || (count & mask) != 0) {
        if ((count & mask) == 0) {
            if (i >= n) break;
            int32_t x0, x1, c;
            get(i, x0, x1, c);
            xx = x0;
            count = static_cast<int32_t>(static_cast<uint32_t>(count) + static_cast<uint32_t>(c));
            ++i;
            continue;
        }
        int32_t span_x1;
        bool ran_out = false;
        for (;;) {
            if (i >= n) {
                span_x1 = aa_width;
                ran_out = true;
                break;
            }
            int32_t x0, x1, c;
            get(i, x0, x1, c);
            count = static_cast<int32_t>(static_cast<uint32_t>(count) + static_cast<uint32_t>(c));
            int32_t end = static_cast<int32_t>(static_cast<uint32_t>(x1) + 1u);
            ++i;
            if ((count & mask) == 0) {
                span_x1 = end;
                break;
            }
        }
        int32_t bx0 = max(xx, lo);
        int32_t bx1 = max(min(span_x1, hi), lo);
        if (bx0 < bx1) {
            if (have && bx0 <= ce) {
                ce = max(ce, bx1);
            } else {
                if (have) put(ns++, cs, ce);
                cs = bx0;
                ce = bx1;
                have = true;
            }
        }
        xx = span_x1;
        if (ran_out) {
            ++nonterm;
            break;
        }
    }
    if (have) put(ns++, cs, ce);
    return ns;
}

// Coverage cells of one pixel row from the sorted, disjoint span lists of its
// four AA sub-rows (draw_aa_line's per-pixel nibble popcount, fill/mod.rs:
// 344-401, computed from spans): the coverage of pixel x is the number of
// (sub-row, AA column) pairs covered in columns [4x, 4x+4), 0..16. Boundaries
// of all four lists are merged in column order; pixels that contain a
// boundary get their own cell, the pixels between two such pixels share one
// run cell of coverage 4 x depth. Cells come out sorted by x, disjoint, with
// coverage > 0; at most one per boundary plus one run per gap, i.e. at most
// 2 x (number of boundaries). Cell: x0 (bits 0-13) | len-1 (14-27) | cov-1 (28-31).
template <typename Bound, typename Put>
__host__ __device__ __forceinline__ int sweep_cells(const int (&n)[4], Bound bound, Put put) {
    // Each list's next boundary (INT32_MAX once the list is used up) and its
    // index (bit 0: a span end). The sweep takes the least head, lowest list
    // first among equal ones, and reloads only that list's head.
    int bi[4];
    int32_t hd[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        bi[k] = 0;
        hd[k] = n[k] > 0 ? bound(k, 0, false) : INT32_MAX;
    }
    int depth = 0, nc = 0;
    int32_t prev_px = -1;
    auto next = [&](int& kmin) -> int32_t {
        int32_t best = hd[0];
        kmin = 0;
#pragma unroll
        for (int k = 1; k < 4; ++k) {
            if (hd[k] < best) {
                best = hd[k];
                kmin = k;
            }
        }
        if (best == INT32_MAX) kmin = -1;
        return best;
    };
    auto advance = [&](int kk) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (k == kk) {
                depth += (bi[k] & 1) ? -1 : 1;
                ++bi[k];
                hd[k] = bi[k] < 2 * n[k] ? bound(k, bi[k] >> 1, (bi[k] & 1) != 0) : INT32_MAX;
            }
        }
    };
    auto emit = [&](int32_t x0, int32_t len, int32_t cov) {
        put(nc++, static_cast<uint32_t>(x0) | (static_cast<uint32_t>(len - 1) << 14) |
                      (static_cast<uint32_t>(cov - 1) << 28));
    };
    int k;
    int32_t b = next(k);
    while (k >= 0) {
        const int32_t px = b >> 2;
        if (depth > 0 && px - 1 >= prev_px + 1) emit(prev_px + 1, px - 1 - prev_px, 4 * depth);
        int32_t col = 4 * px, cov = 0;
        while (k >= 0 && b < 4 * px + 4) {
            cov += depth * (b - col);
            col = b;
            advance(k);
            b = next(k);
        }
        cov += depth * (4 * px + 4 - col);
        if (cov > 0) emit(px, 1, cov);
        prev_px = px;
    }
    return nc;
}

// Merged Intersect lists of up to 32 consecutive AA rows of one path, one
// row per lane, in shared memory: entry k of lane l at [k * LS + l].
//
// The path's edges are visited in order, 32 at a time: a ballot finds those
// overlapping [lo, hi], a 32x32 bit transpose gives each lane the edges that
// cover its row, and each lane folds its entries in edge order, so every row
// sees its entries in segment order and the write_intersect merge (merge only
// with the last entry written to the row, scanner/mod.rs:600-642) is exact.
// Groups of 32 edges whose row range misses [lo, hi] are skipped from the
// per-group bounds gmin/gmax. GS groups are staged at once (sedge holds GS x
// 32 edges) and folded in one loop, so the warp runs as many fold steps as
// its busiest row has entries in those groups together, not per group.
// Returns the entry count; entries past K are counted but not stored (the
// caller treats n > K as overflow).
template <int K, int LS, int GS = 1>
__device__ __forceinline__ int gather_row(const PathInfo& P, int32_t lo, int32_t hi, int32_t r, bool valid,
                                          const Edge* __restrict__ edges, const int32_t* __restrict__ gmin,
                                          const int32_t* __restrict__ gmax, Edge* sedge, int32_t* x0s,
                                          int32_t* x1s, int32_t* cns, int lane) {
    static_assert(GS == 1 || GS == 2, "one or two staged edge groups");
    int n = 0;
    bool has_last = false;
    int32_t lx0 = 0, lx1 = 0, lc = 0;
    auto fold = [&](int bb) {
        const Edge E = sedge[bb];  // two 16-byte shared loads
        int32_t elo, ehi, ec;
        edge_entry(E, r, elo, ehi, ec);
        if (has_last && sat_inc(lx1) >= elo && lx0 <= sat_inc(ehi)) {
            lc = static_cast<int32_t>(static_cast<uint32_t>(lc) + static_cast<uint32_t>(ec));
            lx0 = min(lx0, elo);
            lx1 = max(lx1, ehi);
        } else {
            if (has_last) {
                if (n < K) {
                    x0s[n * LS + lane] = lx0;
                    x1s[n * LS + lane] = lx1;
                    cns[n * LS + lane] = lc;
                }
                ++n;
            }
            lx0 = elo;
            lx1 = ehi;
            lc = ec;
            has_last = true;
        }
    };
    // 32 groups' bounds at a time, one per lane: the warp visits only the
    // groups whose rows meet [lo, hi], in ascending order.
    for (uint32_t gb = P.e_begin >> 5; 32ull * gb < P.e_end; gb += 32) {
      const uint32_t gl = gb + lane;
      const bool g_hit = 32ull * gl < P.e_end && !(gmin[gl] > hi || gmax[gl] < lo);
      uint32_t gm = __ballot_sync(0xffffffffu, g_hit);
      while (gm) {
        uint32_t mine[GS];
#pragma unroll
        for (int s = 0; s < GS; ++s) {
            mine[s] = 0;
            // The next group with an edge on [lo, hi] goes to slot s.
            while (gm) {
                const uint32_t eb = (gb + static_cast<uint32_t>(__ffs(gm) - 1)) << 5;
                gm &= gm - 1;
                const uint32_t j = eb + lane;
                Edge e;
                bool hit = false;
                if (j >= P.e_begin && j < P.e_end) {
                    e = edges[j];
                    hit = !(e.flags & EF_EMPTY) && e.row0 <= hi && e.row1 >= lo;
                }
                if (!__any_sync(0xffffffffu, hit)) continue;
                uint32_t rows_of_edge = 0;
                if (hit) {
                    const int q = 32 * s + lane;
                    sedge[q] = e;
                    const int32_t ra = max(e.row0, lo) - lo, rb = min(e.row1, hi) - lo;
                    rows_of_edge = (0xffffffffu >> (31 - rb)) & (0xffffffffu << ra);
                }
                mine[s] = warp_transpose32(rows_of_edge, lane);
                break;
            }
            if (!valid) mine[s] = 0;
        }
        __syncwarp();
        if constexpr (GS == 1) {
            uint32_t m = mine[0];
            while (m) {
                const int bb = __ffs(m) - 1;
                m &= m - 1;
                fold(bb);
            }
        } else {
            // Slot 0's group precedes slot 1's: bit order is edge order.
            uint64_t m = (static_cast<uint64_t>(mine[1]) << 32) | mine[0];
            while (m) {
                const int bb = __ffsll(static_cast<long long>(m)) - 1;
                m &= m - 1;
                fold(bb);
            }
        }
        __syncwarp();
      }
    }
    if (has_last) {
        if (n < K) {
            x0s[n * LS + lane] = lx0;
            x1s[n * LS + lane] = lx1;
            cns[n * LS + lane] = lc;
        }
        ++n;
    }
    return n;
}

// sort_unstable_by_key(x0) on a lane's list (stable insertion sort, as Rust
// std sorts slices of up to 20 elements) followed by the render_aa_line
// winding walk; the row's union of spans replaces the list in place.
template <int LS>
__device__ __forceinline__ int sort_and_walk(int n, int32_t mask, int32_t aa_width, int32_t lo, int32_t hi,
                                             int32_t* x0s, int32_t* x1s,
                                             int32_t* cns, int lane, uint32_t& nonterm) {
    for (int a = 1; a < n; ++a) {
        const int32_t t0 = x0s[a * LS + lane], t1 = x1s[a * LS + lane], tc = cns[a * LS + lane];
        int b = a;
        while (b > 0 && t0 < x0s[(b - 1) * LS + lane]) {
            x0s[b * LS + lane] = x0s[(b - 1) * LS + lane];
            x1s[b * LS + lane] = x1s[(b - 1) * LS + lane];
            cns[b * LS + lane] = cns[(b - 1) * LS + lane];
            --b;
        }
        x0s[b * LS + lane] = t0;
        x1s[b * LS + lane] = t1;
        cns[b * LS + lane] = tc;
    }
    return walk_row(
        n, mask, aa_width, lo, hi,
        [&](int i, int32_t& x0, int32_t& x1, int32_t& cc) {
            x0 = x0s[i * LS + lane];
            x1 = x1s[i * LS + lane];
            cc = cns[i * LS + lane];
        },
        [&](int k, int32_t s0, int32_t e0) {
            x0s[k * LS + lane] = s0;
            x1s[k * LS + lane] = e0;
        },
        nonterm);
}

// Owner path of every row chunk (one warp per path writes its chunk range).
__global__ void k_chunk_paths(const uint32_t* __restrict__ chunk_off, uint32_t n_paths,
                              uint32_t* __restrict__ chunk_path) {
    const int lane = threadIdx.x & 31;
    const uint32_t warp_g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t p = warp_g; p < n_paths; p += nwarps)
        for (uint32_t c = chunk_off[p] + lane; c < chunk_off[p + 1]; c += 32) chunk_path[c] = p;
}

// Row stage: one warp per chunk of 32 AA rows of one path, lane = row.
// Chunks start on a multiple of 4 AA rows, so lanes 4k..4k+3 are the four
// sub-rows of one pixel row; their spans are merged into coverage cells by
// lane 4k. Pixel rows with a list over KCAP go to k_groups_mid.
// k_rows' shared memory (dynamic: it exceeds the 48 KB of static shared
// memory): per warp the three entry lists, GS staged edge groups (32 edge
// records of 32 bytes each) and the span counts. A block stages
// WARPS x GS x 32 edges at a time.
template <int KCAP, int WARPS, int GS = 2>
constexpr size_t rows_smem_bytes() {
    return sizeof(int32_t) * WARPS * (3 * KCAP * 32 + 8 * 32 * GS + 32);
}

template <int KCAP, int WARPS = ROWS_WARPS, int GS = 2>
__global__ void __launch_bounds__(WARPS * 32) k_rows(
    const PathInfo* __restrict__ info, const uint32_t* __restrict__ chunk_off, const uint32_t* __restrict__ group_off,
    const Edge* __restrict__ edges, const int32_t* __restrict__ gmin, const int32_t* __restrict__ gmax,
    const uint32_t* __restrict__ page_w, uint32_t n_paths, uint2* __restrict__ group_idx, uint32_t* __restrict__ cells,
    uint32_t cell_cap, uint2* __restrict__ ovf, uint32_t ovf_cap, BatchCounters* __restrict__ ctr,
    const uint32_t* __restrict__ chunk_path, const int4* __restrict__ path_clip) {
    extern __shared__ __align__(16) int32_t rows_smem[];
    constexpr int LIST = WARPS * KCAP * 32;
    auto sx0 = reinterpret_cast<int32_t (*)[KCAP * 32]>(rows_smem);
    auto sx1 = reinterpret_cast<int32_t (*)[KCAP * 32]>(rows_smem + LIST);
    auto scn = reinterpret_cast<int32_t (*)[KCAP * 32]>(rows_smem + 2 * LIST);
    auto sedge = reinterpret_cast<Edge (*)[32 * GS]>(rows_smem + 3 * LIST);  // 16-byte aligned: LIST is a multiple of 4
    auto sns = reinterpret_cast<int32_t (*)[32]>(rows_smem + 3 * LIST + WARPS * 8 * 32 * GS);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t total_chunks = chunk_off[n_paths];
    uint32_t nonterm = 0;
    for (uint32_t c = blockIdx.x * WARPS + w; c < total_chunks; c += gridDim.x * WARPS) {
        const uint32_t p = chunk_path[c];  // path owning chunk c
        const PathInfo P = info[p];
        const int32_t chunk_lo = (P.y0 & ~3) + static_cast<int32_t>(c - chunk_off[p]) * 32;
        const int32_t chunk_hi = min(chunk_lo + 31, P.y1);
        const int32_t r = chunk_lo + lane;
        const bool valid = r >= P.y0 && r <= chunk_hi;
        const int32_t mask = (P.paint >> 16) & 1 ? 1 : ~0;
        const int32_t aa_width = 4 * static_cast<int32_t>(page_w[P.page]);
        const int n = gather_row<KCAP, 32, GS>(P, chunk_lo, chunk_hi, r, valid, edges, gmin, gmax, sedge[w], sx0[w],
                                              sx1[w], scn[w], lane);
        const bool overflow = valid && n > KCAP;
        int ns = 0;
        const int2 cx = path_clip ? make_int2(path_clip[p].x, path_clip[p].y) : make_int2(0, aa_width);
        if (valid && !overflow)
            ns = sort_and_walk<32>(n, mask, aa_width, cx.x, cx.y, sx0[w], sx1[w], scn[w], lane, nonterm);
        // ---- one pixel row per 4 lanes: merge the sub-rows' spans into cells
        sns[w][lane] = (valid && !overflow) ? ns : 0;
        const uint32_t ovf_lanes = __ballot_sync(0xffffffffu, overflow);
        __syncwarp();
        const bool leader = (lane & 3) == 0 && r <= P.y1;  // this pixel row has an AA row in [y0, y1]
        const bool g_ovf = ((ovf_lanes >> (lane & ~3)) & 0xFu) != 0;
        int n4[4] = {0, 0, 0, 0};
        uint32_t need = 0;
        if (leader && !g_ovf) {
#pragma unroll
            for (int k = 0; k < 4; ++k) n4[k] = sns[w][lane + k];
            need = 4u * static_cast<uint32_t>(n4[0] + n4[1] + n4[2] + n4[3]);  // 2 cells per span boundary
        }
        uint32_t incl = need;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        uint32_t base = 0;
        if (lane == 31 && total) base = atomicAdd(&ctr->cell_cursor, total);
        base = __shfl_sync(0xffffffffu, base, 31);
        const bool fits = static_cast<uint64_t>(base) + total <= cell_cap;
        if (lane == 0 && total && !fits) atomicOr(&ctr->err, ERR_SPAN_CAP);
        if (leader) {
            const int32_t g = r >> 2;
            const uint32_t gi = group_off[p] + static_cast<uint32_t>(g - (P.y0 >> 2));
            if (g_ovf) {
                const uint32_t k = atomicAdd(&ctr->ovf_count, 1u);
                if (k < ovf_cap) ovf[k] = make_uint2(p, static_cast<uint32_t>(g));
                else atomicOr(&ctr->err, ERR_OVF_CAP);
                group_idx[gi] = make_uint2(0u, 0u);
            } else if (fits) {
                const uint32_t o0 = base + incl - need;
                const int nc = sweep_cells(
                    n4,
                    [&](int k, int i, bool end) {
                        return end ? sx1[w][i * 32 + lane + k] : sx0[w][i * 32 + lane + k];
                    },
                    [&](int q, uint32_t cell) { cells[o0 + q] = cell; });
                group_idx[gi] = make_uint2(o0, static_cast<uint32_t>(nc));
            } else {
                group_idx[gi] = make_uint2(0u, 0u);
            }
        }
        __syncwarp();
    }
    if (nonterm) atomicAdd(&ctr->nonterminating, nonterm);
}

// ---------------------------------------------------------------------------
// Rectilinear paths (every edge horizontal or vertical, at most 32 edges: all
// rectangles). Between "event rows" — a vertical edge's first row, the row
// after it (the first row's count is 0 when it is not below seg_y_min) and
// the row after its last; a horizontal edge's row and the row after — every
// AA row has the same merged entries, so one row per band is computed and
// pixel rows whose four sub-rows lie in one band share one cell list. The
// path gets a list of runs (group range, cells) instead of a per-row index,
// and a solid box (pixels of coverage 16) for the composite's full-tile path.
// ---------------------------------------------------------------------------
constexpr int RECTI_MAX_EVENTS = 4 * RECTI_MAX_EDGES + 2;
constexpr int RECTI_MAX_SPANS = RECTI_MAX_EDGES / 2 + 1;

// Spans of AA row r of a rectilinear path (fold, sort, walk over <= 32 edges).
__host__ __device__ __forceinline__ int recti_row_spans(const PathInfo& P, const Edge* __restrict__ edges,
                                                        int32_t r, int32_t aa_width, int32_t lo, int32_t hi,
                                                        int32_t* sx0, int32_t* sx1, uint32_t& nonterm) {
    int32_t x0s[RECTI_MAX_EDGES], x1s[RECTI_MAX_EDGES], cs[RECTI_MAX_EDGES];
    int n = 0;
    for (uint32_t j = P.e_begin; j < P.e_end; ++j) {
        const Edge E = edges[j];
        if ((E.flags & EF_EMPTY) || r < E.row0 || r > E.row1) continue;
        int32_t elo, ehi, ec;
        edge_entry(E, r, elo, ehi, ec);
        if (n > 0 && sat_inc(x1s[n - 1]) >= elo && x0s[n - 1] <= sat_inc(ehi)) {
            cs[n - 1] = static_cast<int32_t>(static_cast<uint32_t>(cs[n - 1]) + static_cast<uint32_t>(ec));
            x0s[n - 1] = min(x0s[n - 1], elo);
            x1s[n - 1] = max(x1s[n - 1], ehi);
        } else {
            x0s[n] = elo;
            x1s[n] = ehi;
            cs[n] = ec;
            ++n;
        }
    }
    for (int a = 1; a < n; ++a) {
        const int32_t t0 = x0s[a], t1 = x1s[a], tc = cs[a];
        int b = a;
        while (b > 0 && t0 < x0s[b - 1]) {
            x0s[b] = x0s[b - 1];
            x1s[b] = x1s[b - 1];
            cs[b] = cs[b - 1];
            --b;
        }
        x0s[b] = t0;
        x1s[b] = t1;
        cs[b] = tc;
    }
    const int32_t mask = (P.paint >> 16) & 1 ? 1 : ~0;
    return walk_row(
        n, mask, aa_width, lo, hi,
        [&](int i, int32_t& a, int32_t& b, int32_t& c) {
            a = x0s[i];
            b = x1s[i];
            c = cs[i];
        },
        [&](int k, int32_t s0, int32_t e0) {
            sx0[k] = s0;
            sx1[k] = e0;
        },
        nonterm);
}

// Event rows of a rectilinear path, sorted and unique, within [y0, y1 + 1]:
// its first row, the row after its last; a horizontal edge's row and the row
// after; a vertical edge's first row, the row after it and the row after its
// last. All AA rows of one band [ev[b], ev[b+1]) have the same merged entries.
__host__ __device__ __forceinline__ int recti_events(const PathInfo& P, const Edge* __restrict__ edges, int32_t* ev) {
    int nev = 0;
    auto push = [&](int32_t v) {
        if (v >= P.y0 && v <= P.y1 + 1) ev[nev++] = v;
    };
    push(P.y0);
    push(P.y1 + 1);
    for (uint32_t j = P.e_begin; j < P.e_end; ++j) {
        const Edge E = edges[j];
        if (E.flags & EF_EMPTY) continue;
        push(E.row0);
        push(E.row0 + 1);
        if ((E.flags & EF_KIND_MASK) == EK_VERT) push(E.row1 + 1);
    }
    for (int a = 1; a < nev; ++a) {
        const int32_t t = ev[a];
        int b = a;
        while (b > 0 && t < ev[b - 1]) {
            ev[b] = ev[b - 1];
            --b;
        }
        ev[b] = t;
    }
    int m = 0;
    for (int a = 0; a < nev; ++a)
        if (m == 0 || ev[a] != ev[m - 1]) ev[m++] = ev[a];
    return m;
}

// Whether a rectilinear path is a box (PI_BOX): the bands of identical AA
// rows [ev[b], ev[b+1]) that paint anything are consecutive, each has exactly
// one span, the same in all of them, and every row's winding closes. Returns
// the span [s0, s1) and the painted AA rows [r0, r1]. (A rectangle's first
// and last AA rows paint nothing: their merged entry has a zero count.)
__host__ __device__ __forceinline__ bool recti_box(const PathInfo& P, const Edge* __restrict__ edges,
                                                   const int32_t* ev, int nev, int32_t aa_width, int32_t lo,
                                                   int32_t hi, int32_t& s0, int32_t& s1, int32_t& r0, int32_t& r1) {
    bool seen = false, ended = false;
    for (int b = 0; b + 1 < nev; ++b) {
        int32_t a0[RECTI_MAX_SPANS], a1[RECTI_MAX_SPANS];
        uint32_t open_rows = 0;
        const int n = recti_row_spans(P, edges, ev[b], aa_width, lo, hi, a0, a1, open_rows);
        if (open_rows || n > 1) return false;
        if (n == 0) {
            ended = seen;
            continue;
        }
        if (ended) return false;  // painted bands with a gap between them
        if (!seen) {
            s0 = a0[0];
            s1 = a1[0];
            r0 = ev[b];
            seen = true;
        } else if (a0[0] != s0 || a1[0] != s1) {
            return false;
        }
        r1 = ev[b + 1] - 1;
    }
    return seen && s0 < s1;
}

template <bool WRITE>
__global__ void k_recti(PathInfo* __restrict__ info, uint32_t n_paths, const Edge* __restrict__ edges,
                        const uint32_t* __restrict__ page_w, int rowmap, uint32_t* __restrict__ run_count,
                        const uint32_t* __restrict__ run_off, int4* __restrict__ runs, uint32_t* __restrict__ cells,
                        uint32_t cell_cap, BatchCounters* __restrict__ ctr, const int4* __restrict__ path_clip) {
    uint32_t nonterm = 0;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n_paths; p += gridDim.x * blockDim.x) {
        PathInfo P = info[p];
        if (P.paint & PI_SOLID) continue;  // hairline layers: runs from k_hl_count / k_hl_write
        if (!(P.paint & PI_RECTI)) {
            if (!WRITE) run_count[p] = 0;
            continue;
        }
        if (WRITE && (P.paint & PI_BOX)) continue;  // boxes have no runs or cells
        int32_t ev[RECTI_MAX_EVENTS];
        const int nev = recti_events(P, edges, ev);  // ev[0] = y0, ev[nev-1] = y1 + 1
        auto band_of = [&](int32_t r) {  // last k with ev[k] <= r
            int lo = 0, hi = nev - 1;
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (ev[mid] <= r) lo = mid;
                else hi = mid;
            }
            return lo;
        };
        const int32_t g0 = P.y0 >> 2, g1 = P.y1 >> 2;
        const int32_t aa_width = 4 * static_cast<int32_t>(page_w[P.page]);
        const int2 cx = path_clip ? make_int2(path_clip[p].x, path_clip[p].y) : make_int2(0, aa_width);
        if (!WRITE) {
            int32_t s0 = 0, s1 = 0, r0 = 0, r1 = -1;
            if (recti_box(P, edges, ev, nev, aa_width, cx.x, cx.y, s0, s1, r0, r1)) {
                // Solid box: pixels whose four AA columns and whose AA rows under
                // the row map all lie inside the box.
                int32_t by0, by1;
                if (rowmap == 0) {
                    by0 = floor_div(r0 + 3, 4);
                    by1 = floor_div(r1 + 1, 4) - 1;
                } else {  // pixel row y shows AA rows 16y+12 .. 16y+15
                    by0 = floor_div(r0 - 12 + 15, 16);
                    by1 = floor_div(r1 - 15, 16);
                }
                by0 = max(by0, P.py0);
                by1 = min(by1, P.py1);
                const int32_t bx0 = floor_div(s0 + 3, 4), bx1 = floor_div(s1, 4) - 1;
                // From here on a box's y0, y1 are the AA rows it paints.
                info[p].y0 = r0;
                info[p].y1 = r1;
                info[p].paint = P.paint | PI_BOX;
                info[p].run_off = static_cast<uint32_t>(s0);
                info[p].run_cnt = static_cast<uint32_t>(s1);
                if (bx0 <= bx1 && by0 <= by1) {
                    info[p].bx0 = bx0;
                    info[p].bx1 = bx1;
                    info[p].by0 = by0;
                    info[p].by1 = by1;
                }
                run_count[p] = 0;
                continue;
            }
        }
        uint32_t nrun = 0;
        uint32_t ro = WRITE ? run_off[p] : 0u;
        int32_t best_rows = 0, bx0 = 1, bx1 = 0, bg0 = 1, bg1 = 0;
        for (int32_t g = g0; g <= g1;) {
            const int32_t r_lo = 4 * g, r_hi = 4 * g + 3;
            const bool inside = r_lo >= P.y0 && r_hi <= P.y1;
            int32_t g_end = g;
            bool uniform = false;
            int b = 0;
            if (inside) {
                b = band_of(r_lo);
                if (band_of(r_hi) == b) {
                    uniform = true;
                    g_end = min((ev[b + 1] - 4) >> 2, (P.y1 - 3) >> 2);
                }
            }
            if (WRITE) {
                int32_t s0[4][RECTI_MAX_SPANS], s1[4][RECTI_MAX_SPANS];
                int n4[4] = {0, 0, 0, 0};
                if (uniform) {
                    n4[0] = recti_row_spans(P, edges, r_lo, aa_width, cx.x, cx.y, s0[0], s1[0], nonterm);
                    n4[1] = n4[2] = n4[3] = n4[0];
                } else {
                    for (int k = 0; k < 4; ++k) {
                        const int32_t r = r_lo + k;
                        if (r >= P.y0 && r <= P.y1) n4[k] = recti_row_spans(P, edges, r, aa_width, cx.x, cx.y, s0[k], s1[k], nonterm);
                    }
                }
                const uint32_t need = 4u * static_cast<uint32_t>(n4[0] + n4[1] + n4[2] + n4[3]);
                const uint32_t o0 = need ? atomicAdd(&ctr->cell_cursor, need) : 0u;
                int nc = 0;
                if (static_cast<uint64_t>(o0) + need > cell_cap) {
                    atomicOr(&ctr->err, ERR_SPAN_CAP);
                } else {
                    int32_t f0 = 1, f1 = 0;  // widest coverage-16 cell of a uniform run
                    nc = sweep_cells(
                        n4,
                        [&](int k, int i, bool end) {
                            const int kk = uniform ? 0 : k;
                            return end ? s1[kk][i] : s0[kk][i];
                        },
                        [&](int q, uint32_t cell) {
                            cells[o0 + q] = cell;
                            const int32_t len = static_cast<int32_t>((cell >> 14) & 0x3fffu) + 1;
                            if ((cell >> 28) == 15u && len > f1 - f0 + 1) {
                                f0 = static_cast<int32_t>(cell & 0x3fffu);
                                f1 = f0 + len - 1;
                            }
                        });
                    if (uniform && f0 <= f1) {
                        const int32_t rows = g_end - g + 1;
                        if (static_cast<int64_t>(rows) * (f1 - f0 + 1) > static_cast<int64_t>(best_rows) * (bx1 - bx0 + 1)) {
                            best_rows = rows;
                            bx0 = f0;
                            bx1 = f1;
                            bg0 = g;
                            bg1 = g_end;
                        }
                    }
                }
                runs[ro + nrun] = make_int4(g, g_end, static_cast<int32_t>(o0), nc);
            }
            ++nrun;
            g = g_end + 1;
        }
        if (!WRITE) {
            run_count[p] = nrun;
        } else {
            P.run_off = ro;
            P.run_cnt = nrun;
            // Solid box in pixel rows of the row map, inside the rows the path draws.
            int32_t by0, by1;
            if (rowmap == 0) {
                by0 = bg0;
                by1 = bg1;
            } else {  // pixel row y shows group 4y + 3
                by0 = (bg0 - 3 + 3) >> 2;
                by0 = (4 * by0 + 3 < bg0) ? by0 + 1 : by0;
                by1 = bg1 >= 3 ? (bg1 - 3) >> 2 : -1;
            }
            by0 = max(by0, P.py0);
            by1 = min(by1, P.py1);
            if (bx0 <= bx1 && by0 <= by1) {
                info[p].bx0 = bx0;
                info[p].bx1 = bx1;
                info[p].by0 = by0;
                info[p].by1 = by1;
            }
            info[p].run_off = ro;
            info[p].run_cnt = nrun;
        }
    }
    if (WRITE && nonterm) atomicAdd(&ctr->nonterminating, nonterm);
}

// Pixel rows whose sub-row lists overflowed KCAP: one warp per pixel row
// (lanes 0-3 = its AA rows) with MID_K entries per row in shared memory.
// Rows longer than that go to k_groups_slow through ovf2.
constexpr int MID_K = 128;
constexpr int MID_WARPS = 4;

__global__ void __launch_bounds__(MID_WARPS * 32) k_groups_mid(
    const PathInfo* __restrict__ info, const uint32_t* __restrict__ group_off, const Edge* __restrict__ edges,
    const int32_t* __restrict__ gmin, const int32_t* __restrict__ gmax, const uint32_t* __restrict__ page_w,
    const uint2* __restrict__ ovf, uint32_t ovf_cap, uint2* __restrict__ group_idx, uint32_t* __restrict__ cells,
    uint32_t cell_cap, uint2* __restrict__ ovf2, BatchCounters* __restrict__ ctr, const int4* __restrict__ path_clip) {
    __shared__ int32_t sx0[MID_WARPS][MID_K * 4];
    __shared__ int32_t sx1[MID_WARPS][MID_K * 4];
    __shared__ int32_t scn[MID_WARPS][MID_K * 4];
    __shared__ Edge sedge[MID_WARPS][32];
    __shared__ int32_t sns[MID_WARPS][4];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t n_ovf = min(ctr->ovf_count, ovf_cap);
    uint32_t nonterm = 0;
    for (uint32_t k = blockIdx.x * MID_WARPS + w; k < n_ovf; k += gridDim.x * MID_WARPS) {
        const uint32_t p = ovf[k].x;
        const int32_t g = static_cast<int32_t>(ovf[k].y);
        const PathInfo P = info[p];
        const int32_t lo = 4 * g, hi = min(4 * g + 3, P.y1);
        const int32_t r = lo + lane;
        const bool valid = lane < 4 && r >= P.y0 && r <= hi;
        const int32_t mask = (P.paint >> 16) & 1 ? 1 : ~0;
        const int32_t aa_width = 4 * static_cast<int32_t>(page_w[P.page]);
        const int n = gather_row<MID_K, 4>(P, lo, hi, r, valid, edges, gmin, gmax, sedge[w], sx0[w], sx1[w], scn[w],
                                           lane);
        const bool overflow = valid && n > MID_K;
        int ns = 0;
        const int2 cx = path_clip ? make_int2(path_clip[p].x, path_clip[p].y) : make_int2(0, aa_width);
        if (valid && !overflow)
            ns = sort_and_walk<4>(n, mask, aa_width, cx.x, cx.y, sx0[w], sx1[w], scn[w], lane, nonterm);
        if (lane < 4) sns[w][lane] = (valid && !overflow) ? ns : 0;
        const bool any_ovf = __any_sync(0xffffffffu, overflow);
        __syncwarp();
        if (lane == 0) {
            const uint32_t gi = group_off[p] + static_cast<uint32_t>(g - (P.y0 >> 2));
            if (any_ovf) {
                const uint32_t k2 = atomicAdd(&ctr->ovf2_count, 1u);
                if (k2 < ovf_cap) ovf2[k2] = make_uint2(p, static_cast<uint32_t>(g));
                else atomicOr(&ctr->err, ERR_OVF_CAP);
                group_idx[gi] = make_uint2(0u, 0u);
            } else {
                int n4[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) n4[q] = sns[w][q];
                const uint32_t need = 4u * static_cast<uint32_t>(n4[0] + n4[1] + n4[2] + n4[3]);
                const uint32_t o0 = need ? atomicAdd(&ctr->cell_cursor, need) : 0u;
                if (static_cast<uint64_t>(o0) + need > cell_cap) {
                    atomicOr(&ctr->err, ERR_SPAN_CAP);
                    group_idx[gi] = make_uint2(0u, 0u);
                } else {
                    const int nc = sweep_cells(
                        n4, [&](int q, int i, bool end) { return end ? sx1[w][i * 4 + q] : sx0[w][i * 4 + q]; },
                        [&](int q, uint32_t cell) { cells[o0 + q] = cell; });
                    group_idx[gi] = make_uint2(o0, static_cast<uint32_t>(nc));
                }
            }
        }
        __syncwarp();
    }
    if (nonterm) atomicAdd(&ctr->nonterminating, nonterm);
}

// Pixel rows with a sub-row whose merged list exceeded MID_K: one thread per
// pixel row, the four sub-row lists in a global scratch slice of 4 x the
// path's edge count.
constexpr int SLOW_WARPS = 4;  // warps per block of k_groups_slow

__global__ void k_groups_slow(const PathInfo* __restrict__ info, const uint32_t* __restrict__ group_off,
                              const Edge* __restrict__ edges, const int32_t* __restrict__ gmin,
                              const int32_t* __restrict__ gmax, const uint32_t* __restrict__ page_w,
                              const uint2* __restrict__ ovf, uint32_t ovf_cap, int3* __restrict__ scratch,
                              uint32_t scratch_cap, uint2* __restrict__ group_idx, uint32_t* __restrict__ cells,
                              uint32_t cell_cap, BatchCounters* __restrict__ ctr, const int4* __restrict__ path_clip) {
    // One warp per overflowing pixel row. The warp loads the path's edges 32
    // at a time (aligned groups whose row bounds miss the row are skipped) and
    // stages each lane's entries for the four AA sub-rows in shared memory;
    // lanes 0-3 then fold them, in edge order, into their sub-row's list
    // (merging into the list's last entry as fill_intersections does). Lane 0
    // sorts, walks and writes the cells.
    __shared__ int3 stage[SLOW_WARPS][4][32];
    const uint32_t lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const uint32_t n_ovf = min(ctr->ovf2_count, ovf_cap);
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    uint32_t nonterm = 0;
    for (uint32_t k = blockIdx.x * (blockDim.x >> 5) + wib; k < n_ovf; k += warps) {
        const uint32_t p = ovf[k].x;
        const int32_t g = static_cast<int32_t>(ovf[k].y);
        const PathInfo P = info[p];
        const uint32_t ne = P.e_end - P.e_begin;
        // Four sub-row lists of up to ne entries, and one list of merge-sort temporary.
        uint32_t sb = 0;
        if (lane == 0) sb = atomicAdd(&ctr->scratch_cursor, 5u * ne);
        sb = __shfl_sync(0xffffffffu, sb, 0);
        if (static_cast<uint64_t>(sb) + 5ull * ne > scratch_cap) {
            if (lane == 0) atomicOr(&ctr->err, ERR_SCRATCH_CAP);
            continue;
        }
        const int32_t mask = (P.paint >> 16) & 1 ? 1 : ~0;
        const int32_t aa_width = 4 * static_cast<int32_t>(page_w[P.page]);
        const int2 cx = path_clip ? make_int2(path_clip[p].x, path_clip[p].y) : make_int2(0, aa_width);
        const int32_t rlo = max(4 * g, P.y0), rhi = min(4 * g + 3, P.y1);
        // Lane s < 4: sub-row s's list length and its last entry (not yet stored).
        int n_s = 0;
        int3 last = make_int3(0, 0, 0);
        bool has_last = false;
        int3* const Ls = scratch + sb + min(lane, 3u) * ne;
        // 32 groups' bounds at a time, one per lane; only groups meeting the
        // pixel row's AA rows are visited, in ascending order.
        for (uint32_t gb = P.e_begin >> 5; 32ull * gb < P.e_end; gb += 32) {
          const uint32_t gl = gb + lane;
          const bool g_hit = 32ull * gl < P.e_end && !(gmax[gl] < rlo || gmin[gl] > rhi);
          uint32_t gm = __ballot_sync(0xffffffffu, g_hit);
          while (gm) {
            const uint32_t base = (gb + static_cast<uint32_t>(__ffs(gm) - 1)) << 5;
            gm &= gm - 1;
            const uint32_t j = base + lane;
            uint32_t bits = 0;  // sub-rows this lane's edge has an entry in
            if (j >= P.e_begin && j < P.e_end) {
                const Edge E = edges[j];
                if (!(E.flags & EF_EMPTY) && E.row1 >= rlo && E.row0 <= rhi) {
                    const int32_t r0 = max(rlo, E.row0), r1 = min(rhi, E.row1);
                    for (int32_t r = r0; r <= r1; ++r) {
                        int32_t elo, ehi, ec;
                        edge_entry(E, r, elo, ehi, ec);
                        stage[wib][r - 4 * g][lane] = make_int3(elo, ehi, ec);
                        bits |= 1u << (r - 4 * g);
                    }
                }
            }
            const uint32_t m0 = __ballot_sync(0xffffffffu, bits & 1), m1 = __ballot_sync(0xffffffffu, bits & 2);
            const uint32_t m2 = __ballot_sync(0xffffffffu, bits & 4), m3 = __ballot_sync(0xffffffffu, bits & 8);
            __syncwarp();
            if (lane < 4) {
                uint32_t m = lane == 0 ? m0 : lane == 1 ? m1 : lane == 2 ? m2 : m3;
                while (m) {
                    const int q = __ffs(m) - 1;
                    m &= m - 1;
                    const int3 e = stage[wib][lane][q];
                    if (has_last && sat_inc(last.y) >= e.x && last.x <= sat_inc(e.y)) {
                        last.z = static_cast<int32_t>(static_cast<uint32_t>(last.z) + static_cast<uint32_t>(e.z));
                        last.x = min(last.x, e.x);
                        last.y = max(last.y, e.y);
                    } else {
                        if (has_last) Ls[n_s++] = last;
                        last = e;
                        has_last = true;
                    }
                }
            }
            __syncwarp();
          }
        }
        if (lane < 4 && has_last) Ls[n_s++] = last;
        int n4[4];
#pragma unroll
        for (int sub = 0; sub < 4; ++sub) n4[sub] = __shfl_sync(0xffffffffu, n_s, sub);
        __syncwarp();
        if (lane != 0) continue;
        for (int sub = 0; sub < 4; ++sub) {
            const int32_t r = 4 * g + sub;
            if (r < P.y0 || r > P.y1) continue;
            int3* L = scratch + sb + static_cast<uint32_t>(sub) * ne;
            int n = n4[sub];
            // Stable sort by x0 (a row of more than 20 entries: see the tie
            // note in the oracle): bottom-up merge sort through the temporary
            // list, skipped when the entries already come in order.
            bool sorted = true;
            for (int a = 1; a < n && sorted; ++a) sorted = L[a - 1].x <= L[a].x;
            if (!sorted) {
                int3* A = L;
                int3* T = scratch + sb + 4u * ne;
                for (int w = 1; w < n; w *= 2) {
                    for (int lo = 0; lo < n; lo += 2 * w) {
                        const int mid = min(lo + w, n), hi = min(lo + 2 * w, n);
                        int i = lo, j = mid, k = lo;
                        while (i < mid && j < hi) T[k++] = A[j].x < A[i].x ? A[j++] : A[i++];
                        while (i < mid) T[k++] = A[i++];
                        while (j < hi) T[k++] = A[j++];
                    }
                    int3* t = A;
                    A = T;
                    T = t;
                }
                if (A != L)
                    for (int a = 0; a < n; ++a) L[a] = A[a];
            }
            n4[sub] = walk_row(
                n, mask, aa_width, cx.x, cx.y,
                [&](int i, int32_t& x0, int32_t& x1, int32_t& cc) {
                    x0 = L[i].x;
                    x1 = L[i].y;
                    cc = L[i].z;
                },
                [&](int q, int32_t s0, int32_t e0) {
                    L[q].x = s0;
                    L[q].y = e0;
                },
                nonterm);
        }
        const uint32_t need = 4u * static_cast<uint32_t>(n4[0] + n4[1] + n4[2] + n4[3]);
        const uint32_t gi = group_off[p] + static_cast<uint32_t>(g - (P.y0 >> 2));
        const uint32_t o0 = need ? atomicAdd(&ctr->cell_cursor, need) : 0u;
        if (static_cast<uint64_t>(o0) + need > cell_cap) {
            atomicOr(&ctr->err, ERR_SPAN_CAP);
            group_idx[gi] = make_uint2(0u, 0u);
            continue;
        }
        const int3* base = scratch + sb;
        const int nc = sweep_cells(
            n4,
            [&](int sub, int i, bool end) {
                const int3 v = base[static_cast<uint32_t>(sub) * ne + i];
                return end ? v.y : v.x;
            },
            [&](int q, uint32_t cell) { cells[o0 + q] = cell; });
        group_idx[gi] = make_uint2(o0, static_cast<uint32_t>(nc));
    }
    if (nonterm) atomicAdd(&ctr->nonterminating, nonterm);
}

// ---------------------------------------------------------------------------
// Composite: one CTA per TW x TH page tile. The tile's bytes are loaded once
// into registers, every path of the tile's supertile list whose rectangle
// overlaps the tile is applied in path order (coverage from its four AA
// sub-row span lists -> AA_GAMMA -> div255 source-over), and the tile is
// stored once.
// ---------------------------------------------------------------------------
// Tiles of 4,096 pixels or more run RRB_COMP_BIG_THREADS threads per CTA
// (512: a thread holds 8 pixels, as in the smaller tiles' 256-thread CTAs).
// The composite is compiled for RRB_COMP_SM_THREADS resident threads per SM,
// which sets its register budget. With two path hits' loads in flight, 1280
// threads (five 256-thread CTAs, 48 registers) ran the 64-page mixed batch's
// composite 5% faster than 1024 (64 registers) and 4% faster than 1536 (40);
// with one (a buffer of registers fewer), 1536 threads (six CTAs, 40
// registers) ran it 3% faster again (53.97 against 55.78 ms).
#ifndef RRB_COMP_BIG_THREADS
#define RRB_COMP_BIG_THREADS 512
#endif
#ifndef RRB_COMP_SM_THREADS
#define RRB_COMP_SM_THREADS 1536
#endif
// Path hits whose loads are in flight ahead of the one being blended (1, or
// 2 with a buffer of registers more).
#ifndef RRB_COMP_PIPE_DEPTH
#define RRB_COMP_PIPE_DEPTH 1
#endif
__host__ __device__ constexpr int comp_threads(int tw, int th) {
    return tw * th >= 4096 ? RRB_COMP_BIG_THREADS : 256;
}
__host__ __device__ constexpr int comp_ctas_per_sm(int tw, int th) {
    return RRB_COMP_SM_THREADS / comp_threads(tw, th) > 0 ? RRB_COMP_SM_THREADS / comp_threads(tw, th) : 1;
}

__constant__ uint8_t c_gamma[17] = {0, 4, 11, 21, 32, 45, 59, 74, 90, 108, 126, 145, 166, 187, 209, 231, 255};

struct HitInfo {
    int32_t g0, g1, py0, py1;  // pixel-row groups [g0, g1] (AA rows >> 2), pixel rows touched
    uint32_t goff, paint;      // first group index entry (or first run), paint word (| HIT_FULL)
    uint32_t run_cnt, rgb;     // rectilinear paths: number of runs; Rgb8 pages: the path's colour
};

constexpr uint32_t HIT_FULL = 1u << 18;  // every pixel of this tile has coverage 16 for this path

template <int TW, int TH>
struct CompLayout {
    static constexpr int NT = comp_threads(TW, TH);  // threads per CTA = candidates per chunk
    static constexpr int LPR = TW < 32 ? TW : 32;      // lanes per pixel row
    static constexpr int PX = TW / LPR;                // pixels per lane
    static constexpr int RPW = 32 / LPR;               // rows per warp step
    static constexpr int NW = NT / 32;
    static constexpr int NPIX = TW * TH / NT;          // pixels per thread
};

// Loads of one hit for this thread's tile rows: the pixel row's entry in the
// group index (g = y, or 4y+3 under the as-shipped row map) and this lane's
// first cell. k_composite issues them two and one hits ahead of use.
template <int TW, int TH>
struct HitRows {
    static constexpr int ITERS = TH / (CompLayout<TW, TH>::NW * CompLayout<TW, TH>::RPW);
    uint2 ix[ITERS];
    uint32_t cell0[ITERS];
};

// A box hit (PI_BOX): its coverage over this thread's pixels is cx * cy,
// from the box's AA columns [S0, S1) (h.goff, h.run_cnt) and AA rows
// [h.g0, h.g1]; the pixel row y shows AA rows 4y..4y+3 (documented row map)
// or 16y+12..16y+15 (as-shipped). No loads: every operand is in the hit.
// Then AA_GAMMA and the blend of composite_path_rows.
template <int TW, int TH, bool RGB>
__device__ __forceinline__ void composite_box(const HitInfo& h, int rowmap, int X0, int Y0, const uint8_t* gamma,
                                              uint32_t (&pix)[CompLayout<TW, TH>::NPIX]);

constexpr uint32_t kFewRuns = 4;   // rectilinear paths with at most this many runs: no search
constexpr uint32_t kFewCells = 4;  // rectilinear rows with at most this many cells: direct lookup
constexpr int kLoopCells = 6;      // rows with at most this many cells in the tile: tested one by one
constexpr uint32_t kDirectRun = 4; // runs of at most this many full-tile layers: blended per pixel

template <int TW, int TH>
__device__ __forceinline__ void load_hit_index(const HitInfo& h, int rowmap, int Y0, int H,
                                               const uint2* __restrict__ gidx, const int4* __restrict__ runs,
                                               HitRows<TW, TH>& hr) {
    using L = CompLayout<TW, TH>;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int slot = lane / L::LPR;
#pragma unroll
    for (int it = 0; it < HitRows<TW, TH>::ITERS; ++it) {
        const int y = Y0 + (w * L::RPW + slot) + it * L::NW * L::RPW;
        const int32_t grp = rowmap ? 4 * y + 3 : y;
        const bool rowok = !(h.paint & (PI_BOX | HIT_FULL)) && y >= h.py0 && y <= h.py1 && y < H && grp >= h.g0 &&
                           grp <= h.g1;
        uint2 ix = make_uint2(0u, 0u);
        if (rowok) {
            if (h.paint & PI_RECTI) {
                // Runs cover [g0, g1] in order: the last run starting at or before grp.
                uint32_t lo = 0;
                if (h.run_cnt <= kFewRuns) {
                    // A rectangle has a handful of runs: their starts are loaded
                    // at once instead of by a chain of dependent search steps.
                    int32_t s[kFewRuns - 1];
#pragma unroll
                    for (uint32_t q = 1; q < kFewRuns; ++q) s[q - 1] = q < h.run_cnt ? runs[h.goff + q].x : INT32_MAX;
#pragma unroll
                    for (uint32_t q = 1; q < kFewRuns; ++q)
                        if (s[q - 1] <= grp) lo = q;
                } else {
                    uint32_t hi = h.run_cnt;
                    while (hi - lo > 1) {
                        const uint32_t mid = (lo + hi) >> 1;
                        if (runs[h.goff + mid].x <= grp) lo = mid;
                        else hi = mid;
                    }
                }
                const int4 rn = runs[h.goff + lo];
                if (rn.x <= grp && grp <= rn.y) ix = make_uint2(static_cast<uint32_t>(rn.z), static_cast<uint32_t>(rn.w));
            } else {
                ix = gidx[h.goff + static_cast<uint32_t>(grp - h.g0)];
            }
        }
        hr.ix[it] = ix;
    }
}

template <int TW, int TH>
__device__ __forceinline__ void load_hit_cells(const uint32_t* __restrict__ cells, HitRows<TW, TH>& hr) {
    using L = CompLayout<TW, TH>;
    const int sub = (threadIdx.x & 31) % L::LPR;
#pragma unroll
    for (int it = 0; it < HitRows<TW, TH>::ITERS; ++it)
        hr.cell0[it] = static_cast<uint32_t>(sub) < hr.ix[it].y ? cells[hr.ix[it].x + sub] : 0u;
}

// One path over the rows of this thread's tile slots: find each pixel's
// coverage cell (start marks in shared memory + a prefix max across the row's
// lanes), then AA_GAMMA and the div255 source-over of render_span_aa_inner's
// no-alpha arm (pipe/aa.rs:192-208).
// Rgb8 pages (A12, composite_aa_rgb8_opaque, simd/composite.rs:56+): pixels
// and colours packed r | g << 8 | b << 16; per channel
// c = ((255 - a) * dst + a * src + 255) >> 8.
__device__ __forceinline__ uint32_t rgb_over(uint32_t d, uint32_t a, uint32_t s) {
    const uint32_t inv = 255u - a;
    uint32_t out = 0;
#pragma unroll
    for (int c = 0; c < 24; c += 8)
        out |= (((inv * ((d >> c) & 0xffu) + a * ((s >> c) & 0xffu) + 255u) >> 8) & 0xffu) << c;
    return out;
}

// render_span's general arm on an Rgb8 page without alpha plane, per channel
// div255((255 - a) * dst + a * src) (pipe/general.rs:261-312).
__device__ __forceinline__ uint32_t rgb_over_div255(uint32_t d, uint32_t a, uint32_t s) {
    uint32_t out = 0;
#pragma unroll
    for (int c = 0; c < 24; c += 8)
        out |= div255((255u - a) * ((d >> c) & 0xffu) + a * ((s >> c) & 0xffu)) << c;
    return out;
}

// a_src of the Rgb8 path: (a_input * shape + 255) >> 8.
__device__ __forceinline__ uint32_t rgb_a_src(uint32_t alpha, uint32_t shape) { return (alpha * shape + 255u) >> 8; }

// div255 for x <= 255 * 255, where its clamp never applies: every product
// of two bytes and every source-over sum (255 - a) * d + a * s.
__device__ __forceinline__ uint32_t div255_small(uint32_t x) { return (x + (x >> 8) + 0x80u) >> 8; }

// Source-over of one Gray8 pixel at AA coverage cov (1..16): a_src =
// div255(alpha * AA_GAMMA[cov]), then div255((255 - a_src) * d + a_src * g).
// Full coverage takes the hit's constants: AA_GAMMA[16] = 255 and
// div255(alpha * 255) = alpha, so a_src = alpha (inv16 = 255 - alpha,
// ag16 = alpha * g).
__device__ __forceinline__ uint32_t gray_over(uint32_t d, int32_t cov, const uint8_t* gamma, uint32_t alpha,
                                              uint32_t g, uint32_t inv16, uint32_t ag16) {
    if (cov >= 16) return div255_small(inv16 * d + ag16);
    const uint32_t a_src = div255_small(alpha * gamma[cov]);
    return div255_small((255u - a_src) * d + a_src * g);
}

// FEW: the batch has rectilinear paths, whose rows take the direct lookup.
template <int TW, int TH, bool RGB, bool FEW>
__device__ __forceinline__ void composite_path_rows(const HitInfo& h, const HitRows<TW, TH>& hr, int X0,
                                                    const uint32_t* __restrict__ cells, const uint8_t* gamma,
                                                    int32_t (*mark)[TW], uint32_t (&pix)[CompLayout<TW, TH>::NPIX]) {
    using L = CompLayout<TW, TH>;
    constexpr int ITERS = HitRows<TW, TH>::ITERS;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int sub = lane % L::LPR;
    const int slot = lane / L::LPR;
    const int col = sub * L::PX;
    const uint32_t g = h.paint & 0xff, alpha = (h.paint >> 8) & 0xff;
#pragma unroll
    for (int it = 0; it < ITERS; ++it) {
        const uint2 ix = hr.ix[it];
        // No cells in this warp's row(s) of the tile: nothing to do (a vote,
        // so the shuffles below stay warp-uniform when a warp holds 2 rows).
        if (__all_sync(0xffffffffu, ix.y == 0u)) continue;
        int32_t cov[L::PX];
#pragma unroll
        for (int q = 0; q < L::PX; ++q) cov[q] = 0;
        // Rectilinear paths (rectangle edges crossing the tile) have at most a
        // few cells per pixel row, held in the row's first lanes (cell0): each
        // pixel takes the last cell that reaches into the tile and starts
        // (clipped to the tile) at or before it, and is covered if it lies
        // before that cell's end — the rule of the marking pass below,
        // without shared memory.
        bool few = false;
        if constexpr (FEW) {
            if constexpr (L::RPW > 1) few = (h.paint & PI_RECTI) && __all_sync(0xffffffffu, ix.y <= kFewCells);
            else few = (h.paint & PI_RECTI) && ix.y <= kFewCells;
        }
        if (few) {
            uint32_t sel[L::PX];
            bool has[L::PX];
#pragma unroll
            for (int q = 0; q < L::PX; ++q) {
                sel[q] = 0;
                has[q] = false;
            }
#pragma unroll
            for (uint32_t k = 0; k < kFewCells; ++k) {
                const uint32_t c = __shfl_sync(0xffffffffu, hr.cell0[it], static_cast<int>(k), L::LPR);
                const int32_t x0 = static_cast<int32_t>(c & 0x3fffu);
                const int32_t x1 = x0 + static_cast<int32_t>((c >> 14) & 0x3fffu) + 1;
                const int32_t sx = max(x0, X0);
                const bool marks = k < ix.y && sx < min(x1, X0 + TW);
#pragma unroll
                for (int q = 0; q < L::PX; ++q) {
                    if (marks && sx <= X0 + col + q) {
                        sel[q] = c;
                        has[q] = true;
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < L::PX; ++q) {
                const int32_t x0 = static_cast<int32_t>(sel[q] & 0x3fffu);
                const int32_t x1 = x0 + static_cast<int32_t>((sel[q] >> 14) & 0x3fffu) + 1;
                if (has[q] && X0 + col + q < x1) cov[q] = static_cast<int32_t>(sel[q] >> 28) + 1;
            }
        }
        // A warp holding one pixel row whose cells all sit in its lanes
        // (cell0): when few of them reach into the tile, each pixel tests
        // those few directly (cells are sorted and disjoint, so the one that
        // contains a pixel is the last one starting at or before it).
        if constexpr (L::RPW == 1) {
            if (!few && ix.y <= static_cast<uint32_t>(L::LPR)) {
                const uint32_t c = hr.cell0[it];
                const int32_t x0 = static_cast<int32_t>(c & 0x3fffu);
                const int32_t x1 = x0 + static_cast<int32_t>((c >> 14) & 0x3fffu) + 1;
                const bool in_tile = static_cast<uint32_t>(sub) < ix.y && max(x0, X0) < min(x1, X0 + TW);
                uint32_t bm = __ballot_sync(0xffffffffu, in_tile);
                if (__popc(bm) <= kLoopCells) {
                    while (bm) {
                        const int t = __ffs(bm) - 1;
                        bm &= bm - 1;
                        const uint32_t cc = __shfl_sync(0xffffffffu, c, t);
                        const int32_t cx0 = static_cast<int32_t>(cc & 0x3fffu);
                        const int32_t cx1 = cx0 + static_cast<int32_t>((cc >> 14) & 0x3fffu) + 1;
#pragma unroll
                        for (int q = 0; q < L::PX; ++q) {
                            const int32_t x = X0 + col + q;
                            if (x >= cx0 && x < cx1) cov[q] = static_cast<int32_t>(cc >> 28) + 1;
                        }
                    }
                    few = true;  // done: skip the marking pass
                }
            }
        }
        // Otherwise the clipped cell starts are marked in shared memory, LPR
        // cells at a time, and each pixel takes a prefix max across its row.
        uint32_t nb = 0;
        if (!few) {
            nb = (ix.y + L::LPR - 1) / L::LPR;
            // With one pixel row per warp step every lane holds the same entry.
            if constexpr (L::RPW > 1)
                for (int o = 16; o; o >>= 1) nb = max(nb, __shfl_xor_sync(0xffffffffu, nb, o));
        }
        for (uint32_t bt = 0; bt < nb; ++bt) {
#pragma unroll
            for (int q = 0; q < L::PX; ++q) mark[w * L::RPW + slot][q * L::LPR + sub] = -1;
            __syncwarp();
            const uint32_t j = bt * L::LPR + sub;
            uint32_t cell = 0;
            if (j < ix.y) {
                cell = bt == 0 ? hr.cell0[it] : cells[ix.x + j];
                const int32_t x0 = static_cast<int32_t>(cell & 0x3fffu);
                const int32_t x1 = x0 + static_cast<int32_t>((cell >> 14) & 0x3fffu) + 1;
                const int32_t sx = max(x0, X0);
                if (sx < min(x1, X0 + TW)) {
                    // Pixel p = lane * PX + q of the row lives at [q * LPR + lane] (no bank conflicts).
                    const int32_t pp = sx - X0;
                    mark[w * L::RPW + slot][(pp % L::PX) * L::LPR + pp / L::PX] = sub;
                }
            }
            __syncwarp();
            int32_t v[L::PX];
            int32_t run = -1;
#pragma unroll
            for (int q = 0; q < L::PX; ++q) {
                run = max(run, mark[w * L::RPW + slot][q * L::LPR + sub]);
                v[q] = run;
            }
            // Exclusive prefix max of `run` over the lanes before this one in the row.
            int32_t incl = run;
#pragma unroll
            for (int o = 1; o < L::LPR; o <<= 1) {
                const int32_t t = __shfl_up_sync(0xffffffffu, incl, o, L::LPR);
                if (sub >= o) incl = max(incl, t);
            }
            int32_t before = __shfl_up_sync(0xffffffffu, incl, 1, L::LPR);
            if (sub == 0) before = -1;
#pragma unroll
            for (int q = 0; q < L::PX; ++q) {
                const int32_t idx = max(before, v[q]);
                const uint32_t c = __shfl_sync(0xffffffffu, cell, idx >= 0 ? idx : sub, L::LPR);
                const int32_t x0 = static_cast<int32_t>(c & 0x3fffu);
                const int32_t x1 = x0 + static_cast<int32_t>((c >> 14) & 0x3fffu) + 1;
                const int32_t x = X0 + col + q;
                if (idx >= 0 && x < x1) cov[q] = static_cast<int32_t>(c >> 28) + 1;
            }
        }
#pragma unroll
        for (int q = 0; q < L::PX; ++q) {
            if (cov[q] == 0) continue;
            const int k = it * L::PX + q;
            if (RGB) {
                const uint32_t shape = gamma[min(cov[q], 16)];
                pix[k] = (h.paint & PI_SOLID) ? rgb_over_div255(pix[k], alpha, h.rgb)
                                              : rgb_over(pix[k], rgb_a_src(alpha, shape), h.rgb);
            } else {
                pix[k] = gray_over(pix[k], cov[q], gamma, alpha, g, 255u - alpha, alpha * g);
            }
        }
    }
}

template <int TW, int TH, bool RGB>
__device__ __forceinline__ void composite_box(const HitInfo& h, int rowmap, int X0, int Y0, const uint8_t* gamma,
                                              uint32_t (&pix)[CompLayout<TW, TH>::NPIX]) {
    using L = CompLayout<TW, TH>;
    constexpr int ITERS = HitRows<TW, TH>::ITERS;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int slot = lane / L::LPR, col = (lane % L::LPR) * L::PX;
    const int32_t S0 = static_cast<int32_t>(h.goff), S1 = static_cast<int32_t>(h.run_cnt);
    const uint32_t g = h.paint & 0xff, alpha = (h.paint >> 8) & 0xff;
    int32_t cx[L::PX];
#pragma unroll
    for (int q = 0; q < L::PX; ++q) {
        const int32_t a = 4 * (X0 + col + q);
        cx[q] = max(0, min(a + 4, S1) - max(a, S0));
    }
#pragma unroll
    for (int it = 0; it < ITERS; ++it) {
        const int y = Y0 + (w * L::RPW + slot) + it * L::NW * L::RPW;
        const int32_t r = rowmap ? 16 * y + 12 : 4 * y;
        const int32_t cy = (y >= h.py0 && y <= h.py1) ? max(0, min(r + 4, h.g1 + 1) - max(r, h.g0)) : 0;
        if (cy == 0) continue;  // the box misses this row
#pragma unroll
        for (int q = 0; q < L::PX; ++q) {
            const int32_t cov = cx[q] * cy;
            if (cov == 0) continue;
            const int k = it * L::PX + q;
            if (RGB) {
                pix[k] = rgb_over(pix[k], rgb_a_src(alpha, gamma[cov]), h.rgb);
            } else {
                pix[k] = gray_over(pix[k], cov, gamma, alpha, g, 255u - alpha, alpha * g);
            }
        }
    }
}

// RGB: the pages are Rgb8 (3 bytes per pixel) and path_rgb[p] is path p's
// colour; otherwise Gray8 pages painted with each path's gray.
template <int TW, int TH, bool RGB, bool FEW>
__global__ void __launch_bounds__(comp_threads(TW, TH), comp_ctas_per_sm(TW, TH)) k_composite(
    const PathInfo* __restrict__ info, const PageGeom* __restrict__ pages, uint32_t n_pages, uint32_t n_tiles,
    int stw, int sth, const uint32_t* __restrict__ super_off, const uint32_t* __restrict__ super_list,
    const uint32_t* __restrict__ group_off, const uint2* __restrict__ gidx, const uint32_t* __restrict__ cells,
    const int4* __restrict__ runs, uint8_t* __restrict__ arena, int rowmap, BatchCounters* __restrict__ ctr,
    const uint32_t* __restrict__ path_rgb, const uint32_t* __restrict__ super_start) {
    using L = CompLayout<TW, TH>;
    constexpr int ITERS = TH / (L::NW * L::RPW);
    constexpr int NPIX = L::NPIX;
    constexpr int COMP_CHUNK = L::NT;
    static_assert(ITERS * L::PX == NPIX, "tile shape must cover the CTA exactly");
    __shared__ HitInfo hits[COMP_CHUNK];
    // Gray pages: per hit, the full-coverage blend's constants packed as
    // (255 - a) | a * g << 8 (a_src = div255(a * AA_GAMMA[16]) = a).
    __shared__ uint32_t hcoef[RGB ? 1 : COMP_CHUNK];
    __shared__ uint32_t wcnt[L::NW];
    __shared__ uint8_t gamma[17];
    __shared__ int32_t mark[L::NW * L::RPW][TW];
    // Two maps, used in turn: a run's map is written while no thread can still
    // be reading the one before it (one barrier per run).
    __shared__ uint8_t lut[2][RGB ? 768 : 256];
    // Gray pages: the values a run of full-tile layers meets. A tile holds few
    // distinct values, so the run's map is composed for those alone: every
    // thread marks its pixels' values, warp 0 lists and clears the marks and
    // composes the layers for each listed value (seen[] is all zero between runs).
    __shared__ __align__(8) uint8_t seen[RGB ? 8 : 256];
    __shared__ uint8_t vals[RGB ? 4 : 256];
    __shared__ uint32_t red[L::NW];
    // Bit k: hit k of the chunk is not a full-tile layer (where a run of full layers ends).
    __shared__ uint32_t partial[COMP_CHUNK / 32];
    // Bit k: hit k reads coverage cells (neither a full-tile layer nor a box):
    // the hits the load pipeline runs over.
    __shared__ uint32_t pathbits[COMP_CHUNK / 32];
    __shared__ uint32_t next_tile;
    if (threadIdx.x < 17) gamma[threadIdx.x] = c_gamma[threadIdx.x];
    if (!RGB && threadIdx.x < 256) seen[threadIdx.x] = 0;  // ordered before use by take()'s barrier
    if (ctr->err) return;  // a capacity overflow upstream: leave the pages untouched
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int col = (lane % L::LPR) * L::PX;
    int lut_sel = 0;
    // Persistent CTAs take tiles from a work queue (ctr->tile_cursor, zeroed
    // with the batch counters): a tile's cost ranges from nothing to
    // thousands of layers, so tiles go to whichever CTA is free.
    auto take = [&]() {
        __syncthreads();  // every thread is done with the previous index
        if (threadIdx.x == 0) next_tile = atomicAdd(&ctr->tile_cursor, 1u);
        __syncthreads();
        return next_tile;
    };
    for (uint32_t t = take(); t < n_tiles; t = take()) {
        const uint32_t pg = find_page_by(pages, n_pages, t, false);
        const PageGeom G = pages[pg];
        const uint32_t lt = t - G.tile_base;
        const int tx = static_cast<int>(lt % G.ntx), ty = static_cast<int>(lt / G.ntx);
        const int X0 = tx * TW, Y0 = ty * TH;
        const int W = static_cast<int>(G.w), H = static_cast<int>(G.h);
        uint8_t* page = arena + G.offset;
        uint32_t pix[NPIX];
#pragma unroll
        for (int it = 0; it < ITERS; ++it) {
            const int y = Y0 + (w * L::RPW + lane / L::LPR) + it * L::NW * L::RPW;
#pragma unroll
            for (int q = 0; q < L::PX; ++q) {
                const int x = X0 + col + q;
                uint32_t v = 0;
                if (y < H && x < W) {
                    if (RGB) {
                        const uint8_t* p = page + 3 * (static_cast<size_t>(y) * W + x);
                        v = p[0] | (uint32_t(p[1]) << 8) | (uint32_t(p[2]) << 16);
                    } else {
                        v = page[static_cast<size_t>(y) * W + x];
                    }
                }
                pix[it * L::PX + q] = v;
            }
        }
        const uint32_t sx = static_cast<uint32_t>(X0 / stw), sy = static_cast<uint32_t>(Y0 / sth);
        const uint32_t q0 = G.work_base + (sy * G.nsx + sx) * G.nblk;
        const uint32_t l0 = super_off[q0], l1 = super_off[q0 + G.nblk];
        // The supertile's last opaque full layer (position + 1, or 0).
        const uint32_t s_open = super_start[G.super_base + sy * G.nsx + sx];
        // The tile clipped to the page: a path whose solid box holds it covers
        // every pixel that matters with coverage 16.
        const int TX1 = min(X0 + TW, W) - 1, TY1 = min(Y0 + TH, H) - 1;
        auto full_over = [&](const PathInfo& P) {
            return P.bx0 <= X0 && P.bx1 >= TX1 && P.by0 <= Y0 && P.by1 >= TY1;
        };
        // Pre-pass: the last opaque layer covering the whole tile sets every
        // pixel to its colour (div255(255 * g) = g; on Rgb8 pages
        // (255 * s + 255) >> 8 = s), so compositing starts there.
        uint32_t start = l0;
        {
            // Only layers from the supertile's opaque start on can start the tile.
            uint32_t best = s_open;
            const uint32_t scan0 = s_open ? s_open : l0;
            for (uint32_t c0 = scan0; c0 < l1; c0 += COMP_CHUNK) {
                const uint32_t q = c0 + threadIdx.x;
                if (q < l1) {
                    const PathInfo P = info[super_list[q]];
                    if (((P.paint >> 8) & 0xff) == 255u && full_over(P)) best = q + 1;
                }
            }
            for (int o = 16; o; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
            if (lane == 0) red[w] = best;
            __syncthreads();
#pragma unroll
            for (int k = 0; k < L::NW; ++k) best = max(best, red[k]);
            __syncthreads();
            if (best) start = best - 1;
        }
        for (uint32_t c0 = l0 + ((start - l0) / COMP_CHUNK) * COMP_CHUNK; c0 < l1; c0 += COMP_CHUNK) {
            const uint32_t q = c0 + threadIdx.x;
            bool hit = false;
            PathInfo P;
            if (q < l1 && q >= start) {
                P = info[super_list[q]];
                hit = P.px0 <= X0 + TW - 1 && P.px1 >= X0 && P.py0 <= Y0 + TH - 1 && P.py1 >= Y0 && P.px0 <= P.px1;
            }
            const uint32_t m = __ballot_sync(0xffffffffu, hit);
            if (lane == 0) wcnt[w] = __popc(m);
            if (threadIdx.x < COMP_CHUNK / 32) partial[threadIdx.x] = pathbits[threadIdx.x] = 0u;
            __syncthreads();
            uint32_t before = 0, total = 0;
#pragma unroll
            for (int k = 0; k < L::NW; ++k) {
                const uint32_t v = wcnt[k];
                before += k < w ? v : 0u;
                total += v;
            }
            if (hit) {
                const uint32_t pos = before + __popc(m & lanemask_lt());
                HitInfo hi;
                const bool box = (P.paint & PI_BOX) != 0;  // boxes keep AA rows, the others pixel-row groups
                hi.g0 = box ? P.y0 : P.y0 >> 2;
                hi.g1 = box ? P.y1 : P.y1 >> 2;
                hi.py0 = P.py0;
                hi.py1 = P.py1;
                hi.goff = (P.paint & PI_RECTI) ? P.run_off : group_off[super_list[q]];
                hi.run_cnt = P.run_cnt;
                hi.rgb = RGB ? path_rgb[super_list[q]] : 0u;
                const bool full = full_over(P);
                hi.paint = P.paint | (full ? HIT_FULL : 0u);
                hits[pos] = hi;
                if (!full) atomicOr(&partial[pos >> 5], 1u << (pos & 31));
                if (!full && !box) atomicOr(&pathbits[pos >> 5], 1u << (pos & 31));
                if (!RGB) {
                    const uint32_t a = (P.paint >> 8) & 0xffu, g = P.paint & 0xffu;
                    hcoef[pos] = (255u - a) | ((a * g) << 8);
                }
            }
            __syncthreads();
            // The first hit at or after `from` whose bit is set in bits[] (or total).
            auto next_set = [&](const uint32_t* bits, uint32_t from) {
                uint32_t wd = from >> 5;
                uint32_t b = from < total ? bits[wd] & (0xffffffffu << (from & 31)) : 0u;
                while (!b && 32 * (wd + 1) < total) b = bits[++wd];
                return b ? 32 * wd + static_cast<uint32_t>(__ffs(b) - 1) : total;
            };
            // Software pipeline over the hits that read cells (path hits): the
            // index entries of the path hit after next and the first cells of
            // the next one are in flight while a path hit is blended, and across
            // the boxes and full-tile runs between them, which load nothing.
            // A run of layers covering the whole tile is applied as one 256-entry
            // map (one blend per thread per layer) instead of per pixel.
#if RRB_COMP_PIPE_DEPTH >= 2
            HitRows<TW, TH> cur, nxt, nxt2;
#else
            HitRows<TW, TH> cur, nxt;
#endif
            const uint32_t p0 = next_set(pathbits, 0);
            uint32_t p1 = p0 < total ? next_set(pathbits, p0 + 1) : total;  // the path hit after the next one
            if (p0 < total) load_hit_index<TW, TH>(hits[p0], rowmap, Y0, H, gidx, runs, cur);
            if (p1 < total) load_hit_index<TW, TH>(hits[p1], rowmap, Y0, H, gidx, runs, nxt);
            if (p0 < total) load_hit_cells<TW, TH>(cells, cur);
            uint32_t k = 0;
            while (k < total) {
                const uint32_t kpaint = hits[k].paint;
                if (kpaint & HIT_FULL) {
                    const uint32_t m = next_set(partial, k + 1);
                    if (RGB) {
                        // One map per channel (each channel composes on its own).
                        if (m - k >= 2) {
                            uint8_t* map = lut[lut_sel];
                            lut_sel ^= 1;
                            if (threadIdx.x < 256) {
                                uint32_t v = threadIdx.x | (threadIdx.x << 8) | (threadIdx.x << 16);
                                for (uint32_t i = k; i < m; ++i)
                                    v = rgb_over(v, rgb_a_src((hits[i].paint >> 8) & 0xff, 255u), hits[i].rgb);
                                map[threadIdx.x] = static_cast<uint8_t>(v);
                                map[256 + threadIdx.x] = static_cast<uint8_t>(v >> 8);
                                map[512 + threadIdx.x] = static_cast<uint8_t>(v >> 16);
                            }
                            __syncthreads();
#pragma unroll
                            for (int j = 0; j < NPIX; ++j)
                                pix[j] = map[pix[j] & 0xffu] | (uint32_t(map[256 + ((pix[j] >> 8) & 0xffu)]) << 8) |
                                         (uint32_t(map[512 + (pix[j] >> 16)]) << 16);
                        } else {
                            const uint32_t a = rgb_a_src((hits[k].paint >> 8) & 0xff, 255u), s = hits[k].rgb;
#pragma unroll
                            for (int j = 0; j < NPIX; ++j) pix[j] = rgb_over(pix[j], a, s);
                        }
                    } else if (m - k > kDirectRun) {
                        uint8_t* map = lut[lut_sel];
                        lut_sel ^= 1;
#pragma unroll
                        for (int j = 0; j < NPIX; ++j) seen[pix[j]] = 1;
                        __syncthreads();
                        if (w == 0) {
                            // List the marked values (lane l owns seen[8l .. 8l+7]) and clear them.
                            const uint2 wd = reinterpret_cast<const uint2*>(seen)[lane];
                            const uint32_t n_mine = __popc(__vcmpne4(wd.x, 0u)) / 8 + __popc(__vcmpne4(wd.y, 0u)) / 8;
                            uint32_t at = n_mine;
                            for (int o = 1; o < 32; o <<= 1) {
                                const uint32_t t = __shfl_up_sync(0xffffffffu, at, o);
                                if (lane >= o) at += t;
                            }
                            const uint32_t n_vals = __shfl_sync(0xffffffffu, at, 31);
                            at -= n_mine;
#pragma unroll
                            for (int b = 0; b < 8; ++b) {
                                const uint32_t byte = ((b < 4 ? wd.x : wd.y) >> (8 * (b & 3))) & 0xffu;
                                if (byte) vals[at++] = static_cast<uint8_t>(8 * lane + b);
                            }
                            reinterpret_cast<uint2*>(seen)[lane] = make_uint2(0u, 0u);
                            __syncwarp();
                            for (uint32_t q = lane; q < n_vals; q += 32) {
                                const uint32_t v0 = vals[q];
                                uint32_t v = v0;
                                // div255 of x <= 255 * 255 needs no clamp.
#pragma unroll 4
                                for (uint32_t i = k; i < m; ++i) {
                                    const uint32_t cf = hcoef[i];
                                    const uint32_t x = (cf & 0xffu) * v + (cf >> 8);
                                    v = (x + (x >> 8) + 0x80u) >> 8;
                                }
                                map[v0] = static_cast<uint8_t>(v);
                            }
                        }
                        __syncthreads();
#pragma unroll
                        for (int j = 0; j < NPIX; ++j) pix[j] = map[pix[j]];
                    } else {
                        // A short run: each pixel takes the layers one by one
                        // (no map, no barrier).
                        for (uint32_t i = k; i < m; ++i) {
                            const uint32_t cf = hcoef[i], inv = cf & 0xffu, ag = cf >> 8;
#pragma unroll
                            for (int j = 0; j < NPIX; ++j) pix[j] = div255_small(inv * pix[j] + ag);
                        }
                    }
                    k = m;
                    continue;
                }
                if (kpaint & PI_BOX) {
                    composite_box<TW, TH, RGB>(hits[k], rowmap, X0, Y0, gamma, pix);
                    ++k;
                    continue;
                }
                // A path hit (k is the pipeline's current one): the index loads
                // of the path hit after p1 and the cells of p1 go out first.
                const uint32_t p2 = p1 < total ? next_set(pathbits, p1 + 1) : total;
#if RRB_COMP_PIPE_DEPTH >= 2
                if (p2 < total) load_hit_index<TW, TH>(hits[p2], rowmap, Y0, H, gidx, runs, nxt2);
#endif
                if (p1 < total) load_hit_cells<TW, TH>(cells, nxt);
                composite_path_rows<TW, TH, RGB, FEW>(hits[k], cur, X0, cells, gamma, mark, pix);
                cur = nxt;
#if RRB_COMP_PIPE_DEPTH >= 2
                nxt = nxt2;
#else
                // One buffer fewer: p2's index loads go out once p1 is current.
                if (p2 < total) load_hit_index<TW, TH>(hits[p2], rowmap, Y0, H, gidx, runs, nxt);
#endif
                p1 = p2;
                ++k;
            }
            __syncthreads();
        }
#pragma unroll
        for (int it = 0; it < ITERS; ++it) {
            const int y = Y0 + (w * L::RPW + lane / L::LPR) + it * L::NW * L::RPW;
#pragma unroll
            for (int q = 0; q < L::PX; ++q) {
                const int x = X0 + col + q;
                if (y < H && x < W) {
                    const uint32_t v = pix[it * L::PX + q];
                    if (RGB) {
                        uint8_t* p = page + 3 * (static_cast<size_t>(y) * W + x);
                        p[0] = static_cast<uint8_t>(v);
                        p[1] = static_cast<uint8_t>(v >> 8);
                        p[2] = static_cast<uint8_t>(v >> 16);
                    } else {
                        page[static_cast<size_t>(y) * W + x] = static_cast<uint8_t>(v);
                    }
                }
            }
        }
    }
}

// rgb_to_gray (crates/pdf_raster/src/render.rs:1306-1324): BT.709 luma,
// (2126 r + 7152 g + 722 b + 5000) / 10000, exact in integers.
__global__ void k_rgb_to_gray(const uint8_t* __restrict__ rgb, uint8_t* __restrict__ gray, uint64_t n) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t r = rgb[3 * i], g = rgb[3 * i + 1], b = rgb[3 * i + 2];
        gray[i] = static_cast<uint8_t>((2126u * r + 7152u * g + 722u * b + 5000u) / 10000u);
    }
}

}  // namespace rrb
