// rrb_features.cpp — page features of the learned cost model.
//
// The cost model predicts the device time of rendering one page with one
// composite tile shape from features that are cheap to compute on the host
// before the page is rendered (one pass over its points and a difference
// array over the tile grid), so that a scheduler can use them to choose the
// tile shape and the order in which queued pages are admitted.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/rrb.h"

namespace {

// Flattened line count of one cubic (an estimate of the De Casteljau piece
// count at this flatness: the largest second difference of the control
// polygon bounds the deviation of a chord, which falls by 4 per halving).
double cubic_pieces(const double* p, double flatness) {
    const double ax = p[0] - 2 * p[2] + p[4], ay = p[1] - 2 * p[3] + p[5];
    const double bx = p[2] - 2 * p[4] + p[6], by = p[3] - 2 * p[5] + p[7];
    const double dd = std::sqrt(std::max(ax * ax + ay * ay, bx * bx + by * by));
    const double f = std::max(flatness, 1e-3);
    return std::min(1024.0, std::max(1.0, std::ceil(std::sqrt(0.75 * dd / f))));
}

int tile_index(uint32_t w, uint32_t h) {
    if (w == 16 && h == 16) return 0;
    if (w == 32 && h == 32) return 1;
    if (w == 64 && h == 16) return 2;
    return -1;
}

// All three tile shapes of one page in one pass over its points: the
// shape-independent features once, then one difference-array histogram per
// tile shape. out: [3][RRB_MLP_IN], rows in the order 16x16, 32x32, 64x16.
int features_all(const rrb_path_batch_params* p, uint32_t page, float* out) {
    if (!p || !out || page >= p->n_pages || !p->page_width || !p->page_height) return RRB_ERR_INVARIANT;
    if (p->n_paths && (!p->path_page || !p->path_pt_off || !p->pts || !p->flags || !p->fill_rule || !p->alpha))
        return RRB_ERR_INVARIANT;
    const double W = p->page_width[page], H = p->page_height[page];
    const double* m = p->matrix;
    const bool ident = m[0] == 1.0 && m[1] == 0.0 && m[2] == 0.0 && m[3] == 1.0 && m[4] == 0.0 && m[5] == 0.0;
    const uint32_t* pp = p->path_page;
    const uint64_t b = p->n_paths ? static_cast<uint64_t>(std::lower_bound(pp, pp + p->n_paths, page) - pp) : 0;
    const uint64_t e = p->n_paths ? static_cast<uint64_t>(std::upper_bound(pp, pp + p->n_paths, page) - pp) : 0;
    struct Box {
        double x0, y0, x1, y1;
    };
    std::vector<Box> boxes;
    boxes.reserve(e - b);
    double n_pts = 0, n_lines = 0, n_curves = 0, edges = 0, length = 0, area_sum = 0;
    double eo = 0, translucent = 0, recti = 0;
    for (uint64_t k = b; k < e; ++k) {
        const uint64_t a0 = p->path_pt_off[k], a1 = p->path_pt_off[k + 1];
        n_pts += static_cast<double>(a1 - a0);
        eo += p->fill_rule[k] ? 1 : 0;
        translucent += p->alpha[k] < 255 ? 1 : 0;
        double x0 = 1e300, y0 = 1e300, x1 = -1e300, y1 = -1e300;
        bool axis = true;
        double px = 0, py = 0;
        for (uint64_t i = a0; i < a1; ++i) {
            const double sx = p->pts[2 * i], sy = p->pts[2 * i + 1];
            const double x = ident ? sx : m[0] * sx + m[2] * sy + m[4];
            const double y = ident ? sy : m[1] * sx + m[3] * sy + m[5];
            x0 = std::min(x0, x);
            y0 = std::min(y0, y);
            x1 = std::max(x1, x);
            y1 = std::max(y1, y);
            const uint8_t f = p->flags[i];
            if (i > a0 && !(f & RRB_PATH_FIRST)) {
                if (f & RRB_PATH_CURVE) {
                    // The first of two control points starts a cubic: (prev, c1, c2, end).
                    if (i + 2 < a1 && (p->flags[i + 1] & RRB_PATH_CURVE)) {
                        double q[8] = {px, py, x, y, 0, 0, 0, 0};
                        for (int j = 1; j <= 2; ++j) {
                            const double cx = p->pts[2 * (i + j)], cy = p->pts[2 * (i + j) + 1];
                            q[2 + 2 * j] = m[0] * cx + m[2] * cy + m[4];
                            q[3 + 2 * j] = m[1] * cx + m[3] * cy + m[5];
                        }
                        n_curves += 1;
                        edges += cubic_pieces(q, p->flatness);
                        const double dx = q[6] - q[0], dy = q[7] - q[1];
                        length += std::sqrt(dx * dx + dy * dy);
                        axis = false;
                    }
                } else if (!(i > a0 + 1 && (p->flags[i - 1] & RRB_PATH_CURVE))) {
                    n_lines += 1;
                    edges += 1;
                    const double dx = x - px, dy = y - py;
                    length += std::sqrt(dx * dx + dy * dy);
                    axis = axis && (x == px || y == py);
                }
            }
            px = x;
            py = y;
        }
        if (x0 > x1) continue;
        recti += axis ? 1 : 0;
        const double cx0 = std::max(0.0, x0), cy0 = std::max(0.0, y0);
        const double cx1 = std::min(W, x1), cy1 = std::min(H, y1);
        if (cx0 >= cx1 || cy0 >= cy1) continue;
        area_sum += (cx1 - cx0) * (cy1 - cy0);
        boxes.push_back({cx0, cy0, cx1, cy1});
    }
    const double n_paths = static_cast<double>(e - b), segs = n_lines + n_curves;
    float base[13];
    base[0] = static_cast<float>(std::log1p(W * H));
    base[1] = static_cast<float>(std::log1p(n_paths));
    base[2] = static_cast<float>(std::log1p(n_pts));
    base[3] = static_cast<float>(segs > 0 ? n_lines / segs : 0);
    base[4] = static_cast<float>(std::log1p(n_curves));
    base[5] = static_cast<float>(std::log1p(edges));
    base[6] = static_cast<float>(std::log1p(segs > 0 ? length / segs : 0));
    base[7] = static_cast<float>(std::log1p(area_sum / (W * H)));
    base[8] = static_cast<float>(std::log1p(n_paths > 0 ? area_sum / n_paths : 0));
    base[9] = static_cast<float>(n_paths > 0 ? eo / n_paths : 0);
    base[10] = static_cast<float>(n_paths > 0 ? translucent / n_paths : 0);
    base[11] = static_cast<float>(n_paths > 0 ? recti / n_paths : 0);
    static const uint32_t kShape[3][2] = {{16, 16}, {32, 32}, {64, 16}};
    std::vector<int32_t> diff;
    for (int t = 0; t < 3; ++t) {
        const uint32_t tw = kShape[t][0], th = kShape[t][1];
        const uint32_t gw = static_cast<uint32_t>((W + tw - 1) / tw), gh = static_cast<uint32_t>((H + th - 1) / th);
        diff.assign(static_cast<size_t>(gw + 1) * (gh + 1), 0);
        const size_t st = gw + 1;
        for (const Box& bx : boxes) {
            const uint32_t tx0 = static_cast<uint32_t>(bx.x0 / tw), ty0 = static_cast<uint32_t>(bx.y0 / th);
            const uint32_t tx1 = std::min(gw - 1, static_cast<uint32_t>(bx.x1 / tw));
            const uint32_t ty1 = std::min(gh - 1, static_cast<uint32_t>(bx.y1 / th));
            diff[ty0 * st + tx0] += 1;
            diff[ty0 * st + tx1 + 1] -= 1;
            diff[(ty1 + 1) * st + tx0] -= 1;
            diff[(ty1 + 1) * st + tx1 + 1] += 1;
        }
        // Paths per tile (2-D prefix sum of the rectangle marks) -> 8-bin
        // histogram in powers of 4.
        double hist[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        std::vector<int32_t> col(gw + 1, 0);
        for (uint32_t y = 0; y < gh; ++y) {
            int32_t run = 0;
            for (uint32_t x = 0; x < gw; ++x) {
                col[x] += diff[static_cast<size_t>(y) * st + x];
                run += col[x];
                int bin = 0;
                for (int32_t v = run; v > 0 && bin < 7; v >>= 2) ++bin;  // 0, 1-3, 4-15, ..., >= 4096
                hist[bin] += 1;
            }
        }
        const double tiles = static_cast<double>(gw) * gh;
        float* o = out + t * RRB_MLP_IN;
        for (int k = 0; k < 12; ++k) o[k] = base[k];
        o[12] = static_cast<float>(tiles > 0 ? 1.0 - hist[0] / tiles : 0);
        for (int k = 0; k < 8; ++k) o[13 + k] = static_cast<float>(tiles > 0 ? hist[k] / tiles : 0);
        o[21] = t == 0 ? 1.f : 0.f;
        o[22] = t == 1 ? 1.f : 0.f;
        o[23] = t == 2 ? 1.f : 0.f;
    }
    return RRB_OK;
}

}  // namespace

extern "C" int rrb_page_features_all(const rrb_path_batch_params* p, uint32_t page, float* out) {
    return features_all(p, page, out);
}

extern "C" int rrb_page_features(const rrb_path_batch_params* p, uint32_t page, uint32_t tile_w, uint32_t tile_h,
                                 float* out) {
    const int ti = tile_index(tile_w, tile_h);
    if (ti < 0 || !out) return RRB_ERR_INVARIANT;
    float all[3 * RRB_MLP_IN];
    const int rc = features_all(p, page, all);
    if (rc) return rc;
    std::memcpy(out, all + ti * RRB_MLP_IN, RRB_MLP_IN * sizeof(float));
    return RRB_OK;
}
