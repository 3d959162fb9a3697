// fill_oracle.cpp — CPU restatement of the reference's aa_fill / tile_fill
// operators and its tile-record builder. TEST INFRASTRUCTURE ONLY.
//
// Compiled with -ffp-contract=off: every multiply-add below is unfused
// unless written as std::fmaf, which is exactly where the reference's Rust
// uses f32::mul_add (fill.rs). tile_fill.cu is restated as written, every
// operation rounded on its own (IEEE f32, no contraction).

#include "fill_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace {

constexpr uint32_t kTileW = 16, kTileH = 16;  // TILE_W / TILE_H (lib.rs:122-124)

// The 64 sample offsets of aa_fill (fill.rs:272-345, aa_fill.cu JITTER_X/Y):
// x = Halton base 2 of n = 1..64 (exact binary fractions); y = Halton base 3
// of n = 1..64 written with 6 decimals, so the f32 value is the one nearest
// to the 6-decimal rounding, not to the exact 1/3-based fraction.
double radical_inverse(uint32_t n, uint32_t base) {
    double inv = 1.0 / base, f = inv, r = 0.0;
    while (n) {
        r += f * static_cast<double>(n % base);
        n /= base;
        f *= inv;
    }
    return r;
}

struct Jitter {
    float x[64], y[64];
    Jitter() {
        for (uint32_t i = 0; i < 64; ++i) {
            x[i] = static_cast<float>(radical_inverse(i + 1, 2));
            const double h3 = radical_inverse(i + 1, 3);
            y[i] = static_cast<float>(std::nearbyint(h3 * 1e6) / 1e6);
        }
    }
};
const Jitter kJitter;

// aa_fill_cpu_sample (fill.rs:400-421).
bool sample_inside(const float* segs, uint32_t n, float sx, float sy, int eo) {
    int32_t w = 0;
    for (uint32_t k = 0; k < n; ++k) {
        const float x0 = segs[4 * k], y0 = segs[4 * k + 1], x1 = segs[4 * k + 2], y1 = segs[4 * k + 3];
        if (y0 <= sy && sy < y1) {
            const float t = (sy - y0) / (y1 - y0);
            const float xi = std::fmaf(t, x1 - x0, x0);
            if (xi >= sx) w += 1;
        } else if (y1 <= sy && sy < y0) {
            const float t = (sy - y1) / (y0 - y1);
            const float xi = std::fmaf(t, x0 - x1, x1);
            if (xi >= sx) w -= 1;
        }
    }
    return eo ? (w & 1) != 0 : w != 0;
}

// Rust `f32 as i32` / `as u32`: truncation toward zero, saturating, NaN -> 0.
int32_t sat_i32(float v) {
    if (std::isnan(v)) return 0;
    if (v <= -2147483648.0f) return INT32_MIN;
    if (v >= 2147483648.0f) return INT32_MAX;
    return static_cast<int32_t>(v);
}
uint32_t sat_u32(float v) {
    if (std::isnan(v) || v <= 0.0f) return 0;
    if (v >= 4294967296.0f) return UINT32_MAX;
    return static_cast<uint32_t>(v);
}

// segment_pixel_area (tile_fill.cu:64-115).
float segment_pixel_area(float x_enter, float dxdy, float iy0, float iy1, float sign, float px) {
    const float y_len = iy1 - iy0;
    if (y_len <= 0.0f) return 0.0f;
    const float x0 = x_enter;
    const float x1 = x_enter + dxdy * y_len;
    const float xl = std::fmin(x0, x1), xr = std::fmax(x0, x1);
    float cover;
    if (xr <= px) {
        cover = 0.0f;
    } else if (xl >= px + 1.0f) {
        cover = y_len;
    } else {
        const float dx = xr - xl;
        if (dx < 1e-6f) {
            const float xmid = 0.5f * (x0 + x1);
            cover = (xmid >= px + 0.5f) ? y_len : 0.0f;
        } else {
            const float left = std::fmax(xl, px);
            const float right = std::fmin(xr, px + 1.0f);
            const float yf_left = (left - xl) / dx * y_len;
            const float yf_right = (right - xl) / dx * y_len;
            const float above = y_len - yf_right;
            cover = (yf_right - yf_left) + above;
        }
    }
    return sign * cover;
}

}  // namespace

extern "C" {

void or_aa_jitter(float* x, float* y) {
    std::memcpy(x, kJitter.x, sizeof kJitter.x);
    std::memcpy(y, kJitter.y, sizeof kJitter.y);
}

void or_aa_fill_cpu(const float* segs, uint32_t n_segs, float x_min, float y_min, uint32_t width,
                    uint32_t height, int eo, uint8_t* out) {
    for (uint32_t py = 0; py < height; ++py) {
        for (uint32_t px = 0; px < width; ++px) {
            const float cx = x_min + static_cast<float>(px) + 0.5f;
            const float cy = y_min + static_cast<float>(py) + 0.5f;
            uint32_t hits = 0;
            for (int s = 0; s < 64; ++s) {
                const float sx = cx + kJitter.x[s] - 0.5f;
                const float sy = cy + kJitter.y[s] - 0.5f;
                hits += sample_inside(segs, n_segs, sx, sy, eo) ? 1u : 0u;
            }
            out[static_cast<size_t>(py) * width + px] = static_cast<uint8_t>((hits * 255 + 32) >> 6);
        }
    }
}

int64_t or_build_tile_records(const float* segs, uint32_t n_segs, float x_min, float y_min, uint32_t width,
                              uint32_t height, or_tile_record* records, uint32_t* tile_starts,
                              uint32_t* tile_counts, uint32_t* grid_w_out) {
    const uint32_t grid_w = (width + kTileW - 1) / kTileW, grid_h = (height + kTileH - 1) / kTileH;
    if (grid_w > 0xFFFF || grid_h > 0xFFFF) return -1;
    if (grid_w_out) *grid_w_out = grid_w;
    const float tw = static_cast<float>(kTileW), th = static_cast<float>(kTileH);
    std::vector<or_tile_record> recs;
    for (uint32_t k = 0; k < n_segs; ++k) {
        float sx0 = segs[4 * k] - x_min, sy0 = segs[4 * k + 1] - y_min;
        float sx1 = segs[4 * k + 2] - x_min, sy1 = segs[4 * k + 3] - y_min;
        const float dy = std::fabs(sy1 - sy0);
        if (!std::isfinite(dy) || dy < 1e-6f || !std::isfinite(sx0) || !std::isfinite(sx1)) continue;
        float sign = 1.0f;
        if (sy0 > sy1) {
            std::swap(sx0, sx1);
            std::swap(sy0, sy1);
            sign = -1.0f;
        }
        const float dxdy = (sx1 - sx0) / (sy1 - sy0);
        const float ey0 = std::fmax(sy0, 0.0f);
        const float ey1 = std::fmin(sy1, static_cast<float>(height));
        if (ey0 >= ey1) continue;
        const uint32_t ty0 = sat_u32(std::floor(ey0 / th));
        const uint32_t ty1 = sat_u32(std::floor(std::fmax(ey1 - 1e-6f, 0.0f) / th));
        const uint32_t ty_end = std::min(ty1, grid_h - 1);
        for (uint64_t ty = ty0; ty <= ty_end; ++ty) {
            const float tile_top = static_cast<float>(static_cast<uint32_t>(ty) * kTileH);
            const float tile_bot = tile_top + th;
            const float seg_y0_tile = std::fmax(ey0, tile_top) - tile_top;
            const float seg_y1_tile = std::fmin(ey1, tile_bot) - tile_top;
            if (seg_y0_tile >= seg_y1_tile) continue;
            const float x_enter_global = std::fmaf(dxdy, std::fmax(ey0, tile_top) - sy0, sx0);
            const float x_at_exit = std::fmaf(dxdy, seg_y1_tile - seg_y0_tile, x_enter_global);
            const float xl = std::fmin(x_enter_global, x_at_exit);
            const float xr = std::fmax(x_enter_global, x_at_exit);
            const int32_t tx0_i = sat_i32(std::floor(xl / tw));
            const int32_t tx1_i = sat_i32(std::floor(xr / tw));
            if (tx1_i < 0) continue;
            const uint32_t tx0 = static_cast<uint32_t>(std::max(tx0_i, 0));
            const uint32_t tx1 = std::min(static_cast<uint32_t>(tx1_i), grid_w - 1);
            for (uint64_t tx = tx0; tx <= tx1; ++tx) {
                or_tile_record r;
                r.key = (static_cast<uint32_t>(ty) << 16) | static_cast<uint32_t>(tx);
                r.x_enter = x_enter_global - static_cast<float>(static_cast<uint32_t>(tx) * kTileW);
                r.dxdy = dxdy;
                r.y0_tile = seg_y0_tile;
                r.y1_tile = seg_y1_tile;
                r.sign = sign;
                r.pad = r.pad2 = 0;
                recs.push_back(r);
            }
        }
    }
    std::stable_sort(recs.begin(), recs.end(),
                     [](const or_tile_record& a, const or_tile_record& b) { return a.key < b.key; });
    const size_t n_tiles = static_cast<size_t>(grid_w) * grid_h;
    std::vector<uint32_t> counts(n_tiles, 0);
    for (const or_tile_record& r : recs) {
        const size_t t = static_cast<size_t>(r.key >> 16) * grid_w + (r.key & 0xFFFF);
        if (t < n_tiles) counts[t] += 1;
    }
    if (tile_counts) std::memcpy(tile_counts, counts.data(), n_tiles * sizeof(uint32_t));
    if (tile_starts) {
        uint32_t run = 0;
        for (size_t t = 0; t < n_tiles; ++t) {
            tile_starts[t] = run;
            run += counts[t];
        }
    }
    if (records && !recs.empty()) std::memcpy(records, recs.data(), recs.size() * sizeof(or_tile_record));
    return static_cast<int64_t>(recs.size());
}

void or_tile_fill(const or_tile_record* records, const uint32_t* tile_starts, const uint32_t* tile_counts,
                  uint32_t grid_w, uint32_t width, uint32_t height, int eo, uint8_t* coverage) {
    for (uint32_t py = 0; py < height; ++py) {
        for (uint32_t px = 0; px < width; ++px) {
            const uint32_t tile_idx = (py / kTileH) * grid_w + (px / kTileW);
            const uint32_t start = tile_starts[tile_idx], count = tile_counts[tile_idx];
            const float py_f = static_cast<float>(py % kTileH), px_f = static_cast<float>(px % kTileW);
            float area = 0.0f;
            for (uint32_t r = start; r < start + count; ++r) {
                const or_tile_record& rec = records[r];
                const float iy0 = std::fmax(rec.y0_tile, py_f);
                const float iy1 = std::fmin(rec.y1_tile, py_f + 1.0f);
                if (iy0 >= iy1) continue;
                const float x_at_iy0 = rec.x_enter + rec.dxdy * (iy0 - rec.y0_tile);
                area += segment_pixel_area(x_at_iy0, rec.dxdy, iy0, iy1, rec.sign, px_f);
            }
            int32_t cov;
            if (eo) {
                float a = std::fabs(area);
                a = a - std::floor(a);
                if (a > 0.5f) a = 1.0f - a;
                cov = sat_i32(a * 2.0f * 255.5f);
            } else {
                cov = sat_i32(std::fmin(std::fabs(area), 1.0f) * 255.5f);
            }
            coverage[static_cast<size_t>(py) * width + px] = static_cast<uint8_t>(std::min(cov, 255));
        }
    }
}

}  // extern "C"
