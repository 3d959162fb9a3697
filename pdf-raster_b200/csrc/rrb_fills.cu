// rrb_fills.cu — the reference's two GPU coverage operators behind their own
// parameter layouts: record_aa_fill (64-sample Halton-jittered coverage) and
// record_tile_fill (analytic signed-area coverage over 16x16 tiles), the
// GpuBackend entry points of crates/gpu/src/backend/mod.rs with AaFillParams /
// TileFillParams (backend/params.rs:90-103,170-185). Both write a u8 coverage
// buffer of width x height; neither composites.
//
// aa_fill. The reference launches one 64-thread block per pixel and tests
// every segment at every sample: O(pixels x 64 x segments). Here a CTA owns a
// band of 8 pixel rows (one warp per row) and a 512-column chunk. The band's
// segments are filtered once into shared memory by the exact y-range of its
// samples. All 64 samples of a pixel row share one y per sample index, so
// for each of the row's 64 sample lines the warp gathers that line's
// crossings (x and winding sign), sorts them by x and forms suffix sums of
// the signs; then a pixel's sample is inside iff the suffix sum at the first
// crossing with x >= sample x passes the fill rule — the same set of
// crossings the per-sample test counts, so the result is bit-identical to
// aa_fill_cpu (crates/gpu/src/fill.rs:346-421): IEEE division and the fma of
// its mul_add, evaluated once per (line, segment) instead of per pixel.
//
// tile_fill. Same decomposition as the reference (one 16x16 tile per CTA,
// one pixel per thread), with the tile's records staged through shared
// memory 256 at a time and every operation of tile_fill.cu rounded on its
// own (products via __fmul_rn so that none is contracted into an fma).
// A tile whose [start, start + count) runs past the records buffer is
// treated as empty instead of being read out of bounds.
//
// record_tile_fill_segs builds the records on the device from the same
// segments as aa_fill (build_tile_records, fill.rs:82-264: count, write in
// segment order, stable radix sort by tile key, per-tile ranges by binary
// search), then runs tile_fill: no CPU record build and no upload.

#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>

#include "../../include/rrb.h"
#include "rrb_device_scope.h"

int rrb_ctx_device(const rrb_ctx* c);
bool rrb_ctx_page_open(const rrb_ctx* c);
int rrb_ctx_fail(rrb_ctx* c, int code, const char* msg);
int rrb_ctx_sm_count(const rrb_ctx* c);
int rrb_ctx_fill_scratch(rrb_ctx* c, int k, size_t bytes, void** out);

namespace {

// ---- sample offsets ----------------------------------------------------------
// x: Halton base 2 of n = 1..64 (exact binary fractions). y: Halton base 3 of
// n = 1..64 as the reference writes it, rounded to 6 decimals, then to f32.
struct AaJitter {
    float x[64];
    float y[64];
};

double radical_inverse(uint32_t n, uint32_t base) {
    const double inv = 1.0 / base;
    double f = inv, r = 0.0;
    while (n) {
        r += f * static_cast<double>(n % base);
        n /= base;
        f *= inv;
    }
    return r;
}

const AaJitter& jitter() {
    static const AaJitter j = [] {
        AaJitter t;
        for (uint32_t i = 0; i < 64; ++i) {
            t.x[i] = static_cast<float>(radical_inverse(i + 1, 2));
            t.y[i] = static_cast<float>(std::nearbyint(radical_inverse(i + 1, 3) * 1e6) / 1e6);
        }
        return t;
    }();
    return j;
}

// ---- aa_fill -------------------------------------------------------------------
constexpr int AA_WARPS = 8;              // pixel rows per band
constexpr int AA_PPL = 16;               // pixels per lane
constexpr int AA_CW = 32 * AA_PPL;       // columns per chunk
constexpr int AA_SEG_CAP = 1024;         // band segments kept in shared memory
constexpr int AA_X_CAP = 128;            // crossings per sample line kept in shared memory

// The winding crossing of aa_fill_cpu_sample (fill.rs:400-421) for a sample
// line at sy: true with the crossing x and its sign, false if the segment
// does not span sy or x is NaN (a NaN x never passes `xi >= sx`).
__device__ __forceinline__ bool crossing(const float4 s, float sy, float& xi, int& d) {
    if (s.y <= sy && sy < s.w) {
        const float t = (sy - s.y) / (s.w - s.y);
        xi = fmaf(t, s.z - s.x, s.x);
        d = 1;
    } else if (s.w <= sy && sy < s.y) {
        const float t = (sy - s.w) / (s.y - s.w);
        xi = fmaf(t, s.x - s.z, s.z);
        d = -1;
    } else {
        return false;
    }
    return !isnan(xi);
}

__global__ void __launch_bounds__(AA_WARPS * 32) k_aa_fill(const float4* __restrict__ segs, uint32_t n_segs,
                                                           float x_min, float y_min, uint32_t width,
                                                           uint32_t height, int eo, const __grid_constant__ AaJitter J,
                                                           uint8_t* __restrict__ coverage) {
    __shared__ float4 sseg[AA_SEG_CAP];
    __shared__ float lx[AA_WARPS][AA_X_CAP];     // crossings as gathered
    __shared__ int ld[AA_WARPS][AA_X_CAP];
    __shared__ float sxs[AA_WARPS][AA_X_CAP];    // sorted by x
    __shared__ int suf[AA_WARPS][AA_X_CAP + 1];  // suffix sums of the sorted signs
    __shared__ uint32_t s_count;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t bands = (height + AA_WARPS - 1) / AA_WARPS, chunks = (width + AA_CW - 1) / AA_CW;
    float jy_lo = J.y[0], jy_hi = J.y[0];
    for (int s = 1; s < 64; ++s) {
        jy_lo = fminf(jy_lo, J.y[s]);
        jy_hi = fmaxf(jy_hi, J.y[s]);
    }
    for (uint64_t item = blockIdx.x; item < static_cast<uint64_t>(bands) * chunks; item += gridDim.x) {
        const uint32_t band = static_cast<uint32_t>(item / chunks), chunk = static_cast<uint32_t>(item % chunks);
        const uint32_t r0 = band * AA_WARPS, r1 = min(height, r0 + AA_WARPS) - 1;
        const uint32_t c0 = chunk * AA_CW;
        // Exact extremes of the band's sample y values (each step is monotone).
        const float lo = ((y_min + static_cast<float>(r0)) + 0.5f + jy_lo) - 0.5f;
        const float hi = ((y_min + static_cast<float>(r1)) + 0.5f + jy_hi) - 0.5f;
        if (threadIdx.x == 0) s_count = 0;
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < n_segs; k += blockDim.x) {
            const float4 s = segs[k];
            if (fminf(s.y, s.w) <= hi && fmaxf(s.y, s.w) > lo) {
                const uint32_t at = atomicAdd(&s_count, 1u);
                if (at < AA_SEG_CAP) sseg[at] = s;
            }
        }
        __syncthreads();
        const bool band_ovf = s_count > AA_SEG_CAP;  // then every line reads the global list
        const uint32_t n_src = band_ovf ? n_segs : s_count;
        const float4* src = band_ovf ? segs : sseg;
        const uint32_t py = r0 + w;
        if (py < height) {
            uint32_t hits[AA_PPL];
#pragma unroll
            for (int j = 0; j < AA_PPL; ++j) hits[j] = 0;
            const float cy = (y_min + static_cast<float>(py)) + 0.5f;
            for (int smp = 0; smp < 64; ++smp) {
                const float sy = (cy + J.y[smp]) - 0.5f;
                const float jx = J.x[smp];
                // Gather this sample line's crossings.
                uint32_t n = 0;
                for (uint32_t b = 0; b < n_src; b += 32) {
                    const uint32_t k = b + lane;
                    float xi = 0.f;
                    int d = 0;
                    const bool hit = k < n_src && crossing(src[k], sy, xi, d);
                    const uint32_t m = __ballot_sync(0xffffffffu, hit);
                    const uint32_t at = n + __popc(m & ((1u << lane) - 1u));
                    if (hit && at < AA_X_CAP) {
                        lx[w][at] = xi;
                        ld[w][at] = d;
                    }
                    n += __popc(m);
                }
                __syncwarp();
                if (n <= AA_X_CAP) {
                    // Rank sort by x (ties by gather order), then suffix sums of the signs.
                    for (uint32_t i = lane; i < n; i += 32) {
                        const float xv = lx[w][i];
                        uint32_t rank = 0;
                        for (uint32_t j = 0; j < n; ++j) {
                            const float xj = lx[w][j];
                            rank += (xj < xv || (xj == xv && j < i)) ? 1u : 0u;
                        }
                        sxs[w][rank] = xv;
                        suf[w][rank] = ld[w][i];
                    }
                    __syncwarp();
                    int carry = 0;
                    for (int base = static_cast<int>((n + 31) & ~31u) - 32; base >= 0; base -= 32) {
                        const int i = base + lane;
                        int v = i < static_cast<int>(n) ? suf[w][i] : 0;
                        for (int o = 1; o < 32; o <<= 1) {
                            const int t = __shfl_down_sync(0xffffffffu, v, o);
                            if (lane + o < 32) v += t;
                        }
                        const int total = __shfl_sync(0xffffffffu, v, 0);
                        __syncwarp();
                        if (i < static_cast<int>(n)) suf[w][i] = v + carry;
                        carry += total;
                        __syncwarp();
                    }
                    if (lane == 0) suf[w][n] = 0;
                    __syncwarp();
#pragma unroll
                    for (int j = 0; j < AA_PPL; ++j) {
                        const uint32_t px = c0 + lane + 32u * j;
                        if (px >= width) continue;
                        const float sx = ((x_min + static_cast<float>(px)) + 0.5f + jx) - 0.5f;
                        uint32_t a = 0, z = n;  // first sorted crossing with x >= sx
                        while (a < z) {
                            const uint32_t mid = (a + z) >> 1;
                            if (sxs[w][mid] >= sx) z = mid;
                            else a = mid + 1;
                        }
                        const int wv = suf[w][a];
                        hits[j] += (eo ? (wv & 1) != 0 : wv != 0) ? 1u : 0u;
                    }
                } else {
                    // More crossings than the line's list holds: count per sample.
#pragma unroll
                    for (int j = 0; j < AA_PPL; ++j) {
                        const uint32_t px = c0 + lane + 32u * j;
                        if (px >= width) continue;
                        const float sx = ((x_min + static_cast<float>(px)) + 0.5f + jx) - 0.5f;
                        int wv = 0;
                        for (uint32_t k = 0; k < n_src; ++k) {
                            float xi;
                            int d;
                            if (crossing(src[k], sy, xi, d) && xi >= sx) wv += d;
                        }
                        hits[j] += (eo ? (wv & 1) != 0 : wv != 0) ? 1u : 0u;
                    }
                }
                __syncwarp();
            }
            uint8_t* row = coverage + static_cast<size_t>(py) * width;
#pragma unroll
            for (int j = 0; j < AA_PPL; ++j) {
                const uint32_t px = c0 + lane + 32u * j;
                if (px < width) row[px] = static_cast<uint8_t>((hits[j] * 255u + 32u) >> 6);
            }
        }
        __syncthreads();
    }
}

// ---- tile_fill -----------------------------------------------------------------
constexpr uint32_t TILE = 16;
constexpr int TF_THREADS = TILE * TILE;

struct __align__(16) TileRec {
    uint32_t key;
    float x_enter, dxdy, y0_tile, y1_tile, sign;
    uint32_t pad, pad2;
};
static_assert(sizeof(TileRec) == 32 && sizeof(TileRec) == sizeof(rrb_tile_record), "TileRecord is 32 bytes");

// segment_pixel_area of tile_fill.cu:64-115, every operation rounded on its own.
__device__ __forceinline__ float segment_pixel_area(float x_enter, float dxdy, float iy0, float iy1, float sign,
                                                    float px) {
    const float y_len = iy1 - iy0;
    if (y_len <= 0.0f) return 0.0f;
    const float x0 = x_enter;
    const float x1 = __fadd_rn(x_enter, __fmul_rn(dxdy, y_len));
    const float xl = fminf(x0, x1), xr = fmaxf(x0, x1);
    float cover;
    if (xr <= px) {
        cover = 0.0f;
    } else if (xl >= px + 1.0f) {
        cover = y_len;
    } else {
        const float dx = xr - xl;
        if (dx < 1e-6f) {
            const float xmid = __fmul_rn(0.5f, x0 + x1);
            cover = (xmid >= px + 0.5f) ? y_len : 0.0f;
        } else {
            const float left = fmaxf(xl, px);
            const float right = fminf(xr, px + 1.0f);
            const float yf_left = __fmul_rn(__fdiv_rn(left - xl, dx), y_len);
            const float yf_right = __fmul_rn(__fdiv_rn(right - xl, dx), y_len);
            const float above = y_len - yf_right;
            cover = (yf_right - yf_left) + above;
        }
    }
    return __fmul_rn(sign, cover);
}

// Rust / PTX float -> int conversion: truncate, saturate, NaN -> 0.
__device__ __forceinline__ int32_t sat_i32(float v) {
    if (isnan(v)) return 0;
    if (v <= -2147483648.0f) return INT32_MIN;
    if (v >= 2147483648.0f) return INT32_MAX;
    return static_cast<int32_t>(v);
}

__global__ void __launch_bounds__(TF_THREADS) k_tile_fill(const TileRec* __restrict__ recs, uint64_t n_recs,
                                                          const uint32_t* __restrict__ starts,
                                                          const uint32_t* __restrict__ counts, uint32_t grid_w,
                                                          uint32_t grid_h, uint32_t width, uint32_t height, int eo,
                                                          uint8_t* __restrict__ coverage) {
    __shared__ TileRec srec[TF_THREADS];
    const uint32_t tid = threadIdx.x, pxl = tid % TILE, pyl = tid / TILE;
    const float px_f = static_cast<float>(pxl), py_f = static_cast<float>(pyl);
    const uint64_t n_tiles = static_cast<uint64_t>(grid_w) * grid_h;
    for (uint64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const uint32_t tx = static_cast<uint32_t>(tile % grid_w), ty = static_cast<uint32_t>(tile / grid_w);
        const uint64_t start = starts[tile];
        uint64_t cnt = counts[tile];
        if (start + cnt > n_recs) cnt = 0;
        float area = 0.0f;
        for (uint64_t base = 0; base < cnt; base += TF_THREADS) {
            const uint32_t m = cnt - base < TF_THREADS ? static_cast<uint32_t>(cnt - base) : TF_THREADS;
            __syncthreads();
            if (tid < m) srec[tid] = recs[start + base + tid];
            __syncthreads();
            for (uint32_t r = 0; r < m; ++r) {
                const TileRec rec = srec[r];
                const float iy0 = fmaxf(rec.y0_tile, py_f);
                const float iy1 = fminf(rec.y1_tile, py_f + 1.0f);
                if (iy0 >= iy1) continue;
                const float x_at_iy0 = __fadd_rn(rec.x_enter, __fmul_rn(rec.dxdy, iy0 - rec.y0_tile));
                area = __fadd_rn(area, segment_pixel_area(x_at_iy0, rec.dxdy, iy0, iy1, rec.sign, px_f));
            }
        }
        int32_t cov;
        if (eo) {
            float a = fabsf(area);
            a = a - floorf(a);
            if (a > 0.5f) a = 1.0f - a;
            cov = sat_i32(__fmul_rn(__fmul_rn(a, 2.0f), 255.5f));
        } else {
            cov = sat_i32(__fmul_rn(fminf(fabsf(area), 1.0f), 255.5f));
        }
        const uint32_t px = tx * TILE + pxl, py = ty * TILE + pyl;
        if (px < width && py < height) coverage[static_cast<size_t>(py) * width + px] = static_cast<uint8_t>(min(cov, 255));
    }
}

// ---- tile records on the device (build_tile_records, fill.rs:82-264) ----------
__device__ __forceinline__ uint32_t sat_u32(float v) {
    if (isnan(v) || v <= 0.0f) return 0;
    if (v >= 4294967296.0f) return UINT32_MAX;
    return static_cast<uint32_t>(v);
}

// Records of segment k in the reference's order (tile rows, then columns);
// with out == nullptr only counts them.
__device__ uint32_t segment_records(const float4 sg, float x_min, float y_min, uint32_t height, uint32_t grid_w,
                                    uint32_t grid_h, TileRec* out, uint32_t* keys) {
    float sx0 = sg.x - x_min, sy0 = sg.y - y_min, sx1 = sg.z - x_min, sy1 = sg.w - y_min;
    const float dy = fabsf(sy1 - sy0);
    if (!isfinite(dy) || dy < 1e-6f || !isfinite(sx0) || !isfinite(sx1)) return 0;
    float sign = 1.0f;
    if (sy0 > sy1) {
        float t = sx0;
        sx0 = sx1;
        sx1 = t;
        t = sy0;
        sy0 = sy1;
        sy1 = t;
        sign = -1.0f;
    }
    const float dxdy = __fdiv_rn(sx1 - sx0, sy1 - sy0);
    const float ey0 = fmaxf(sy0, 0.0f);
    const float ey1 = fminf(sy1, static_cast<float>(height));
    if (ey0 >= ey1) return 0;
    const float th = static_cast<float>(TILE), tw = static_cast<float>(TILE);
    const uint32_t ty0 = sat_u32(floorf(__fdiv_rn(ey0, th)));
    const uint32_t ty1 = sat_u32(floorf(__fdiv_rn(fmaxf(ey1 - 1e-6f, 0.0f), th)));
    const uint32_t ty_end = min(ty1, grid_h - 1);
    uint32_t n = 0;
    for (uint64_t ty = ty0; ty <= ty_end; ++ty) {
        const float tile_top = static_cast<float>(static_cast<uint32_t>(ty) * TILE);
        const float tile_bot = tile_top + th;
        const float seg_y0_tile = fmaxf(ey0, tile_top) - tile_top;
        const float seg_y1_tile = fminf(ey1, tile_bot) - tile_top;
        if (seg_y0_tile >= seg_y1_tile) continue;
        const float x_enter_global = fmaf(dxdy, fmaxf(ey0, tile_top) - sy0, sx0);
        const float x_at_exit = fmaf(dxdy, seg_y1_tile - seg_y0_tile, x_enter_global);
        const float xl = fminf(x_enter_global, x_at_exit), xr = fmaxf(x_enter_global, x_at_exit);
        const int32_t tx0_i = sat_i32(floorf(__fdiv_rn(xl, tw)));
        const int32_t tx1_i = sat_i32(floorf(__fdiv_rn(xr, tw)));
        if (tx1_i < 0) continue;
        const uint32_t tx0 = static_cast<uint32_t>(max(tx0_i, 0));
        const uint32_t tx1 = min(static_cast<uint32_t>(tx1_i), grid_w - 1);
        if (tx0 > tx1) continue;
        if (out) {
            for (uint32_t tx = tx0; tx <= tx1; ++tx) {
                TileRec r;
                r.key = (static_cast<uint32_t>(ty) << 16) | tx;
                r.x_enter = x_enter_global - static_cast<float>(tx * TILE);
                r.dxdy = dxdy;
                r.y0_tile = seg_y0_tile;
                r.y1_tile = seg_y1_tile;
                r.sign = sign;
                r.pad = r.pad2 = 0;
                out[n + (tx - tx0)] = r;
                keys[n + (tx - tx0)] = r.key;
            }
        }
        n += tx1 - tx0 + 1;
    }
    return n;
}

__global__ void k_tile_count(const float4* __restrict__ segs, uint32_t n_segs, uint32_t height, uint32_t grid_w,
                             uint32_t grid_h, unsigned long long* __restrict__ counts) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n_segs; k += gridDim.x * blockDim.x)
        counts[k] = segment_records(segs[k], 0.f, 0.f, height, grid_w, grid_h, nullptr, nullptr);
}

// Exclusive scan of n u64 counts in place (one CTA; the offsets of each
// segment's records in segment order); out[n] = total.
__global__ void __launch_bounds__(1024) k_scan_u64(unsigned long long* __restrict__ v, uint32_t n) {
    __shared__ unsigned long long part[1024];
    const uint32_t t = threadIdx.x, per = (n + 1023) / 1024;
    const uint32_t b = min(n, t * per), e = min(n, b + per);
    unsigned long long s = 0;
    for (uint32_t i = b; i < e; ++i) s += v[i];
    part[t] = s;
    __syncthreads();
    for (uint32_t o = 1; o < 1024; o <<= 1) {
        const unsigned long long x = t >= o ? part[t - o] : 0ull;
        __syncthreads();
        part[t] += x;
        __syncthreads();
    }
    unsigned long long run = part[t] - s;
    for (uint32_t i = b; i < e; ++i) {
        const unsigned long long c = v[i];
        v[i] = run;
        run += c;
    }
    if (t == 1023) v[n] = part[1023];
}

__global__ void k_tile_write(const float4* __restrict__ segs, uint32_t n_segs, uint32_t height, uint32_t grid_w,
                             uint32_t grid_h, const unsigned long long* __restrict__ off, TileRec* __restrict__ recs,
                             uint32_t* __restrict__ keys, uint32_t* __restrict__ idx) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n_segs; k += gridDim.x * blockDim.x) {
        const unsigned long long o = off[k];
        const uint32_t n = segment_records(segs[k], 0.f, 0.f, height, grid_w, grid_h, recs + o, keys + o);
        for (uint32_t i = 0; i < n; ++i) idx[o + i] = static_cast<uint32_t>(o + i);
    }
}

// Sorted records and, per tile, the range of its key in the sorted keys.
__global__ void k_tile_gather(const TileRec* __restrict__ recs, const uint32_t* __restrict__ order, uint32_t n,
                              TileRec* __restrict__ sorted) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        sorted[i] = recs[order[i]];
}

__global__ void k_tile_ranges(const uint32_t* __restrict__ keys, uint32_t n, uint32_t grid_w, uint32_t grid_h,
                              uint32_t* __restrict__ starts, uint32_t* __restrict__ counts) {
    const uint64_t n_tiles = static_cast<uint64_t>(grid_w) * grid_h;
    for (uint64_t t = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; t < n_tiles;
         t += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t key = (static_cast<uint32_t>(t / grid_w) << 16) | static_cast<uint32_t>(t % grid_w);
        auto lower = [&](uint32_t k) {
            uint32_t a = 0, z = n;
            while (a < z) {
                const uint32_t m = (a + z) >> 1;
                if (keys[m] < k) a = m + 1;
                else z = m;
            }
            return a;
        };
        const uint32_t s = lower(key);
        starts[t] = s;
        counts[t] = lower(key + 1) - s;
    }
}

#define FILL_CUDA(ctx, call)                                                                             \
    do {                                                                                                 \
        cudaError_t e__ = (call);                                                                        \
        if (e__ != cudaSuccess) {                                                                        \
            cudaGetLastError();                                                                          \
            return rrb_ctx_fail(ctx, RRB_ERR_DEVICE, (std::string(#call ": ") + cudaGetErrorString(e__)).c_str()); \
        }                                                                                                \
    } while (0)

// Checks shared by the coverage operators; `dev` is the status of the
// caller's DeviceScope (the context's device made current for the call).
int begin(rrb_ctx* c, cudaError_t dev) {
    if (!rrb_ctx_page_open(c)) return rrb_ctx_fail(c, RRB_ERR_STATE, "record_* outside begin_page/submit_page");
    FILL_CUDA(c, dev);
    return RRB_OK;
}

int check_cov(rrb_ctx* c, const rrb_buf* cov, uint32_t w, uint32_t h) {
    if (!cov) return rrb_ctx_fail(c, RRB_ERR_INVARIANT, "coverage buffer is null");
    if (static_cast<uint64_t>(w) * h > rrb_device_buffer_len(cov))
        return rrb_ctx_fail(c, RRB_ERR_INVARIANT, "coverage buffer is smaller than width * height");
    return RRB_OK;
}

int check_segs(rrb_ctx* c, const rrb_buf* segs, uint32_t n) {
    if (n && !segs) return rrb_ctx_fail(c, RRB_ERR_INVARIANT, "segs buffer is null");
    if (n && 16ull * n > rrb_device_buffer_len(segs))
        return rrb_ctx_fail(c, RRB_ERR_INVARIANT, "segs buffer is smaller than 16 * n_segs bytes");
    if (n && (reinterpret_cast<uintptr_t>(rrb_device_ptr(segs)) & 15))
        return rrb_ctx_fail(c, RRB_ERR_INVARIANT, "segs buffer is not 16-byte aligned");
    return RRB_OK;
}

int launch_tile_fill(rrb_ctx* c, const TileRec* recs, uint64_t n_recs, const uint32_t* starts,
                     const uint32_t* counts, uint32_t w, uint32_t h, int eo, uint8_t* cov) {
    const uint32_t gw = (w + TILE - 1) / TILE, gh = (h + TILE - 1) / TILE;
    const uint64_t tiles = static_cast<uint64_t>(gw) * gh;
    const int grid = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>(tiles, 8ull * rrb_ctx_sm_count(c))));
    cudaStream_t s = static_cast<cudaStream_t>(rrb_stream(c));
    k_tile_fill<<<grid, TF_THREADS, 0, s>>>(recs, n_recs, starts, counts, gw, gh, w, h, eo, cov);
    FILL_CUDA(c, cudaGetLastError());
    return RRB_OK;
}

// record_scan's phases (ScanPhase, crates/gpu/src/backend/params.rs:221-289).
// A block of SCAN_THREADS threads owns a tile of 2 * SCAN_THREADS u32; thread
// t holds elements 2t and 2t + 1. The exclusive scan of the pair sums is a
// warp shuffle scan, then a scan of the warp totals by warp 0; u32 sums wrap.
constexpr int SCAN_THREADS = static_cast<int>(RRB_SCAN_WORKGROUP_SIZE);
constexpr uint32_t SCAN_TILE = 2u * RRB_SCAN_WORKGROUP_SIZE;

// Exclusive scan of v over the block; *total receives the block's sum.
__device__ __forceinline__ uint32_t scan_block_excl(uint32_t v, uint32_t* warp_sums, uint32_t* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_sums[w] = incl;
    __syncthreads();
    if (w == 0) {
        constexpr int NW = SCAN_THREADS / 32;
        uint32_t x = lane < NW ? warp_sums[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += t;
        }
        if (lane < NW) warp_sums[lane] = x;  // inclusive over the warps
    }
    __syncthreads();
    *total = warp_sums[SCAN_THREADS / 32 - 1];
    return (w ? warp_sums[w - 1] : 0u) + incl - v;
}

// Phase 0 (and phase 1 with tile_sums == nullptr over the block sums): each
// block scans its tile of data[0, n) in place; tile_sums[block] = its total.
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tiles(uint32_t* __restrict__ data, uint32_t n,
                                                             uint32_t* __restrict__ tile_sums) {
    __shared__ uint32_t warp_sums[SCAN_THREADS / 32];
    const uint64_t i0 = static_cast<uint64_t>(blockIdx.x) * SCAN_TILE + 2u * threadIdx.x;
    const uint32_t a = i0 < n ? data[i0] : 0u, b = i0 + 1 < n ? data[i0 + 1] : 0u;
    uint32_t total;
    const uint32_t excl = scan_block_excl(a + b, warp_sums, &total);
    if (i0 < n) data[i0] = excl;
    if (i0 + 1 < n) data[i0 + 1] = excl + a;
    if (tile_sums && threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// Phase 2: block b adds the scanned tile_sums[b] to its tile.
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_scatter(uint32_t* __restrict__ data, uint32_t n,
                                                               const uint32_t* __restrict__ tile_sums) {
    const uint32_t add = tile_sums[blockIdx.x];
    const uint64_t i0 = static_cast<uint64_t>(blockIdx.x) * SCAN_TILE + threadIdx.x;
    if (i0 < n) data[i0] += add;
    if (i0 + SCAN_THREADS < n) data[i0 + SCAN_THREADS] += add;
}

}  // namespace

extern "C" {

int rrb_record_scan(rrb_ctx* c, const rrb_scan_params* p) {
    if (!c || !p) return RRB_ERR_INVARIANT;
    const rrb_host::DeviceScope dev_scope(rrb_ctx_device(c));
    int rc;
    if ((rc = begin(c, dev_scope.status()))) return rc;
    // ScanParams::validate (crates/gpu/src/backend/params.rs:338-372).
    if (p->len_elems == 0) return rrb_ctx_fail(c, RRB_ERR_INVARIANT, "len_elems must be > 0");
    if (!p->data || 4ull * p->len_elems > rrb_device_buffer_len(p->data))
        return rrb_ctx_fail(c, RRB_ERR_INVARIANT, "data buffer is smaller than len_elems * 4 bytes");
    const uint32_t blocks = (p->len_elems + SCAN_TILE - 1) / SCAN_TILE;
    if (blocks > RRB_SCAN_MAX_BLOCKS)
        return rrb_ctx_fail(c, RRB_ERR_INVARIANT, "block_count exceeds SCAN_MAX_BLOCKS (1024)");
    if (!p->block_sums || 4ull * blocks > rrb_device_buffer_len(p->block_sums))
        return rrb_ctx_fail(c, RRB_ERR_INVARIANT, "block_sums buffer is smaller than block_count * 4 bytes");
    if (p->phase > RRB_SCAN_SCATTER_BLOCK_SUMS) return rrb_ctx_fail(c, RRB_ERR_INVARIANT, "unknown scan phase");
    if (reinterpret_cast<uintptr_t>(rrb_device_ptr(p->data)) & 3 ||
        reinterpret_cast<uintptr_t>(rrb_device_ptr(p->block_sums)) & 3)
        return rrb_ctx_fail(c, RRB_ERR_INVARIANT, "scan buffers must be 4-byte aligned");
    cudaStream_t s = static_cast<cudaStream_t>(rrb_stream(c));
    uint32_t* data = static_cast<uint32_t*>(rrb_device_ptr(p->data));
    uint32_t* sums = static_cast<uint32_t*>(rrb_device_ptr(p->block_sums));
    if (p->phase == RRB_SCAN_PER_WORKGROUP) k_scan_tiles<<<blocks, SCAN_THREADS, 0, s>>>(data, p->len_elems, sums);
    else if (p->phase == RRB_SCAN_BLOCK_SUMS) k_scan_tiles<<<1, SCAN_THREADS, 0, s>>>(sums, blocks, nullptr);
    else k_scan_scatter<<<blocks, SCAN_THREADS, 0, s>>>(data, p->len_elems, sums);
    FILL_CUDA(c, cudaGetLastError());
    return RRB_OK;
}

void rrb_aa_fill_jitter(float* x, float* y) {
    if (x) std::memcpy(x, jitter().x, sizeof jitter().x);
    if (y) std::memcpy(y, jitter().y, sizeof jitter().y);
}

int rrb_record_aa_fill(rrb_ctx* c, const rrb_aa_fill_params* p) {
    if (!c || !p) return RRB_ERR_INVARIANT;
    const rrb_host::DeviceScope dev_scope(rrb_ctx_device(c));
    int rc;
    if ((rc = begin(c, dev_scope.status())) || (rc = check_cov(c, p->coverage, p->width, p->height)) ||
        (rc = check_segs(c, p->segs, p->n_segs)))
        return rc;
    if (!p->width || !p->height) return RRB_OK;
    cudaStream_t s = static_cast<cudaStream_t>(rrb_stream(c));
    uint8_t* cov = static_cast<uint8_t*>(rrb_device_ptr(p->coverage));
    if (!p->n_segs) {
        FILL_CUDA(c, cudaMemsetAsync(cov, 0, static_cast<size_t>(p->width) * p->height, s));
        return RRB_OK;
    }
    const uint64_t items = static_cast<uint64_t>((p->height + AA_WARPS - 1) / AA_WARPS) * ((p->width + AA_CW - 1) / AA_CW);
    const int grid = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>(items, 3ull * rrb_ctx_sm_count(c))));
    k_aa_fill<<<grid, AA_WARPS * 32, 0, s>>>(static_cast<const float4*>(rrb_device_ptr(p->segs)), p->n_segs, 0.f,
                                            0.f, p->width, p->height, p->fill_rule != 0, jitter(), cov);
    FILL_CUDA(c, cudaGetLastError());
    return RRB_OK;
}

int rrb_record_tile_fill(rrb_ctx* c, const rrb_tile_fill_params* p) {
    if (!c || !p) return RRB_ERR_INVARIANT;
    const rrb_host::DeviceScope dev_scope(rrb_ctx_device(c));
    int rc;
    if ((rc = begin(c, dev_scope.status())) || (rc = check_cov(c, p->coverage, p->width, p->height))) return rc;
    if (!p->width || !p->height) return RRB_OK;
    const uint32_t gw = (p->width + TILE - 1) / TILE, gh = (p->height + TILE - 1) / TILE;
    const uint64_t tiles = static_cast<uint64_t>(gw) * gh;
    if (!p->records || !p->tile_starts || !p->tile_counts)
        return rrb_ctx_fail(c, RRB_ERR_INVARIANT, "records / tile_starts / tile_counts buffer is null");
    if (rrb_device_buffer_len(p->tile_starts) < 4 * tiles || rrb_device_buffer_len(p->tile_counts) < 4 * tiles)
        return rrb_ctx_fail(c, RRB_ERR_INVARIANT, "tile_starts / tile_counts hold fewer than grid_w * grid_h entries");
    if (reinterpret_cast<uintptr_t>(rrb_device_ptr(p->records)) & 15)
        return rrb_ctx_fail(c, RRB_ERR_INVARIANT, "records buffer is not 16-byte aligned");
    return launch_tile_fill(c, static_cast<const TileRec*>(rrb_device_ptr(p->records)),
                            rrb_device_buffer_len(p->records) / sizeof(TileRec),
                            static_cast<const uint32_t*>(rrb_device_ptr(p->tile_starts)),
                            static_cast<const uint32_t*>(rrb_device_ptr(p->tile_counts)), p->width, p->height,
                            p->fill_rule != 0, static_cast<uint8_t*>(rrb_device_ptr(p->coverage)));
}

int rrb_record_tile_fill_segs(rrb_ctx* c, const rrb_aa_fill_params* p, uint64_t* n_records) {
    if (!c || !p) return RRB_ERR_INVARIANT;
    const rrb_host::DeviceScope dev_scope(rrb_ctx_device(c));
    int rc;
    if ((rc = begin(c, dev_scope.status())) || (rc = check_cov(c, p->coverage, p->width, p->height)) ||
        (rc = check_segs(c, p->segs, p->n_segs)))
        return rc;
    if (n_records) *n_records = 0;
    if (!p->width || !p->height) return RRB_OK;
    const uint32_t gw = (p->width + TILE - 1) / TILE, gh = (p->height + TILE - 1) / TILE;
    if (gw > 0xFFFF || gh > 0xFFFF) return rrb_ctx_fail(c, RRB_ERR_INVARIANT, "raster exceeds the 16-bit tile key range");
    const uint64_t tiles = static_cast<uint64_t>(gw) * gh;
    cudaStream_t s = static_cast<cudaStream_t>(rrb_stream(c));
    const int sm = rrb_ctx_sm_count(c);
    const uint32_t n = p->n_segs;
    const float4* segs = static_cast<const float4*>(rrb_device_ptr(p->segs));
    void *v_off, *v_rec, *v_key, *v_idx, *v_key2, *v_idx2, *v_sorted, *v_ranges;
    if ((rc = rrb_ctx_fill_scratch(c, 0, 8ull * (n + 1), &v_off))) return rc;
    auto* off = static_cast<unsigned long long*>(v_off);
    uint64_t total = 0;
    if (n) {
        const int g = static_cast<int>(std::max<uint32_t>(1, std::min<uint32_t>((n + 255) / 256, 8u * sm)));
        k_tile_count<<<g, 256, 0, s>>>(segs, n, p->height, gw, gh, off);
        k_scan_u64<<<1, 1024, 0, s>>>(off, n);
        FILL_CUDA(c, cudaGetLastError());
        FILL_CUDA(c, cudaMemcpyAsync(&total, off + n, 8, cudaMemcpyDeviceToHost, s));
        FILL_CUDA(c, cudaStreamSynchronize(s));
    }
    if (total >= (1ull << 31)) return rrb_ctx_fail(c, RRB_ERR_POOL_EXHAUSTED, "more than 2^31 tile records");
    const uint32_t nr = static_cast<uint32_t>(total);
    if (n_records) *n_records = nr;
    const size_t nr1 = std::max<uint32_t>(1, nr);
    if ((rc = rrb_ctx_fill_scratch(c, 1, nr1 * sizeof(TileRec), &v_rec)) ||
        (rc = rrb_ctx_fill_scratch(c, 2, nr1 * 4, &v_key)) || (rc = rrb_ctx_fill_scratch(c, 3, nr1 * 4, &v_idx)) ||
        (rc = rrb_ctx_fill_scratch(c, 4, nr1 * 4, &v_key2)) || (rc = rrb_ctx_fill_scratch(c, 5, nr1 * 4, &v_idx2)) ||
        (rc = rrb_ctx_fill_scratch(c, 6, nr1 * sizeof(TileRec), &v_sorted)) ||
        (rc = rrb_ctx_fill_scratch(c, 7, 8 * tiles, &v_ranges)))
        return rc;
    auto* starts = static_cast<uint32_t*>(v_ranges);
    auto* counts = starts + tiles;
    if (nr) {
        const int g = static_cast<int>(std::max<uint32_t>(1, std::min<uint32_t>((n + 255) / 256, 8u * sm)));
        k_tile_write<<<g, 256, 0, s>>>(segs, n, p->height, gw, gh, off, static_cast<TileRec*>(v_rec),
                                       static_cast<uint32_t*>(v_key), static_cast<uint32_t*>(v_idx));
        size_t temp = 0;
        FILL_CUDA(c, cub::DeviceRadixSort::SortPairs(nullptr, temp, static_cast<uint32_t*>(v_key),
                                                     static_cast<uint32_t*>(v_key2), static_cast<uint32_t*>(v_idx),
                                                     static_cast<uint32_t*>(v_idx2), static_cast<int>(nr), 0, 32, s));
        // The sort's temporary storage reuses the offsets slot (no longer needed).
        if ((rc = rrb_ctx_fill_scratch(c, 0, std::max<size_t>(temp, 8ull * (n + 1)), &v_off))) return rc;
        FILL_CUDA(c, cub::DeviceRadixSort::SortPairs(v_off, temp, static_cast<uint32_t*>(v_key),
                                                     static_cast<uint32_t*>(v_key2), static_cast<uint32_t*>(v_idx),
                                                     static_cast<uint32_t*>(v_idx2), static_cast<int>(nr), 0, 32, s));
        const int g2 = static_cast<int>(std::max<uint32_t>(1, std::min<uint32_t>((nr + 255) / 256, 8u * sm)));
        k_tile_gather<<<g2, 256, 0, s>>>(static_cast<const TileRec*>(v_rec), static_cast<const uint32_t*>(v_idx2), nr,
                                         static_cast<TileRec*>(v_sorted));
    }
    const int g3 = static_cast<int>(std::max<uint64_t>(1, std::min<uint64_t>((tiles + 255) / 256, 8ull * sm)));
    k_tile_ranges<<<g3, 256, 0, s>>>(static_cast<const uint32_t*>(v_key2), nr, gw, gh, starts, counts);
    FILL_CUDA(c, cudaGetLastError());
    return launch_tile_fill(c, static_cast<const TileRec*>(v_sorted), nr, starts, counts, p->width, p->height,
                            p->fill_rule != 0, static_cast<uint8_t*>(rrb_device_ptr(p->coverage)));
}

}  // extern "C"
