// rrb_backend.cu — the C ABI (include/rrb.h): context, device memory,
// transfers, the per-page state machine of GpuBackend
// (crates/gpu/src/backend/mod.rs:216-503) and the path-fill batch driver.
//
// One rrb_ctx = one device + one non-blocking stream, as GpuCtx serialises
// every call on one stream (crates/gpu/src/lib.rs:197-208). Scratch buffers
// for a batch are owned by the context and grow on demand, so repeated
// batches of similar size allocate nothing.

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/rrb.h"
#include "rrb_device_scope.h"
#include "rrb_hairline.cuh"
#include "rrb_kernels.cuh"
#include "rrb_stroke.h"

using namespace rrb;

struct rrb_buf {
    void* p = nullptr;
    size_t len = 0;
};
struct rrb_host_buf {
    void* p = nullptr;
    size_t len = 0;
};

namespace {

struct Scratch {
    void* p = nullptr;
    size_t cap = 0;
};

constexpr int KCAP = 12;        // merged Intersect entries per AA row kept in shared memory
constexpr int KCAP_WIDE = 16;   // the same for the 4-warp row-stage shapes
// Row-stage shapes (rrb_batch::row_shape): entries per AA row kept in shared
// memory x warps per block x 32-edge groups a warp stages at once; a block
// stages warps x groups x 32 edges (512, 256, 256, 1024, 128).
constexpr int kRowShapes = 5;
constexpr uint64_t kLaneCountCurves = 1ull << 22;  // big curves whose lane counts are kept (128 MiB)
constexpr int SUPER = 256;      // supertile edge in pixels (a multiple of every tile shape)

}  // namespace

struct rrb_ctx {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    uint64_t budget = 0;
    uint64_t used = 0;
    std::string err;
    bool in_page = false;
    rrb_tuning tuning{};
    rrb_batch_stats stats{};
    uint64_t next_fence = 1;
    std::unordered_map<uint64_t, cudaEvent_t> fences;
    std::vector<cudaEvent_t> free_events;
    // Batch scratch.
    Scratch s_pts, s_flags, s_off, s_rule, s_gray, s_alpha, s_page, s_geom, s_pw, s_ph, s_mtx;
    Scratch s_pieces, s_clip, s_edge_off, s_edges, s_info, s_rows, s_chunks, s_super_cnt, s_super_list;
    Scratch s_super_start;  // per supertile: one past its last opaque full layer
    Scratch s_big;          // piece slots of curves flattened by a warp each
    Scratch s_lanes;        // per big curve: each lane's segment count (u8 x 32), from the count pass
    Scratch s_row_idx, s_spans, s_ovf, s_scratch, s_ctr, s_block, s_stats, s_groups, s_slots, s_path_pieces, s_ovf2;
    Scratch s_run_off, s_runs, s_chunk_path, s_clip_lo, s_hl_clip;
    Scratch s_fill[8];           // scratch of the aa_fill / tile_fill operators (rrb_fills.cu)
    uint32_t* h_read = nullptr;  // pinned readback area
    uint64_t launches = 0;
    uint64_t host_syncs = 0;  // stream waits for device-side sizes in the current run_resident_one
    // Replays with cached sizes: each wave's counters are copied here (page-
    // locked, one slot per wave) and read after the render's one wait.
    rrb::BatchCounters* h_waves = nullptr;
    uint32_t h_waves_cap = 0;
    bool deferred = false;  // the last run_resident_one left its counters in h_waves
    // Page-locked staging of the page geometry of a render's waves (wave i at
    // its first page): a copy from pageable memory would wait on the stream.
    rrb::PageGeom* h_geom = nullptr;
    uint32_t h_geom_cap = 0;
    uint32_t geom_slot = 0;  // where the next run_resident_one stages its geometry
    // Set while the pages are still on their way up (rrb_render_pages_host):
    // the next composite waits for this event first.
    cudaEvent_t pages_up = nullptr;
    bool wait_pages_up = false;
    uint64_t scratch_grows = 0;  // ensure() reallocations since the last record call began
    struct rrb_batch* tmp_batch = nullptr;  // inputs of rrb_record_path_batch
    struct rrb_batch* wave_batch = nullptr; // view of a group of pages of a larger batch
    struct StageTimer* timer = nullptr;
    float stage_ms[16] = {};
    uint32_t stage_launches[16] = {};
    // Per-stage sums over the waves of one resident render.
    float stage_sum_ms[16] = {};
    uint32_t stage_sum_launches[16] = {};
    rrb_stroke::PaintBatch* paint = nullptr;  // host arrays of rrb_record_stroke_batch, reused
    cudaStream_t copy_stream = nullptr;       // streamed batches: point uploads ahead of the render
    cudaStream_t down_stream = nullptr;       // host page renders: page downloads beside the uploads
    uint64_t tuning_epoch = 0;                // bumped by rrb_set_tuning: resident batches re-run their trials
    // With automatic tiles: the tile shape the last resident batch settled on
    // by its trials (0: none yet, 64x16), the default of batches uploaded per
    // call on this context until another batch settles or the tuning changes.
    uint32_t settled_tw = 0, settled_th = 0;
    cudaEvent_t trial_ev[2] = {nullptr, nullptr};  // timing of a resident batch's trial render
};

namespace {

int set_err(rrb_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

int cuda_err(rrb_ctx* c, cudaError_t e, const char* what) {
    return set_err(c, RRB_ERR_DEVICE, std::string(what) + ": " + cudaGetErrorString(e));
}

#define RRB_CUDA(ctx, call)                                   \
    do {                                                      \
        cudaError_t e__ = (call);                             \
        if (e__ != cudaSuccess) return cuda_err(ctx, e__, #call); \
    } while (0)

int dev_alloc(rrb_ctx* c, size_t bytes, void** out) {
    if (c->budget && c->used + bytes > c->budget)
        return set_err(c, RRB_ERR_OUT_OF_MEMORY,
                       "device allocation of " + std::to_string(bytes) + " bytes exceeds the budget");
    cudaError_t e = cudaMalloc(out, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_err(c, RRB_ERR_OUT_OF_MEMORY, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    c->used += bytes;
    return RRB_OK;
}

void dev_free(rrb_ctx* c, void* p, size_t bytes) {
    if (!p) return;
    cudaFree(p);
    c->used -= std::min<uint64_t>(c->used, bytes);
}

// Grow a scratch buffer to at least `bytes` (x1.25 headroom); contents are not kept.
int ensure(rrb_ctx* c, Scratch& s, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (s.cap >= bytes) return RRB_OK;
    if (s.p) {
        cudaError_t e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) return cuda_err(c, e, "cudaStreamSynchronize");
        dev_free(c, s.p, s.cap);
        s.p = nullptr;
        s.cap = 0;
    }
    size_t want = bytes + bytes / 4;
    want = (want + 255) & ~size_t(255);
    int rc = dev_alloc(c, want, &s.p);
    if (rc) return rc;
    s.cap = want;
    c->scratch_grows += 1;
    return RRB_OK;
}

template <typename T>
T* as(Scratch& s) {
    return static_cast<T*>(s.p);
}

int grid_for(rrb_ctx* c, uint64_t n, int threads, int per_sm = 8) {
    uint64_t need = (n + threads - 1) / threads;
    uint64_t cap = static_cast<uint64_t>(c->sm_count) * per_sm;
    return static_cast<int>(std::max<uint64_t>(1, std::min(need, cap)));
}

// Exclusive scan of n u32 at d_in into d_out[0..n] (d_out[n] = total).
int scan_u32(rrb_ctx* c, const uint32_t* d_in, uint32_t* d_out, uint32_t n) {
    uint32_t* bs = as<uint32_t>(c->s_block);
    if (n == 0) {
        RRB_CUDA(c, cudaMemsetAsync(d_out, 0, sizeof(uint32_t), c->stream));
        return RRB_OK;
    }
    uint32_t nb = std::min<uint32_t>(SCAN_MAX_BLOCKS, std::max<uint32_t>(1, (n + 4095) / 4096));
    uint32_t per = (n + nb - 1) / nb;
    nb = (n + per - 1) / per;
    k_scan_reduce<<<nb, SCAN_THREADS, 0, c->stream>>>(d_in, n, per, bs);
    k_scan_blocks<<<1, 1024, 0, c->stream>>>(bs, nb);
    k_scan_down<<<nb, SCAN_THREADS, 0, c->stream>>>(d_in, d_out, n, per, bs);
    c->launches += 3;
    RRB_CUDA(c, cudaGetLastError());
    return RRB_OK;
}

template <typename T>
int upload(rrb_ctx* c, Scratch& s, const T* src, size_t count) {
    int rc = ensure(c, s, count * sizeof(T));
    if (rc) return rc;
    if (count) RRB_CUDA(c, cudaMemcpyAsync(s.p, src, count * sizeof(T), cudaMemcpyHostToDevice, c->stream));
    return RRB_OK;
}

int read_back(rrb_ctx* c, const void* dev, size_t bytes) {
    ++c->host_syncs;
    RRB_CUDA(c, cudaMemcpyAsync(c->h_read, dev, bytes, cudaMemcpyDeviceToHost, c->stream));
    RRB_CUDA(c, cudaStreamSynchronize(c->stream));
    return RRB_OK;
}

bool valid_tile(uint32_t w, uint32_t h) {
    return (w == 16 && h == 16) || (w == 32 && h == 32) || (w == 64 && h == 16) || (w == 128 && h == 16) ||
           (w == 128 && h == 32);
}

// The kernels a resident batch's trials choose between, loaded when the
// context is made: with CUDA's lazy module loading the first launch of a
// kernel also loads it, and that time would land inside the first trial
// render that uses it, making that tile or row shape look slower.
void preload_trial_kernels() {
    cudaFuncAttributes a{};
#define RRB_PRELOAD(...) cudaFuncGetAttributes(&a, reinterpret_cast<const void*>(__VA_ARGS__))
#define RRB_PRELOAD_COMP(TW, TH)                      \
    do {                                              \
        RRB_PRELOAD(k_composite<TW, TH, false, false>); \
        RRB_PRELOAD(k_composite<TW, TH, false, true>);  \
        RRB_PRELOAD(k_composite<TW, TH, true, false>);  \
        RRB_PRELOAD(k_composite<TW, TH, true, true>);   \
    } while (0)
    RRB_PRELOAD_COMP(16, 16);
    RRB_PRELOAD_COMP(32, 32);
    RRB_PRELOAD_COMP(64, 16);
    RRB_PRELOAD_COMP(128, 16);
    RRB_PRELOAD_COMP(128, 32);
    RRB_PRELOAD(k_rows<KCAP, ROWS_WARPS>);
    RRB_PRELOAD(k_rows<KCAP_WIDE, 4>);
    RRB_PRELOAD(k_rows<KCAP, ROWS_WARPS, 1>);
    RRB_PRELOAD(k_rows<8, 16>);
    RRB_PRELOAD(k_rows<KCAP_WIDE, 4, 1>);
#undef RRB_PRELOAD_COMP
#undef RRB_PRELOAD
    cudaGetLastError();
}

int launch_composite(rrb_ctx* c, int tw, int th, int grid, const PathInfo* info, const PageGeom* geom,
                     uint32_t n_pages, uint32_t n_tiles, const uint32_t* super_off, const uint32_t* super_list,
                     const uint32_t* row_off, const uint2* row_idx, const uint32_t* spans, const int4* runs,
                     uint8_t* arena, int rowmap, BatchCounters* ctr, const uint32_t* path_rgb,
                     bool rectilinear, const uint32_t* super_start) {
#define RRB_COMP(TW, TH, RGB, FEW)                                                                           \
    k_composite<TW, TH, RGB, FEW><<<grid, comp_threads(TW, TH), 0, c->stream>>>(                              \
        info, geom, n_pages, n_tiles, SUPER, SUPER, super_off, super_list, row_off, row_idx, spans, runs, arena, \
        rowmap, ctr, path_rgb, super_start)
#define RRB_COMP_SHAPE(RGB, FEW)                                  \
    do {                                                          \
        if (tw == 64 && th == 16) RRB_COMP(64, 16, RGB, FEW);     \
        else if (tw == 128 && th == 16) RRB_COMP(128, 16, RGB, FEW); \
        else if (tw == 128 && th == 32) RRB_COMP(128, 32, RGB, FEW); \
        else if (tw == 32 && th == 32) RRB_COMP(32, 32, RGB, FEW); \
        else RRB_COMP(16, 16, RGB, FEW);                          \
    } while (0)
    // Batches with rectilinear paths (rectangles) use the variant with the
    // direct cell lookup for their rows; others keep the plain kernel, whose
    // register allocation the extra path would disturb.
    if (path_rgb) {
        if (rectilinear) RRB_COMP_SHAPE(true, true);
        else RRB_COMP_SHAPE(true, false);
    } else {
        if (rectilinear) RRB_COMP_SHAPE(false, true);
        else RRB_COMP_SHAPE(false, false);
    }
#undef RRB_COMP_SHAPE
#undef RRB_COMP
    c->launches += 1;
    RRB_CUDA(c, cudaGetLastError());
    return RRB_OK;
}

// Host-side checks of a batch (the params.validate() of the reference,
// crates/gpu/src/backend/params.rs:57,334), plus the page geometry the
// kernels need. No device access.
int validate_batch(const rrb_path_batch_params* h, size_t arena_len, uint32_t tw, uint32_t th,
                   std::vector<PageGeom>& geom, uint64_t& tiles, uint64_t& supers, std::string& msg, uint32_t bpp = 1,
                   uint8_t max_rule = 1) {
    const uint64_t n_paths = h->n_paths, n_pts = h->n_pts;
    const uint32_t n_pages = h->n_pages;
    tiles = supers = 0;
    if (h->rowmap > 1) return msg = "rowmap must be 0 or 1", RRB_ERR_INVARIANT;
    if (!(h->flatness >= 0.0)) return msg = "flatness must be >= 0", RRB_ERR_INVARIANT;
    for (int i = 0; i < 6; ++i)
        if (!std::isfinite(h->matrix[i])) return msg = "matrix must be finite", RRB_ERR_INVARIANT;
    if (!valid_tile(tw, th)) return msg = "tile shape must be 16x16, 32x32, 64x16, 128x16 or 128x32", RRB_ERR_INVARIANT;
    if (n_paths == 0) return RRB_OK;
    if (!h->pts || !h->flags || !h->path_pt_off || !h->fill_rule || !h->gray || !h->alpha || !h->path_page ||
        !h->page_width || !h->page_height || !h->page_offset || !n_pages)
        return msg = "null array in path batch", RRB_ERR_INVARIANT;
    if (n_pts >= (1ull << 30) || n_paths >= (1ull << 31))
        return msg = "batch exceeds 2^30 points or 2^31 paths", RRB_ERR_INVARIANT;
    if (h->path_pt_off[0] != 0 || h->path_pt_off[n_paths] != n_pts)
        return msg = "path_pt_off must start at 0 and end at n_pts", RRB_ERR_INVARIANT;
    for (uint64_t p = 0; p < n_paths; ++p)
        if (h->path_pt_off[p + 1] < h->path_pt_off[p]) return msg = "path_pt_off must be non-decreasing", RRB_ERR_INVARIANT;
    geom.assign(n_pages, PageGeom{});
    for (uint32_t pg = 0; pg < n_pages; ++pg) {
        uint32_t w = h->page_width[pg], ht = h->page_height[pg];
        if (w == 0 || ht == 0 || w > 16383 || ht > (1u << 28))
            return msg = "page width must be 1..16383 and height 1..2^28", RRB_ERR_INVARIANT;
        // Overflow-safe form of offset + bytes > arena_len (an offset near 2^64 must not wrap).
        const uint64_t page_bytes = static_cast<uint64_t>(bpp) * w * ht;
        if (h->page_offset[pg] > arena_len || page_bytes > arena_len - h->page_offset[pg])
            return msg = "page extends past the page buffer", RRB_ERR_INVARIANT;
        PageGeom& G = geom[pg];
        G.w = w;
        G.h = ht;
        G.offset = h->page_offset[pg];
        G.ntx = (w + tw - 1) / tw;
        G.nsx = (w + SUPER - 1) / SUPER;
        G.tile_base = static_cast<uint32_t>(tiles);
        G.super_base = static_cast<uint32_t>(supers);
        tiles += static_cast<uint64_t>(G.ntx) * ((ht + th - 1) / th);
        supers += static_cast<uint64_t>(G.nsx) * ((ht + SUPER - 1) / SUPER);
    }
    uint32_t prev = 0;
    for (uint64_t p = 0; p < n_paths; ++p) {
        uint32_t pg = h->path_page[p];
        if (pg >= n_pages || pg < prev)
            return msg = "path_page must be < n_pages and non-decreasing", RRB_ERR_INVARIANT;
        if (h->fill_rule[p] > max_rule) return msg = "fill_rule must be 0 or 1", RRB_ERR_INVARIANT;
        prev = pg;
    }
    uint64_t p = 0, work = 0;
    for (uint32_t pg = 0; pg < n_pages; ++pg) {
        PageGeom& G = geom[pg];
        G.path_begin = static_cast<uint32_t>(p);
        while (p < n_paths && h->path_page[p] == pg) ++p;
        G.path_end = static_cast<uint32_t>(p);
        G.nblk = std::max<uint32_t>(1, (G.path_end - G.path_begin + BIN_BLOCK - 1) / BIN_BLOCK);
        G.work_base = static_cast<uint32_t>(work);
        work += static_cast<uint64_t>(G.nsx) * ((G.h + SUPER - 1) / SUPER) * G.nblk;
    }
    if (tiles >= (1ull << 31) || supers >= (1ull << 31) || work >= (1ull << 31))
        return msg = "too many tiles", RRB_ERR_INVARIANT;
    supers = work;  // binning work items
    return RRB_OK;
}

// Recompute per-tile geometry for tile shape (tw, th).
void set_tiles(std::vector<PageGeom>& geom, uint32_t tw, uint32_t th, uint64_t& tiles) {
    tiles = 0;
    for (PageGeom& G : geom) {
        G.ntx = (G.w + tw - 1) / tw;
        G.tile_base = static_cast<uint32_t>(tiles);
        tiles += static_cast<uint64_t>(G.ntx) * ((G.h + th - 1) / th);
    }
}

}  // namespace

// The sizes one render of a wave found on the device between its stages. A
// resident batch renders the same inputs every time, so a later render of
// the same wave with the same tile shape, row-stage shape and row map finds
// the same sizes: it takes them from here and launches every stage without
// waiting on the stream.
struct WaveSizes {
    bool valid = false;
    uint32_t tw = 0, th = 0;
    uint8_t row_shape = 0;
    int rowmap = -1;
    uint64_t n_pieces = 0, n_edges = 0, n_groups = 0, n_chunks = 0, n_pairs = 0, n_runs = 0;
    uint64_t raw_entries = 0, hl_rows = 0, mid = 0, slow = 0, slow_need = 0;
    bool matches(uint32_t w, uint32_t h, uint8_t rs, int rm) const {
        return valid && tw == w && th == h && row_shape == rs && rowmap == rm;
    }
};

// A batch whose inputs live in device memory: uploaded once, rendered any
// number of times (the serving loop keeps these resident).
struct rrb_batch {
    Scratch pts, flags, off, rule, gray, alpha, page, geom, pw, ph, mtx;
    Scratch rgb;                    // Rgb8 pages: per-path colour r | g << 8 | b << 16
    uint32_t bpp = 1;               // page bytes per pixel: 1 Gray8, 3 Rgb8
    Scratch clip;                   // per-path clip in AA units (int4), when has_clip
    Scratch clipf;                  // the clip rectangles as given (4 doubles per path), when has_clip
    bool has_clip = false;
    Scratch visit;                  // per-path visited pixel rows (int2) under the shipped row map, when has_visit
    bool has_visit = false;
    bool has_hairline = false;      // some paths are hairline segments (RULE_HAIRLINE)
    // Page groups [plan[i], plan[i+1]) that rendered without running out of
    // scratch or cell capacity last time (with plan_wave_points); reused so a
    // resident batch does not fail and split on every render.
    std::vector<uint32_t> plan;
    uint64_t plan_wave_points = 0;
    // Per wave of `plan`: the sizes its last render found on the device.
    std::vector<WaveSizes> sizes;
    // Row-stage shape (kRowShapes of them, 0 the default) and tile shape (0 x 0:
    // the context's) of the next render. A resident batch renders once per
    // trial, timed by events on its stream (a trial whose render grew scratch
    // is repeated): first each candidate tile shape with row shape 0 (with
    // automatic tiles 64x16, 128x16 and 128x32; else the context's), then the
    // other row shapes with the fastest tile; it keeps the fastest pair.
    uint8_t row_shape = 0;
    uint32_t tile_w = 0, tile_h = 0;
    struct Trial {
        uint32_t tw, th;
        uint8_t rs;
        float ms;
    };
    std::vector<Trial> trials;  // empty: not planned yet
    bool row_trials_planned = false;  // the second phase (row shapes) is in trials
    size_t trial = 0;           // next trial to run (trials.size(): settled)
    uint64_t trial_epoch = ~0ull;
    std::vector<PageGeom> geom_h;
    std::vector<uint64_t> page_pt;  // first point of each page's paths (n_pages + 1)
    bool view = false;              // a wave: inputs point into another batch (only off/page/geom owned)
    uint64_t supers = 0, arena_need = 0;
    uint64_t n_paths = 0, n_pts = 0;
    uint32_t n_pages = 0;
    double flat_sq = 0.0;
    uint8_t rowmap = 0;
};

namespace {

// Stage names for the optional per-stage event timing.
const char* const kStageNames[] = {"walk",   "seg_count",   "scan_edges", "seg_write", "path_bbox",
                                   "scan_rows_chunks", "super_count", "scan_super", "super_write", "rows",
                                   "rows_slow", "composite"};
constexpr int kStages = sizeof(kStageNames) / sizeof(kStageNames[0]);

}  // namespace

// Events of up to kTimedWaves waves of one render: a render whose waves do
// not wait on the stream (a replay with cached sizes) reads them all after
// its one synchronisation.
constexpr int kTimedWaves = 64;
struct StageTimer {
    bool on = false;
    int slot = 0;  // the wave whose events are being recorded
    cudaEvent_t begin[kTimedWaves][kStages] = {}, end[kTimedWaves][kStages] = {};
    bool used[kTimedWaves][kStages] = {};
    uint32_t launches[kTimedWaves][kStages] = {};
    uint64_t launch_mark = 0;
};

namespace {

// Per-stage CUDA events on the launching stream (profiling mode only).
void stage(rrb_ctx* c, int k) {
    StageTimer* t = c->timer;
    if (!t || !t->on || k >= kStages) return;
    cudaEventRecord(t->begin[t->slot][k], c->stream);
    t->used[t->slot][k] = true;
    t->launch_mark = c->launches;
}

void stage_end(rrb_ctx* c, int k) {
    StageTimer* t = c->timer;
    if (!t || !t->on || k >= kStages) return;
    cudaEventRecord(t->end[t->slot][k], c->stream);
    t->launches[t->slot][k] = static_cast<uint32_t>(c->launches - t->launch_mark);
}

void free_batch_bufs(rrb_ctx* c, rrb_batch* B) {
    Scratch* all[] = {&B->pts, &B->flags, &B->off, &B->rule, &B->gray, &B->alpha, &B->page, &B->geom, &B->pw, &B->ph,
                      &B->mtx, &B->rgb, &B->clip, &B->clipf, &B->visit};
    for (Scratch* s : all) {
        if (B->view && s != &B->off && s != &B->page && s != &B->geom) {
            s->p = nullptr;
            s->cap = 0;
            continue;
        }
        dev_free(c, s->p, s->cap);
        s->p = nullptr;
        s->cap = 0;
    }
}

// Upload a batch's inputs. rgb (host, 3 bytes per path) selects Rgb8 pages;
// clip (host, 4 doubles per path) clips each path to a device-space rectangle.
int batch_upload(rrb_ctx* c, const rrb_path_batch_params* h, rrb_batch* B, const uint8_t* rgb = nullptr,
                 const double* clip = nullptr, bool hairlines = false, bool defer_points = false,
                 const int32_t* visit = nullptr) {
    std::string msg;
    uint64_t tiles = 0;
    B->bpp = rgb ? 3 : 1;
    int v = validate_batch(h, SIZE_MAX, 64, 16, B->geom_h, tiles, B->supers, msg, B->bpp,
                           hairlines ? RULE_HAIRLINE : 1);
    if (v) return set_err(c, v, msg);
    B->sizes.clear();  // new inputs: no render has seen their sizes
    B->n_paths = h->n_paths;
    B->n_pts = h->n_pts;
    B->n_pages = h->n_pages;
    B->flat_sq = h->flatness * h->flatness;
    B->rowmap = h->rowmap;
    B->arena_need = 0;
    for (const PageGeom& G : B->geom_h)
        B->arena_need = std::max<uint64_t>(B->arena_need, G.offset + static_cast<uint64_t>(B->bpp) * G.w * G.h);
    B->plan.clear();
    B->row_shape = 0;
    B->tile_w = B->tile_h = 0;
    B->trials.clear();
    B->trial = 0;
    B->trial_epoch = ~0ull;
    B->row_trials_planned = false;
    B->has_hairline = false;
    if (hairlines)
        for (uint64_t p = 0; p < h->n_paths && !B->has_hairline; ++p) B->has_hairline = h->fill_rule[p] == RULE_HAIRLINE;
    B->page_pt.assign(B->n_pages + 1, 0);
    for (uint32_t pg = 0; pg < B->n_pages; ++pg) B->page_pt[pg] = h->path_pt_off[B->geom_h[pg].path_begin];
    B->page_pt[B->n_pages] = h->n_paths ? h->path_pt_off[h->n_paths] : 0;
    if (B->n_paths == 0) return RRB_OK;
    int rc;
    if (defer_points) {
        // The caller copies the points itself, range by range (run_streamed).
        if ((rc = ensure(c, B->pts, 2 * h->n_pts * sizeof(double)))) return rc;
        if ((rc = ensure(c, B->flags, h->n_pts))) return rc;
    } else {
        if ((rc = upload(c, B->pts, h->pts, 2 * h->n_pts))) return rc;
        if ((rc = upload(c, B->flags, h->flags, h->n_pts))) return rc;
    }
    if ((rc = upload(c, B->off, h->path_pt_off, h->n_paths + 1))) return rc;
    if ((rc = upload(c, B->rule, h->fill_rule, h->n_paths))) return rc;
    if ((rc = upload(c, B->gray, h->gray, h->n_paths))) return rc;
    if ((rc = upload(c, B->alpha, h->alpha, h->n_paths))) return rc;
    if ((rc = upload(c, B->page, h->path_page, h->n_paths))) return rc;
    if ((rc = upload(c, B->pw, h->page_width, h->n_pages))) return rc;
    if ((rc = upload(c, B->ph, h->page_height, h->n_pages))) return rc;
    if ((rc = ensure(c, B->geom, h->n_pages * sizeof(PageGeom)))) return rc;
    if ((rc = upload(c, B->mtx, h->matrix, 6))) return rc;
    B->has_clip = clip != nullptr;
    if (clip) {
        // Clip::new(0, 0, W, H) then clip_to_rect (clip.rs:73-88,116-125,266-271),
        // in AA units: columns [4 x_min_i, 4 (x_max_i + 1)), rows [4 y_min_i, 4 (y_max_i + 1) - 1].
        std::vector<int4> ci(h->n_paths);
        for (uint64_t p = 0; p < h->n_paths; ++p) {
            const double* r = clip + 4 * p;
            for (int k = 0; k < 4; ++k)
                if (!std::isfinite(r[k])) return set_err(c, RRB_ERR_INVARIANT, "clip rectangles must be finite");
            const uint32_t pg = h->path_page[p];
            const double W = h->page_width[pg], H = h->page_height[pg];
            const double x_min = std::max(0.0, std::min(r[0], r[2])), x_max = std::min(W, std::max(r[0], r[2]));
            const double y_min = std::max(0.0, std::min(r[1], r[3])), y_max = std::min(H, std::max(r[1], r[3]));
            auto fl = [](double v) { return static_cast<int32_t>(std::max(-1e9, std::min(1e9, std::floor(v)))); };
            auto ce = [](double v) { return static_cast<int32_t>(std::max(-1e9, std::min(1e9, std::ceil(v)))); };
            const int32_t x_min_i = fl(x_min), y_min_i = fl(y_min), x_max_i = ce(x_max) - 1, y_max_i = ce(y_max) - 1;
            ci[p] = make_int4(4 * x_min_i, 4 * (x_max_i + 1), 4 * y_min_i, 4 * (y_max_i + 1) - 1);
            if (ci[p].x > ci[p].y) ci[p].y = ci[p].x;      // empty column range
            if (ci[p].z > ci[p].w + 1) ci[p].w = ci[p].z - 1;  // empty row range
        }
        if ((rc = upload(c, B->clip, ci.data(), ci.size()))) return rc;
        if ((rc = upload(c, B->clipf, clip, 4 * h->n_paths))) return rc;
        RRB_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    B->has_visit = visit != nullptr && h->rowmap == RRB_ROWMAP_AS_SHIPPED;
    if (B->has_visit) {
        if ((rc = upload(c, B->visit, reinterpret_cast<const int2*>(visit), h->n_paths))) return rc;
        RRB_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    if (rgb) {
        std::vector<uint32_t> packed(h->n_paths);
        for (uint64_t p = 0; p < h->n_paths; ++p)
            packed[p] = rgb[3 * p] | (uint32_t(rgb[3 * p + 1]) << 8) | (uint32_t(rgb[3 * p + 2]) << 16);
        if ((rc = upload(c, B->rgb, packed.data(), packed.size()))) return rc;
        // The staging vector is released on return: let the copy finish first.
        RRB_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    return RRB_OK;
}

// The pipeline over a device-resident batch into the device page arena.
// ws: the wave's cached sizes (see WaveSizes), or nullptr. When they match,
// every stage is launched without waiting on the stream, and the counters
// are copied into the page-locked slot c->h_waves[slot] for the caller to
// read after its one wait (c->deferred is set); otherwise the sizes are read
// back between the stages and, if ws is given, stored there.
int run_resident_one(rrb_ctx* c, rrb_batch* B, uint8_t* arena, size_t arena_len, int rowmap,
                     WaveSizes* ws = nullptr, uint32_t slot = 0) {
    c->launches = 0;
    c->host_syncs = 0;
    c->deferred = false;
    std::memset(&c->stats, 0, sizeof c->stats);
    std::memset(c->stage_ms, 0, sizeof c->stage_ms);
    std::memset(c->stage_launches, 0, sizeof c->stage_launches);
    if (c->timer) std::memset(c->timer->used[c->timer->slot], 0, sizeof c->timer->used[0]);
    if (B->n_paths == 0) return RRB_OK;
    if (B->arena_need > arena_len) return set_err(c, RRB_ERR_INVARIANT, "page extends past the page buffer");
    if (rowmap < 0 || rowmap > 1) return set_err(c, RRB_ERR_INVARIANT, "rowmap must be 0 or 1");
    const bool settled = c->tuning.auto_tile == 1 && c->settled_tw;
    const uint32_t tw = B->tile_w ? B->tile_w : settled ? c->settled_tw : (c->tuning.tile_w ? c->tuning.tile_w : 64);
    const uint32_t th = B->tile_h ? B->tile_h : settled ? c->settled_th : (c->tuning.tile_h ? c->tuning.tile_h : 16);
    c->stats.tile_w = tw;
    c->stats.tile_h = th;
    c->stats.row_shape = B->row_shape;
    uint64_t tiles = 0;
    set_tiles(B->geom_h, tw, th, tiles);
    if (tiles >= (1ull << 31)) return set_err(c, RRB_ERR_INVARIANT, "too many tiles");
    const bool cached = ws && ws->matches(tw, th, B->row_shape, rowmap) && slot < c->h_waves_cap;
    const uint64_t n_paths = B->n_paths, n_pts = B->n_pts, supers = B->supers;
    const uint32_t n_pages = B->n_pages;
    const uint32_t NP = static_cast<uint32_t>(n_paths);
    const double flat_sq = B->flat_sq;
    const int4* pclip = B->has_clip ? as<int4>(B->clip) : nullptr;
    int rc;
    if (cached && c->h_geom && c->geom_slot + n_pages <= c->h_geom_cap) {
        PageGeom* st = c->h_geom + c->geom_slot;
        std::memcpy(st, B->geom_h.data(), n_pages * sizeof(PageGeom));
        RRB_CUDA(c, cudaMemcpyAsync(B->geom.p, st, n_pages * sizeof(PageGeom), cudaMemcpyHostToDevice, c->stream));
    } else {
        RRB_CUDA(c, cudaMemcpyAsync(B->geom.p, B->geom_h.data(), n_pages * sizeof(PageGeom), cudaMemcpyHostToDevice,
                                    c->stream));
    }
    // ---- stage 1: walk, compact pieces, flatten counts, edge offsets
    if ((rc = ensure(c, c->s_slots, n_pts * sizeof(uint2)))) return rc;
    if ((rc = ensure(c, c->s_path_pieces, (n_paths + 1) * sizeof(uint32_t)))) return rc;
    if ((rc = ensure(c, c->s_block, (SCAN_MAX_BLOCKS + 1) * sizeof(uint32_t)))) return rc;
    if ((rc = ensure(c, c->s_ctr, sizeof(BatchCounters)))) return rc;
    RRB_CUDA(c, cudaMemsetAsync(c->s_ctr.p, 0, sizeof(BatchCounters), c->stream));
    stage(c, 0);
    // Paths of up to kLongWalk points: a thread each; longer ones: a warp each.
    constexpr uint32_t kLongWalk = 64;
    k_walk<<<grid_for(c, n_paths, 128, 32), 128, 0, c->stream>>>(as<double>(B->pts), as<uint8_t>(B->flags),
                                                             as<uint64_t>(B->off), NP, as<double>(B->mtx),
                                                             as<uint32_t>(B->page), as<uint32_t>(B->ph),
                                                             as<uint2>(c->s_slots), as<uint32_t>(c->s_path_pieces),
                                                             B->has_hairline ? as<uint8_t>(B->rule) : nullptr,
                                                             kLongWalk);
    c->launches += 1;
    k_walk_long<<<grid_for(c, n_paths * 32, 256, 16), 256, 0, c->stream>>>(
        as<double>(B->pts), as<uint8_t>(B->flags), as<uint64_t>(B->off), NP, as<double>(B->mtx),
        as<uint2>(c->s_slots), as<uint32_t>(c->s_path_pieces), B->has_hairline ? as<uint8_t>(B->rule) : nullptr,
        kLongWalk);
    c->launches += 1;
    RRB_CUDA(c, cudaGetLastError());
    if ((rc = scan_u32(c, as<uint32_t>(c->s_path_pieces), as<uint32_t>(c->s_path_pieces), NP))) return rc;
    if (!cached && (rc = read_back(c, as<uint32_t>(c->s_path_pieces) + NP, sizeof(uint32_t)))) return rc;
    const uint64_t n_pieces = cached ? ws->n_pieces : c->h_read[0];
    const uint32_t NPC = static_cast<uint32_t>(n_pieces);
    if ((rc = ensure(c, c->s_pieces, std::max<uint64_t>(1, n_pieces) * sizeof(uint2)))) return rc;
    if ((rc = ensure(c, c->s_clip, std::max<uint64_t>(1, n_pieces) * sizeof(uint32_t)))) return rc;
    if (pclip && (rc = ensure(c, c->s_clip_lo, std::max<uint64_t>(1, n_pieces) * sizeof(uint32_t)))) return rc;
    uint32_t* clip_lo = pclip ? as<uint32_t>(c->s_clip_lo) : nullptr;
    if ((rc = ensure(c, c->s_edge_off, (n_pieces + 1) * sizeof(uint32_t)))) return rc;
    k_compact_pieces<<<grid_for(c, n_paths * 32, 256, 16), 256, 0, c->stream>>>(
        as<uint64_t>(B->off), as<uint32_t>(c->s_path_pieces), NP, as<uint32_t>(B->page), as<uint32_t>(B->ph),
        as<uint2>(c->s_slots), as<uint2>(c->s_pieces), as<uint32_t>(c->s_clip), pclip, clip_lo);
    c->launches += 1;
    stage_end(c, 0);
    RRB_CUDA(c, cudaGetLastError());
    stage(c, 1);
    // Curves of more than CURVE_BIG segments: listed here, counted by a warp each.
    if ((rc = ensure(c, c->s_big, std::max<uint64_t>(1, n_pieces) * sizeof(uint32_t)))) return rc;
    // Lane counts of the first lane_cap big curves: the write pass places each
    // lane's leaves from them instead of counting again (later curves recount).
    const uint32_t lane_cap = static_cast<uint32_t>(std::min<uint64_t>(n_pieces, kLaneCountCurves));
    if ((rc = ensure(c, c->s_lanes, std::max<uint64_t>(1, lane_cap) * CURVE_LANES))) return rc;
    k_seg_count<true><<<grid_for(c, n_pieces, 128, 32), 128, 0, c->stream>>>(
        as<double>(B->pts), as<uint2>(c->s_pieces), NPC, as<double>(B->mtx), flat_sq, as<uint32_t>(c->s_edge_off),
        as<uint32_t>(c->s_big), as<BatchCounters>(c->s_ctr));
    k_seg_count_big<<<c->sm_count * 16, 128, 0, c->stream>>>(as<double>(B->pts), as<uint2>(c->s_pieces),
                                                            as<double>(B->mtx), flat_sq, as<uint32_t>(c->s_big),
                                                            as<BatchCounters>(c->s_ctr), as<uint32_t>(c->s_edge_off),
                                                            as<uint8_t>(c->s_lanes), lane_cap);
    c->launches += 2;
    stage_end(c, 1);
    RRB_CUDA(c, cudaGetLastError());
    stage(c, 2);
    if ((rc = scan_u32(c, as<uint32_t>(c->s_edge_off), as<uint32_t>(c->s_edge_off), NPC))) return rc;
    stage_end(c, 2);
    if (!cached && (rc = read_back(c, as<uint32_t>(c->s_edge_off) + NPC, sizeof(uint32_t)))) return rc;
    const uint64_t n_edges = cached ? ws->n_edges : c->h_read[0];
    // ---- stage 2: edges, path boxes, row/chunk offsets, supertile bins
    if ((rc = ensure(c, c->s_edges, std::max<uint64_t>(1, n_edges) * sizeof(Edge)))) return rc;
    if ((rc = ensure(c, c->s_info, n_paths * sizeof(PathInfo)))) return rc;
    if ((rc = ensure(c, c->s_rows, (n_paths + 1) * sizeof(uint32_t)))) return rc;
    if ((rc = ensure(c, c->s_chunks, (n_paths + 1) * sizeof(uint32_t)))) return rc;
    if ((rc = ensure(c, c->s_super_cnt, (supers + 1) * sizeof(uint32_t)))) return rc;
    const uint64_t n_egroups = (n_edges + 31) / 32 + 1;
    if ((rc = ensure(c, c->s_groups, n_egroups * 2 * sizeof(int32_t)))) return rc;
    int32_t* gmin = as<int32_t>(c->s_groups);
    int32_t* gmax = gmin + n_egroups;
    // 0x7f7f7f7f / 0x80808080: beyond any AA row, so they act as +inf / -inf.
    RRB_CUDA(c, cudaMemsetAsync(gmin, 0x7f, n_egroups * sizeof(int32_t), c->stream));
    RRB_CUDA(c, cudaMemsetAsync(gmax, 0x80, n_egroups * sizeof(int32_t), c->stream));
    stage(c, 3);
    k_seg_write<true><<<grid_for(c, n_pieces, 128, 32), 128, 0, c->stream>>>(
        as<double>(B->pts), as<uint2>(c->s_pieces), NPC, as<double>(B->mtx), flat_sq, as<uint32_t>(c->s_edge_off),
        static_cast<uint32_t>(n_edges), as<Edge>(c->s_edges), as<uint32_t>(c->s_clip), clip_lo);
    k_seg_write_big<<<c->sm_count * 16, 128, 0, c->stream>>>(
        as<double>(B->pts), as<uint2>(c->s_pieces), as<double>(B->mtx), flat_sq, as<uint32_t>(c->s_big),
        as<BatchCounters>(c->s_ctr), as<uint32_t>(c->s_edge_off), static_cast<uint32_t>(n_edges),
        as<Edge>(c->s_edges), as<uint32_t>(c->s_clip), clip_lo, as<uint8_t>(c->s_lanes), lane_cap);
    c->launches += 2;
    stage_end(c, 3);
    const int chunk_rows = 32;
    stage(c, 4);
    k_path_bbox<<<grid_for(c, n_paths * 32, 256), 256, 0, c->stream>>>(
        as<uint32_t>(c->s_path_pieces), as<uint32_t>(c->s_edge_off), as<Edge>(c->s_edges), NP, as<uint8_t>(B->rule),
        as<uint8_t>(B->gray), as<uint8_t>(B->alpha), as<uint32_t>(B->page), as<uint32_t>(B->pw),
        as<uint32_t>(B->ph), rowmap, as<PathInfo>(c->s_info), as<uint32_t>(c->s_rows), as<uint32_t>(c->s_chunks),
        chunk_rows, as<BatchCounters>(c->s_ctr), gmin, gmax, pclip, B->has_visit ? as<int2>(B->visit) : nullptr);
    c->launches += 1;
    // Hairline segments: their layers' PathInfo and run counts (before the
    // binning, which reads the layers' rectangles).
    if ((rc = ensure(c, c->s_run_off, (n_paths + 1) * sizeof(uint32_t)))) return rc;
    const double* hl_clip = B->has_clip ? as<double>(B->clipf) : nullptr;
    if (B->has_hairline) {
        k_hl_count<<<grid_for(c, n_paths, 128, 16), 128, 0, c->stream>>>(
            as<double>(B->pts), as<uint64_t>(B->off), as<uint8_t>(B->rule), as<double>(B->mtx),
            as<uint32_t>(B->page), as<uint32_t>(B->pw), as<uint32_t>(B->ph), hl_clip, as<uint8_t>(B->gray),
            as<uint8_t>(B->alpha), NP, rowmap, as<PathInfo>(c->s_info), as<uint32_t>(c->s_run_off),
            as<BatchCounters>(c->s_ctr));
        c->launches += 1;
    }
    stage_end(c, 4);
    RRB_CUDA(c, cudaGetLastError());
    stage(c, 5);
    if ((rc = scan_u32(c, as<uint32_t>(c->s_rows), as<uint32_t>(c->s_rows), NP))) return rc;
    if ((rc = scan_u32(c, as<uint32_t>(c->s_chunks), as<uint32_t>(c->s_chunks), NP))) return rc;
    stage_end(c, 5);
    const uint32_t NSUP = static_cast<uint32_t>(supers);
    stage(c, 6);
    k_super_bin<false><<<grid_for(c, supers * 32, 256), 256, 0, c->stream>>>(
        as<PathInfo>(c->s_info), as<PageGeom>(B->geom), n_pages, NSUP, SUPER, SUPER, as<uint32_t>(c->s_super_cnt),
        nullptr, nullptr, nullptr);
    c->launches += 1;
    stage_end(c, 6);
    RRB_CUDA(c, cudaGetLastError());
    stage(c, 7);
    if ((rc = scan_u32(c, as<uint32_t>(c->s_super_cnt), as<uint32_t>(c->s_super_cnt), NSUP))) return rc;
    // Rectilinear paths: runs per path, then their offsets.
    k_recti<false><<<grid_for(c, n_paths, 128, 16), 128, 0, c->stream>>>(
        as<PathInfo>(c->s_info), NP, as<Edge>(c->s_edges), as<uint32_t>(B->pw), rowmap, as<uint32_t>(c->s_run_off),
        nullptr, nullptr, nullptr, 0, as<BatchCounters>(c->s_ctr), pclip);
    c->launches += 1;
    RRB_CUDA(c, cudaGetLastError());
    if ((rc = scan_u32(c, as<uint32_t>(c->s_run_off), as<uint32_t>(c->s_run_off), NP))) return rc;
    stage_end(c, 7);
    uint64_t n_groups, n_chunks, n_pairs, n_runs, raw_entries, hl_rows;
    if (cached) {
        n_groups = ws->n_groups;
        n_chunks = ws->n_chunks;
        n_pairs = ws->n_pairs;
        n_runs = ws->n_runs;
        raw_entries = ws->raw_entries;
        hl_rows = ws->hl_rows;
    } else {
        RRB_CUDA(c, cudaMemcpyAsync(c->h_read + 0, as<uint32_t>(c->s_rows) + NP, 4, cudaMemcpyDeviceToHost,
                                    c->stream));
        RRB_CUDA(c, cudaMemcpyAsync(c->h_read + 1, as<uint32_t>(c->s_chunks) + NP, 4, cudaMemcpyDeviceToHost,
                                    c->stream));
        RRB_CUDA(c, cudaMemcpyAsync(c->h_read + 2, as<uint32_t>(c->s_super_cnt) + NSUP, 4, cudaMemcpyDeviceToHost,
                                    c->stream));
        RRB_CUDA(c, cudaMemcpyAsync(c->h_read + 4, &as<BatchCounters>(c->s_ctr)->raw_entries, 8,
                                    cudaMemcpyDeviceToHost, c->stream));
        RRB_CUDA(c, cudaMemcpyAsync(c->h_read + 6, as<uint32_t>(c->s_run_off) + NP, 4, cudaMemcpyDeviceToHost,
                                    c->stream));
        RRB_CUDA(c, cudaMemcpyAsync(c->h_read + 8, &as<BatchCounters>(c->s_ctr)->hl_rows, 8, cudaMemcpyDeviceToHost,
                                    c->stream));
        ++c->host_syncs;
        RRB_CUDA(c, cudaStreamSynchronize(c->stream));
        n_groups = c->h_read[0];
        n_chunks = c->h_read[1];
        n_pairs = c->h_read[2];
        n_runs = c->h_read[6];
        std::memcpy(&raw_entries, c->h_read + 4, 8);
        std::memcpy(&hl_rows, c->h_read + 8, 8);
    }
    // The run offsets were scanned in 32 bits: refuse totals that could wrap.
    if (hl_rows > 0x7FFFFFFFull || n_runs > 0x7FFFFFFFull)
        return set_err(c, RRB_ERR_POOL_EXHAUSTED, "batch needs more than 2^31 row runs");
    // ---- stage 3: rows -> coverage cells. An AA row with m merged entries
    // yields at most m/2 + 1 spans, and a pixel row at most 2 cells per span
    // boundary: cells <= 4 * spans <= 2 * raw entries + 4 * AA rows.
    const uint64_t aa_rows = 4 * n_groups;
    uint64_t cell_cap = 2 * raw_entries + 4 * aa_rows + hl_rows + 1024;
    if (cell_cap > 0xFFFFFF00ull) return set_err(c, RRB_ERR_POOL_EXHAUSTED, "batch needs more than 2^32 cells");
    if (n_groups > 0x3FFFFFFFull) return set_err(c, RRB_ERR_POOL_EXHAUSTED, "batch needs more than 2^30 pixel rows");
    if ((rc = ensure(c, c->s_row_idx, std::max<uint64_t>(1, n_groups) * sizeof(uint2)))) return rc;
    if ((rc = ensure(c, c->s_spans, cell_cap * sizeof(uint32_t)))) return rc;
    if ((rc = ensure(c, c->s_ovf, std::max<uint64_t>(1, n_groups) * sizeof(uint2)))) return rc;
    if ((rc = ensure(c, c->s_super_list, std::max<uint64_t>(1, n_pairs) * sizeof(uint32_t)))) return rc;
    if ((rc = ensure(c, c->s_runs, std::max<uint64_t>(1, n_runs) * sizeof(int4)))) return rc;
    const PageGeom& last_page = B->geom_h[n_pages - 1];
    const uint64_t n_super_tiles =
        last_page.super_base + static_cast<uint64_t>(last_page.nsx) * ((last_page.h + SUPER - 1) / SUPER);
    if ((rc = ensure(c, c->s_super_start, n_super_tiles * sizeof(uint32_t)))) return rc;
    RRB_CUDA(c, cudaMemsetAsync(c->s_super_start.p, 0, n_super_tiles * sizeof(uint32_t), c->stream));
    stage(c, 8);
    k_super_bin<true><<<grid_for(c, supers * 32, 256), 256, 0, c->stream>>>(
        as<PathInfo>(c->s_info), as<PageGeom>(B->geom), n_pages, NSUP, SUPER, SUPER, nullptr,
        as<uint32_t>(c->s_super_cnt), as<uint32_t>(c->s_super_list), as<uint32_t>(c->s_super_start));
    c->launches += 1;
    stage_end(c, 8);
    stage(c, 9);
    if (n_chunks) {
        if ((rc = ensure(c, c->s_chunk_path, n_chunks * sizeof(uint32_t)))) return rc;
        k_chunk_paths<<<grid_for(c, n_paths * 32, 256), 256, 0, c->stream>>>(as<uint32_t>(c->s_chunks), NP,
                                                                            as<uint32_t>(c->s_chunk_path));
        c->launches += 1;
        // Shapes of the row stage: 12 list entries per AA row with 8 warps per
        // block (the default), 16 entries with 4 warps (fewer rows go to
        // k_groups_mid: pages whose rows carry more crossings), 8 entries with
        // 16 warps, each with one or two edge groups staged per warp.
        auto rows = [&](auto kernel, int warps, size_t smem) -> int {
            RRB_CUDA(c, cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(smem)));
            kernel<<<grid_for(c, n_chunks * 32, warps * 32, 16), warps * 32, smem, c->stream>>>(
                as<PathInfo>(c->s_info), as<uint32_t>(c->s_chunks), as<uint32_t>(c->s_rows), as<Edge>(c->s_edges),
                gmin, gmax, as<uint32_t>(B->pw), NP, as<uint2>(c->s_row_idx), as<uint32_t>(c->s_spans),
                static_cast<uint32_t>(cell_cap), as<uint2>(c->s_ovf), static_cast<uint32_t>(std::max<uint64_t>(1, n_groups)),
                as<BatchCounters>(c->s_ctr), as<uint32_t>(c->s_chunk_path), pclip);
            return RRB_OK;
        };
        switch (B->row_shape) {
            case 1: rc = rows(k_rows<KCAP_WIDE, 4>, 4, rows_smem_bytes<KCAP_WIDE, 4>()); break;
            case 2: rc = rows(k_rows<KCAP, ROWS_WARPS, 1>, ROWS_WARPS, rows_smem_bytes<KCAP, ROWS_WARPS, 1>()); break;
            case 3: rc = rows(k_rows<8, 16>, 16, rows_smem_bytes<8, 16>()); break;
            case 4: rc = rows(k_rows<KCAP_WIDE, 4, 1>, 4, rows_smem_bytes<KCAP_WIDE, 4, 1>()); break;
            default: rc = rows(k_rows<KCAP, ROWS_WARPS>, ROWS_WARPS, rows_smem_bytes<KCAP, ROWS_WARPS>());
        }
        if (rc) return rc;
        c->launches += 1;
    }
    if (n_runs) {
        k_recti<true><<<grid_for(c, n_paths, 128, 16), 128, 0, c->stream>>>(
            as<PathInfo>(c->s_info), NP, as<Edge>(c->s_edges), as<uint32_t>(B->pw), rowmap, nullptr,
            as<uint32_t>(c->s_run_off), as<int4>(c->s_runs), as<uint32_t>(c->s_spans), static_cast<uint32_t>(cell_cap),
            as<BatchCounters>(c->s_ctr), pclip);
        c->launches += 1;
    }
    if (B->has_hairline && hl_rows) {
        k_hl_write<<<grid_for(c, n_paths * 32, 256, 8), 256, 0, c->stream>>>(
            as<double>(B->pts), as<uint64_t>(B->off), as<uint8_t>(B->rule), as<double>(B->mtx),
            as<uint32_t>(B->page), as<uint32_t>(B->pw), as<uint32_t>(B->ph), hl_clip, NP, rowmap,
            as<uint32_t>(c->s_run_off), as<PathInfo>(c->s_info), as<int4>(c->s_runs), as<uint32_t>(c->s_spans),
            static_cast<uint32_t>(cell_cap), as<BatchCounters>(c->s_ctr));
        c->launches += 1;
    }
    stage_end(c, 9);
    RRB_CUDA(c, cudaGetLastError());
    // Overflowing pixel rows, if any: the warp-per-row middle path, then the
    // sequential path for rows longer than its shared lists.
    BatchCounters hc;
    std::memset(&hc, 0, sizeof hc);
    if (!cached) {
        if ((rc = read_back(c, as<BatchCounters>(c->s_ctr), sizeof(BatchCounters)))) return rc;
        std::memcpy(&hc, c->h_read, sizeof hc);
    }
    const uint32_t ovf_cap = static_cast<uint32_t>(std::max<uint64_t>(1, n_groups));
    const uint64_t mid = cached ? ws->mid : std::min<uint64_t>(hc.ovf_count, n_groups);
    uint64_t slow = 0, slow_need = 0;
    if (mid) {
        if ((rc = ensure(c, c->s_ovf2, std::max<uint64_t>(1, n_groups) * sizeof(uint2)))) return rc;
        stage(c, 10);
        k_groups_mid<<<grid_for(c, mid * 32, MID_WARPS * 32, 16), MID_WARPS * 32, 0, c->stream>>>(
            as<PathInfo>(c->s_info), as<uint32_t>(c->s_rows), as<Edge>(c->s_edges), gmin, gmax,
            as<uint32_t>(B->pw), as<uint2>(c->s_ovf), ovf_cap, as<uint2>(c->s_row_idx), as<uint32_t>(c->s_spans),
            static_cast<uint32_t>(cell_cap), as<uint2>(c->s_ovf2), as<BatchCounters>(c->s_ctr), pclip);
        c->launches += 1;
        RRB_CUDA(c, cudaGetLastError());
        if (!cached) {
            if ((rc = read_back(c, as<BatchCounters>(c->s_ctr), sizeof(BatchCounters)))) return rc;
            std::memcpy(&hc, c->h_read, sizeof hc);
        }
        slow = cached ? ws->slow : std::min<uint64_t>(hc.ovf2_count, n_groups);
        if (slow && cached) {
            // The scratch the last render settled on; the cursors are where the
            // faster paths left them on the device.
            slow_need = ws->slow_need;
            if ((rc = ensure(c, c->s_scratch, slow_need * sizeof(int3)))) return rc;
            k_groups_slow<<<grid_for(c, slow * 32, SLOW_WARPS * 32, 16), SLOW_WARPS * 32, 0, c->stream>>>(
                as<PathInfo>(c->s_info), as<uint32_t>(c->s_rows), as<Edge>(c->s_edges), gmin, gmax,
                as<uint32_t>(B->pw), as<uint2>(c->s_ovf2), ovf_cap, as<int3>(c->s_scratch),
                static_cast<uint32_t>(std::min<uint64_t>(c->s_scratch.cap / sizeof(int3), 0xFFFFFFFFull)),
                as<uint2>(c->s_row_idx), as<uint32_t>(c->s_spans), static_cast<uint32_t>(cell_cap),
                as<BatchCounters>(c->s_ctr), pclip);
            c->launches += 1;
            RRB_CUDA(c, cudaGetLastError());
        } else if (slow) {
            uint64_t need = std::min<uint64_t>(slow * 4096 + 4 * n_edges, 0x7FFFFFFFull);
            // Every attempt re-runs all slow rows, so it restarts the cell
            // allocation where the faster paths left it.
            c->h_read[64] = hc.cell_cursor;
            c->h_read[65] = 0;
            for (int attempt = 0; attempt < 4; ++attempt) {
                if ((rc = ensure(c, c->s_scratch, need * sizeof(int3)))) return rc;
                RRB_CUDA(c, cudaMemcpyAsync(&as<BatchCounters>(c->s_ctr)->cell_cursor, &c->h_read[64], 4,
                                            cudaMemcpyHostToDevice, c->stream));
                RRB_CUDA(c, cudaMemcpyAsync(&as<BatchCounters>(c->s_ctr)->scratch_cursor, &c->h_read[65], 4,
                                            cudaMemcpyHostToDevice, c->stream));
                k_groups_slow<<<grid_for(c, slow * 32, SLOW_WARPS * 32, 16), SLOW_WARPS * 32, 0, c->stream>>>(
                    as<PathInfo>(c->s_info), as<uint32_t>(c->s_rows), as<Edge>(c->s_edges), gmin, gmax,
                    as<uint32_t>(B->pw),
                    as<uint2>(c->s_ovf2), ovf_cap, as<int3>(c->s_scratch),
                    static_cast<uint32_t>(std::min<uint64_t>(c->s_scratch.cap / sizeof(int3), 0xFFFFFFFFull)),
                    as<uint2>(c->s_row_idx), as<uint32_t>(c->s_spans), static_cast<uint32_t>(cell_cap),
                    as<BatchCounters>(c->s_ctr), pclip);
                c->launches += 1;
                RRB_CUDA(c, cudaGetLastError());
                if ((rc = read_back(c, as<BatchCounters>(c->s_ctr), sizeof(BatchCounters)))) return rc;
                std::memcpy(&hc, c->h_read, sizeof hc);
                slow_need = need;
                if (!(hc.err & ERR_SCRATCH_CAP)) break;
                // Not enough scratch: grow to what was asked for and run again.
                need = std::min<uint64_t>(static_cast<uint64_t>(hc.scratch_cursor) + 4 * n_edges, 0x7FFFFFFFull);
                c->h_read[66] = hc.err & ~ERR_SCRATCH_CAP;
                RRB_CUDA(c, cudaMemcpyAsync(&as<BatchCounters>(c->s_ctr)->err, &c->h_read[66], 4,
                                            cudaMemcpyHostToDevice, c->stream));
            }
        }
        stage_end(c, 10);
    }
    // ---- stage 4: composite
    stage(c, 11);
    if (c->wait_pages_up) {  // the first composite of a host render: its pages must have landed
        RRB_CUDA(c, cudaStreamWaitEvent(c->stream, c->pages_up, 0));
        c->wait_pages_up = false;
    }
    // Persistent: as many CTAs as fit on the device at once (the CTAs per SM
    // the composite is compiled for), taking tiles from the work queue.
    const int comp_per_sm = comp_ctas_per_sm(static_cast<int>(tw), static_cast<int>(th));
    if ((rc = launch_composite(c, static_cast<int>(tw), static_cast<int>(th), grid_for(c, tiles, 1, comp_per_sm),
                               as<PathInfo>(c->s_info), as<PageGeom>(B->geom), n_pages, static_cast<uint32_t>(tiles),
                               as<uint32_t>(c->s_super_cnt), as<uint32_t>(c->s_super_list), as<uint32_t>(c->s_rows),
                               as<uint2>(c->s_row_idx), as<uint32_t>(c->s_spans), as<int4>(c->s_runs), arena,
                               rowmap, as<BatchCounters>(c->s_ctr), B->bpp == 3 ? as<uint32_t>(B->rgb) : nullptr,
                               n_runs > 0, as<uint32_t>(c->s_super_start))))
        return rc;
    stage_end(c, 11);
    c->stats.paths = n_paths;
    c->stats.pieces = n_pieces;
    c->stats.segments = n_edges;
    c->stats.tiles = tiles;
    c->stats.tile_pairs = n_pairs;
    c->stats.kernel_launches = c->launches;
    c->stats.row_groups = n_groups;
    if (cached) {
        // The counters go to this wave's page-locked slot; the caller reads
        // them (and the stage events) after its one wait on the stream.
        RRB_CUDA(c, cudaMemcpyAsync(c->h_waves + slot, c->s_ctr.p, sizeof(BatchCounters), cudaMemcpyDeviceToHost,
                                    c->stream));
        c->deferred = true;
        c->stats.host_syncs = c->host_syncs;
        return RRB_OK;
    }
    if ((rc = read_back(c, as<BatchCounters>(c->s_ctr), sizeof(BatchCounters)))) return rc;
    std::memcpy(&hc, c->h_read, sizeof hc);
    if (ws && !hc.err) {
        ws->valid = true;
        ws->tw = tw;
        ws->th = th;
        ws->row_shape = B->row_shape;
        ws->rowmap = rowmap;
        ws->n_pieces = n_pieces;
        ws->n_edges = n_edges;
        ws->n_groups = n_groups;
        ws->n_chunks = n_chunks;
        ws->n_pairs = n_pairs;
        ws->n_runs = n_runs;
        ws->raw_entries = raw_entries;
        ws->hl_rows = hl_rows;
        ws->mid = mid;
        ws->slow = slow;
        ws->slow_need = slow_need;
    }
    c->stats.paths = n_paths;
    c->stats.pieces = n_pieces;
    c->stats.segments = n_edges;
    c->stats.aa_rows = hc.aa_rows;
    c->stats.spans = hc.cell_cursor;
    c->stats.row_overflows = hc.ovf_count;
    c->stats.pieces = n_pieces;
    c->stats.tiles = tiles;
    c->stats.tile_pairs = n_pairs;
    c->stats.nonterminating_rows = hc.nonterminating;
    c->stats.kernel_launches = c->launches;
    c->stats.row_groups = n_groups;
    c->stats.host_syncs = c->host_syncs;
    if (c->timer && c->timer->on) {
        // The final read_back synchronised the stream: every event is complete.
        const int sl = c->timer->slot;
        for (int k = 0; k < kStages; ++k) {
            float ms = 0.f;
            if (c->timer->used[sl][k]) cudaEventElapsedTime(&ms, c->timer->begin[sl][k], c->timer->end[sl][k]);
            c->stage_ms[k] = ms;
            c->stage_launches[k] = c->timer->used[sl][k] ? c->timer->launches[sl][k] : 0;
        }
    }
    if (hc.err) {
        char buf[128];
        std::snprintf(buf, sizeof buf, "batch capacity exceeded (error bits 0x%x); pages left untouched", hc.err);
        return set_err(c, RRB_ERR_POOL_EXHAUSTED, buf);
    }
    return RRB_OK;
}

// Binning geometry (supertiles, (supertile x path block) work items) of pages
// whose path ranges are already set.
void set_binning(std::vector<PageGeom>& geom, uint64_t& supers_out) {
    uint64_t supers = 0, work = 0;
    for (PageGeom& G : geom) {
        G.nsx = (G.w + SUPER - 1) / SUPER;
        G.super_base = static_cast<uint32_t>(supers);
        supers += static_cast<uint64_t>(G.nsx) * ((G.h + SUPER - 1) / SUPER);
        G.nblk = std::max<uint32_t>(1, (G.path_end - G.path_begin + BIN_BLOCK - 1) / BIN_BLOCK);
        G.work_base = static_cast<uint32_t>(work);
        work += static_cast<uint64_t>(G.nsx) * ((G.h + SUPER - 1) / SUPER) * G.nblk;
    }
    supers_out = work;
}

void release_scratch(rrb_ctx* c) {
    cudaStreamSynchronize(c->stream);
    Scratch* all[] = {&c->s_pieces, &c->s_clip, &c->s_edge_off, &c->s_edges, &c->s_info, &c->s_rows, &c->s_chunks,
                      &c->s_super_cnt, &c->s_super_list, &c->s_super_start, &c->s_big, &c->s_lanes, &c->s_row_idx, &c->s_spans, &c->s_ovf, &c->s_scratch,
                      &c->s_groups, &c->s_slots, &c->s_path_pieces, &c->s_ovf2, &c->s_run_off, &c->s_runs,
                      &c->s_chunk_path, &c->s_clip_lo, &c->s_hl_clip};
    for (Scratch* x : all) {
        dev_free(c, x->p, x->cap);
        x->p = nullptr;
        x->cap = 0;
    }
}

// Pages [pg0, pg1) of B as a batch of their own: the inputs are views into
// B's device arrays; only the per-path offsets and page indices are rebased.
int make_wave(rrb_ctx* c, rrb_batch* B, uint32_t pg0, uint32_t pg1, rrb_batch* W) {
    W->view = true;  // off / page / geom are owned (and reused across waves), the rest are views
    const uint32_t pb = B->geom_h[pg0].path_begin, pe = B->geom_h[pg1 - 1].path_end;
    const uint64_t ptb = B->page_pt[pg0], pte = B->page_pt[pg1];
    W->n_paths = pe - pb;
    W->n_pts = pte - ptb;
    W->n_pages = pg1 - pg0;
    W->flat_sq = B->flat_sq;
    W->rowmap = B->rowmap;
    W->arena_need = B->arena_need;
    auto view = [](Scratch& dst, const Scratch& src, size_t byte_off) {
        dst.p = static_cast<char*>(src.p) + byte_off;
        dst.cap = 0;
    };
    view(W->pts, B->pts, 2 * ptb * sizeof(double));
    view(W->flags, B->flags, ptb);
    view(W->rule, B->rule, pb);
    view(W->gray, B->gray, pb);
    view(W->alpha, B->alpha, pb);
    view(W->pw, B->pw, pg0 * sizeof(uint32_t));
    view(W->ph, B->ph, pg0 * sizeof(uint32_t));
    view(W->mtx, B->mtx, 0);
    W->bpp = B->bpp;
    if (B->bpp == 3) view(W->rgb, B->rgb, pb * sizeof(uint32_t));
    W->has_clip = B->has_clip;
    W->has_hairline = B->has_hairline;
    W->row_shape = B->row_shape;
    W->tile_w = B->tile_w;
    W->tile_h = B->tile_h;
    if (B->has_clip) view(W->clip, B->clip, pb * sizeof(int4));
    if (B->has_clip) view(W->clipf, B->clipf, pb * 4 * sizeof(double));
    W->has_visit = B->has_visit;
    if (B->has_visit) view(W->visit, B->visit, pb * sizeof(int2));
    int rc;
    if ((rc = ensure(c, W->off, (W->n_paths + 1) * sizeof(uint64_t)))) return rc;
    if ((rc = ensure(c, W->page, std::max<uint64_t>(1, W->n_paths) * sizeof(uint32_t)))) return rc;
    if ((rc = ensure(c, W->geom, W->n_pages * sizeof(PageGeom)))) return rc;
    k_rebase_paths<<<grid_for(c, W->n_paths + 1, 256), 256, 0, c->stream>>>(
        as<uint64_t>(B->off) + pb, as<uint64_t>(W->off), ptb, as<uint32_t>(B->page) + pb, as<uint32_t>(W->page), pg0,
        static_cast<uint32_t>(W->n_paths));
    c->launches += 1;
    RRB_CUDA(c, cudaGetLastError());
    W->geom_h.assign(B->geom_h.begin() + pg0, B->geom_h.begin() + pg1);
    for (PageGeom& G : W->geom_h) {
        G.path_begin -= pb;
        G.path_end -= pb;
    }
    set_binning(W->geom_h, W->supers);
    W->page_pt.clear();
    return RRB_OK;
}

// Points per wave: a page is never split, consecutive pages are grouped up
// to this many path points; a wave that runs out of device memory is split
// in half and retried.
constexpr uint64_t kWavePoints = 40ull << 20;

// ws / slot: the wave's cached sizes and counter slot (run_resident_one);
// the halves of a wave that had to be split get none.
int run_pages(rrb_ctx* c, rrb_batch* B, uint32_t pg0, uint32_t pg1, uint8_t* arena, size_t arena_len, int rowmap,
              rrb_batch_stats& acc, int depth, std::vector<uint32_t>& done_plan, WaveSizes* ws = nullptr,
              uint32_t slot = 0) {
    int rc;
    if (pg0 == 0 && pg1 == B->n_pages) {
        rc = run_resident_one(c, B, arena, arena_len, rowmap, ws, slot);
    } else {
        rc = make_wave(c, B, pg0, pg1, c->wave_batch);
        if (!rc) rc = run_resident_one(c, c->wave_batch, arena, arena_len, rowmap, ws, slot);
    }
    if (rc == RRB_OK) {
        const rrb_batch_stats& s = c->stats;
        acc.paths += s.paths;
        acc.pieces += s.pieces;
        acc.segments += s.segments;
        acc.aa_rows += s.aa_rows;
        acc.spans += s.spans;
        acc.row_overflows += s.row_overflows;
        acc.tiles += s.tiles;
        acc.tile_pairs += s.tile_pairs;
        acc.nonterminating_rows += s.nonterminating_rows;
        acc.kernel_launches += s.kernel_launches;
        acc.row_groups += s.row_groups;
        acc.host_syncs += s.host_syncs;
        acc.waves += 1;
        acc.tile_w = s.tile_w;
        acc.tile_h = s.tile_h;
        acc.row_shape = s.row_shape;
        for (int k = 0; k < 16; ++k) {
            c->stage_sum_ms[k] += c->stage_ms[k];
            c->stage_sum_launches[k] += c->stage_launches[k];
        }
        done_plan.push_back(pg1);
        return RRB_OK;
    }
    const bool splittable = (rc == RRB_ERR_OUT_OF_MEMORY || rc == RRB_ERR_POOL_EXHAUSTED) && pg1 - pg0 > 1 && depth < 20;
    if (!splittable) return rc;
    // The composite had not run, so the pages are untouched: split. Out of
    // memory also gives the scratch back first; a cell-capacity overflow
    // (more than 2^32 coverage cells) keeps it.
    cudaGetLastError();
    if (rc == RRB_ERR_OUT_OF_MEMORY) release_scratch(c);
    const uint32_t mid = pg0 + (pg1 - pg0) / 2;
    if ((rc = run_pages(c, B, pg0, mid, arena, arena_len, rowmap, acc, depth + 1, done_plan))) return rc;
    return run_pages(c, B, mid, pg1, arena, arena_len, rowmap, acc, depth + 1, done_plan);
}

int run_resident_waves(rrb_ctx* c, rrb_batch* B, uint8_t* arena, size_t arena_len, int rowmap);

int run_resident(rrb_ctx* c, rrb_batch* B, uint8_t* arena, size_t arena_len, int rowmap) {
    if (B->trial_epoch != c->tuning_epoch) {
        // Plan the first phase of the trials: the tile shapes (the context's,
        // or with automatic tiles 64x16, 128x16 and 128x32), row shape 0.
        B->trial_epoch = c->tuning_epoch;
        B->trials.clear();
        B->trial = 0;
        B->row_trials_planned = false;
        const uint32_t cw = c->tuning.tile_w ? c->tuning.tile_w : 64, ch = c->tuning.tile_h ? c->tuning.tile_h : 16;
        if (c->tuning.auto_tile == 1) {
            // The shape the context last settled on goes first: a batch
            // uploaded per call renders once, with the first trial's shapes.
            uint32_t shapes[3][2] = {{64u, 16u}, {128u, 16u}, {128u, 32u}};
            for (int k = 1; k < 3; ++k)
                if (shapes[k][0] == c->settled_tw && shapes[k][1] == c->settled_th) std::swap(shapes[0], shapes[k]);
            for (const auto& t : shapes) B->trials.push_back({t[0], t[1], 0, 0.f});
        } else {
            B->trials.push_back({cw, ch, 0, 0.f});
        }
    }
    auto settled = [&]() {
        c->stats.trials_left = B->trials.size() - B->trial;
    };
    if (B->trial >= B->trials.size()) {
        const int rc = run_resident_waves(c, B, arena, arena_len, rowmap);
        settled();
        return rc;
    }
    const rrb_batch::Trial& T = B->trials[B->trial];
    B->tile_w = T.tw;
    B->tile_h = T.th;
    B->row_shape = T.rs;
    for (cudaEvent_t& e : c->trial_ev)
        if (!e) RRB_CUDA(c, cudaEventCreate(&e));
    const uint64_t g0 = c->scratch_grows;
    RRB_CUDA(c, cudaEventRecord(c->trial_ev[0], c->stream));
    const int rc = run_resident_waves(c, B, arena, arena_len, rowmap);
    if (rc != RRB_OK) return rc;
    RRB_CUDA(c, cudaEventRecord(c->trial_ev[1], c->stream));
    ++c->stats.host_syncs;
    RRB_CUDA(c, cudaEventSynchronize(c->trial_ev[1]));
    float ms = 0.f;
    RRB_CUDA(c, cudaEventElapsedTime(&ms, c->trial_ev[0], c->trial_ev[1]));
    if (c->scratch_grows == g0) {  // a render that grew scratch is repeated
        B->trials[B->trial].ms = ms;
        if (++B->trial == B->trials.size()) {
            size_t best = 0;
            for (size_t k = 1; k < B->trials.size(); ++k)
                if (B->trials[k].ms < B->trials[best].ms) best = k;
            if (!B->row_trials_planned) {
                // Second phase: the other row shapes with the fastest tile.
                B->row_trials_planned = true;
                const rrb_batch::Trial T0 = B->trials[best];
                for (uint8_t rs = 1; rs < kRowShapes; ++rs) B->trials.push_back({T0.tw, T0.th, rs, 0.f});
            } else {
                B->tile_w = B->trials[best].tw;
                B->tile_h = B->trials[best].th;
                B->row_shape = B->trials[best].rs;
                if (c->tuning.auto_tile == 1) {
                    c->settled_tw = B->tile_w;
                    c->settled_th = B->tile_h;
                }
            }
        }
    }
    settled();
    return RRB_OK;
}

int run_resident_waves(rrb_ctx* c, rrb_batch* B, uint8_t* arena, size_t arena_len, int rowmap) {
    rrb_batch_stats acc{};
    const uint64_t grows0 = c->scratch_grows;
    struct Done {
        rrb_ctx* c;
        uint64_t g0;
        ~Done() { c->stats.scratch_grows = c->scratch_grows - g0; }
    } done{c, grows0};
    const uint64_t wave_pts = c->tuning.wave_points ? c->tuning.wave_points : kWavePoints;
    // Wave plan: the groups that worked last time, else consecutive pages up
    // to wave_pts points each (any group that fails is split in two).
    std::vector<uint32_t> plan;
    const bool reused = !B->plan.empty() && B->plan_wave_points == wave_pts && B->plan.back() == B->n_pages;
    if (!reused) B->sizes.clear();  // sizes belong to the plan's waves
    if (reused) {
        plan = B->plan;
    } else if (B->n_paths == 0 || B->n_pts <= wave_pts) {
        plan = {0, B->n_pages};
    } else {
        plan.push_back(0);
        uint32_t pg = 0;
        while (pg < B->n_pages) {
            uint32_t end = pg + 1;
            while (end < B->n_pages && B->page_pt[end + 1] - B->page_pt[pg] <= wave_pts) ++end;
            plan.push_back(end);
            pg = end;
        }
    }
    std::memset(c->stage_sum_ms, 0, sizeof c->stage_sum_ms);
    std::memset(c->stage_sum_launches, 0, sizeof c->stage_sum_launches);
    // Waves whose sizes the last render of this plan found: launched without
    // waiting on the stream, their counters read after one wait at the end.
    const size_t n_waves = plan.size() - 1;
    if (B->sizes.size() != n_waves) B->sizes.assign(n_waves, WaveSizes{});
    if (c->h_waves_cap < n_waves) {
        if (c->h_waves) cudaFreeHost(c->h_waves);
        c->h_waves = nullptr;
        c->h_waves_cap = 0;
        void* h = nullptr;
        if (cudaMallocHost(&h, std::max<size_t>(n_waves, 8) * sizeof(BatchCounters)) == cudaSuccess) {
            c->h_waves = static_cast<BatchCounters*>(h);
            c->h_waves_cap = static_cast<uint32_t>(std::max<size_t>(n_waves, 8));
        } else {
            cudaGetLastError();  // no slots: every wave reads its sizes back
        }
    }
    if (c->h_geom_cap < B->n_pages) {
        if (c->h_geom) cudaFreeHost(c->h_geom);
        c->h_geom = nullptr;
        c->h_geom_cap = 0;
        void* h = nullptr;
        if (cudaMallocHost(&h, std::max<size_t>(B->n_pages, 64) * sizeof(PageGeom)) == cudaSuccess) {
            c->h_geom = static_cast<PageGeom*>(h);
            c->h_geom_cap = static_cast<uint32_t>(std::max<size_t>(B->n_pages, 64));
        } else {
            cudaGetLastError();  // geometry then comes from pageable memory
        }
    }
    std::vector<uint32_t> done_plan{plan.front()}, deferred;
    for (size_t i = 0; i < n_waves; ++i) {
        const uint32_t slot = static_cast<uint32_t>(i);
        if (c->timer) c->timer->slot = static_cast<int>(std::min<size_t>(i, kTimedWaves - 1));
        c->geom_slot = plan[i];
        int rc = run_pages(c, B, plan[i], plan[i + 1], arena, arena_len, rowmap, acc, 0, done_plan, &B->sizes[i],
                           slot);
        if (rc) {
            c->stats = acc;
            B->plan.clear();
            B->sizes.clear();
            if (c->timer) c->timer->slot = 0;
            return rc;
        }
        if (c->deferred) deferred.push_back(slot);
    }
    if (c->timer) c->timer->slot = 0;
    if (!deferred.empty()) {
        // The render's one wait: then every deferred wave's counters and events.
        ++acc.host_syncs;
        RRB_CUDA(c, cudaStreamSynchronize(c->stream));
        uint32_t err = 0;
        for (uint32_t w : deferred) {
            const BatchCounters& hc = c->h_waves[w];
            err |= hc.err;
            acc.aa_rows += hc.aa_rows;
            acc.spans += hc.cell_cursor;
            acc.row_overflows += hc.ovf_count;
            acc.nonterminating_rows += hc.nonterminating;
            if (c->timer && c->timer->on) {
                const int sl = static_cast<int>(std::min<uint32_t>(w, kTimedWaves - 1));
                for (int k = 0; k < kStages; ++k) {
                    float ms = 0.f;
                    if (c->timer->used[sl][k]) cudaEventElapsedTime(&ms, c->timer->begin[sl][k], c->timer->end[sl][k]);
                    c->stage_sum_ms[k] += ms;
                    c->stage_sum_launches[k] += c->timer->used[sl][k] ? c->timer->launches[sl][k] : 0;
                }
            }
        }
        if (err) {
            // Cannot happen for the inputs the sizes came from; drop them.
            B->sizes.clear();
            c->stats = acc;
            char buf[128];
            std::snprintf(buf, sizeof buf, "batch capacity exceeded on a replay (error bits 0x%x)", err);
            return set_err(c, RRB_ERR_POOL_EXHAUSTED, buf);
        }
    }
    if (done_plan != plan) B->sizes.assign(done_plan.size() - 1, WaveSizes{});  // waves were split
    B->plan = done_plan;
    B->plan_wave_points = wave_pts;
    c->stats = acc;
    // Stage times of the whole render: the sums over its waves.
    std::memcpy(c->stage_ms, c->stage_sum_ms, sizeof c->stage_ms);
    std::memcpy(c->stage_launches, c->stage_sum_launches, sizeof c->stage_launches);
    return RRB_OK;
}

// Paths [pa, pb) of B as a batch of their own (a path-range wave): the pages
// they lie on, each keeping only those paths. Rendering consecutive path
// ranges one after another composites every page in path order, the same
// pixels as one pass. ptb / pte: the range's first point and end.
int make_path_wave(rrb_ctx* c, rrb_batch* B, uint32_t pa, uint32_t pb, uint64_t ptb, uint64_t pte, rrb_batch* W) {
    auto page_of = [&](uint32_t path) {  // the page whose path range holds `path`
        uint32_t lo = 0, hi = B->n_pages;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) / 2;
            if (B->geom_h[mid].path_begin <= path) lo = mid;
            else hi = mid;
        }
        while (lo + 1 < B->n_pages && B->geom_h[lo].path_end <= path) ++lo;
        return lo;
    };
    const uint32_t pg0 = page_of(pa), pg1 = page_of(pb - 1) + 1;
    W->view = true;
    W->n_paths = pb - pa;
    W->n_pts = pte - ptb;
    W->n_pages = pg1 - pg0;
    W->flat_sq = B->flat_sq;
    W->rowmap = B->rowmap;
    W->arena_need = B->arena_need;
    W->bpp = B->bpp;
    W->has_clip = B->has_clip;
    W->has_hairline = B->has_hairline;
    W->row_shape = B->row_shape;
    W->tile_w = B->tile_w;
    W->tile_h = B->tile_h;
    auto view = [](Scratch& dst, const Scratch& src, size_t byte_off) {
        dst.p = static_cast<char*>(src.p) + byte_off;
        dst.cap = 0;
    };
    view(W->pts, B->pts, 2 * ptb * sizeof(double));
    view(W->flags, B->flags, ptb);
    view(W->rule, B->rule, pa);
    view(W->gray, B->gray, pa);
    view(W->alpha, B->alpha, pa);
    view(W->pw, B->pw, pg0 * sizeof(uint32_t));
    view(W->ph, B->ph, pg0 * sizeof(uint32_t));
    view(W->mtx, B->mtx, 0);
    if (B->bpp == 3) view(W->rgb, B->rgb, pa * sizeof(uint32_t));
    W->has_visit = B->has_visit;
    if (B->has_visit) view(W->visit, B->visit, pa * sizeof(int2));
    if (B->has_clip) {
        view(W->clip, B->clip, pa * sizeof(int4));
        view(W->clipf, B->clipf, pa * 4 * sizeof(double));
    }
    int rc;
    if ((rc = ensure(c, W->off, (W->n_paths + 1) * sizeof(uint64_t)))) return rc;
    if ((rc = ensure(c, W->page, std::max<uint64_t>(1, W->n_paths) * sizeof(uint32_t)))) return rc;
    if ((rc = ensure(c, W->geom, W->n_pages * sizeof(PageGeom)))) return rc;
    k_rebase_paths<<<grid_for(c, W->n_paths + 1, 256), 256, 0, c->stream>>>(
        as<uint64_t>(B->off) + pa, as<uint64_t>(W->off), ptb, as<uint32_t>(B->page) + pa, as<uint32_t>(W->page), pg0,
        static_cast<uint32_t>(W->n_paths));
    c->launches += 1;
    RRB_CUDA(c, cudaGetLastError());
    W->geom_h.assign(B->geom_h.begin() + pg0, B->geom_h.begin() + pg1);
    for (PageGeom& G : W->geom_h) {
        G.path_begin = std::min(std::max(G.path_begin, pa), pb) - pa;
        G.path_end = std::max(std::min(G.path_end, pb), pa) - pa;
        if (G.path_end < G.path_begin) G.path_end = G.path_begin;
    }
    set_binning(W->geom_h, W->supers);
    W->page_pt.clear();
    W->plan.clear();
    return RRB_OK;
}

// Path range [pa, pb) of B; a range that runs out of memory or cell capacity
// is split in two (its composite had not run, so the pages are untouched).
int run_path_range(rrb_ctx* c, rrb_batch* B, const uint64_t* path_pt_off, uint32_t pa, uint32_t pb, uint8_t* arena,
                   size_t arena_len, int rowmap, rrb_batch_stats& acc, int depth) {
    int rc = make_path_wave(c, B, pa, pb, path_pt_off[pa], path_pt_off[pb], c->wave_batch);
    if (!rc) rc = run_resident_one(c, c->wave_batch, arena, arena_len, rowmap);
    if (rc == RRB_OK) {
        const rrb_batch_stats& s = c->stats;
        acc.paths += s.paths;
        acc.pieces += s.pieces;
        acc.segments += s.segments;
        acc.aa_rows += s.aa_rows;
        acc.spans += s.spans;
        acc.row_overflows += s.row_overflows;
        acc.tiles += s.tiles;
        acc.tile_pairs += s.tile_pairs;
        acc.nonterminating_rows += s.nonterminating_rows;
        acc.kernel_launches += s.kernel_launches;
        acc.row_groups += s.row_groups;
        acc.host_syncs += s.host_syncs;
        acc.waves += 1;
        acc.tile_w = s.tile_w;
        acc.tile_h = s.tile_h;
        acc.row_shape = s.row_shape;
        for (int k = 0; k < 16; ++k) {
            c->stage_sum_ms[k] += c->stage_ms[k];
            c->stage_sum_launches[k] += c->stage_launches[k];
        }
        return RRB_OK;
    }
    const bool splittable = (rc == RRB_ERR_OUT_OF_MEMORY || rc == RRB_ERR_POOL_EXHAUSTED) && pb - pa > 1 && depth < 24;
    if (!splittable) return rc;
    cudaGetLastError();
    if (rc == RRB_ERR_OUT_OF_MEMORY) release_scratch(c);
    const uint32_t mid = pa + (pb - pa) / 2;
    if ((rc = run_path_range(c, B, path_pt_off, pa, mid, arena, arena_len, rowmap, acc, depth + 1))) return rc;
    return run_path_range(c, B, path_pt_off, mid, pb, arena, arena_len, rowmap, acc, depth + 1);
}

// Points per batch from which host batches in page-locked memory are
// streamed: their points are copied range by range on a second stream while
// the ranges before them render, so the upload hides behind the render.
constexpr uint64_t kStreamMinPoints = 4ull << 20;
constexpr uint64_t kStreamRanges = 4;

bool page_locked(const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Host pages of rrb_render_pages_host: up before the render (or, with
// init >= 0, filled with that byte on the device instead), down after it.
struct HostPages {
    uint8_t* p = nullptr;
    size_t len = 0;
    int init = -1;
};

// io (optional): the streamed render also moves the pages. They go up on the
// copy stream behind the first range's points, and the first composite
// waits for them (pages filled on the device instead: a fill ahead of the
// first range); each page goes down on its own stream, beside the uploads,
// as soon as the last range with a path on it has composited, while later
// ranges render.
int run_streamed(rrb_ctx* c, const rrb_path_batch_params* h, rrb_batch* B, uint8_t* arena, size_t arena_len,
                 const HostPages* io = nullptr) {
    if (!c->copy_stream) RRB_CUDA(c, cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    if (io && !c->down_stream) RRB_CUDA(c, cudaStreamCreateWithFlags(&c->down_stream, cudaStreamNonBlocking));
    // Ranges of consecutive paths: a first one of about a tenth of the
    // points (the render starts once its copy lands), then kStreamRanges - 1
    // equal ones (copies run a little faster than renders, so they stay ahead).
    const uint64_t first = std::max<uint64_t>(1ull << 20, h->n_pts / 10);
    const uint64_t target = std::max<uint64_t>(
        1ull << 20, (h->n_pts - std::min(first, h->n_pts) + kStreamRanges - 2) / (kStreamRanges - 1));
    std::vector<uint32_t> cut{0};
    for (uint64_t p = 1; p < h->n_paths; ++p)
        if (h->path_pt_off[p] - h->path_pt_off[cut.back()] >= (cut.size() == 1 ? first : target))
            cut.push_back(static_cast<uint32_t>(p));
    cut.push_back(static_cast<uint32_t>(h->n_paths));
    const size_t nr = cut.size() - 1;
    // ev[0 .. nr-1]: range r's points landed; ev[nr]: previous work done;
    // ev[nr+1]: pages landed; ev[nr+2 ..]: range r composited.
    std::vector<cudaEvent_t> ev(2 * nr + 2, nullptr);
    for (auto& e : ev) RRB_CUDA(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    auto done = [&](int rc) {
        cudaStreamSynchronize(c->copy_stream);  // no copy from the caller's memory may outlive the call
        if (io) cudaStreamSynchronize(c->down_stream);
        for (auto& e : ev) cudaEventDestroy(e);
        return rc;
    };
    // The copies start once the device is done with the previous batch in these buffers.
    RRB_CUDA(c, cudaEventRecord(ev[nr], c->stream));
    RRB_CUDA(c, cudaStreamWaitEvent(c->copy_stream, ev[nr], 0));
    if (io && io->init >= 0) RRB_CUDA(c, cudaMemsetAsync(arena, io->init, io->len, c->stream));
    for (size_t r = 0; r < nr; ++r) {
        const uint64_t a = h->path_pt_off[cut[r]], b = h->path_pt_off[cut[r + 1]];
        if (b > a) {
            if (cudaMemcpyAsync(as<double>(B->pts) + 2 * a, h->pts + 2 * a, 2 * (b - a) * sizeof(double),
                                cudaMemcpyHostToDevice, c->copy_stream) != cudaSuccess ||
                cudaMemcpyAsync(as<uint8_t>(B->flags) + a, h->flags + a, b - a, cudaMemcpyHostToDevice,
                                c->copy_stream) != cudaSuccess)
                return done(set_err(c, RRB_ERR_DEVICE, "point upload failed"));
        }
        if (cudaEventRecord(ev[r], c->copy_stream) != cudaSuccess) return done(set_err(c, RRB_ERR_DEVICE, "event"));
        if (r == 0 && io && io->init < 0) {
            if (cudaMemcpyAsync(arena, io->p, io->len, cudaMemcpyHostToDevice, c->copy_stream) != cudaSuccess ||
                cudaEventRecord(ev[nr + 1], c->copy_stream) != cudaSuccess)
                return done(set_err(c, RRB_ERR_DEVICE, "page upload failed"));
            c->pages_up = ev[nr + 1];
            c->wait_pages_up = true;
        }
    }
    uint32_t next_down = 0;  // first page not yet on its way down
    auto send_down = [&](uint32_t upto, cudaEvent_t after) -> bool {
        if (!io || next_down >= upto) return true;
        if (cudaEventRecord(after, c->stream) != cudaSuccess || cudaStreamWaitEvent(c->down_stream, after, 0) != cudaSuccess)
            return false;
        for (; next_down < upto; ++next_down) {
            const uint64_t off = h->page_offset[next_down];
            const uint64_t bytes = static_cast<uint64_t>(B->bpp) * h->page_width[next_down] * h->page_height[next_down];
            const uint64_t end = std::min<uint64_t>(off + bytes, io->len);
            if (off < end && cudaMemcpyAsync(io->p + off, arena + off, end - off, cudaMemcpyDeviceToHost,
                                             c->down_stream) != cudaSuccess)
                return false;
        }
        return true;
    };
    rrb_batch_stats acc{};
    const uint64_t grows0 = c->scratch_grows;
    std::memset(c->stage_sum_ms, 0, sizeof c->stage_sum_ms);
    std::memset(c->stage_sum_launches, 0, sizeof c->stage_sum_launches);
    for (size_t r = 0; r < nr; ++r) {
        if (cudaStreamWaitEvent(c->stream, ev[r], 0) != cudaSuccess) return done(set_err(c, RRB_ERR_DEVICE, "event"));
        const int rc = run_path_range(c, B, h->path_pt_off, cut[r], cut[r + 1], arena, arena_len, h->rowmap, acc, 0);
        if (rc) {
            c->wait_pages_up = false;
            c->stats = acc;
            return done(rc);
        }
        // Pages whose paths all lie in ranges 0..r are final.
        uint32_t upto = next_down;
        while (upto < B->n_pages && (r + 1 == nr || B->geom_h[upto].path_end <= cut[r + 1])) ++upto;
        if (!send_down(upto, ev[nr + 2 + r])) return done(set_err(c, RRB_ERR_DEVICE, "page download failed"));
    }
    if (c->wait_pages_up) {  // no range reached a composite: the pages still go up and come back
        RRB_CUDA(c, cudaStreamWaitEvent(c->stream, c->pages_up, 0));
        c->wait_pages_up = false;
        if (!send_down(B->n_pages, ev[2 * nr + 1])) return done(set_err(c, RRB_ERR_DEVICE, "page download failed"));
    }
    c->stats = acc;
    c->stats.scratch_grows = c->scratch_grows - grows0;
    std::memcpy(c->stage_ms, c->stage_sum_ms, sizeof c->stage_ms);
    std::memcpy(c->stage_launches, c->stage_sum_launches, sizeof c->stage_launches);
    return done(RRB_OK);
}

// stream: allow the streamed form. Paint batches do not stream: their points
// are built on the host first, and their slow rows (one thread per row, a
// few long ones) cost more split over ranges than the copy they would hide.
// t0: when the caller's own host work began (default: now); the stats'
// host_ns is the time from it to the first kernel.
// io (optional): host pages to upload before and download after the render
// (overlapped with it when the batch streams).
int run_batch(rrb_ctx* c, const rrb_path_batch_params* h, uint8_t* arena, size_t arena_len,
              const uint8_t* rgb = nullptr, const double* clip = nullptr, bool hairlines = false, bool stream = true,
              const std::chrono::steady_clock::time_point* t0 = nullptr, const int32_t* visit = nullptr,
              const HostPages* io = nullptr) {
    const auto start = t0 ? *t0 : std::chrono::steady_clock::now();
    rrb_batch* B = c->tmp_batch;
    const bool streamed = stream && h->n_paths > 1 && h->n_pts >= kStreamMinPoints && page_locked(h->pts) &&
                          page_locked(h->flags);
    int rc = batch_upload(c, h, B, rgb, clip, hairlines, streamed, visit);
    if (rc) return rc;
    const uint64_t host_ns = static_cast<uint64_t>(
        std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - start).count());
    if (streamed) {
        rc = run_streamed(c, h, B, arena, arena_len, io);
    } else {
        if (io && io->init >= 0) RRB_CUDA(c, cudaMemsetAsync(arena, io->init, io->len, c->stream));
        else if (io) RRB_CUDA(c, cudaMemcpyAsync(arena, io->p, io->len, cudaMemcpyHostToDevice, c->stream));
        rc = run_resident(c, B, arena, arena_len, h->rowmap);
        if (io && !rc) RRB_CUDA(c, cudaMemcpyAsync(io->p, arena, io->len, cudaMemcpyDeviceToHost, c->stream));
    }
    c->stats.host_ns = host_ns;
    return rc;
}

// Page-locked host memory for the paint batch arrays: the upload of the
// (often large) stroke outlines is then a DMA, and the buffers are reused.
struct PinnedAlloc : rrb_stroke::HostAlloc {
    void* alloc(size_t bytes) override {
        void* p = nullptr;
        return cudaHostAlloc(&p, std::max<size_t>(bytes, 1), cudaHostAllocDefault) == cudaSuccess ? p : nullptr;
    }
    void release(void* p) override {
        if (p) cudaFreeHost(p);
    }
};

int paint_batch(rrb_ctx* c, const rrb_path_batch_params* p, const rrb_stroke_params* sp, const uint8_t* path_rgb,
                const double* clip_rects) {
    const auto t0 = std::chrono::steady_clock::now();
    std::string msg;
    if (!c->paint) c->paint = new rrb_stroke::PaintBatch();
    rrb_stroke::PaintBatch& pb = *c->paint;
    PinnedAlloc alloc;
    int rc = rrb_stroke::build(p, sp, path_rgb, clip_rects, alloc, pb, msg);
    if (rc) return set_err(c, rc, msg);
    if (pb.n_paths == 0) return RRB_OK;
    rrb_path_batch_params q = *p;
    q.pts = pb.pts.p;
    q.flags = pb.flags.p;
    q.n_pts = pb.n_pts;
    q.path_pt_off = pb.off.p;
    q.fill_rule = pb.rule.p;
    q.gray = pb.gray.p;
    q.alpha = pb.alpha.p;
    q.path_page = pb.page.p;
    q.n_paths = pb.n_paths;
    return run_batch(c, &q, static_cast<uint8_t*>(p->pages->p), p->pages->len, path_rgb ? pb.rgb.p : nullptr,
                     clip_rects ? pb.clip.p : nullptr, true, false, &t0);
}

}  // namespace

// Library-internal hooks for the other translation units (C++ linkage, not
// part of the C ABI): the context's device, whether a page is open, and its
// last error message.
int rrb_ctx_device(const rrb_ctx* c) { return c->device; }
bool rrb_ctx_page_open(const rrb_ctx* c) { return c->in_page; }
int rrb_ctx_fail(rrb_ctx* c, int code, const char* msg) { return set_err(c, code, msg); }
int rrb_ctx_sm_count(const rrb_ctx* c) { return c->sm_count; }
// Scratch slot k (0..7) of the fill operators, grown to at least `bytes`
// within the context's memory budget; contents are not kept across growth.
int rrb_ctx_fill_scratch(rrb_ctx* c, int k, size_t bytes, void** out) {
    if (k < 0 || k >= 8) return set_err(c, RRB_ERR_INVARIANT, "fill scratch slot out of range");
    int rc = ensure(c, c->s_fill[k], bytes);
    if (rc) return rc;
    *out = c->s_fill[k].p;
    return RRB_OK;
}

extern "C" {

const char* rrb_version(void) { return "rrb 0.1 sm_100a"; }

const char* rrb_status_name(int s) {
    switch (s) {
        case RRB_OK: return "ok";
        case RRB_ERR_ZERO_SIZE_ALLOC: return "ZeroSizeAlloc";
        case RRB_ERR_UNALIGNED_FILL: return "UnalignedFill";
        case RRB_ERR_POOL_EXHAUSTED: return "PoolExhausted";
        case RRB_ERR_INVARIANT: return "InvariantViolation";
        case RRB_ERR_OTHER: return "Other";
        case RRB_ERR_TIMEOUT: return "Timeout";
        case RRB_ERR_DEVICE: return "DeviceError";
        case RRB_ERR_OUT_OF_MEMORY: return "OutOfMemory";
        case RRB_ERR_STATE: return "StateError";
        default: return "unknown";
    }
}

int rrb_init(int device, uint64_t mem_budget_bytes, rrb_ctx** out) {
    if (!out) return RRB_ERR_INVARIANT;
    *out = nullptr;
    rrb_ctx* c = new rrb_ctx();
    c->device = device;
    c->budget = mem_budget_bytes;
    const rrb_host::DeviceScope dev_scope(device);
    cudaError_t e = dev_scope.status();
    if (e != cudaSuccess) {
        delete c;
        return RRB_ERR_DEVICE;
    }
    int sm = 0;
    if (cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, device) == cudaSuccess && sm > 0)
        c->sm_count = sm;
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        return RRB_ERR_DEVICE;
    }
    e = cudaMallocHost(reinterpret_cast<void**>(&c->h_read), 4096);
    if (e != cudaSuccess) {
        cudaStreamDestroy(c->stream);
        delete c;
        return RRB_ERR_DEVICE;
    }
    c->tmp_batch = new rrb_batch();
    c->wave_batch = new rrb_batch();
    preload_trial_kernels();
    c->tuning.tile_w = 64;
    c->tuning.tile_h = 16;
    c->tuning.rows_per_chunk = 32;
    c->tuning.auto_tile = 1;
    *out = c;
    return RRB_OK;
}

int rrb_destroy(rrb_ctx* c) {
    if (!c) return RRB_OK;
    const rrb_host::DeviceScope dev_scope(c->device);
    cudaStreamSynchronize(c->stream);
    Scratch* all[] = {&c->s_pts, &c->s_flags, &c->s_off, &c->s_rule, &c->s_gray, &c->s_alpha, &c->s_page,
                      &c->s_geom, &c->s_pw, &c->s_ph, &c->s_mtx, &c->s_pieces, &c->s_clip, &c->s_edge_off,
                      &c->s_edges, &c->s_info, &c->s_rows, &c->s_chunks, &c->s_super_cnt, &c->s_super_list, &c->s_super_start, &c->s_big, &c->s_lanes,
                      &c->s_row_idx, &c->s_spans, &c->s_ovf, &c->s_scratch, &c->s_ctr, &c->s_block, &c->s_stats,
                      &c->s_groups, &c->s_slots, &c->s_path_pieces, &c->s_ovf2, &c->s_run_off, &c->s_runs,
                      &c->s_chunk_path, &c->s_clip_lo};
    for (Scratch* s : all) dev_free(c, s->p, s->cap);
    for (Scratch& s : c->s_fill) dev_free(c, s.p, s.cap);
    for (cudaEvent_t e : c->trial_ev)
        if (e) cudaEventDestroy(e);
    if (c->tmp_batch) {
        free_batch_bufs(c, c->tmp_batch);
        delete c->tmp_batch;
    }
    if (c->wave_batch) {
        free_batch_bufs(c, c->wave_batch);
        delete c->wave_batch;
    }
    if (c->timer) {
        for (int w = 0; w < kTimedWaves; ++w)
            for (int k = 0; k < kStages; ++k) {
                cudaEventDestroy(c->timer->begin[w][k]);
                cudaEventDestroy(c->timer->end[w][k]);
            }
        delete c->timer;
    }
    if (c->h_waves) cudaFreeHost(c->h_waves);
    if (c->h_geom) cudaFreeHost(c->h_geom);
    if (c->paint) {
        PinnedAlloc alloc;
        c->paint->release(alloc);
        delete c->paint;
    }
    for (auto& kv : c->fences) cudaEventDestroy(kv.second);
    for (cudaEvent_t ev : c->free_events) cudaEventDestroy(ev);
    if (c->h_read) cudaFreeHost(c->h_read);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    if (c->down_stream) cudaStreamDestroy(c->down_stream);
    cudaStreamDestroy(c->stream);
    delete c;
    return RRB_OK;
}

const char* rrb_last_error_message(const rrb_ctx* c) { return c ? c->err.c_str() : "no context"; }

int rrb_alloc_device(rrb_ctx* c, size_t size, rrb_buf** out) {
    if (!c || !out) return RRB_ERR_INVARIANT;
    if (size == 0) return set_err(c, RRB_ERR_ZERO_SIZE_ALLOC, "alloc_device called with size = 0");
    const rrb_host::DeviceScope dev_scope(c->device);
    void* p = nullptr;
    int rc = dev_alloc(c, size, &p);
    if (rc) return rc;
    *out = new rrb_buf{p, size};
    return RRB_OK;
}

int rrb_alloc_device_zeroed(rrb_ctx* c, size_t size, rrb_buf** out) {
    if (!c || !out) return RRB_ERR_INVARIANT;
    const rrb_host::DeviceScope dev_scope(c->device);
    if (size == 0) return set_err(c, RRB_ERR_ZERO_SIZE_ALLOC, "alloc_device_zeroed called with size = 0");
    int rc = rrb_alloc_device(c, size, out);
    if (rc) return rc;
    RRB_CUDA(c, cudaMemsetAsync((*out)->p, 0, size, c->stream));
    RRB_CUDA(c, cudaStreamSynchronize(c->stream));
    return RRB_OK;
}

size_t rrb_device_buffer_len(const rrb_buf* b) { return b ? b->len : 0; }
void* rrb_device_ptr(const rrb_buf* b) { return b ? b->p : nullptr; }

int rrb_free_device(rrb_ctx* c, rrb_buf* b) {
    if (!c || !b) return RRB_ERR_INVARIANT;
    const rrb_host::DeviceScope dev_scope(c->device);
    cudaStreamSynchronize(c->stream);
    dev_free(c, b->p, b->len);
    delete b;
    return RRB_OK;
}

int rrb_alloc_host_pinned(rrb_ctx* c, size_t size, rrb_host_buf** out) {
    if (!c || !out) return RRB_ERR_INVARIANT;
    const rrb_host::DeviceScope dev_scope(c->device);
    if (size == 0) return set_err(c, RRB_ERR_ZERO_SIZE_ALLOC, "alloc_host_pinned called with size = 0");
    void* p = nullptr;
    RRB_CUDA(c, cudaMallocHost(&p, size));
    *out = new rrb_host_buf{p, size};
    return RRB_OK;
}

void* rrb_host_ptr(const rrb_host_buf* b) { return b ? b->p : nullptr; }

int rrb_free_host_pinned(rrb_ctx* c, rrb_host_buf* b) {
    if (!c || !b) return RRB_ERR_INVARIANT;
    const rrb_host::DeviceScope dev_scope(c->device);
    cudaStreamSynchronize(c->stream);
    cudaFreeHost(b->p);
    delete b;
    return RRB_OK;
}

static int record_fence(rrb_ctx* c, rrb_fence* out) {
    cudaEvent_t ev;
    if (!c->free_events.empty()) {
        ev = c->free_events.back();
        c->free_events.pop_back();
    } else {
        RRB_CUDA(c, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    }
    RRB_CUDA(c, cudaEventRecord(ev, c->stream));
    uint64_t id = c->next_fence++;
    c->fences[id] = ev;
    if (out) *out = id;
    return RRB_OK;
}

static int wait_fence(rrb_ctx* c, rrb_fence f, uint64_t timeout_ns) {
    auto it = c->fences.find(f);
    if (it == c->fences.end()) return set_err(c, RRB_ERR_INVARIANT, "unknown fence");
    cudaEvent_t ev = it->second;
    auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        cudaError_t e = cudaEventQuery(ev);
        if (e == cudaSuccess) break;
        if (e != cudaErrorNotReady) return cuda_err(c, e, "cudaEventQuery");
        if (timeout_ns) {
            auto dt = std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0);
            if (static_cast<uint64_t>(dt.count()) > timeout_ns)
                return set_err(c, RRB_ERR_TIMEOUT, "fence not signalled within timeout");
        }
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
    c->fences.erase(it);
    c->free_events.push_back(ev);
    return RRB_OK;
}

int rrb_upload_async(rrb_ctx* c, const rrb_buf* dst, size_t off, const void* src, size_t len, rrb_fence* out) {
    if (!c || !dst || (!src && len)) return RRB_ERR_INVARIANT;
    if (off > dst->len || len > dst->len - off)
        return set_err(c, RRB_ERR_INVARIANT, "upload exceeds the device buffer");
    const rrb_host::DeviceScope dev_scope(c->device);
    if (len) RRB_CUDA(c, cudaMemcpyAsync(static_cast<char*>(dst->p) + off, src, len, cudaMemcpyHostToDevice, c->stream));
    return record_fence(c, out);
}

int rrb_download_async(rrb_ctx* c, const rrb_buf* src, size_t off, void* dst, size_t len, rrb_fence* out) {
    if (!c || !src || (!dst && len)) return RRB_ERR_INVARIANT;
    if (off > src->len || len > src->len - off)
        return set_err(c, RRB_ERR_INVARIANT, "download exceeds the device buffer");
    const rrb_host::DeviceScope dev_scope(c->device);
    if (len) RRB_CUDA(c, cudaMemcpyAsync(dst, static_cast<const char*>(src->p) + off, len, cudaMemcpyDeviceToHost, c->stream));
    return record_fence(c, out);
}

int rrb_wait_download(rrb_ctx* c, rrb_fence f) { return c ? wait_fence(c, f, 0) : RRB_ERR_INVARIANT; }
int rrb_submit_transfer(rrb_ctx* c, rrb_fence* out) { return c ? record_fence(c, out) : RRB_ERR_INVARIANT; }
int rrb_wait_transfer(rrb_ctx* c, rrb_fence f, uint64_t t) { return c ? wait_fence(c, f, t) : RRB_ERR_INVARIANT; }

int rrb_detect_vram_budget(rrb_ctx* c, rrb_vram_budget* out) {
    if (!c || !out) return RRB_ERR_INVARIANT;
    const rrb_host::DeviceScope dev_scope(c->device);
    size_t fr = 0, tot = 0;
    RRB_CUDA(c, cudaMemGetInfo(&fr, &tot));
    out->total_bytes = tot;
    out->free_bytes = fr;
    out->budget_bytes = c->budget;
    out->used_bytes = c->used;
    return RRB_OK;
}

int rrb_begin_page(rrb_ctx* c) {
    if (!c) return RRB_ERR_INVARIANT;
    if (c->in_page) return set_err(c, RRB_ERR_STATE, "begin_page while a page is open");
    c->in_page = true;
    return RRB_OK;
}

int rrb_record_zero_buffer(rrb_ctx* c, const rrb_buf* b) {
    if (!c || !b) return RRB_ERR_INVARIANT;
    const rrb_host::DeviceScope dev_scope(c->device);
    if (!c->in_page) return set_err(c, RRB_ERR_STATE, "record_* outside begin_page/submit_page");
    RRB_CUDA(c, cudaMemsetAsync(b->p, 0, b->len, c->stream));
    return RRB_OK;
}

int rrb_submit_page(rrb_ctx* c, rrb_fence* out) {
    if (!c) return RRB_ERR_INVARIANT;
    if (!c->in_page) return set_err(c, RRB_ERR_STATE, "submit_page without begin_page");
    c->in_page = false;
    return record_fence(c, out);
}

int rrb_wait_page(rrb_ctx* c, rrb_fence f, uint64_t timeout_ns) {
    return c ? wait_fence(c, f, timeout_ns) : RRB_ERR_INVARIANT;
}

int rrb_set_tuning(rrb_ctx* c, const rrb_tuning* t) {
    if (!c || !t) return RRB_ERR_INVARIANT;
    uint32_t w = t->tile_w ? t->tile_w : c->tuning.tile_w, h = t->tile_h ? t->tile_h : c->tuning.tile_h;
    if (!valid_tile(w, h)) return set_err(c, RRB_ERR_INVARIANT, "tile shape must be 16x16, 32x32, 64x16, 128x16 or 128x32");
    if (t->auto_tile > 2) return set_err(c, RRB_ERR_INVARIANT, "auto_tile must be 0, 1 or 2");
    c->tuning.tile_w = w;
    c->tuning.tile_h = h;
    if (t->auto_tile) c->tuning.auto_tile = t->auto_tile;
    else if (t->tile_w || t->tile_h) c->tuning.auto_tile = 2;  // an explicit tile shape
    if (t->wave_points != 0xFFFFFFFFu) c->tuning.wave_points = t->wave_points;  // all ones: keep
    ++c->tuning_epoch;
    c->settled_tw = c->settled_th = 0;
    return RRB_OK;
}

int rrb_get_tuning(rrb_ctx* c, rrb_tuning* t) {
    if (!c || !t) return RRB_ERR_INVARIANT;
    *t = c->tuning;
    return RRB_OK;
}

int rrb_last_batch_stats(rrb_ctx* c, rrb_batch_stats* out) {
    if (!c || !out) return RRB_ERR_INVARIANT;
    *out = c->stats;
    return RRB_OK;
}

int rrb_record_path_batch(rrb_ctx* c, const rrb_path_batch_params* p) {
    if (!c || !p) return RRB_ERR_INVARIANT;
    if (!c->in_page) return set_err(c, RRB_ERR_STATE, "record_* outside begin_page/submit_page");
    if (!p->pages) return set_err(c, RRB_ERR_INVARIANT, "pages buffer is null");
    const rrb_host::DeviceScope dev_scope(c->device);
    return run_batch(c, p, static_cast<uint8_t*>(p->pages->p), p->pages->len);
}

int rrb_validate_path_batch(const rrb_path_batch_params* p, size_t pages_len, char* msg, size_t msg_len) {
    if (!p) return RRB_ERR_INVARIANT;
    std::vector<PageGeom> geom;
    uint64_t tiles = 0, supers = 0;
    std::string m;
    int rc = validate_batch(p, pages_len, 64, 16, geom, tiles, supers, m);
    if (msg && msg_len) {
        std::snprintf(msg, msg_len, "%s", m.c_str());
    }
    return rc;
}

int rrb_record_path_fill(rrb_ctx* c, const rrb_path_fill_params* p) {
    if (!c || !p) return RRB_ERR_INVARIANT;
    if (!p->page) return set_err(c, RRB_ERR_INVARIANT, "page buffer is null");
    if (p->n_pts && (!p->pts || !p->flags)) return set_err(c, RRB_ERR_INVARIANT, "null path arrays");
    if (p->fill_rule > 1) return set_err(c, RRB_ERR_INVARIANT, "fill_rule must be 0 or 1");
    rrb_path_batch_params b;
    std::memset(&b, 0, sizeof b);
    uint64_t off[2] = {0, p->n_pts};
    uint32_t page = 0, w = p->width, h = p->height;
    uint64_t po = p->page_offset;
    b.pts = p->pts;
    b.flags = p->flags;
    b.n_pts = p->n_pts;
    b.path_pt_off = off;
    b.fill_rule = &p->fill_rule;
    b.gray = &p->gray;
    b.alpha = &p->alpha;
    b.path_page = &page;
    b.n_paths = p->n_pts ? 1 : 0;
    b.page_width = &w;
    b.page_height = &h;
    b.page_offset = &po;
    b.n_pages = 1;
    b.pages = p->page;
    std::memcpy(b.matrix, p->matrix, sizeof b.matrix);
    b.flatness = p->flatness;
    b.rowmap = p->rowmap;
    return rrb_record_path_batch(c, &b);
}

int rrb_batch_upload(rrb_ctx* c, const rrb_path_batch_params* p, rrb_batch** out) {
    if (!c || !p || !out) return RRB_ERR_INVARIANT;
    const rrb_host::DeviceScope dev_scope(c->device);
    rrb_batch* B = new rrb_batch();
    int rc = batch_upload(c, p, B);
    if (rc) {
        free_batch_bufs(c, B);
        delete B;
        return rc;
    }
    RRB_CUDA(c, cudaStreamSynchronize(c->stream));
    *out = B;
    return RRB_OK;
}

int rrb_record_batch(rrb_ctx* c, rrb_batch* B, const rrb_buf* pages, int rowmap) {
    if (!c || !B || !pages) return RRB_ERR_INVARIANT;
    if (!c->in_page) return set_err(c, RRB_ERR_STATE, "record_* outside begin_page/submit_page");
    const rrb_host::DeviceScope dev_scope(c->device);
    return run_resident(c, B, static_cast<uint8_t*>(pages->p), pages->len, rowmap);
}

int rrb_batch_free(rrb_ctx* c, rrb_batch* B) {
    if (!c || !B) return RRB_ERR_INVARIANT;
    const rrb_host::DeviceScope dev_scope(c->device);
    cudaStreamSynchronize(c->stream);
    free_batch_bufs(c, B);
    delete B;
    return RRB_OK;
}

int rrb_record_fill_buffer(rrb_ctx* c, const rrb_buf* b, size_t off, size_t len, uint8_t value) {
    if (!c || !b) return RRB_ERR_INVARIANT;
    const rrb_host::DeviceScope dev_scope(c->device);
    if (!c->in_page) return set_err(c, RRB_ERR_STATE, "record_* outside begin_page/submit_page");
    if (off > b->len || len > b->len - off) return set_err(c, RRB_ERR_INVARIANT, "fill exceeds the device buffer");
    RRB_CUDA(c, cudaMemsetAsync(static_cast<char*>(b->p) + off, value, len, c->stream));
    return RRB_OK;
}

void* rrb_stream(rrb_ctx* c) { return c ? static_cast<void*>(c->stream) : nullptr; }

int rrb_set_profiling(rrb_ctx* c, int enable) {
    if (!c) return RRB_ERR_INVARIANT;
    const rrb_host::DeviceScope dev_scope(c->device);
    if (!c->timer) {
        c->timer = new StageTimer();
        for (int w = 0; w < kTimedWaves; ++w)
            for (int k = 0; k < kStages; ++k) {
                RRB_CUDA(c, cudaEventCreate(&c->timer->begin[w][k]));
                RRB_CUDA(c, cudaEventCreate(&c->timer->end[w][k]));
            }
    }
    c->timer->on = enable != 0;
    return RRB_OK;
}

int rrb_last_stage_times(rrb_ctx* c, rrb_stage_time* out, int cap, int* n) {
    if (!c || !n) return RRB_ERR_INVARIANT;
    int m = 0;
    for (int k = 0; k < kStages; ++k) {
        if (m < cap && out) {
            std::snprintf(out[m].name, sizeof out[m].name, "%s", kStageNames[k]);
            out[m].ms = c->stage_ms[k];
            out[m].launches = c->stage_launches[k];
        }
        ++m;
    }
    *n = m;
    return RRB_OK;
}

int rrb_record_stroke_batch(rrb_ctx* c, const rrb_path_batch_params* p, const rrb_stroke_params* stroke,
                            const uint8_t* path_rgb, const double* clip_rects) {
    if (!c || !p) return RRB_ERR_INVARIANT;
    if (!c->in_page) return set_err(c, RRB_ERR_STATE, "record_* outside begin_page/submit_page");
    if (!p->pages) return set_err(c, RRB_ERR_INVARIANT, "pages buffer is null");
    if (p->n_paths && !stroke) return set_err(c, RRB_ERR_INVARIANT, "stroke params array is null");
    const rrb_host::DeviceScope dev_scope(c->device);
    {
        std::vector<PageGeom> geom;
        uint64_t tiles = 0, supers = 0;
        std::string m;
        int v = validate_batch(p, p->pages->len, 64, 16, geom, tiles, supers, m, path_rgb ? 3 : 1);
        if (v) return set_err(c, v, m);
        if (clip_rects)
            for (uint64_t k = 0; k < 4 * p->n_paths; ++k)
                if (!std::isfinite(clip_rects[k])) return set_err(c, RRB_ERR_INVARIANT, "clip rectangles must be finite");
    }
    if (p->n_paths == 0) return RRB_OK;
    return paint_batch(c, p, stroke, path_rgb, clip_rects);
}

int rrb_record_path_batch_ex(rrb_ctx* c, const rrb_path_batch_params* p, const uint8_t* path_rgb,
                             const double* clip_rects) {
    return rrb_record_path_batch_visit(c, p, path_rgb, clip_rects, nullptr);
}

int rrb_record_path_batch_visit(rrb_ctx* c, const rrb_path_batch_params* p, const uint8_t* path_rgb,
                                const double* clip_rects, const int32_t* visit_rows) {
    if (!c || !p) return RRB_ERR_INVARIANT;
    if (!c->in_page) return set_err(c, RRB_ERR_STATE, "record_* outside begin_page/submit_page");
    if (!p->pages) return set_err(c, RRB_ERR_INVARIANT, "pages buffer is null");
    const rrb_host::DeviceScope dev_scope(c->device);
    {
        std::vector<PageGeom> geom;
        uint64_t tiles = 0, supers = 0;
        std::string m;
        int v = validate_batch(p, p->pages->len, 64, 16, geom, tiles, supers, m, path_rgb ? 3 : 1);
        if (v) return set_err(c, v, m);
    }
    static const uint8_t kNone[3] = {0, 0, 0};
    const uint8_t* rgb = path_rgb ? (p->n_paths ? path_rgb : kNone) : nullptr;
    return run_batch(c, p, static_cast<uint8_t*>(p->pages->p), p->pages->len, rgb, p->n_paths ? clip_rects : nullptr,
                     false, true, nullptr, p->n_paths ? visit_rows : nullptr);
}

int rrb_record_path_batch_rgb(rrb_ctx* c, const rrb_path_batch_params* p, const uint8_t* path_rgb) {
    if (c && p && p->n_paths && !path_rgb) return set_err(c, RRB_ERR_INVARIANT, "path_rgb is null");
    static const uint8_t kNone[3] = {0, 0, 0};
    return rrb_record_path_batch_ex(c, p, path_rgb ? path_rgb : kNone, nullptr);
}

int rrb_record_rgb_to_gray(rrb_ctx* c, const rrb_buf* rgb, size_t rgb_offset, const rrb_buf* gray,
                           size_t gray_offset, uint64_t n_px) {
    if (!c || !rgb || !gray) return RRB_ERR_INVARIANT;
    if (!c->in_page) return set_err(c, RRB_ERR_STATE, "record_* outside begin_page/submit_page");
    if (rgb_offset > rgb->len || n_px > (rgb->len - rgb_offset) / 3 || gray_offset > gray->len ||
        n_px > gray->len - gray_offset)
        return set_err(c, RRB_ERR_INVARIANT, "rgb_to_gray range past a buffer");
    if (!n_px) return RRB_OK;
    const rrb_host::DeviceScope dev_scope(c->device);
    k_rgb_to_gray<<<grid_for(c, n_px, 256), 256, 0, c->stream>>>(static_cast<const uint8_t*>(rgb->p) + rgb_offset,
                                                                static_cast<uint8_t*>(gray->p) + gray_offset, n_px);
    RRB_CUDA(c, cudaGetLastError());
    return RRB_OK;
}

namespace {
int render_pages_host(rrb_ctx* c, const rrb_path_batch_params* p, uint8_t* host_pages, size_t len, int init) {
    if (!c || !p || !host_pages || !p->pages) return RRB_ERR_INVARIANT;
    if (len > p->pages->len) return set_err(c, RRB_ERR_INVARIANT, "host pages larger than the device arena");
    if (init > 255) return set_err(c, RRB_ERR_INVARIANT, "init_value must be 0..255");
    const rrb_host::DeviceScope dev_scope(c->device);
    int rc = rrb_begin_page(c);
    if (rc) return rc;
    // The pages travel inside the render: overlapped with it when the batch
    // streams (page-locked points), before and after it otherwise.
    const HostPages io{host_pages, len, init < 0 ? -1 : init};
    rc = run_batch(c, p, static_cast<uint8_t*>(p->pages->p), p->pages->len, nullptr, nullptr, false, true, nullptr,
                   nullptr, &io);
    rrb_fence f = 0;
    int rc2 = rrb_submit_page(c, &f);
    if (rc) return rc;
    if (rc2) return rc2;
    return rrb_wait_page(c, f, 0) ? RRB_ERR_DEVICE : (cudaStreamSynchronize(c->stream) == cudaSuccess ? RRB_OK : RRB_ERR_DEVICE);
}
}  // namespace

int rrb_render_pages_host(rrb_ctx* c, const rrb_path_batch_params* p, uint8_t* host_pages, size_t len) {
    return render_pages_host(c, p, host_pages, len, -1);
}

int rrb_render_pages_host_init(rrb_ctx* c, const rrb_path_batch_params* p, uint8_t* host_pages, size_t len,
                               int init_value) {
    if (init_value < 0) return c ? set_err(c, RRB_ERR_INVARIANT, "init_value must be 0..255") : RRB_ERR_INVARIANT;
    return render_pages_host(c, p, host_pages, len, init_value);
}

}  // extern "C"
