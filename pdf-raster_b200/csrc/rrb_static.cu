// rrb_static.cu — rrb_record_path_fill_static: the single-path AA fill of
// rrb_record_path_fill with every intermediate in one statically reserved
// device array, so that a call allocates no device memory at all.
//
// Who needs it: a renderer that cannot allocate device memory while it draws.
// cudaMalloc / cudaFree synchronise the whole device (cudaFree waits for all
// work on it), so a page thread on a busy serving GPU that allocated per path
// would stall every other stream; a process whose device memory is handed out
// up front by an external pool, or whose admission control has already
// granted its budget, must not meet an out-of-memory error in the middle of a
// page. This entry point draws from a fixed array instead; its limits are
// the array's partition below, and paths beyond them are rejected up front
// or, for limits only known on the device, before any pixel is written.
//
// The array lives in this file's own device module, so it is reserved only in
// processes that call this entry point (when the module loads), not in every
// process that uses the library.
//
// Pipeline (one path, all on the context's stream): the subpath walk, piece
// compaction, flatten counts and edge records of the batched pipeline (the
// same kernels), then k_static_rows — one warp per pixel row, the merged
// crossings of its four AA rows in shared memory, sort, winding walk and
// coverage cells into the array — and k_static_blend, which applies the cells
// to the page only when no limit was hit.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/rrb.h"
#include "rrb_device_scope.h"

// The pipeline's kernels with internal linkage in this translation unit: this
// module carries its own copies, so it can load apart from the main one.
namespace {
#include "rrb_kernels.cuh"
}  // namespace

// Library-internal hooks into the context, defined with the context.
int rrb_ctx_device(const rrb_ctx* c);
bool rrb_ctx_page_open(const rrb_ctx* c);
int rrb_ctx_fail(rrb_ctx* c, int code, const char* msg);

namespace {

using namespace rrb;

constexpr uint32_t kMaxPoints = RRB_STATIC_MAX_POINTS;
constexpr uint32_t kMaxEdges = RRB_STATIC_MAX_EDGES;
constexpr int kRowK = RRB_STATIC_MAX_ROW_CROSSINGS;
constexpr size_t kBytes = RRB_STATIC_SCRATCH_BYTES;

// Per-call parameters and small results; the whole struct is uploaded at the
// start of every call, which also zeroes the counters.
struct StaticHeader {
    PathInfo info;
    BatchCounters ctr;
    double mtx[6];
    uint64_t off[2];
    uint32_t page, pw, ph, pad0;
    uint8_t rule, gray, alpha, pad1[5];
    uint32_t path_pieces[2];
    uint32_t rows[2], chunks[2];
    uint32_t block[SCAN_MAX_BLOCKS + 1];
};

constexpr size_t up256(size_t x) { return (x + 255) & ~size_t(255); }

// Partition of the array (byte offsets, each 256-byte aligned).
constexpr size_t kOffHdr = 0;
constexpr size_t kOffPts = up256(kOffHdr + sizeof(StaticHeader));
constexpr size_t kOffFlags = up256(kOffPts + 16ull * kMaxPoints);
constexpr size_t kOffSlots = up256(kOffFlags + kMaxPoints);
constexpr size_t kOffPieces = up256(kOffSlots + 8ull * kMaxPoints);
constexpr size_t kOffClip = up256(kOffPieces + 8ull * kMaxPoints);
constexpr size_t kOffEdgeOff = up256(kOffClip + 4ull * kMaxPoints);
constexpr size_t kOffEdges = up256(kOffEdgeOff + 4ull * (kMaxPoints + 1));
constexpr uint32_t kGroups = kMaxEdges / 32 + 1;
constexpr size_t kOffGmin = up256(kOffEdges + sizeof(Edge) * kMaxEdges);
constexpr size_t kOffGmax = up256(kOffGmin + 4ull * kGroups);
constexpr size_t kOffCells = up256(kOffGmax + 4ull * kGroups);
constexpr uint32_t kMaxCells = static_cast<uint32_t>((kBytes - kOffCells) / sizeof(uint2));
static_assert(kOffCells < kBytes && kMaxCells >= (1u << 20), "scratch partition");
static_assert(kMaxCells == RRB_STATIC_MAX_CELLS, "RRB_STATIC_MAX_CELLS must match the partition");
static_assert(kRowK <= 1024, "row lists live in shared memory");

// The scratch array. Every call uses all of it, from one call to the next.
static __device__ __align__(256) unsigned char g_fill_scratch[kBytes];

constexpr int kMaxDevices = 64;
struct DeviceScratch {
    unsigned char* base = nullptr;
    int sm_count = 0;
};
std::mutex g_lock;                     // held for a whole call: one call at a time per process
DeviceScratch g_dev[kMaxDevices];

// Set-up, once per device, with that device current: the array's device
// address (this also loads the module that holds it) and the SM count.
int scratch_for(rrb_ctx* c, int device, DeviceScratch*& out) {
    if (device < 0 || device >= kMaxDevices) return rrb_ctx_fail(c, RRB_ERR_DEVICE, "device index out of range");
    DeviceScratch& d = g_dev[device];
    if (!d.base) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_fill_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return rrb_ctx_fail(c, RRB_ERR_DEVICE,
                                (std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e)).c_str());
        }
        int sm = 0;
        if (cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || sm <= 0) sm = 148;
        d.base = static_cast<unsigned char*>(p);
        d.sm_count = sm;
    }
    out = &d;
    return RRB_OK;
}

constexpr int kRowWarps = 4;

// One warp per pixel row of the path (rows under the row map, clipped to the
// page): lanes 0-3 gather, sort and walk the four AA sub-rows in shared
// memory; lane 0 merges their spans into coverage cells (row, cell) appended
// to `cells`. A sub-row with more than kRowK merged crossings sets
// ERR_ROW_CAP, a full cell array ERR_SPAN_CAP; either stops the blend.
__global__ void __launch_bounds__(kRowWarps * 32) k_static_rows(const PathInfo* __restrict__ info,
                                                                const Edge* __restrict__ edges,
                                                                const int32_t* __restrict__ gmin,
                                                                const int32_t* __restrict__ gmax, uint32_t page_w,
                                                                int rowmap, uint2* __restrict__ cells,
                                                                uint32_t cell_cap, BatchCounters* __restrict__ ctr) {
    __shared__ int32_t sx0[kRowWarps][kRowK * 4];
    __shared__ int32_t sx1[kRowWarps][kRowK * 4];
    __shared__ int32_t scn[kRowWarps][kRowK * 4];
    __shared__ Edge sedge[kRowWarps][32];
    __shared__ int32_t sns[kRowWarps][4];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const PathInfo P = info[0];
    if (P.y0 > P.y1 || P.py0 > P.py1) return;
    const int32_t g_lo = P.y0 >> 2, g_hi = P.y1 >> 2;
    const int32_t mask = (P.paint >> 16) & 1 ? 1 : ~0;
    const int32_t aa_width = 4 * static_cast<int32_t>(page_w);
    uint32_t nonterm = 0;
    for (int32_t y = P.py0 + static_cast<int32_t>(blockIdx.x * kRowWarps + w); y <= P.py1;
         y += static_cast<int32_t>(gridDim.x * kRowWarps)) {
        const int32_t grp = rowmap ? 4 * y + 3 : y;
        if (grp < g_lo || grp > g_hi) continue;
        const int32_t lo = 4 * grp, hi = min(4 * grp + 3, P.y1);
        const int32_t r = lo + lane;
        const bool valid = lane < 4 && r >= P.y0 && r <= hi;
        const int n = gather_row<kRowK, 4>(P, lo, hi, r, valid, edges, gmin, gmax, sedge[w], sx0[w], sx1[w], scn[w],
                                           lane);
        const bool overflow = valid && n > kRowK;
        int ns = 0;
        if (valid && !overflow) ns = sort_and_walk<4>(n, mask, aa_width, 0, aa_width, sx0[w], sx1[w], scn[w], lane, nonterm);
        if (lane < 4) sns[w][lane] = (valid && !overflow) ? ns : 0;
        const bool any_ovf = __any_sync(0xffffffffu, overflow);
        __syncwarp();
        if (lane == 0) {
            if (any_ovf) {
                atomicOr(&ctr->err, ERR_ROW_CAP);
            } else {
                int n4[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) n4[q] = sns[w][q];
                auto bound = [&](int q, int i, bool end) { return end ? sx1[w][i * 4 + q] : sx0[w][i * 4 + q]; };
                const int nc = sweep_cells(n4, bound, [](int, uint32_t) {});
                const uint32_t o0 = nc ? atomicAdd(&ctr->cell_cursor, static_cast<uint32_t>(nc)) : 0u;
                if (static_cast<uint64_t>(o0) + static_cast<uint32_t>(nc) > cell_cap) {
                    atomicOr(&ctr->err, ERR_SPAN_CAP);
                } else if (nc) {
                    const uint32_t yy = static_cast<uint32_t>(y);
                    sweep_cells(n4, bound, [&](int q, uint32_t cell) { cells[o0 + q] = make_uint2(yy, cell); });
                }
            }
        }
        __syncwarp();
    }
    if (nonterm) atomicAdd(&ctr->nonterminating, nonterm);
}

// Applies the cells: AA_GAMMA of the coverage, then the div255 source-over of
// the solid gray (pipe/aa.rs:192-208), one thread per cell. Cells are
// disjoint, so every pixel has one writer. Does nothing if a limit was hit.
__global__ void k_static_blend(const PathInfo* __restrict__ info, const uint2* __restrict__ cells, uint32_t cell_cap,
                               const BatchCounters* __restrict__ ctr, uint8_t* __restrict__ page, uint32_t width) {
    if (ctr->err) return;
    const uint32_t n = min(ctr->cell_cursor, cell_cap);
    const uint32_t paint = info[0].paint;
    const uint32_t g = paint & 0xff, alpha = (paint >> 8) & 0xff;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint2 c = cells[i];
        const uint32_t x0 = c.y & 0x3fffu, len = ((c.y >> 14) & 0x3fffu) + 1, cov = (c.y >> 28) + 1;
        const uint32_t a_src = div255(alpha * static_cast<uint32_t>(c_gamma[cov]));
        uint8_t* row = page + static_cast<size_t>(c.x) * width;
        for (uint32_t x = x0; x < x0 + len; ++x) row[x] = static_cast<uint8_t>(div255((255u - a_src) * row[x] + a_src * g));
    }
}

#define RRB_STATIC_CUDA(ctx, call)                                                                     \
    do {                                                                                               \
        cudaError_t e__ = (call);                                                                      \
        if (e__ != cudaSuccess) {                                                                      \
            cudaGetLastError();                                                                        \
            return rrb_ctx_fail(ctx, RRB_ERR_DEVICE, (std::string(#call ": ") + cudaGetErrorString(e__)).c_str()); \
        }                                                                                              \
    } while (0)

// Exclusive scan of n u32 in place (d[n] = total), block sums in the header.
int scan_static(rrb_ctx* c, cudaStream_t s, uint32_t* d, uint32_t n, uint32_t* block) {
    const uint32_t nb0 = std::min<uint32_t>(SCAN_MAX_BLOCKS, std::max<uint32_t>(1, (n + 4095) / 4096));
    const uint32_t per = (n + nb0 - 1) / nb0;
    const uint32_t nb = (n + per - 1) / per;
    k_scan_reduce<<<nb, SCAN_THREADS, 0, s>>>(d, n, per, block);
    k_scan_blocks<<<1, 1024, 0, s>>>(block, nb);
    k_scan_down<<<nb, SCAN_THREADS, 0, s>>>(d, d, n, per, block);
    RRB_STATIC_CUDA(c, cudaGetLastError());
    return RRB_OK;
}

int read_u32(rrb_ctx* c, cudaStream_t s, const uint32_t* dev, uint32_t& out) {
    RRB_STATIC_CUDA(c, cudaMemcpyAsync(&out, dev, sizeof out, cudaMemcpyDeviceToHost, s));
    RRB_STATIC_CUDA(c, cudaStreamSynchronize(s));
    return RRB_OK;
}

int fill_static(rrb_ctx* c, const rrb_path_fill_params* p, unsigned char* base, int sm_count) {
    cudaStream_t s = static_cast<cudaStream_t>(rrb_stream(c));
    StaticHeader* hdr = reinterpret_cast<StaticHeader*>(base + kOffHdr);
    double* pts = reinterpret_cast<double*>(base + kOffPts);
    uint8_t* flags = base + kOffFlags;
    uint2* slots = reinterpret_cast<uint2*>(base + kOffSlots);
    uint2* pieces = reinterpret_cast<uint2*>(base + kOffPieces);
    uint32_t* clip = reinterpret_cast<uint32_t*>(base + kOffClip);
    uint32_t* edge_off = reinterpret_cast<uint32_t*>(base + kOffEdgeOff);
    Edge* edges = reinterpret_cast<Edge*>(base + kOffEdges);
    int32_t* gmin = reinterpret_cast<int32_t*>(base + kOffGmin);
    int32_t* gmax = reinterpret_cast<int32_t*>(base + kOffGmax);
    uint2* cells = reinterpret_cast<uint2*>(base + kOffCells);
    auto grid = [&](uint64_t n, int threads, int per_sm) {
        const uint64_t need = (n + threads - 1) / threads, cap = static_cast<uint64_t>(sm_count) * per_sm;
        return static_cast<int>(std::max<uint64_t>(1, std::min(need, cap)));
    };

    // Header: parameters, zeroed counters (cell cursor, error bits).
    StaticHeader h;
    std::memset(&h, 0, sizeof h);
    std::memcpy(h.mtx, p->matrix, sizeof h.mtx);
    h.off[0] = 0;
    h.off[1] = p->n_pts;
    h.page = 0;
    h.pw = p->width;
    h.ph = p->height;
    h.rule = p->fill_rule;
    h.gray = p->gray;
    h.alpha = p->alpha;
    RRB_STATIC_CUDA(c, cudaMemcpyAsync(hdr, &h, offsetof(StaticHeader, block), cudaMemcpyHostToDevice, s));
    RRB_STATIC_CUDA(c, cudaMemcpyAsync(pts, p->pts, 16ull * p->n_pts, cudaMemcpyHostToDevice, s));
    RRB_STATIC_CUDA(c, cudaMemcpyAsync(flags, p->flags, p->n_pts, cudaMemcpyHostToDevice, s));
    const double flat_sq = p->flatness * p->flatness;

    // Subpath walk -> pieces (at most one per point).
    k_walk<<<1, 32, 0, s>>>(pts, flags, hdr->off, 1, hdr->mtx, &hdr->page, &hdr->ph, slots, hdr->path_pieces,
                            nullptr);
    int rc;
    if ((rc = scan_static(c, s, hdr->path_pieces, 1, hdr->block))) return rc;
    uint32_t n_pieces = 0;
    if ((rc = read_u32(c, s, hdr->path_pieces + 1, n_pieces))) return rc;
    if (n_pieces == 0) return RRB_OK;
    k_compact_pieces<<<1, 32, 0, s>>>(hdr->off, hdr->path_pieces, 1, &hdr->page, &hdr->ph, slots, pieces, clip,
                                      nullptr, nullptr);
    k_seg_count<false><<<grid(n_pieces, 128, 32), 128, 0, s>>>(pts, pieces, n_pieces, hdr->mtx, flat_sq, edge_off,
                                                                nullptr, &hdr->ctr);
    if ((rc = scan_static(c, s, edge_off, n_pieces, hdr->block))) return rc;
    uint32_t n_edges = 0;
    if ((rc = read_u32(c, s, edge_off + n_pieces, n_edges))) return rc;
    if (n_edges > kMaxEdges) {
        char msg[160];
        std::snprintf(msg, sizeof msg,
                      "path flattens to %u edges; rrb_record_path_fill_static holds at most %u (page untouched)",
                      n_edges, kMaxEdges);
        return rrb_ctx_fail(c, RRB_ERR_POOL_EXHAUSTED, msg);
    }
    if (n_edges == 0) return RRB_OK;

    // Edge records, the path box and per-32-edge row bounds.
    const uint32_t groups = n_edges / 32 + 1;
    RRB_STATIC_CUDA(c, cudaMemsetAsync(gmin, 0x7f, groups * sizeof(int32_t), s));  // +inf rows
    RRB_STATIC_CUDA(c, cudaMemsetAsync(gmax, 0x80, groups * sizeof(int32_t), s));  // -inf rows
    k_seg_write<false><<<grid(n_pieces, 128, 32), 128, 0, s>>>(pts, pieces, n_pieces, hdr->mtx, flat_sq, edge_off, n_edges,
                                                         edges, clip, nullptr);
    k_path_bbox<<<1, 32, 0, s>>>(hdr->path_pieces, edge_off, edges, 1, &hdr->rule, &hdr->gray, &hdr->alpha,
                                 &hdr->page, &hdr->pw, &hdr->ph, p->rowmap, &hdr->info, hdr->rows, hdr->chunks, 32,
                                 &hdr->ctr, gmin, gmax, nullptr, nullptr);
    RRB_STATIC_CUDA(c, cudaGetLastError());

    // Rows -> cells, then the blend (skipped on the device if a limit was hit).
    const uint64_t pix_rows = p->height;  // an upper bound on the path's pixel rows
    k_static_rows<<<grid(pix_rows * 32, kRowWarps * 32, 8), kRowWarps * 32, 0, s>>>(
        &hdr->info, edges, gmin, gmax, p->width, p->rowmap, cells, kMaxCells, &hdr->ctr);
    uint8_t* page = static_cast<uint8_t*>(rrb_device_ptr(p->page)) + p->page_offset;
    k_static_blend<<<sm_count * 4, 256, 0, s>>>(&hdr->info, cells, kMaxCells, &hdr->ctr, page, p->width);
    RRB_STATIC_CUDA(c, cudaGetLastError());
    uint32_t err = 0;
    if ((rc = read_u32(c, s, &hdr->ctr.err, err))) return rc;
    if (err & ERR_ROW_CAP) {
        char msg[160];
        std::snprintf(msg, sizeof msg,
                      "an AA row of this path has more than %d merged crossings, the limit of "
                      "rrb_record_path_fill_static (page untouched)",
                      kRowK);
        return rrb_ctx_fail(c, RRB_ERR_POOL_EXHAUSTED, msg);
    }
    if (err) {
        char msg[160];
        std::snprintf(msg, sizeof msg,
                      "path needs more than %u coverage cells, the limit of rrb_record_path_fill_static "
                      "(page untouched)",
                      kMaxCells);
        return rrb_ctx_fail(c, RRB_ERR_POOL_EXHAUSTED, msg);
    }
    return RRB_OK;
}

}  // namespace

extern "C" int rrb_record_path_fill_static(rrb_ctx* c, const rrb_path_fill_params* p) {
    if (!c || !p) return RRB_ERR_INVARIANT;
    if (!rrb_ctx_page_open(c)) return rrb_ctx_fail(c, RRB_ERR_STATE, "record_* outside begin_page/submit_page");
    if (!p->page) return rrb_ctx_fail(c, RRB_ERR_INVARIANT, "page buffer is null");
    if (p->n_pts && (!p->pts || !p->flags)) return rrb_ctx_fail(c, RRB_ERR_INVARIANT, "null path arrays");
    if (p->fill_rule > 1) return rrb_ctx_fail(c, RRB_ERR_INVARIANT, "fill_rule must be 0 or 1");
    if (p->rowmap > 1) return rrb_ctx_fail(c, RRB_ERR_INVARIANT, "rowmap must be 0 or 1");
    if (!(p->flatness >= 0.0)) return rrb_ctx_fail(c, RRB_ERR_INVARIANT, "flatness must be >= 0");
    for (int i = 0; i < 6; ++i)
        if (!std::isfinite(p->matrix[i])) return rrb_ctx_fail(c, RRB_ERR_INVARIANT, "matrix must be finite");
    if (p->width == 0 || p->height == 0 || p->width > 16383 || p->height > (1u << 28))
        return rrb_ctx_fail(c, RRB_ERR_INVARIANT, "page width must be 1..16383 and height 1..2^28");
    const uint64_t page_len = rrb_device_buffer_len(p->page);
    if (p->page_offset > page_len || static_cast<uint64_t>(p->width) * p->height > page_len - p->page_offset)
        return rrb_ctx_fail(c, RRB_ERR_INVARIANT, "page extends past the page buffer");
    if (p->n_pts > kMaxPoints) {
        char msg[160];
        std::snprintf(msg, sizeof msg, "path has %u points; rrb_record_path_fill_static takes at most %u",
                      p->n_pts, kMaxPoints);
        return rrb_ctx_fail(c, RRB_ERR_POOL_EXHAUSTED, msg);
    }
    if (p->n_pts == 0) return RRB_OK;
    std::lock_guard<std::mutex> lk(g_lock);
    const int device = rrb_ctx_device(c);
    const rrb_host::DeviceScope dev_scope(device);
    RRB_STATIC_CUDA(c, dev_scope.status());
    DeviceScratch* d = nullptr;
    int rc = scratch_for(c, device, d);
    if (rc) return rc;
    return fill_static(c, p, d->base, d->sm_count);
}
