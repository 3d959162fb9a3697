// rrb_stroke.h — library-internal interface of the host stroker (rrb_stroke.cpp).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/rrb.h"

namespace rrb_stroke {

// What one path of a paint batch draws.
enum Kind : uint8_t {
    NOTHING = 0,   // nothing (empty path, all-gap dash, degenerate stroke)
    OUTLINE = 1,   // the stroke outline, filled nonzero with AA
    HAIRLINE = 2,  // a hairline polyline, drawn as one-pixel spans
    FILL = 3,      // not a stroke: the input path, filled with its own rule
};

// Internal fill-rule value of a hairline segment in a paint batch (the
// device pipeline's RULE_HAIRLINE).
constexpr uint8_t kRuleHairline = 2;

// Source of host memory for the batch arrays (the backend hands out
// page-locked memory, so the upload is a DMA).
struct HostAlloc {
    virtual void* alloc(size_t bytes) = 0;
    virtual void release(void* p) = 0;
    virtual ~HostAlloc() = default;
};

template <typename T>
struct HostArray {
    T* p = nullptr;
    size_t cap = 0;
    void reserve(HostAlloc& a, size_t n) {
        if (n <= cap) return;
        a.release(p);
        p = nullptr;
        cap = 0;
        p = static_cast<T*>(a.alloc(n * sizeof(T)));
        if (p) cap = n;
    }
    void release(HostAlloc& a) {
        a.release(p);
        p = nullptr;
        cap = 0;
    }
};

// Geometry a worker made for one chunk of consecutive paths (reused from
// call to call, so steady-state calls allocate nothing).
struct Chunk {
    std::vector<double> xy;       // outline / hairline points of the chunk's paths
    std::vector<uint8_t> fl;
    std::vector<uint8_t> kind;    // per path
    std::vector<uint64_t> len;    // per path: points in xy / fl
    std::vector<uint32_t> segs;   // per path: hairline segments
    uint64_t out_paths = 0, out_pts = 0;
};

// The batch the device renders for a paint batch: fills (the input paths),
// stroke outlines (rule nonzero) and hairline segments (two-point paths with
// rule kRuleHairline), in path order, with their paint, page and clip.
struct PaintBatch {
    HostArray<double> pts, clip;
    HostArray<uint8_t> flags, rule, gray, alpha, rgb;
    HostArray<uint64_t> off;
    HostArray<uint32_t> page;
    uint64_t n_paths = 0, n_pts = 0;
    std::vector<Chunk> chunks;
    void release(HostAlloc& a) {
        pts.release(a);
        clip.release(a);
        flags.release(a);
        rule.release(a);
        gray.release(a);
        alpha.release(a);
        rgb.release(a);
        off.release(a);
        page.release(a);
    }
};

// Checks one path's stroke parameters (params.validate() style).
int check_params(const rrb_stroke_params& sp, std::string& msg);
// Strokes every path of p with sp[p] and lays out the batch to render:
// host threads stroke chunks of paths, then write the chunks' output paths
// at their offsets. path_rgb / clip_rects (per input path, or null) are
// carried to the output paths.
int build(const rrb_path_batch_params* p, const rrb_stroke_params* sp, const uint8_t* path_rgb,
          const double* clip_rects, HostAlloc& alloc, PaintBatch& out, std::string& msg);

}  // namespace rrb_stroke
