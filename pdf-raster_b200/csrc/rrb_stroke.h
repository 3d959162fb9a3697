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

// Geometry of a paint batch: kind per path, and for outlines and hairlines
// their points at [off[p], off[p+1]) of xy (x, y pairs) / fl (path flags).
struct Plan {
    std::vector<uint8_t> kind;
    std::vector<uint64_t> off;
    std::vector<double> xy;
    std::vector<uint8_t> fl;
};

// Checks one path's stroke parameters (params.validate() style).
int check_params(const rrb_stroke_params& sp, std::string& msg);
// Strokes every path of p with sp[p] (host threads over chunks of paths).
int plan(const rrb_path_batch_params* p, const rrb_stroke_params* sp, Plan& out, std::string& msg);

}  // namespace rrb_stroke
