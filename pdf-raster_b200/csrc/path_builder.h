// path_builder.h — the object behind the opaque rrb_path handle of
// path_builder.cpp, shared with the scene generator (scenes/scene_gen.cpp),
// which builds its paths through the same functions.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

struct rrb_path {
    std::vector<double> pts;
    std::vector<uint8_t> flags;
    size_t cur_subpath = 0;
    size_t len() const { return flags.size(); }
    bool no_current_point() const { return cur_subpath == len(); }
    bool one_point_subpath() const { return len() != 0 && cur_subpath == len() - 1; }
};
