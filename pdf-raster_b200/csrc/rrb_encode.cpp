// rrb_encode.cpp — Netpbm output of rendered pages (the page output step of
// crates/encode: write_pgm for Gray8, pgm.rs, and write_ppm for Rgb8,
// ppm.rs): the header "P5\n{w} {h}\n255\n" or "P6\n{w} {h}\n255\n"
// followed by the rows' pixel bytes (row stride = width * channels).

#include <cstdio>
#include <cstring>

#include "../../include/rrb.h"

extern "C" int rrb_encode_netpbm(const uint8_t* pixels, uint32_t width, uint32_t height, uint32_t channels,
                                 uint8_t* out, size_t out_cap, size_t* out_len) {
    if (!out_len || (channels != 1 && channels != 3)) return RRB_ERR_INVARIANT;
    char head[64];
    const int n = std::snprintf(head, sizeof head, "P%c\n%u %u\n255\n", channels == 1 ? '5' : '6', width, height);
    if (n <= 0) return RRB_ERR_OTHER;
    const size_t body = static_cast<size_t>(width) * height * channels;
    *out_len = static_cast<size_t>(n) + body;
    if (!out) return RRB_OK;  // size query
    if (out_cap < *out_len) return RRB_ERR_INVARIANT;
    if (body && !pixels) return RRB_ERR_INVARIANT;
    std::memcpy(out, head, static_cast<size_t>(n));
    if (body) std::memcpy(out + n, pixels, body);
    return RRB_OK;
}
