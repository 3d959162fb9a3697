/* fill_oracle.h — CPU restatement of the reference's two GPU fill operators
 * (TEST INFRASTRUCTURE ONLY; the checker for rrb_record_aa_fill and
 * rrb_record_tile_fill).
 *
 *   or_aa_fill_cpu         aa_fill_cpu + aa_fill_cpu_sample
 *                          (crates/gpu/src/fill.rs:346-421): 64 Halton(2,3)
 *                          jittered samples per pixel, crossing-number winding.
 *   or_build_tile_records  build_tile_records (crates/gpu/src/fill.rs:82-264)
 *                          with a STABLE sort by key (the reference's
 *                          sort_unstable_by_key only pins the order of equal
 *                          keys for lists of at most 20 records).
 *   or_tile_fill           tile_fill (crates/gpu/kernels/tile_fill.cu:60-177)
 *                          as written, in IEEE f32 with every operation
 *                          rounded on its own. (The reference builds its
 *                          kernels with --use_fast_math: approximate division,
 *                          contraction and flush-to-zero, so its own bytes
 *                          are only within rounding of this restatement.)
 *
 * All arithmetic is f32 with no implicit contraction (-ffp-contract=off). */
#pragma once
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    uint32_t key; /* (tile_y << 16) | tile_x */
    float x_enter, dxdy, y0_tile, y1_tile, sign;
    uint32_t pad, pad2;
} or_tile_record;

/* The 64 (x, y) sample offsets, as f32. */
void or_aa_jitter(float* x64, float* y64);

void or_aa_fill_cpu(const float* segs, uint32_t n_segs, float x_min, float y_min, uint32_t width,
                    uint32_t height, int eo, uint8_t* out);

/* Records of every segment; returns the record count. With records == NULL
 * only counts. tile_starts / tile_counts (grid_w * grid_h entries each) may be
 * NULL. Returns -1 when the grid exceeds the 16-bit tile key range. */
int64_t or_build_tile_records(const float* segs, uint32_t n_segs, float x_min, float y_min, uint32_t width,
                              uint32_t height, or_tile_record* records, uint32_t* tile_starts,
                              uint32_t* tile_counts, uint32_t* grid_w);

void or_tile_fill(const or_tile_record* records, const uint32_t* tile_starts, const uint32_t* tile_counts,
                  uint32_t grid_w, uint32_t width, uint32_t height, int eo, uint8_t* coverage);

#ifdef __cplusplus
}
#endif
