/*
 * rrb_scenes.h — C ABI of librrb_scenes.so, the seeded synthetic workloads
 * of the benchmark and the tests.
 *
 * The generator is a library of its own, not part of the fill backend
 * (librrb.so): a process that only needs scenes, such as the CPU baseline
 * that times the reference's CPU path, never maps the backend. Paths are built
 * with the same PathBuilder restatement the backend exports (rrb_path_*,
 * crates/raster/src/path/mod.rs:310-448), compiled into this library too.
 */
#ifndef RRB_SCENES_H
#define RRB_SCENES_H

#include "rrb.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- seeded synthetic scenes (the benchmark workloads) ----------------------
 * kind 0: polygon page (2,000 paths of 1-3 contours x 4-32 line/cubic
 *         segments on jittered circles, NZ 70% / EO 30%, opaque);
 * kind 1: glyph-dense text page (150,000 quadratic glyphs on 60 baselines);
 * kind 2: mixed pages of uneven size (30% glyphs, 40% polygons, 30% rects,
 *         alpha 32-255). Zero fields take the defaults of each kind. */
typedef struct {
    uint32_t kind;
    uint64_t seed;
    uint32_t n_pages;      /* kind 2 (default 64); kinds 0/1 always 1 */
    uint32_t n_paths;      /* kinds 0/1: paths on the page; kind 2: 0 = log-normal count */
    uint32_t page_w, page_h; /* kinds 0/1 page size (default 2550x3300) */
    double page_scale;     /* kind 2: page dimensions multiplied by this (default 1) */
    double paths_scale;    /* kind 2: median path count multiplied by this (default 1) */
    uint32_t path_cap;     /* kind 2: max paths per page (default 50,000) */
    uint32_t reserved;
} rrb_scene_params;
typedef struct rrb_scene rrb_scene;
int rrb_scene_generate(const rrb_scene_params* p, rrb_scene** out);
void rrb_scene_free(rrb_scene* s);
/* Fills a batch view of the scene (pages = NULL, caller binds a device arena). */
void rrb_scene_view(const rrb_scene* s, rrb_path_batch_params* out);
uint64_t rrb_scene_arena_bytes(const rrb_scene* s);
/* Input segment counts of the scene: [lines, cubics, points]. */
void rrb_scene_counts(const rrb_scene* s, uint64_t out[3]);

#ifdef __cplusplus
}
#endif
#endif /* RRB_SCENES_H */
