// scene_gen.cpp — the seeded synthetic workloads of the benchmark and the
// tests (librrb_scenes.so, a library of its own: it is not part of the fill
// backend, and a process that only generates scenes, such as the CPU
// baseline, never maps the backend library).
//
// rrb_scene_generate builds the workloads from a SplitMix64 stream:
//   kind 0  polygon page: closed paths of 1-3 contours, 4-32 line or cubic
//           segments on jittered circles with log-normal radius;
//   kind 1  glyph-dense text page: quadratic glyph outlines on 60 baselines;
//   kind 2  mixed pages: {A4, Letter, A3} x {150, 300, 600} dpi, 30% glyphs,
//           40% polygons, 30% axis-aligned rectangles, alpha 32-255.
// Every path is built through the product's PathBuilder restatement
// (path_builder.cpp, compiled into this library too), so the generated
// Path::{pts, flags} arrays are exactly what the reference's builder would
// produce for the same calls.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/rrb_scenes.h"
#include "../csrc/path_builder.h"

// ---------------------------------------------------------------------------
// Scene generator
// ---------------------------------------------------------------------------
namespace {

// SplitMix64 (Steele, Lea, Flood 2014).
struct Rng {
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double u01() { return static_cast<double>(next() >> 11) * (1.0 / 9007199254740992.0); }
    double uniform(double a, double b) { return a + (b - a) * u01(); }
    int64_t randint(int64_t a, int64_t b) {  // inclusive
        int64_t v = a + static_cast<int64_t>(u01() * static_cast<double>(b - a + 1));
        return v > b ? b : v;
    }
    double normal() {  // Box-Muller, one variate per call
        double u1 = 1.0 - u01();
        double u2 = u01();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

constexpr double kPi = 3.141592653589793;

struct Scene {
    std::vector<double> pts;
    std::vector<uint8_t> flags;
    std::vector<uint64_t> path_pt_off{0};
    std::vector<uint8_t> rule, gray, alpha;
    std::vector<uint32_t> path_page;
    std::vector<uint32_t> page_w, page_h;
    std::vector<uint64_t> page_off;
    uint64_t arena = 0;
    uint64_t n_lines = 0, n_cubics = 0;
    rrb_path builder;

    void add_page(uint32_t w, uint32_t h) {
        page_w.push_back(w);
        page_h.push_back(h);
        page_off.push_back(arena);
        arena += (static_cast<uint64_t>(w) * h + 255) & ~uint64_t(255);
    }
    void commit(uint32_t page, uint8_t r, uint8_t g, uint8_t a) {
        const rrb_path& b = builder;
        pts.insert(pts.end(), b.pts.begin(), b.pts.end());
        flags.insert(flags.end(), b.flags.begin(), b.flags.end());
        for (size_t i = 0; i < b.flags.size(); ++i) {
            if (b.flags[i] & RRB_PATH_FIRST) continue;
            if (b.flags[i] & RRB_PATH_CURVE) {
                ++n_cubics;
                i += 2;
            } else {
                ++n_lines;
            }
        }
        path_pt_off.push_back(flags.size());
        rule.push_back(r);
        gray.push_back(g);
        alpha.push_back(a);
        path_page.push_back(page);
        rrb_path_clear(&builder);
    }
};

inline double clampd(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Polygon path: 1-3 contours of 4-32 segments on a jittered circle; each
// segment a line (p=.5) or a cubic (p=.5); vertices clipped to the page; the
// last segment returns exactly to the first vertex, then close(false).
void gen_polygon(Rng& r, Scene& s, double W, double H, double radius_scale) {
    int ncont = static_cast<int>(r.randint(1, 3));
    double cx = r.uniform(0.0, W), cy = r.uniform(0.0, H);
    double rad = std::exp(std::log(60.0) + 1.0 * r.normal()) * radius_scale;
    rad = std::min(rad, std::max(W, H));
    rrb_path* b = &s.builder;
    std::vector<double> vx, vy;
    for (int c = 0; c < ncont; ++c) {
        int nseg = static_cast<int>(r.randint(4, 32));
        double rc = rad * (c == 0 ? 1.0 : r.uniform(0.25, 0.95));
        double ox = c == 0 ? 0.0 : r.uniform(-0.3, 0.3) * rad;
        double oy = c == 0 ? 0.0 : r.uniform(-0.3, 0.3) * rad;
        double dir = (c == 0 || r.u01() < 0.5) ? 1.0 : -1.0;
        double phase = r.uniform(0.0, 2.0 * kPi);
        vx.resize(nseg);
        vy.resize(nseg);
        for (int k = 0; k < nseg; ++k) {
            double th = phase + dir * 2.0 * kPi * (k + r.uniform(-0.35, 0.35)) / nseg;
            double rr = rc * r.uniform(0.7, 1.3);
            vx[k] = clampd(cx + ox + rr * std::cos(th), 0.0, W);
            vy[k] = clampd(cy + oy + rr * std::sin(th), 0.0, H);
        }
        rrb_path_move_to(b, vx[0], vy[0]);
        for (int k = 0; k < nseg; ++k) {
            int n = (k + 1) % nseg;
            if (r.u01() < 0.5) {
                rrb_path_line_to(b, vx[n], vy[n]);
            } else {
                double dx = vx[n] - vx[k], dy = vy[n] - vy[k];
                double j1 = r.uniform(-0.4, 0.4), j2 = r.uniform(-0.4, 0.4);
                double c1x = clampd(vx[k] + dx / 3.0 - dy * j1, 0.0, W);
                double c1y = clampd(vy[k] + dy / 3.0 + dx * j1, 0.0, H);
                double c2x = clampd(vx[k] + 2.0 * dx / 3.0 - dy * j2, 0.0, W);
                double c2y = clampd(vy[k] + 2.0 * dy / 3.0 + dx * j2, 0.0, H);
                rrb_path_curve_to(b, c1x, c1y, c2x, c2y, vx[n], vy[n]);
            }
        }
        rrb_path_close(b, 0);
    }
}

// Glyph-like path in an em box whose left edge is x0 and baseline is yb:
// an outer contour plus 0-2 reversed counters, 12-60 quadratic segments each,
// on-curve points on jittered ellipses and control points on the tangent
// intersections, every quadratic elevated by conic_to_cubic.
void gen_glyph(Rng& r, Scene& s, double x0, double yb, double em) {
    int ncont = static_cast<int>(r.randint(1, 3));
    rrb_path* b = &s.builder;
    double ocx = x0 + 0.35 * em, ocy = yb - 0.38 * em;
    double orx = 0.30 * em * r.uniform(0.8, 1.1), ory = 0.38 * em * r.uniform(0.8, 1.1);
    std::vector<double> px, py, qx, qy;
    for (int c = 0; c < ncont; ++c) {
        int nq = static_cast<int>(r.randint(12, 60));
        double cxc = ocx, cyc = ocy, rx = orx, ry = ory, dir = 1.0;
        if (c > 0) {
            double f = r.uniform(0.25, 0.5);
            rx = orx * f;
            ry = ory * f;
            cxc = ocx + r.uniform(-0.3, 0.3) * (orx - rx);
            cyc = ocy + r.uniform(-0.3, 0.3) * (ory - ry);
            dir = -1.0;
        }
        double phase = r.uniform(0.0, 2.0 * kPi);
        px.resize(nq); py.resize(nq); qx.resize(nq); qy.resize(nq);
        double kc = 1.0 / std::cos(kPi / nq);
        for (int k = 0; k < nq; ++k) {
            double th = phase + dir * 2.0 * kPi * k / nq;
            double j = 1.0 + r.uniform(-0.08, 0.08);
            px[k] = cxc + rx * j * std::cos(th);
            py[k] = cyc + ry * j * std::sin(th);
            double tm = phase + dir * 2.0 * kPi * (k + 0.5) / nq;
            double jm = kc * (1.0 + r.uniform(-0.08, 0.08));
            qx[k] = cxc + rx * jm * std::cos(tm);
            qy[k] = cyc + ry * jm * std::sin(tm);
        }
        rrb_path_move_to(b, px[0], py[0]);
        for (int k = 0; k < nq; ++k) {
            int n = (k + 1) % nq;
            rrb_path_conic_to(b, qx[k], qy[k], px[n], py[n]);
        }
        rrb_path_close(b, 0);
    }
}

// Axis-aligned rectangle covering `frac` of the page area.
void gen_rect(Rng& r, Scene& s, double W, double H) {
    double frac = r.uniform(0.05, 0.8);
    double aspect = std::exp(r.uniform(-0.7, 0.7));
    double area = frac * W * H;
    double w = std::min(std::sqrt(area * aspect), W);
    double h = std::min(area / w, H);
    double x0 = r.uniform(0.0, W - w), y0 = r.uniform(0.0, H - h);
    rrb_path* b = &s.builder;
    rrb_path_move_to(b, x0, y0);
    rrb_path_line_to(b, x0 + w, y0);
    rrb_path_line_to(b, x0 + w, y0 + h);
    rrb_path_line_to(b, x0, y0 + h);
    rrb_path_close(b, 0);
}

// Page sizes {A4, Letter, A3} x {150, 300, 600} dpi, round(pts * dpi / 72).
const uint32_t kPageSizes[9][3] = {
    {1240, 1754, 150}, {2480, 3508, 300}, {4961, 7016, 600},
    {1275, 1650, 150}, {2550, 3300, 300}, {5100, 6600, 600},
    {1754, 2480, 150}, {3508, 4961, 300}, {7016, 9921, 600},
};

}  // namespace

struct rrb_scene {
    Scene s;
};

extern "C" {

int rrb_scene_generate(const rrb_scene_params* p, rrb_scene** out) {
    if (!p || !out) return RRB_ERR_INVARIANT;
    rrb_scene* sc = new rrb_scene();
    Scene& s = sc->s;
    Rng r(p->seed);
    if (p->kind == 0 || p->kind == 1) {
        uint32_t W = p->page_w ? p->page_w : 2550, H = p->page_h ? p->page_h : 3300;
        s.add_page(W, H);
        if (p->kind == 0) {
            uint32_t n = p->n_paths ? p->n_paths : 2000;
            for (uint32_t i = 0; i < n; ++i) {
                gen_polygon(r, s, W, H, 1.0);
                uint8_t rule = r.u01() < 0.7 ? RRB_FILL_NONZERO : RRB_FILL_EVEN_ODD;
                uint8_t g = static_cast<uint8_t>(r.randint(0, 255));
                s.commit(0, rule, g, 255);
            }
        } else {
            uint32_t n = p->n_paths ? p->n_paths : 150000;
            const uint32_t lines = 60;
            uint32_t per_line = (n + lines - 1) / lines;
            double pitch = static_cast<double>(H) / (lines + 1);
            double adv = static_cast<double>(W) / per_line;
            uint32_t made = 0;
            for (uint32_t l = 0; l < lines && made < n; ++l) {
                double yb = (l + 1) * pitch;
                double x = 0.0;
                for (uint32_t g = 0; g < per_line && made < n; ++g, ++made) {
                    double em = r.uniform(8.0, 12.0) * 300.0 / 72.0;
                    gen_glyph(r, s, x, yb, em);
                    s.commit(0, RRB_FILL_NONZERO, 0, 255);
                    x += adv * r.uniform(0.9, 1.1);
                }
            }
        }
    } else if (p->kind == 2) {
        uint32_t n_pages = p->n_pages ? p->n_pages : 64;
        double pscale = p->page_scale > 0 ? p->page_scale : 1.0;
        double nscale = p->paths_scale > 0 ? p->paths_scale : 1.0;
        uint32_t cap = p->path_cap ? p->path_cap : 50000;
        for (uint32_t pg = 0; pg < n_pages; ++pg) {
            const uint32_t* sz = kPageSizes[r.randint(0, 8)];
            uint32_t W = std::max<uint32_t>(16, static_cast<uint32_t>(std::lround(sz[0] * pscale)));
            uint32_t H = std::max<uint32_t>(16, static_cast<uint32_t>(std::lround(sz[1] * pscale)));
            double dpi_f = sz[2] / 300.0 * pscale;
            s.add_page(W, H);
            double cnt = std::exp(std::log(5000.0 * nscale) + 1.2 * r.normal());
            uint32_t n = static_cast<uint32_t>(std::min<double>(std::max(1.0, std::round(cnt)), cap));
            for (uint32_t i = 0; i < n; ++i) {
                double u = r.u01();
                uint8_t rule = RRB_FILL_NONZERO;
                if (u < 0.3) {
                    double em = r.uniform(8.0, 12.0) * sz[2] / 72.0 * pscale;
                    double x0 = r.uniform(0.0, std::max(1.0, W - em));
                    double yb = r.uniform(em, std::max(em + 1.0, static_cast<double>(H)));
                    gen_glyph(r, s, x0, yb, em);
                } else if (u < 0.7) {
                    gen_polygon(r, s, W, H, dpi_f);
                    rule = r.u01() < 0.7 ? RRB_FILL_NONZERO : RRB_FILL_EVEN_ODD;
                } else {
                    gen_rect(r, s, W, H);
                }
                uint8_t g = static_cast<uint8_t>(r.randint(0, 255));
                uint8_t a = static_cast<uint8_t>(r.randint(32, 255));
                s.commit(pg, rule, g, a);
            }
        }
    } else {
        delete sc;
        return RRB_ERR_INVARIANT;
    }
    *out = sc;
    return RRB_OK;
}

void rrb_scene_free(rrb_scene* s) { delete s; }

void rrb_scene_view(const rrb_scene* sc, rrb_path_batch_params* o) {
    const Scene& s = sc->s;
    std::memset(o, 0, sizeof *o);
    o->pts = s.pts.data();
    o->flags = s.flags.data();
    o->n_pts = s.flags.size();
    o->path_pt_off = s.path_pt_off.data();
    o->fill_rule = s.rule.data();
    o->gray = s.gray.data();
    o->alpha = s.alpha.data();
    o->path_page = s.path_page.data();
    o->n_paths = s.rule.size();
    o->page_width = s.page_w.data();
    o->page_height = s.page_h.data();
    o->page_offset = s.page_off.data();
    o->n_pages = static_cast<uint32_t>(s.page_w.size());
    o->pages = nullptr;
    o->matrix[0] = 1.0;
    o->matrix[3] = 1.0;
    o->flatness = 0.1;
    o->rowmap = RRB_ROWMAP_DOCUMENTED;
}

uint64_t rrb_scene_arena_bytes(const rrb_scene* s) { return s->s.arena; }

void rrb_scene_counts(const rrb_scene* s, uint64_t out[3]) {
    out[0] = s->s.n_lines;
    out[1] = s->s.n_cubics;
    out[2] = s->s.flags.size();
}

}  // extern "C"
