// rrb_server.cpp — continuous-batching page-render server over the C ABI.
//
// Requests are page renders (a path batch over its own pages). Worker threads,
// each with its own backend context (own stream and scratch), take the queue
// in arrival order and form batches at every batch boundary: as many queued
// requests as fit the device-memory budget (estimated resident bytes of all
// in-flight batches) and the per-batch page cap. A request that arrives while
// batches are on the device joins the next batch that has room, so work from
// different requests overlaps on the device across workers. Each request's
// pages come back to its own host buffer; latency is submit -> pages on host.
//
// With a cost model (rrb_server_set_cost_model) every request gets, at
// submit, the predicted device time of its pages for each tile shape; batches
// then admit queued requests shortest-predicted first and/or render with the
// tile shape of least predicted total time (autotuner table as fallback).

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <system_error>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/rrb.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t id = 0;
    rrb_path_batch_params p{};  // host arrays, valid until the request completes
    uint8_t* out = nullptr;     // host pages (arena layout of p.page_offset)
    size_t out_len = 0;
    uint8_t init = 255;
    uint64_t est_bytes = 0;
    int status = RRB_OK;
    bool done = false;
    float pred[3] = {0, 0, 0};  // predicted device ms per tile shape (cost model)
    float pred_best = 0;
    int table_shape = -1;       // autotuner table's shape for its largest page
    Clock::time_point t_submit, t_start, t_done;
};

constexpr uint32_t kTiles[3][2] = {{16, 16}, {32, 32}, {64, 16}};
constexpr size_t kStageThreads = 8;  // host threads per worker that copy a batch's requests into staging

}  // namespace

struct rrb_server {
    rrb_server_config cfg{};
    std::vector<rrb_ctx*> ctx;
    std::vector<std::thread> threads;
    std::mutex m;
    std::condition_variable cv_work, cv_done, cv_pred;
    std::deque<Request*> queue;
    std::deque<Request*> pending;  // waiting for their cost-model prediction
    std::vector<std::thread> predictors;
    std::unordered_map<uint64_t, Request*> live;
    uint64_t next_id = 1;
    uint64_t in_use = 0, peak_in_use = 0;
    uint64_t batches = 0, batched_requests = 0, completed = 0;
    uint64_t tile_batches[3] = {0, 0, 0};
    uint64_t prep_ns = 0, render_ns = 0, download_ns = 0;
    bool stop = false;
    // Cost model (set before traffic; read by submitters and workers).
    std::vector<float> params;  // MLP parameters (evaluated on the host)
    bool have_params = false, have_table = false;
    uint32_t policy = 0;
    float x_mean[RRB_MLP_IN], x_std[RRB_MLP_IN], y_mean = 0, y_std = 1;
    int32_t table[16];
};

namespace {

// Device bytes a request needs while it is on the device: its pages, its
// inputs, and the intermediate edge / row data (about 3.5 edges of 32 B per
// input point on curve-heavy content, and a few bytes per pixel row), plus
// the 32 lane counts kept per curve flattened by a warp (at most one curve
// per point, at most 4 Mi curves).
uint64_t estimate_bytes(const rrb_path_batch_params& p) {
    uint64_t pages = 0;
    for (uint32_t i = 0; i < p.n_pages; ++i) pages += static_cast<uint64_t>(p.page_width[i]) * p.page_height[i];
    return 3 * pages + p.n_pts * (17 + 112) + std::min<uint64_t>(p.n_pts, 1ull << 22) * 32 + p.n_paths * 256 +
           (1u << 20);
}

// A growable array in page-locked host memory (rrb_alloc_host_pinned): the
// batch upload from it is a DMA, and a batch of 4 Mi points or more streams
// its path ranges to the device while earlier ranges render.
template <typename T>
struct PinnedVec {
    rrb_ctx* c = nullptr;
    rrb_host_buf* buf = nullptr;
    T* p = nullptr;
    size_t n = 0, cap = 0;
    ~PinnedVec() {
        if (buf) rrb_free_host_pinned(c, buf);
    }
    bool reserve(size_t want) {
        if (want <= cap) return true;
        size_t nc = std::max<size_t>(want, cap + cap / 2 + 1024);
        rrb_host_buf* nb = nullptr;
        if (rrb_alloc_host_pinned(c, nc * sizeof(T), &nb)) return false;
        T* np = static_cast<T*>(rrb_host_ptr(nb));
        if (n) std::memcpy(np, p, n * sizeof(T));
        if (buf) rrb_free_host_pinned(c, buf);
        buf = nb;
        p = np;
        cap = nc;
        return true;
    }
    bool append(const T* src, size_t k) {
        if (!reserve(n + k)) return false;
        if (k) std::memcpy(p + n, src, k * sizeof(T));
        n += k;
        return true;
    }
    bool push(T v) { return append(&v, 1); }
    // Size n (contents past the old size undefined): callers then fill it.
    bool resize(size_t k) {
        if (!reserve(k)) return false;
        n = k;
        return true;
    }
    void clear() { n = 0; }
    T* data() { return p; }
    size_t size() const { return n; }
};

struct Staging {
    PinnedVec<double> pts;
    PinnedVec<uint8_t> flags, rule, gray, alpha;
    PinnedVec<uint64_t> off, page_off;
    PinnedVec<uint32_t> path_page, pw, ph;
    void bind(rrb_ctx* c) {
        pts.c = flags.c = rule.c = gray.c = alpha.c = off.c = page_off.c = path_page.c = pw.c = ph.c = c;
    }
};

void worker(rrb_server* s, int wi) {
    rrb_ctx* c = s->ctx[wi];
    Staging st;
    st.bind(c);
    rrb_buf* arena = nullptr;
    size_t arena_cap = 0;
    for (;;) {
        std::vector<Request*> batch;
        uint64_t bytes = 0;
        {
            std::unique_lock<std::mutex> lk(s->m);
            s->cv_work.wait(lk, [&] { return s->stop || !s->queue.empty(); });
            if (s->stop && s->queue.empty()) break;
            uint32_t pages = 0;
            if (s->policy & RRB_SCHED_SHORTEST_FIRST) {
                // Shortest predicted first (stable: arrival order among equals).
                std::stable_sort(s->queue.begin(), s->queue.end(),
                                 [](const Request* a, const Request* b) { return a->pred_best < b->pred_best; });
            }
            while (!s->queue.empty()) {
                Request* r = s->queue.front();
                const bool fits = s->in_use + bytes + r->est_bytes <= s->cfg.mem_budget_bytes || s->cfg.mem_budget_bytes == 0;
                if (!batch.empty() && (!fits || pages + r->p.n_pages > s->cfg.max_batch_pages)) break;
                if (batch.empty() && !fits && s->in_use > 0) break;  // wait for memory to free up
                s->queue.pop_front();
                batch.push_back(r);
                bytes += r->est_bytes;
                pages += r->p.n_pages;
            }
            if (batch.empty()) {
                // Nothing admissible: let another batch finish first.
                s->cv_work.wait_for(lk, std::chrono::milliseconds(1));
                continue;
            }
            s->in_use += bytes;
            s->peak_in_use = std::max(s->peak_in_use, s->in_use);
            s->batches += 1;
            s->batched_requests += batch.size();
        }
        // Tile shape of this batch.
        int shape = -1;
        if (s->policy & RRB_SCHED_TILE_BY_MODEL) {
            if (s->have_params) {
                float tot[3] = {0, 0, 0};
                for (Request* r : batch)
                    for (int k = 0; k < 3; ++k) tot[k] += r->pred[k];
                shape = static_cast<int>(std::min_element(tot, tot + 3) - tot);
            } else if (s->have_table) {
                shape = batch.front()->table_shape;
            }
        }
        if (shape < 0 && s->cfg.tile_w && s->cfg.tile_h) {
            for (int k = 0; k < 3; ++k)
                if (kTiles[k][0] == s->cfg.tile_w && kTiles[k][1] == s->cfg.tile_h) shape = k;
        }
        if (shape < 0) shape = 2;
        {
            rrb_tuning t{};
            t.tile_w = kTiles[shape][0];
            t.tile_h = kTiles[shape][1];
            t.wave_points = 0xFFFFFFFFu;
            rrb_set_tuning(c, &t);
            std::lock_guard<std::mutex> lk(s->m);
            s->tile_batches[shape] += 1;
        }
        const auto t_start = Clock::now();
        auto ns_since = [](Clock::time_point a) {
            return static_cast<uint64_t>(std::chrono::duration_cast<std::chrono::nanoseconds>(Clock::now() - a).count());
        };
        // Concatenate the requests into one batch over one device arena:
        // each request's place in the staging arrays first, then the copies,
        // requests spread over host threads (the batch's points are most of
        // its bytes, and one thread's memcpy is well below the host link).
        const size_t nb = batch.size();
        std::vector<uint64_t> req_arena_off(nb), req_pt(nb + 1), req_path(nb + 1), req_page(nb + 1);
        uint64_t arena_len = 0;
        for (size_t k = 0; k < nb; ++k) {
            const rrb_path_batch_params& p = batch[k]->p;
            req_arena_off[k] = arena_len;
            req_pt[k + 1] = req_pt[k] + p.n_pts;
            req_path[k + 1] = req_path[k] + p.n_paths;
            req_page[k + 1] = req_page[k] + p.n_pages;
            arena_len += (batch[k]->out_len + 255) & ~size_t(255);
        }
        bool staged = st.pts.resize(2 * req_pt[nb]) && st.flags.resize(req_pt[nb]) &&
                      st.off.resize(req_path[nb] + 1) && st.path_page.resize(req_path[nb]) &&
                      st.rule.resize(req_path[nb]) && st.gray.resize(req_path[nb]) &&
                      st.alpha.resize(req_path[nb]) && st.pw.resize(req_page[nb]) && st.ph.resize(req_page[nb]) &&
                      st.page_off.resize(req_page[nb]);
        if (staged) {
            st.off.p[0] = 0;
            auto copy_req = [&](size_t k) {
                const rrb_path_batch_params& p = batch[k]->p;
                const uint64_t pt0 = req_pt[k], pa0 = req_path[k], pg0 = req_page[k];
                if (p.n_pts) {
                    std::memcpy(st.pts.p + 2 * pt0, p.pts, 2 * p.n_pts * sizeof(double));
                    std::memcpy(st.flags.p + pt0, p.flags, p.n_pts);
                }
                for (uint64_t i = 0; i < p.n_paths; ++i) {
                    st.off.p[pa0 + i + 1] = pt0 + p.path_pt_off[i + 1];
                    st.path_page.p[pa0 + i] = static_cast<uint32_t>(pg0) + p.path_page[i];
                }
                if (p.n_paths) {
                    std::memcpy(st.rule.p + pa0, p.fill_rule, p.n_paths);
                    std::memcpy(st.gray.p + pa0, p.gray, p.n_paths);
                    std::memcpy(st.alpha.p + pa0, p.alpha, p.n_paths);
                }
                for (uint32_t i = 0; i < p.n_pages; ++i) {
                    st.pw.p[pg0 + i] = p.page_width[i];
                    st.ph.p[pg0 + i] = p.page_height[i];
                    st.page_off.p[pg0 + i] = req_arena_off[k] + p.page_offset[i];
                }
            };
            // Threads take requests in turn; a small batch stays on this thread.
            const size_t nt = std::min<size_t>({nb, kStageThreads, req_pt[nb] / (1u << 18) + 1});
            std::atomic<size_t> next{0};
            auto run = [&]() {
                for (size_t k = next.fetch_add(1); k < nb; k = next.fetch_add(1)) copy_req(k);
            };
            std::vector<std::thread> helpers;
            try {
                for (size_t t = 1; t < nt; ++t) helpers.emplace_back(run);
            } catch (const std::system_error&) {
                // No thread to spare: the ones started and this one share the rest.
            }
            run();
            for (std::thread& h : helpers) h.join();
        }
        int rc = staged ? RRB_OK : RRB_ERR_OUT_OF_MEMORY;
        if (!rc && arena_len > arena_cap) {
            if (arena) rrb_free_device(c, arena);
            arena = nullptr;
            arena_cap = 0;
            rc = rrb_alloc_device(c, arena_len + arena_len / 4, &arena);
            if (!rc) arena_cap = arena_len + arena_len / 4;
        }
        rrb_path_batch_params b = batch.front()->p;
        b.pts = st.pts.data();
        b.flags = st.flags.data();
        b.n_pts = st.flags.size();
        b.path_pt_off = st.off.data();
        b.fill_rule = st.rule.data();
        b.gray = st.gray.data();
        b.alpha = st.alpha.data();
        b.path_page = st.path_page.data();
        b.n_paths = st.rule.size();
        b.page_width = st.pw.data();
        b.page_height = st.ph.data();
        b.page_offset = st.page_off.data();
        b.n_pages = static_cast<uint32_t>(st.pw.size());
        b.pages = arena;
        const uint64_t prep = ns_since(t_start);
        const auto t_render = Clock::now();
        rrb_fence f = 0;
        if (!rc) rc = rrb_begin_page(c);
        if (!rc) {
            for (size_t k = 0; k < batch.size() && !rc; ++k)
                rc = rrb_record_fill_buffer(c, arena, req_arena_off[k], batch[k]->out_len, batch[k]->init);
            if (!rc) rc = rrb_record_path_batch(c, &b);
            int rc2 = rrb_submit_page(c, &f);
            if (!rc) rc = rc2;
        }
        if (!rc) rc = rrb_wait_page(c, f, 0);
        const uint64_t render = ns_since(t_render);
        const auto t_down = Clock::now();
        // Every request's pages go down in stream order; one wait for the last.
        rrb_fence df = 0;
        for (size_t k = 0; k < batch.size() && !rc; ++k)
            rc = rrb_download_async(c, arena, req_arena_off[k], batch[k]->out, batch[k]->out_len, &df);
        if (!rc && df) rc = rrb_wait_download(c, df);
        const auto t_done = Clock::now();
        const uint64_t down = ns_since(t_down);
        {
            std::lock_guard<std::mutex> lk(s->m);
            s->prep_ns += prep;
            s->render_ns += render;
            s->download_ns += down;
            s->in_use -= bytes;
            for (Request* r : batch) {
                r->status = rc;
                r->t_start = t_start;
                r->t_done = t_done;
                r->done = true;
                s->completed += 1;
            }
        }
        s->cv_done.notify_all();
        s->cv_work.notify_all();
    }
    if (arena) rrb_free_device(c, arena);
}

// Cost-model predictions of one request (per tile shape, summed over its
// pages) and the table's shape for its largest page.
int predict_request(rrb_server* s, Request* r) {
    const uint32_t n = r->p.n_pages;
    std::vector<float> X(static_cast<size_t>(n) * 3 * RRB_MLP_IN);
    uint64_t biggest = 0;
    for (uint32_t pg = 0; pg < n; ++pg) {
        {
            int rc = rrb_page_features_all(&r->p, pg, &X[static_cast<size_t>(pg) * 3 * RRB_MLP_IN]);
            if (rc) return rc;
        }
        const uint64_t px = static_cast<uint64_t>(r->p.page_width[pg]) * r->p.page_height[pg];
        if (s->have_table && px >= biggest) {
            biggest = px;
            const float* x = &X[static_cast<size_t>(pg) * 3 * RRB_MLP_IN];
            const int b0 = std::min(3, std::max(0, static_cast<int>((x[0] - 13.0f) / 1.0f)));
            const int b1 = std::min(3, std::max(0, static_cast<int>((x[5] - x[0] + 6.0f) / 1.5f)));
            r->table_shape = s->table[b0 * 4 + b1];
        }
    }
    if (!s->have_params) return RRB_OK;
    for (size_t i = 0; i < X.size(); ++i) {
        const size_t j = i % RRB_MLP_IN;
        X[i] = (X[i] - s->x_mean[j]) / s->x_std[j];
    }
    std::vector<float> y(static_cast<size_t>(n) * 3);
    int rc = rrb_mlp_predict_host(s->params.data(), X.data(), n * 3, y.data());
    if (rc) return rc;
    for (int k = 0; k < 3; ++k) r->pred[k] = 0;
    for (uint32_t pg = 0; pg < n; ++pg)
        for (int k = 0; k < 3; ++k) r->pred[k] += std::exp(y[pg * 3 + k] * s->y_std + s->y_mean);
    r->pred_best = *std::min_element(r->pred, r->pred + 3);
    return RRB_OK;
}

// Predictor thread: computes the predictions of submitted requests and moves
// them to the render queue.
void predictor(rrb_server* s) {
    for (;;) {
        Request* r;
        {
            std::unique_lock<std::mutex> lk(s->m);
            s->cv_pred.wait(lk, [&] { return s->stop || !s->pending.empty(); });
            if (s->pending.empty()) break;  // stopping
            r = s->pending.front();
            s->pending.pop_front();
        }
        const int rc = predict_request(s, r);
        {
            std::lock_guard<std::mutex> lk(s->m);
            if (rc) {
                r->status = rc;
                r->t_start = r->t_done = Clock::now();
                r->done = true;
                s->completed += 1;
            } else {
                s->queue.push_back(r);
            }
        }
        if (rc) s->cv_done.notify_all();
        else s->cv_work.notify_one();
    }
}

}  // namespace

extern "C" {

int rrb_server_set_cost_model(rrb_server* s, const rrb_server_cost_model* m) {
    if (!s || !m) return RRB_ERR_INVARIANT;
    if (m->params && (!m->x_mean || !m->x_std)) return RRB_ERR_INVARIANT;
    if (m->table)
        for (int k = 0; k < 16; ++k)
            if (m->table[k] < 0 || m->table[k] > 2) return RRB_ERR_INVARIANT;
    std::lock_guard<std::mutex> lk(s->m);
    if (m->params) {
        s->params.assign(m->params, m->params + RRB_MLP_PARAMS);
        std::memcpy(s->x_mean, m->x_mean, sizeof s->x_mean);
        std::memcpy(s->x_std, m->x_std, sizeof s->x_std);
        s->y_mean = m->y_mean;
        s->y_std = m->y_std;
    }
    s->have_params = m->params != nullptr;
    s->have_table = m->table != nullptr;
    if (m->table) std::memcpy(s->table, m->table, sizeof s->table);
    s->policy = m->policy;
    if ((s->have_params || s->have_table) && s->predictors.empty()) {
        const uint32_t n = s->cfg.predict_threads ? s->cfg.predict_threads : 4;
        for (uint32_t i = 0; i < n; ++i) s->predictors.emplace_back(predictor, s);
    }
    return RRB_OK;
}

int rrb_server_create(const rrb_server_config* cfg, rrb_server** out) {
    if (!cfg || !out) return RRB_ERR_INVARIANT;
    rrb_server* s = new rrb_server();
    s->cfg = *cfg;
    if (!s->cfg.workers) s->cfg.workers = 2;
    if (!s->cfg.max_batch_pages) s->cfg.max_batch_pages = 64;
    for (uint32_t i = 0; i < s->cfg.workers; ++i) {
        rrb_ctx* c = nullptr;
        int rc = rrb_init(cfg->device, 0, &c);
        if (rc) {
            for (rrb_ctx* x : s->ctx) rrb_destroy(x);
            delete s;
            return rc;
        }
        rrb_tuning t{};
        t.tile_w = cfg->tile_w;
        t.tile_h = cfg->tile_h;
        t.wave_points = 0xFFFFFFFFu;
        if (t.tile_w && t.tile_h) rrb_set_tuning(c, &t);
        s->ctx.push_back(c);
    }
    for (uint32_t i = 0; i < s->cfg.workers; ++i) s->threads.emplace_back(worker, s, static_cast<int>(i));
    *out = s;
    return RRB_OK;
}

int rrb_server_submit(rrb_server* s, const rrb_path_batch_params* p, uint8_t* host_pages, size_t host_pages_len,
                      uint8_t init_value, uint64_t* ticket) {
    if (!s || !p || !host_pages || !ticket) return RRB_ERR_INVARIANT;
    char msg[8];
    int rc = rrb_validate_path_batch(p, host_pages_len, msg, sizeof msg);
    if (rc) return rc;
    const auto t0 = Clock::now();
    Request* r = new Request();
    r->p = *p;
    r->out = host_pages;
    r->out_len = host_pages_len;
    r->init = init_value;
    r->est_bytes = estimate_bytes(*p);
    r->t_submit = t0;
    bool predicted = false;
    {
        std::lock_guard<std::mutex> lk(s->m);
        r->id = s->next_id++;
        s->live[r->id] = r;
        predicted = !s->predictors.empty();
        if (predicted) s->pending.push_back(r);
        else s->queue.push_back(r);
    }
    *ticket = r->id;
    if (predicted) s->cv_pred.notify_one();
    else s->cv_work.notify_one();
    return RRB_OK;
}

int rrb_server_wait(rrb_server* s, uint64_t ticket, uint64_t timeout_ns, rrb_request_result* res) {
    if (!s) return RRB_ERR_INVARIANT;
    std::unique_lock<std::mutex> lk(s->m);
    auto it = s->live.find(ticket);
    if (it == s->live.end()) return RRB_ERR_INVARIANT;
    Request* r = it->second;
    auto ready = [&] { return r->done; };
    if (timeout_ns) {
        if (!s->cv_done.wait_for(lk, std::chrono::nanoseconds(timeout_ns), ready)) return RRB_ERR_TIMEOUT;
    } else {
        s->cv_done.wait(lk, ready);
    }
    if (res) {
        res->status = r->status;
        res->latency_ns = static_cast<uint64_t>(std::chrono::duration_cast<std::chrono::nanoseconds>(r->t_done - r->t_submit).count());
        res->queue_ns = static_cast<uint64_t>(std::chrono::duration_cast<std::chrono::nanoseconds>(r->t_start - r->t_submit).count());
    }
    const int st = r->status;
    s->live.erase(it);
    delete r;
    return st;
}

int rrb_server_stats(rrb_server* s, rrb_server_stats_t* out) {
    if (!s || !out) return RRB_ERR_INVARIANT;
    std::lock_guard<std::mutex> lk(s->m);
    out->completed = s->completed;
    out->batches = s->batches;
    out->batched_requests = s->batched_requests;
    out->queued = s->queue.size();
    out->in_use_bytes = s->in_use;
    out->peak_in_use_bytes = s->peak_in_use;
    for (int k = 0; k < 3; ++k) out->tile_batches[k] = s->tile_batches[k];
    out->prep_ns = s->prep_ns;
    out->render_ns = s->render_ns;
    out->download_ns = s->download_ns;
    return RRB_OK;
}

int rrb_server_destroy(rrb_server* s) {
    if (!s) return RRB_OK;
    {
        std::lock_guard<std::mutex> lk(s->m);
        s->stop = true;
    }
    s->cv_pred.notify_all();
    for (std::thread& t : s->predictors) t.join();
    s->cv_work.notify_all();
    for (std::thread& t : s->threads) t.join();
    for (rrb_ctx* c : s->ctx) rrb_destroy(c);
    for (auto& kv : s->live) delete kv.second;
    delete s;
    return RRB_OK;
}

}  // extern "C"
