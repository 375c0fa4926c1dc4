// epp_server.cu -- the native serving loop (include/epp.h, epp_server_*).
//
// Built only on the public entry points of this library (epp_create, epp_upload, epp_search,
// epp_step, epp_query, epp_get_integrals, epp_download, epp_set_priority, the batch calls,
// epp_destroy): every request runs the plain path, alone on a context of its own or, co-batched,
// as one instance of a batch context, so its state equals the same simulation run alone.  The
// loop is the Python serving module's: FIFO admission within an HBM budget measured by
// epp_context_bytes, a stream priority by run size, a few chunks of steps kept queued on every
// resident stream, retirement with the FP64 integrals.  No reference counterpart.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <new>
#include <thread>
#include <vector>

#include "../../include/epp.h"

namespace {

enum class ReqState { Waiting, Active, Done, Failed };

// Columns of the reference layout that upload reads and download writes (the neighbour columns
// are left out: the server never emits lists).
struct Col {
    int32_t index, width;
};

struct Request {
    int64_t id = 0;
    epp_config cfg{};
    epp_physics phys{};
    epp_column_map map{};
    int32_t steps = 0, n = 0;
    bool keep = false;
    int ni = 0, nf = 0;                 // stored int / float columns (leading dimension n)
    std::vector<int32_t> alive, cell, ip;
    std::vector<float> fp;
    int64_t bytes = 0;
    ReqState state = ReqState::Waiting;
    int32_t error = EPP_OK;
    uint32_t status = 0;
    epp_integrals integrals{};
    double t_submit = 0, t_admit = -1, t_done = -1;
};

std::vector<Col> int_cols(const epp_column_map& m) {
    return {{m.tag, 1}, {m.is_movable, 1}, {m.n_count, 1}, {m.instance, 1}};
}

std::vector<Col> float_cols(const epp_column_map& m, int dim) {
    return {{m.position, dim}, {m.velocity, dim}, {m.dvelocity, dim}, {m.mass, 1}, {m.volume, 1},
            {m.density, 1},    {m.ddensity, 1},   {m.pressure, 1},   {m.gap, 1},  {m.h, 1}};
}

int columns_needed(const std::vector<Col>& cols) {
    int k = 0;
    for (const Col& c : cols)
        if (c.index >= 0) k = std::max(k, c.index + c.width);
    return k;
}

// Stream priority by size, as the Python loop: about one level per half decade, smallest first.
int32_t priority_for(int32_t n) {
    const double v = std::round(2.0 * (6.0 - std::log10((double)std::max(n, 1))));
    return -(int32_t)std::max(0.0, std::min(5.0, v));
}

// A resident unit: one request on its own context, or co-batched requests as the instances of
// one batch context (2D only; merged matrices with an Instance column built here).
struct Unit {
    std::vector<Request*> reqs;
    epp_ctx* ctx = nullptr;
    epp_physics phys{};
    int32_t steps = 0, queued = 0;
    int64_t bytes = 0;
    bool batch = false;
    int32_t total = 0, ni = 0, nf = 0;   // merged rows and columns (batch)
    epp_column_map map{};
    std::vector<int32_t> alive, cell, ip;
    std::vector<float> fp;
    std::vector<int32_t> row0;           // first merged row of each request
};

}  // namespace

struct epp_server {
    int32_t device = 0;
    int64_t budget = 0;
    int32_t max_active = 256, chunk = 100, ahead = 2;
    bool co_batch = false;
    int32_t batch_max = 256;
    int64_t next_id = 0, used = 0, peak = 0;
    int32_t max_conc = 0, resident = 0;
    int64_t submitted = 0, completed = 0, failed = 0;
    std::deque<Request*> waiting;
    std::vector<std::unique_ptr<Unit>> active;
    std::map<int64_t, std::unique_ptr<Request>> all;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

void release_state(Request* r) {
    if (r->keep && r->state == ReqState::Done) return;
    std::vector<int32_t>().swap(r->ip);
    std::vector<float>().swap(r->fp);
    std::vector<int32_t>().swap(r->alive);
    std::vector<int32_t>().swap(r->cell);
}

void fail_request(epp_server* s, Request* r, int32_t code) {
    r->state = ReqState::Failed;
    r->error = code;
    r->t_done = s->now();
    ++s->failed;
    release_state(r);
}

void fail_unit(epp_server* s, Unit* u, int32_t code) {
    if (u->ctx) {
        epp_destroy(u->ctx);
        u->ctx = nullptr;
    }
    for (Request* r : u->reqs)
        if (r->state == ReqState::Active) fail_request(s, r, code);
}

void fill(epp_server* s, Unit* u) {
    const int32_t k = std::min(s->chunk * s->ahead, u->steps - u->queued);
    if (k <= 0) return;
    const int32_t rc = epp_step(u->ctx, k, &u->phys);
    if (rc != EPP_OK) return fail_unit(s, u, rc);
    u->queued += k;
}

// Requests that can share a batch context: 2D, no instance column of their own, the same grid,
// tags, column layout, step count and physics apart from dt and c0.
bool batchable(const Request* r) {
    return r->cfg.domain.dim == 2 && r->cfg.n_instances <= 1 && r->map.instance < 0;
}

bool same_group(const Request* a, const Request* b) {
    if (!batchable(a) || !batchable(b) || a->steps != b->steps || a->keep != b->keep) return false;
    if (std::memcmp(&a->cfg.domain, &b->cfg.domain, sizeof a->cfg.domain) != 0) return false;
    if (a->cfg.n_tags != b->cfg.n_tags ||
        std::memcmp(a->cfg.adjacency, b->cfg.adjacency, sizeof a->cfg.adjacency) != 0)
        return false;
    if (std::memcmp(&a->map, &b->map, sizeof a->map) != 0) return false;
    epp_physics pa = a->phys, pb = b->phys;
    pa.dt = pb.dt = 0.0f;
    pa.c0 = pb.c0 = 0.0f;
    return std::memcmp(&pa, &pb, sizeof pa) == 0;
}

// Context, upload and the initial search! (main.jl:157-164) of a single request.
int32_t admit_single(epp_server* s, Unit* u) {
    Request* r = u->reqs[0];
    epp_config cfg = r->cfg;
    cfg.device = s->device;
    cfg.hbm_budget_bytes = 0;
    int32_t rc = epp_create(&cfg, &u->ctx);
    if (rc != EPP_OK) return rc;
    int32_t applied = 0;
    if ((rc = epp_set_priority(u->ctx, priority_for(r->n), &applied)) != EPP_OK) return rc;
    rc = epp_upload(u->ctx, r->n, r->alive.data(), r->cell.data(), r->ip.data(), r->n, r->fp.data(), r->n, &r->map);
    if (rc != EPP_OK) return rc;
    u->phys = r->phys;
    u->steps = r->steps;
    return epp_search(u->ctx, EPP_CRITERION_SYMMETRY, EPP_ACTION_DAMBREAK_CONTINUITY, &u->phys, 0);
}

// The same for co-batched requests: merged matrices (rows of request k after those of k - 1, an
// Instance column after the request's int columns, cells left to the first search), one context
// with per-instance dt and c0.
int32_t admit_batch(epp_server* s, Unit* u) {
    const Request* h = u->reqs[0];
    const int32_t K = (int32_t)u->reqs.size();
    int32_t total = 0;
    for (const Request* r : u->reqs) {
        u->row0.push_back(total);
        total += r->n;
    }
    u->batch = true;
    u->total = total;
    u->ni = h->ni + 1;
    u->nf = h->nf;
    u->map = h->map;
    u->map.instance = h->ni;
    try {
        u->alive.assign((size_t)total, 0);
        u->cell.assign((size_t)total, 0);
        u->ip.assign((size_t)u->ni * total, 0);
        u->fp.assign((size_t)u->nf * total, 0.0f);
    } catch (const std::bad_alloc&) {
        return EPP_ERR_OUT_OF_MEMORY;
    }
    std::vector<float> dt(K), c0(K);
    for (int32_t k = 0; k < K; ++k) {
        const Request* r = u->reqs[k];
        const size_t o = (size_t)u->row0[k];
        std::copy(r->alive.begin(), r->alive.end(), u->alive.begin() + o);
        for (int c = 0; c < h->ni; ++c)
            std::memcpy(&u->ip[(size_t)c * total + o], &r->ip[(size_t)c * r->n], sizeof(int32_t) * r->n);
        std::fill(u->ip.begin() + (size_t)h->ni * total + o, u->ip.begin() + (size_t)h->ni * total + o + r->n, k);
        for (int c = 0; c < h->nf; ++c)
            std::memcpy(&u->fp[(size_t)c * total + o], &r->fp[(size_t)c * r->n], sizeof(float) * r->n);
        dt[k] = r->phys.dt;
        c0[k] = r->phys.c0;
    }
    epp_config cfg = h->cfg;
    cfg.device = s->device;
    cfg.hbm_budget_bytes = 0;
    cfg.n_capacity = total;
    cfg.n_instances = K;
    int32_t rc = epp_create(&cfg, &u->ctx);
    if (rc != EPP_OK) return rc;
    int32_t applied = 0;
    if ((rc = epp_set_priority(u->ctx, priority_for(total), &applied)) != EPP_OK) return rc;
    if ((rc = epp_set_instance_physics(u->ctx, K, dt.data(), c0.data())) != EPP_OK) return rc;
    rc = epp_upload(u->ctx, total, u->alive.data(), u->cell.data(), u->ip.data(), total, u->fp.data(), total, &u->map);
    if (rc != EPP_OK) return rc;
    u->phys = h->phys;
    u->steps = h->steps;
    return epp_search(u->ctx, EPP_CRITERION_SYMMETRY, EPP_ACTION_DAMBREAK_CONTINUITY, &u->phys, 0);
}

void finish_request(epp_server* s, Request* r) {
    r->state = ReqState::Done;
    r->t_done = s->now();
    ++s->completed;
    release_state(r);
}

void retire(epp_server* s, Unit* u) {
    uint32_t status = 0;
    int32_t rc = epp_synchronize(u->ctx, &status);
    if (rc != EPP_OK && rc != EPP_ERR_DEVICE_STATUS) return fail_unit(s, u, rc);
    if (!u->batch) {
        Request* r = u->reqs[0];
        r->status = status;
        rc = epp_get_integrals(u->ctx, &u->phys, &r->integrals);
        if (rc == EPP_OK && r->keep)
            rc = epp_download(u->ctx, r->alive.data(), r->cell.data(), r->ip.data(), r->n, r->fp.data(), r->n, &r->map);
        if (rc != EPP_OK) return fail_unit(s, u, rc);
    } else {
        const int32_t K = (int32_t)u->reqs.size();
        std::vector<epp_integrals> out((size_t)K);
        rc = epp_get_instance_integrals(u->ctx, &u->phys, out.data(), K);
        if (rc == EPP_OK && u->reqs[0]->keep)
            rc = epp_download(u->ctx, u->alive.data(), u->cell.data(), u->ip.data(), u->total, u->fp.data(), u->total,
                              &u->map);
        if (rc != EPP_OK) return fail_unit(s, u, rc);
        for (int32_t k = 0; k < K; ++k) {
            Request* r = u->reqs[k];
            r->status = status;
            r->integrals = out[(size_t)k];
            if (!r->keep) continue;
            const size_t o = (size_t)u->row0[k];
            std::copy(u->alive.begin() + o, u->alive.begin() + o + r->n, r->alive.begin());
            std::copy(u->cell.begin() + o, u->cell.begin() + o + r->n, r->cell.begin());
            for (int c = 0; c < r->ni; ++c)
                std::memcpy(&r->ip[(size_t)c * r->n], &u->ip[(size_t)c * u->total + o], sizeof(int32_t) * r->n);
            for (int c = 0; c < r->nf; ++c)
                std::memcpy(&r->fp[(size_t)c * r->n], &u->fp[(size_t)c * u->total + o], sizeof(float) * r->n);
        }
    }
    epp_destroy(u->ctx);
    u->ctx = nullptr;
    for (Request* r : u->reqs) finish_request(s, r);
}

// One pass: admission, refills, retirements.  Returns whether anything progressed.
bool pass(epp_server* s) {
    bool progressed = false;
    while (!s->waiting.empty() && s->resident < s->max_active) {
        Request* r = s->waiting.front();
        if (r->bytes > s->budget) {   // can never fit: fail it, keep serving the rest
            s->waiting.pop_front();
            fail_request(s, r, EPP_ERR_BUDGET);
            progressed = true;
            continue;
        }
        if (s->used + r->bytes > s->budget) break;
        s->waiting.pop_front();
        progressed = true;
        std::unique_ptr<Unit> u(new Unit());
        u->reqs.push_back(r);
        u->bytes = r->bytes;
        if (s->co_batch && batchable(r)) {   // the waiting requests that can share its batch
            const int32_t cap = std::min(s->batch_max, s->max_active - s->resident);
            for (auto it = s->waiting.begin(); it != s->waiting.end() && (int32_t)u->reqs.size() < cap;) {
                if (same_group(r, *it) && s->used + u->bytes + (*it)->bytes <= s->budget) {
                    u->bytes += (*it)->bytes;
                    u->reqs.push_back(*it);
                    it = s->waiting.erase(it);
                } else {
                    ++it;
                }
            }
        }
        for (Request* m : u->reqs) m->state = ReqState::Active;
        const int32_t rc = u->reqs.size() == 1 ? admit_single(s, u.get()) : admit_batch(s, u.get());
        if (rc != EPP_OK) {
            fail_unit(s, u.get(), rc);
            continue;
        }
        const double t = s->now();
        for (Request* m : u->reqs) m->t_admit = t;
        s->used += u->bytes;
        s->peak = std::max(s->peak, s->used);
        s->resident += (int32_t)u->reqs.size();
        fill(s, u.get());
        s->active.push_back(std::move(u));
    }
    s->max_conc = std::max(s->max_conc, s->resident);
    for (size_t k = 0; k < s->active.size();) {
        Unit* u = s->active[k].get();
        int32_t done = 0;
        if (u->ctx && epp_query(u->ctx, &done) != EPP_OK) {
            fail_unit(s, u, EPP_ERR_CUDA);
        } else if (u->ctx && done) {
            progressed = true;
            if (u->queued < u->steps) fill(s, u);
            else retire(s, u);
        }
        if (!u->ctx) {   // retired or failed
            s->used -= u->bytes;
            s->resident -= (int32_t)u->reqs.size();
            s->active.erase(s->active.begin() + (long)k);
        } else {
            ++k;
        }
    }
    return progressed;
}

void stats_of(const epp_server* s, epp_server_stats* st) {
    if (!st) return;
    st->submitted = s->submitted;
    st->completed = s->completed;
    st->failed = s->failed;
    st->peak_resident_bytes = s->peak;
    st->max_concurrent = s->max_conc;
    st->waiting = (int32_t)s->waiting.size();
    st->active = s->resident;
}

}  // namespace

extern "C" {

int32_t epp_server_create(int32_t device, int64_t budget_bytes, int32_t max_active, int32_t chunk_steps,
                          int32_t ahead, epp_server** out) {
    if (!out || budget_bytes <= 0 || max_active < 1 || chunk_steps < 1 || ahead < 1) return EPP_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return EPP_ERR_NO_DEVICE;
    if (device < 0 || device >= ndev) return EPP_ERR_INVALID_ARGUMENT;
    epp_server* s = new (std::nothrow) epp_server();
    if (!s) return EPP_ERR_OUT_OF_MEMORY;
    s->device = device;
    s->budget = budget_bytes;
    s->max_active = max_active;
    s->chunk = chunk_steps;
    s->ahead = ahead;
    *out = s;
    return EPP_OK;
}

int32_t epp_server_destroy(epp_server* s) {
    if (!s) return EPP_ERR_INVALID_ARGUMENT;
    for (auto& u : s->active)
        if (u->ctx) epp_destroy(u->ctx);
    delete s;
    return EPP_OK;
}

int32_t epp_server_set_co_batch(epp_server* s, int32_t enabled, int32_t batch_max) {
    if (!s || batch_max < 1) return EPP_ERR_INVALID_ARGUMENT;
    s->co_batch = enabled != 0;
    s->batch_max = batch_max;
    return EPP_OK;
}

int32_t epp_server_submit(epp_server* s, const epp_config* config, int32_t n, const int32_t* is_alive,
                          const int32_t* cell_index, const int32_t* ip, int64_t ldi, const float* fp, int64_t ldf,
                          const epp_column_map* map, const epp_physics* phys, int32_t n_steps, int32_t keep_state,
                          int64_t* request_id) {
    if (!s || !config || !is_alive || !ip || !fp || !map || !phys || !request_id || n < 0 || n_steps < 0 ||
        ldi < n || ldf < n || n > config->n_capacity)
        return EPP_ERR_INVALID_ARGUMENT;
    std::unique_ptr<Request> r(new (std::nothrow) Request());
    if (!r) return EPP_ERR_OUT_OF_MEMORY;
    int64_t bytes = 0;
    if (const int32_t rc = epp_context_bytes(config, &bytes)) return rc;
    r->id = s->next_id++;
    r->cfg = *config;
    r->phys = *phys;
    r->map = *map;
    r->map.n_index = r->map.n_rvec = r->map.n_r = r->map.n_w = r->map.n_dw = r->map.n_hinv = -1;
    r->steps = n_steps;
    r->n = n;
    r->keep = keep_state != 0;
    r->bytes = bytes;
    const auto ic = int_cols(r->map);
    const auto fc = float_cols(r->map, config->domain.dim);
    r->ni = std::max(1, columns_needed(ic));
    r->nf = std::max(1, columns_needed(fc));
    try {
        r->alive.assign(is_alive, is_alive + n);
        r->cell.assign((size_t)n, 0);
        if (cell_index) std::copy(cell_index, cell_index + n, r->cell.begin());
        r->ip.assign((size_t)r->ni * n, 0);
        r->fp.assign((size_t)r->nf * n, 0.0f);
    } catch (const std::bad_alloc&) {
        return EPP_ERR_OUT_OF_MEMORY;
    }
    for (const Col& c : ic)
        for (int w = 0; c.index >= 0 && w < c.width; ++w)
            std::memcpy(&r->ip[(size_t)(c.index + w) * n], ip + (size_t)(c.index + w) * ldi, sizeof(int32_t) * n);
    for (const Col& c : fc)
        for (int w = 0; c.index >= 0 && w < c.width; ++w)
            std::memcpy(&r->fp[(size_t)(c.index + w) * n], fp + (size_t)(c.index + w) * ldf, sizeof(float) * n);
    r->t_submit = s->now();
    *request_id = r->id;
    s->waiting.push_back(r.get());
    s->all[r->id] = std::move(r);
    ++s->submitted;
    return EPP_OK;
}

int32_t epp_server_poll(epp_server* s, epp_server_stats* stats) {
    if (!s) return EPP_ERR_INVALID_ARGUMENT;
    pass(s);
    stats_of(s, stats);
    return EPP_OK;
}

int32_t epp_server_drain(epp_server* s, epp_server_stats* stats) {
    if (!s) return EPP_ERR_INVALID_ARGUMENT;
    while (!s->waiting.empty() || !s->active.empty())
        if (!pass(s)) std::this_thread::sleep_for(std::chrono::microseconds(50));
    stats_of(s, stats);
    return EPP_OK;
}

int32_t epp_server_result(epp_server* s, int64_t id, epp_integrals* integrals, uint32_t* device_status,
                          double* admit_s, double* done_s) {
    if (!s) return EPP_ERR_INVALID_ARGUMENT;
    auto it = s->all.find(id);
    if (it == s->all.end()) return EPP_ERR_INVALID_ARGUMENT;
    const Request* r = it->second.get();
    if (r->state == ReqState::Failed) return r->error;
    if (r->state != ReqState::Done) return EPP_ERR_STATE;
    if (integrals) *integrals = r->integrals;
    if (device_status) *device_status = r->status;
    if (admit_s) *admit_s = r->t_admit - r->t_submit;
    if (done_s) *done_s = r->t_done - r->t_submit;
    return EPP_OK;
}

int32_t epp_server_download(epp_server* s, int64_t id, int32_t* is_alive, int32_t* cell_index, int32_t* ip,
                            int64_t ldi, float* fp, int64_t ldf) {
    if (!s) return EPP_ERR_INVALID_ARGUMENT;
    auto it = s->all.find(id);
    if (it == s->all.end()) return EPP_ERR_INVALID_ARGUMENT;
    const Request* r = it->second.get();
    if (r->state == ReqState::Failed) return r->error;
    if (r->state != ReqState::Done || !r->keep) return EPP_ERR_STATE;
    if (ldi < r->n || ldf < r->n) return EPP_ERR_INVALID_ARGUMENT;
    const int n = r->n;
    if (is_alive) std::copy(r->alive.begin(), r->alive.end(), is_alive);
    if (cell_index) std::copy(r->cell.begin(), r->cell.end(), cell_index);
    if (ip)
        for (const Col& c : int_cols(r->map))
            for (int w = 0; c.index >= 0 && w < c.width; ++w)
                std::memcpy(ip + (size_t)(c.index + w) * ldi, &r->ip[(size_t)(c.index + w) * n], sizeof(int32_t) * n);
    if (fp)
        for (const Col& c : float_cols(r->map, r->cfg.domain.dim))
            for (int w = 0; c.index >= 0 && w < c.width; ++w)
                std::memcpy(fp + (size_t)(c.index + w) * ldf, &r->fp[(size_t)(c.index + w) * n], sizeof(float) * n);
    return EPP_OK;
}

}  // extern "C"
