// epp_server.cu -- the native serving loop (include/epp.h, epp_server_*).
//
// Built only on the public entry points of this library (epp_create, epp_upload, epp_search,
// epp_step, epp_query, epp_get_integrals, epp_download, epp_set_priority, epp_destroy): every
// request gets a context of its own and runs the plain path, so its result equals the same
// simulation run alone.  The loop is the Python serving module's: FIFO admission within an HBM
// budget measured by epp_context_bytes, a stream priority by run size, a few chunks of steps kept
// queued on every resident stream, retirement with the FP64 integrals.  No reference counterpart.
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
    epp_ctx* ctx = nullptr;
    int32_t queued = 0;
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

}  // namespace

struct epp_server {
    int32_t device = 0;
    int64_t budget = 0;
    int32_t max_active = 256, chunk = 100, ahead = 2;
    int64_t next_id = 0, used = 0, peak = 0;
    int32_t max_conc = 0;
    int64_t submitted = 0, completed = 0, failed = 0;
    std::deque<Request*> waiting;
    std::vector<Request*> active;
    std::map<int64_t, std::unique_ptr<Request>> all;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

void fail_request(epp_server* s, Request* r, int32_t code) {
    if (r->ctx) {
        epp_destroy(r->ctx);
        r->ctx = nullptr;
    }
    r->state = ReqState::Failed;
    r->error = code;
    r->t_done = s->now();
    ++s->failed;
    r->ip.clear();
    r->fp.clear();
}

void fill(epp_server* s, Request* r) {
    const int32_t k = std::min(s->chunk * s->ahead, r->steps - r->queued);
    if (k <= 0) return;
    const int32_t rc = epp_step(r->ctx, k, &r->phys);
    if (rc != EPP_OK) return fail_request(s, r, rc);
    r->queued += k;
}

// Context, upload and the initial search! (main.jl:157-164) of an admitted request.
int32_t admit(epp_server* s, Request* r) {
    epp_config cfg = r->cfg;
    cfg.device = s->device;
    cfg.hbm_budget_bytes = 0;
    int32_t rc = epp_create(&cfg, &r->ctx);
    if (rc != EPP_OK) return rc;
    int32_t applied = 0;
    if ((rc = epp_set_priority(r->ctx, priority_for(r->n), &applied)) != EPP_OK) return rc;
    rc = epp_upload(r->ctx, r->n, r->alive.data(), r->cell.data(), r->ip.data(), r->n, r->fp.data(), r->n, &r->map);
    if (rc != EPP_OK) return rc;
    return epp_search(r->ctx, EPP_CRITERION_SYMMETRY, EPP_ACTION_DAMBREAK_CONTINUITY, &r->phys, 0);
}

void retire(epp_server* s, Request* r) {
    int32_t rc = epp_synchronize(r->ctx, &r->status);
    if (rc == EPP_OK || rc == EPP_ERR_DEVICE_STATUS) rc = epp_get_integrals(r->ctx, &r->phys, &r->integrals);
    if (rc == EPP_OK && r->keep)
        rc = epp_download(r->ctx, r->alive.data(), r->cell.data(), r->ip.data(), r->n, r->fp.data(), r->n, &r->map);
    if (rc != EPP_OK) return fail_request(s, r, rc);
    epp_destroy(r->ctx);
    r->ctx = nullptr;
    r->state = ReqState::Done;
    r->t_done = s->now();
    ++s->completed;
    if (!r->keep) {
        r->ip.clear();
        r->fp.clear();
        r->alive.clear();
        r->cell.clear();
    }
}

// One pass: admission, refills, retirements.  Returns whether anything progressed.
bool pass(epp_server* s) {
    bool progressed = false;
    while (!s->waiting.empty() && (int32_t)s->active.size() < s->max_active) {
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
        const int32_t rc = admit(s, r);
        if (rc != EPP_OK) {
            fail_request(s, r, rc);
            continue;
        }
        r->state = ReqState::Active;
        r->t_admit = s->now();
        s->used += r->bytes;
        s->peak = std::max(s->peak, s->used);
        s->active.push_back(r);
        fill(s, r);
    }
    s->max_conc = std::max(s->max_conc, (int32_t)s->active.size());
    for (size_t k = 0; k < s->active.size();) {
        Request* r = s->active[k];
        int32_t done = 0;
        if (r->state == ReqState::Active && epp_query(r->ctx, &done) != EPP_OK) {
            fail_request(s, r, EPP_ERR_CUDA);
        } else if (r->state == ReqState::Active && done) {
            progressed = true;
            if (r->queued < r->steps) fill(s, r);
            else retire(s, r);
        }
        if (r->state == ReqState::Done || r->state == ReqState::Failed) {
            s->used -= r->bytes;
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
    st->active = (int32_t)s->active.size();
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
    for (auto& kv : s->all)
        if (kv.second->ctx) epp_destroy(kv.second->ctx);
    delete s;
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
