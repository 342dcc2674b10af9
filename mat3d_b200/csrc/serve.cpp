// Serving loop (m3d_serve_*): continuous admission of RVE solves of mixed
// kinds and grid sizes onto one GPU.
//
// Requests enter a FIFO queue.  Worker threads (one CUDA stream per solver)
// take the first request that fits: a resident idle solver of the same shape
// is reused as is; otherwise a new one is created if its device footprint
// (m3d_footprint_bytes) fits the budget, after releasing idle solvers of other
// shapes, least recently used first.  A request that does not fit yet is
// passed over by later ones at most kMaxBypass times, then it waits at the
// head until memory frees up.  Solves of different requests run on different
// streams and overlap on the device; each request runs alone on its solver,
// so its result does not depend on what else is in flight.
#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "mat3d_b200.h"

void m3d_internal_set_error(const std::string& msg);

namespace {

typedef std::chrono::steady_clock Clock;
typedef std::tuple<int, int, int, int, int, int> ShapeKey;  // kind, behav, Nx, Ny, Nz, precision

constexpr int kMaxBypass = 8;

struct Req {
    long long ticket = 0;
    m3d_request r{};
    std::vector<double> mat;
    std::vector<int32_t> phase;
    double E[6] = {}, X0[6] = {};
    bool hasX0 = false;
    ShapeKey key;
    long long bytes = 0;
    int bypassed = 0;
    Clock::time_point t_submit, t_admit;
};

struct Done {
    m3d_result res{};
    std::vector<double> field;
    bool keep_field = false;
};

struct Idle {
    m3d_solver* h;
    long long bytes;
    Clock::time_point last;
};

int sfail(int code, const std::string& msg) {
    m3d_internal_set_error(msg);
    return code;
}

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace

struct m3d_server {
    int dev = 0;
    double budget = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::unique_ptr<Req>> queue;
    std::map<long long, Done> done;
    std::map<long long, bool> pending;  // submitted, not yet finished
    std::multimap<ShapeKey, Idle> idle;
    long long next_ticket = 1;
    double resident = 0;  // bytes of all solvers held (running + idle)
    int running = 0, peak_running = 0, n_solvers = 0;
    long long submitted = 0, completed = 0, failed = 0;
    bool stop = false;
    std::vector<std::thread> workers;

    void worker();
    std::unique_ptr<Req> pick(m3d_solver** reuse, long long* reserved, std::vector<m3d_solver*>& evict);
    int solve(Req& q, m3d_solver* h, Done& d);
};

// Under `mu`.  The first queued request that can start now: one with an idle
// solver of its shape, or one whose footprint fits after releasing idle
// solvers of other shapes (least recently used first).  Bypassing is bounded.
std::unique_ptr<Req> m3d_server::pick(m3d_solver** reuse, long long* reserved, std::vector<m3d_solver*>& evict) {
    *reuse = nullptr;
    *reserved = 0;
    for (size_t i = 0; i < queue.size(); ++i) {
        Req& q = *queue[i];
        auto it = idle.find(q.key);
        bool ok = false;
        if (it != idle.end()) {
            *reuse = it->second.h;
            idle.erase(it);
            ok = true;
        } else {
            double idle_bytes = 0;
            for (auto& e : idle) idle_bytes += (double)e.second.bytes;
            if (resident - idle_bytes + (double)q.bytes <= budget) {
                while (resident + (double)q.bytes > budget && !idle.empty()) {
                    auto lru = idle.begin();
                    for (auto e = idle.begin(); e != idle.end(); ++e)
                        if (e->second.last < lru->second.last) lru = e;
                    evict.push_back(lru->second.h);
                    resident -= (double)lru->second.bytes;
                    --n_solvers;
                    idle.erase(lru);
                }
                resident += (double)q.bytes;
                ++n_solvers;
                *reserved = q.bytes;
                ok = true;
            }
        }
        if (ok) {
            std::unique_ptr<Req> r = std::move(queue[i]);
            queue.erase(queue.begin() + (long)i);
            for (size_t j = 0; j < i; ++j) queue[j]->bypassed += 1;
            return r;
        }
        if (q.bypassed >= kMaxBypass) break;  // keep FIFO order behind a starved request
    }
    return nullptr;
}

int m3d_server::solve(Req& q, m3d_solver* h, Done& d) {
    const m3d_request& r = q.r;
    int rc = (r.kind == M3D_KIND_MECH)
                 ? m3d_set_material_mech(h, q.mat.data(), r.nph, q.phase.data(), r.scheme)
                 : m3d_set_material_thermal(h, r.km, r.ki, q.phase.data(), r.scheme);
    if (rc) return rc;
    rc = m3d_set_load(h, 0, q.E, q.hasX0 ? q.X0 : nullptr);
    if (rc) return rc;
    const int st = m3d_run(h, r.tol, 0.0, r.nInc, M3D_CRIT_RESIDUAL, r.max_iter);
    if (st != M3D_OK && st != M3D_NOT_CONVERGED) return st;
    rc = m3d_get_means(h, 0, d.res.strain_mean, d.res.stress_mean);
    if (rc) return rc;
    m3d_stats s;
    m3d_get_stats(h, &s);
    d.res.iters = s.iters;
    d.res.sweeps = s.sweeps;
    d.res.residual = s.residual;
    if (r.keep_field) {
        const int C = (r.kind == M3D_KIND_MECH) ? 6 : 3;
        d.field.assign((size_t)C * r.Nx * r.Ny * r.Nz, 0.0);
        rc = m3d_get_field(h, M3D_FIELD_STRAIN, 0, d.field.data());
        if (rc) return rc;
        d.keep_field = true;
    }
    return st;
}

void m3d_server::worker() {
    cudaSetDevice(dev);
    for (;;) {
        std::unique_ptr<Req> q;
        m3d_solver* h = nullptr;
        long long reserved = 0;
        std::vector<m3d_solver*> evict;
        {
            std::unique_lock<std::mutex> lk(mu);
            for (;;) {
                if (!queue.empty()) q = pick(&h, &reserved, evict);
                if (q || (stop && queue.empty())) break;
                cv_work.wait(lk);
            }
            if (!q) return;
            ++running;
            if (running > peak_running) peak_running = running;
        }
        for (m3d_solver* e : evict) m3d_destroy(e);
        q->t_admit = Clock::now();
        Done d;
        int rc = M3D_OK;
        if (!h) {
            const m3d_request& r = q->r;
            rc = m3d_create(r.kind, r.Nx, r.Ny, r.Nz, r.behav, r.precision, 1, &h);
            if (rc) h = nullptr;
        }
        if (h) rc = solve(*q, h, d);
        const auto t_done = Clock::now();
        d.res.status = rc;
        d.res.queue_ms = ms_between(q->t_submit, q->t_admit);
        d.res.solve_ms = ms_between(q->t_admit, t_done);
        d.res.latency_ms = ms_between(q->t_submit, t_done);
        {
            std::lock_guard<std::mutex> lk(mu);
            if (h) {
                idle.insert(std::make_pair(q->key, Idle{h, q->bytes, t_done}));
            } else if (reserved) {
                resident -= (double)reserved;
                --n_solvers;
            }
            --running;
            ++completed;
            if (rc != M3D_OK && rc != M3D_NOT_CONVERGED) ++failed;
            pending.erase(q->ticket);
            done[q->ticket] = std::move(d);
        }
        cv_done.notify_all();
        cv_work.notify_all();
    }
}

extern "C" {

int m3d_serve_create(double mem_budget_bytes, int workers, m3d_server** out) {
    if (!out) return sfail(M3D_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (workers < 1 || workers > 64) return sfail(M3D_ERR_ARG, "workers must be in [1, 64]");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return sfail(M3D_ERR_CUDA, "no CUDA device");
    if (!(mem_budget_bytes > 0)) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return sfail(M3D_ERR_CUDA, "no CUDA device");
        mem_budget_bytes = 0.85 * (double)fr;
    }
    m3d_server* s = new m3d_server();
    s->dev = dev;
    s->budget = mem_budget_bytes;
    for (int i = 0; i < workers; ++i) s->workers.emplace_back([s] { s->worker(); });
    *out = s;
    return M3D_OK;
}

int m3d_serve_submit(m3d_server* s, const m3d_request* req, long long* ticket) {
    if (!s || !req || !ticket) return sfail(M3D_ERR_ARG, "NULL argument");
    const m3d_request& r = *req;
    if (r.kind != M3D_KIND_MECH && r.kind != M3D_KIND_THERMAL) return sfail(M3D_ERR_ARG, "invalid kind");
    if (!r.phase || !r.E) return sfail(M3D_ERR_ARG, "phase and E are required");
    if (r.kind == M3D_KIND_MECH && (!r.mat || r.nph < 1 || r.nph > 16)) return sfail(M3D_ERR_ARG, "mech needs mat, nph in [1, 16]");
    if (r.Nx < 2 || r.Ny < 2 || r.Nz < 2 || r.Nx > 1024 || r.Ny > 1024 || r.Nz > 1024)
        return sfail(M3D_ERR_ARG, "grid sizes must be in [2, 1024]");
    if (!(r.tol > 0)) return sfail(M3D_ERR_ARG, "tol must be positive");
    const long long bytes = m3d_footprint_bytes(r.kind, r.Nx, r.Ny, r.Nz, r.behav, r.precision, 1, 1);
    if (bytes < 0) return sfail(M3D_ERR_ARG, "invalid shape or precision");
    if ((double)bytes > s->budget) return sfail(M3D_ERR_OOM, "request footprint exceeds the memory budget");
    std::unique_ptr<Req> q(new Req());
    q->r = r;
    const size_t V = (size_t)r.Nx * r.Ny * r.Nz;
    q->phase.assign(r.phase, r.phase + V);
    if (r.kind == M3D_KIND_MECH) q->mat.assign(r.mat, r.mat + (size_t)r.nph * 7);
    const int C = (r.kind == M3D_KIND_MECH) ? 6 : 3;
    for (int i = 0; i < C; ++i) q->E[i] = r.E[i];
    if (r.X0) {
        for (int i = 0; i < 6; ++i) q->X0[i] = r.X0[i];
        q->hasX0 = true;
    }
    q->r.mat = nullptr;
    q->r.phase = nullptr;
    q->r.E = nullptr;
    q->r.X0 = nullptr;
    if (q->r.nInc < 1) q->r.nInc = 1;
    q->key = std::make_tuple(r.kind, r.behav, r.Nx, r.Ny, r.Nz, r.precision);
    q->bytes = bytes;
    q->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) return sfail(M3D_ERR_STATE, "server is shutting down");
        q->ticket = s->next_ticket++;
        *ticket = q->ticket;
        s->pending[q->ticket] = true;
        ++s->submitted;
        s->queue.push_back(std::move(q));
    }
    s->cv_work.notify_one();
    return M3D_OK;
}

static int take_result(m3d_server* s, long long ticket, m3d_result* out) {
    auto it = s->done.find(ticket);
    if (it == s->done.end()) return s->pending.count(ticket) ? M3D_PENDING : sfail(M3D_ERR_ARG, "unknown ticket");
    if (out) *out = it->second.res;
    if (!it->second.keep_field) s->done.erase(it);
    return M3D_OK;
}

int m3d_serve_poll(m3d_server* s, long long ticket, m3d_result* out) {
    if (!s) return sfail(M3D_ERR_ARG, "NULL server");
    std::lock_guard<std::mutex> lk(s->mu);
    return take_result(s, ticket, out);
}

int m3d_serve_wait(m3d_server* s, long long ticket, double timeout_ms, m3d_result* out) {
    if (!s) return sfail(M3D_ERR_ARG, "NULL server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto ready = [&] { return s->done.count(ticket) || !s->pending.count(ticket); };
    if (timeout_ms < 0) s->cv_done.wait(lk, ready);
    else s->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), ready);
    return take_result(s, ticket, out);
}

int m3d_serve_get_field(m3d_server* s, long long ticket, double* out) {
    if (!s || !out) return sfail(M3D_ERR_ARG, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->done.find(ticket);
    if (it == s->done.end() || !it->second.keep_field)
        return s->pending.count(ticket) ? M3D_PENDING : sfail(M3D_ERR_ARG, "no kept field for this ticket");
    std::memcpy(out, it->second.field.data(), it->second.field.size() * sizeof(double));
    s->done.erase(it);
    return M3D_OK;
}

int m3d_serve_get_stats(m3d_server* s, m3d_serve_stats* out) {
    if (!s || !out) return sfail(M3D_ERR_ARG, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    out->submitted = s->submitted;
    out->completed = s->completed;
    out->failed = s->failed;
    out->queued = (int)s->queue.size();
    out->running = s->running;
    out->peak_running = s->peak_running;
    out->resident_solvers = s->n_solvers;
    out->resident_bytes = s->resident;
    out->budget_bytes = s->budget;
    return M3D_OK;
}

int m3d_serve_destroy(m3d_server* s) {
    if (!s) return M3D_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (std::thread& t : s->workers) t.join();
    for (auto& e : s->idle) m3d_destroy(e.second.h);
    delete s;
    return M3D_OK;
}

}  // extern "C"
