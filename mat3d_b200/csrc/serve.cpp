// Serving loop (m3d_serve_*): continuous batching of RVE solves of mixed
// kinds and grid sizes onto one GPU.
//
// Requests enter a FIFO queue.  Worker threads take the first request that can
// start, together with up to kMaxMerge - 1 later queued requests that share its
// shape, precision and stop rule when they are linear (elastic or thermal):
// those run as ONE multi-RVE solve, each request an entry of the batch with its
// own phase map, material, load, stop rule state and result (an entry of a
// multi-RVE solve equals the same solve alone, bitwise).  A resident idle
// solver of the same shape and entry count is reused as is; otherwise a new
// one is created if its device footprint (m3d_footprint_bytes) fits the
// budget, after releasing idle solvers of other shapes, least recently used
// first (a merge that does not fit is halved until it does).  A request that
// cannot start is passed over by later ones at most kMaxBypass times, then it
// waits at the head until memory frees up.
//
// Large solves (a 256^3 grid, or an inelastic one from 96^3) run on
// low-priority streams and at most half the workers hold one at a time; the
// others keep serving small requests, whose streams have the highest
// priority, so a long J2 request neither blocks them in the queue nor starves
// them of SMs.  Solves of different workers overlap on the device.
#include <cuda_runtime.h>

#include <algorithm>
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
constexpr int kMaxMerge = 8;

struct Req {
    long long ticket = 0;
    m3d_request r{};
    std::vector<double> mat;
    std::vector<int32_t> phase;
    double E[6] = {}, X0[6] = {};
    bool hasX0 = false;
    ShapeKey key;
    long long bytes = 0;
    bool linear = false;  // elastic or thermal: may share a multi-RVE solve
    bool big = false;     // runs on a low-priority stream, at most half the workers
    int bypassed = 0;
    Clock::time_point t_submit, t_admit;
};

// requests solved together (one solver, one entry each)
struct Group {
    std::vector<std::unique_ptr<Req>> reqs;
    long long bytes = 0;
    bool big = false;
};

// idle solvers are keyed by shape and entry count
typedef std::pair<ShapeKey, int> SolverKey;

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

bool same_rule(const Req& a, const Req& b) {
    return a.key == b.key && a.linear && b.linear && a.r.tol == b.r.tol && a.r.max_iter == b.r.max_iter;
}

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
    std::multimap<SolverKey, Idle> idle;
    long long next_ticket = 1;
    double resident = 0;  // bytes of all solvers held (running + idle)
    int running = 0, peak_running = 0, n_solvers = 0, running_big = 0, big_max = 1;
    long long submitted = 0, completed = 0, failed = 0, merged_solves = 0, merged_requests = 0;
    bool stop = false;
    std::vector<std::thread> workers;

    void worker();
    bool pick(Group& g, m3d_solver** reuse, long long* reserved, std::vector<m3d_solver*>& evict);
    int solve(Group& g, m3d_solver* h, std::vector<Done>& d);
};

// Under `mu`.  The first queued request that can start now, with the later
// requests it can share a solve with: an idle solver of that shape and entry
// count is reused, or the group's footprint must fit after releasing idle
// solvers of other shapes (least recently used first); a merge that does not
// fit is halved.  Bypassing is bounded; big requests wait (without counting
// as bypassed) while half the workers hold big solves.
bool m3d_server::pick(Group& g, m3d_solver** reuse, long long* reserved, std::vector<m3d_solver*>& evict) {
    *reuse = nullptr;
    *reserved = 0;
    for (size_t i = 0; i < queue.size(); ++i) {
        Req& q = *queue[i];
        if (q.big && running_big >= big_max) continue;
        std::vector<size_t> mates{i};
        if (q.linear)
            for (size_t j = i + 1; j < queue.size() && (int)mates.size() < kMaxMerge; ++j)
                if (same_rule(q, *queue[j])) mates.push_back(j);
        bool ok = false;
        long long bytes = 0;
        for (int k = (int)mates.size(); k >= 1 && !ok; k /= 2) {
            const m3d_request& r = q.r;
            bytes = (k == 1) ? q.bytes : m3d_footprint_bytes(r.kind, r.Nx, r.Ny, r.Nz, r.behav, r.precision, k, k);
            auto it = idle.find(SolverKey(q.key, k));
            if (it != idle.end()) {
                *reuse = it->second.h;
                idle.erase(it);
                ok = true;
            } else {
                double idle_bytes = 0;
                for (auto& e : idle) idle_bytes += (double)e.second.bytes;
                if (resident - idle_bytes + (double)bytes <= budget) {
                    while (resident + (double)bytes > budget && !idle.empty()) {
                        auto lru = idle.begin();
                        for (auto e = idle.begin(); e != idle.end(); ++e)
                            if (e->second.last < lru->second.last) lru = e;
                        evict.push_back(lru->second.h);
                        resident -= (double)lru->second.bytes;
                        --n_solvers;
                        idle.erase(lru);
                    }
                    resident += (double)bytes;
                    ++n_solvers;
                    *reserved = bytes;
                    ok = true;
                }
            }
            if (ok) mates.resize(k);
        }
        if (ok) {
            g.bytes = bytes;
            g.big = q.big;
            for (size_t m = mates.size(); m-- > 0;) {  // highest index first: erasing keeps lower indices valid
                g.reqs.push_back(std::move(queue[mates[m]]));
                queue.erase(queue.begin() + (long)mates[m]);
            }
            std::reverse(g.reqs.begin(), g.reqs.end());
            for (size_t j = 0; j < i; ++j) queue[j]->bypassed += 1;
            return true;
        }
        if (q.bypassed >= kMaxBypass) break;  // keep FIFO order behind a starved request
    }
    return false;
}

// One solve for the group: entry b holds request b (its RVE, load and stop
// rule state); each request's result is its own entry's.
int m3d_server::solve(Group& g, m3d_solver* h, std::vector<Done>& d) {
    const int n = (int)g.reqs.size();
    for (int b = 0; b < n; ++b) {
        const Req& q = *g.reqs[b];
        const m3d_request& r = q.r;
        int rc = (r.kind == M3D_KIND_MECH)
                     ? m3d_set_material_mech_rve(h, b, q.mat.data(), r.nph, q.phase.data(), r.scheme)
                     : m3d_set_material_thermal_rve(h, b, r.km, r.ki, q.phase.data(), r.scheme);
        if (rc) return rc;
        rc = m3d_set_load(h, b, q.E, q.hasX0 ? q.X0 : nullptr);
        if (rc) return rc;
    }
    const m3d_request& r0 = g.reqs[0]->r;
    const int st = m3d_run(h, r0.tol, 0.0, r0.nInc, M3D_CRIT_RESIDUAL, r0.max_iter);
    if (st != M3D_OK && st != M3D_NOT_CONVERGED) return st;
    m3d_stats s;
    m3d_get_stats(h, &s);
    for (int b = 0; b < n; ++b) {
        const Req& q = *g.reqs[b];
        m3d_result& res = d[b].res;
        int rc = m3d_get_means(h, b, res.strain_mean, res.stress_mean);
        if (rc) return rc;
        if (q.linear) {
            rc = m3d_get_entry_stats(h, b, &res.iters, &res.sweeps, &res.residual, &res.status);
            if (rc) return rc;
        } else {
            res.iters = s.iters;
            res.sweeps = s.sweeps;
            res.residual = s.residual;
            res.status = st;
        }
        if (q.r.keep_field) {
            const int C = (q.r.kind == M3D_KIND_MECH) ? 6 : 3;
            d[b].field.assign((size_t)C * q.r.Nx * q.r.Ny * q.r.Nz, 0.0);
            rc = m3d_get_field(h, M3D_FIELD_STRAIN, b, d[b].field.data());
            if (rc) return rc;
            d[b].keep_field = true;
        }
    }
    return M3D_OK;
}

void m3d_server::worker() {
    cudaSetDevice(dev);
    // two streams per worker: the highest priority for small solves, the
    // lowest for big ones (a solver runs on the worker's stream while it is
    // held, and goes back to its own stream when idle)
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    cudaStream_t s_hi = nullptr, s_lo = nullptr;
    cudaStreamCreateWithPriority(&s_hi, cudaStreamNonBlocking, hi);
    cudaStreamCreateWithPriority(&s_lo, cudaStreamNonBlocking, lo);
    for (;;) {
        Group g;
        m3d_solver* h = nullptr;
        long long reserved = 0;
        std::vector<m3d_solver*> evict;
        {
            std::unique_lock<std::mutex> lk(mu);
            bool got = false;
            for (;;) {
                if (!queue.empty()) got = pick(g, &h, &reserved, evict);
                if (got || (stop && queue.empty())) break;
                cv_work.wait(lk);
            }
            if (!got) break;
            ++running;
            if (g.big) ++running_big;
            if (running > peak_running) peak_running = running;
            if (g.reqs.size() > 1) {
                ++merged_solves;
                merged_requests += (long long)g.reqs.size();
            }
        }
        for (m3d_solver* e : evict) m3d_destroy(e);
        const auto t_admit = Clock::now();
        const int n = (int)g.reqs.size();
        std::vector<Done> d((size_t)n);
        int rc = M3D_OK;
        const m3d_request& r = g.reqs[0]->r;
        if (!h) {
            rc = g.reqs[0]->linear ? m3d_create_multi(r.kind, r.Nx, r.Ny, r.Nz, r.precision, n, 1, &h)
                                   : m3d_create(r.kind, r.Nx, r.Ny, r.Nz, r.behav, r.precision, 1, &h);
            if (rc) h = nullptr;
        }
        if (h) {
            m3d_set_stream(h, g.big ? s_lo : s_hi);
            rc = solve(g, h, d);
            m3d_set_stream(h, nullptr);
        }
        const auto t_done = Clock::now();
        {
            std::lock_guard<std::mutex> lk(mu);
            if (h) {
                idle.insert(std::make_pair(SolverKey(g.reqs[0]->key, n), Idle{h, g.bytes, t_done}));
            } else if (reserved) {
                resident -= (double)reserved;
                --n_solvers;
            }
            --running;
            if (g.big) --running_big;
            for (int b = 0; b < n; ++b) {
                Req& q = *g.reqs[b];
                Done& dd = d[b];
                if (rc != M3D_OK) dd.res.status = rc;
                dd.res.queue_ms = ms_between(q.t_submit, t_admit);
                dd.res.solve_ms = ms_between(t_admit, t_done);
                dd.res.latency_ms = ms_between(q.t_submit, t_done);
                ++completed;
                if (dd.res.status != M3D_OK && dd.res.status != M3D_NOT_CONVERGED) ++failed;
                pending.erase(q.ticket);
                done[q.ticket] = std::move(dd);
            }
        }
        cv_done.notify_all();
        cv_work.notify_all();
    }
    cudaStreamDestroy(s_hi);
    cudaStreamDestroy(s_lo);
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
    s->big_max = std::max(1, workers / 2);
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
    q->linear = (r.kind == M3D_KIND_THERMAL || r.behav == M3D_BEHAV_ELASTIC);
    q->big = (long long)V >= 192LL * 192 * 192 || (!q->linear && (long long)V >= 96LL * 96 * 96);
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
    out->merged_solves = s->merged_solves;
    out->merged_requests = s->merged_requests;
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
