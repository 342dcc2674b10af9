// Batched homogenization of many RVEs of mixed grid sizes (m3d_batch_*).
//
// The reference homogenizes one RVE per FFT_Analysis3D / FFT_analysis3d_thermal
// object, its load cases one after another (src/3d/FFT_analysis3D.cpp:856-903,
// src/3dTherm/FFT_thermal3D.cpp:489-580).  Here the RVEs added to a batch are
// grouped by grid size; each group runs as multi-RVE solvers (every RVE with
// all its load cases as entries of one batch, the whole iteration one CUDA
// graph launch).  When all groups fit the device-memory budget together they
// run concurrently -- one host thread and stream per group, their graph
// launches overlapping on the device -- otherwise one after another, each
// split into as few launches as the budget allows.  Each RVE keeps the reference's own setup (scheme, reference
// medium, load magnitudes and tensor assembly), so its tensor is the one
// m3d_homogenize gives for it alone.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "mat3d_b200.h"

void m3d_internal_set_error(const std::string& msg);

namespace {

struct BatchRve {
    int Nx, Ny, Nz;
    std::vector<double> mat;  // mech: nph x 7
    int nph = 0;
    double km = 0, ki = 0;    // thermal
    std::vector<int32_t> phase;
    int scheme = 0;
};

int bfail(int code, const std::string& msg) {
    m3d_internal_set_error(msg);
    return code;
}

}  // namespace

struct m3d_batch {
    int kind = 0, prec = 0;
    double budget = 0;  // bytes
    std::vector<BatchRve> rves;
    m3d_batch_stats st{};
    bool autotune = false;
};

extern "C" {

int m3d_batch_create(int kind, int precision, double mem_budget_bytes, m3d_batch** out) {
    if (!out) return bfail(M3D_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (kind != M3D_KIND_MECH && kind != M3D_KIND_THERMAL) return bfail(M3D_ERR_ARG, "kind must be MECH or THERMAL");
    if (precision < 0 || precision > 2) return bfail(M3D_ERR_ARG, "invalid precision");
    if (!(mem_budget_bytes > 0)) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return bfail(M3D_ERR_CUDA, "no CUDA device");
        mem_budget_bytes = 0.85 * (double)fr;
    }
    m3d_batch* b = new m3d_batch();
    b->kind = kind;
    b->prec = precision;
    b->budget = mem_budget_bytes;
    *out = b;
    return M3D_OK;
}

int m3d_batch_destroy(m3d_batch* b) {
    delete b;
    return M3D_OK;
}

int m3d_batch_clear(m3d_batch* b) {
    if (!b) return bfail(M3D_ERR_ARG, "NULL batch");
    b->rves.clear();
    return M3D_OK;
}

static int add_common(m3d_batch* b, int Nx, int Ny, int Nz, const int32_t* phase, int scheme, BatchRve& r) {
    if (!b || !phase) return bfail(M3D_ERR_ARG, "NULL argument");
    if (Nx < 2 || Ny < 2 || Nz < 2 || Nx > 1024 || Ny > 1024 || Nz > 1024)
        return bfail(M3D_ERR_ARG, "grid sizes must be in [2, 1024]");
    if (scheme < 0 || scheme > 2) return bfail(M3D_ERR_ARG, "invalid scheme");
    r.Nx = Nx; r.Ny = Ny; r.Nz = Nz;
    r.scheme = scheme;
    r.phase.assign(phase, phase + (size_t)Nx * Ny * Nz);
    return M3D_OK;
}

int m3d_batch_add_mech(m3d_batch* b, int Nx, int Ny, int Nz, const double* mat, int nph, const int32_t* phase,
                       int scheme, int* index) {
    if (!b || !mat) return bfail(M3D_ERR_ARG, "NULL argument");
    if (b->kind != M3D_KIND_MECH) return bfail(M3D_ERR_ARG, "not a mechanical batch");
    if (nph < 1 || nph > 16) return bfail(M3D_ERR_ARG, "nph must be in [1, 16]");
    BatchRve r;
    int rc = add_common(b, Nx, Ny, Nz, phase, scheme, r);
    if (rc) return rc;
    r.nph = nph;
    r.mat.assign(mat, mat + (size_t)nph * 7);
    b->rves.push_back(std::move(r));
    if (index) *index = (int)b->rves.size() - 1;
    return M3D_OK;
}

int m3d_batch_add_thermal(m3d_batch* b, int Nx, int Ny, int Nz, double km, double ki, const int32_t* phase,
                          int scheme, int* index) {
    if (!b) return bfail(M3D_ERR_ARG, "NULL batch");
    if (b->kind != M3D_KIND_THERMAL) return bfail(M3D_ERR_ARG, "not a thermal batch");
    if (!(km > 0) || !(ki > 0)) return bfail(M3D_ERR_ARG, "conductivities must be positive");
    BatchRve r;
    int rc = add_common(b, Nx, Ny, Nz, phase, scheme, r);
    if (rc) return rc;
    r.km = km;
    r.ki = ki;
    b->rves.push_back(std::move(r));
    if (index) *index = (int)b->rves.size() - 1;
    return M3D_OK;
}

// One grid-size group: its RVE ids, launch chunk size and the handle of its
// first chunk (made and, when autotuning, tuned before the groups run).
struct GroupPlan {
    int Nx = 0, Ny = 0, Nz = 0;
    std::vector<int> ids;
    int R = 1;                  // RVEs per launch
    long long bytes = 0;        // device footprint of one launch
    m3d_solver* h = nullptr;    // first chunk's handle
    int hR = 0;
    // results of the run
    int rc = M3D_OK, status = M3D_OK;
    std::string err;
    double ms = 0;
    long long sweeps = 0, s64 = 0, s32 = 0, vi = 0, kl = 0;
    int launches = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;  // first start / last end on the group's stream
};

static int set_rves(m3d_batch* b, m3d_solver* h, const std::vector<int>& ids, int c0, int r) {
    for (int k = 0; k < r; ++k) {
        const BatchRve& m = b->rves[ids[c0 + k]];
        const int rc = (b->kind == M3D_KIND_MECH)
                           ? m3d_set_material_mech_rve(h, k, m.mat.data(), m.nph, m.phase.data(), m.scheme)
                           : m3d_set_material_thermal_rve(h, k, m.km, m.ki, m.phase.data(), m.scheme);
        if (rc) return rc;
    }
    return M3D_OK;
}

// Runs every chunk of one group on its own handle(s) and stream.
static void run_group(m3d_batch* b, GroupPlan& gp, int C, double tol_field, int max_iter, double* Ceff, double* Seff) {
    const long long V = (long long)gp.Nx * gp.Ny * gp.Nz;
    const int n = (int)gp.ids.size();
    std::vector<double> Ce, Se;
    cudaEvent_t a = nullptr, z = nullptr;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&z) != cudaSuccess) {
        gp.rc = M3D_ERR_CUDA;
        gp.err = "event creation failed";
        return;
    }
    for (int c0 = 0; c0 < n; c0 += gp.R) {
        const int r = std::min(gp.R, n - c0);
        if (gp.h && gp.hR != r) {
            m3d_stats hst;
            m3d_get_stats(gp.h, &hst);
            gp.kl += hst.kernel_launches;
            m3d_destroy(gp.h);
            gp.h = nullptr;
        }
        int rc = M3D_OK;
        if (!gp.h) {
            rc = m3d_create_multi(b->kind, gp.Nx, gp.Ny, gp.Nz, b->prec, r, C, &gp.h);
            if (!rc) gp.hR = r;
            if (!rc && b->autotune) { m3d_tune t; rc = m3d_autotune(gp.h, 0, &t); }  // the group's tuned choice
        }
        if (!rc && c0 > 0) rc = set_rves(b, gp.h, gp.ids, c0, r);
        if (rc) { gp.rc = rc; gp.err = m3d_last_error(); break; }
        Ce.assign((size_t)r * C * C, 0.0);
        Se.assign((size_t)r * C * C, 0.0);
        cudaStream_t s = (cudaStream_t)m3d_get_stream(gp.h);
        cudaEventRecord(a, s);
        if (c0 == 0) cudaEventRecord(gp.e0, s);
        const int hs = m3d_homogenize(gp.h, tol_field, 0, M3D_CRIT_RESIDUAL, max_iter, Ce.data(), Se.data(), nullptr,
                                      nullptr);
        cudaEventRecord(z, s);
        cudaEventRecord(gp.e1, s);
        if (hs != M3D_OK && hs != M3D_NOT_CONVERGED) { gp.rc = hs; gp.err = m3d_last_error(); break; }
        if (hs == M3D_NOT_CONVERGED) gp.status = M3D_NOT_CONVERGED;
        cudaEventSynchronize(z);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, z);
        m3d_stats hst;
        m3d_get_stats(gp.h, &hst);
        gp.ms += ms;
        gp.sweeps += hst.sweeps;
        gp.s64 += hst.sweeps_fp64;
        gp.s32 += hst.sweeps_fp32;
        gp.vi += hst.sweeps * V;
        gp.launches += 1;
        for (int k = 0; k < r; ++k) {
            const int i = gp.ids[c0 + k];
            if (Ceff) std::memcpy(Ceff + (size_t)i * C * C, &Ce[(size_t)k * C * C], C * C * sizeof(double));
            if (Seff) std::memcpy(Seff + (size_t)i * C * C, &Se[(size_t)k * C * C], C * C * sizeof(double));
        }
    }
    if (gp.h) {
        m3d_stats hst;
        m3d_get_stats(gp.h, &hst);
        gp.kl += hst.kernel_launches;
        m3d_destroy(gp.h);
        gp.h = nullptr;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(z);
}

int m3d_batch_homogenize(m3d_batch* b, double tol_field, int max_iter, double* Ceff, double* Seff) {
    if (!b) return bfail(M3D_ERR_ARG, "NULL batch");
    if (!(tol_field > 0)) return bfail(M3D_ERR_ARG, "tolerance must be positive");
    const auto w0 = std::chrono::steady_clock::now();
    const int C = (b->kind == M3D_KIND_MECH) ? 6 : 3;
    std::memset(&b->st, 0, sizeof(b->st));
    // groups by grid, largest grids first
    std::map<std::tuple<int, int, int>, std::vector<int>> groups;
    for (int i = 0; i < (int)b->rves.size(); ++i) {
        const BatchRve& r = b->rves[i];
        groups[std::make_tuple(r.Nx, r.Ny, r.Nz)].push_back(i);
    }
    std::vector<GroupPlan> plans;
    for (auto& kv : groups) {
        GroupPlan gp;
        gp.Nx = std::get<0>(kv.first); gp.Ny = std::get<1>(kv.first); gp.Nz = std::get<2>(kv.first);
        gp.ids = kv.second;
        plans.push_back(std::move(gp));
    }
    std::sort(plans.begin(), plans.end(), [](const GroupPlan& a, const GroupPlan& c) {
        return (long long)a.Nx * a.Ny * a.Nz > (long long)c.Nx * c.Ny * c.Nz;
    });
    // Launch sizes.  All groups run at once (one host thread and stream each,
    // their graph launches overlapping on the device) when their launches fit
    // the budget together; otherwise one group after another, each using the
    // whole budget.  The footprint is affine in the RVE count.
    auto chunking = [&](GroupPlan& gp, double budget) -> int {
        const long long f1 = m3d_footprint_bytes(b->kind, gp.Nx, gp.Ny, gp.Nz, M3D_BEHAV_ELASTIC, b->prec, 1, C);
        const long long f2 = m3d_footprint_bytes(b->kind, gp.Nx, gp.Ny, gp.Nz, M3D_BEHAV_ELASTIC, b->prec, 2, 2 * C);
        const long long per = f2 - f1, base = f1 - per;
        if ((double)(base + per) > budget) return bfail(M3D_ERR_OOM, "one RVE of this grid exceeds the memory budget");
        long long rmax = (long long)((budget - (double)base) / (double)per);
        rmax = std::max(1LL, std::min<long long>(rmax, 8192 / C));
        const int n = (int)gp.ids.size();
        const int nchunks = (int)((n + rmax - 1) / rmax);
        gp.R = (n + nchunks - 1) / nchunks;
        gp.bytes = base + per * gp.R;
        return M3D_OK;
    };
    int rc = M3D_OK;
    bool together = plans.size() > 1;
    long long need = 0;
    for (GroupPlan& gp : plans) {
        rc = chunking(gp, b->budget);
        if (rc) return rc;
        const long long f1 = m3d_footprint_bytes(b->kind, gp.Nx, gp.Ny, gp.Nz, M3D_BEHAV_ELASTIC, b->prec, 1, C);
        const long long f2 = m3d_footprint_bytes(b->kind, gp.Nx, gp.Ny, gp.Nz, M3D_BEHAV_ELASTIC, b->prec, 2, 2 * C);
        need += (f1 - (f2 - f1)) + (f2 - f1) * (long long)gp.ids.size();  // the whole group in one launch
    }
    together = together && (double)need <= b->budget;
    if (together)
        for (GroupPlan& gp : plans) gp.R = (int)gp.ids.size();
    // handles of the first chunks, materials set and (sequentially, on an idle
    // device) the schedules tuned and the solve graphs captured
    for (GroupPlan& gp : plans) {
        const int r = std::min<int>(gp.R, (int)gp.ids.size());
        rc = m3d_create_multi(b->kind, gp.Nx, gp.Ny, gp.Nz, b->prec, r, C, &gp.h);
        if (rc) break;
        gp.hR = r;
        rc = set_rves(b, gp.h, gp.ids, 0, r);
        if (rc) break;
        if (b->autotune) {
            m3d_tune t;
            rc = m3d_autotune(gp.h, 3, &t);
            if (rc) break;
            b->st.autotuned += 1;
        }
        // capture the handle's solve graph now (a one-sweep solve), so that
        // the group's timed launch below carries no host-side capture
        {
            const int hs = m3d_homogenize(gp.h, tol_field, 0, M3D_CRIT_RESIDUAL, 1, nullptr, nullptr, nullptr, nullptr);
            if (hs != M3D_OK && hs != M3D_NOT_CONVERGED) { rc = hs; break; }
        }
        if (cudaEventCreate(&gp.e0) != cudaSuccess || cudaEventCreate(&gp.e1) != cudaSuccess) {
            rc = bfail(M3D_ERR_CUDA, "event creation failed");
            break;
        }
    }
    if (rc == M3D_OK) {
        if (together) {
            std::vector<std::thread> th;
            int dev = 0;
            cudaGetDevice(&dev);
            for (GroupPlan& gp : plans)
                th.emplace_back([&, dev, p = &gp] {
                    cudaSetDevice(dev);
                    run_group(b, *p, C, tol_field, max_iter, Ceff, Seff);
                });
            for (auto& t : th) t.join();
        } else {
            for (GroupPlan& gp : plans) run_group(b, gp, C, tol_field, max_iter, Ceff, Seff);
        }
    }
    // device time: from the first group's start to the last group's end
    int status = M3D_OK;
    cudaEvent_t first = nullptr, last = nullptr;
    float span = 0;
    for (GroupPlan& gp : plans) {
        if (gp.h) { m3d_destroy(gp.h); gp.h = nullptr; }
        if (rc == M3D_OK && gp.rc != M3D_OK) {
            rc = gp.rc;
            m3d_internal_set_error(gp.err);
        }
        if (gp.status == M3D_NOT_CONVERGED) status = M3D_NOT_CONVERGED;
        b->st.sweeps += gp.sweeps;
        b->st.sweeps_fp64 += gp.s64;
        b->st.sweeps_fp32 += gp.s32;
        b->st.voxel_iters += gp.vi;
        b->st.launches += gp.launches;
        b->st.kernel_launches += gp.kl;
        b->st.groups += 1;
        if (gp.e0 && gp.e1 && gp.launches) {
            float t = 0;
            if (!first || (cudaEventElapsedTime(&t, first, gp.e0) == cudaSuccess && t < 0)) first = gp.e0;
            if (!last || (cudaEventElapsedTime(&t, last, gp.e1) == cudaSuccess && t > 0)) last = gp.e1;
        }
    }
    if (first && last && cudaEventElapsedTime(&span, first, last) == cudaSuccess) b->st.device_ms = span;
    else for (GroupPlan& gp : plans) b->st.device_ms += gp.ms;
    for (GroupPlan& gp : plans) {
        if (gp.e0) cudaEventDestroy(gp.e0);
        if (gp.e1) cudaEventDestroy(gp.e1);
    }
    (void)cudaGetLastError();
    b->st.concurrent = together ? 1 : 0;
    b->st.wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - w0).count();
    b->st.rves = (int)b->rves.size();
    if (rc) return rc;
    return status;
}

int m3d_batch_set_autotune(m3d_batch* b, int on) {
    if (!b) return bfail(M3D_ERR_ARG, "NULL batch");
    b->autotune = on != 0;
    return M3D_OK;
}

int m3d_batch_get_stats(const m3d_batch* b, m3d_batch_stats* out) {
    if (!b || !out) return bfail(M3D_ERR_ARG, "NULL argument");
    *out = b->st;
    return M3D_OK;
}

}  // extern "C"
