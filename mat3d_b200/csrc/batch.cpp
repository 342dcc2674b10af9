// Batched homogenization of many RVEs of mixed grid sizes (m3d_batch_*).
//
// The reference homogenizes one RVE per FFT_Analysis3D / FFT_analysis3d_thermal
// object, its load cases one after another (src/3d/FFT_analysis3D.cpp:856-903,
// src/3dTherm/FFT_thermal3D.cpp:489-580).  Here the RVEs added to a batch are
// grouped by grid size; each group runs as multi-RVE solvers (every RVE with
// all its load cases as entries of one batch, the whole iteration one CUDA
// graph launch), split into as few launches as the device-memory budget
// allows.  Each RVE keeps the reference's own setup (scheme, reference
// medium, load magnitudes and tensor assembly), so its tensor is the one
// m3d_homogenize gives for it alone.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <string>
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
    std::vector<std::pair<std::tuple<int, int, int>, std::vector<int>>> order(groups.begin(), groups.end());
    std::sort(order.begin(), order.end(), [](const auto& a, const auto& c) {
        const auto& x = a.first;
        const auto& y = c.first;
        return (long long)std::get<0>(x) * std::get<1>(x) * std::get<2>(x) >
               (long long)std::get<0>(y) * std::get<1>(y) * std::get<2>(y);
    });
    int status = M3D_OK;
    std::vector<double> Ce, Se;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
        return bfail(M3D_ERR_CUDA, "event creation failed");
    int rc = M3D_OK;
    for (auto& grp : order) {
        const int Nx = std::get<0>(grp.first), Ny = std::get<1>(grp.first), Nz = std::get<2>(grp.first);
        const std::vector<int>& ids = grp.second;
        const long long V = (long long)Nx * Ny * Nz;
        // RVEs per launch within the memory budget (footprint is affine in the RVE count)
        const long long f1 = m3d_footprint_bytes(b->kind, Nx, Ny, Nz, M3D_BEHAV_ELASTIC, b->prec, 1, C);
        const long long f2 = m3d_footprint_bytes(b->kind, Nx, Ny, Nz, M3D_BEHAV_ELASTIC, b->prec, 2, 2 * C);
        const long long per = f2 - f1, base = f1 - per;
        long long rmax = (long long)((b->budget - (double)base) / (double)per);
        rmax = std::max(1LL, std::min<long long>(rmax, 8192 / C));
        if ((double)(base + per) > b->budget) { rc = bfail(M3D_ERR_OOM, "one RVE of this grid exceeds the memory budget"); break; }
        const int n = (int)ids.size();
        const int nchunks = (int)((n + rmax - 1) / rmax);
        const int R = (n + nchunks - 1) / nchunks;
        m3d_solver* h = nullptr;
        int hR = 0;
        for (int c0 = 0; c0 < n && rc == M3D_OK; c0 += R) {
            const int r = std::min(R, n - c0);
            if (h && hR != r) { m3d_destroy(h); h = nullptr; }
            if (!h) {
                rc = m3d_create_multi(b->kind, Nx, Ny, Nz, b->prec, r, C, &h);
                if (rc) break;
                hR = r;
            }
            for (int k = 0; k < r && rc == M3D_OK; ++k) {
                const BatchRve& m = b->rves[ids[c0 + k]];
                rc = (b->kind == M3D_KIND_MECH)
                         ? m3d_set_material_mech_rve(h, k, m.mat.data(), m.nph, m.phase.data(), m.scheme)
                         : m3d_set_material_thermal_rve(h, k, m.km, m.ki, m.phase.data(), m.scheme);
            }
            if (rc) break;
            if (b->autotune) {
                // time the schedules on the group's first solver, reuse the choice afterwards
                m3d_tune t;
                rc = m3d_autotune(h, c0 == 0 ? 3 : 0, &t);
                if (rc) break;
                if (c0 == 0) b->st.autotuned += 1;
            }
            Ce.assign((size_t)r * C * C, 0.0);
            Se.assign((size_t)r * C * C, 0.0);
            cudaStream_t s = (cudaStream_t)m3d_get_stream(h);
            cudaEventRecord(e0, s);
            const int hs = m3d_homogenize(h, tol_field, 0, M3D_CRIT_RESIDUAL, max_iter, Ce.data(), Se.data(), nullptr, nullptr);
            cudaEventRecord(e1, s);
            if (hs != M3D_OK && hs != M3D_NOT_CONVERGED) { rc = hs; break; }
            if (hs == M3D_NOT_CONVERGED) status = M3D_NOT_CONVERGED;
            cudaEventSynchronize(e1);
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            m3d_stats hst;
            m3d_get_stats(h, &hst);
            b->st.device_ms += ms;
            b->st.sweeps += hst.sweeps;
            b->st.sweeps_fp64 += hst.sweeps_fp64;
            b->st.sweeps_fp32 += hst.sweeps_fp32;
            b->st.voxel_iters += hst.sweeps * V;
            b->st.launches += 1;
            for (int k = 0; k < r; ++k) {
                const int i = ids[c0 + k];
                if (Ceff) std::memcpy(Ceff + (size_t)i * C * C, &Ce[(size_t)k * C * C], C * C * sizeof(double));
                if (Seff) std::memcpy(Seff + (size_t)i * C * C, &Se[(size_t)k * C * C], C * C * sizeof(double));
            }
        }
        if (h) {
            m3d_stats hst;
            m3d_get_stats(h, &hst);
            b->st.kernel_launches += hst.kernel_launches;
            m3d_destroy(h);
        }
        b->st.groups += 1;
        if (rc) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
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
