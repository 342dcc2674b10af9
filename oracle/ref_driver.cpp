// oracle/ref_driver.cpp -- TEST INFRASTRUCTURE ONLY (part of the CPU oracle).
//
// A C entry layer over the reference's own solver classes, compiled together
// with the unmodified reference sources src/3d/FFT_analysis3D.cpp and
// src/3dTherm/FFT_thermal3D.cpp (see oracle/Makefile) into
// oracle/_ref/libmat3d_ref.so.  Tests and the CPU baseline call it through
// ctypes; nothing in the product links it.
//
// The driver follows the call order of the reference's example drivers
// (example/3d/main.cpp:117-128, example/3d_thermal/main.cpp:93-102) with one
// deliberate change: the thermal single run calls material() before
// setLoad(), because example/3d_thermal/main.cpp:94-95 calls setLoad first and
// then reads uninitialised scheme flags.
//
// Private members (iteration counter, scheme flags, setGF) are read through
// the usual test-harness `#define private public`; class layout is unchanged.

#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <streambuf>
#include <string>
#include <vector>
#include <omp.h>

#include "fftw3.h"
#include <eigen/Eigen/Dense>
#include <CImg.h>
#include "m3d_vtk_stub.h"

#define private public
#include "FFT_analysis3D.hpp"
#include "FFT_thermal3D.hpp"
#undef private

namespace {

// Discards solver chatter but counts the per-iteration lines the reference
// prints from convergenceCheck (src/3d/FFT_analysis3D.cpp:394,
// src/3dTherm/FFT_thermal3D.cpp:340), which gives the total sweep count across
// load increments.
class CountingNullBuf : public std::streambuf {
public:
    long long iter_lines = 0;
    std::string line;
    bool echo = false;

protected:
    int overflow(int ch) override {
        if (ch == EOF) return 0;
        if (echo) std::fputc(ch, stderr);
        if (ch == '\n') {
            if (line.rfind("Itter=", 0) == 0 || line.rfind("Iter=", 0) == 0) ++iter_lines;
            line.clear();
        } else if (line.size() < 16) {
            line.push_back((char)ch);
        }
        return ch;
    }
};

// Wall time of the last run's set-up (constructor: allocation and FFT plans;
// material(): tables and the Green operator; setLoad()) and of its solve
// (runAnalysis / homogenization), for the CPU baseline timing.
double g_setup_s = 0, g_run_s = 0;
double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct QuietScope {
    CountingNullBuf buf;
    std::streambuf* old;
    QuietScope() {
        const char* e = std::getenv("M3D_REF_ECHO");
        buf.echo = e && e[0] == '1';
        old = std::cout.rdbuf(&buf);
    }
    ~QuietScope() { std::cout.rdbuf(old); }
};

}  // namespace

extern "C" {

// Mechanical single analysis (FFT_Analysis3D::runAnalysis,
// src/3d/FFT_analysis3D.cpp:749-854).  `behav` is "e", "ep" or "ed".
// force_scheme: 0 = the reference's automatic choice, 1 = strain-based,
// 2 = stress-based (elastic only; the flags are reset and setGF re-run).
// Outputs are AoS 6 x V column-major (voxel-major), as MatrixDdd::data().
int ref_mech_run(int Nx, int Ny, int Nz, const char* behav, const double* mat, int nph, const int32_t* rve,
                 const double* E6, const double* X06, double tol_field, double tol_eq, int nInc, int force_scheme,
                 int fft_threads, double* eps_out, double* sig_out, double* extra_out, double* prop_out,
                 long long* sweeps_out, int* scheme_out, int* ninc_out, double* la0mu0_out) {
    QuietScope q;
    const int V = Nx * Ny * Nz;
    MatrixDdd m(nph, 7);
    for (int i = 0; i < nph; ++i)
        for (int j = 0; j < 7; ++j) m(i, j) = mat[i * 7 + j];
    MatrixIdd R(1, V);
    for (int i = 0; i < V; ++i) R(i) = rve[i];
    MatrixDdd E(6, 1), X(6, 1);
    for (int i = 0; i < 6; ++i) { E(i) = E6[i]; X(i) = X06[i]; }

    fftw_plan_with_nthreads(fft_threads > 0 ? fft_threads : 3);
    const double t0 = now_s();
    FFT_Analysis3D a(Nx, Ny, Nz, std::string(behav));
    a.material(m, R, nph);
    if (force_scheme == 1 || force_scheme == 2) {
        a.strainBase = (force_scheme == 1);
        a.stressBase = (force_scheme == 2);
        a.setGF();
    }
    a.setLoad(E, X);
    // The constructor sizes the 6x1 mean buffers used by updateE() only for
    // "ep" (src/3d/FFT_analysis3D.cpp:64-65); for "ed" updateE() would write
    // through empty matrices (:575-579) and crash.  Size them here.
    if (a.mater_behav == "ed") {
        a.sigma_iter_old.resize(6, 1);
        a.epsilon_iter_old.resize(6, 1);
    }
    const double t1 = now_s();
    a.runAnalysis(tol_field, tol_eq, nInc);
    g_setup_s = t1 - t0;
    g_run_s = now_s() - t1;

    if (eps_out) std::memcpy(eps_out, a.epsilon.data(), sizeof(double) * 6 * (size_t)V);
    if (sig_out) std::memcpy(sig_out, a.sigma.data(), sizeof(double) * 6 * (size_t)V);
    if (extra_out) {
        if (a.mater_behav == "ep") std::memcpy(extra_out, a.epsilon_p_eff.data(), sizeof(double) * (size_t)V);
        if (a.mater_behav == "ed") std::memcpy(extra_out, a.d.data(), sizeof(double) * (size_t)V);
    }
    if (prop_out && a.mater_behav != "e") {
        const int n = a.prop_homogenized.rows();
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < 9; ++j) prop_out[i * 9 + j] = a.prop_homogenized(i, j);
    }
    if (ninc_out) *ninc_out = (a.mater_behav == "e") ? 1 : (int)a.nInc;
    if (sweeps_out) *sweeps_out = q.buf.iter_lines;
    if (scheme_out) *scheme_out = a.strainBase ? 1 : (a.stressBase ? 2 : 0);
    if (la0mu0_out) { la0mu0_out[0] = a.la0; la0mu0_out[1] = a.mu0; }
    return 0;
}

// Mechanical homogenization (src/3d/FFT_analysis3D.cpp:856-999): six load
// cases -> CHomo, SHomo (6x6), epHomo, sigHomo; the report goes to out_name.txt.
int ref_mech_homog(int Nx, int Ny, int Nz, const double* mat, int nph, const int32_t* rve, double tol_field,
                   double tol_eq, int force_scheme, int fft_threads, const char* out_name, double* C36, double* S36,
                   double* ep36, double* sig36, long long* sweeps_out, int* scheme_out, double* E123) {
    QuietScope q;
    const int V = Nx * Ny * Nz;
    MatrixDdd m(nph, 7);
    for (int i = 0; i < nph; ++i)
        for (int j = 0; j < 7; ++j) m(i, j) = mat[i * 7 + j];
    MatrixIdd R(1, V);
    for (int i = 0; i < V; ++i) R(i) = rve[i];
    fftw_plan_with_nthreads(fft_threads > 0 ? fft_threads : 3);
    FFT_Analysis3D a(Nx, Ny, Nz, "e");
    a.material(m, R, nph);
    if (force_scheme == 1 || force_scheme == 2) {
        a.strainBase = (force_scheme == 1);
        a.stressBase = (force_scheme == 2);
        a.setGF();
    }
    a.homogenization(tol_field, tol_eq, std::string(out_name ? out_name : "/dev/null/x"));
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            C36[i * 6 + j] = a.CHomo(i, j);
            S36[i * 6 + j] = a.SHomo(i, j);
            if (ep36) ep36[i * 6 + j] = a.epHomo(i, j);
            if (sig36) sig36[i * 6 + j] = a.sigHomo(i, j);
        }
    if (sweeps_out) *sweeps_out = q.buf.iter_lines;
    if (scheme_out) *scheme_out = a.strainBase ? 1 : 2;
    if (E123) { E123[0] = a.E11; E123[1] = a.E22; E123[2] = a.E33; }
    return 0;
}

// Thermal single analysis (src/3dTherm/FFT_thermal3D.cpp:446-485).
int ref_therm_run(int Nx, int Ny, int Nz, double km, double ki, const int32_t* rve, const double* E3, double tol_field,
                  double tol_eq, int fft_threads, double* grad_out, double* flux_out, long long* sweeps_out,
                  int* scheme_out) {
    QuietScope q;
    const int V = Nx * Ny * Nz;
    MatrixIdd R(1, V);
    for (int i = 0; i < V; ++i) R(i) = rve[i];
    MatrixDdd E(3, 1);
    for (int i = 0; i < 3; ++i) E(i) = E3[i];
    fftw_plan_with_nthreads(fft_threads > 0 ? fft_threads : 3);
    const double t0 = now_s();
    FFT_analysis3d_thermal a(Nx, Ny, Nz);
    a.material(km, ki, R);
    a.setLoad(E);
    const double t1 = now_s();
    a.runAnalysis(tol_field, tol_eq);
    g_setup_s = t1 - t0;
    g_run_s = now_s() - t1;
    if (grad_out) std::memcpy(grad_out, a.tempGradient.data(), sizeof(double) * 3 * (size_t)V);
    if (flux_out) std::memcpy(flux_out, a.heatFlux.data(), sizeof(double) * 3 * (size_t)V);
    if (sweeps_out) *sweeps_out = q.buf.iter_lines;
    if (scheme_out) *scheme_out = a.tempGradientBase ? 1 : (a.heatFluxBase ? 2 : 0);
    return 0;
}

// Thermal homogenization (src/3dTherm/FFT_thermal3D.cpp:489-622): three unit
// load cases -> KHomo, RHomo (3x3).
int ref_therm_homog(int Nx, int Ny, int Nz, double km, double ki, const int32_t* rve, double tol_field, double tol_eq,
                    int fft_threads, const char* out_name, double* K9, double* R9, long long* sweeps_out,
                    int* scheme_out) {
    QuietScope q;
    const int V = Nx * Ny * Nz;
    MatrixIdd R(1, V);
    for (int i = 0; i < V; ++i) R(i) = rve[i];
    fftw_plan_with_nthreads(fft_threads > 0 ? fft_threads : 3);
    FFT_analysis3d_thermal a(Nx, Ny, Nz);
    a.material(km, ki, R);
    a.homogenization(tol_field, tol_eq, std::string(out_name ? out_name : "/dev/null/x"));
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            K9[i * 3 + j] = a.KHomo(i, j);
            R9[i * 3 + j] = a.RHomo(i, j);
        }
    if (sweeps_out) *sweeps_out = q.buf.iter_lines;
    if (scheme_out) *scheme_out = a.tempGradientBase ? 1 : 2;
    return 0;
}

// The stand-in FFT alone (same guru64 layout as the 3-D solver's forward plan,
// src/3d/FFT_analysis3D.cpp:115-147): c interleaved real fields -> half spectrum.
int ref_fft_r2c(int Nx, int Ny, int Nz, int c, const double* in, double* out_c128) {
    fftw_iodim64 d[3], h[1];
    d[0].n = Nx; d[0].is = (std::ptrdiff_t)Nz * Ny * c; d[0].os = (std::ptrdiff_t)(Nz / 2 + 1) * Ny * c;
    d[1].n = Ny; d[1].is = (std::ptrdiff_t)Nz * c;      d[1].os = (std::ptrdiff_t)(Nz / 2 + 1) * c;
    d[2].n = Nz; d[2].is = c;                           d[2].os = c;
    h[0].n = c; h[0].is = 1; h[0].os = 1;
    std::vector<double> tin(in, in + (size_t)c * Nx * Ny * Nz);
    fftw_plan p = fftw_plan_guru64_dft_r2c(3, d, 1, h, tin.data(), (fftw_complex*)out_c128, FFTW_ESTIMATE);
    fftw_execute(p);
    fftw_destroy_plan(p);
    return 0;
}

int ref_fft_c2r(int Nx, int Ny, int Nz, int c, const double* in_c128, double* out) {
    fftw_iodim64 d[3], h[1];
    d[0].n = Nx; d[0].is = (std::ptrdiff_t)(Nz / 2 + 1) * Ny * c; d[0].os = (std::ptrdiff_t)Nz * Ny * c;
    d[1].n = Ny; d[1].is = (std::ptrdiff_t)(Nz / 2 + 1) * c;      d[1].os = (std::ptrdiff_t)Nz * c;
    d[2].n = Nz; d[2].is = c;                                     d[2].os = c;
    h[0].n = c; h[0].is = 1; h[0].os = 1;
    std::vector<double> tin(in_c128, in_c128 + (size_t)2 * c * Nx * Ny * (Nz / 2 + 1));
    fftw_plan p = fftw_plan_guru64_dft_c2r(3, d, 1, h, (fftw_complex*)tin.data(), out, FFTW_ESTIMATE);
    fftw_execute(p);
    fftw_destroy_plan(p);
    return 0;
}

// set-up and solve wall times (seconds) of the last ref_mech_run / ref_therm_run
void ref_last_timing(double* setup_s, double* run_s) {
    if (setup_s) *setup_s = g_setup_s;
    if (run_s) *run_s = g_run_s;
}

}  // extern "C"
