// oracle/ref_driver_rec.cpp -- TEST INFRASTRUCTURE ONLY (part of the CPU oracle).
//
// A C entry layer over the reference's microstructure reconstruction
// (recon::recPlan, src/rec/reconstruction.cpp), compiled unmodified into
// oracle/_ref/libmat3d_ref.so.  Uses the constructor from a full two-point
// correlation function (:213-240) and runRec(n, beta) (:283-400).  The
// stand-in Eigen's setRandom is a seeded counter-based generator (the
// reference's draws come from std::rand, which is implementation defined), so
// the random initial field and restarts can be reproduced exactly elsewhere.

#include <cstdint>
#include <iostream>
#include <streambuf>

#include "reconstruction.hpp"

namespace {
struct NullBuf : std::streambuf {
    int overflow(int c) override { return c; }
};
struct Quiet {
    NullBuf nb;
    std::streambuf* old;
    Quiet() : old(std::cout.rdbuf(&nb)) {}
    ~Quiet() { std::cout.rdbuf(old); }
};
}  // namespace

extern "C" {

// rve_out: the reconstructed phase field (real part of mTilda after the
// final thresholding), err_out: trackrealerrorA (n values, 0 past the last
// iteration); returns the number of iterations whose error was recorded.
int ref_rec_run(int Nx, int Ny, int Nz, const double* tpcf, int n, double beta, unsigned long long seed,
                double* rve_out, double* err_out) {
    Quiet q;
    Eigen::m3d_rand_seed(seed);
    std::vector<double> t(tpcf, tpcf + (size_t)Nx * Ny * Nz);
    recon::recPlan a(t.data(), Nx, Ny, Nz);
    a.runRec(n, beta);
    const size_t xyz = (size_t)Nx * Ny * Nz;
    for (size_t s = 0; s < xyz; ++s) rve_out[s] = a.mTilda[s][0];
    int cnt = 0;
    for (int i = 0; i < n; ++i) {
        err_out[i] = a.trackrealerrorA(i);
        if (err_out[i] != 0) cnt = i + 1;
    }
    return cnt;
}

// one 3-D complex transform through the same stand-in FFTW plan type the
// reconstruction uses (sign -1 forward, +1 backward, unnormalised), so the
// restatement can be run on exactly the reference's transform when pinning it
int ref_fft3(const double* in, double* out, int Nx, int Ny, int Nz, int sign) {
    const size_t xyz = (size_t)Nx * Ny * Nz;
    fftw_complex* a = new fftw_complex[xyz];
    fftw_complex* b = new fftw_complex[xyz];
    fftw_plan p = fftw_plan_dft_3d(Nx, Ny, Nz, a, b, sign < 0 ? FFTW_FORWARD : FFTW_BACKWARD, FFTW_ESTIMATE);
    for (size_t s = 0; s < xyz; ++s) { a[s][0] = in[2 * s]; a[s][1] = in[2 * s + 1]; }
    fftw_execute(p);
    for (size_t s = 0; s < xyz; ++s) { out[2 * s] = b[s][0]; out[2 * s + 1] = b[s][1]; }
    fftw_destroy_plan(p);
    delete[] a;
    delete[] b;
    return 0;
}

// the reference's ifftshift (:100-140), for building a TPCF centred on index 0
int ref_ifftshift(const double* in, double* out, int Nx, int Ny, int Nz) {
    Quiet q;
    recon::ifftshift(const_cast<double*>(in), out, Nx, Ny, Nz);
    return 0;
}

}  // extern "C"
