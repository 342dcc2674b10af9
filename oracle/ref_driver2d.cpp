// oracle/ref_driver2d.cpp -- TEST INFRASTRUCTURE ONLY (part of the CPU oracle).
//
// A C entry layer over the reference's own 2-D solver class FFT_Analysis2D,
// compiled with the unmodified src/2d/FFT_analysis2D.cpp into
// oracle/_ref/libmat3d_ref.so (its own translation unit: the 2-D and 3-D
// headers both define file-scope helpers).  Follows example/2d/main.cpp:
// material(q, RVE), setLoad(E), runAnalysis() (25 basic-scheme iterations).
// The class prints every iteration; its output is discarded here.

#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <streambuf>
#include <string>
#include <unistd.h>

#include "fftw3.h"
#include <eigen/Eigen/Dense>
#include <CImg.h>

#include "FFT_analysis2D.hpp"

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

void setup(FFT_Analysis2D& a, const double* props4, const int32_t* rve, int xy) {
    MatrixDdd R(1, xy);
    for (int i = 0; i < xy; ++i) R(i) = (double)rve[i];
    double q[4] = {props4[0], props4[1], props4[2], props4[3]};
    a.material(q, R);
}
}  // namespace

extern "C" {

// E: 3 complex values as (re, im) pairs; eps/sig out: the class's 3 x xy
// complex matrices as stored (column-major: voxel-major, 3 complex per voxel)
int ref_2d_run(int Nx, int Ny, const double* props4, const int32_t* rve, const double* E, double* eps, double* sig) {
    Quiet q;
    const int xy = Nx * Ny;
    FFT_Analysis2D a(Nx, Ny);
    setup(a, props4, rve, xy);
    MatrixCdd E1(3, 1);
    for (int i = 0; i < 3; ++i) E1(i) = std::complex<double>(E[2 * i], E[2 * i + 1]);
    a.setLoad(E1);
    a.runAnalysis();
    std::memcpy(eps, a.epsilon.data(), sizeof(double) * 2 * 3 * xy);
    std::memcpy(sig, a.sigma.data(), sizeof(double) * 2 * 3 * xy);
    return 0;
}

// setLoad(E) then homogenization(): CHomo (3x3, column-major), epHomo, sigHomo.
// homogenization() writes "Homogenized_Properties" into the working
// directory; it runs in a scratch directory that is removed afterwards.
int ref_2d_homog(int Nx, int Ny, const double* props4, const int32_t* rve, const double* E, double* CH, double* epH,
                 double* sigH) {
    Quiet q;
    const int xy = Nx * Ny;
    FFT_Analysis2D a(Nx, Ny);
    setup(a, props4, rve, xy);
    MatrixCdd E1(3, 1);
    for (int i = 0; i < 3; ++i) E1(i) = std::complex<double>(E[2 * i], E[2 * i + 1]);
    a.setLoad(E1);
    char cwd[4096];
    if (!getcwd(cwd, sizeof(cwd))) return 1;
    char tmpl[] = "/tmp/m3d_ref2d_XXXXXX";
    if (!mkdtemp(tmpl)) return 2;
    if (chdir(tmpl) != 0) return 3;
    a.homogenization();
    if (chdir(cwd) != 0) return 4;
    std::string f = std::string(tmpl) + "/Homogenized_Properties";
    std::remove(f.c_str());
    rmdir(tmpl);
    std::memcpy(CH, a.CHomo.data(), sizeof(double) * 9);
    std::memcpy(epH, a.epHomo.data(), sizeof(double) * 9);
    std::memcpy(sigH, a.sigHomo.data(), sizeof(double) * 9);
    return 0;
}

}  // extern "C"
