// oracle/ref_driver_rec.cpp -- TEST INFRASTRUCTURE ONLY (part of the CPU oracle).
//
// A C entry layer over the reference's microstructure reconstruction
// (recon::recPlan, src/rec/reconstruction.cpp), compiled unmodified into
// oracle/_ref/libmat3d_ref.so.  Uses the constructor from a full two-point
// correlation function (:213-240) and runRec(n, beta) (:283-400).  The
// stand-in Eigen's setRandom is a seeded counter-based generator (the
// reference's draws come from std::rand, which is implementation defined), so
// the random initial field and restarts can be reproduced exactly elsewhere.

#include <unistd.h>

#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <streambuf>

// Everything reconstruction.hpp includes, first, so that the access override
// below reaches only the recPlan class (the section pin reads its private
// normC after estimateNormFFT_RVE).  M3D_REF_CIMG is the reference's own
// vendored CImg.h, the file reconstruction.hpp includes by a quoted path.
#include <eigen/Eigen/Dense>
#include "fftw3.h"
#include M3D_REF_CIMG
#include "omp.h"
#include <vtkActor.h>
#include <vtkImageData.h>
#include <vtkImageDataGeometryFilter.h>
#include <vtkPolyDataMapper.h>
#include <vtkProperty.h>
#include <vtkRenderWindow.h>
#include <vtkRenderWindowInteractor.h>
#include <vtkRenderer.h>
#include <vtkSmartPointer.h>
#include <vtkVersion.h>
#include <vtkXMLImageDataReader.h>
#include <vtkXMLImageDataWriter.h>
#define private public
#include "reconstruction.hpp"
#undef private

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

// recPlan(CImg c1, CImg c2) (:145-206) from 8-bit sections stored x fastest,
// then estimateNormFFT_RVE() (:245-281); normC out (xyz = w1 * h1 * h2).
// estimateNormFFT_RVE writes normc.txt into the working directory; it runs in
// a scratch directory that is removed afterwards.
int ref_rec_sections(const unsigned char* c1, int w1, int h1, const unsigned char* c2, int w2, int h2,
                     double* normC_out) {
    Quiet q;
    cimg_library::CImg<unsigned char> C1(c1, w1, h1, 1, 1), C2(c2, w2, h2, 1, 1);
    recon::recPlan a(C1, C2);
    char cwd[4096];
    if (!getcwd(cwd, sizeof(cwd))) return 1;
    char tmpl[] = "/tmp/m3d_refrec_XXXXXX";
    if (!mkdtemp(tmpl)) return 2;
    if (chdir(tmpl) != 0) return 3;
    a.estimateNormFFT_RVE();
    if (chdir(cwd) != 0) return 4;
    std::string f = std::string(tmpl) + "/normc.txt";
    std::remove(f.c_str());
    rmdir(tmpl);
    const size_t xyz = (size_t)a.Nx * a.Ny * a.Nz;
    for (size_t s = 0; s < xyz; ++s) normC_out[s] = a.normC[s];
    return 0;
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
