// reconstruction.hpp -- drop-in replacement for the reference's microstructure
// reconstruction header (include/reconstruction.hpp:1-98 of FayyazNo/MAT3d).
//
// Same namespace (recon), free functions fftshift / ifftshift, class recPlan
// with its two constructors, estimateNormFFT_RVE, runRec, saveRecImages,
// vtiWriter and the public members trackrealerrorA and mTilda; the work runs
// on the GPU through the C ABI in mat3d_b200.h (link -lmat3d_b200).
// Differences from the reference, all deliberate:
//   * no FFTW, Eigen, CImg or VTK dependency: the header carries the subset a
//     caller of the reference uses -- fftw_complex and one-shot 2-D/3-D complex
//     plans (executed on the GPU; skipped when the real fftw3.h came first), a
//     minimal 8-bit image type cimg_library::CImg (skipped when the real CImg
//     came first) and the matrix type MatrixDdd of mat3d_matrix.hpp;
//   * the random draws come from the library's seeded generator (seed(),
//     default 1) instead of std::rand;
//   * saveRecImages writes each x slice as an Ny x Nz PNG itself (the
//     reference's Nx x Ny CImg image, identical for cubic grids, is saved
//     through CImg's external converters), rve_rec.txt and err.txt;
//     estimateNormFFT_RVE does not write normc.txt;
//   * the section constructor needs two sections of one size with a nonzero
//     pixel each (other inputs overrun or divide by zero in the reference);
//   * errors throw std::runtime_error.
#ifndef MAT3D_RECONSTRUCTION_HPP
#define MAT3D_RECONSTRUCTION_HPP

#include <cmath>
#include <cstddef>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "mat3d_b200.h"
#include "mat3d_matrix.hpp"

#ifndef FFTW3_H
typedef double fftw_complex[2];
struct m3d_fftw_plan_s {
    int n0, n1, n2, sign;
    fftw_complex* in;
    fftw_complex* out;
};
typedef m3d_fftw_plan_s* fftw_plan;
#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)
static inline fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex* in, fftw_complex* out, int sign,
                                         unsigned) {
    return new m3d_fftw_plan_s{n0, n1, n2, sign, in, out};
}
static inline fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex* in, fftw_complex* out, int sign, unsigned) {
    return new m3d_fftw_plan_s{n0, n1, 1, sign, in, out};
}
static inline void fftw_execute(const fftw_plan p) {
    if (m3drec_fft3(&p->in[0][0], &p->out[0][0], p->n0, p->n1, p->n2, p->sign, 0) != M3D_OK)
        throw std::runtime_error(std::string("fftw_execute (GPU): ") + m3d_last_error());
}
static inline void fftw_destroy_plan(fftw_plan p) { delete p; }
static inline int fftw_init_threads() { return 1; }
static inline void fftw_plan_with_nthreads(int) {}
static inline void fftw_cleanup_threads() {}
#endif

#ifndef cimg_version
namespace cimg_library {
// 8-bit single-channel image, pixel (x, y) at x + width * y (CImg's layout)
template <class T>
class CImg {
public:
    CImg() {}
    CImg(int w, int h, int d = 1, int c = 1) : w_(w), h_(h), px_((std::size_t)w * h * d * c) {}
    CImg(const T* values, int w, int h, int d = 1, int c = 1)
        : w_(w), h_(h), px_(values, values + (std::size_t)w * h * d * c) {}
    int width() const { return w_; }
    int height() const { return h_; }
    T* data() { return px_.data(); }
    const T* data() const { return px_.data(); }
    T& operator()(int x, int y, int z = 0, int c = 0) { return px_[(std::size_t)x + (std::size_t)w_ * y]; }
    // Neumann boundary, as CImg's atXY
    T atXY(int x, int y) const {
        x = x < 0 ? 0 : (x >= w_ ? w_ - 1 : x);
        y = y < 0 ? 0 : (y >= h_ ? h_ - 1 : y);
        return px_[(std::size_t)x + (std::size_t)w_ * y];
    }

private:
    int w_ = 0, h_ = 0;
    std::vector<T> px_;
};
}  // namespace cimg_library
#endif

using namespace std;
using namespace cimg_library;

namespace recon {
// fftshift / ifftshift of an Nx x Ny x Nz array (src/rec/reconstruction.cpp:47-140)
void fftshift(double* in, double* out, int Nx, int Ny, int Nz);
void ifftshift(double* in, double* out, int Nx, int Ny, int Nz);

// mean | |MTilda| - normC | (include/reconstruction.hpp:37-44)
inline double funcNormC(fftw_complex* MTilda, double* normC, int xyz) {
    double err = 0;
    for (int k = 0; k < xyz; ++k)
        err += std::fabs(std::sqrt(MTilda[k][0] * MTilda[k][0] + MTilda[k][1] * MTilda[k][1]) - normC[k]);
    return err / xyz;
}

class recPlan {
public:
    // two perpendicular cut sections (8-bit; the grid is w x h x h)
    recPlan(CImg<unsigned char> c1, CImg<unsigned char> c2);
    // the full two-point correlation function on Nx1 x Ny1 x Nz1
    recPlan(double* TPCF, int Nx1, int Ny1, int Nz1);
    ~recPlan();
    recPlan(const recPlan&) = delete;
    recPlan& operator=(const recPlan&) = delete;

    void estimateNormFFT_RVE();
    void runRec(int n, double b);
    void saveRecImages(string locFldr);
    void vtiWriter(string fileName, double* tpcf);

    MatrixDdd trackrealerrorA;
    fftw_complex* mTilda = nullptr;  // Nx*Ny*Nz complex, index z + Nz*(y + Ny*x)
    void fftShift(double* in, double* out, int Nx, int Ny, int Nz) { fftshift(in, out, Nx, Ny, Nz); }
    void ifftShift(double* in, double* out, int Nx, int Ny, int Nz) { ifftshift(in, out, Nx, Ny, Nz); }

    // beyond the reference: the seed of the random draws (default 1)
    void seed(unsigned long long s);

private:
    m3d_rec* h_ = nullptr;
    int Nx = 0, Ny = 0, Nz = 0, xyz = 0;
    void sync_fields(int n);
};
}  // namespace recon

#endif
