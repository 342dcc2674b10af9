// rec_compat.cpp -- the drop-in recon::recPlan of include/reconstruction.hpp
// over the m3drec_* C ABI (the reconstruction itself runs on the GPU, rec.cu).
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/reconstruction.hpp"

namespace {
void check(int rc, const char* what) {
    if (rc != M3D_OK) throw std::runtime_error(std::string(what) + ": " + m3d_last_error());
}
}  // namespace

namespace recon {

void fftshift(double* in, double* out, int Nx, int Ny, int Nz) {
    check(m3drec_fftshift(in, out, Nx, Ny, Nz), "fftshift");
}

void ifftshift(double* in, double* out, int Nx, int Ny, int Nz) {
    check(m3drec_ifftshift(in, out, Nx, Ny, Nz), "ifftshift");
}

recPlan::recPlan(CImg<unsigned char> c1, CImg<unsigned char> c2) {
    check(m3drec_create_from_sections(c1.data(), c1.width(), c1.height(), c2.data(), c2.width(), c2.height(), 0, &h_),
          "recPlan(c1, c2)");
    Nx = c1.width();
    Ny = c1.height();
    Nz = c2.height();
    xyz = Nx * Ny * Nz;
    mTilda = new fftw_complex[(std::size_t)xyz];
    std::memset(mTilda, 0, sizeof(fftw_complex) * (std::size_t)xyz);
    check(m3drec_seed(h_, 1), "seed");
}

recPlan::recPlan(double* TPCF, int Nx1, int Ny1, int Nz1) : Nx(Nx1), Ny(Ny1), Nz(Nz1), xyz(Nx1 * Ny1 * Nz1) {
    check(m3drec_create(Nx, Ny, Nz, TPCF, 0, &h_), "recPlan(TPCF, Nx, Ny, Nz)");
    mTilda = new fftw_complex[(std::size_t)xyz];
    std::memset(mTilda, 0, sizeof(fftw_complex) * (std::size_t)xyz);
    check(m3drec_seed(h_, 1), "seed");
}

recPlan::~recPlan() {
    m3drec_destroy(h_);
    delete[] mTilda;
}

void recPlan::seed(unsigned long long s) { check(m3drec_seed(h_, s), "seed"); }

void recPlan::estimateNormFFT_RVE() { check(m3drec_estimate_norm(h_), "estimateNormFFT_RVE"); }

// mTilda (complex) and trackrealerrorA (1 x n, 0 past the last pass run) from the device
void recPlan::sync_fields(int n) {
    int i = 0, j = 0;
    unsigned long long call = 0;
    check(m3drec_get_state(h_, &mTilda[0][0], &i, &j, &call), "runRec");
    trackrealerrorA.resize(1, n);
    trackrealerrorA.setZero();
    std::vector<double> e((std::size_t)std::max(n, 1));
    int cnt = 0;
    check(m3drec_get_error(h_, e.data(), n, &cnt), "runRec");
    for (int k = 0; k < std::min(n, cnt); ++k) trackrealerrorA(k) = e[(std::size_t)k];
}

void recPlan::runRec(int n, double b) {
    check(m3drec_run(h_, n, b), "runRec");
    sync_fields(n);
}

void recPlan::saveRecImages(string locFldr) { check(m3drec_save_images(h_, locFldr.c_str()), "saveRecImages"); }

void recPlan::vtiWriter(string fileName, double* tpcf) {
    check(m3drec_write_vti(h_, fileName.c_str(), tpcf), "vtiWriter");
}

}  // namespace recon
