// FFT_analysis3D.hpp -- drop-in replacement for the reference's mechanical
// FFT solver class (include/FFT_analysis3D.hpp:36-215 of FayyazNo/MAT3d).
//
// Same class name, constructor, methods, argument order and public result
// fields; the solve runs on the GPU through the C ABI in mat3d_b200.h
// (link -lmat3d_b200).  Differences from the reference, all deliberate:
//   * errors throw std::runtime_error instead of exit()/std::terminate;
//   * fields are m3d::DMatrix (column-major, Eigen-compatible layout) rather
//     than Eigen matrices; epsilon/sigma are 6 x N^3 as in the reference;
//   * vtiWriter writes the 14 documented components (the reference reads
//     sigma(i+6, .), past the end of sigma, at src/3d/FFT_analysis3D.cpp:1080);
//   * arithmetic is FP64 by default; set precision before material() to use
//     the FP32 or FP32-with-FP64-refinement solvers.
#ifndef MAT3D_FFT_ANALYSIS3D_HPP
#define MAT3D_FFT_ANALYSIS3D_HPP

#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>

#include "mat3d_b200.h"
#include "mat3d_matrix.hpp"

using namespace std;

class FFT_Analysis3D {
public:
    // stiffness / compliance of every phase and of the reference medium
    MatrixDdd* C = nullptr;
    MatrixDdd C0;
    MatrixDdd* C_acc = nullptr;
    MatrixDdd* S_acc = nullptr;
    MatrixDdd* S = nullptr;
    MatrixDdd S0;
    // fields, 6 x Nx*Ny*Nz, Voigt [11,22,33,23,13,12], tensor shear
    MatrixDdd epsilon;
    MatrixDdd sigma;
    // macroscopic load, its increment and the mixed-control stress direction
    MatrixDdd E;
    MatrixDdd dE;
    MatrixDdd X0;
    int Nx, Ny, Nz;
    int xyz;
    double la0 = 0, mu0 = 0;
    double *la = nullptr, *mu = nullptr, *El = nullptr, *v = nullptr, *K = nullptr;
    double *H = nullptr, *n = nullptr, *Sy = nullptr;
    double *P = nullptr, *Y0 = nullptr;
    int noPhases = 0;
    double E11 = 0, E22 = 0, E33 = 0;
    MatrixDdd epHomo;
    MatrixDdd sigHomo;
    MatrixDdd SHomo;
    MatrixDdd CHomo;
    double* vol_fractions = nullptr;
    MatrixDdd epsilon_p_eff;
    MatrixDdd sigma_eff;
    MatrixDdd d;
    MatrixDdd prop_homogenized;

    FFT_Analysis3D(int Nx1, int Ny1, int Nz1, string mater_behav);
    ~FFT_Analysis3D();
    FFT_Analysis3D(const FFT_Analysis3D&) = delete;
    FFT_Analysis3D& operator=(const FFT_Analysis3D&) = delete;

    void material(MatrixDdd& mat, MatrixIdd& RVE1, int noPhases);
    void setLoad(MatrixDdd& E1, MatrixDdd& X0);
    void runAnalysis(double tol_field, double tol_eq, int nInc1);
    double homogenization(double tol_field, double tol_eq, string outputName);
    void printer(std::string outFldr = "results");
    void vtiWriter(std::string fileName);

    // extensions (not in the reference)
    void setPrecision(int m3d_precision);   // M3D_PREC_FP64 (default), _FP32, _FP32_REFINE
    void setCriterion(int m3d_criterion);   // M3D_CRIT_REFERENCE (default) or _RESIDUAL
    m3d_stats stats() const;
    int iterations() const;

private:
    m3d_solver* h_ = nullptr;
    string mater_behav_;
    int prec_ = M3D_PREC_FP64;
    int crit_ = M3D_CRIT_REFERENCE;
    MatrixDdd mat_;
    MatrixIdd RVE_;
    bool strainBase_ = true;
    void ensure_handle();
    void fetch_fields();
};

#endif
