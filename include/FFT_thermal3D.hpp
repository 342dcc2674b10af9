// FFT_thermal3D.hpp -- drop-in replacement for the reference's thermal FFT
// solver class (include/FFT_thermal3D.hpp:37-154 of FayyazNo/MAT3d).
//
// Same class name, constructor, methods and public fields; the solve runs on
// the GPU through the C ABI in mat3d_b200.h (link -lmat3d_b200).  Errors throw
// std::runtime_error.  As in the reference, phase id 0 is the inclusion (ki)
// and any nonzero id the matrix (km).  setLoad may be called before material()
// (example/3d_thermal/main.cpp:94-95 does so); the load is then applied when
// material() has chosen the scheme.
#ifndef MAT3D_FFT_THERMAL3D_HPP
#define MAT3D_FFT_THERMAL3D_HPP

#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>

#include "mat3d_b200.h"
#include "mat3d_matrix.hpp"

using namespace std;

class FFT_analysis3d_thermal {
public:
    MatrixDdd Ki, Km, K0;
    MatrixDdd tempGradient;  // 3 x Nx*Ny*Nz
    MatrixDdd heatFlux;      // 3 x Nx*Ny*Nz
    MatrixDdd E;
    MatrixDdd tempGradHomo;
    MatrixDdd KHomo;
    MatrixDdd RHomo;
    MatrixDdd Ri, Rm, R0;
    MatrixDdd heatFluxHomo;
    int Nx, Ny, Nz;
    int xyz;
    double K11 = 0, K22 = 0, K33 = 0;

    FFT_analysis3d_thermal(int Nx1, int Ny1, int Nz1);
    ~FFT_analysis3d_thermal();
    FFT_analysis3d_thermal(const FFT_analysis3d_thermal&) = delete;
    FFT_analysis3d_thermal& operator=(const FFT_analysis3d_thermal&) = delete;

    void material(double km, double ki, MatrixIdd& RVE1);
    void setLoad(MatrixDdd& E1);
    void runAnalysis(double tol_field, double tol_eq);
    void homogenization(double tol_field, double tol_eq, string filename);
    void printer(string folderName);
    void vtiWriter(std::string fileName);

    // extensions (not in the reference)
    void setPrecision(int m3d_precision);
    void setCriterion(int m3d_criterion);
    m3d_stats stats() const;

private:
    m3d_solver* h_ = nullptr;
    int prec_ = M3D_PREC_FP64;
    int crit_ = M3D_CRIT_REFERENCE;
    MatrixIdd RVE_;
    double km_ = 0, ki_ = 0;
    bool material_set_ = false;
    void ensure_handle();
    void fetch_fields();
};

#endif
