// compat.cpp -- the drop-in classes FFT_Analysis3D and FFT_analysis3d_thermal
// implemented over the C ABI (compiled into libmat3d_b200.so).
//
// Output formats follow the reference: homogenization report
// (src/3d/FFT_analysis3D.cpp:944-996, src/3dTherm/FFT_thermal3D.cpp:597-620),
// single-column field files (printer, :1001-1053 / :628-692), and a VTK XML
// ImageData (.vti) file written directly, without VTK (vtiWriter, :1056-1104 /
// :697-746).
#include <sys/stat.h>
#include <sys/types.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "FFT_analysis3D.hpp"
#include "FFT_thermal3D.hpp"

namespace {

void check(int rc, const char* what) {
    if (rc != M3D_OK && rc != M3D_NOT_CONVERGED) {
        throw std::runtime_error(std::string(what) + ": " + m3d_status_string(rc) + ": " + m3d_last_error());
    }
    if (rc == M3D_NOT_CONVERGED) std::cout << " iteration excede from the allowable number" << std::endl;
}

MatrixDdd iso_C(double la, double mu) {
    MatrixDdd C(6, 6);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C(i, j) = la;
    for (int i = 0; i < 3; ++i) C(i, i) = la + 2 * mu;
    for (int i = 3; i < 6; ++i) C(i, i) = 2 * mu;
    return C;
}

// VTK XML ImageData writer: one point-data array with `ncomp` components,
// x fastest in the file (VTK order), taken from fields stored v = z + Nz*(y + Ny*x)
// exactly as the reference's GetScalarPointer(x,y,z) loop does
// (len = x + y*dims[0] + z*dims[0]*dims[1], src/3d/FFT_analysis3D.cpp:1071-1076).
void write_vti(const std::string& name, int Nx, int Ny, int Nz, int ncomp,
               const std::vector<const double*>& comps) {
    std::ofstream f(name);
    if (!f) throw std::runtime_error("cannot open " + name);
    f << "<?xml version=\"1.0\"?>\n";
    f << "<VTKFile type=\"ImageData\" version=\"0.1\" byte_order=\"LittleEndian\">\n";
    f << "  <ImageData WholeExtent=\"0 " << Nx - 1 << " 0 " << Ny - 1 << " 0 " << Nz - 1
      << "\" Origin=\"0 0 0\" Spacing=\"1 1 1\">\n";
    f << "    <Piece Extent=\"0 " << Nx - 1 << " 0 " << Ny - 1 << " 0 " << Nz - 1 << "\">\n";
    f << "      <PointData Scalars=\"ImageScalars\">\n";
    f << "        <DataArray type=\"Float64\" Name=\"ImageScalars\" NumberOfComponents=\"" << ncomp
      << "\" format=\"ascii\">\n";
    f.precision(10);
    const long long n = (long long)Nx * Ny * Nz;
    for (long long len = 0; len < n; ++len) {
        for (int c = 0; c < ncomp; ++c) f << (c ? " " : "") << (comps[c] ? comps[c][len] : 0.0);
        f << "\n";
    }
    f << "        </DataArray>\n      </PointData>\n      <CellData/>\n    </Piece>\n  </ImageData>\n</VTKFile>\n";
}

}  // namespace

// ============================================================================
// FFT_Analysis3D
// ============================================================================
FFT_Analysis3D::FFT_Analysis3D(int Nx1, int Ny1, int Nz1, string mater_behav) {
    Nx = Nx1; Ny = Ny1; Nz = Nz1;
    xyz = Nx * Ny * Nz;
    mater_behav_ = mater_behav;
    if (mater_behav != "e" && mater_behav != "ep" && mater_behav != "ed")
        throw std::invalid_argument("mater_behav must be \"e\", \"ep\" or \"ed\"");
    epsilon.resize(6, xyz);
    sigma.resize(6, xyz);
    E.resize(6, 1);
    X0.resize(6, 1);
}

FFT_Analysis3D::~FFT_Analysis3D() {
    m3d_destroy(h_);
    delete[] C; delete[] S; delete[] C_acc; delete[] S_acc;
    delete[] la; delete[] mu; delete[] El; delete[] v; delete[] K;
    delete[] H; delete[] n; delete[] Sy; delete[] P; delete[] Y0;
    delete[] vol_fractions;
}

void FFT_Analysis3D::setPrecision(int p) { prec_ = p; }
void FFT_Analysis3D::setCriterion(int c) { crit_ = c; }

void FFT_Analysis3D::ensure_handle() {
    if (h_) return;
    const int behav = mater_behav_ == "e" ? M3D_BEHAV_ELASTIC : (mater_behav_ == "ep" ? M3D_BEHAV_J2 : M3D_BEHAV_DAMAGE);
    check(m3d_create(M3D_KIND_MECH, Nx, Ny, Nz, behav, prec_, 1, &h_), "m3d_create");
}

void FFT_Analysis3D::material(MatrixDdd& mat, MatrixIdd& RVE1, int noPhases1) {
    if (RVE1.size() != xyz) throw std::invalid_argument("RVE must have Nx*Ny*Nz entries");
    ensure_handle();
    noPhases = noPhases1;
    std::vector<double> m((size_t)noPhases * 7);
    for (int i = 0; i < noPhases; ++i)
        for (int j = 0; j < 7; ++j) m[i * 7 + j] = mat(i, j);
    mat_ = mat;
    RVE_ = RVE1;
    check(m3d_set_material_mech(h_, m.data(), noPhases, RVE1.data(), M3D_SCHEME_AUTO), "material");
    m3d_stats st;
    m3d_get_stats(h_, &st);
    strainBase_ = (st.scheme == 1);
    std::cout << (strainBase_ ? " Strain-Based Algorithm is Running" : " Stress-Based Algorithm is Running") << std::endl;
    la0 = st.la0;
    mu0 = st.mu0;
    // public copies of the phase data (material(), src/3d/FFT_analysis3D.cpp:441-546)
    delete[] C; delete[] S; delete[] C_acc; delete[] S_acc;
    delete[] la; delete[] mu; delete[] El; delete[] v; delete[] K;
    delete[] H; delete[] n; delete[] Sy; delete[] P; delete[] Y0; delete[] vol_fractions;
    C = new MatrixDdd[noPhases]; S = new MatrixDdd[noPhases];
    C_acc = new MatrixDdd[noPhases]; S_acc = new MatrixDdd[noPhases];
    la = new double[noPhases]; mu = new double[noPhases]; El = new double[noPhases]; v = new double[noPhases];
    K = new double[noPhases]; H = new double[noPhases]; n = new double[noPhases]; Sy = new double[noPhases];
    P = new double[noPhases]; Y0 = new double[noPhases]; vol_fractions = new double[noPhases];
    C0 = iso_C(la0, mu0);
    S0 = C0.inverse();
    for (int i = 0; i < noPhases; ++i) {
        El[i] = mat(i, 0); v[i] = mat(i, 1); Sy[i] = mat(i, 2); H[i] = mat(i, 3);
        n[i] = mat(i, 4); P[i] = mat(i, 5); Y0[i] = mat(i, 6);
        mu[i] = El[i] / (1 + v[i]) / 2.;
        la[i] = v[i] * El[i] / (1 + v[i]) / (1 - 2 * v[i]);
        K[i] = la[i] + (2. / 3.) * mu[i];
        C[i] = iso_C(la[i], mu[i]);
        S[i] = C[i].inverse();
        vol_fractions[i] = st.vol_fraction[i];
        MatrixDdd a(6, 6), b(6, 6);
        MatrixDdd ci = MatrixDdd(6, 6), si = MatrixDdd(6, 6);
        for (int r = 0; r < 6; ++r)
            for (int c = 0; c < 6; ++c) { ci(r, c) = C[i](r, c) + C0(r, c); si(r, c) = S[i](r, c) + S0(r, c); }
        const MatrixDdd cinv = ci.inverse(), sinv = si.inverse();
        for (int r = 0; r < 6; ++r)
            for (int c = 0; c < 6; ++c) {
                double s1 = 0, s2 = 0;
                for (int k = 0; k < 6; ++k) { s1 += cinv(r, k) * C0(k, c); s2 += sinv(r, k) * S0(k, c); }
                a(r, c) = 2 * s1;
                b(r, c) = 2 * s2;
            }
        C_acc[i] = a;
        S_acc[i] = b;
    }
}

void FFT_Analysis3D::setLoad(MatrixDdd& E1, MatrixDdd& X01) {
    E = E1;
    X0 = X01;
    if (!h_) throw std::logic_error("setLoad before material");
    check(m3d_set_load(h_, 0, E.data(), X0.data()), "setLoad");
}

void FFT_Analysis3D::fetch_fields() {
    epsilon.resize(6, xyz);
    sigma.resize(6, xyz);
    check(m3d_get_field(h_, M3D_FIELD_STRAIN, 0, epsilon.data()), "epsilon");
    check(m3d_get_field(h_, M3D_FIELD_STRESS, 0, sigma.data()), "sigma");
    if (mater_behav_ == "ep") {
        epsilon_p_eff.resize(1, xyz);
        check(m3d_get_field(h_, M3D_FIELD_EPS_P, 0, epsilon_p_eff.data()), "epsilon_p_eff");
        sigma_eff.resize(1, xyz);
        for (int i = 0; i < xyz; ++i) {
            const double* s = sigma.data() + (size_t)6 * i;
            const double sm = (s[0] + s[1] + s[2]) / 3.;
            const double d0 = s[0] - sm, d1 = s[1] - sm, d2 = s[2] - sm;
            sigma_eff(i) = std::sqrt(1.5) * std::sqrt(d0 * d0 + d1 * d1 + d2 * d2 + 2 * s[3] * s[3] + 2 * s[4] * s[4] + 2 * s[5] * s[5]);
        }
    }
    if (mater_behav_ == "ed") {
        d.resize(1, xyz);
        check(m3d_get_field(h_, M3D_FIELD_DAMAGE, 0, d.data()), "d");
    }
    if (mater_behav_ != "e") {
        m3d_stats st;
        m3d_get_stats(h_, &st);
        prop_homogenized.resize(st.n_increments, 9);
        std::vector<double> rows((size_t)std::max(1, st.n_increments) * 9);
        const int nr = m3d_get_increments(h_, rows.data(), st.n_increments);
        for (int i = 0; i < nr; ++i)
            for (int j = 0; j < 9; ++j) prop_homogenized(i, j) = rows[(size_t)i * 9 + j];
    }
}

void FFT_Analysis3D::runAnalysis(double tol_field, double tol_eq, int nInc1) {
    if (!h_) throw std::logic_error("runAnalysis before material");
    check(m3d_run(h_, tol_field, tol_eq, nInc1, crit_, 0), "runAnalysis");
    fetch_fields();
}

double FFT_Analysis3D::homogenization(double tol_field, double tol_eq, string outputName) {
    if (!h_) throw std::logic_error("homogenization before material");
    if (mater_behav_ != "e") {
        // the reference switches its own object to elastic (:858); here a
        // separate elastic solve is run on the same material
        m3d_solver* he = nullptr;
        check(m3d_create(M3D_KIND_MECH, Nx, Ny, Nz, M3D_BEHAV_ELASTIC, prec_, 6, &he), "m3d_create");
        std::vector<double> m((size_t)noPhases * 7);
        for (int i = 0; i < noPhases; ++i)
            for (int j = 0; j < 7; ++j) m[i * 7 + j] = mat_(i, j);
        std::swap(h_, he);
        mater_behav_ = "e";
        check(m3d_set_material_mech(h_, m.data(), noPhases, RVE_.data(), M3D_SCHEME_AUTO), "material");
        m3d_destroy(he);
        m3d_stats st;
        m3d_get_stats(h_, &st);
        strainBase_ = st.scheme == 1;
    }
    CHomo.resize(6, 6); SHomo.resize(6, 6); epHomo.resize(6, 6); sigHomo.resize(6, 6);
    double c36[36], s36[36], e36[36], g36[36];
    check(m3d_homogenize(h_, tol_field, tol_eq, crit_, 0, c36, s36, e36, g36), "homogenization");
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            CHomo(i, j) = c36[i * 6 + j];
            SHomo(i, j) = s36[i * 6 + j];
            epHomo(i, j) = e36[i * 6 + j];
            sigHomo(i, j) = g36[i * 6 + j];
        }
    E11 = 1. / SHomo(0, 0); E22 = 1. / SHomo(1, 1); E33 = 1. / SHomo(2, 2);
    // fields of the last load case, as the reference leaves them
    epsilon.resize(6, xyz);
    sigma.resize(6, xyz);
    check(m3d_get_field(h_, M3D_FIELD_STRAIN, 5, epsilon.data()), "epsilon");
    check(m3d_get_field(h_, M3D_FIELD_STRESS, 5, sigma.data()), "sigma");
    // Hashin-Shtrikman bounds (:911-942)
    double Gn = mu[0], G1 = mu[0], Kn = K[0], K1 = K[0];
    for (int i = 1; i < noPhases; ++i) {
        Gn = std::max(Gn, mu[i]); G1 = std::min(G1, mu[i]);
        Kn = std::max(Kn, K[i]); K1 = std::min(K1, K[i]);
    }
    const double alfa1 = -3 / (3 * K1 + 4 * G1), alfan = -3 / (3 * Kn + 4 * Gn);
    const double beta1 = -(3 * (K1 + 2 * G1)) / ((3 * K1 + 4 * G1) * 5 * G1);
    const double betan = -(3 * (Kn + 2 * Gn)) / ((3 * Kn + 4 * Gn) * 5 * Gn);
    double A1 = 0, An = 0, B1 = 0, Bn = 0;
    for (int i = 0; i < noPhases; ++i) {
        if (K[i] != K1) A1 += vol_fractions[i] / ((1. / (K[i] - K1)) - alfa1);
        if (K[i] != Kn) An += vol_fractions[i] / ((1. / (K[i] - Kn)) - alfan);
        if (mu[i] != G1) B1 += vol_fractions[i] / ((0.5 / (mu[i] - G1)) - beta1);
        if (mu[i] != Gn) Bn += vol_fractions[i] / ((0.5 / (mu[i] - Gn)) - betan);
    }
    const double K_min = K1 + A1 / (1 + alfa1 * A1), K_max = Kn + An / (1 + alfan * An);
    const double G_min = G1 + 0.5 * B1 / (1 + beta1 * B1), G_max = Gn + 0.5 * Bn / (1 + betan * Bn);
    const double E_min = 9 * K_min * G_min / (3 * K_min + G_min), E_max = 9 * K_max * G_max / (3 * K_max + G_max);
    std::ofstream homo(outputName + ".txt");
    homo << "*************************************************************************" << endl << endl;
    homo << "        F F T     H O M O G E N I Z A T I O N    B Y   M A T 3 D" << endl << endl;
    homo << (strainBase_ ? "                      Stran-Based Algorithm Is Used" : "                      Stress-Based Algorithm Is Used") << endl;
    homo << "                           Nx=" << Nx << "   " << "Ny=" << Ny << "   " << "Nz=" << Nz << endl << endl;
    homo << "      ----------------------------------------------------------------" << endl;
    for (int i = 0; i < noPhases; ++i) {
        string k = to_string(i) + " = ";
        homo << "                      Volume Fraction Phase " << k << vol_fractions[i] << endl;
        homo << "     E" << k << El[i] << "     " << "v" << k << v[i] << "     " << "K" << k << K[i] << "     " << "G" << k << mu[i] << "     " << endl << endl;
    }
    homo << "      ----------------------------------------------------------------" << endl << endl;
    homo << "                        Hashin-Shtrikman Bounds" << endl;
    homo << "         E_min=" << E_min << "   " << "K_min=" << K_min << "   " << "G_min=" << G_min << endl;
    homo << "         E_max=" << E_max << "   " << "K_max=" << K_max << "   " << "G_max=" << G_max << endl << endl << endl;
    homo << "************************************************************************" << endl << endl;
    homo << "Homogenized Elastic Modules:" << endl;
    homo << "E11=" << E11 << "     " << "E22=" << E22 << "     " << "E33=" << E33 << "     " << endl << endl;
    homo << endl << "C_Homogenized=" << endl << endl << CHomo << endl;
    homo << "      ----------------------------------------------------------------" << endl;
    homo << endl << "S_Homogenized=" << endl << endl << SHomo << endl;
    homo << "      ----------------------------------------------------------------" << endl;
    for (int i = 0; i < noPhases; ++i) {
        homo << endl << "C" << to_string(i) << "=" << endl << C[i] << endl;
        homo << "      ----------------------------------------------------------------" << endl;
        homo << endl << "S" << to_string(i) << "=" << endl << S[i] << endl;
        homo << "      ----------------------------------------------------------------" << endl;
    }
    homo << endl << "Homogenized Load Cases (Each row is one load case i.e (E11 E22 E33 E32 E31 E12) and Eij is summation of strain components in in  all voxels )" << endl << endl;
    homo << epHomo << endl;
    homo << endl << "Homogenized stess (Each coulemn is (SS11 SS22 SS33 SS32 SS31 SS12) and SSij is summation of stress components in in all voxels )" << endl << endl;
    homo << sigHomo << endl;
    return E11 + E22 + E33;
}

void FFT_Analysis3D::printer(std::string outFldr) {
    mkdir(outFldr.c_str(), S_IRWXU | S_IRWXG | S_IROTH | S_IXOTH);
    const char* names[13] = {"ep1.txt", "ep2.txt", "ep3.txt", "ep4.txt", "ep5.txt", "ep6.txt",
                             "sig1.txt", "sig2.txt", "sig3.txt", "sig4.txt", "sig5.txt", "sig6.txt", "ep_p"};
    for (int j = 0; j < 13; ++j) {
        string nm = names[j];
        if (j == 12 && mater_behav_ == "ed") nm = "d";
        std::ofstream o(outFldr + "/" + nm);
        for (int i = 0; i < xyz; ++i) {
            if (j < 6) o << epsilon(j, i) << endl;
            else if (j < 12) o << sigma(j - 6, i) << endl;
            else if (mater_behav_ == "ep") o << epsilon_p_eff(i) << endl;
            else if (mater_behav_ == "ed") o << d(i) << endl;
        }
    }
    if (mater_behav_ != "e") {
        std::ofstream op("epsilon_sigma.txt");
        op << "epsilon" << "  " << "sigma1" << "   " << "sigma2" << "   " << "sigma3" << "   " << "tau23" << "   " << "tau13"
           << "   " << "tau12" << "   " << (mater_behav_ == "ep" ? "sigma_eff" : "d") << "   " << "epsilon_p_eff" << endl;
        op << 0 << "  " << 0 << "  " << 0 << "  " << 0 << "  " << 0 << "  " << 0 << "  " << 0 << "  " << 0 << "  " << 0 << endl;
        for (int i = 0; i < prop_homogenized.rows(); ++i) {
            for (int j = 0; j < 9; ++j) op << (j ? "  " : "") << prop_homogenized(i, j);
            op << endl;
        }
    }
}

void FFT_Analysis3D::vtiWriter(std::string fileName) {
    std::vector<std::vector<double>> cols(14, std::vector<double>(xyz, 0.0));
    for (int i = 0; i < xyz; ++i)
        for (int c = 0; c < 6; ++c) {
            cols[c][i] = epsilon(c, i);
            cols[6 + c][i] = sigma(c, i);
        }
    if (mater_behav_ == "ep")
        for (int i = 0; i < xyz; ++i) { cols[12][i] = epsilon_p_eff(i); cols[13][i] = sigma_eff(i); }
    if (mater_behav_ == "ed")
        for (int i = 0; i < xyz; ++i) cols[12][i] = d(i);
    // the reference maps VTK point (x,y,z) to field index x + y*Nx + z*Nx*Ny
    std::vector<const double*> ptr(14);
    for (int c = 0; c < 14; ++c) ptr[c] = cols[c].data();
    write_vti(fileName, Nx, Ny, Nz, 14, ptr);
}

m3d_stats FFT_Analysis3D::stats() const {
    m3d_stats s;
    std::memset(&s, 0, sizeof(s));
    if (h_) m3d_get_stats(h_, &s);
    return s;
}
int FFT_Analysis3D::iterations() const { return stats().iters; }

// ============================================================================
// FFT_analysis3d_thermal
// ============================================================================
FFT_analysis3d_thermal::FFT_analysis3d_thermal(int Nx1, int Ny1, int Nz1) {
    Nx = Nx1; Ny = Ny1; Nz = Nz1;
    xyz = Nx * Ny * Nz;
    tempGradient.resize(3, xyz);
    heatFlux.resize(3, xyz);
    E.resize(3, 1);
}

FFT_analysis3d_thermal::~FFT_analysis3d_thermal() { m3d_destroy(h_); }

void FFT_analysis3d_thermal::setPrecision(int p) { prec_ = p; }
void FFT_analysis3d_thermal::setCriterion(int c) { crit_ = c; }

void FFT_analysis3d_thermal::ensure_handle() {
    if (h_) return;
    check(m3d_create(M3D_KIND_THERMAL, Nx, Ny, Nz, M3D_BEHAV_ELASTIC, prec_, 1, &h_), "m3d_create");
}

void FFT_analysis3d_thermal::material(double km, double ki, MatrixIdd& RVE1) {
    if (RVE1.size() != xyz) throw std::invalid_argument("RVE must have Nx*Ny*Nz entries");
    ensure_handle();
    km_ = km;
    ki_ = ki;
    RVE_ = RVE1;
    check(m3d_set_material_thermal(h_, km, ki, RVE1.data(), M3D_SCHEME_AUTO), "material");
    m3d_stats st;
    m3d_get_stats(h_, &st);
    std::cout << (st.scheme == 1 ? " temperature Gradient-Based Algorithm is Running" : " Heat Flux-Based  Algorithm is Running") << std::endl;
    Km.setZero(3, 3); Ki.setZero(3, 3); K0.setZero(3, 3);
    for (int i = 0; i < 3; ++i) { Km(i, i) = km; Ki(i, i) = ki; K0(i, i) = st.k0; }
    Rm = Km.inverse(); Ri = Ki.inverse(); R0 = K0.inverse();
    material_set_ = true;
    if (E.size() == 3) check(m3d_set_load(h_, 0, E.data(), nullptr), "setLoad");
}

void FFT_analysis3d_thermal::setLoad(MatrixDdd& E1) {
    E = E1;
    if (material_set_) check(m3d_set_load(h_, 0, E.data(), nullptr), "setLoad");
}

void FFT_analysis3d_thermal::fetch_fields() {
    tempGradient.resize(3, xyz);
    heatFlux.resize(3, xyz);
    check(m3d_get_field(h_, M3D_FIELD_STRAIN, 0, tempGradient.data()), "tempGradient");
    check(m3d_get_field(h_, M3D_FIELD_STRESS, 0, heatFlux.data()), "heatFlux");
}

void FFT_analysis3d_thermal::runAnalysis(double tol_field, double tol_eq) {
    if (!material_set_) throw std::logic_error("runAnalysis before material");
    check(m3d_run(h_, tol_field, tol_eq, 1, crit_, 0), "runAnalysis");
    fetch_fields();
}

void FFT_analysis3d_thermal::homogenization(double tol_field, double tol_eq, string filename) {
    if (!material_set_) throw std::logic_error("homogenization before material");
    double k9[9], r9[9], g9[9], q9[9];
    check(m3d_homogenize(h_, tol_field, tol_eq, crit_, 0, k9, r9, g9, q9), "homogenization");
    KHomo.resize(3, 3); RHomo.resize(3, 3); tempGradHomo.resize(3, 3); heatFluxHomo.resize(3, 3);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            KHomo(i, j) = k9[i * 3 + j];
            RHomo(i, j) = r9[i * 3 + j];
            tempGradHomo(i, j) = g9[i * 3 + j];
            heatFluxHomo(i, j) = q9[i * 3 + j];
        }
    tempGradient.resize(3, xyz);
    heatFlux.resize(3, xyz);
    check(m3d_get_field(h_, M3D_FIELD_STRAIN, 2, tempGradient.data()), "tempGradient");
    check(m3d_get_field(h_, M3D_FIELD_STRESS, 2, heatFlux.data()), "heatFlux");
    // Mori-Tanaka and HS bounds (src/3dTherm/FFT_thermal3D.cpp:582-592); fi_m
    // is RVE.sum()/xyz there, an integer division, reproduced here
    long long s = 0;
    for (int i = 0; i < xyz; ++i) s += RVE_(i);
    const double fi_m = (double)(s / xyz), fi_i = 1 - fi_m;
    const double km = km_, ki = ki_;
    const double k_mt = km + (fi_i * (ki - km)) / (1 + fi_m * (ki - km) / (3 * km));
    const double k_up = fi_i * ki + fi_m * km - fi_i * fi_m * (km - ki) * (km - ki) / (3 * ki - fi_i * (ki - km));
    const double k_lo = fi_i * ki + fi_m * km - fi_i * fi_m * (km - ki) * (km - ki) / (3 * km + fi_m * (ki - km));
    K11 = KHomo(0, 0); K22 = KHomo(1, 1); K33 = KHomo(2, 2);
    std::ofstream homo(filename + ".txt");
    homo << "Volume Fraction of the White Phase (or 1)=" << fi_m << endl << endl;
    homo << "K phase matrix  ( or 1)=" << endl << Km << "     " << endl;
    homo << "K phase inclusion(or 0)=" << endl << Ki << "     " << endl;
    homo << "Nx=" << Nx << "   " << "Ny=" << Ny << "   " << Nz << endl << endl;
    homo << endl << "KHomogenized Mori-Tanaka=" << endl << endl << k_mt << endl;
    homo << endl << "Lower bound HS=" << endl << endl << k_lo << endl;
    homo << endl << "Upper bound LS=" << endl << endl << k_up << endl;
    homo << endl << "KHomogenized=" << endl << endl << KHomo << endl;
    homo << endl << "RHomogenized(Homogenized Resistivity tensor)=" << endl << endl << RHomo << endl;
    homo << endl << "Rm=" << endl << endl << Rm << endl;
    homo << endl << "Ri=" << endl << endl << Ri << endl;
    homo << endl << endl << "--------------------------------------------------------------------" << endl << endl;
    homo << endl << "Homogenized Load Cases (Each row is one load case i.e (E11 E22 E33 ) and Eij is summation of temperatur gradient components in in  all voxels )" << endl << endl;
    homo << tempGradHomo << endl;
    homo << endl << "Homogenized stess (Each coulemn is (SS11 SS22 SS33) and SSij is summation of heat flux in in all voxels )" << endl << endl;
    homo << heatFluxHomo << endl;
}

void FFT_analysis3d_thermal::printer(string folderName) {
    mkdir(folderName.c_str(), S_IRWXU | S_IRWXG | S_IROTH | S_IXOTH);
    for (int c = 0; c < 3; ++c) {
        std::ofstream a(folderName + "/heatFlux" + to_string(c + 1) + ".txt");
        for (int i = 0; i < xyz; ++i) a << heatFlux(c, i) << endl;
        std::ofstream b(folderName + "/tempGradient" + to_string(c + 1) + ".txt");
        for (int i = 0; i < xyz; ++i) b << tempGradient(c, i) << endl;
    }
}

void FFT_analysis3d_thermal::vtiWriter(std::string fileName) {
    std::vector<std::vector<double>> cols(6, std::vector<double>(xyz, 0.0));
    for (int i = 0; i < xyz; ++i)
        for (int c = 0; c < 3; ++c) { cols[c][i] = tempGradient(c, i); cols[3 + c][i] = heatFlux(c, i); }
    std::vector<const double*> ptr(6);
    for (int c = 0; c < 6; ++c) ptr[c] = cols[c].data();
    write_vti(fileName, Nx, Ny, Nz, 6, ptr);
}

m3d_stats FFT_analysis3d_thermal::stats() const {
    m3d_stats s;
    std::memset(&s, 0, sizeof(s));
    if (h_) m3d_get_stats(h_, &s);
    return s;
}
