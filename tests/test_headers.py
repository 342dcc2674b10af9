"""The drop-in headers are self-contained: a caller's translation unit that
includes only them (and the C ABI header, compiled as C) compiles.  CPU only;
no library is linked."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")

CXX = shutil.which("g++")
CC = shutil.which("gcc")

SNIPPETS = {
    "FFT_analysis3D.hpp": """
        #include "FFT_analysis3D.hpp"
        int main() { FFT_Analysis3D* a = nullptr; (void)a; return 0; }
    """,
    "FFT_thermal3D.hpp": """
        #include "FFT_thermal3D.hpp"
        int main() { FFT_analysis3d_thermal* t = nullptr; (void)t; return 0; }
    """,
    "reconstruction.hpp": """
        #include "reconstruction.hpp"
        int main() {
            fftw_complex* a = new fftw_complex[8];
            fftw_plan p = fftw_plan_dft_3d(2, 2, 2, a, a, FFTW_FORWARD, FFTW_ESTIMATE);
            fftw_destroy_plan(p);
            CImg<unsigned char> c(4, 4);
            c(1, 2) = 255;
            double e = recon::funcNormC(a, nullptr, 0);
            recon::recPlan* r = nullptr;
            (void)r; (void)e;
            delete[] a;
            return c.atXY(9, -3) == 0 ? 0 : 1;
        }
    """,
}


@pytest.mark.skipif(CXX is None, reason="no C++ compiler")
@pytest.mark.parametrize("header", sorted(SNIPPETS))
def test_cpp_header_compiles(header):
    r = subprocess.run([CXX, "-std=c++14", "-fsyntax-only", "-Wall", "-I", INC, "-x", "c++", "-"],
                       input=SNIPPETS[header], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


@pytest.mark.skipif(CC is None, reason="no C compiler")
def test_c_abi_header_is_c():
    src = '#include "mat3d_b200.h"\nint main(void) { m3d_rec* r = 0; (void)r; return m3d_abi_version() < 0; }\n'
    r = subprocess.run([CC, "-std=c99", "-fsyntax-only", "-Wall", "-I", INC, "-x", "c", "-"],
                       input=src, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
