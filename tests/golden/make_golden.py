"""Generate the golden fixtures in tests/golden/ from the reference's own solver.

Runs oracle/_ref/libmat3d_ref.so -- the reference sources
src/3d/FFT_analysis3D.cpp, src/3dTherm/FFT_thermal3D.cpp, src/2d/FFT_analysis2D.cpp
and src/rec/reconstruction.cpp compiled unmodified by oracle/Makefile against
stand-in FFTW/Eigen/VTK headers -- on
small seeded inputs and stores inputs and outputs as compressed .npz files.
The reference project ships no tests or expected outputs of its own, so these
fixtures are the parity pin for the numpy oracle (tests/test_oracle_golden.py)
and, through it, for the CUDA solver.

    make -C oracle REF=<reference sources> && python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle.ref_lib import RefLib  # noqa: E402


def sphere(shape, r, center=None):
    Nx, Ny, Nz = shape
    X, Y, Z = np.meshgrid(np.arange(Nx), np.arange(Ny), np.arange(Nz), indexing="ij")
    c = center or (Nx / 2, Ny / 2, Nz / 2)
    rve = np.ones(shape, np.int32)
    rve[(X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2 <= r * r] = 0
    return rve.ravel()


MAT_A = np.array([[70e9, 0.2, 40e6, 100e6, 1, 8e-2, 8e2], [3e9, 0.35, 250e6, 8006, 0.2, 8e-4, 8e3]])
MAT_J2 = np.array([[400e9, 0.2, 1e30, 0, 1, 0, 1e30], [70e9, 0.33, 100e6, 1e9, 1, 0, 1e30]])


def main():
    ref = RefLib()
    out = {}
    rng = np.random.default_rng(1234)
    # FFT layout pins (guru64 r2c / c2r of the 3-D solver's plans)
    for (shape, c) in (((6, 8, 10), 6), ((5, 6, 7), 3)):
        x = rng.standard_normal(shape + (c,))
        spec = ref.fft_r2c(x)
        back = ref.fft_c2r(spec, shape)
        np.savez_compressed(os.path.join(HERE, f"fft_{shape[0]}x{shape[1]}x{shape[2]}_c{c}.npz"),
                            x=x, spec=spec, back=back)
    # elastic runs: stress-based (auto) and strain-based (forced), non-cubic
    for name, shape, force, E in (("elastic_auto_12", (12, 12, 12), 0, [1e-3, 0, 0, 0, 2e-4, 0]),
                                  ("elastic_strain_10x12x14", (10, 12, 14), 1, [0, 1e-3, 0, 3e-4, 0, 0])):
        rve = sphere(shape, 3.1)
        r = ref.mech_run(shape, "e", MAT_A, rve, np.array(E, float), np.array([0, 1, 0, 0, 0, 0.0]),
                         1e-10, 1e-10, 1, force)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), shape=shape, rve=rve, mat=MAT_A, E=E,
                            force=force, tol=1e-10, **r)
    # elastic homogenization
    shape = (10, 10, 10)
    rve = sphere(shape, 2.6)
    r = ref.mech_homog(shape, MAT_A, rve, 1e-10, 1e-10)
    np.savez_compressed(os.path.join(HERE, "homog_elastic_10.npz"), shape=shape, rve=rve, mat=MAT_A, tol=1e-10, **r)
    # J2 and damage, 3 increments under uniaxial stress direction X0 = e_1
    for name, behav, mat in (("j2_10", "ep", MAT_J2), ("damage_10", "ed", MAT_A)):
        shape = (10, 10, 10)
        rve = sphere(shape, 2.8, center=(5, 5, 5))
        E = np.array([0.02, 0, 0, 0, 0, 0.0])
        X0 = np.array([1.0, 0, 0, 0, 0, 0])
        r = ref.mech_run(shape, behav, mat, rve, E, X0, 1e-8, 1e-8, 3, 0)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), shape=shape, rve=rve, mat=mat, E=E, X0=X0,
                            tol=1e-8, ninc_req=3, **r)
    # thermal: gradient-based (km < ki) and flux-based (km > ki), run + homogenization
    for name, km, ki in (("thermal_grad_12", 1.0, 100.0), ("thermal_flux_12", 30.0, 25.0)):
        shape = (12, 12, 12)
        rve = sphere(shape, 3.3)
        E = np.array([0.0, 0.3, 1.0])
        r = ref.therm_run(shape, km, ki, rve, E, 1e-10, 1e-10)
        h = ref.therm_homog(shape, km, ki, rve, 1e-10, 1e-10)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), shape=shape, rve=rve, km=km, ki=ki, E=E, tol=1e-10,
                            **r, K=h["K"], R=h["R"], homog_sweeps=h["sweeps"])
    # 2-D solver (src/2d/FFT_analysis2D.cpp): single run (25 iterations) and
    # homogenization, an even and an odd square grid (non-square grids make
    # the reference divide by a zero wave vector: x wraps with Ny)
    props = np.array([68.9e9, 0.35, 400e9, 0.23])
    for N in (16, 15):
        X, Y = np.meshgrid(np.arange(N), np.arange(N), indexing="ij")
        rve = np.ones((N, N), np.int32)
        rve[(X - N / 2) ** 2 + (Y - N / 2.5) ** 2 <= 16] = 0
        rve = rve.ravel()
        E = np.array([0, 0.001j, 0.005], np.complex128)
        r = ref.mech2d_run((N, N), props, rve, E)
        h = ref.mech2d_homog((N, N), props, rve, E)
        np.savez_compressed(os.path.join(HERE, f"mech2d_{N}.npz"), shape=(N, N), rve=rve, props=props, E=E,
                            eps=r["eps"], sig=r["sig"], C=h["C"], epHomo=h["epHomo"], sigHomo=h["sigHomo"])
    # microstructure reconstruction (src/rec/reconstruction.cpp): the TPCF of
    # example/reconst3d/main.cpp (f(r) = exp(-r/A) sin(Qr)/(Qr)), shifted to
    # index 0 and transformed as the example does; 320 passes cover the
    # hybrid input-output phase, the box projection (j >= 100), the restarts
    # at i + 1 = 150 and 300 and the reset of j after 200.  Odd lengths: for
    # an even length the transform of a real field has real coefficients at
    # the Nyquist frequencies whose phase (0 or +-pi) hangs on the sign of a
    # rounding-level imaginary part, which differs between FFT implementations
    from oracle.mat3d_oracle import ifftshift3, tpcf_isotropic
    for shape, seed, (A, Q, phi1) in (((9, 9, 9), 1, (3.0, 0.8, 0.4)), ((7, 9, 11), 2, (4.0, 0.6, 0.5))):
        Nx, Ny, Nz = shape
        t = tpcf_isotropic(max(shape), A, Q, phi1).reshape((max(shape),) * 3)[:Nx, :Ny, :Nz].ravel()
        T = np.real(np.fft.fftn(ifftshift3(t, Nx, Ny, Nz).reshape(shape))).ravel()
        n, beta = 320, 0.8
        r = ref.rec_run(shape, T, n, beta, seed)
        np.savez_compressed(os.path.join(HERE, f"rec_{Nx}x{Ny}x{Nz}.npz"), shape=shape, tpcf=T, seed=seed, n=n,
                            beta=beta, err=r["err"], rve=r["rve"], iterations=r["iterations"])
    # the cut-section constructor + estimateNormFFT_RVE: seeded 8-bit sections
    # (discs at 200, scattered pixels at 90, which the reference's integer
    # division by the maximum maps to 0), square and non-square
    rng = np.random.default_rng(7)
    for (h, w) in ((12, 12), (9, 11)):
        img = np.zeros((h, w), np.uint8)
        yy, xx = np.mgrid[0:h, 0:w]
        for _ in range(4):
            cy, cx, rr = rng.uniform(0, h), rng.uniform(0, w), rng.uniform(1.5, 3)
            img[(yy - cy) ** 2 + (xx - cx) ** 2 <= rr * rr] = 200
        img[rng.random((h, w)) < 0.05] = 90
        np.savez_compressed(os.path.join(HERE, f"rec_sections_{w}x{h}.npz"), c1=img, c2=img,
                            normC=ref.rec_sections(img, img))
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
