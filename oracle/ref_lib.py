"""ctypes wrapper of oracle/_ref/libmat3d_ref.so (the reference's own solver
sources built by oracle/Makefile).  TEST INFRASTRUCTURE ONLY: used by the
fixture generator, the CPU tests and the CPU-baseline legs of bench.py.

Fields come back in the reference's AoS layout (voxel-major, c values per
voxel), reshaped here to (c, V) like the reference's Eigen c x N^3 matrices.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libmat3d_ref.so")


def available() -> bool:
    return os.path.exists(REF_SO)


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class RefLib:
    def __init__(self, path: str = REF_SO, fft_threads: int = 3):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle` where the reference sources exist")
        self.L = ctypes.CDLL(path)
        self.threads = fft_threads

    def fft_r2c(self, x):
        Nx, Ny, Nz, c = x.shape
        xin = np.ascontiguousarray(x, np.float64)
        out = np.zeros((Nx, Ny, Nz // 2 + 1, c), np.complex128)
        self.L.ref_fft_r2c(Nx, Ny, Nz, c, _p(xin), _p(out))
        return out

    def fft_c2r(self, spec, shape):
        Nx, Ny, Nz = shape
        c = spec.shape[-1]
        sin = np.ascontiguousarray(spec, np.complex128)
        out = np.zeros((Nx, Ny, Nz, c))
        self.L.ref_fft_c2r(Nx, Ny, Nz, c, _p(sin), _p(out))
        return out

    def mech_run(self, shape, behav, mat, rve, E, X0, tol_field, tol_eq, nInc=1, force_scheme=0):
        Nx, Ny, Nz = shape
        V = Nx * Ny * Nz
        mat = np.ascontiguousarray(mat, np.float64)
        rve = np.ascontiguousarray(np.asarray(rve).ravel(), np.int32)
        E = np.ascontiguousarray(E, np.float64)
        X0 = np.ascontiguousarray(X0, np.float64)
        eps, sig, ex = np.zeros(6 * V), np.zeros(6 * V), np.zeros(V)
        prop = np.zeros(max(nInc, 1) * 9)
        sw, sch, ni, lm = ctypes.c_longlong(), ctypes.c_int(), ctypes.c_int(), np.zeros(2)
        D = ctypes.c_double
        self.L.ref_mech_run(Nx, Ny, Nz, behav.encode(), _p(mat), mat.shape[0], _p(rve), _p(E), _p(X0), D(tol_field),
                            D(tol_eq), nInc, force_scheme, self.threads, _p(eps), _p(sig), _p(ex), _p(prop),
                            ctypes.byref(sw), ctypes.byref(sch), ctypes.byref(ni), _p(lm))
        return dict(eps=eps.reshape(V, 6).T.copy(), sig=sig.reshape(V, 6).T.copy(), extra=ex,
                    prop=prop.reshape(-1, 9)[: ni.value], sweeps=sw.value, scheme=sch.value, ninc=ni.value,
                    la0=lm[0], mu0=lm[1])

    def mech_homog(self, shape, mat, rve, tol_field, tol_eq, force_scheme=0):
        Nx, Ny, Nz = shape
        mat = np.ascontiguousarray(mat, np.float64)
        rve = np.ascontiguousarray(np.asarray(rve).ravel(), np.int32)
        C, S, ep, sg, E3 = np.zeros(36), np.zeros(36), np.zeros(36), np.zeros(36), np.zeros(3)
        sw, sch = ctypes.c_longlong(), ctypes.c_int()
        D = ctypes.c_double
        self.L.ref_mech_homog(Nx, Ny, Nz, _p(mat), mat.shape[0], _p(rve), D(tol_field), D(tol_eq), force_scheme,
                              self.threads, None, _p(C), _p(S), _p(ep), _p(sg), ctypes.byref(sw), ctypes.byref(sch),
                              _p(E3))
        return dict(C=C.reshape(6, 6), S=S.reshape(6, 6), epHomo=ep.reshape(6, 6), sigHomo=sg.reshape(6, 6),
                    sweeps=sw.value, scheme=sch.value, E123=E3)

    def therm_run(self, shape, km, ki, rve, E, tol_field, tol_eq):
        Nx, Ny, Nz = shape
        V = Nx * Ny * Nz
        rve = np.ascontiguousarray(np.asarray(rve).ravel(), np.int32)
        E = np.ascontiguousarray(E, np.float64)
        g, q = np.zeros(3 * V), np.zeros(3 * V)
        sw, sch = ctypes.c_longlong(), ctypes.c_int()
        D = ctypes.c_double
        self.L.ref_therm_run(Nx, Ny, Nz, D(km), D(ki), _p(rve), _p(E), D(tol_field), D(tol_eq), self.threads, _p(g),
                             _p(q), ctypes.byref(sw), ctypes.byref(sch))
        return dict(grad=g.reshape(V, 3).T.copy(), flux=q.reshape(V, 3).T.copy(), sweeps=sw.value, scheme=sch.value)

    def last_timing(self):
        """(set-up seconds, solve seconds) of the last mech_run / therm_run:
        constructor + material() + setLoad() versus runAnalysis()."""
        a, b = ctypes.c_double(), ctypes.c_double()
        self.L.ref_last_timing(ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def therm_homog(self, shape, km, ki, rve, tol_field, tol_eq):
        Nx, Ny, Nz = shape
        rve = np.ascontiguousarray(np.asarray(rve).ravel(), np.int32)
        K, R = np.zeros(9), np.zeros(9)
        sw, sch = ctypes.c_longlong(), ctypes.c_int()
        D = ctypes.c_double
        self.L.ref_therm_homog(Nx, Ny, Nz, D(km), D(ki), _p(rve), D(tol_field), D(tol_eq), self.threads, None, _p(K),
                               _p(R), ctypes.byref(sw), ctypes.byref(sch))
        return dict(K=K.reshape(3, 3), R=R.reshape(3, 3), sweeps=sw.value, scheme=sch.value)

    # ---- 2-D solver (src/2d/FFT_analysis2D.cpp) -----------------------------
    def mech2d_run(self, shape, props, rve, E):
        """material(props, RVE), setLoad(E), runAnalysis() (25 iterations);
        epsilon and sigma as (3, Nx*Ny) complex arrays."""
        Nx, Ny = shape
        xy = Nx * Ny
        props = np.ascontiguousarray(props, np.float64)
        rve = np.ascontiguousarray(np.asarray(rve).ravel(), np.int32)
        Ec = np.ascontiguousarray(np.asarray(E, np.complex128))
        eps, sig = np.zeros(3 * xy, np.complex128), np.zeros(3 * xy, np.complex128)
        self.L.ref_2d_run(Nx, Ny, _p(props), _p(rve), _p(Ec), _p(eps), _p(sig))
        return dict(eps=eps.reshape(xy, 3).T.copy(), sig=sig.reshape(xy, 3).T.copy())

    def mech2d_homog(self, shape, props, rve, E):
        """setLoad(E) then homogenization(): CHomo, epHomo, sigHomo (3 x 3)."""
        Nx, Ny = shape
        props = np.ascontiguousarray(props, np.float64)
        rve = np.ascontiguousarray(np.asarray(rve).ravel(), np.int32)
        Ec = np.ascontiguousarray(np.asarray(E, np.complex128))
        C, ep, sg = np.zeros(9), np.zeros(9), np.zeros(9)
        rc = self.L.ref_2d_homog(Nx, Ny, _p(props), _p(rve), _p(Ec), _p(C), _p(ep), _p(sg))
        if rc:
            raise RuntimeError(f"ref_2d_homog failed ({rc})")
        # Eigen storage is column-major
        return dict(C=C.reshape(3, 3).T, epHomo=ep.reshape(3, 3).T, sigHomo=sg.reshape(3, 3).T)

    # ---- microstructure reconstruction (src/rec/reconstruction.cpp) -----------
    def rec_run(self, shape, tpcf, n, beta, seed):
        """recPlan(TPCF, Nx, Ny, Nz).runRec(n, beta) with the stand-in generator
        seeded by `seed`: the binary field, the error track, iterations run."""
        Nx, Ny, Nz = shape
        t = np.ascontiguousarray(np.asarray(tpcf, np.float64).ravel())
        rve, err = np.zeros(t.size), np.zeros(n)
        self.L.ref_rec_run.restype = ctypes.c_int
        its = self.L.ref_rec_run(Nx, Ny, Nz, _p(t), n, ctypes.c_double(beta), ctypes.c_ulonglong(seed), _p(rve),
                                 _p(err))
        return dict(rve=rve, err=err, iterations=its)

    def ifftshift(self, a, shape):
        Nx, Ny, Nz = shape
        x = np.ascontiguousarray(np.asarray(a, np.float64).ravel())
        out = np.zeros_like(x)
        self.L.ref_ifftshift(_p(x), _p(out), Nx, Ny, Nz)
        return out

    def fft3(self, a, shape, sign):
        """One unnormalised 3-D complex transform through the stand-in FFTW
        plan the reconstruction runs on (sign -1 forward, +1 backward)."""
        Nx, Ny, Nz = shape
        x = np.ascontiguousarray(np.asarray(a, np.complex128).ravel())
        out = np.zeros_like(x)
        self.L.ref_fft3(ctypes.c_void_p(x.ctypes.data), ctypes.c_void_p(out.ctypes.data), Nx, Ny, Nz, sign)
        return out

    def rec_sections(self, c1, c2):
        """recPlan(CImg c1, CImg c2) + estimateNormFFT_RVE(): normC.  c1, c2:
        uint8 images indexed [y, x] (height x width)."""
        a1, a2 = (np.ascontiguousarray(np.asarray(c, np.uint8)) for c in (c1, c2))
        (h1, w1), (h2, w2) = a1.shape, a2.shape
        out = np.zeros(w1 * h1 * h2)
        self.L.ref_rec_sections.restype = ctypes.c_int
        rc = self.L.ref_rec_sections(ctypes.c_void_p(a1.ctypes.data), w1, h1, ctypes.c_void_p(a2.ctypes.data), w2, h2,
                                     _p(out))
        assert rc == 0, rc
        return out
