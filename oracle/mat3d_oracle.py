"""CPU oracle: a numpy restatement of the reference's FFT homogenization path.

TEST INFRASTRUCTURE ONLY.  Only tests/, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of bench.py may import this
module, and only as the checker or the timed CPU baseline -- never as a
product code path.

Parity pin: this restatement is checked (tests/test_oracle_ref.py) against
``oracle/_ref/libmat3d_ref.so``, the reference's own solver sources
(src/3d/FFT_analysis3D.cpp, src/3dTherm/FFT_thermal3D.cpp) compiled unmodified
against stand-in headers for FFTW/Eigen/VTK (oracle/Makefile), and against the
golden fixtures in tests/golden/ that were generated from that library.

Everything is FP64.  Fields are stored component-major (SoA) as arrays of shape
``[c, Nx, Ny, Nz]``; the reference stores them voxel-major (AoS, Eigen 6 x N^3
column-major) with voxel index ``z + Nz*(y + Ny*x)``.  The R2C halving axis is z
(the fastest axis), the frequency vector is ``xi = (kz, ky, kx)`` (index 0 is
the z axis) and Voigt order is [11,22,33,23,13,12] with tensor shear, all as in
src/3d/FFT_analysis3D.cpp:115-150,198-211.

numpy.fft.irfftn has FFTW's c2r semantics for a non-Hermitian half spectrum
(complex passes first, imaginary parts of the DC/Nyquist bins of the last axis
ignored); numpy's 1/N normalisation equals the reference's ``/xyz``
(src/3d/FFT_analysis3D.cpp:268-279).
"""
from __future__ import annotations

import math

import numpy as np

VOIGT_PAIRS = [(0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1)]
SHEAR_W = np.array([1.0, 1.0, 1.0, 2.0, 2.0, 2.0])

CRIT_REFERENCE = 0  # the reference's stationarity stop rule
CRIT_RESIDUAL = 1   # product criterion: rms |x_c - x| / |E|


# ----------------------------------------------------------------------------
# shared helpers
# ----------------------------------------------------------------------------
def signed_freq(n: int, positive_nyquist: bool) -> np.ndarray:
    """Signed integer frequency of each FFT index.

    ``positive_nyquist=False``: x <= (N-1)/2 -> x, else x-N
    (src/3d/FFT_analysis3D.cpp:202-209, src/3dTherm/FFT_thermal3D.cpp:150-157).
    ``positive_nyquist=True``: x <= N/2 -> x, else x-N
    (src/3dTherm/FFT_thermal3D.cpp:113-120, :321-328).
    """
    idx = np.arange(n)
    lim = n // 2 if positive_nyquist else (n - 1) // 2
    return np.where(idx <= lim, idx, idx - n).astype(np.float64)


def xi_grid(Nx, Ny, Nz, positive_nyquist, x_wrap=None):
    """(xi0, xi1, xi2) = (kz, ky, kx) broadcast over the half spectrum [Nx, Ny, Nz//2+1].

    ``x_wrap`` replaces Nx in the wrap of the x index (the flux-based thermal
    Green operator wraps x with Ny, src/3dTherm/FFT_thermal3D.cpp:151)."""
    kx = signed_freq(Nx, positive_nyquist)
    if x_wrap is not None:
        idx = np.arange(Nx)
        lim = Nx // 2 if positive_nyquist else (Nx - 1) // 2
        kx = np.where(idx <= lim, idx, idx - x_wrap).astype(np.float64)
    ky = signed_freq(Ny, positive_nyquist)
    kz = signed_freq(Nz, positive_nyquist)[: Nz // 2 + 1]
    return (kz[None, None, :], ky[None, :, None], kx[:, None, None])


def fwd(field):
    """3-D R2C over the grid axes of an SoA field [c, Nx, Ny, Nz]."""
    return np.fft.rfftn(field, axes=(1, 2, 3))


def bwd(spec, shape):
    """3-D C2R (normalised by 1/N^3) over the grid axes."""
    return np.fft.irfftn(spec, s=shape, axes=(1, 2, 3))


def matvec(M_by_phase, phase, x):
    """y[:, v] = M[phase[v]] @ x[:, v] for SoA x (src/3d/FFT_analysis3D.cpp:236-247)."""
    out = np.empty_like(x)
    for p in range(M_by_phase.shape[0]):
        m = phase == p
        if np.any(m):
            out[:, m] = M_by_phase[p] @ x[:, m]
    return out


def iso_stiffness(la, mu):
    """Voigt (tensor-shear) isotropic stiffness (src/3d/FFT_analysis3D.cpp:457-462)."""
    C = np.zeros((6, 6))
    C[:3, :3] = la
    C[0, 0] = C[1, 1] = C[2, 2] = la + 2 * mu
    C[3, 3] = C[4, 4] = C[5, 5] = 2 * mu
    return C


def aos_to_soa(a, c, Nx, Ny, Nz):
    return np.ascontiguousarray(np.asarray(a, np.float64).reshape(Nx, Ny, Nz, c).transpose(3, 0, 1, 2))


def soa_to_aos(a):
    return np.ascontiguousarray(np.moveaxis(a, 0, -1)).reshape(-1)


# ----------------------------------------------------------------------------
# mechanics: FFT_Analysis3D
# ----------------------------------------------------------------------------
class MechOracle:
    """Restatement of ``FFT_Analysis3D`` (include/FFT_analysis3D.hpp:36-215)."""

    def __init__(self, Nx, Ny, Nz, behav="e"):
        # ctor, src/3d/FFT_analysis3D.cpp:25-152
        self.Nx, self.Ny, self.Nz = Nx, Ny, Nz
        self.shape = (Nx, Ny, Nz)
        self.V = Nx * Ny * Nz
        self.behav = behav
        self.sweeps = 0
        self.iters_per_inc = []

    # material(), src/3d/FFT_analysis3D.cpp:420-549
    def material(self, mat, rve, nph=None, force_scheme=0):
        mat = np.asarray(mat, np.float64)
        nph = mat.shape[0] if nph is None else nph
        El, v = mat[:nph, 0], mat[:nph, 1]
        self.Sy, self.Hh, self.n = mat[:nph, 2], mat[:nph, 3], mat[:nph, 4]
        self.P, self.Y0 = mat[:nph, 5], mat[:nph, 6]
        self.mu = El / (1 + v) / 2.0
        self.la = v * El / (1 + v) / (1 - 2 * v)
        self.K = self.la + (2.0 / 3.0) * self.mu
        self.El, self.v = El, v
        self.C = np.stack([iso_stiffness(self.la[i], self.mu[i]) for i in range(nph)])
        self.S = np.stack([np.linalg.inv(c) for c in self.C])
        self.phase = np.asarray(rve, np.int64).reshape(self.shape)
        self.nph = nph
        self.vol = np.array([np.count_nonzero(self.phase == k) / self.V for k in range(nph)])
        # max_min_Array keeps the FIRST index of a strict maximum (:5-23)
        idx_mu_max = int(np.argmax(self.mu))
        if self.behav == "e":
            K0 = np.sqrt(self.K.min() * self.K.max())
            self.mu0 = np.sqrt(self.mu.min() * self.mu.max())
            self.la0 = K0 - self.mu0 * 2.0 / 3.0
            self.strain_based = bool(self.vol[idx_mu_max] == self.vol.max())
        else:
            # non-elastic: strain-based, arithmetic-mean reference medium (:515-522)
            self.strain_based = True
            self.mu0 = (self.mu.min() + self.mu.max()) / 2
            self.la0 = (self.la.min() + self.la.max()) / 2
        if force_scheme in (1, 2):
            self.strain_based = force_scheme == 1
        self.C0 = iso_stiffness(self.la0, self.mu0)
        self.S0 = np.linalg.inv(self.C0)
        self.C_acc = np.stack([2 * np.linalg.inv(self.C[i] + self.C0) @ self.C0 for i in range(nph)])
        self.S_acc = np.stack([2 * np.linalg.inv(self.S[i] + self.S0) @ self.S0 for i in range(nph)])
        self.xi = xi_grid(self.Nx, self.Ny, self.Nz, positive_nyquist=False)

    # setGF()/multiplyGF(), src/3d/FFT_analysis3D.cpp:155-233, 297-348
    def apply_green(self, tau_hat):
        """-(Gamma0 : tau_hat) (strain-based) or -(Delta0 : tau_hat) (stress-based),
        shear inputs doubled, at every half-spectrum mode except k=0 (left 0)."""
        la0, mu0 = self.la0, self.mu0
        xi = self.xi
        nrm = xi[0] ** 2 + xi[1] ** 2 + xi[2] ** 2
        nrm = np.where(nrm == 0, 1.0, nrm)  # k = 0 is overwritten by the caller
        out = np.zeros_like(tau_hat)
        if self.strain_based:
            d1 = 1 / (4 * mu0)
            d2 = (la0 + mu0) / (mu0 * (la0 + 2 * mu0))

            def G(i, j, k, h):
                dl = lambda a, b: 1.0 if a == b else 0.0
                return (d1 / nrm) * (dl(k, i) * xi[h] * xi[j] + dl(h, i) * xi[k] * xi[j]
                                     + dl(k, j) * xi[h] * xi[i] + dl(h, j) * xi[k] * xi[i]) \
                    - (d2 * xi[i] * xi[j] * xi[k] * xi[h]) / (nrm * nrm)
        else:
            c1 = 2 * mu0 * (3 * la0 + 2 * mu0) / (la0 + 2 * mu0)
            c2 = 2 * mu0
            c3, c4 = (c1 - c2) / 2.0, c2 / 2.0

            def G(i, j, k, h):
                dl = lambda a, b: 1.0 if a == b else 0.0
                pr = lambda a, b: dl(a, b) - xi[a] * xi[b] / nrm
                return c3 * pr(i, j) * pr(k, h) + c4 * pr(i, k) * pr(j, h) + c4 * pr(i, h) * pr(j, k)
        for a, (i, j) in enumerate(VOIGT_PAIRS):
            acc = 0
            for b, (k, h) in enumerate(VOIGT_PAIRS):
                acc = acc + G(i, j, k, h) * tau_hat[b] * SHEAR_W[b]
            out[a] = -acc
        out[:, 0, 0, 0] = 0
        return out

    # setLoad(), src/3d/FFT_analysis3D.cpp:551-564
    def set_load(self, E, X0=None):
        self.E = np.asarray(E, np.float64).copy()
        self.X0 = np.zeros(6) if X0 is None else np.asarray(X0, np.float64).copy()
        full = np.broadcast_to(self.E[:, None, None, None], (6,) + self.shape).copy()
        if self.strain_based:
            self.eps = full
            if not hasattr(self, "sig"):
                self.sig = np.zeros_like(full)
        else:
            self.sig = full
            if not hasattr(self, "eps"):
                self.eps = np.zeros_like(full)

    # convergenceCheck(), src/3d/FFT_analysis3D.cpp:351-416
    def _convergence_terms(self, sig):
        t2 = fwd(sig)
        dd = np.sqrt(np.sum(SHEAR_W * (t2[:, 0, 0, 0].real ** 2 + t2[:, 0, 0, 0].imag ** 2)))
        xi = self.xi
        p = t2.real ** 2 + t2.imag ** 2
        z0, z1, z2 = xi
        s = (p[0] * z0 * z0 + p[1] * z1 * z1 + p[2] * z2 * z2
             + p[3] * ((z1 + z1) + (z2 + z2)) + p[4] * ((z0 + z0) + (z2 + z2)) + p[5] * ((z0 + z0) + (z1 + z1)))
        cc = np.sum(np.sqrt(np.abs(s[:, :, 1:])))
        return cc / dd / self.V

    def _stop_reference(self, it, sum_old):
        eq = self._convergence_terms(self.sig)
        if self.strain_based:
            diff_sum = abs((self.sig.sum() - sum_old) /
                           (self.V * (0.5 * self.C[0][0, 0] + 0.5 * self.C[min(1, self.nph - 1)][0, 0]) * self.E.sum()))
        else:
            diff_sum = abs((self.eps.sum() - sum_old) /
                           (self.V * (0.5 * self.S[0][0, 0] + 0.5 * self.S[min(1, self.nph - 1)][0, 0]) * self.E.sum()))
        diff_eq = abs(eq - self._eq_old)
        self._eq_old = eq
        self.last_eqvar = eq
        return diff_sum, diff_eq

    # runAnalysis() elastic branch, src/3d/FFT_analysis3D.cpp:749-794
    def _run_elastic(self, tol_field, tol_eq, criterion, max_iter):
        ph = self.phase
        if self.strain_based:
            self.sig = matvec(self.C, ph, self.eps)
        else:
            self.eps = matvec(self.S, ph, self.sig)
        it = 0
        self._eq_old = getattr(self, "_eq_old", 0.0)
        Enorm = np.sqrt(np.sum(SHEAR_W * self.E ** 2))
        self.residual = np.inf
        while True:
            if self.strain_based:
                sum_old = self.sig.sum()
                tau = self.sig - np.einsum("ab,bxyz->axyz", self.C0, self.eps)
                state = self.eps
            else:
                sum_old = self.eps.sum()
                tau = self.eps - np.einsum("ab,bxyz->axyz", self.S0, self.sig)
                state = self.sig
            t3 = self.apply_green(fwd(tau))
            t3[:, 0, 0, 0] = self.E * self.V
            xc = bwd(t3, self.shape)
            if criterion == CRIT_RESIDUAL:
                d = xc - state
                self.residual = np.sqrt(np.sum(SHEAR_W[:, None, None, None] * d * d) / self.V) / Enorm
            if self.strain_based:
                self.eps = self.eps + matvec(self.C_acc, ph, xc - self.eps)
                self.sig = matvec(self.C, ph, self.eps)
            else:
                self.sig = self.sig + matvec(self.S_acc, ph, xc - self.sig)
                self.eps = matvec(self.S, ph, self.sig)
            it += 1
            self.sweeps += 1
            if criterion == CRIT_REFERENCE:
                diff_sum, diff_eq = self._stop_reference(it, sum_old)
                if it > 1 and diff_eq < tol_eq and diff_sum < tol_field:
                    break
                if it > max_iter:
                    break
            else:
                if self.residual < tol_field:
                    break
                if it >= max_iter:
                    break
        self.iters_per_inc.append(it)
        return it

    # elastoPlastic(), sigma_eff_calculator(), src/3d/FFT_analysis3D.cpp:597-606, 640-691
    def _elasto_plastic(self):
        ph = self.phase
        self._sum_old = self.sig.sum()
        sig = self.sig_old + matvec(self.C, ph, self.eps - self.eps_old)
        sm = (sig[0] + sig[1] + sig[2]) / 3.0
        sd = sig.copy()
        sd[:3] -= sm
        seff = np.sqrt(1.5) * np.sqrt(np.sum(SHEAR_W[:, None, None, None] * sd * sd, axis=0))
        Sy, H, n, mu = self.Sy[ph], self.Hh[ph], self.n[ph], self.mu[ph]
        ep = self.ep_eff
        phi = seff - Sy - H * np.power(ep, n)
        dp = np.zeros_like(seff)
        act = phi > 0
        if np.any(act):
            s_e, S_, H_, n_, mu_, e_ = seff[act], Sy[act], H[act], n[act], mu[act], ep[act]
            x_o = np.zeros_like(s_e)
            x = np.zeros_like(s_e)
            live = np.ones(s_e.shape, bool)
            for _ in range(200):
                if not live.any():
                    break
                xl = x_o[live] - (s_e[live] - 3 * mu_[live] * x_o[live] - S_[live] - H_[live] * np.power(e_[live] + x_o[live], n_[live])) \
                    / (-3 * mu_[live] - H_[live] * n_[live] * np.power(e_[live] + x_o[live], n_[live] - 1))
                x[live] = xl
                x_o[live] = xl
                res = s_e[live] - 3 * mu_[live] * xl - S_[live] - H_[live] * np.power(e_[live] + xl, n_[live])
                if np.any(np.isnan(xl)):
                    raise FloatingPointError("Newton-Raphson failed (reference throws here, :672-673)")
                done = np.abs(res) < 1e-5
                li = np.flatnonzero(live)
                live[li[done]] = False
            dp[act] = x
            # sigma -= (1.5 x / sigma_eff) C sigma_d
            corr = np.zeros_like(sig)
            fac = np.where(act, 1.5 * dp / np.where(act, seff, 1.0), 0.0)
            Csd = matvec(self.C, ph, sd)
            corr = fac[None] * Csd
            sig = sig - corr
            sm = (sig[0] + sig[1] + sig[2]) / 3.0
            sd2 = sig.copy()
            sd2[:3] -= sm
            seff = np.where(act, np.sqrt(1.5) * np.sqrt(np.sum(SHEAR_W[:, None, None, None] * sd2 * sd2, axis=0)), seff)
        self.sig = sig
        self.seff = seff
        self.phi = phi
        self.dp = dp

    # elastoDamage(), src/3d/FFT_analysis3D.cpp:619-638
    def _elasto_damage(self):
        ph = self.phase
        self._sum_old = self.sig.sum() if hasattr(self, "sig") else 0.0
        Ce = matvec(self.C, ph, self.eps)
        Y = np.sqrt(np.sum(SHEAR_W[:, None, None, None] * Ce * self.eps, axis=0))
        self.d_old = self.d.copy()
        P, Y0 = self.P[ph], self.Y0[ph]
        dn = np.maximum(1 - np.exp(-P * (Y - Y0)), self.d_old)
        self.d = np.where(Y > Y0, dn, self.d)
        self.Y = Y
        self.sig = (1 - self.d)[None] * Ce

    def _constitutive(self):
        if self.behav == "ep":
            self._elasto_plastic()
        else:
            self._elasto_damage()

    # updateE(), old_iter_fields_update(), prod(), src/3d/FFT_analysis3D.cpp:566-594
    def _update_E(self):
        prod = lambda a, b: a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + 2 * a[3] * b[3] + 2 * a[4] * b[4] + 2 * a[5] * b[5]
        s_mean = self.sig.reshape(6, -1).sum(1) / self.V
        e_mean = self.eps.reshape(6, -1).sum(1) / self.V
        x = self.S0 @ s_mean - e_mean
        y = self.S0 @ self.X0
        k = (self.dE.sum() * self.incNo + prod(x, self.X0)) / prod(y, self.X0)
        self.E = k * (self.S0 @ self.X0) - self.S0 @ s_mean + e_mean

    # runAnalysis() ep/ed branch, src/3d/FFT_analysis3D.cpp:796-853
    def _run_inelastic(self, tol_field, tol_eq, nInc, criterion, max_iter, damage_stop):
        V = self.V
        self.nInc = nInc
        self.dE = self.E / (nInc * 1.0)
        self.E = self.dE.copy()
        self.set_load(self.E, self.X0)
        self.eps_old = np.zeros_like(self.eps)
        self.sig_old = np.zeros_like(self.eps)
        self.sig = np.zeros_like(self.eps)
        self.ep_eff = np.full(self.shape, 1.236547e-9)
        self.d = np.zeros(self.shape)
        self.d_old = np.zeros(self.shape)
        self.prop = np.zeros((nInc, 9))
        self.incNo = 0
        nx = 0
        self.ninc_done = nInc
        for i in range(nInc):
            self.incNo += 1
            it = 0
            self._eq_old = getattr(self, "_eq_old", 0.0)
            self._constitutive()
            while True:
                sig_hat = fwd(self.sig)
                eps_hat = fwd(self.eps)
                self._update_E()
                t3 = eps_hat + self.apply_green(sig_hat)
                t3[:, 0, 0, 0] = self.E * V
                eps_prev = self.eps
                self.eps = bwd(t3, self.shape)
                sum_old_before = self.sig.sum()
                self._constitutive()
                it += 1
                self.sweeps += 1
                if criterion == CRIT_REFERENCE:
                    eq = self._convergence_terms(self.sig)
                    diff_sum = abs((self.sig.sum() - self._sum_old) /
                                   (V * (0.5 * self.C[0][0, 0] + 0.5 * self.C[min(1, self.nph - 1)][0, 0]) * self.E.sum()))
                    diff_eq = abs(eq - self._eq_old)
                    self._eq_old = eq
                    if it > 1 and diff_eq < tol_eq and diff_sum < tol_field:
                        break
                    if it > max_iter:
                        break
                else:
                    d = self.eps - eps_prev
                    En = np.sqrt(np.sum(SHEAR_W * self.E ** 2))
                    self.residual = np.sqrt(np.sum(SHEAR_W[:, None, None, None] * d * d) / V) / En
                    if self.residual < tol_field or it >= max_iter:
                        break
            self.iters_per_inc.append(it)
            if self.behav == "ed" and i != 0 and damage_stop:
                # softening stop rule (:829-847) compares the increment's homogenized
                # stress with the previous one.  The reference reads row i before
                # export_homogen_var(i) fills it (an uninitialised read); the oracle
                # reads the fresh value here, which is what the rule intends.
                cur = self.sig.reshape(6, -1).sum(1) / V
                for j in range(6):
                    if self.X0[j] != 0 and cur[j] < self.prop[i - 1, j + 1]:
                        nx += 1
            if nx == 3:
                self.ninc_done = i
                break
            # export_homogen_var(), :722-746
            t = int(np.flatnonzero(self.X0 != 0)[0])
            self.prop[i, 0] = self.eps[t].sum() / V
            self.prop[i, 1:7] = self.sig.reshape(6, -1).sum(1) / V
            if self.behav == "ep":
                self.prop[i, 7] = self.seff.sum() / V
                self.prop[i, 8] = self.ep_eff.sum() / V
            else:
                self.prop[i, 7] = self.d.sum() / V
                self.prop[i, 8] = 0
            # update_old_Variable(), :693-719
            if self.behav == "ep":
                self.ep_eff = np.where(self.phi > 0, self.ep_eff + self.dp, self.ep_eff)
                self.sig_old = self.sig.copy()
            tmp = self.eps_old
            self.eps_old = self.eps.copy()
            self.eps = self.eps + (self.eps - tmp)
            self.E = self.E + self.dE
        return sum(self.iters_per_inc)

    def run(self, tol_field, tol_eq, nInc=1, criterion=CRIT_REFERENCE, max_iter=2000, damage_stop=True):
        if self.behav == "e":
            return self._run_elastic(tol_field, tol_eq, criterion, max_iter)
        return self._run_inelastic(tol_field, tol_eq, nInc, criterion, max_iter, damage_stop)

    # homogenization(), src/3d/FFT_analysis3D.cpp:856-903
    def homogenization(self, tol_field, tol_eq, criterion=CRIT_REFERENCE, max_iter=2000):
        self.behav = "e"
        ep = np.zeros((6, 6))
        sg = np.zeros((6, 6))
        for w in range(6):
            E = np.zeros(6)
            E[w] = 0.0005 if self.strain_based else 1.0e6
            self.set_load(E, E)
            self._run_elastic(tol_field, tol_eq, criterion, max_iter)
            sg[w, :] = self.sig.reshape(6, -1).sum(1) / self.V
            ep[:, w] = self.eps.reshape(6, -1).sum(1) / self.V
        if self.strain_based:
            CH = np.linalg.inv(ep) @ sg
            SH = np.linalg.inv(CH)
        else:
            SH = np.linalg.inv(sg) @ ep
            CH = np.linalg.inv(SH)
        self.CHomo, self.SHomo, self.epHomo, self.sigHomo = CH, SH, ep, sg
        return CH, SH

    # Hashin-Shtrikman bounds, src/3d/FFT_analysis3D.cpp:911-942
    def hs_bounds(self):
        mu, K, vf = self.mu, self.K, self.vol
        Gn, G1, Kn, K1 = mu.max(), mu.min(), K.max(), K.min()
        a1, an = -3 / (3 * K1 + 4 * G1), -3 / (3 * Kn + 4 * Gn)
        b1 = -(3 * (K1 + 2 * G1)) / ((3 * K1 + 4 * G1) * 5 * G1)
        bn = -(3 * (Kn + 2 * Gn)) / ((3 * Kn + 4 * Gn) * 5 * Gn)
        A1 = sum(vf[i] / ((1 / (K[i] - K1)) - a1) for i in range(len(K)) if K[i] != K1)
        An = sum(vf[i] / ((1 / (K[i] - Kn)) - an) for i in range(len(K)) if K[i] != Kn)
        B1 = sum(vf[i] / ((0.5 / (mu[i] - G1)) - b1) for i in range(len(K)) if mu[i] != G1)
        Bn = sum(vf[i] / ((0.5 / (mu[i] - Gn)) - bn) for i in range(len(K)) if mu[i] != Gn)
        Kmin, Kmax = K1 + A1 / (1 + a1 * A1), Kn + An / (1 + an * An)
        Gmin, Gmax = G1 + 0.5 * B1 / (1 + b1 * B1), Gn + 0.5 * Bn / (1 + bn * Bn)
        Emin, Emax = 9 * Kmin * Gmin / (3 * Kmin + Gmin), 9 * Kmax * Gmax / (3 * Kmax + Gmax)
        return dict(E_min=Emin, E_max=Emax, K_min=Kmin, K_max=Kmax, G_min=Gmin, G_max=Gmax)


# ----------------------------------------------------------------------------
# thermal: FFT_analysis3d_thermal
# ----------------------------------------------------------------------------
class ThermOracle:
    """Restatement of ``FFT_analysis3d_thermal`` (include/FFT_thermal3D.hpp:37-154)."""

    def __init__(self, Nx, Ny, Nz):
        self.Nx, self.Ny, self.Nz = Nx, Ny, Nz
        self.shape = (Nx, Ny, Nz)
        self.V = Nx * Ny * Nz
        self.sweeps = 0

    # material(), src/3dTherm/FFT_thermal3D.cpp:373-422
    def material(self, km, ki, rve, force_scheme=0):
        self.km, self.ki = float(km), float(ki)
        self.phase = np.asarray(rve, np.int64).reshape(self.shape)
        # vol_1 = RVE.sum()/xyz is an INTEGER division in the reference (:399):
        # it is 1 only when every voxel is phase 1, else 0.
        vol_1 = int(self.phase.sum()) // self.V
        self.grad_based = bool((vol_1 >= 0.5 and km > ki) or (vol_1 < 0.5 and km < ki))
        if force_scheme in (1, 2):
            self.grad_based = force_scheme == 1
        self.k0 = np.sqrt(ki * km)
        if self.grad_based:
            self.xi = xi_grid(self.Nx, self.Ny, self.Nz, positive_nyquist=True)
        else:
            self.xi = xi_grid(self.Nx, self.Ny, self.Nz, positive_nyquist=False, x_wrap=self.Ny)
        # K1 = 2(Km+K0)^-1 K0 etc. (:244-245, :257-258), all isotropic scalars
        k0 = self.k0
        self.acc_g = np.array([2 * k0 / (ki + k0), 2 * k0 / (km + k0)])  # by phase 0, 1
        r0, rm, ri = 1 / k0, 1 / km, 1 / ki
        self.acc_f = np.array([2 * r0 / (ri + r0), 2 * r0 / (rm + r0)])
        self.kph = np.array([ki, km])

    def _is_matrix(self):
        # multipKx()/strainUpdate() test `if (RVE(i))`: any nonzero id is the matrix (:186, :249)
        return (self.phase != 0).astype(np.int64)

    # setLoad(), :426-441
    def set_load(self, E):
        self.E = np.asarray(E, np.float64).copy()
        full = np.broadcast_to(self.E[:, None, None, None], (3,) + self.shape).copy()
        if self.grad_based:
            self.grad = full
            if not hasattr(self, "flux"):
                self.flux = np.zeros_like(full)
        else:
            self.flux = full
            if not hasattr(self, "grad"):
                self.grad = np.zeros_like(full)

    # setGF()/multiplyGF(), :98-175, :270-297
    def apply_green(self, t2):
        z = self.xi
        if self.grad_based:
            mm = self.k0 * (z[0] ** 2 + z[1] ** 2 + z[2] ** 2)
            mm = np.where(mm == 0, 1.0, mm)
            G = [[z[a] * z[b] / mm for b in range(3)] for a in range(3)]
        else:
            mm = z[0] ** 2 + z[1] ** 2 + z[2] ** 2
            mm = np.where(mm == 0, 1.0, mm)
            G = [[((1.0 if a == b else 0.0) - z[a] * z[b] / mm) * self.k0 for b in range(3)] for a in range(3)]
        out = np.empty_like(t2)
        for a in range(3):
            out[a] = G[a][0] * t2[0] + G[a][1] * t2[1] + G[a][2] * t2[2]
        out[:, 0, 0, 0] = 0
        return out

    # convergenceCheck(), :303-365
    def _convergence_terms(self):
        t2 = fwd(self.flux)
        dd = np.sqrt(np.sum(t2[:, 0, 0, 0].real ** 2 + t2[:, 0, 0, 0].imag ** 2))
        z = xi_grid(self.Nx, self.Ny, self.Nz, positive_nyquist=True)
        p = t2.real ** 2 + t2.imag ** 2
        cc = np.sum(np.sqrt(p[0] * z[0] ** 2 + p[1] * z[1] ** 2 + p[2] * z[2] ** 2))
        return cc / dd / self.V

    # runAnalysis(), :446-485
    def run(self, tol_field, tol_eq, criterion=CRIT_REFERENCE, max_iter=500):
        ph = self._is_matrix()
        kv = self.kph[ph]
        if self.grad_based:
            self.flux = kv[None] * self.grad
        else:
            self.grad = self.flux / kv[None]
        it = 0
        self._eq_old = getattr(self, "_eq_old", 0.0)
        En = np.sqrt(np.sum(self.E ** 2))
        while True:
            if self.grad_based:
                sum_old = self.flux.sum()
                pol = self.k0 * self.grad - self.flux
                state = self.grad
            else:
                sum_old = self.grad.sum()
                pol = self.flux / self.k0 - self.grad
                state = self.flux
            t3 = self.apply_green(fwd(pol))
            t3[:, 0, 0, 0] = self.E * self.V
            xc = bwd(t3, self.shape)
            if criterion == CRIT_RESIDUAL:
                d = xc - state
                self.residual = np.sqrt(np.sum(d * d) / self.V) / En
            if self.grad_based:
                self.grad = self.grad + self.acc_g[ph][None] * (xc - self.grad)
                self.flux = kv[None] * self.grad
            else:
                self.flux = self.flux + self.acc_f[ph][None] * (xc - self.flux)
                self.grad = self.flux / kv[None]
            it += 1
            self.sweeps += 1
            if criterion == CRIT_REFERENCE:
                eq = self._convergence_terms()
                if self.grad_based:
                    diff_sum = abs((self.flux.sum() - sum_old) / (self.V * (0.5 * self.ki + 0.5 * self.km) * self.E.sum()))
                else:
                    diff_sum = abs((self.grad.sum() - sum_old) /
                                   (self.V * (0.5 / self.ki + 0.5 / self.km) * self.E.sum()))
                diff_eq = abs(eq - self._eq_old)
                self._eq_old = eq
                if it > 1 and diff_eq < tol_eq and diff_sum < tol_field:
                    break
                if it > max_iter:
                    break
            else:
                if self.residual < tol_field or it >= max_iter:
                    break
        self.iters = it
        return it

    # homogenization(), :489-581
    def homogenization(self, tol_field, tol_eq, criterion=CRIT_REFERENCE, max_iter=500):
        G = np.zeros((3, 3))
        Q = np.zeros((3, 3))
        for w in range(3):
            E = np.zeros(3)
            E[w] = 1.0
            self.set_load(E)
            self.run(tol_field, tol_eq, criterion, max_iter)
            g = self.grad.reshape(3, -1).sum(1) / self.V
            q = self.flux.reshape(3, -1).sum(1) / self.V
            if self.grad_based:
                G[w, :] = g
                Q[:, w] = q
            else:
                Q[w, :] = q
                G[:, w] = g
        if self.grad_based:
            KH = np.linalg.inv(G) @ Q
            RH = np.linalg.inv(KH)
        else:
            RH = np.linalg.inv(Q) @ G
            KH = np.linalg.inv(RH)
        self.KHomo, self.RHomo = KH, RH
        return KH, RH

    # Mori-Tanaka and HS bounds, :582-592 (fi_m is an integer division there, too)
    def bounds(self):
        km, ki = self.km, self.ki
        fi_m = int(self.phase.sum()) // self.V
        fi_i = 1 - fi_m
        mt = km + (fi_i * (ki - km)) / (1 + fi_m * (ki - km) / (3 * km))
        up = fi_i * ki + fi_m * km - fi_i * fi_m * (km - ki) ** 2 / (3 * ki - fi_i * (ki - km))
        lo = fi_i * ki + fi_m * km - fi_i * fi_m * (km - ki) ** 2 / (3 * km + fi_m * (ki - km))
        return dict(mori_tanaka=mt, hs_low=lo, hs_up=up)


# ============================================================================
# 2-D elastic solver, src/2d/FFT_analysis2D.cpp (plane, 3 components
# [11, 22, 12] with tensor shear, complex fields, basic scheme, fixed number
# of iterations).
# ============================================================================
class Mech2DOracle:
    """Restatement of FFT_Analysis2D.  Fields are (3, Nx*Ny) complex with
    voxel index y + Ny*x (src/2d/FFT_analysis2D.cpp:11-19 allocates 3 x xy)."""

    # GF component s -> tensor indices (i, j, k, h)  (:64-70)
    Q = ((0, 0, 0, 0), (0, 0, 1, 1), (0, 0, 0, 1), (1, 1, 1, 1), (1, 1, 0, 1), (0, 1, 0, 1))
    # row j of the symmetric 3 x 3 operator -> GF component (:107-110)
    W = ((0, 1, 2), (1, 3, 4), (2, 4, 5))

    def __init__(self, Nx, Ny):
        self.Nx, self.Ny, self.xy = Nx, Ny, Nx * Ny
        self.eps = np.zeros((3, self.xy), np.complex128)
        self.sig = np.zeros((3, self.xy), np.complex128)
        self.E = np.zeros(3, np.complex128)

    def material(self, props, rve):  # :189-224
        Em, vm, Ei, vi = [float(p) for p in props[:4]]
        mum = Em / (1 + vm) / 2
        lam = vm * Em / (1 + vm) / (1 - 2 * vm)
        mui = Ei / (1 + vi) / 2
        lai = vi * Ei / (1 + vi) / (1 - 2 * vi)
        self.Cm = np.array([[lam + 2 * mum, lam, 0], [lam, lam + 2 * mum, 0], [0, 0, 2 * mum]])
        self.Ci = np.array([[lai + 2 * mui, lai, 0], [lai, lai + 2 * mui, 0], [0, 0, 2 * mui]])
        self.C0 = 1.0 * (self.Cm + self.Ci) / 2.0
        self.la0 = 1.0 * (lai + lam) / 2.0
        self.mu0 = 1.0 * (mui + mum) / 2.0
        self.rve = np.asarray(rve).ravel().astype(np.float64)

    def setLoad(self, E):  # :226-233
        self.E = np.asarray(E, np.complex128).copy()
        self.eps[:] = self.E[:, None]

    def green(self):  # setGF, :49-103 (x wraps with Ny as in :85-86)
        Nx, Ny = self.Nx, self.Ny
        d1 = 1 / (4 * self.mu0)
        d2 = (self.la0 + self.mu0) / (self.mu0 * (self.la0 + 2 * self.mu0))
        x = np.arange(Nx)
        y = np.arange(Ny)
        x1 = np.where(x <= (Nx - 1) // 2, x, -(Ny - x)).astype(np.float64)
        y1 = np.where(y <= (Ny - 1) // 2, y, -(Ny - y)).astype(np.float64)
        X, Y = np.meshgrid(x1, y1, indexing="ij")
        z = (X.ravel(), Y.ravel())
        n2 = z[0] * z[0] + z[1] * z[1]
        dl = lambda a, b: 1.0 if a == b else 0.0
        GF = np.zeros((6, self.xy))
        with np.errstate(divide="ignore", invalid="ignore"):
            for s, (i, j, k, h) in enumerate(self.Q):
                GF[s] = (d1 / n2) * (dl(k, i) * z[h] * z[j] + dl(h, i) * z[k] * z[j] + dl(k, j) * z[h] * z[i]
                                     + dl(h, j) * z[k] * z[i]) - (d2 * z[i] * z[j] * z[k] * z[h]) / (n2 * n2)
        return GF

    def iterate(self, GF):
        Nx, Ny, xy = self.Nx, self.Ny, self.xy
        # multipCx (:106-116): sigma = C(x) eps
        mtx = self.rve == 1
        self.sig = np.where(mtx[None, :], self.Cm @ self.eps, self.Ci @ self.eps)
        tau = self.sig - self.C0 @ self.eps  # runAnalysis :240
        t2 = np.fft.fft2(tau.reshape(3, Nx, Ny), axes=(1, 2)).reshape(3, xy)  # FFT_tau :118-122
        t1 = np.empty_like(t2)
        for j in range(3):  # multiplyGF :124-137
            w = self.W[j]
            t1[j] = -(GF[w[0]] * t2[0] + GF[w[1]] * t2[1] + GF[w[2]] * t2[2] * 2)
        t1[:, 0] = self.E * xy
        t2 = np.fft.ifft2(t1.reshape(3, Nx, Ny), axes=(1, 2)).reshape(3, xy) * xy  # FFTW backward, unnormalised
        self.eps = t2 / xy  # FFTBCKWRD_epsilon :140-145

    def runAnalysis(self, iterations=25):  # :235-247
        GF = self.green()
        for _ in range(iterations):
            self.iterate(GF)

    def homogenization(self, iterations=25):  # :250-283 (no setLoad between load cases)
        epH = np.zeros((3, 3))
        sgH = np.zeros((3, 3))
        for w in range(3):
            self.E = np.zeros(3, np.complex128)
            self.E[w] = 0.005
            self.runAnalysis(iterations)
            epH[w, :] = self.eps.real.sum(axis=1) / self.xy
            sgH[:, w] = self.sig.real.sum(axis=1) / self.xy
        C = np.linalg.inv(epH) @ sgH
        return C, epH, sgH


# ============================================================================
# Microstructure reconstruction by phase retrieval, src/rec/reconstruction.cpp
# (recon::recPlan from a two-point correlation function, runRec).
# ============================================================================
def _mix64(z):
    z = z + np.uint64(0x9E3779B97F4A7C15)
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def rand_pm1(seed, call, n):
    """The seeded counter-based draws that stand in for Eigen's setRandom:
    2 u - 1 with u = (mix(mix(seed * 0x100000001B3 + call) + i) >> 11) * 2^-53."""
    with np.errstate(over="ignore"):
        b = _mix64(np.uint64(seed) * np.uint64(0x100000001B3) + np.uint64(call))
        v = _mix64(b + np.arange(n, dtype=np.uint64))
    return 2.0 * ((v >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)) - 1.0


def tpcf_isotropic(N, A=25.0, Q=0.4, phi1=0.5):
    """The example TPCF of example/reconst3d/main.cpp:37-80 (scaled
    autocovariance f(r) = exp(-r/A) sin(Q r)/(Q r), S2 = f phi1 phi2 + phi1^2),
    centred at (N/2, N/2, N/2), before the driver's ifftshift."""
    m = N // 2
    i = np.arange(N) - m
    X, Y, Z = np.meshgrid(i, i, i, indexing="ij")
    r = np.sqrt(X * X + Y * Y + Z * Z * 1.0)
    with np.errstate(invalid="ignore", divide="ignore"):
        fr = np.exp(-r / A) * np.sin(Q * r) / (Q * r)
    fr[r == 0] = 1.0
    phi2 = 1 - phi1
    return (fr * phi1 * phi2 + phi1 * phi1).ravel()


def ifftshift3(a, Nx, Ny, Nz):
    """recon::ifftshift (:100-140): inverse of the centring shift, per axis
    by floor(n/2) (even n) or floor(n/2)+1 (odd n)."""
    return np.fft.ifftshift(np.asarray(a).reshape(Nx, Ny, Nz)).ravel()


class RecOracle:
    """recPlan(TPCF, Nx, Ny, Nz) (:213-240) and runRec(n, beta) (:283-400).

    `fft(a, sign)` is the unnormalised 3-D complex transform (sign -1 forward,
    +1 backward); numpy's by default.  The iteration is chaotic: a rounding
    difference of one unit grows by a factor of about three per iteration, so
    two implementations agree bit for bit only when they share every rounding
    step -- `fft` lets the pin tests run this restatement on the reference's
    own transform, and every other operation below keeps the reference's
    order (sequential error sum, sqrt(re^2 + im^2), atan2, division by xyz).
    """

    def __init__(self, tpcf, Nx, Ny, Nz, fft=None, libm_atan2=False):
        self.shape = (Nx, Ny, Nz)
        # numpy's arctan2 rounds differently from the C library's atan2 (which
        # std::arg calls) in a few ulps of cases; the pin tests take libm's
        self.atan2 = np.frompyfunc(math.atan2, 2, 1) if libm_atan2 else np.arctan2
        self.xyz = Nx * Ny * Nz
        self.normC = np.sqrt(np.abs(np.asarray(tpcf, np.float64).ravel()) * self.xyz)
        sh = self.shape
        self.fft = fft or (lambda a, sign: (np.fft.fftn(a.reshape(sh)) if sign < 0 else
                                            np.fft.ifftn(a.reshape(sh), norm="forward")).ravel())

    @classmethod
    def from_sections(cls, c1, c2, fft=None, fft2=None):
        """recPlan(CImg c1, CImg c2) (:145-206) + estimateNormFFT_RVE (:245-281).
        c1, c2: 8-bit images indexed [y, x]; grid width1 x height1 x height2.
        `fft2(a, (n0, n1), sign)` is the unnormalised 2-D complex transform."""
        c1 = np.asarray(c1).astype(np.int64)
        c2 = np.asarray(c2).astype(np.int64)
        (Ny, Nx), (Nz, Nzz) = c1.shape, c2.shape
        # CC1[k + j*Ny] = (int)C1(j, k) / Max, over j < Nx, k < Ny for both sections
        cc1 = (c1.T // c1.max()).ravel().astype(np.float64)
        cc2 = (c2[:Ny, :Nx].T // c2[:Ny, :Nx].max()).ravel().astype(np.float64)
        f2 = fft2 or (lambda a, sh, sign: (np.fft.fft2(a.reshape(sh)) if sign < 0 else
                                          np.fft.ifft2(a.reshape(sh), norm="forward")).ravel())

        def autocorr(cc, sh):
            sp = f2(cc.astype(np.complex128), sh, -1)
            v = sh[0] * sh[1] * sh[0] * sh[1]  # int arithmetic in the reference: wraps past 2^31
            den = float((v + 2 ** 31) % 2 ** 32 - 2 ** 31)
            p = (sp.real * sp.real + sp.imag * sp.imag) / den
            return f2(p.astype(np.complex128), sh, +1)

        cc3 = autocorr(cc1, (Nx, Ny))
        cc4 = autocorr(cc2, (Nz, Nzz))
        xyz = Nx * Ny * Nz
        f1 = cc3[0].real
        c3 = cc3.real.reshape(Nx, Ny)[:, :, None]
        c4 = cc4.real[:Nz][None, None, :]
        mh = ((c3 * c4 / f1 + (f1 - c3) * (f1 - c4) / (1 - f1)) * xyz).ravel()
        o = cls(np.zeros(xyz), Nx, Ny, Nz, fft=fft)
        MH = o.fft(mh.astype(np.complex128), -1)
        o.normC = np.sqrt(np.sqrt(MH.real * MH.real + MH.imag * MH.imag))
        return o

    def error(self, MT):
        """funcNormC (include/reconstruction.hpp:37-44): mean |(|MTilda| - normC)|, summed in voxel order."""
        a = np.abs(np.sqrt(MT.real * MT.real + MT.imag * MT.imag) - self.normC)
        return float(np.add.accumulate(a)[-1]) / self.xyz

    def start(self, seed):
        """The state runRec starts from (:289-293): mTilda = (U + 1) / 2 from the first draw."""
        st = dict(mT=((rand_pm1(seed, 0, self.xyz) + 1.0) * 0.5).astype(np.complex128), i=0, j=0, call=1,
                  seed=seed)
        return st

    def step(self, st, beta):
        """One pass of the runRec loop (:296-364) on state `st` (mTilda, i, j,
        draw counter); returns the recorded error.  The caller checks i < n
        before and err < 0.1 after, as the loop does."""
        xyz = self.xyz
        st["j"] += 1
        MT = self.fft(st["mT"], -1)
        err = self.error(MT)
        st["MT"] = MT
        if err < 0.1:
            return err
        at = lambda z: np.asarray(self.atan2(z.imag, z.real), np.float64)
        ang = at(MT)
        if np.remainder(st["i"] + 1, 150) == 0:  # restart the phases from a fresh draw
            r = rand_pm1(st["seed"], st["call"], xyz)
            st["call"] += 1
            MH = self.fft(r.astype(np.complex128), -1)
            ang = at(MH) * 0.3 + at(MT) * 0.7
        MH = self.normC * np.cos(ang) + 1j * (self.normC * np.sin(ang))
        mH = self.fft(MH, +1)
        re, im = mH.real / xyz, mH.imag / xyz
        mT = st["mT"]
        if st["j"] < 100:  # hybrid input-output projection
            k = re < 0
            re[k] = mT.real[k] - beta * re[k]
            im[k] = 0
            k = re > 1
            re[k] = mT.real[k] - beta * (re[k] - 1)
            im[k] = 0
            k = re > 1
            re[k] = 1
            im[k] = 0
        else:  # plain box projection
            k = re < 0
            re[k] = 0
            im[k] = 0
            k = re > 1
            re[k] = 1
            im[k] = 0
            if st["j"] > 200:
                st["j"] = 0
        st["mT"] = re + 1j * im
        st["i"] += 1
        return err

    def threshold(self, field):
        """The closing loop of runRec (:370-395): shift the 0.5 cut by 0.001 at a
        time until the phase-1 fraction is within 1e-4 of normC[0] / xyz (at
        most 202 tries)."""
        xyz = self.xyz
        ctr, x = 0, 0.0
        while True:
            b = np.where(field < 0.5 - x, 0.0, 1.0)
            vol_dif = b.sum() / (1.0 * xyz) - self.normC[0] / (1.0 * xyz)
            if vol_dif > 0:
                x -= 0.001
            else:
                x += 0.001
            if abs(vol_dif) < 0.0001 or ctr > 200:
                break
            ctr += 1
        return b

    def runRec(self, n, beta, seed):
        st = self.start(seed)
        err = np.zeros(n)
        while True:
            if st["i"] >= n:
                break
            i = st["i"]
            err[i] = self.step(st, beta)
            if err[i] < 0.1:
                break
        self.err = err
        self.iterations = int(np.count_nonzero(err))
        self.field = st["mT"].real.copy()
        self.rve = self.threshold(self.field)
        return self.rve
