"""The x turnaround with a warp per component (`k_xturn_cp`,
passes_fast.cuh) against the staged kernel whose warps hold all six
components of their own columns (`M3D_XTURN_CP=0`).  Per line and per mode
both do the same arithmetic, so the elastic linear solves (residual rule: the
operator keeps no sums) give equal bits and sweep counts; under the
reference stop rule and in J2 the turnaround also sums the convergence
check, in another order, so those agree to rounding.  Both elastic schemes
(strain-based: the stiff phase is the majority; stress-based: it is not),
compile-time grids with a short last column group, FP32 / FP64 /
refinement, multi-RVE entries.
"""
import numpy as np
import pytest

import mat3d_b200 as m3d

pytestmark = pytest.mark.gpu


def sphere_rve(N, r, center):
    X, Y, Z = np.meshgrid(np.arange(N), np.arange(N), np.arange(N), indexing="ij")
    rve = np.ones((N, N, N), np.int32)
    rve[(X - center[0]) ** 2 + (Y - center[1]) ** 2 + (Z - center[2]) ** 2 <= r * r] = 0
    return rve.ravel()


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


STIFF_INCLUSION = np.array([[70e9, 0.2, 1e30, 0, 1, 0, 1e30], [3e9, 0.35, 1e30, 0, 1, 0, 1e30]])  # stress-based
STIFF_MATRIX = np.array([[3e9, 0.35, 1e30, 0, 1, 0, 1e30], [70e9, 0.2, 1e30, 0, 1, 0, 1e30]])  # strain-based
J2_MAT = np.array([[400e9, 0.2, 1e30, 0, 1, 0, 1e30], [70e9, 0.33, 100e6, 1e9, 1, 0, 1e30]])


def solve(N, mat, prec, tol, cp, monkeypatch, criterion=m3d.CRIT_RESIDUAL, behav=m3d.ELASTIC, ninc=1):
    monkeypatch.setenv("M3D_XTURN_CP", "1" if cp else "0")
    rve = sphere_rve(N, N / 4, (N / 2 + 1, N / 2, N / 2 - 1))
    s = m3d.Solver(m3d.KIND_MECH, N, N, N, behav, prec, 1)
    s.set_material_mech(mat, rve)
    E = np.array([1e-3, 0, 0, 0, 0, 2e-4])
    s.set_load(E, np.array([1.0, 0, 0, 0, 0, 0]) if behav != m3d.ELASTIC else None)
    s.run(tol, tol, ninc, criterion)
    f = s.field(m3d.FIELD_STRAIN)
    sw = s.stats()["sweeps"]
    s.close()
    return f, sw


@pytest.mark.parametrize("N", [32, 48, 64, 96, 128])
@pytest.mark.parametrize("mat", [STIFF_INCLUSION, STIFF_MATRIX], ids=["stress_based", "strain_based"])
@pytest.mark.parametrize("prec,tol", [("fp32", 1e-5), ("fp32_refine", 1e-9), ("fp64", 1e-10)])
def test_component_parallel_equals_staged(N, mat, prec, tol, monkeypatch):
    a, sa = solve(N, mat, prec, tol, True, monkeypatch)
    b, sb = solve(N, mat, prec, tol, False, monkeypatch)
    assert sa == sb
    assert np.array_equal(a, b)


def test_component_parallel_multi_rve(monkeypatch):
    N = 48
    out = []
    for cp in ("1", "0"):
        monkeypatch.setenv("M3D_XTURN_CP", cp)
        s = m3d.Solver(m3d.KIND_MECH, N, N, N, m3d.ELASTIC, "fp32_refine", nrve=2, nload=6)
        s.set_material_mech(STIFF_INCLUSION, sphere_rve(N, 10, (20, 24, 26)), rve=0)
        s.set_material_mech(STIFF_MATRIX, sphere_rve(N, 12, (24, 22, 25)), rve=1)
        C, *_ = s.homogenize(1e-9, 0, m3d.CRIT_RESIDUAL)
        out.append(C)
        s.close()
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("N", [32, 64])
def test_component_parallel_reference_rule(N, monkeypatch):
    a, sa = solve(N, STIFF_INCLUSION, "fp64", 1e-8, True, monkeypatch, criterion=m3d.CRIT_REFERENCE)
    b, sb = solve(N, STIFF_INCLUSION, "fp64", 1e-8, False, monkeypatch, criterion=m3d.CRIT_REFERENCE)
    assert abs(sa - sb) <= 1
    assert rel(a, b) < 1e-9, rel(a, b)


@pytest.mark.parametrize("prec,bound", [("fp64", 1e-9), ("fp32", 1e-4)])
def test_component_parallel_j2(prec, bound, monkeypatch):
    a, sa = solve(32, J2_MAT, prec, 1e-6, True, monkeypatch, behav=m3d.J2, ninc=2)
    b, sb = solve(32, J2_MAT, prec, 1e-6, False, monkeypatch, behav=m3d.J2, ninc=2)
    assert abs(sa - sb) <= max(2, sb // 50), (sa, sb)
    assert rel(a, b) < bound, rel(a, b)


@pytest.mark.parametrize("N", [48, 96, 128])
@pytest.mark.parametrize("prec,tol", [("fp32", 1e-6), ("fp64", 1e-10)])
def test_component_parallel_thermal(N, prec, tol, monkeypatch):
    """Three components (the thermal operators with their rank-one kernels
    turned off): equal bits to the staged kernel."""
    monkeypatch.setenv("M3D_XTURN_R1", "0")
    out = []
    for cp in ("1", "0"):
        monkeypatch.setenv("M3D_XTURN_CP", cp)
        s = m3d.Solver(m3d.KIND_THERMAL, N, N, N, 0, prec, 1)
        s.set_material_thermal(1.0, 50.0, sphere_rve(N, N / 4, (N / 2 + 1, N / 2, N / 2 - 1)))
        s.set_load(np.array([0.2, 0.3, 1.0]))
        s.run(tol, 0, 1, m3d.CRIT_RESIDUAL)
        out.append((s.field(m3d.FIELD_STRAIN), s.stats()["sweeps"]))
        s.close()
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][0], out[1][0])
