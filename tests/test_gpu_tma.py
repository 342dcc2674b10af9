"""The TMA-staged y pass (M3D_TMA_Y=1: persistent CTAs, tiles copied by the
Tensor Memory Accelerator into swizzled shared memory and stored back by it)
against the default y pass.  The per-column FFT arithmetic is the same, so
fields must be bitwise identical; covered: one-box and two-box tiles (FP32
lines of 32/48 points use 32-column tiles), FP64 (two boxes per tile) and a
partial last kz tile."""
import numpy as np
import pytest

import mat3d_b200 as m3d

pytestmark = pytest.mark.gpu

MAT = np.array([[70e9, 0.2, 1e30, 0, 1, 0, 1e30], [3e9, 0.35, 1e30, 0, 1, 0, 1e30]])


def sphere_rve(N, r):
    X, Y, Z = np.meshgrid(np.arange(N), np.arange(N), np.arange(N), indexing="ij")
    g = np.ones((N, N, N), np.int32)
    g[(X - N / 2) ** 2 + (Y - N / 2) ** 2 + (Z - N / 2) ** 2 <= r * r] = 0
    return g.ravel()


def solve(N, prec, kind, tma, monkeypatch):
    monkeypatch.setenv("M3D_TMA_Y", "1" if tma else "0")
    s = m3d.Solver(kind, N, N, N, 0, prec, 2)
    rve = sphere_rve(N, 0.3 * N)
    if kind == m3d.KIND_MECH:
        s.set_material_mech(MAT, rve)
        loads = [np.array([1e-3, 0, 0, 0, 0, 0.0]), np.array([0, 0, 0, 4e-4, 0, 0.0])]
    else:
        s.set_material_thermal(1.0, 30.0, rve)
        loads = [np.array([0, 0, 1.0]), np.array([0.5, 1.0, 0])]
    for b in range(2):
        s.set_load(loads[b], None, b=b)
    s.run(1e-5 if prec == "fp32" else 1e-9, 0, 1, m3d.CRIT_RESIDUAL)
    out = [s.field(m3d.FIELD_STRAIN, b) for b in range(2)], s.stats()
    s.close()
    return out


@pytest.mark.parametrize("N,prec,kind", [(32, "fp32", m3d.KIND_MECH), (48, "fp32", m3d.KIND_THERMAL),
                                         (64, "fp64", m3d.KIND_MECH), (128, "fp32", m3d.KIND_THERMAL),
                                         (32, "fp32_refine", m3d.KIND_THERMAL)])
def test_tma_ypass_equals_default(N, prec, kind, monkeypatch):
    (fa, sa) = solve(N, prec, kind, False, monkeypatch)
    (fb, sb) = solve(N, prec, kind, True, monkeypatch)
    assert sa["sweeps"] == sb["sweeps"]
    for a, b in zip(fa, fb):
        assert np.array_equal(a, b)
