"""Compacted sweeps of multi-entry graph solves (mat3d_b200/csrc/solver.cu,
`compact_levels`): once entries converge, each sweep's CTAs are mapped to the
entries still iterating (a live list rebuilt after every sweep) and the loop
moves to smaller launch grids (B, B/2, B/4, ...); opt-in with
`M3D_COMPACT=1`.  Only the CTA-to-entry mapping changes -- every entry runs
the same arithmetic and the same fixed-order reductions -- so a compacted
solve equals the uncompacted one bit for bit, entry by entry, with the same
sweep counts.

The cases mix RVEs and load directions whose sweep counts differ, so the live
list shrinks during the solve, and cover the two-pass (thermal) and five-pass
(elastic) sweeps, the refinement's inner loop, the generic line-FFT kernels
(a 40^3 grid) and the TMA-staged y pass.
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


def rves(N, n):
    rng = np.random.default_rng(7)
    return [sphere_rve(N, N * rng.uniform(0.15, 0.35), rng.uniform(0.3, 0.7, 3) * N) for _ in range(n)]


def thermal_homogenize(N, prec, tol, compact, monkeypatch, extra_env=()):
    monkeypatch.setenv("M3D_COMPACT", "1" if compact else "0")
    for k, v in extra_env:
        monkeypatch.setenv(k, v)
    contrasts = [(1.0, 3.0), (1.0, 100.0), (30.0, 25.0), (1.0, 40.0)]  # gradient- and flux-based schemes
    rs = rves(N, len(contrasts))
    s = m3d.Solver(m3d.KIND_THERMAL, N, N, N, 0, prec, nrve=len(rs), nload=3)
    for r, (g, (km, ki)) in enumerate(zip(rs, contrasts)):
        s.set_material_thermal(km, ki, g, rve=r)
    K, *_ = s.homogenize(tol, 0, m3d.CRIT_RESIDUAL)
    ent = [s.entry_stats(b) for b in range(len(rs) * 3)]
    fields = [s.field(m3d.FIELD_STRAIN, b) for b in range(len(rs) * 3)]
    st = s.stats()
    s.close()
    return K, ent, fields, st


def mech_homogenize(N, prec, tol, compact, monkeypatch, extra_env=()):
    monkeypatch.setenv("M3D_COMPACT", "1" if compact else "0")
    for k, v in extra_env:
        monkeypatch.setenv(k, v)
    contrasts = [2.0, 30.0, 80.0]
    rs = rves(N, len(contrasts))
    s = m3d.Solver(m3d.KIND_MECH, N, N, N, m3d.ELASTIC, prec, nrve=len(rs), nload=6)
    for r, (g, c) in enumerate(zip(rs, contrasts)):
        mat = np.array([[c * 3e9, 0.2, 1e30, 0, 1, 0, 1e30], [3e9, 0.35, 1e30, 0, 1, 0, 1e30]])
        s.set_material_mech(mat, g, rve=r)
    C, *_ = s.homogenize(tol, 0, m3d.CRIT_RESIDUAL)
    ent = [s.entry_stats(b) for b in range(len(rs) * 6)]
    fields = [s.field(m3d.FIELD_STRAIN, b) for b in range(len(rs) * 6)]
    st = s.stats()
    s.close()
    return C, ent, fields, st


def check_equal(a, b):
    Ka, ea, fa, sa = a
    Kb, eb, fb, sb = b
    assert [e["sweeps"] for e in ea] == [e["sweeps"] for e in eb]
    assert [e["iters"] for e in ea] == [e["iters"] for e in eb]
    assert len(set(e["sweeps"] for e in ea)) > 1  # the entries do converge at different sweeps
    assert sa["sweeps"] == sb["sweeps"]
    assert np.array_equal(Ka, Kb)
    for x, y in zip(fa, fb):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("prec,tol", [("fp32", 1e-5), ("fp64", 1e-9), ("fp32_refine", 1e-9)])
def test_compacted_thermal_equals_uncompacted(prec, tol, monkeypatch):
    check_equal(thermal_homogenize(32, prec, tol, True, monkeypatch),
                thermal_homogenize(32, prec, tol, False, monkeypatch))


@pytest.mark.parametrize("prec,tol", [("fp32", 1e-5), ("fp32_refine", 1e-8)])
def test_compacted_elastic_equals_uncompacted(prec, tol, monkeypatch):
    check_equal(mech_homogenize(32, prec, tol, True, monkeypatch),
                mech_homogenize(32, prec, tol, False, monkeypatch))


def test_compacted_generic_and_tma_y_kernels(monkeypatch):
    # 40^3: generic (shared-memory Stockham) line FFTs; 32^3 with the TMA-staged y pass
    check_equal(mech_homogenize(40, "fp32_refine", 1e-8, True, monkeypatch),
                mech_homogenize(40, "fp32_refine", 1e-8, False, monkeypatch))
    env = (("M3D_TMA_Y", "1"),)
    check_equal(thermal_homogenize(32, "fp32", 1e-5, True, monkeypatch, env),
                thermal_homogenize(32, "fp32", 1e-5, False, monkeypatch, env))
