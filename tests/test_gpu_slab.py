"""Two-pass sweeps (x turnaround + y-z slab pass, mat3d_b200/csrc/passes_slab.cuh)
against the five-pass sweeps and the CPU oracle.

The slab pass runs wherever the per-phase operators act on each component
separately (every thermal scheme) and the grid has Ny == Nz of a compile-time
line length.  It changes only which real lines share a complex FFT, so:
  * FP32 solves: slab vs five-pass fields within 1e-5 relative, both within
    2e-4 of the FP64 oracle (the FP32 bound of tests/test_gpu_parity.py);
  * FP64 solves: slab vs five-pass within 1e-10;
  * FP32 + FP64 refinement to 1e-9: within 1e-7 of the oracle (the refinement
    bound), whichever sweep runs inside.
"""
import numpy as np
import pytest

import mat3d_b200 as m3d
from oracle import mat3d_oracle as O

pytestmark = pytest.mark.gpu


def sphere_rve(shape, r, center=None):
    Nx, Ny, Nz = shape
    X, Y, Z = np.meshgrid(np.arange(Nx), np.arange(Ny), np.arange(Nz), indexing="ij")
    c = center or (Nx / 2, Ny / 2, Nz / 2)
    rve = np.ones(shape, np.int32)
    rve[(X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2 <= r * r] = 0
    return rve.ravel()


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


def thermal_solve(shape, km, ki, rve, E, prec, tol, monkeypatch, slab, graph=True, batch=1):
    monkeypatch.setenv("M3D_NO_SLAB", "0" if slab else "1")
    monkeypatch.setenv("M3D_NO_GRAPH", "0" if graph else "1")
    s = m3d.Solver(m3d.KIND_THERMAL, *shape, 0, prec, batch)
    s.set_material_thermal(km, ki, rve)
    for b in range(batch):
        s.set_load(np.roll(E, b), None, b=b)
    s.run(tol, 0, 1, m3d.CRIT_RESIDUAL)
    st = s.stats()
    out = [s.field(m3d.FIELD_STRAIN, b) for b in range(batch)]
    s.close()
    return out, st


def oracle_grad(shape, km, ki, rve, E):
    o = O.ThermOracle(*shape)
    o.material(km, ki, rve)
    o.set_load(E)
    o.run(1e-12, 0, criterion=O.CRIT_RESIDUAL)
    return o.grad.reshape(3, -1)


@pytest.mark.parametrize("N", [32, 48, 64, 96, 128])
@pytest.mark.parametrize("km,ki", [(1.0, 100.0), (30.0, 25.0)])  # gradient-based, flux-based
def test_slab_fp32_matches_five_pass(N, km, ki, monkeypatch):
    shape = (N, N, N)
    rve = sphere_rve(shape, N / 4)
    E = np.array([0.2, 0.3, 1.0])
    (a,), sa = thermal_solve(shape, km, ki, rve, E, "fp32", 1e-6, monkeypatch, slab=True)
    (b,), sb = thermal_solve(shape, km, ki, rve, E, "fp32", 1e-6, monkeypatch, slab=False)
    assert sa["passes_per_sweep"] == 2 and sb["passes_per_sweep"] == 5
    assert abs(sa["iters"] - sb["iters"]) <= 2
    assert rel(a, b) < 1e-5, rel(a, b)
    if N <= 64:
        ref = oracle_grad(shape, km, ki, rve, E)
        assert rel(a, ref) < 2e-4


@pytest.mark.parametrize("N", [32, 48, 64])
def test_slab_fp64_matches_five_pass(N, monkeypatch):
    shape = (N, N, N)
    rve = sphere_rve(shape, N / 4 + 0.5)
    E = np.array([0.0, 0.3, 1.0])
    (a,), sa = thermal_solve(shape, 1.0, 100.0, rve, E, "fp64", 1e-10, monkeypatch, slab=True)
    (b,), sb = thermal_solve(shape, 1.0, 100.0, rve, E, "fp64", 1e-10, monkeypatch, slab=False)
    assert sa["passes_per_sweep"] == 2 and sb["passes_per_sweep"] == 5
    assert abs(sa["iters"] - sb["iters"]) <= 1
    assert rel(a, b) < 1e-10, rel(a, b)


@pytest.mark.parametrize("N", [64, 128])
def test_slab_refine_against_oracle(N, monkeypatch):
    shape = (N, N, N)
    rve = sphere_rve(shape, N / 4 - 2)
    E = np.array([0.0, 0.0, 1.0])
    (a,), sa = thermal_solve(shape, 1.0, 100.0, rve, E, "fp32_refine", 1e-9, monkeypatch, slab=True)
    assert sa["passes_per_sweep"] == 2 and sa["sweeps_fp32"] > 0 and sa["residual"] < 1e-9
    (b,), _ = thermal_solve(shape, 1.0, 100.0, rve, E, "fp32_refine", 1e-9, monkeypatch, slab=False)
    assert rel(a, b) < 1e-8
    if N == 64:
        assert rel(a, oracle_grad(shape, 1.0, 100.0, rve, E)) < 1e-7


def test_slab_non_cubic_x_and_batch(monkeypatch):
    """Nx != Ny = Nz, three load cases in one batch."""
    shape = (48, 64, 64)
    rve = sphere_rve(shape, 13.0)
    E = np.array([0.0, 0.0, 1.0])
    a, sa = thermal_solve(shape, 1.0, 100.0, rve, E, "fp64", 1e-10, monkeypatch, slab=True, batch=3)
    b, sb = thermal_solve(shape, 1.0, 100.0, rve, E, "fp64", 1e-10, monkeypatch, slab=False, batch=3)
    assert sa["passes_per_sweep"] == 2
    for w in range(3):
        assert rel(a[w], b[w]) < 1e-10


def test_slab_graph_equals_host_loop(monkeypatch):
    shape = (64, 64, 64)
    rve = sphere_rve(shape, 15.0)
    E = np.array([0.1, 0.0, 1.0])
    (a,), sa = thermal_solve(shape, 1.0, 100.0, rve, E, "fp32_refine", 1e-9, monkeypatch, slab=True, graph=True)
    (b,), sb = thermal_solve(shape, 1.0, 100.0, rve, E, "fp32_refine", 1e-9, monkeypatch, slab=True, graph=False)
    assert sa["sweeps_fp32"] == sb["sweeps_fp32"] and sa["sweeps_fp64"] == sb["sweeps_fp64"]
    assert np.array_equal(a, b)


def test_slab_multi_rve(monkeypatch):
    """Two RVEs with different schemes (gradient- and flux-based) in one multi-RVE
    solve: each equals its own single-RVE slab solve bitwise."""
    monkeypatch.setenv("M3D_NO_SLAB", "0")
    shape = (32, 32, 32)
    rves = [sphere_rve(shape, 8.0), sphere_rve(shape, 10.0)]
    ks = [(1.0, 100.0), (30.0, 25.0)]
    mb = m3d.Solver(m3d.KIND_THERMAL, *shape, 0, "fp32_refine", nrve=2, nload=3)
    for r in range(2):
        mb.set_material_thermal(*ks[r], rves[r], rve=r)
    K, *_ = mb.homogenize(1e-9, 0, m3d.CRIT_RESIDUAL)
    assert mb.stats()["passes_per_sweep"] == 2
    for r in range(2):
        s = m3d.Solver(m3d.KIND_THERMAL, *shape, 0, "fp32_refine", 3)
        s.set_material_thermal(*ks[r], rves[r])
        K1, *_ = s.homogenize(1e-9, 0, m3d.CRIT_RESIDUAL)
        assert np.array_equal(K[r], K1)


@pytest.mark.parametrize("N", [32, 64, 128])
@pytest.mark.parametrize("km,ki", [(1.0, 100.0), (30.0, 25.0)])  # gradient-based, flux-based
@pytest.mark.parametrize("prec,tol", [("fp32", 1e-6), ("fp32_refine", 1e-9), ("fp64", 1e-10)])
def test_rank_one_x_turnaround_matches_staged(N, km, ki, prec, tol, monkeypatch):
    """The thermal x turnaround in rank-one form (three forward, two inverse
    line FFTs) against the staged kernel that applies the Green operator mode
    by mode: FP32 fields within 1e-5, refined and FP64 fields within 1e-8."""
    shape = (N, N, N)
    rve = sphere_rve(shape, N / 4, center=(N / 2 + 1, N / 2, N / 2 - 1))
    E = np.array([0.2, 0.3, 1.0])
    out = []
    for r1 in ("1", "0"):
        monkeypatch.setenv("M3D_XTURN_R1", r1)
        (a,), st = thermal_solve(shape, km, ki, rve, E, prec, tol, monkeypatch, slab=True)
        out.append(a)
    assert rel(out[0], out[1]) < (1e-5 if prec == "fp32" else 1e-8), rel(out[0], out[1])


@pytest.mark.parametrize("N", [32, 48, 64, 96, 128])
@pytest.mark.parametrize("km,ki", [(1.0, 100.0), (30.0, 25.0)])  # gradient-based, flux-based
@pytest.mark.parametrize("prec,tol,batch", [("fp32", 1e-6, 1), ("fp32_refine", 1e-9, 1), ("fp32", 1e-6, 3)])
def test_tma_staged_rank_one_is_bitwise_equal(N, km, ki, prec, tol, batch, monkeypatch):
    """The rank-one x turnaround with its column loads staged by TMA does the
    plain rank-one kernel's arithmetic: equal fields and sweep counts, also
    with several entries converging at different sweeps (batch 3: the load
    rolled per entry) and on a grid whose last column group is short."""
    shape = (N, N, N)
    rve = sphere_rve(shape, N / 4, center=(N / 2 + 1, N / 2, N / 2 - 1))
    E = np.array([0.2, 0.3, 1.0])
    out, sts = [], []
    for tma in ("1", "0"):
        monkeypatch.setenv("M3D_XTURN_TMA", tma)
        f, st = thermal_solve(shape, km, ki, rve, E, prec, tol, monkeypatch, slab=True, batch=batch)
        out.append(f)
        sts.append(st)
    assert sts[0]["sweeps"] == sts[1]["sweeps"]
    for a, b in zip(*out):
        assert np.array_equal(a, b)
