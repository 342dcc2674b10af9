"""The graph-captured solve (one CUDA graph launch whose loops are conditional
while nodes re-armed on the device) against the host-driven loop (chunks of
sweeps with a host check of the done flags between chunks; selected here by
enabling per-sweep profiling).  Both run the same kernels on the same
entries, so fields, means and sweep counts must be identical."""
import numpy as np
import pytest

import mat3d_b200 as m3d

pytestmark = pytest.mark.gpu

MAT = np.array([[70e9, 0.2, 1e30, 0, 1, 0, 1e30], [3e9, 0.35, 1e30, 0, 1, 0, 1e30]])


def sphere_rve(shape, r):
    Nx, Ny, Nz = shape
    X, Y, Z = np.meshgrid(np.arange(Nx), np.arange(Ny), np.arange(Nz), indexing="ij")
    rve = np.ones(shape, np.int32)
    rve[(X - Nx / 2) ** 2 + (Y - Ny / 2) ** 2 + (Z - Nz / 2) ** 2 <= r * r] = 0
    return rve.ravel()


def solve(kind, shape, prec, crit, tol, host_loop, batch=2):
    s = m3d.Solver(kind, *shape, 0, prec, batch)
    rve = sphere_rve(shape, 0.3 * shape[0])
    if kind == m3d.KIND_MECH:
        s.set_material_mech(MAT, rve)
        loads = [np.array([1e-3, 0, 0, 0, 0, 0.0]), np.array([0, 0, 0, 0, 5e-4, 0.0])]
    else:
        s.set_material_thermal(1.0, 50.0, rve)
        loads = [np.array([0, 0, 1.0]), np.array([1.0, 0.5, 0])]
    for b in range(batch):
        s.set_load(loads[b % 2], None, b=b)
    if host_loop:
        s.set_profiling(True)
    s.run(tol, tol, 1, crit)
    out = dict(st=s.stats(), f=[s.field(m3d.FIELD_STRAIN, b) for b in range(batch)],
               m=[s.means(b) for b in range(batch)])
    s.close()
    return out


@pytest.mark.parametrize("kind,prec,crit", [
    (m3d.KIND_MECH, "fp64", m3d.CRIT_RESIDUAL),
    (m3d.KIND_MECH, "fp64", m3d.CRIT_REFERENCE),
    (m3d.KIND_MECH, "fp32", m3d.CRIT_RESIDUAL),
    (m3d.KIND_MECH, "fp32_refine", m3d.CRIT_RESIDUAL),
    (m3d.KIND_THERMAL, "fp64", m3d.CRIT_REFERENCE),
    (m3d.KIND_THERMAL, "fp32_refine", m3d.CRIT_RESIDUAL),
])
def test_graph_equals_host_loop(kind, prec, crit):
    shape = (16, 16, 16)
    tol = 1e-5 if prec == "fp32" else 1e-9
    g = solve(kind, shape, prec, crit, tol, host_loop=False)
    h = solve(kind, shape, prec, crit, tol, host_loop=True)
    for k in ("sweeps", "sweeps_fp64", "sweeps_fp32", "iters", "status"):
        assert g["st"][k] == h["st"][k], (k, g["st"][k], h["st"][k])
    assert g["st"]["residual"] == h["st"]["residual"]
    for a, b in zip(g["f"], h["f"]):
        assert np.array_equal(a, b)
    for (e1, s1), (e2, s2) in zip(g["m"], h["m"]):
        assert np.array_equal(e1, e2) and np.array_equal(s1, s2)


def test_graph_reused_across_runs_and_iteration_cap():
    """A second run on the same handle replays the cached graph; a run that
    hits its iteration cap ends with NOT_CONVERGED after exactly max_iter sweeps."""
    shape = (16, 16, 16)
    s = m3d.Solver(m3d.KIND_MECH, *shape, 0, "fp64", 1)
    s.set_material_mech(MAT, sphere_rve(shape, 5.0))
    s.set_load(np.array([1e-3, 0, 0, 0, 0, 0.0]))
    s.run(1e-9, 0, 1, m3d.CRIT_RESIDUAL)
    f1, st1 = s.field(m3d.FIELD_STRAIN), s.stats()
    s.set_load(np.array([1e-3, 0, 0, 0, 0, 0.0]))
    s.run(1e-9, 0, 1, m3d.CRIT_RESIDUAL)
    assert np.array_equal(f1, s.field(m3d.FIELD_STRAIN))
    assert s.stats()["iters"] == st1["iters"]
    rc = s.run(1e-30, 0, 1, m3d.CRIT_RESIDUAL, max_iter=7)
    assert rc == m3d.NOT_CONVERGED
    assert s.stats()["iters"] == 7
    s.close()


def test_field_into_caller_buffer():
    """Solver.field(out=...) writes the voxel-major field into a caller-owned
    buffer (pinned here) and equals the allocating form."""
    import torch
    shape = (16, 16, 16)
    s = m3d.Solver(m3d.KIND_THERMAL, *shape, 0, "fp64", 1)
    s.set_material_thermal(1.0, 20.0, sphere_rve(shape, 5.0))
    s.set_load(np.array([0, 0, 1.0]))
    s.run(1e-9, 0, 1, m3d.CRIT_RESIDUAL)
    want = s.field(m3d.FIELD_STRAIN)
    buf = torch.empty(3 * 16 ** 3, dtype=torch.float64).pin_memory().numpy()
    got = s.field(m3d.FIELD_STRAIN, out=buf)
    assert np.array_equal(got, want) and np.shares_memory(got, buf)
    with pytest.raises(ValueError):
        s.field(m3d.FIELD_STRAIN, out=np.empty(10))
    s.close()
