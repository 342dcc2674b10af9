"""The autotuner (m3d_autotune, m3d_batch_set_autotune): it times the launch
schedules that compute the same sweep and keeps the fastest.  Results under
the tuned schedule agree with the default schedule to rounding (the generic
and compile-time FFT kernels associate sums differently)."""
import numpy as np
import pytest

import mat3d_b200 as m3d

pytestmark = pytest.mark.gpu

MAT = np.array([[70e9, 0.2, 1e30, 0, 1, 0, 1e30], [3e9, 0.35, 1e30, 0, 1, 0, 1e30]])


def sphere_rve(shape, r):
    Nx, Ny, Nz = shape
    X, Y, Z = np.meshgrid(np.arange(Nx), np.arange(Ny), np.arange(Nz), indexing="ij")
    g = np.ones(shape, np.int32)
    g[(X - Nx / 2) ** 2 + (Y - Ny / 2) ** 2 + (Z - Nz / 2) ** 2 <= r * r] = 0
    return g.ravel()


def homog(shape, prec, tune):
    s = m3d.Solver(m3d.KIND_MECH, *shape, 0, prec, 6)
    s.set_material_mech(MAT, sphere_rve(shape, 0.3 * min(shape)))
    t = s.autotune(tune) if tune is not None else None
    Ce, *_ = s.homogenize(1e-9, 0, m3d.CRIT_RESIDUAL)
    s.close()
    return Ce, t


@pytest.mark.parametrize("shape,prec", [((32, 32, 32), "fp32_refine"), ((24, 20, 28), "fp64")])
def test_tuned_schedule_matches_default(shape, prec):
    C0, _ = homog(shape, prec, None)
    C1, t = homog(shape, prec, 3)
    assert t["candidates"] >= 2 and t["sweep_us"] > 0
    if shape[0] == 24:
        assert t["fast"] == 0  # no compile-time kernel for these lengths
    assert np.abs(C1 - C0).max() / np.abs(C0).max() < 1e-8
    # a later handle of the same shape reuses the remembered schedule without timing
    C2, t2 = homog(shape, prec, 0)
    keys = ("fast", "tma_y", "G", "tzy", "tzx", "slab")
    assert {k: t2[k] for k in keys} == {k: t[k] for k in keys}
    assert np.array_equal(C2, C1)


def test_apply_without_tuning_first_fails():
    s = m3d.Solver(m3d.KIND_THERMAL, 14, 14, 14, 0, "fp64", 3)
    s.set_material_thermal(1.0, 10.0, sphere_rve((14, 14, 14), 4.0))
    with pytest.raises(m3d.M3DError):
        s.autotune(0)
    s.close()


def test_batch_autotune():
    members = [((16, 16, 16), 3.0 + i) for i in range(3)] + [((32, 32, 32), 8.0)]
    out = []
    for tune in (False, True):
        bt = m3d.Batch(m3d.KIND_MECH, "fp32_refine")
        bt.set_autotune(tune)
        for shape, r in members:
            bt.add_mech(shape, MAT, sphere_rve(shape, r))
        Ce, _, _ = bt.homogenize(1e-9)
        st = bt.stats()
        assert st["autotuned"] == (2 if tune else 0)
        out.append(Ce)
        bt.close()
    assert np.abs(out[1] - out[0]).max() / np.abs(out[0]).max() < 1e-8


@pytest.mark.parametrize("shape", [(45, 45, 45), (48, 40, 36)])
def test_radix_schedules_agree(shape, monkeypatch):
    """Every radix-stage order of the generic line FFTs (the autotuner's
    schedule candidates) gives the same FP64 field to 1e-12."""
    monkeypatch.setenv("M3D_GENERIC_FFT", "1")
    Nx, Ny, Nz = shape
    X, Y, Z = np.meshgrid(np.arange(Nx), np.arange(Ny), np.arange(Nz), indexing="ij")
    rve = np.ones(shape, np.int32)
    rve[(X - Nx / 2) ** 2 + (Y - Ny / 2) ** 2 + (Z - Nz / 2) ** 2 <= (min(shape) / 4) ** 2] = 0
    rve = rve.ravel()
    out = []
    for sched in range(4):
        monkeypatch.setenv("M3D_FFT_SCHEDULE", str(sched))
        s = m3d.Solver(m3d.KIND_THERMAL, *shape, 0, "fp64", 1)
        s.set_material_thermal(1.0, 20.0, rve)
        s.set_load(np.array([0.1, 0.0, 1.0]))
        s.run(1e-10, 0, 1, m3d.CRIT_RESIDUAL)
        out.append(s.field(m3d.FIELD_STRAIN))
        s.close()
    for f in out[1:]:
        assert np.linalg.norm(f - out[0]) / np.linalg.norm(out[0]) < 1e-12
