"""Asynchronous field export (m3d_get_field_async / m3d_wait_field): the
field is written into the handle's export buffer on the device and copied to
host memory on a copy stream, so a following solve may run while the copy is
in flight.  The copied field equals the synchronous m3d_get_field of the same
solve, also when the next solve (another load) has already overwritten the
state, and two exports in a row keep their order."""
import numpy as np
import pytest
import torch

import mat3d_b200 as m3d

pytestmark = pytest.mark.gpu


def sphere_rve(N, r):
    X, Y, Z = np.meshgrid(np.arange(N), np.arange(N), np.arange(N), indexing="ij")
    rve = np.ones((N, N, N), np.int32)
    rve[(X - N / 2) ** 2 + (Y - N / 2) ** 2 + (Z - N / 2) ** 2 <= r * r] = 0
    return rve.ravel()


@pytest.mark.parametrize("kind", ["thermal", "mech"])
def test_async_export_matches_sync(kind):
    N = 32
    rve = sphere_rve(N, 8)
    if kind == "thermal":
        s = m3d.Solver(m3d.KIND_THERMAL, N, N, N, 0, "fp32_refine", 1)
        s.set_material_thermal(1.0, 30.0, rve)
        loads = [np.array([0.0, 0.0, 1.0]), np.array([1.0, 0.5, 0.0])]
    else:
        s = m3d.Solver(m3d.KIND_MECH, N, N, N, m3d.ELASTIC, "fp64", 1)
        s.set_material_mech(np.array([[70e9, 0.2, 1e30, 0, 1, 0, 1e30], [3e9, 0.35, 1e30, 0, 1, 0, 1e30]]), rve)
        loads = [np.array([1e-3, 0, 0, 0, 0, 0.0]), np.array([0, 2e-4, 0, 0, 0, 1e-3])]
    n = s.V * s.C
    pinned = [torch.empty(n, dtype=torch.float64).pin_memory().numpy() for _ in range(2)]
    ref = []
    for E in loads:
        s.set_load(E)
        s.run(1e-9, 1e-9, 1, m3d.CRIT_RESIDUAL)
        ref.append(s.field(m3d.FIELD_STRAIN).copy())
    for k in range(2):  # two rounds: the handle's copy stream is reused
        for i, E in enumerate(loads):
            s.set_load(E)
            s.run(1e-9, 1e-9, 1, m3d.CRIT_RESIDUAL)
            s.field_async(pinned[i], m3d.FIELD_STRAIN)  # copy of solve i overlaps solve i + 1
        s.wait_field()
        for i in range(2):
            assert np.array_equal(pinned[i].reshape(s.V, s.C).T, ref[i])
    s.close()
