"""The numpy oracle against the live reference library (oracle/_ref), on
inputs other than the committed fixtures.  Skipped where the library was not
built (it is built from the reference sources by oracle/Makefile).  CPU only."""
import numpy as np
import pytest

from oracle import mat3d_oracle as O
from oracle import ref_lib

pytestmark = pytest.mark.skipif(not ref_lib.available(), reason="oracle/_ref/libmat3d_ref.so not built")

MAT = np.array([[70e9, 0.2, 40e6, 100e6, 1, 8e-2, 8e2], [3e9, 0.35, 250e6, 8006, 0.2, 8e-4, 8e3]])


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def random_rve(shape, vf, seed, nph=2):
    rng = np.random.default_rng(seed)
    r = (rng.random(shape) >= vf).astype(np.int32)
    if nph > 2:
        r[rng.random(shape) < 0.1] = 2
    return r.ravel()


@pytest.mark.parametrize("shape,seed,force", [((9, 10, 11), 0, 0), ((8, 8, 8), 1, 1), ((8, 8, 8), 2, 2)])
def test_elastic_random_rves(shape, seed, force):
    ref = ref_lib.RefLib()
    rve = random_rve(shape, 0.3, seed)
    E = np.array([2e-4, -1e-4, 3e-4, 1e-4, 0, 5e-5])
    r = ref.mech_run(shape, "e", MAT, rve, E, np.zeros(6), 1e-9, 1e-9, 1, force)
    o = O.MechOracle(*shape, "e")
    o.material(MAT, rve, force_scheme=force)
    o.set_load(E)
    assert o.run(1e-9, 1e-9) == r["sweeps"]
    assert rel(o.eps.reshape(6, -1), r["eps"]) < 1e-11


def test_three_phase_elastic():
    ref = ref_lib.RefLib()
    mat = np.vstack([MAT, [[200e9, 0.3, 1e30, 0, 1, 0, 1e30]]])
    shape = (8, 8, 8)
    rve = random_rve(shape, 0.25, 7, nph=3)
    E = np.array([1e-3, 0, 0, 0, 0, 0.0])
    r = ref.mech_run(shape, "e", mat, rve, E, np.zeros(6), 1e-9, 1e-9, 1, 0)
    o = O.MechOracle(*shape, "e")
    o.material(mat, rve)
    o.set_load(E)
    assert o.run(1e-9, 1e-9) == r["sweeps"]
    assert rel(o.sig.reshape(6, -1), r["sig"]) < 1e-11


def test_thermal_noncubic_is_flux_based_quirk():
    """Integer-division scheme choice: km > ki with any inclusion -> flux-based."""
    ref = ref_lib.RefLib()
    shape = (8, 8, 8)
    rve = random_rve(shape, 0.2, 3)
    r = ref.therm_run(shape, 5.0, 2.0, rve, np.array([1.0, 0, 0]), 1e-9, 1e-9)
    o = O.ThermOracle(*shape)
    o.material(5.0, 2.0, rve)
    assert r["scheme"] == 2 and not o.grad_based
    o.set_load(np.array([1.0, 0, 0]))
    assert o.run(1e-9, 1e-9) == r["sweeps"]
    assert rel(o.grad.reshape(3, -1), r["grad"]) < 1e-11
