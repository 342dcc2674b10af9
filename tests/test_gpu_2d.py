"""The 2-D solver (m3d2d_*) against the reference's own FFT_Analysis2D
(golden fixtures made from it, tests/golden/make_golden.py) and the numpy
restatement.  Tolerances: fields rel-L2 < 1e-10 after the 25 iterations;
homogenized tensors: diagonal entries < 1e-8 relative, every entry
< 1e-6 of the largest (the off-diagonal means are sums of large cancelling
terms, and C = epHomo^-1 sigHomo carries their rounding into every entry;
the numpy restatement differs from the reference by as much)."""
import os

import numpy as np
import pytest

import mat3d_b200 as m3d
from oracle import mat3d_oracle as O

pytestmark = pytest.mark.gpu

G = os.path.join(os.path.dirname(__file__), "golden")
PROPS = np.array([68.9e9, 0.35, 400e9, 0.23])


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def disc(N, r, off=0.0):
    X, Y = np.meshgrid(np.arange(N), np.arange(N), indexing="ij")
    g = np.ones((N, N), np.int32)
    g[(X - N / 2 - off) ** 2 + (Y - N / 2.5) ** 2 <= r * r] = 0
    return g.ravel()


@pytest.mark.parametrize("name", ["mech2d_16", "mech2d_15"])
def test_2d_vs_reference_fixture(name):
    f = np.load(os.path.join(G, name + ".npz"))
    Nx, Ny = (int(v) for v in f["shape"])
    s = m3d.Solver2D(Nx, Ny)
    s.material(f["props"], f["rve"])
    s.set_load(f["E"])
    s.run(25)
    eps, sig = s.fields()
    assert rel(eps, f["eps"]) < 1e-10
    assert rel(sig, f["sig"]) < 1e-10
    C, ep, sg = s.homogenize(25)
    Cr = f["C"]
    assert np.abs(np.diag(C) - np.diag(Cr)).max() / np.abs(np.diag(Cr)).max() < 1e-8
    assert np.abs(C - Cr).max() / np.abs(Cr).max() < 1e-6
    assert np.abs(ep - f["epHomo"]).max() < 1e-15
    s.close()


@pytest.mark.parametrize("N", [20, 48, 64, 96])
def test_2d_vs_oracle(N):
    rve = disc(N, 0.2 * N, 0.5)
    E = np.array([0.002, -0.001, 0.004 + 0.0005j])
    o = O.Mech2DOracle(N, N)
    o.material(PROPS, rve)
    o.setLoad(E)
    o.runAnalysis(25)
    s = m3d.Solver2D(N, N)
    s.material(PROPS, rve)
    s.set_load(E)
    s.run(25)
    eps, sig = s.fields()
    assert rel(eps, o.eps) < 1e-10 and rel(sig, o.sig) < 1e-10
    s.close()


def test_2d_class_mirror():
    N = 32
    rve = disc(N, 6.0)
    a = m3d.FFT_Analysis2D(N, N)
    a.material(PROPS, rve)
    a.setLoad([0, 0, 0.005])
    a.runAnalysis()
    o = O.Mech2DOracle(N, N)
    o.material(PROPS, rve)
    o.setLoad(np.array([0, 0, 0.005]))
    o.runAnalysis()
    assert rel(a.epsilon, o.eps) < 1e-10
    C = a.homogenization()
    Co, _, _ = o.homogenization()
    assert np.abs(np.diag(C) - np.diag(Co)).max() / np.abs(np.diag(Co)).max() < 1e-8
    assert np.allclose(a.SHomo @ C, np.eye(3), atol=1e-9)


def test_2d_errors():
    with pytest.raises(m3d.M3DError):
        m3d.Solver2D(1, 8)
    s = m3d.Solver2D(8, 8)
    with pytest.raises(m3d.M3DError):
        s.run(25)  # no material / load yet
    s.close()


def test_handles_of_different_sizes_coexist():
    """A smaller handle made after a larger one must not lower the larger
    one's shared-memory launch limit (both above the 48 KB default here)."""
    big = m3d.Solver2D(1024, 1024)
    rve = np.ones(1024 * 1024, np.int32)
    rve[: 1024 * 300] = 0
    big.material([68.9e9, 0.35, 400e9, 0.23], rve)
    big.set_load(np.array([0, 0, 0.005], np.complex128))
    big.run(2)
    e1, _ = big.fields()
    small = m3d.Solver2D(512, 512)
    small.material([68.9e9, 0.35, 400e9, 0.23], np.ones(512 * 512, np.int32))
    small.set_load(np.array([0, 0, 0.005], np.complex128))
    small.run(2)
    big.set_load(np.array([0, 0, 0.005], np.complex128))
    big.run(2)
    e2, _ = big.fields()
    assert np.array_equal(e1, e2)
    small.close()
    big.close()
