"""The numpy oracle reproduces the golden fixtures made from the reference's own
solver sources (tests/golden/make_golden.py).  CPU only."""
import glob
import os

import numpy as np
import pytest

from oracle import mat3d_oracle as O

G = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    return np.load(os.path.join(G, name + ".npz"))


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(G, "fft_*.npz"))))
def test_fft_layout(path):
    f = np.load(path)
    x = f["x"]  # [Nx, Ny, Nz, c] AoS, as the reference's interleaved buffers
    spec = np.fft.rfftn(np.moveaxis(x, -1, 0), axes=(1, 2, 3))
    assert np.abs(np.moveaxis(spec, 0, -1) - f["spec"]).max() / np.abs(f["spec"]).max() < 1e-13
    back = np.fft.irfftn(np.moveaxis(f["spec"], -1, 0), s=x.shape[:3], axes=(1, 2, 3)) * np.prod(x.shape[:3])
    assert np.abs(np.moveaxis(back, 0, -1) - f["back"]).max() / np.abs(f["back"]).max() < 1e-13


@pytest.mark.parametrize("name", ["elastic_auto_12", "elastic_strain_10x12x14"])
def test_elastic(name):
    f = load(name)
    shape = tuple(int(v) for v in f["shape"])
    o = O.MechOracle(*shape, "e")
    o.material(f["mat"], f["rve"], force_scheme=int(f["force"]))
    assert (1 if o.strain_based else 2) == int(f["scheme"])
    o.set_load(f["E"])
    it = o.run(float(f["tol"]), float(f["tol"]))
    assert it == int(f["sweeps"])
    assert rel(o.eps.reshape(6, -1), f["eps"]) < 1e-11
    assert rel(o.sig.reshape(6, -1), f["sig"]) < 1e-11
    assert o.la0 == pytest.approx(float(f["la0"]), rel=1e-15)


def test_elastic_homogenization():
    f = load("homog_elastic_10")
    shape = tuple(int(v) for v in f["shape"])
    o = O.MechOracle(*shape, "e")
    o.material(f["mat"], f["rve"])
    C, S = o.homogenization(float(f["tol"]), float(f["tol"]))
    assert o.sweeps == int(f["sweeps"])
    assert np.abs(C - f["C"]).max() / np.abs(f["C"]).max() < 1e-12
    assert np.abs(o.epHomo - f["epHomo"]).max() / np.abs(f["epHomo"]).max() < 1e-12


@pytest.mark.parametrize("name,behav", [("j2_10", "ep"), ("damage_10", "ed")])
def test_inelastic(name, behav):
    f = load(name)
    shape = tuple(int(v) for v in f["shape"])
    o = O.MechOracle(*shape, behav)
    o.material(f["mat"], f["rve"])
    o.set_load(f["E"], f["X0"])
    total = o.run(float(f["tol"]), float(f["tol"]), int(f["ninc_req"]))
    assert total == int(f["sweeps"])
    assert o.ninc_done == int(f["ninc"])
    assert rel(o.eps.reshape(6, -1), f["eps"]) < 1e-10
    assert rel(o.sig.reshape(6, -1), f["sig"]) < 1e-10
    assert np.abs(o.prop - f["prop"]).max() / np.abs(f["prop"]).max() < 1e-10
    extra = o.ep_eff.ravel() if behav == "ep" else o.d.ravel()
    assert np.abs(extra - f["extra"]).max() <= 1e-10 * max(1.0, np.abs(f["extra"]).max())


@pytest.mark.parametrize("name", ["thermal_grad_12", "thermal_flux_12"])
def test_thermal(name):
    f = load(name)
    shape = tuple(int(v) for v in f["shape"])
    o = O.ThermOracle(*shape)
    o.material(float(f["km"]), float(f["ki"]), f["rve"])
    assert (1 if o.grad_based else 2) == int(f["scheme"])
    o.set_load(f["E"])
    it = o.run(float(f["tol"]), float(f["tol"]))
    assert it == int(f["sweeps"])
    assert rel(o.grad.reshape(3, -1), f["grad"]) < 1e-11
    assert rel(o.flux.reshape(3, -1), f["flux"]) < 1e-11
    o2 = O.ThermOracle(*shape)
    o2.material(float(f["km"]), float(f["ki"]), f["rve"])
    K, R = o2.homogenization(float(f["tol"]), float(f["tol"]))
    assert np.abs(K - f["K"]).max() / np.abs(f["K"]).max() < 1e-12


@pytest.mark.parametrize("name", ["mech2d_16", "mech2d_15"])
def test_mech2d(name):
    """The 2-D solver (src/2d/FFT_analysis2D.cpp): 25 basic-scheme iterations
    from setLoad(E), complex fields, and homogenization() continuing from that
    field."""
    f = load(name)
    Nx, Ny = (int(v) for v in f["shape"])
    o = O.Mech2DOracle(Nx, Ny)
    o.material(f["props"], f["rve"])
    o.setLoad(f["E"])
    o.runAnalysis()
    assert rel(o.eps, f["eps"]) < 1e-12
    assert rel(o.sig, f["sig"]) < 1e-12
    C, ep, sg = o.homogenization()
    # the near-zero off-diagonal means are sums of large cancelling terms: they
    # (and C = epHomo^-1 sigHomo) agree to 1e-6 of the largest entry only
    # (sequential sums in the reference, pairwise in numpy)
    assert np.abs(ep - f["epHomo"]).max() < 1e-15
    assert np.abs(sg - f["sigHomo"]).max() / np.abs(f["sigHomo"]).max() < 1e-6
    assert np.abs(C - f["C"]).max() / np.abs(f["C"]).max() < 1e-6
