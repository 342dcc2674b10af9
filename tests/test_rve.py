"""Seeded microstructure generators and the RVE text format.  CPU only."""
import numpy as np

from mat3d_b200 import rve


def test_spheres_rsa_deterministic_and_vf():
    g1, m1 = rve.spheres_rsa(32, radius=3.0, vf=0.2, seed=5)
    g2, m2 = rve.spheres_rsa(32, radius=3.0, vf=0.2, seed=5)
    assert np.array_equal(g1, g2)
    assert 0.2 <= m1["vf"] < 0.25
    assert set(np.unique(g1)) <= {0, 1}


def test_ellipsoids_and_lognormal():
    g, m = rve.ellipsoids(32, vf=0.3, n_target=20, seed=1)
    assert 0.3 <= m["vf"] < 0.36
    g, m = rve.lognormal_spheres(40, vf=0.15, seed=2)
    assert 0.15 <= m["vf"] < 0.2


def test_txt_roundtrip(tmp_path):
    g, _ = rve.spheres_rsa(8, radius=2.0, vf=0.1, seed=0)
    p = tmp_path / "r.txt"
    rve.write_rve_txt(p, g)
    back = rve.read_rve_txt(p, 512)
    assert np.array_equal(back, g.ravel())


def test_batch_descriptors():
    d = rve.batch_rves(16)
    assert len(d) == 16 and all(n in (32, 48, 64, 96) for _, n, _, _ in d)
    assert d == rve.batch_rves(16)
