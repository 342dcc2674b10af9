"""The reconstruction restatement (oracle RecOracle, recon::recPlan / runRec
of src/rec/reconstruction.cpp) against the reference's own outputs, plus the
host-side index shifts of the C ABI.  CPU only.

The phase-retrieval loop amplifies a rounding difference by about three per
pass, so agreement over hundreds of passes needs identical arithmetic: those
tests run the restatement on the reference's own transform (exported by the
reference library) with the C library's atan2, and then every recorded error
and the final 0/1 field must match bit for bit.  With numpy's FFT the first
passes agree to rounding."""
import numpy as np
import pytest

from oracle import mat3d_oracle as O
from oracle import ref_lib

GOLDEN = ["rec_9x9x9", "rec_7x9x11"]
have_ref = pytest.mark.skipif(not ref_lib.available(), reason="oracle/_ref/libmat3d_ref.so not built")


def load(name):
    import os
    return np.load(os.path.join(os.path.dirname(__file__), "golden", f"{name}.npz"))


def test_generator_formula():
    """The counter-based draws: first values for seed 1, draw 0 (SplitMix64
    finaliser of the seed-and-draw base plus the voxel index)."""
    def mix(z):
        M = (1 << 64) - 1
        z = (z + 0x9E3779B97F4A7C15) & M
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        return z ^ (z >> 31)
    base = mix((1 * 0x100000001B3 + 0) & ((1 << 64) - 1))
    want = [2.0 * ((mix((base + i) & ((1 << 64) - 1)) >> 11) * 2.0 ** -53) - 1.0 for i in range(5)]
    assert np.array_equal(O.rand_pm1(1, 0, 5), np.array(want))
    u = O.rand_pm1(7, 3, 100000)
    assert u.min() >= -1 and u.max() < 1 and abs(u.mean()) < 0.01


@pytest.mark.parametrize("name", GOLDEN)
def test_golden_first_passes_numpy(name):
    """numpy's transform: the error of the first passes agrees to rounding."""
    g = load(name)
    shape = tuple(int(v) for v in g["shape"])
    o = O.RecOracle(g["tpcf"], *shape)
    st = o.start(int(g["seed"]))
    e = [o.step(st, float(g["beta"])) for _ in range(8)]
    assert np.abs(np.array(e) - g["err"][:8]).max() / g["err"][0] < 1e-11


@have_ref
@pytest.mark.parametrize("name", GOLDEN)
def test_golden_bit_exact_on_reference_transform(name):
    g = load(name)
    shape = tuple(int(v) for v in g["shape"])
    R = ref_lib.RefLib()
    o = O.RecOracle(g["tpcf"], *shape, fft=lambda a, sg: R.fft3(a, shape, sg), libm_atan2=True)
    rve = o.runRec(int(g["n"]), float(g["beta"]), int(g["seed"]))
    assert np.array_equal(o.err, g["err"])
    assert o.iterations == int(g["iterations"])
    assert np.array_equal(rve, g["rve"])


@have_ref
@pytest.mark.parametrize("shape,seed,n", [((6, 6, 6), 3, 400), ((5, 7, 9), 4, 200), ((12, 12, 12), 5, 160)])
def test_live_reference_bit_exact(shape, seed, n):
    """Other grids (odd lengths included) and seeds, live against the reference."""
    Nx, Ny, Nz = shape
    R = ref_lib.RefLib()
    m = max(shape)
    t = O.tpcf_isotropic(m, 3.0, 0.7, 0.45).reshape(m, m, m)[:Nx, :Ny, :Nz].ravel()
    T = np.real(np.fft.fftn(O.ifftshift3(t, *shape).reshape(shape))).ravel()
    r = R.rec_run(shape, T, n, 0.75, seed)
    o = O.RecOracle(T, *shape, fft=lambda a, sg: R.fft3(a, shape, sg), libm_atan2=True)
    o.runRec(n, 0.75, seed)
    assert np.array_equal(o.err, r["err"])
    assert np.array_equal(o.rve, r["rve"])


@have_ref
@pytest.mark.parametrize("shape", [(6, 8, 10), (5, 6, 7), (7, 7, 7), (4, 9, 6)])
def test_ifftshift_vs_reference(shape):
    R = ref_lib.RefLib()
    a = np.random.default_rng(0).random(int(np.prod(shape)))
    assert np.array_equal(O.ifftshift3(a, *shape), R.ifftshift(a, shape))


@pytest.mark.parametrize("shape", [(6, 8, 10), (5, 6, 7), (7, 7, 7), (1, 3, 4)])
def test_abi_shifts(shape):
    """m3drec_fftshift / m3drec_ifftshift (host code of the library): the
    inverse pair, and ifftshift equal to the restatement of recon::ifftshift."""
    m3d = pytest.importorskip("mat3d_b200")
    try:
        m3d.load_library()
    except ImportError as e:
        pytest.skip(str(e))
    a = np.random.default_rng(1).random(int(np.prod(shape)))
    f = m3d.fftshift(a, *shape)
    assert np.array_equal(m3d.ifftshift(f, *shape), a)
    assert np.array_equal(m3d.ifftshift(a, *shape), O.ifftshift3(a, *shape))
    assert np.array_equal(f, np.fft.fftshift(a.reshape(shape)).ravel())


def test_threshold_walk():
    """The closing walk on a planted field: cut moves in 0.001 steps until the
    fraction of ones is within 1e-4 of normC[0] / xyz."""
    shape = (10, 10, 10)
    xyz = 1000
    T = np.zeros(xyz)
    T[0] = 0.3 ** 2 * xyz  # normC[0] = sqrt(T[0] * xyz) = 0.3 xyz
    o = O.RecOracle(T, *shape)
    field = (np.arange(xyz) + 0.5) / xyz  # uniform in (0, 1): 30 % ones needs a cut near 0.7
    b = o.threshold(field)
    assert abs(b.mean() - 0.3) < 1e-4 or abs(b.mean() - 0.3) <= 0.0015


SECTIONS = ["rec_sections_12x12", "rec_sections_11x9"]


@pytest.mark.parametrize("name", SECTIONS)
def test_sections_golden_numpy(name):
    """recPlan(CImg, CImg) + estimateNormFFT_RVE restated with numpy's FFT:
    normC within 1e-7 of its maximum (sqrt(sqrt(|M|)) magnifies the rounding of
    the near-zero coefficients)."""
    g = load(name)
    o = O.RecOracle.from_sections(g["c1"], g["c2"])
    assert np.abs(o.normC - g["normC"]).max() / g["normC"].max() < 1e-7


@have_ref
@pytest.mark.parametrize("name", SECTIONS)
def test_sections_bit_exact_on_reference_transform(name):
    g = load(name)
    R = ref_lib.RefLib()
    h, w = g["c1"].shape
    o = O.RecOracle.from_sections(g["c1"], g["c2"], fft=lambda a, sg: R.fft3(a, (w, h, h), sg),
                                  fft2=lambda a, sh, sg: R.fft3(a, (sh[0], sh[1], 1), sg))
    assert np.array_equal(o.normC, g["normC"])
    assert np.array_equal(R.rec_sections(g["c1"], g["c2"]), g["normC"])


@have_ref
@pytest.mark.parametrize("beta,n", [(0.5, 230), (0.95, 230), (0.0, 60)])
def test_live_reference_other_betas(beta, n):
    """The hybrid input-output step for other feedback constants (beta = 0
    reduces it to an error-reduction step) stays bit-exact with the reference."""
    shape = (7, 8, 9)
    R = ref_lib.RefLib()
    m = max(shape)
    t = O.tpcf_isotropic(m, 2.5, 0.9, 0.35).reshape(m, m, m)[:7, :8, :9].ravel()
    T = np.real(np.fft.fftn(O.ifftshift3(t, *shape).reshape(shape))).ravel()
    r = R.rec_run(shape, T, n, beta, 11)
    o = O.RecOracle(T, *shape, fft=lambda a, sg: R.fft3(a, shape, sg), libm_atan2=True)
    o.runRec(n, beta, 11)
    assert np.array_equal(o.err, r["err"])
    assert np.array_equal(o.rve, r["rve"])
