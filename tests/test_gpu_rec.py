"""Microstructure reconstruction on the GPU (m3drec_*) against the
restatement of recon::recPlan / runRec (src/rec/reconstruction.cpp) and the
reference's fixtures.

The random draws and the threshold walk are exact (integer work and exact
double steps), so the initial field and a thresholded field must be equal bit
for bit.  The transforms round differently from numpy's, and the iteration
amplifies a rounding difference about threefold per pass, so the loop is
checked pass by pass from the same state (every branch: hybrid input-output,
box projection, the restart at i + 1 = 150, the reset of j after 200,
convergence) to 1e-9, short runs to 1e-8, and long runs through what they must
achieve (error track of the reference's size, volume fraction on target).

Grids with an even length are avoided where transforms are compared: the
transform of a real field (the initial field, the restart draws) has real
coefficients at the Nyquist frequencies, and where such a coefficient is
negative its phase is +pi or -pi by the sign of a rounding-level imaginary
part -- a choice that differs between FFT implementations (numpy's, the GPU's)
and changes the next field by O(1).  With odd lengths only the zero frequency
is self-conjugate, and its imaginary part is an exact +0 everywhere."""
import numpy as np
import pytest

import mat3d_b200 as m3d
from oracle import mat3d_oracle as O

pytestmark = pytest.mark.gpu


def load(name):
    import os
    return np.load(os.path.join(os.path.dirname(__file__), "golden", f"{name}.npz"))


def example_tpcf(shape, A=3.0, Q=0.8, phi1=0.4):
    """The example's TPCF (example/reconst3d/main.cpp): centred S2, shifted to
    index 0, real part of its transform."""
    m = max(shape)
    t = O.tpcf_isotropic(m, A, Q, phi1).reshape(m, m, m)[:shape[0], :shape[1], :shape[2]].ravel()
    return np.real(np.fft.fftn(O.ifftshift3(t, *shape).reshape(shape))).ravel()


def state_close(gpu, st, tol=1e-9):
    f = gpu["field"]
    assert gpu["i"] == st["i"] and gpu["j"] == st["j"] and gpu["call"] == st["call"]
    d = np.abs(f - st["mT"]).max()
    assert d < tol, d


@pytest.mark.parametrize("shape", [(8, 8, 8), (6, 8, 10), (16, 12, 9), (9, 9, 9), (7, 9, 11)])
def test_initial_field_and_threshold_exact(shape):
    """n = 0: the initial draws (m = (U + 1) / 2) thresholded; both steps exact."""
    T = example_tpcf(shape)
    r = m3d.Reconstruction(T, *shape)
    r.seed(11)
    r.run(0, 0.8)
    o = O.RecOracle(T, *shape)
    st = o.start(11)
    want = o.threshold(st["mT"].real)
    assert np.array_equal(r.field(), want)
    assert r.errors().size == 0
    r.close()


@pytest.mark.parametrize("name", ["rec_9x9x9", "rec_7x9x11"])
def test_first_passes_vs_reference_fixture(name):
    """The reference's recorded errors for the first passes (fixture made by
    the reference itself) agree to 1e-9."""
    g = load(name)
    shape = tuple(int(v) for v in g["shape"])
    r = m3d.Reconstruction(g["tpcf"], *shape)
    r.seed(int(g["seed"]))
    r.run(10, float(g["beta"]))
    e = r.errors()
    assert e.size == 10
    assert np.abs(e - g["err"][:10]).max() / g["err"][0] < 1e-9
    r.close()


@pytest.mark.parametrize("shape,k", [((15, 15, 15), 12), ((11, 13, 9), 12), ((27, 21, 25), 8)])
def test_short_run_state_vs_oracle(shape, k):
    T = example_tpcf(shape)
    r = m3d.Reconstruction(T, *shape)
    r.seed(5)
    r.run(k, 0.8)  # k passes then the threshold
    o = O.RecOracle(T, *shape)
    o.runRec(k, 0.8, 5)
    assert np.abs(r.errors() - o.err).max() / o.err[0] < 1e-8
    # the same passes without the threshold: the complex field itself
    r.seed(5)
    r.run(0, 0.8)
    o2 = O.RecOracle(T, *shape)
    st = o2.start(5)
    r.set_state(st["mT"], 0, 0, 1)
    r.iterate(k, 0.8)
    for _ in range(k):
        o2.step(st, 0.8)
    state_close(r.get_state(), st, 1e-8)
    r.close()


@pytest.mark.parametrize("i,j", [(148, 149), (298, 99), (98, 99), (199, 200), (149, 0), (40, 150)])
def test_branches_step_by_step(i, j):
    """Two passes from the same state at the loop's branch points: restart
    (i + 1 = 150, 300), the switch to the box projection (j = 100), the reset
    of j after 200, and an ordinary box-projection pass."""
    shape = (11, 13, 15)
    T = example_tpcf(shape)
    o = O.RecOracle(T, *shape)
    st = o.start(3)
    for _ in range(5):
        o.step(st, 0.8)
    st.update(i=i, j=j, call=1 + i // 150)  # draws taken: the initial one and one per earlier restart
    r = m3d.Reconstruction(T, *shape)
    r.seed(3)
    r.set_state(st["mT"], i, j, st["call"])
    r.iterate(2, 0.8)
    e = [o.step(st, 0.8) for _ in range(2)]
    state_close(r.get_state(), st)
    got = r.errors()
    assert got.size == i + 2
    assert np.abs(got[i:] - np.array(e)).max() / e[0] < 1e-9
    r.close()


def test_converged_pass_leaves_field():
    """A field whose transform already has the target modulus: the first pass
    records err < 0.1 and stops without touching the field (:310-314)."""
    shape = (8, 10, 12)
    rng = np.random.default_rng(2)
    m = (rng.random(shape) < 0.4).astype(np.float64)
    M = np.fft.fftn(m)
    T = (np.abs(M) ** 2 / m.size).ravel()  # normC = |M|
    r = m3d.Reconstruction(T, *shape)
    r.seed(1)
    r.set_state(m.ravel().astype(np.complex128), 0, 0, 1)
    r.iterate(50, 0.8)
    s = r.get_state()
    e = r.errors()
    assert e.size == 1 and e[0] < 1e-12
    assert s["i"] == 0 and s["j"] == 1
    assert np.array_equal(s["field"], m.ravel().astype(np.complex128))
    r.close()


@pytest.mark.parametrize("shape", [(20, 20, 20), (21, 21, 21)])  # even and odd voxel counts
def test_threshold_exact_on_planted_field(shape):
    T = example_tpcf(shape)
    rng = np.random.default_rng(4)
    f = rng.random(int(np.prod(shape))) * 1.2 - 0.1 + 1j * rng.random(int(np.prod(shape)))
    r = m3d.Reconstruction(T, *shape)
    r.set_state(f, 0, 0, 1)
    r.threshold()
    o = O.RecOracle(T, *shape)
    got = r.get_state()["field"]
    assert np.array_equal(got.real, o.threshold(f.real))
    assert np.array_equal(got.imag, f.imag)  # the walk writes the real part only (:397)
    r.close()


def test_graph_equals_host_loop():
    """The graph-captured loop and the host-driven loop (per-kernel timing)
    launch the same kernels: identical errors, fields and counters."""
    shape = (16, 16, 16)
    T = example_tpcf(shape)
    out = []
    for prof in (False, True):
        r = m3d.Reconstruction(T, *shape)
        r.seed(9)
        r.set_profiling(prof)
        r.run(160, 0.8)  # crosses the restart at i + 1 = 150
        out.append((r.errors(), r.field(), r.get_state()))
        if prof:
            ms, n = r.profile()
            assert n == out[0][0].size and ms[3] > 0
        r.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert {k: out[0][2][k] for k in ("i", "j", "call")} == {k: out[1][2][k] for k in ("i", "j", "call")}


@pytest.mark.parametrize("name", ["rec_9x9x9", "rec_7x9x11"])
def test_long_run_properties(name):
    """320 passes (every branch) on the reference's fixture input: the run
    completes the same number of passes or converges as the reference did,
    its error track stays at the reference's level, and the volume fraction
    of the 0/1 field meets the walk's target like the reference's does."""
    g = load(name)
    shape = tuple(int(v) for v in g["shape"])
    n = int(g["n"])
    r = m3d.Reconstruction(g["tpcf"], *shape)
    r.seed(int(g["seed"]))
    r.run(n, float(g["beta"]))
    e, f = r.errors(), r.field()
    ref_e = g["err"][: int(g["iterations"])]
    assert set(np.unique(f)) <= {0.0, 1.0}
    assert 0 < e.size <= n
    assert np.median(e[-50:]) < 2 * np.median(ref_e[-50:]) + 0.1
    target = np.sqrt(abs(g["tpcf"][0]) * f.size) / f.size
    assert abs(f.mean() - target) <= max(abs(g["rve"].mean() - target), 1e-4) + 0.01
    r.close()


def test_recplan_mirror():
    shape = (15, 15, 15)
    T = example_tpcf(shape, phi1=0.5)
    a = m3d.recPlan(T, *shape, seed=2)
    a.runRec(30, 0.8)
    assert a.trackrealerrorA.shape == (30,)
    assert a.mTilda.shape == (15 ** 3,)
    assert set(np.unique(a.mTilda)) <= {0.0, 1.0}
    o = O.RecOracle(T, *shape)
    o.runRec(30, 0.8, 2)
    assert np.abs(a.trackrealerrorA[:8] - o.err[:8]).max() / o.err[0] < 1e-9
    a.close()


def test_errors():
    T = example_tpcf((8, 8, 8))
    with pytest.raises(m3d.M3DError):
        m3d.Reconstruction(np.ones(37 * 4 * 4), 37, 4, 4)  # prime factor 37
    r = m3d.Reconstruction(T, 8, 8, 8)
    with pytest.raises(m3d.M3DError):
        r.iterate(3, 0.8)  # no field yet
    with pytest.raises(m3d.M3DError):
        r.run(-1, 0.8)
    with pytest.raises(m3d.M3DError):
        r.set_state(np.zeros(512, np.complex128), 0, 300, 0)
    r.close()


# ---- cut-section constructor, one-shot transform, writers -------------------
@pytest.mark.parametrize("name", ["rec_sections_12x12", "rec_sections_11x9"])
def test_sections_norm_vs_reference_fixture(name):
    """recPlan(CImg, CImg) + estimateNormFFT_RVE: normC against the
    reference's (fixture) within 1e-7 of its maximum, as the numpy
    restatement; then a short run against the restatement."""
    g = load(name)
    r = m3d.Reconstruction(None, sections=(g["c1"], g["c2"]))
    with pytest.raises(m3d.M3DError):
        r.run(3, 0.8)  # no target modulus before the estimate
    r.estimate_norm()
    nc = r.norm()
    assert np.abs(nc - g["normC"]).max() / g["normC"].max() < 1e-7
    h, w = g["c1"].shape
    shape = (w, h, h)
    assert (r.Nx, r.Ny, r.Nz) == shape
    r.seed(4)
    r.run(6, 0.8)
    o = O.RecOracle(np.zeros(r.xyz), *shape)
    o.normC = nc.copy()  # the same target, so the loop itself is compared
    o.runRec(6, 0.8, 4)
    assert np.abs(r.errors() - o.err).max() / o.err[0] < 1e-8
    r.close()


def test_sections_errors():
    a = np.zeros((8, 8), np.uint8)
    a[2:5, 2:5] = 255
    with pytest.raises(m3d.M3DError):
        m3d.Reconstruction(None, sections=(a, np.zeros((8, 8), np.uint8)))  # all-zero section
    with pytest.raises(m3d.M3DError):
        m3d.Reconstruction(None, sections=(a, a[:, :6]))  # sizes differ


@pytest.mark.parametrize("shape", [(9, 10, 11), (171, 1, 1), (16, 16, 16)])
def test_fft3_vs_numpy(shape):
    rng = np.random.default_rng(1)
    a = rng.standard_normal(int(np.prod(shape))) + 1j * rng.standard_normal(int(np.prod(shape)))
    f = m3d.fft3(a, shape, -1)
    want = np.fft.fftn(a.reshape(shape)).ravel()
    assert np.abs(f - want).max() / np.abs(want).max() < 1e-13
    b = m3d.fft3(f, shape, +1)
    assert np.abs(b / a.size - a).max() < 1e-13


def _png_pixels(path):
    import struct
    import zlib
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat = 8, b""
    w = h = None
    while pos < len(data):
        n, = struct.unpack(">I", data[pos:pos + 4])
        typ, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        crc, = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])
        assert crc == zlib.crc32(typ + body) & 0xFFFFFFFF
        if typ == b"IHDR":
            w, h, depth, ctype = struct.unpack(">IIBB", body[:10])
            assert depth == 8 and ctype == 0
        elif typ == b"IDAT":
            idat += body
        pos += 12 + n
    raw = zlib.decompress(idat)
    rows = [raw[y * (w + 1):(y + 1) * (w + 1)] for y in range(h)]
    assert all(r[0] == 0 for r in rows)
    return np.array([list(r[1:]) for r in rows], np.uint8)  # [y, x]


def test_writers(tmp_path):
    """saveRecImages (PNG slices, rve_rec.txt, err.txt) and vtiWriter."""
    shape = (9, 10, 11)
    T = example_tpcf(shape)
    a = m3d.recPlan(T, *shape, seed=3)
    a.runRec(12, 0.8)
    f = a.mTilda
    folder = tmp_path / "ar1"
    a.saveRecImages(str(folder))
    Nx, Ny, Nz = shape
    F = f.reshape(shape)
    for i in range(Nx):
        px = _png_pixels(folder / f"{i + 1}.png")  # [y = k, x = j]
        assert px.shape == (Nz, Ny)
        assert np.array_equal(px.T, (F[i] * 255).astype(np.uint8))
    vals = np.loadtxt(folder / "rve_rec.txt")
    assert np.array_equal(vals, f)
    lines = open(folder / "err.txt").read().splitlines()
    assert lines[0] == f"voloum fraction= {f.mean():.6g}"
    e = np.array([float(x) for x in lines[1:]])
    assert e.size == 11 and np.allclose(e, a.trackrealerrorA[:11], rtol=1e-5)
    a.vtiWriter(str(folder / "rec.vti"), T)
    txt = open(folder / "rec.vti").read()
    assert 'WholeExtent="0 8 0 9 0 10"' in txt and 'NumberOfComponents="2"' in txt
    body = txt.split('format="ascii">')[1].split("</DataArray>")[0]
    arr = np.array(body.split(), float).reshape(-1, 2)
    assert np.array_equal(arr[:, 0], f) and np.allclose(arr[:, 1], T, rtol=1e-9, atol=1e-12)
    a.close()


def test_handles_of_different_sizes_coexist():
    """A small handle made after a large one must not lower the large one's
    shared-memory launch limit (the limit is a property of the kernel)."""
    big_shape = (96, 96, 96)  # 99 KB of dynamic shared memory in the x turnaround
    T = example_tpcf(big_shape)
    big = m3d.Reconstruction(T, *big_shape)
    big.seed(1)
    big.run(2, 0.8)
    e1 = big.errors()
    small = m3d.Reconstruction(example_tpcf((4, 4, 4)), 4, 4, 4)
    small.seed(1)
    small.run(2, 0.8)
    big.run(2, 0.8)
    assert np.array_equal(big.errors(), e1)
    small.close()
    big.close()


@pytest.mark.parametrize("shape", [(256, 200, 64), (96, 243, 35)])
def test_larger_grids_vs_oracle(shape):
    """Long lines and other tile sizes (256-point x lines, radices 5 and 9,
    27-point stages): three passes against the restatement."""
    # S2 centred per axis (a cube cut to a non-cubic grid would leave a
    # modulus the first pass already meets)
    Nx, Ny, Nz = shape
    X, Y, Z = np.meshgrid(np.arange(Nx) - Nx // 2, np.arange(Ny) - Ny // 2, np.arange(Nz) - Nz // 2, indexing="ij")
    rr = np.sqrt(X * X + Y * Y + Z * Z * 1.0)
    with np.errstate(invalid="ignore", divide="ignore"):
        fr = np.exp(-rr / 3.0) * np.sin(0.8 * rr) / (0.8 * rr)
    fr[rr == 0] = 1.0
    t = (fr * 0.4 * 0.6 + 0.16).ravel()
    T = np.real(np.fft.fftn(O.ifftshift3(t, *shape).reshape(shape))).ravel()
    r = m3d.Reconstruction(T, *shape)
    r.seed(2)
    r.run(0, 0.8)
    o = O.RecOracle(T, *shape)
    st = o.start(2)
    r.set_state(st["mT"], 0, 0, 1)
    r.iterate(3, 0.8)
    e = []
    for _ in range(3):  # the loop's own stop rule: a pass with err < 0.1 ends it
        e.append(o.step(st, 0.8))
        if e[-1] < 0.1:
            break
    got = r.errors()
    assert got.size == len(e) == 3, (got, e)
    assert np.abs(got - np.array(e)).max() / e[0] < 1e-10
    state_close(r.get_state(), st, 1e-9)
    r.close()
