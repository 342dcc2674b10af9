"""The reference's own example drivers, compiled unchanged against this
repository's drop-in headers (tests/dropin/Makefile -> tests/_bin/), run on
the GPU with input files in the reference's key/value text format
(example/3d/in_struct.txt, example/3d_thermal/in_therm.txt layout) and a
generated single-column RVE.  Their outputs (.vti field file, homogenization
report) are checked against the CPU oracle."""
import os
import re
import subprocess

import numpy as np
import pytest

from oracle import mat3d_oracle as O

pytestmark = pytest.mark.gpu

BIN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_bin")


def sphere(N, r):
    X, Y, Z = np.meshgrid(np.arange(N), np.arange(N), np.arange(N), indexing="ij")
    g = np.ones((N, N, N), np.int32)
    g[(X - N / 2) ** 2 + (Y - N / 2) ** 2 + (Z - N / 2) ** 2 <= r * r] = 0
    return g.ravel()


def need(binary):
    p = os.path.join(BIN, binary)
    if not os.path.exists(p):
        pytest.skip(f"{p} not built (tests/dropin/Makefile needs the reference sources)")
    return p


def write_mech_input(d, N, mode, E_str, E0, v0, E1, v1, tol):
    np.savetxt(os.path.join(d, "rve.txt"), sphere(N, N / 4), fmt="%d")
    txt = (f"Nx=Ny=Nz=\n{N}\n\nRVE_Name\nrve.txt\n\nE_0=\n{E0}\n\nv_0=\n{v0}\n\nE_1=\n{E1}\n\nv_1=\n{v1}\n\n"
           f"vtiOutput_YorN=\nY\n\nvtiOutputFileName\nfields.vti\n\nErorr_strss=\n{tol}\n\nErorr_equlibrium=\n{tol}\n\n"
           f"SingleAnalysisOrHomogenization=\n{mode}\n\nHomogenizationOutPutFileName=\nreport\n\nE=\n{E_str}\n")
    with open(os.path.join(d, "in_struct.txt"), "w") as f:
        f.write(txt)


def read_vti(path, ncomp):
    vals = []
    with open(path) as f:
        inside = False
        for line in f:
            if "<DataArray" in line:
                inside = True
                continue
            if "</DataArray>" in line:
                break
            if inside:
                vals.append([float(x) for x in line.split()])
    a = np.array(vals)
    assert a.shape[1] == ncomp
    return a.T


def test_mechanical_example_driver_single_analysis(tmp_path):
    exe = need("mat3d_example")
    N = 32
    write_mech_input(tmp_path, N, "S", ".001,0.1,0,0,0,0", "31e9", ".3", "30e9", ".2", "1e-9")
    r = subprocess.run([exe, "in_struct.txt"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    f = read_vti(os.path.join(tmp_path, "fields.vti"), 14)
    # the same analysis in the oracle (mat table of example/3d/main.cpp:110-111)
    mat = np.array([[31e9, .3, 40e6, 100e6, 1, 8e-2, 8e2], [30e9, .2, 250e6, 8006, .2, 8e-4, 8e3]])
    o = O.MechOracle(N, N, N, "e")
    o.material(mat, sphere(N, N / 4))
    o.set_load(np.array([.001, 0.1, 0, 0, 0, 0]), np.array([0, 1.0, 0, 0, 0, 0]))
    o.run(1e-9, 1e-9)
    eps = o.eps.reshape(6, -1)
    assert np.linalg.norm(f[:6] - eps) / np.linalg.norm(eps) < 1e-7


def test_mechanical_example_driver_homogenization(tmp_path):
    exe = need("mat3d_example")
    N = 32
    write_mech_input(tmp_path, N, "H", ".001,0.1,0,0,0,0", "70e9", ".2", "3e9", ".35", "1e-9")
    r = subprocess.run([exe, "in_struct.txt"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    rep = open(os.path.join(tmp_path, "report.txt")).read()
    block = rep.split("C_Homogenized=")[1].split("----")[0]
    C = np.array([[float(x) for x in ln.split()] for ln in block.strip().splitlines()[:6]])
    mat = np.array([[70e9, .2, 40e6, 100e6, 1, 8e-2, 8e2], [3e9, .35, 250e6, 8006, .2, 8e-4, 8e3]])
    o = O.MechOracle(N, N, N, "e")
    o.material(mat, sphere(N, N / 4))
    CH, _ = o.homogenization(1e-9, 1e-9)
    assert np.abs(C - CH).max() / np.abs(CH).max() < 1e-5  # report printed with 6 significant digits
    assert "Hashin-Shtrikman Bounds" in rep


def test_thermal_example_driver_homogenization(tmp_path):
    exe = need("therm3d_example")
    N = 32
    np.savetxt(os.path.join(tmp_path, "rve.txt"), sphere(N, N / 4), fmt="%d")
    txt = ("Nx=Ny=Nz=\n32\n\nRVE_Name\nrve.txt\n\nk_1=\n25\n\nk_0=\n30\n\nvtiOutput_YorN=\nN\n\n"
           "vtiOutputFileName\nt.vti\n\nErorr_heatFlux=\n1e-9\n\nErorr_equlibrium=\n1e-9\n\n"
           "SingleAnalysisOrHomogenization=\nH\n\nHomogenizationOutPutFileName=\nreport\n\nTG=\n.000,0.1,0\n")
    with open(os.path.join(tmp_path, "in_therm.txt"), "w") as f:
        f.write(txt)
    r = subprocess.run([exe, "in_therm.txt"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    rep = open(os.path.join(tmp_path, "report.txt")).read()
    block = rep.split("KHomogenized=")[1].split("RHomogenized")[0]
    K = np.array([[float(x) for x in ln.split()] for ln in block.strip().splitlines()[:3]])
    o = O.ThermOracle(N, N, N)
    o.material(25.0, 30.0, sphere(N, N / 4))
    KH, _ = o.homogenization(1e-9, 1e-9)
    assert np.abs(K - KH).max() / np.abs(KH).max() < 1e-5
    assert re.search(r"Mori-Tanaka", rep)


def test_reconstruction_example_driver(tmp_path):
    """example/reconst3d/main.cpp unchanged: the 171^3 isotropic TPCF, its
    shift and transform through the header's FFTW subset (GPU), recPlan +
    runRec(100, 0.8), saveRecImages("ar1") and vtiWriter("ar1/rec.vti", tpcf)."""
    exe = need("reconst3d_example")
    r = subprocess.run([exe], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    N = 171
    d = os.path.join(tmp_path, "ar1")
    assert all(os.path.exists(os.path.join(d, f"{i + 1}.png")) for i in range(N))
    lines = open(os.path.join(d, "err.txt")).read().splitlines()
    assert lines[0].startswith("voloum fraction= ")
    vf = float(lines[0].split("=")[1])
    assert abs(vf - 0.5) < 0.01  # the walk's target normC[0] / xyz = phi1 = 0.5 of the example's TPCF
    errs = np.array([float(x) for x in lines[1:]])
    assert errs.size == 99 and np.all(errs > 0) and errs[-1] < errs[0]
    with open(os.path.join(d, "rve_rec.txt"), "rb") as f:
        body = f.read()
    vals = np.array(body.split(), float)
    assert vals.size == N ** 3 and set(np.unique(vals)) <= {0.0, 1.0}
    assert abs(vals.mean() - vf) < 1e-5
    # the vti: 2 components (field, the centred TPCF), flat order
    with open(os.path.join(d, "rec.vti")) as f:
        head = []
        for ln in f:
            head.append(ln)
            if "<DataArray" in ln:
                break
        first = [next(f) for _ in range(3)]
    assert 'NumberOfComponents="2"' in "".join(head) and 'WholeExtent="0 170 0 170 0 170"' in "".join(head)
    t = O.tpcf_isotropic(N, 25.0, 0.4, 0.5)
    for k, ln in enumerate(first):
        a, b = (float(x) for x in ln.split())
        assert a == vals[k] and abs(b - t[k]) < 1e-9
