"""Golden fixtures at the benchmarked configurations, from the reference's own solver.

Runs oracle/_ref/libmat3d_ref.so (the reference sources src/3d/FFT_analysis3D.cpp
and src/3dTherm/FFT_thermal3D.cpp compiled unmodified by oracle/Makefile) on:

  config_thermal128.npz  the bench's default workload: 128^3 steady conduction,
                         ~100 prolate ellipsoids (3a, a, a) of random orientation
                         at 30%, k_matrix 1 : k_inclusion 100 (mat3d_b200.rve.ellipsoids,
                         seed 0), gradient along z; runAnalysis with the
                         reference stop rule at 1e-8 and homogenization at 1e-8
  config_elastic64.npz   64^3 elastic, non-overlapping spheres r = 6 at 20%
                         (random sequential addition, seed 0), matrix 3 GPa / 0.35,
                         inclusions 70 GPa / 0.2, E = (1e-3, 0, ...); runAnalysis at
                         1e-6 and homogenization at 1e-9
  example_rve65.npz      the reference's shipped example input
                         (example/3d/in_struct.txt with example/3d/rve65.txt, a 65^3
                         RVE: odd grid, the generic line-FFT path): the elastic
                         single analysis the example driver runs, and the thermal
                         homogenization of example/3d_thermal/in_therm.txt

Full fields do not fit in a fixture: each run stores the sweep count, the
scheme, per-component sums and sums of squares of every output field, the
field values at every 97th voxel (509th at 128^3; a fixed strided sample) and, for
homogenizations, the effective tensors.  The RVEs are stored bit-packed, so the
GPU tests need neither the generators' exact reproduction nor the reference
tree.  Slow (about 20 minutes on 8 host cores); run it where the reference
sources and oracle/_ref exist:

    make -C oracle REF=<reference sources> && python tests/golden/make_config_golden.py [names...]
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle.ref_lib import RefLib  # noqa: E402

STRIDE = 97
STRIDE128 = 509  # 128^3: about 4100 sampled voxels
MAT_ELASTIC64 = np.array([[70e9, 0.2, 1e30, 0, 1, 0, 1e30], [3e9, 0.35, 1e30, 0, 1, 0, 1e30]])
# example/3d/main.cpp:110-111 with in_struct.txt's E_0, v_0, E_1, v_1
MAT_EXAMPLE = np.array([[31e9, .3, 40e6, 100e6, 1, 8e-2, 8e2], [30e9, .2, 250e6, 8006, .2, 8e-4, 8e3]])


def field_summary(prefix, f, stride=STRIDE):
    """f: (c, V) -> sums, sums of squares and the strided sample."""
    f = np.asarray(f)
    return {f"{prefix}_sum": f.sum(axis=1), f"{prefix}_sumsq": (f * f).sum(axis=1),
            f"{prefix}_sample": f[:, ::stride].copy()}


def packed(rve):
    r = np.asarray(rve).ravel()
    assert set(np.unique(r)) <= {0, 1}
    return np.packbits(r.astype(np.uint8))


def thermal128(ref):
    from mat3d_b200 import rve as R
    g, meta = R.ellipsoids(128, vf=0.30, aspect=3.0, n_target=100, seed=0)
    rve = g.ravel().astype(np.int32)
    shape, km, ki, E, tol = (128, 128, 128), 1.0, 100.0, np.array([0.0, 0.0, 1.0]), 1e-8
    t = time.time()
    r = ref.therm_run(shape, km, ki, rve, E, tol, tol)
    print(f"thermal128 run: {r['sweeps']} sweeps, scheme {r['scheme']}, {time.time() - t:.0f} s", flush=True)
    t = time.time()
    h = ref.therm_homog(shape, km, ki, rve, tol, tol)
    print(f"thermal128 homogenization: {h['sweeps']} sweeps, {time.time() - t:.0f} s", flush=True)
    np.savez_compressed(os.path.join(HERE, "config_thermal128.npz"), shape=shape, rve_bits=packed(rve), km=km, ki=ki,
                        E=E, tol=tol, stride=STRIDE128, sweeps=r["sweeps"], scheme=r["scheme"],
                        **field_summary("grad", r["grad"], STRIDE128), **field_summary("flux", r["flux"], STRIDE128),
                        K=h["K"], R=h["R"], homog_sweeps=h["sweeps"], n_inclusions=meta["n_inclusions"],
                        vf=meta["vf"])


def elastic64(ref):
    from mat3d_b200 import rve as R
    g, meta = R.spheres_rsa(64, radius=6.0, vf=0.20, seed=0)
    rve = g.ravel().astype(np.int32)
    shape, E, X0, tol = (64, 64, 64), np.array([1e-3, 0, 0, 0, 0, 0.0]), np.zeros(6), 1e-6
    t = time.time()
    r = ref.mech_run(shape, "e", MAT_ELASTIC64, rve, E, X0, tol, tol, 1, 0)
    print(f"elastic64 run: {r['sweeps']} sweeps, scheme {r['scheme']}, {time.time() - t:.0f} s", flush=True)
    htol = 1e-9
    t = time.time()
    h = ref.mech_homog(shape, MAT_ELASTIC64, rve, htol, htol)
    print(f"elastic64 homogenization: {h['sweeps']} sweeps, {time.time() - t:.0f} s", flush=True)
    np.savez_compressed(os.path.join(HERE, "config_elastic64.npz"), shape=shape, rve_bits=packed(rve),
                        mat=MAT_ELASTIC64, E=E, X0=X0, tol=tol, stride=STRIDE, sweeps=r["sweeps"],
                        scheme=r["scheme"], **field_summary("eps", r["eps"]), **field_summary("sig", r["sig"]),
                        htol=htol, C=h["C"], S=h["S"], homog_sweeps=h["sweeps"], n_inclusions=meta["n_inclusions"],
                        vf=meta["vf"])


def example_rve65(ref, reference_tree):
    rve = np.loadtxt(os.path.join(reference_tree, "example", "3d", "rve65.txt")).astype(np.int32)
    shape = (65, 65, 65)
    assert rve.size == 65 ** 3
    # example/3d/in_struct.txt: single analysis, E = (0, 0.1, 0, 0, 0, 0), X0 = e_2
    # (example/3d/main.cpp:114), tolerances 1e-6 / 1e-6, nInc 15 (ignored by "e")
    E, X0, tol = np.array([0, 0.1, 0, 0, 0, 0.0]), np.array([0, 1.0, 0, 0, 0, 0]), 1e-6
    t = time.time()
    r = ref.mech_run(shape, "e", MAT_EXAMPLE, rve, E, X0, tol, tol, 15, 0)
    print(f"rve65 elastic run: {r['sweeps']} sweeps, scheme {r['scheme']}, {time.time() - t:.0f} s", flush=True)
    # example/3d_thermal/in_therm.txt: k_1 = 25 (matrix), k_0 = 30 (inclusion),
    # homogenization at 1e-6 / 1e-6
    km, ki = 25.0, 30.0
    t = time.time()
    h = ref.therm_homog(shape, km, ki, rve, tol, tol)
    print(f"rve65 thermal homogenization: {h['sweeps']} sweeps, {time.time() - t:.0f} s", flush=True)
    np.savez_compressed(os.path.join(HERE, "example_rve65.npz"), shape=shape, rve_bits=packed(rve), mat=MAT_EXAMPLE,
                        E=E, X0=X0, tol=tol, stride=STRIDE, sweeps=r["sweeps"], scheme=r["scheme"],
                        **field_summary("eps", r["eps"]), **field_summary("sig", r["sig"]),
                        km=km, ki=ki, K=h["K"], R=h["R"], homog_sweeps=h["sweeps"])


def main(argv):
    ref = RefLib(fft_threads=os.cpu_count() or 3)
    names = argv or ["example_rve65", "elastic64", "thermal128"]
    tree = os.environ.get("MAT3D_REF", "/root/reference")
    for n in names:
        if n == "thermal128":
            thermal128(ref)
        elif n == "elastic64":
            elastic64(ref)
        elif n == "example_rve65":
            example_rve65(ref, tree)
        else:
            raise SystemExit(f"unknown fixture {n}")
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main(sys.argv[1:])
