"""The allocation-free thermal solve, called through the C ABI.

m3d_thermal_solve_noalloc serves callers that cannot allocate device memory
(code that runs inside another framework's memory pool, or serving paths that
must not block on the allocator or fail with out-of-memory half-way): it
solves on device buffers the caller owns and keeps its own working memory in
a fixed array inside the library.  Its gradient field must equal the handle
API's (m3d_run + m3d_get_field) within the FP64 tolerance of the other parity
tests, on two calls in a row -- the second call starts from whatever the first
left in that shared array.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

import mat3d_b200 as m3d

pytestmark = pytest.mark.gpu


def sphere(N, r):
    X, Y, Z = np.meshgrid(np.arange(N), np.arange(N), np.arange(N), indexing="ij")
    g = np.ones((N, N, N), np.int32)
    g[(X - N / 2) ** 2 + (Y - N / 2) ** 2 + (Z - N / 2) ** 2 <= r * r] = 0
    return g.ravel()


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def sphere_grid(shape, r):
    Nx, Ny, Nz = shape
    X, Y, Z = np.meshgrid(np.arange(Nx), np.arange(Ny), np.arange(Nz), indexing="ij")
    g = np.ones(shape, np.int32)
    g[(X - Nx / 2) ** 2 + (Y - Ny / 2) ** 2 + (Z - Nz / 2) ** 2 <= r * r] = 0
    return g.ravel()


def two_calls_against_handle(shape, km, ki, rve, tol=1e-10):
    """The handle API's gradient field, then two allocation-free calls in a row."""
    import torch

    Nx, Ny, Nz = shape
    V = Nx * Ny * Nz
    E = np.array([0.2, 0.3, 1.0])
    s = m3d.Solver(m3d.KIND_THERMAL, Nx, Ny, Nz, m3d.ELASTIC, "fp64", 1)
    s.set_material_thermal(km, ki, rve)
    s.set_load(E)
    s.run(tol, 0.0, 1, m3d.CRIT_RESIDUAL)
    ref = s.field(m3d.FIELD_STRAIN)
    iters_ref = s.stats()["iters"]
    s.close()

    L = m3d.load_library()
    phase = torch.from_numpy(rve.astype(np.uint8)).cuda()
    stream = torch.cuda.current_stream()
    for call in range(2):
        out = torch.full((3 * V,), float("nan"), dtype=torch.float64, device="cuda")
        it, res = ctypes.c_int(), ctypes.c_double()
        rc = L.m3d_thermal_solve_noalloc(Nx, Ny, Nz, km, ki, ctypes.c_void_p(phase.data_ptr()),
                                         E.ctypes.data_as(ctypes.c_void_p), tol, 0,
                                         ctypes.c_void_p(out.data_ptr()), ctypes.byref(it), ctypes.byref(res),
                                         ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, L.m3d_last_error().decode()
        torch.cuda.synchronize()
        got = out.cpu().numpy().reshape(3, V)
        assert rel(got, ref) < 1e-9, (call, rel(got, ref))
        assert abs(it.value - iters_ref) <= 1
        assert res.value < tol


@pytest.mark.parametrize("km,ki", [(1.0, 100.0), (30.0, 25.0)])  # gradient-based, flux-based
def test_noalloc_matches_handle_api(km, ki):
    two_calls_against_handle((32, 32, 32), km, ki, sphere(32, 9.0))


def test_noalloc_phase_ids_above_one():
    """Matrix voxels marked 2: the scheme follows the raw id sum, as in the handle API."""
    rve = sphere(32, 11.0) * 2  # about half the voxels 2, the rest 0
    two_calls_against_handle((32, 32, 32), 1.0, 100.0, rve)


def test_noalloc_non_cubic_grid():
    two_calls_against_handle((24, 30, 40), 1.0, 100.0, sphere_grid((24, 30, 40), 7.0))


def test_noalloc_near_the_scratch_limit():
    """96^3 needs about 23 MiB of the 32 MiB array."""
    two_calls_against_handle((96, 96, 96), 1.0, 10.0, sphere(96, 24.0), tol=1e-9)


def test_noalloc_rejects_grids_beyond_its_scratch():
    L = m3d.load_library()
    it, res = ctypes.c_int(), ctypes.c_double()
    E = np.array([0.0, 0.0, 1.0])
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    rc = L.m3d_thermal_solve_noalloc(256, 256, 256, 1.0, 10.0, dummy, E.ctypes.data_as(ctypes.c_void_p), 1e-6, 0,
                                     dummy, ctypes.byref(it), ctypes.byref(res), None)
    assert rc == 1  # M3D_ERR_ARG
    assert b"MiB" in L.m3d_last_error()
