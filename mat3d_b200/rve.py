"""Seeded synthetic microstructures (voxel RVEs) and the reference's RVE text format.

Phase ids follow the reference: 1 = matrix, 0 = inclusion
(include/FFT_analysis3D.hpp:44-45).  Grids are ``[Nx, Ny, Nz]`` with z the
fastest axis, flattened as ``z + Nz*(y + Ny*x)`` exactly like the single-column
RVE files the reference's drivers read (example/3d/main.cpp:66-88).

Each generator is deterministic for a given seed (numpy PCG64) and periodic
(minimum-image distances), so the same seed gives the same RVE on every host.
"""
from __future__ import annotations

import math

import numpy as np


def _periodic_delta(coord, c, n):
    d = coord - c
    return d - n * np.round(d / n)


def _paint_ellipsoid(grid, center, axes_mat, semi, phase=0):
    """Set voxels whose centre lies inside the (periodic) ellipsoid to ``phase``.

    axes_mat: 3x3 rotation whose rows are the principal directions; semi: semi-axes."""
    N = grid.shape
    r = float(max(semi))
    lo = [int(math.floor(center[i] - r)) for i in range(3)]
    hi = [int(math.ceil(center[i] + r)) for i in range(3)]
    ix = np.arange(lo[0], hi[0] + 1)
    iy = np.arange(lo[1], hi[1] + 1)
    iz = np.arange(lo[2], hi[2] + 1)
    X, Y, Z = np.meshgrid(ix, iy, iz, indexing="ij")
    d = np.stack([X - center[0], Y - center[1], Z - center[2]], axis=-1).astype(np.float64)
    loc = d @ np.asarray(axes_mat, np.float64).T
    q = (loc[..., 0] / semi[0]) ** 2 + (loc[..., 1] / semi[1]) ** 2 + (loc[..., 2] / semi[2]) ** 2
    m = q <= 1.0
    flat = np.unique(np.ravel_multi_index((X[m] % N[0], Y[m] % N[1], Z[m] % N[2]), N))
    changed = int(np.count_nonzero(grid.ravel()[flat] != phase))
    grid.ravel()[flat] = phase
    return changed


def spheres_rsa(N, radius=6.0, vf=0.20, seed=0, gap=1.0, max_tries=200000, radii_fn=None):
    """Non-overlapping spheres by periodic random sequential addition until the
    inclusion fraction reaches ``vf``.  ``radii_fn(rng)`` draws a radius per
    sphere (default: the fixed ``radius``).  Returns (int32 grid [N,N,N], meta)."""
    Nx, Ny, Nz = (N, N, N) if np.isscalar(N) else tuple(N)
    rng = np.random.default_rng(seed)
    grid = np.ones((Nx, Ny, Nz), np.int32)
    box = np.array([Nx, Ny, Nz], np.float64)
    cs = np.zeros((0, 3))
    rs = np.zeros(0)
    n_inc = 0  # inclusion voxels, kept up to date as spheres are painted
    tries = 0
    while n_inc / grid.size < vf and tries < max_tries:
        tries += 1
        r = float(radii_fn(rng)) if radii_fn else float(radius)
        c = rng.uniform(0, 1, 3) * box
        if len(rs):
            d = _periodic_delta(c[None, :], cs, box)
            if np.any(np.einsum("ij,ij->i", d, d) < (r + rs + gap) ** 2):
                continue
        cs = np.vstack([cs, c])
        rs = np.append(rs, r)
        n_inc += _paint_ellipsoid(grid, c, np.eye(3), (r, r, r))
    meta = dict(n_inclusions=len(rs), vf=float(np.count_nonzero(grid == 0) / grid.size), seed=seed)
    return grid, meta


def penetrable_spheres(N, radius, vf, seed=0, max_spheres=100000):
    """Overlapping (penetrable) spheres of one radius at uniform random
    periodic centres, added until the inclusion fraction reaches ``vf``; any
    fraction is reachable (non-overlapping placement jams near 38%)."""
    Nx, Ny, Nz = (N, N, N) if np.isscalar(N) else tuple(N)
    rng = np.random.default_rng(seed)
    grid = np.ones((Nx, Ny, Nz), np.int32)
    box = np.array([Nx, Ny, Nz], np.float64)
    n_inc, n = 0, 0
    while n_inc / grid.size < vf and n < max_spheres:
        c = rng.uniform(0, 1, 3) * box
        n_inc += _paint_ellipsoid(grid, c, np.eye(3), (radius, radius, radius))
        n += 1
    return grid, dict(n_inclusions=n, vf=float(n_inc / grid.size), seed=seed, radius=radius)


def _random_rotation(rng):
    """Uniform rotation on SO(3) from a uniform unit quaternion."""
    q = rng.standard_normal(4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def ellipsoids(N, vf=0.30, aspect=3.0, n_target=100, seed=0):
    """Prolate ellipsoids (aspect*a, a, a), uniformly random orientation, overlap
    allowed, added until the inclusion fraction reaches ``vf``.  ``a`` is chosen
    so that ``n_target`` non-overlapping ellipsoids would fill ``vf``."""
    Nx, Ny, Nz = (N, N, N) if np.isscalar(N) else tuple(N)
    V = Nx * Ny * Nz
    a = (vf * V / (n_target * 4.0 / 3.0 * math.pi * aspect)) ** (1.0 / 3.0)
    rng = np.random.default_rng(seed)
    grid = np.ones((Nx, Ny, Nz), np.int32)
    n = 0
    while np.count_nonzero(grid == 0) / V < vf and n < 100 * n_target:
        c = rng.uniform(0, 1, 3) * np.array([Nx, Ny, Nz])
        R = _random_rotation(rng)
        _paint_ellipsoid(grid, c, R.T, (aspect * a, a, a))
        n += 1
    meta = dict(n_inclusions=n, a=a, aspect=aspect, vf=float(np.count_nonzero(grid == 0) / V), seed=seed)
    return grid, meta


def lognormal_spheres(N, vf=0.15, median=5.0, sigma=0.4, rmin=3.0, rmax=10.0, seed=0):
    """Non-overlapping spheres with log-normal radii (median, sigma of ln r),
    clipped to [rmin, rmax]."""
    mu = math.log(median)
    fn = lambda rng: float(np.clip(rng.lognormal(mu, sigma), rmin, rmax))
    g, meta = spheres_rsa(N, vf=vf, seed=seed, radii_fn=fn)
    meta.update(mu_ln_r=mu, sigma_ln_r=sigma)
    return g, meta


def batch_rves(count=512, sizes=(32, 48, 64, 96), seed0=0, vf_range=(0.05, 0.40), contrast_range=(2.0, 100.0)):
    """The batched-homogenization workload: per seed s, N uniform on ``sizes``,
    sphere vf uniform in ``vf_range`` and stiffness contrast uniform in
    ``contrast_range`` (inclusion E = contrast * 3 GPa, nu 0.2; matrix 3 GPa, 0.35).
    Yields (seed, N, vf, contrast) descriptors; ``batch_member`` builds one."""
    out = []
    for s in range(seed0, seed0 + count):
        rng = np.random.default_rng(10_000 + s)
        N = int(sizes[rng.integers(len(sizes))])
        vf = float(rng.uniform(*vf_range))
        con = float(rng.uniform(*contrast_range))
        out.append((s, N, vf, con))
    return out


def batch_member(seed, N, vf, contrast):
    """RVE ``seed`` of the batched workload: penetrable spheres of radius N/10
    to inclusion fraction ``vf``; inclusion E = contrast * 3 GPa, nu 0.2."""
    r = max(2.0, N / 10.0)
    g, meta = penetrable_spheres(N, radius=r, vf=vf, seed=seed)
    mat = np.array([[contrast * 3e9, 0.2, 1e30, 0, 1, 0, 1e30], [3e9, 0.35, 1e30, 0, 1, 0, 1e30]])
    return g, mat, meta


def read_rve_txt(path, n_expected=None):
    """Single-column 0/1 text RVE (example/3d/main.cpp:69-88): one phase id per
    line in voxel order z + Nz*(y + Ny*x).  Raises if the count is wrong."""
    vals = np.loadtxt(path, dtype=np.float64).astype(np.int32).ravel()
    if n_expected is not None and vals.size != n_expected:
        raise ValueError(f"Dimension is not correct: {vals.size} values, expected {n_expected}")
    return vals


def write_rve_txt(path, grid):
    np.savetxt(path, np.asarray(grid).ravel().astype(np.int32), fmt="%d")


# Material tables of the benchmark workloads: rows [E, nu, sigma_y, H, n, P, Y0]
# per phase (the reference's mat table, example/3d/main.cpp:103-111).
MAT_ELASTIC_SPHERES = np.array([[70e9, 0.2, 1e30, 0.0, 1.0, 0.0, 1e30],   # inclusion (phase 0)
                                [3e9, 0.35, 1e30, 0.0, 1.0, 0.0, 1e30]])  # matrix (phase 1)
MAT_J2_PARTICLES = np.array([[400e9, 0.2, 1e30, 0.0, 1.0, 0.0, 1e30],      # elastic particles
                             [70e9, 0.33, 100e6, 1e9, 1.0, 0.0, 1e30]])    # J2 matrix, linear hardening


def tpcf_isotropic(shape, A=25.0, Q=0.4, phi1=0.5):
    """Two-point correlation function S2 of a statistically isotropic two-phase
    medium, centred on (Nx/2, Ny/2, Nz/2), as example/reconst3d/main.cpp
    builds it: S2 = f(r) phi1 phi2 + phi1^2 with the scaled autocovariance
    f(r) = exp(-r/A) sin(Q r) / (Q r) (f(0) = 1), r the distance from the centre."""
    Nx, Ny, Nz = shape
    X, Y, Z = np.meshgrid(np.arange(Nx) - Nx // 2, np.arange(Ny) - Ny // 2, np.arange(Nz) - Nz // 2, indexing="ij")
    r = np.sqrt(X * X + Y * Y + Z * Z * 1.0)
    with np.errstate(invalid="ignore", divide="ignore"):
        fr = np.exp(-r / A) * np.sin(Q * r) / (Q * r)
    fr[r == 0] = 1.0
    return (fr * phi1 * (1 - phi1) + phi1 * phi1).ravel()


def reconstruction_input(shape, A=25.0, Q=0.4, phi1=0.5):
    """What the example hands to recPlan: the centred S2 moved to index 0
    (recon::ifftshift) and replaced by the real part of its 3-D transform."""
    import mat3d_b200 as m3d
    t = m3d.ifftshift(tpcf_isotropic(shape, A, Q, phi1), *shape)
    return np.ascontiguousarray(np.real(np.fft.fftn(t.reshape(shape))).ravel())
