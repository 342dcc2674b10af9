"""Many RVEs in one batch (m3d_create_multi): every RVE's result equals the
same RVE solved on its own handle, bitwise, and one RVE of the batch is
checked against the CPU oracle.

Each entry of a batch evaluates its own stop rule and its own deterministic
fixed-order reductions, and each RVE's tables and Green-operator constants
are its own, so sharing a launch with other RVEs must not change a single bit.
"""
import numpy as np
import pytest

import mat3d_b200 as m3d
from oracle import mat3d_oracle as O

pytestmark = pytest.mark.gpu


def sphere_rve(shape, r, center=None):
    Nx, Ny, Nz = shape
    X, Y, Z = np.meshgrid(np.arange(Nx), np.arange(Ny), np.arange(Nz), indexing="ij")
    c = center or (Nx / 2, Ny / 2, Nz / 2)
    rve = np.ones(shape, np.int32)
    rve[(X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2 <= r * r] = 0
    return rve.ravel()


def mech_mat(contrast, stiff_matrix=False):
    inc = [contrast * 3e9, 0.2, 1e30, 0, 1, 0, 1e30]
    mtx = [3e9, 0.35, 1e30, 0, 1, 0, 1e30]
    return np.array([mtx, inc] if stiff_matrix else [inc, mtx])


# three RVEs that differ in microstructure, contrast and scheme (the third has
# a dominant stiff phase, so the automatic choice is the stress-based scheme)
MECH_CASES = [
    (dict(r=3.0), mech_mat(20.0), m3d.SCHEME_AUTO),
    (dict(r=4.5, center=(5, 9, 7)), mech_mat(3.0), m3d.SCHEME_AUTO),
    (dict(r=5.0), mech_mat(50.0, stiff_matrix=True), m3d.SCHEME_AUTO),
]


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-10), ("fp32_refine", 1e-9), ("fp32", 1e-5)])
def test_multi_elastic_homogenize_equals_single(prec, tol):
    shape = (16, 16, 16)
    R = len(MECH_CASES)
    mb = m3d.Solver(m3d.KIND_MECH, *shape, 0, prec, nrve=R, nload=6)
    rves = [sphere_rve(shape, **geo) for geo, _, _ in MECH_CASES]
    for r, (_, mat, sch) in enumerate(MECH_CASES):
        mb.set_material_mech(mat, rves[r], sch, rve=r)
    Cm, Sm, epm, sgm, _ = mb.homogenize(tol, 0, m3d.CRIT_RESIDUAL)
    assert Cm.shape == (R, 6, 6)
    schemes = []
    for r, (_, mat, sch) in enumerate(MECH_CASES):
        s1 = m3d.Solver(m3d.KIND_MECH, *shape, 0, prec, 6)
        s1.set_material_mech(mat, rves[r], sch)
        schemes.append(s1.stats()["scheme"])
        C1, S1, ep1, sg1, _ = s1.homogenize(tol, 0, m3d.CRIT_RESIDUAL)
        assert np.array_equal(Cm[r], C1), (r, np.abs(Cm[r] - C1).max())
        assert np.array_equal(Sm[r], S1)
        assert np.array_equal(epm[r], ep1) and np.array_equal(sgm[r], sg1)
        s1.close()
    assert 1 in schemes and 2 in schemes  # both schemes share the batch
    mb.close()


def test_multi_elastic_vs_oracle():
    shape = (12, 12, 12)
    geo, mat, _ = MECH_CASES[2]
    rves = [sphere_rve(shape, 2.5), sphere_rve(shape, 3.5)]
    mats = [mech_mat(10.0), mat]
    mb = m3d.Solver(m3d.KIND_MECH, *shape, 0, "fp64", nrve=2, nload=6)
    for r in range(2):
        mb.set_material_mech(mats[r], rves[r], rve=r)
    Cm, Sm, *_ = mb.homogenize(1e-10, 1e-10, m3d.CRIT_REFERENCE)
    for r in range(2):
        o = O.MechOracle(*shape, "e")
        o.material(mats[r], rves[r])
        CH, SH = o.homogenization(1e-10, 1e-10)
        assert np.abs(Cm[r] - CH).max() / np.abs(CH).max() < 1e-9
        assert np.abs(Sm[r] - SH).max() / np.abs(SH).max() < 1e-9
    mb.close()


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-10), ("fp32_refine", 1e-9)])
def test_multi_thermal_homogenize_equals_single(prec, tol):
    shape = (16, 16, 16)
    cases = [(1.0, 100.0, sphere_rve(shape, 4.0)),   # gradient-based
             (100.0, 1.0, sphere_rve(shape, 3.0)),   # flux-based
             (1.0, 5.0, sphere_rve(shape, 5.5, (4, 4, 4)))]
    mb = m3d.Solver(m3d.KIND_THERMAL, *shape, 0, prec, nrve=len(cases), nload=3)
    for r, (km, ki, rve) in enumerate(cases):
        mb.set_material_thermal(km, ki, rve, rve=r)
    Km, Rm, *_ = mb.homogenize(tol, 0, m3d.CRIT_RESIDUAL)
    schemes = []
    for r, (km, ki, rve) in enumerate(cases):
        s1 = m3d.Solver(m3d.KIND_THERMAL, *shape, 0, prec, 3)
        s1.set_material_thermal(km, ki, rve)
        schemes.append(s1.stats()["scheme"])
        K1, R1, *_ = s1.homogenize(tol, 0, m3d.CRIT_RESIDUAL)
        assert np.array_equal(Km[r], K1), (r, np.abs(Km[r] - K1).max())
        assert np.array_equal(Rm[r], R1)
        s1.close()
    assert 1 in schemes and 2 in schemes
    mb.close()


def test_multi_run_fields_and_loads():
    """nload = 2 with per-entry loads through m3d_run: fields of every entry
    equal the single-RVE solves."""
    shape = (16, 16, 16)
    R, L = 3, 2
    mb = m3d.Solver(m3d.KIND_MECH, *shape, 0, "fp64", nrve=R, nload=L)
    rves = [sphere_rve(shape, 3.0 + r) for r in range(R)]
    mats = [mech_mat(5.0 + 20 * r) for r in range(R)]
    loads = [np.array([1e-3, 0, 0, 0, 0, 0.0]), np.array([0, 0, 0, 2e-4, 0, 3e-4])]
    for r in range(R):
        mb.set_material_mech(mats[r], rves[r], rve=r)
        for l in range(L):
            mb.set_load(loads[l], None, b=r * L + l)
    mb.run(1e-9, 0, 1, m3d.CRIT_RESIDUAL)
    for r in range(R):
        s1 = m3d.Solver(m3d.KIND_MECH, *shape, 0, "fp64", L)
        s1.set_material_mech(mats[r], rves[r])
        for l in range(L):
            s1.set_load(loads[l], None, b=l)
        s1.run(1e-9, 0, 1, m3d.CRIT_RESIDUAL)
        for l in range(L):
            for which in (m3d.FIELD_STRAIN, m3d.FIELD_STRESS):
                assert np.array_equal(mb.field(which, r * L + l), s1.field(which, l)), (r, l, which)
            em, sm = mb.means(r * L + l)
            e1, s1m = s1.means(l)
            assert np.array_equal(em, e1) and np.array_equal(sm, s1m)
        s1.close()
    mb.close()


def test_multi_rejects_unset_rve_and_bad_index():
    shape = (8, 8, 8)
    mb = m3d.Solver(m3d.KIND_MECH, *shape, 0, "fp64", nrve=2, nload=6)
    mb.set_material_mech(mech_mat(10.0), sphere_rve(shape, 2.0), rve=0)
    with pytest.raises(m3d.M3DError):
        mb.homogenize(1e-8)  # RVE 1 has no material yet
    with pytest.raises(m3d.M3DError):
        mb.set_material_mech(mech_mat(10.0), sphere_rve(shape, 2.0), rve=2)
    mb.close()


# ---- m3d_batch_*: mixed grid sizes, memory-budget chunking ------------------
def _batch_members(kind, n=7):
    out = []
    for i in range(n):
        N = (12, 16, 20)[i % 3]
        shape = (N, N, N)
        rve = sphere_rve(shape, 0.22 * N + 0.3 * (i % 2), (N / 2 + i % 3, N / 2, N / 2 - i % 2))
        if kind == m3d.KIND_MECH:
            out.append((shape, mech_mat(2.0 + 15 * i, stiff_matrix=(i % 4 == 3)), rve))
        else:
            out.append((shape, (1.0, 2.0 + 20 * i) if i % 2 else (30.0 + i, 1.0), rve))
    return out


@pytest.mark.parametrize("kind,prec", [(m3d.KIND_MECH, "fp32_refine"), (m3d.KIND_MECH, "fp64"),
                                       (m3d.KIND_THERMAL, "fp32_refine")])
@pytest.mark.parametrize("budget_rves", [0, 1])
def test_batch_api_equals_single(kind, prec, budget_rves):
    """Every tensor of a mixed-size batch equals m3d_homogenize on its RVE alone;
    a budget of one RVE of the largest grid forces several launches per size."""
    members = _batch_members(kind)
    C = 6 if kind == m3d.KIND_MECH else 3
    budget = 0.0
    if budget_rves:
        budget = float(m3d.footprint_bytes(kind, (20, 20, 20), 0, prec, budget_rves, budget_rves * C))
    bt = m3d.Batch(kind, prec, budget)
    for shape, mat, rve in members:
        if kind == m3d.KIND_MECH:
            bt.add_mech(shape, mat, rve)
        else:
            bt.add_thermal(shape, mat[0], mat[1], rve)
    Ce, Se, _ = bt.homogenize(1e-9)
    st = bt.stats()
    assert st["rves"] == len(members) and st["groups"] == 3
    assert (st["launches"] >= 5) if budget_rves else (st["launches"] == 3)
    # with the whole batch in budget the three grid sizes run at once (own
    # threads and streams); a one-RVE budget runs them one after another
    assert st["concurrent"] == (0 if budget_rves else 1)
    assert st["voxel_iters"] > 0 and st["device_ms"] > 0
    for i, (shape, mat, rve) in enumerate(members):
        s1 = m3d.Solver(kind, *shape, 0, prec, C)
        if kind == m3d.KIND_MECH:
            s1.set_material_mech(mat, rve)
        else:
            s1.set_material_thermal(mat[0], mat[1], rve)
        C1, S1, *_ = s1.homogenize(1e-9, 0, m3d.CRIT_RESIDUAL)
        assert np.array_equal(Ce[i], C1), (i, np.abs(Ce[i] - C1).max())
        assert np.array_equal(Se[i], S1)
        s1.close()
    bt.close()


def test_batch_budget_too_small():
    bt = m3d.Batch(m3d.KIND_MECH, "fp64", 1e6)
    bt.add_mech((16, 16, 16), mech_mat(10.0), sphere_rve((16, 16, 16), 3.0))
    with pytest.raises(m3d.M3DError):
        bt.homogenize(1e-8)
    bt.close()


def test_phase_map_ids_on_device():
    """The phase map is converted on the device: an id outside [0, nph) is
    reported at its first voxel and leaves the RVE unset (a solve is refused
    until it is set again); thermal ids are tested only for != 0, so a map of
    0/5 gives the field of the same map as 0/1 under the same scheme."""
    N = 16
    rve = sphere_rve((N, N, N), 4.0)
    bad = rve.copy()
    bad[37] = 2
    bad[900] = -1
    s = m3d.Solver(m3d.KIND_MECH, N, N, N, m3d.ELASTIC, "fp64", 1)
    s.set_material_mech(mech_mat(5.0), rve)
    with pytest.raises(m3d.M3DError) as ei:
        s.set_material_mech(mech_mat(5.0), bad)
    assert "at voxel 37" in str(ei.value)
    s.set_load(np.array([1e-3, 0, 0, 0, 0, 0.0]))
    with pytest.raises(m3d.M3DError):
        s.run(1e-8, 1e-8, 1, m3d.CRIT_RESIDUAL)
    s.set_material_mech(mech_mat(5.0), rve)
    s.run(1e-8, 1e-8, 1, m3d.CRIT_RESIDUAL)
    s.close()
    out = []
    for ids in (rve, rve * 5):
        t = m3d.Solver(m3d.KIND_THERMAL, N, N, N, 0, "fp64", 1)
        t.set_material_thermal(1.0, 20.0, ids, m3d.SCHEME_PRIMAL)
        t.set_load(np.array([0.0, 0.0, 1.0]))
        t.run(1e-10, 0, 1, m3d.CRIT_RESIDUAL)
        out.append(t.field(m3d.FIELD_STRAIN))
        t.close()
    assert np.array_equal(out[0], out[1])
