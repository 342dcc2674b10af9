"""Serving loop (m3d_serve_*): requests of mixed kinds, behaviours and grid
sizes submitted from several host threads run concurrently on the device,
and every result equals the same request served alone, bitwise: a request
runs on its own solver, or as one entry of a multi-RVE solve shared with
queued requests of the same shape and stop rule, whose entries compute
exactly what they would alone."""
import threading

import numpy as np
import pytest

import mat3d_b200 as m3d

pytestmark = pytest.mark.gpu

MAT_E = np.array([[70e9, 0.2, 1e30, 0, 1, 0, 1e30], [3e9, 0.35, 1e30, 0, 1, 0, 1e30]])
MAT_J2 = np.array([[400e9, 0.2, 1e30, 0, 1, 0, 1e30], [70e9, 0.33, 100e6, 1e9, 1, 0, 1e30]])


def sphere_rve(N, r, off=0):
    X, Y, Z = np.meshgrid(np.arange(N), np.arange(N), np.arange(N), indexing="ij")
    c = N / 2 + off
    g = np.ones((N, N, N), np.int32)
    g[(X - c) ** 2 + (Y - N / 2) ** 2 + (Z - N / 2) ** 2 <= r * r] = 0
    return g.ravel()


def requests():
    out = []
    for i in range(12):
        N = (16, 24, 32)[i % 3]
        k = i % 4
        if k == 0:
            out.append(dict(kind=m3d.KIND_MECH, shape=(N,) * 3, phase=sphere_rve(N, 0.3 * N, i % 2),
                            E=[1e-3, 0, 0, 0, 2e-4, 0], mat=MAT_E, precision="fp32_refine", tol=1e-6,
                            keep_field=True))
        elif k == 1:
            out.append(dict(kind=m3d.KIND_THERMAL, shape=(N,) * 3, phase=sphere_rve(N, 0.25 * N), E=[0, 0, 1.0],
                            km=1.0, ki=20.0 + i, precision="fp32_refine", tol=1e-6, keep_field=(i % 2 == 1)))
        elif k == 2:
            out.append(dict(kind=m3d.KIND_MECH, shape=(16,) * 3, phase=sphere_rve(16, 4.0), E=[1e-3, 0, 0, 0, 0, 0],
                            mat=MAT_J2, behav=m3d.J2, X0=[1, 0, 0, 0, 0, 0], nInc=2, precision="fp64", tol=1e-6))
        else:
            out.append(dict(kind=m3d.KIND_MECH, shape=(N,) * 3, phase=sphere_rve(N, 0.2 * N), E=[0, 0, 0, 0, 0, 1e-3],
                            mat=MAT_E, precision="fp64", tol=1e-7, keep_field=True))
    return out


def submit(srv, q):
    q = dict(q)
    return srv.submit(q.pop("kind"), q.pop("shape"), q.pop("phase"), q.pop("E"), **q)


def collect(srv, tickets, reqs):
    res = []
    for t, q in zip(tickets, reqs):
        r = srv.wait(t, 120000.0)
        assert r is not None, "request did not finish"
        f = srv.field(t) if q.get("keep_field") else None
        res.append((r, f))
    return res


def serve_alone(reqs):
    srv = m3d.Server(workers=1)
    out = []
    for q in reqs:
        t = submit(srv, q)
        out.extend(collect(srv, [t], [q]))
    srv.close()
    return out


def check_same(mixed, alone):
    for (r1, f1), (r2, f2) in zip(mixed, alone):
        assert r1["status"] in (m3d.OK, m3d.NOT_CONVERGED) and r1["status"] == r2["status"]
        assert r1["iters"] == r2["iters"] and r1["sweeps"] == r2["sweeps"]
        assert np.array_equal(r1["strain_mean"], r2["strain_mean"])
        assert np.array_equal(r1["stress_mean"], r2["stress_mean"])
        if f1 is not None:
            assert np.array_equal(f1, f2)


def test_mix_equals_alone_two_submitting_threads():
    reqs = requests()
    srv = m3d.Server(workers=6)
    tickets = [None] * len(reqs)

    def producer(idx):
        for i in idx:
            tickets[i] = submit(srv, reqs[i])

    ths = [threading.Thread(target=producer, args=(range(j, len(reqs), 2),)) for j in range(2)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    mixed = collect(srv, tickets, reqs)
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["peak_running"] >= 2  # solves overlapped
    srv.close()
    check_same(mixed, serve_alone(reqs))


def test_budget_admission_serialises_and_matches():
    """A budget that holds one solver of the largest shape: requests of two
    shapes alternate, so each admission must first release the idle solver of
    the other shape; nothing runs concurrently and results are unchanged."""
    reqs = []
    for i in range(6):
        if i % 2 == 0:
            reqs.append(dict(kind=m3d.KIND_THERMAL, shape=(32,) * 3, phase=sphere_rve(32, 8.0 + i), E=[0, 0, 1.0],
                             km=1.0, ki=10.0 + i, precision="fp32_refine", tol=1e-6))
        else:
            reqs.append(dict(kind=m3d.KIND_MECH, shape=(24,) * 3, phase=sphere_rve(24, 5.0 + i), E=[1e-3, 0, 0, 0, 0, 0],
                             mat=MAT_E, precision="fp32_refine", tol=1e-6))
    fps = [m3d.footprint_bytes(q["kind"], q["shape"], 0, q["precision"]) for q in reqs]
    assert max(fps) < sum(sorted(fps)[:2])  # no two solvers fit together
    srv = m3d.Server(mem_budget_bytes=1.05 * max(fps), workers=4)
    tickets = [submit(srv, q) for q in reqs]
    mixed = collect(srv, tickets, reqs)
    st = srv.stats()
    assert st["peak_running"] == 1  # one footprint at a time fits
    assert st["resident_bytes"] <= st["budget_bytes"]
    srv.close()
    check_same(mixed, serve_alone(reqs))


def test_same_shape_requests_merge_and_match():
    """Linear requests of one shape queued together run as multi-RVE solves
    (continuous batching); each result is still bitwise the request alone."""
    reqs = []
    for i in range(10):
        if i % 2 == 0:
            reqs.append(dict(kind=m3d.KIND_THERMAL, shape=(32,) * 3, phase=sphere_rve(32, 6.0 + i / 2, i % 3),
                             E=[0, 0.2 * (i % 3), 1.0], km=1.0, ki=5.0 + 10 * i, precision="fp32_refine", tol=1e-7,
                             keep_field=(i % 4 == 0)))
        else:
            reqs.append(dict(kind=m3d.KIND_MECH, shape=(24,) * 3, phase=sphere_rve(24, 4.0 + i / 3), E=[1e-3, 0, 0, 0, 0, 0],
                             mat=MAT_E, precision="fp64", tol=1e-8, keep_field=(i % 3 == 0)))
    srv = m3d.Server(workers=1)
    blocker = submit(srv, dict(kind=m3d.KIND_THERMAL, shape=(64,) * 3, phase=sphere_rve(64, 20.0), E=[0, 0, 1.0],
                               km=1.0, ki=50.0, precision="fp64", tol=1e-10))
    tickets = [submit(srv, q) for q in reqs]  # queued behind the blocker, then merged by shape
    srv.wait(blocker, 120000.0)
    mixed = collect(srv, tickets, reqs)
    st = srv.stats()
    assert st["failed"] == 0 and st["merged_solves"] >= 2 and st["merged_requests"] >= 4
    srv.close()
    check_same(mixed, serve_alone(reqs))


def test_failed_request_does_not_stop_the_server():
    srv = m3d.Server(workers=2)
    bad = dict(requests()[0])
    bad["mat"] = np.array([[-1.0, 0.2, 1e30, 0, 1, 0, 1e30], [3e9, 0.35, 1e30, 0, 1, 0, 1e30]])
    good = requests()[1]
    tb = submit(srv, bad)
    tg = submit(srv, good)
    with pytest.raises(m3d.M3DError):
        r = srv.wait(tb, 60000.0)
        if r is not None and r["status"] not in (m3d.OK, m3d.NOT_CONVERGED):
            raise m3d.M3DError(r["status"], "failed as expected")
    rg = srv.wait(tg, 60000.0)
    assert rg["status"] == m3d.OK
    assert srv.stats()["failed"] == 1
    with pytest.raises(m3d.M3DError):
        srv.poll(987654)  # unknown ticket
    srv.close()
