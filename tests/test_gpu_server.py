"""The continuous-batching server (bm_server_*) (GPU).

A request's result must be the same when it runs alone and when it runs in
a mix of requests that arrive before and after it (different co-resident
scenes, admission at other step boundaries): the per-particle arithmetic is
identical, only the order of the FP32 reductions changes. That order differs
between any two runs and its effect grows with the steps in a contact scene,
so the bar is the accuracy bar of the plain step (1e-4 dx at 100 steps); a
step missed, taken twice or taken with another scene's state moves the sand
by ~1e-2 dx. It must also match the reference's own
solver, coupler and integrator run alone on the CPU.
"""
import dataclasses
import time

import numpy as np
import pytest

import basements_b200 as bm
from basements_b200 import scenes
from oracle import oracle as O
from tests.gpu_util import POS_TOL_100, max_err_dx

REF = O.reference_or_port()

pytestmark = pytest.mark.gpu


def req_scene(seed, n, grid=32):
    return scenes.box_drop_scene(seed, grid=grid, n_particles=n)


def test_result_same_alone_and_in_mix_and_matches_reference():
    a = req_scene(21, 6000)
    steps = 60
    srv = bm.Server()
    rid = srv.submit(a, steps)
    assert srv.wait(rid) == 0
    alone = srv.result(rid)
    srv.close()

    srv = bm.Server()
    others = [srv.submit(req_scene(30 + k, n, g), st) for k, (n, g, st) in
              enumerate([(20000, 48, 120), (9000, 32, 30), (15000, 64, 90)])]
    time.sleep(0.05)  # the others are on the device when A arrives
    rid = srv.submit(a, steps)
    late = [srv.submit(req_scene(40 + k, 5000), 25) for k in range(3)]
    for r in others + [rid] + late:
        assert srv.wait(r) == 0, r
    mixed = srv.result(rid)
    st = srv.stats()
    srv.close()
    assert st["completed"] == 7 and st["p99_latency_ms"] >= st["p50_latency_ms"] > 0
    e = max_err_dx(alone["position"], mixed["position"], a.dx)
    print(f"alone vs mixed: {e:.2e} dx; p50 {st['p50_latency_ms']:.1f} ms, p99 {st['p99_latency_ms']:.1f} ms")
    assert e < POS_TOL_100
    np.testing.assert_allclose(alone["body"].center[:], mixed["body"].center[:], atol=1e-5)

    c = O.CpuSolver(REF, a.dx)
    c.set_material(a.E, a.nu, a.rho)
    c.set_plastic_alpha(a.alpha)
    c.add_particles(a.position, None, a.mass)
    body = c.run_dynamic_body(O.collider(**a.bodies[0].as_tuple()), a.gravity, a.dt, steps)
    assert max_err_dx(mixed["position"], c.get_particles()["position"], a.dx) < POS_TOL_100
    np.testing.assert_allclose(mixed["body"].center[:], body.center[:], atol=1e-5)


def test_admission_respects_the_hbm_budget():
    scs = [req_scene(50 + k, 4000) for k in range(4)]
    one = bm.estimate_bytes(scs[0])
    srv = bm.Server(hbm_budget_bytes=1.5 * one)  # room for one scene at a time
    ids = [srv.submit(sc, 10) for sc in scs]
    for r in ids:
        assert srv.wait(r) == 0
    st = srv.stats()
    assert st["completed"] == 4 and st["peak_bytes"] <= 1.5 * one
    with pytest.raises(bm.BMError):
        srv.submit(req_scene(60, 60000), 5)  # larger than the whole budget
    srv.close()


def test_failing_request_is_isolated_and_edge_requests():
    """A request whose sand leaves its box completes with BM_ERR_DOMAIN_ESCAPE
    while the requests beside it complete normally and equal their run alone;
    an empty request (a box, no particles) completes with no particles; zero
    steps is an argument error."""
    good = req_scene(80, 5000)
    srv = bm.Server()
    rid = srv.submit(good, 40)
    assert srv.wait(rid) == 0
    alone = srv.result(rid)
    srv.close()

    bad = req_scene(81, 2000)
    bad.domain = ((8, 0, 8), (4, 4, 4))  # far too small: the sand leaves it
    empty = dataclasses.replace(req_scene(82, 2000), position=np.zeros((0, 3), np.float32),
                                mass=np.zeros(0, np.float32), domain=((0, 0, 0), (32, 32, 32)), bodies=[])
    srv = bm.Server()
    ids = [srv.submit(bad, 30), srv.submit(good, 40), srv.submit(empty, 10)]
    assert [srv.wait(r) for r in ids] == [4, 0, 0]  # BM_ERR_DOMAIN_ESCAPE for the escaping request only
    mixed = srv.result(ids[1])
    e = max_err_dx(alone["position"], mixed["position"], good.dx)
    print(f"beside a failing request: {e:.2e} dx from the run alone")
    assert e < POS_TOL_100
    np.testing.assert_allclose(alone["body"].center[:], mixed["body"].center[:], atol=1e-5)
    assert srv.result(ids[2])["position"].shape == (0, 3)
    with pytest.raises(bm.BMError):
        srv.submit(good, 0)
    st = srv.stats()
    assert st["completed"] == 3
    srv.close()


def test_bounded_wait_and_cancel():
    srv = bm.Server()
    rid = srv.submit(req_scene(70, 20000, 48), 100000)
    assert srv.wait(rid, timeout_ms=50) == 6  # BM_ERR_TIMEOUT
    srv.cancel(rid)
    assert srv.wait(rid, timeout_ms=20000) == 8  # BM_ERR_STATE: cancelled, no result
    assert srv.poll(rid) == bm.REQ_CANCELLED
    ok = srv.submit(req_scene(71, 3000), 5)
    assert srv.wait(ok) == 0
    srv.close()
