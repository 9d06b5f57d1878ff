"""The differentiable run (bm_tape_* / bm_adjoint_backward) (GPU).

The reference has no gradient to compare with (its AutodiffTape records
nothing), so the adjoint is checked against central finite differences of
the same loss on the FP64 oracle running the same split step. A tine is
dragged through a sand bed along a seeded waypoint path; the loss is the L2
distance between the final soft heightfield and a seeded target.

The coupler's inside test is a step function of the body pose: a grid node
jumps between the sand's and the blended velocity when a face of the body
crosses it. The loss is therefore discontinuous in the waypoints, and a
central difference over [w - eps, w + eps] picks up jump/(2 eps) for every
crossing inside the interval (at eps = 1e-4 about one crossing per
coordinate on this scene, a few % of the gradient). The adjoint is the
derivative between crossings, so the waypoint check takes eps = 1e-6, where
a crossing is unlikely (~1e-2 per coordinate) and FP64 rounding is still far
below the signal; the eps = 1e-4 differences are printed beside it.
"""
import numpy as np
import pytest

import basements_b200 as bm
from basements_b200 import scenes
from oracle import oracle as O
from tests import fd_util
from tests.gpu_util import POS_TOL_100, gpu_solver, max_err_dx

pytestmark = pytest.mark.gpu

ADJ_REL_TOL = 1e-3


def small_tine():
    return scenes.tine_pass(grid=32, bed_cells=(32, 8, 32), ppc=2, n_waypoints=6, steps=40, dt=2e-4,
                            tine_half=(0.02, 0.06, 0.04), depth=0.05, speed=1.0, jitter=5e-4, seed=1)


def run_tape(sc, body, wp, steps, K):
    s = gpu_solver(sc.dx, sc.position, None, sc.mass, sc.E, sc.nu, sc.rho, sc.alpha, domain=sc.domain)
    tape = bm.Tape(s, K)
    tape.forward(sc.dt, steps, bm.make_collider(**body.as_tuple()), wp)
    return s, tape


@pytest.fixture(scope="module")
def fdpool():
    p = fd_util.pool()
    yield p
    p.close()
    p.join()


def test_tape_forward_matches_reference_split_path():
    sc, body, wp, target = small_tine()
    s, tape = run_tape(sc, body, wp, sc.steps, 20)
    ref = fd_util.oracle_run(O.reference_or_port(), sc, body, wp, sc.steps)
    e = max_err_dx(s.get_particles()["position"], ref, sc.dx)
    print(f"tape forward vs reference split path, {sc.steps} steps: {e:.2e} dx")
    assert e < POS_TOL_100


def test_waypoint_gradient_matches_fp64_finite_differences(fdpool):
    sc, body, wp, target = small_tine()
    s, tape = run_tape(sc, body, wp, sc.steps, 20)
    L, g = scenes.heightfield_loss(s.get_particles()["position"], target)
    gw = tape.backward(g)["dL_dwaypoints"]
    coords = [(k, a) for k in range(1, 5) for a in (0, 1)]
    fd = fd_util.fd_waypoints(fdpool, sc, body, wp, sc.steps, target, coords, eps=1e-6)
    fd4 = fd_util.fd_waypoints(fdpool, sc, body, wp, sc.steps, target, coords, eps=1e-4)
    ad = np.array([gw[k, a] for k, a in coords])
    rel = np.linalg.norm(ad - fd) / np.linalg.norm(fd)
    for (k, a), x, y, z in zip(coords, ad, fd, fd4):
        print(f"waypoint {k} axis {a}: adjoint {x:+.6e}  fd(1e-6) {y:+.6e}  fd(1e-4) {z:+.6e}")
    print(f"relative error (norm over {len(coords)} coordinates): {rel:.2e}")
    assert rel < ADJ_REL_TOL


def test_initial_state_gradient_matches_fp64_directional_difference(fdpool):
    sc, body, wp, target = small_tine()
    s, tape = run_tape(sc, body, wp, sc.steps, 20)
    L, g = scenes.heightfield_loss(s.get_particles()["position"], target)
    gx0 = tape.backward(g, want_x0=True)["dL_dx0"].astype(np.float64)
    rng = np.random.default_rng(5)
    delta = rng.normal(size=sc.position.shape)
    dL, hi, lo = fd_util.fd_direction_x0(fdpool, sc, body, wp, sc.steps, target, delta, 2e-5)
    pred = float(np.sum(gx0 * (hi.astype(np.float64) - lo.astype(np.float64))))
    print(f"directional: adjoint {pred:+.6e}  fd {dL:+.6e}")
    assert abs(pred - dL) < ADJ_REL_TOL * abs(dL)


def test_checkpoint_interval_does_not_change_the_gradient():
    sc, body, wp, target = small_tine()
    grads = []
    for K in (1, 7, 40):
        s, tape = run_tape(sc, body, wp, sc.steps, K)
        L, g = scenes.heightfield_loss(s.get_particles()["position"], target)
        grads.append(tape.backward(g)["dL_dwaypoints"])
        # backward leaves the solver in the recorded final state
        L2, _ = scenes.heightfield_loss(s.get_particles()["position"], target)
        assert L2 == L
    for G in grads[1:]:
        rel = np.linalg.norm(G - grads[0]) / np.linalg.norm(grads[0])
        print(f"checkpoint interval: relative change {rel:.2e}")
        assert rel < ADJ_REL_TOL


def test_backward_needs_a_forward_and_body_optional():
    sc, body, wp, target = small_tine()
    s = gpu_solver(sc.dx, sc.position, None, sc.mass, sc.E, sc.nu, sc.rho, sc.alpha, domain=sc.domain)
    tape = bm.Tape(s, 10)
    with pytest.raises(bm.BMError):
        tape.backward(np.zeros((sc.n, 3), np.float32))
    tape.forward(sc.dt, 12)  # no body
    L, g = scenes.heightfield_loss(s.get_particles()["position"], target)
    out = tape.backward(g, want_x0=True, want_v0=True)
    assert "dL_dwaypoints" not in out and np.isfinite(out["dL_dx0"]).all() and np.abs(out["dL_dv0"]).max() > 0
