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
# The full tine pass (262k particles, 200 steps): the float adjoint against
# FP64 differences on the branch of an FP32 forward measured 1.04e-3 (1.22e-3
# on the FP64 run's own branch; the same at eps = 3e-7, 1e-6 and 2e-6), so
# its bar is a fixed 2e-3.
ADJ_REL_TOL_FULL = 2e-3


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


def test_tape_can_be_destroyed_after_its_solver():
    """A tape outliving its solver (as when both end in a reference cycle)
    frees its own buffers and leaves no CUDA error behind for the next call."""
    sc, body, wp, target = small_tine()
    s, tape = run_tape(sc, body, wp, 4, 2)
    s.close()
    tape.close()
    g = gpu_solver(sc.dx, sc.position, None, sc.mass, sc.E, sc.nu, sc.rho, sc.alpha, domain=sc.domain)
    g.step(sc.dt, 2)
    assert g.sync() == (0, 0)


def check_waypoint_gradient(gw, fd, coords, what):
    """Adjoint dL/d waypoint against the frozen-decision differences: the
    relative error of the 8-vector (the bar) and of each coordinate (printed
    beside its value)."""
    ad = np.array([gw[k, a] for k, a in coords])
    rel = np.linalg.norm(ad - fd) / np.linalg.norm(fd)
    for (k, a), x, y in zip(coords, ad, fd):
        print(f"waypoint {k:2d} axis {a}: adjoint {x:+.6e}  fd {y:+.6e}  rel {abs(x - y) / abs(y):.1e}")
    print(f"{what}: relative error of the gradient (norm) {rel:.2e}")
    return rel


def test_waypoint_gradient_matches_fp64_finite_differences(fdpool):
    """dL/d(waypoints) of the 40-step tine pass against FP64 central
    differences at eps = 1e-6 with the run's discontinuous decisions frozen
    (the SVD's pair skips and sweep stops and the coupler's inside sets of
    the unperturbed run replayed on both sides, tests/fd_util.py), i.e. the
    derivative of the branch the adjoint differentiates. The free
    differences at eps = 1e-4 are printed for comparison (they include the
    jumps of every decision the perturbation flips). Bar: 1e-3 relative."""
    sc, body, wp, target = small_tine()
    s, tape = run_tape(sc, body, wp, sc.steps, 20)
    L, g = scenes.heightfield_loss(s.get_particles()["position"], target)
    gw = tape.backward(g)["dL_dwaypoints"]
    coords = [(k, a) for k in range(1, 5) for a in (0, 1)]
    fd, consistent = fd_util.fd_waypoints_frozen(fdpool, sc, body, wp, sc.steps, target, coords, eps=1e-6)
    assert consistent
    fd4 = fd_util.fd_waypoints(fdpool, sc, body, wp, sc.steps, target, coords, eps=1e-4)
    print("free differences at eps = 1e-4:", " ".join(f"{v:+.6e}" for v in fd4))
    assert check_waypoint_gradient(gw, fd, coords, "40-step tine pass") < ADJ_REL_TOL


def test_initial_state_gradient_matches_fp64_directional_difference(fdpool):
    """dL/dx0 along a random direction of the particles away from the tine.

    Where the tine shears the sand plastically, the FP64 loss is not smooth
    in the particle positions: the reference SVD stops early (rotation skipped
    below |a_ij| = 1e-6, sweeps stopped below 1e-5), the projected F depends
    on the unconverged U and V, and a perturbation that flips one of those
    decisions moves F by the residual. A difference over all particles then
    does not converge as eps shrinks (measured 0.7 % .. 2.7 % off for eps
    2e-5 .. 2e-7), while over the elastic region it does (1.8e-3 at 2e-5,
    1.5e-4 at 2e-6); the plastic region is covered by the waypoint test and
    the one-step field tests."""
    sc, body, wp, target = small_tine()
    s, tape = run_tape(sc, body, wp, sc.steps, 20)
    L, g = scenes.heightfield_loss(s.get_particles()["position"], target)
    gx0 = tape.backward(g, want_x0=True)["dL_dx0"].astype(np.float64)
    rng = np.random.default_rng(5)
    far = np.abs(sc.position[:, 0] - 0.3) > 0.2
    delta = rng.normal(size=sc.position.shape) * far[:, None]
    dL, hi, lo = fd_util.fd_direction_x0(fdpool, sc, body, wp, sc.steps, target, delta, 2e-6)
    pred = float(np.sum(gx0 * (hi.astype(np.float64) - lo.astype(np.float64))))
    print(f"directional: adjoint {pred:+.6e}  fd {dL:+.6e}")
    assert abs(pred - dL) < ADJ_REL_TOL * abs(dL)


FIELDS = {"position": 3, "velocity": 3, "F": 9, "C": 9}
# Perturbations applied in double around the float32 state. The oracle's
# SVD stops on thresholds (rotation skipped below |a_ij| = 1e-6, sweeps
# stopped below 1e-5), and near F = I those decisions sit at the 1e-6..1e-7
# level: a change of one float32 ulp of F (1e-7) already flips some, and the
# jump (the size of the SVD residual) swamps the signal. So F and x, which
# reach F_trial directly, move by 1e-10 .. 3e-10; v and C reach it through
# dt-scaled terms and take larger steps so that the weak couplings stay well
# above double rounding.
FD_EPS = {"position": 1e-10, "velocity": 1e-7, "F": 3e-10, "C": 1e-6}


@pytest.mark.parametrize("use_body", [False, True])
def test_adjoint_of_each_state_field_matches_fp64_differences(use_body):
    """One step: a loss linear in one field of the final state (x, v, F or
    C), its gradient with respect to each field of a random initial state,
    against directional differences of the FP64 oracle: every path through
    the adjoint kernels, the DP/SVD and Hencky adjoints at F near I included.
    Over several steps the float32 state drifts from the FP64 one by ~1e-7,
    which moves the SVD decisions of later steps, so losses on F are checked
    over one step only; the multi-step chain is covered by the waypoint and
    initial-state tests."""
    steps = 1
    sc, body, wp, _ = scenes.tine_pass(grid=32, bed_cells=(12, 6, 12), ppc=2, n_waypoints=4, steps=steps, dt=2e-4,
                                       tine_half=(0.02, 0.06, 0.04), depth=0.05, speed=1.0, jitter=5e-4, seed=1)
    x0 = (sc.position + np.array([0.22, 0.02, 0.3], np.float32)).astype(np.float32)
    n = len(x0)
    rng = np.random.default_rng(1)
    st0 = {"position": x0, "velocity": (rng.normal(size=(n, 3)) * 0.3).astype(np.float32),
           "F": (np.eye(3)[None] + 1e-3 * rng.normal(size=(n, 3, 3))).astype(np.float32),
           "C": rng.normal(size=(n, 3, 3)).astype(np.float32)}
    bodies = [scenes.body_on_path(body, wp, steps, sc.dt, k) for k in range(steps)]

    def oracle_state(st):
        c = O.CpuSolver("f64", sc.dx)
        c.set_material(sc.E, sc.nu, sc.rho)
        c.set_plastic_alpha(sc.alpha)
        c.add_particles(st0["position"], None, sc.mass)
        c.set_state_f64(st["position"], st["velocity"], st["F"], st["C"])
        for b in bodies:
            c.p2g(sc.dt)
            c.grid_update(sc.dt)
            if use_body:
                c.m1_apply(O.collider(**b.as_tuple()), sc.dt)
            c.g2p(sc.dt)
        return c.state_f64()

    s = bm.MPMSolver(sc.dx, domain=sc.domain)
    s.set_material(sc.E, sc.nu, sc.rho)
    s.set_plastic_alpha(sc.alpha)
    s.add_particles(st0["position"], st0["velocity"], sc.mass)
    s.set_particles(0, F=st0["F"], C_=st0["C"])
    tape = bm.Tape(s, 2)
    tape.forward(sc.dt, steps, bm.make_collider(**body.as_tuple()) if use_body else None,
                 wp if use_body else None)
    worst = 0.0
    for lf, wl in FIELDS.items():
        cvec = rng.normal(size=(n, wl))
        g = tape.backward_state({lf: cvec.astype(np.float32)})
        for inf, wi in FIELDS.items():
            if lf == "position" and inf == "F":
                # x1 = x0 + v1 dt here (no floor clamp): this pair is dt times
                # the (velocity, F) pair, and its difference (~1e-12) sits at
                # the double-rounding floor of the summed positions
                continue
            d = rng.normal(size=(n, wi))
            base = st0[inf].reshape(n, wi).astype(np.float64)
            hi = {k: v.astype(np.float64) for k, v in st0.items()}
            lo = dict(hi)
            hi[inf] = (base + FD_EPS[inf] * d).reshape(st0[inf].shape)
            lo[inf] = (base - FD_EPS[inf] * d).reshape(st0[inf].shape)
            fd = float(np.sum(cvec * oracle_state(hi)[lf].reshape(n, wl)) -
                       np.sum(cvec * oracle_state(lo)[lf].reshape(n, wl)))
            pred = float(np.sum(g[inf].reshape(n, wi).astype(np.float64) * d)) * 2 * FD_EPS[inf]
            rel = abs(pred - fd) / abs(fd)
            worst = max(worst, rel)
            print(f"L on {lf:8s} d/d {inf:8s}: adjoint {pred:+.6e} fd {fd:+.6e} rel {rel:.1e}")
    assert worst < ADJ_REL_TOL


def test_full_tine_pass_waypoint_gradient_matches_fp64_finite_differences(fdpool):
    """The full differentiable workload: 262,144 particles on the 64^3 grid,
    200 steps at dt = 1e-4, 16 waypoints, checkpoints every 20 steps. The
    adjoint's dL/d waypoint on 8 seeded coordinates against FP64 central
    differences at eps = 1e-6 with the decisions frozen on both sides (left
    free, such a difference takes the jumps of the hundreds of SVD decisions
    a 1e-6 change flips in this run). The decisions are those of the float
    restatement's run, the branch an FP32 forward (and so the adjoint)
    follows. Bar: ADJ_REL_TOL_FULL on the gradient's norm; each coordinate's
    error is printed."""
    sc, body, wp, target = scenes.tine_pass()
    s, tape = run_tape(sc, body, wp, sc.steps, 20)
    L, g = scenes.heightfield_loss(s.get_particles()["position"], target)
    gw = tape.backward(g)["dL_dwaypoints"]
    rng = np.random.default_rng(11)
    ks = rng.choice(np.arange(1, 15), 8, replace=False)
    coords = [(int(k), int(rng.integers(0, 3))) for k in ks]
    fd, consistent = fd_util.fd_waypoints_frozen(fdpool, sc, body, wp, sc.steps, target, coords, eps=1e-6,
                                                 branch="f32")
    assert consistent
    assert check_waypoint_gradient(gw, fd, coords, "full tine pass") < ADJ_REL_TOL_FULL
