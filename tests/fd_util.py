"""FP64 finite differences of the tine-pass loss on the CPU oracle
(TEST INFRASTRUCTURE: runs the oracle's split step P2G -> update_grid ->
M1 -> G2P in double, the FP64 path that the adjoint is checked against).

Forwards run in a process pool started with the `spawn` method."""
from __future__ import annotations

import multiprocessing as mp
import os

import numpy as np

from basements_b200 import scenes


def oracle_run(kind, sc, body, waypoints, steps, x0=None):
    """Final positions (double) of `steps` split steps of the oracle with the
    body on the waypoint path (x0 replaces the initial positions when given)."""
    from oracle import oracle as O

    c = O.CpuSolver(kind, sc.dx)
    c.set_material(sc.E, sc.nu, sc.rho)
    c.set_plastic_alpha(sc.alpha)
    c.add_particles(sc.position if x0 is None else x0, None, sc.mass)
    for n in range(steps):
        b = scenes.body_on_path(body, waypoints, steps, sc.dt, n)
        c.p2g(sc.dt)
        c.grid_update(sc.dt)
        c.m1_apply(O.collider(**b.as_tuple()), sc.dt)
        c.g2p(sc.dt)
    pos = c.positions_f64()
    c.close()
    return pos


def _loss_job(args):
    kind, sc, body, waypoints, steps, target, x0 = args
    return scenes.heightfield_loss(oracle_run(kind, sc, body, waypoints, steps, x0), target)[0]


def _frozen_job(args):
    """One central difference on a fixed branch: the base run records its
    SVD and coupler-inside decisions, the two perturbed runs replay them.
    Returns (dL, step taken, replays consistent)."""
    from oracle import oracle as O

    sc, body, wp, steps, target, k, a, eps, branch = args
    tape = O.DecisionTape("f64")

    def loss(w, mode, kind="f64", t=tape):
        c = O.CpuSolver(kind, sc.dx)
        c.set_material(sc.E, sc.nu, sc.rho)
        c.set_plastic_alpha(sc.alpha)
        c.add_particles(sc.position, None, sc.mass)
        c.use_tape(t, mode)
        for n in range(steps):
            b = scenes.body_on_path(body, w, steps, sc.dt, n)
            c.p2g(sc.dt)
            c.grid_update(sc.dt)
            c.m1_apply(O.collider(**b.as_tuple()), sc.dt)
            c.g2p(sc.dt)
        pos = c.positions_f64()
        c.close()
        return scenes.heightfield_loss(pos, target)[0]

    if branch == "f32":
        # the branch of the float restatement's run (the decisions an FP32
        # forward takes), replayed by the double runs
        t32 = O.DecisionTape("f32")
        loss(wp, "record", "f32", t32)
        tape.load(*t32.export())
        t32.close()
    else:
        loss(wp, "record")
    hi, lo = wp.copy(), wp.copy()
    hi[k, a] = np.float32(float(wp[k, a]) + eps)
    lo[k, a] = np.float32(float(wp[k, a]) - eps)
    consistent = True
    Lh = loss(hi, "replay")
    st = tape.status()
    consistent = consistent and st[0] == st[1] and st[2] == st[3] and not st[4]
    Ll = loss(lo, "replay")
    st = tape.status()
    consistent = consistent and st[0] == st[1] and st[2] == st[3] and not st[4]
    tape.close()
    return Lh - Ll, float(hi[k, a]) - float(lo[k, a]), consistent


def fd_waypoints_frozen(p, sc, body, wp, steps, target, coords, eps=1e-6, branch="f64"):
    """Central differences dL/d waypoint[k, a] of the FP64 run with its
    discontinuous decisions frozen: both sides replay the SVD pair-skip and
    sweep-stop decisions and the coupler's inside sets of the unperturbed run
    (oracle DecisionTape), so that the difference is a derivative of one
    branch of the algorithm, the branch an adjoint differentiates. (Left
    free, a 1e-6 change of one waypoint flips hundreds of SVD decisions of
    the 262k-particle tine pass, each adding its jump / 2 eps.) Returns the
    differences and whether every replay consumed exactly the record.
    branch="f32" takes the decisions from a run of the float restatement
    instead (both sides still computed in double): the branch an FP32 forward
    follows."""
    res = p.map(_frozen_job, [(sc, body, wp, steps, target, k, a, eps, branch) for k, a in coords])
    return np.array([d / st for d, st, _ in res]), all(ok for _, _, ok in res)


def pool(n=None):
    return mp.get_context("spawn").Pool(n or min(16, os.cpu_count() or 1))


def fd_waypoints(p, sc, body, wp, steps, target, coords, eps=1e-4, kind="f64"):
    """Central differences dL/d waypoint[k, a] for (k, a) in coords; the step
    actually taken is measured after rounding the waypoints to float32."""
    jobs, steps_taken = [], []
    for k, a in coords:
        hi, lo = wp.copy(), wp.copy()
        hi[k, a] = np.float32(float(wp[k, a]) + eps)
        lo[k, a] = np.float32(float(wp[k, a]) - eps)
        steps_taken.append(float(hi[k, a]) - float(lo[k, a]))
        jobs += [(kind, sc, body, hi, steps, target, None), (kind, sc, body, lo, steps, target, None)]
    L = p.map(_loss_job, jobs)
    return np.array([(L[2 * i] - L[2 * i + 1]) / steps_taken[i] for i in range(len(coords))])


def fd_direction_x0(p, sc, body, wp, steps, target, delta, eps, kind="f64"):
    """L(x0 + eps delta) - L(x0 - eps delta) and the float32 positions used,
    so the caller can form the predicted change sum g . (x+ - x-)."""
    x0 = sc.position.astype(np.float64)
    hi = (x0 + eps * delta).astype(np.float32)
    lo = (x0 - eps * delta).astype(np.float32)
    Lh, Ll = p.map(_loss_job, [(kind, sc, body, wp, steps, target, hi), (kind, sc, body, wp, steps, target, lo)])
    return Lh - Ll, hi, lo
