"""The reference's grid-only research scenes, as a harness loop around a
coupler (M0, M1 or M4.5a) of the CUDA solver or of the oracle.

The loop restates research/mpm_rigid_coupling/bench_compare_all.cpp in float32:

* foot_step (:374-504), box_drop_dense (:505-613) and rover_wheel (:614-800):
  a dynamic body; each
  step applies gravity to the body, calls the coupler, adds its reaction,
  integrates with the reference's semi-implicit Euler
  (include/basements/physics/dynamics/integrator.h:20-45, damping 0 as the
  scenarios set it, body-space inverse inertia = identity as make_box /
  make_wheel leave it), then adds grid gravity and the floor clamp to every
  node with mass;
* tine_drag (:215-292): a kinematic box moved by v*dt before each call; the
  reaction is only measured;
* rigid_drift: benchmarks/bench_mpm_rigid_drift.cpp --method pic (:24-178),
  the same dynamic loop over a smaller patch.

Scenario constants follow research/mpm_rigid_coupling/scenarios/
scenario_box_drop.h, scenario_foot_step.h, scenario_tine_drag.h and
scenario_rover_wheel.h.
"""
from __future__ import annotations

import math

import numpy as np

f32 = np.float32


def _seed_block(lo, hi):
    return np.array([(i, j, k) for i in range(lo[0], hi[0] + 1) for j in range(lo[1], hi[1] + 1)
                     for k in range(lo[2], hi[2] + 1)], np.int32)


def _quat_mul(a, b):
    """Hamilton product in float32, summed left to right (quaternion.h:151-158)."""
    f = f32
    aw, ax, ay, az = a
    bw, bx, by, bz = b
    return (f(f(f(aw * bw) - f(ax * bx)) - f(ay * by)) - f(az * bz),
            f(f(f(aw * bx) + f(ax * bw)) + f(ay * bz)) - f(az * by),
            f(f(f(aw * by) - f(ax * bz)) + f(ay * bw)) + f(az * bx),
            f(f(f(aw * bz) + f(ax * by)) - f(ay * bx)) + f(az * bw))


def _axis_angle_x(angle):
    """Quaternion::from_axis_angle((1,0,0), angle) (quaternion.h:36-46)."""
    h = f32(f32(angle) * f32(0.5))
    return (f32(math.cos(float(h))), f32(math.sin(float(h))), f32(0), f32(0))


SCENES = {
    # scenario_box_drop.h (bench_compare_all.cpp:72-208)
    "box_drop": dict(dx=0.1, seed_lo=(-3, 0, -3), seed_hi=(3, 2, 3), node_mass=0.01,
                     domain=((-8, -4, -8), (16, 16, 16)), center=(0.0, 0.55, 0.0),
                     half=(0.2, 0.2, 0.2), q=(1.0, 0.0, 0.0, 0.0), vel=(0, 0, 0), omg=(0, 0, 0),
                     friction=0.5, mass=1.0, shape=0, steps=720, kinematic=False),
    # scenario_box_drop.h with box_mass = 9 (bench_compare_all.cpp:507)
    "box_drop_dense": dict(dx=0.1, seed_lo=(-3, 0, -3), seed_hi=(3, 2, 3), node_mass=0.01,
                           domain=((-8, -4, -8), (16, 16, 16)), center=(0.0, 0.55, 0.0),
                           half=(0.2, 0.2, 0.2), q=(1.0, 0.0, 0.0, 0.0), vel=(0, 0, 0), omg=(0, 0, 0),
                           friction=0.5, mass=9.0, shape=0, steps=720, kinematic=False),
    # scenario_foot_step.h: a thin dynamic box stamped onto a 7x3x7 patch
    "foot_step": dict(dx=0.1, seed_lo=(-3, 0, -3), seed_hi=(3, 2, 3), node_mass=0.01,
                      domain=((-8, -4, -8), (16, 16, 16)), center=(0.0, 0.55, 0.0),
                      half=(0.10, 0.02, 0.10), q=(1.0, 0.0, 0.0, 0.0), vel=(0, 0, 0), omg=(0, 0, 0),
                      friction=0.5, mass=1.0, shape=0, steps=480, kinematic=False),
    # benchmarks/bench_mpm_rigid_drift.cpp:37-69: the unit box over a 5x3x5 patch
    "rigid_drift": dict(dx=0.1, seed_lo=(-2, 0, -2), seed_hi=(2, 2, 2), node_mass=0.01,
                        domain=((-8, -4, -8), (16, 16, 16)), center=(0.0, 0.55, 0.0),
                        half=(0.2, 0.2, 0.2), q=(1.0, 0.0, 0.0, 0.0), vel=(0, 0, 0), omg=(0, 0, 0),
                        friction=0.5, mass=1.0, shape=0, steps=720, kinematic=False),
    # scenario_tine_drag.h: surface_y = (4 - 1 + 0.5) dx, tip 6 cm below it
    "tine_drag": dict(dx=0.05, seed_lo=(-2, 0, -3), seed_hi=(10, 3, 3), node_mass=0.1875,
                      domain=((-8, -4, -8), (24, 16, 16)), center=None, half=(0.005, 0.05, 0.04),
                      q=(1.0, 0.0, 0.0, 0.0), vel=(0.2, 0, 0), omg=(0, 0, 0), friction=0.55, mass=0.5,
                      shape=0, steps=480, kinematic=True),
    # scenario_rover_wheel.h, ROLL mode: cylinder about world z after a 90 deg turn about x
    "rover_wheel": dict(dx=0.1, seed_lo=(-6, 0, -4), seed_hi=(6, 2, 4), node_mass=0.01,
                        domain=((-16, -12, -12), (32, 24, 24)), center=(0.0, 0.55, 0.0),
                        half=(0.15, 0.05, 0.15), q=_axis_angle_x(1.5707963), vel=(0, 0, 0),
                        omg=(0, 0, -10.0), friction=0.5, mass=1.0, shape=1, steps=720, kinematic=False),
}


def tine_start(dx=0.05):
    surface = f32(f32(f32(4 - 1) + f32(0.5)) * f32(dx))
    return (f32(-0.05), f32(f32(surface - f32(0.06)) + f32(0.05)), f32(0.0))


class GpuGrid:
    """The CUDA solver's grid (bm.MPMSolver) behind the loop; coupler "m0",
    "m1" or "m45a"."""

    def __init__(self, bm, sc, coupler="m1"):
        self.bm = bm
        self.coupler = coupler
        self.s = bm.MPMSolver(sc["dx"], domain=sc["domain"])
        ijk = _seed_block(sc["seed_lo"], sc["seed_hi"])
        self.s.seed_grid(ijk, np.zeros((len(ijk), 3), np.float32), np.full(len(ijk), sc["node_mass"], np.float32))

    def apply(self, body, dt):
        return getattr(self.s, f"{self.coupler}_apply")(self.bm.make_collider(**body), float(dt))

    def gravity_floor(self, g, dt):
        grid = self.s.get_grid()
        v = grid["velocity"].copy()
        act = grid["mass"] > 0
        vy = v[..., 1]
        vy[act] = vy[act] + f32(-g * dt)
        vy[act & (vy < 0)] = 0
        self.s.set_grid_velocity(v)
        return float((v[act][:, 1].astype(np.float64) * grid["mass"][act]).sum())


class OracleGrid:
    """The oracle's grid (oracle.CpuSolver, reference build or port) behind the loop."""

    def __init__(self, O, kind, sc, coupler="m1"):
        self.O = O
        self.coupler = coupler
        self.s = O.CpuSolver(kind, sc["dx"])
        ijk = _seed_block(sc["seed_lo"], sc["seed_hi"])
        self.s.grid_seed(ijk, np.zeros((len(ijk), 3), np.float32), np.full(len(ijk), sc["node_mass"], np.float32))

    def apply(self, body, dt):
        return getattr(self.s, f"{self.coupler}_apply")(self.O.collider(**body), float(dt))

    def gravity_floor(self, g, dt):
        n = self.s.grid_nodes()
        sel = (n["active"] > 0) & (n["mass"] > 0)
        v = n["velocity"][sel].copy()
        v[:, 1] = v[:, 1] + f32(-g * dt)
        v[v[:, 1] < 0, 1] = 0
        self.s.grid_seed(n["ijk"][sel], v, n["mass"][sel])
        return float((v[:, 1].astype(np.float64) * n["mass"][sel]).sum())


def run(name, grid, steps=None):
    """Runs one scene; returns per-step rows.

    dynamic scenes: [t, x, y, z, vy, p_body_y, p_grid_y, p_sum_y, KE, nodes_inside]
    (the columns of the reference's FrameExporter::log_step);
    tine_drag: [t, tine_x, fx, fy, fz].
    """
    sc = SCENES[name]
    dt, g, m = f32(1.0 / 240.0), f32(9.81), f32(sc["mass"])
    inv_m = f32(f32(1) / m)
    pos = np.array(tine_start(sc["dx"]) if sc["kinematic"] else sc["center"], np.float32)
    vel = np.array(sc["vel"], np.float32)
    omg = np.array(sc["omg"], np.float32)
    q = tuple(f32(c) for c in sc["q"])
    n_steps = sc["steps"] if steps is None else steps
    rows = []
    for i in range(n_steps):
        t = f32(f32(i + 1) * dt)
        if sc["kinematic"]:
            pos[0] = f32(pos[0] + f32(vel[0] * dt))
        body = dict(center=pos, half_extents=sc["half"], orientation=q, linear_velocity=vel,
                    angular_velocity=omg, friction=sc["friction"], mass=float(m), shape=sc["shape"])
        fr, tq, n = grid.apply(body, dt)
        if sc["kinematic"]:
            grid.gravity_floor(g, dt)
            rows.append([t, pos[0], fr[0], fr[1], fr[2]])
            continue
        force = (np.array([0, -g * m, 0], np.float32) + fr.astype(np.float32)).astype(np.float32)
        vel = (vel + (force * inv_m) * dt).astype(np.float32)
        omg = (omg + tq.astype(np.float32) * dt).astype(np.float32)
        pos = (pos + vel * dt).astype(np.float32)
        dq = _quat_mul((f32(0), omg[0], omg[1], omg[2]), q)
        h = f32(f32(0.5) * dt)
        q = tuple(f32(q[a] + f32(dq[a] * h)) for a in range(4))
        nrm = f32(np.sqrt(f32(f32(f32(q[0] * q[0]) + f32(q[1] * q[1])) + f32(q[2] * q[2])) + f32(q[3] * q[3])))
        q = tuple(f32(c * f32(f32(1) / nrm)) for c in q)
        pg = grid.gravity_floor(g, dt)
        pb = float(vel[1] * m)
        ke = 0.5 * float(m) * float((vel.astype(np.float64) ** 2).sum())
        rows.append([t, pos[0], pos[1], pos[2], vel[1], pb, pg, pb + pg, ke, n])
    return np.array(rows, np.float64)


def tine_summary(rows, start=0.5):
    """Average draft -Fx and vertical Fy over t > start (bench_compare_all.cpp:259-275)."""
    sel = rows[:, 0].astype(np.float32) > f32(start)
    return -rows[sel, 2].mean(), rows[sel, 3].mean(), int(sel.sum())


def rebound(rows, settle=0.05):
    """ReboundTracker (scenario_foot_step.h:84-113) over the body's v_y:
    returns (v_down_peak, v_up_peak)."""
    state, down, up = 0, f32(0), f32(0)
    for t, vy in zip(rows[:, 0].astype(np.float32), rows[:, 4].astype(np.float32)):
        if t < f32(settle):
            continue
        if state == 0:
            down = min(down, vy)
            if vy >= 0 and down < 0:
                state = 1
        if state == 1:
            up = max(up, vy)
            if vy <= 0 and up > 0:
                state = 2
    return float(down), float(up)


# rigid_drift CSV columns [t, box_y, box_vy, p_body_y, p_grid_y, p_sum_y, KE_box,
# nodes_inside] as columns of the dynamic rows above
DRIFT_COLUMNS = [0, 2, 4, 5, 6, 7, 8, 9]


def first_divergence(a, b, atol):
    """First row index where |a - b| > atol in any column, or None."""
    bad = np.nonzero((np.abs(a - b) > atol).any(axis=1))[0]
    return int(bad[0]) if len(bad) else None
