"""The reference's rigid-coupling research bench on the CUDA solver.

research/mpm_rigid_coupling/bench_compare_all.cpp runs grid-only scenes (a
rigid body dropped, stamped, dragged or rolled on a patch of seeded grid
nodes, no particles) through each coupler and writes time series, run
metrics and per-scene summaries that scripts/reproduce_findings.py checks.
This module holds the same pieces for the CUDA couplers:

* ``SCENES``: the scenario registry (scenarios/scenario_*.h constants,
  bench_compare_all.cpp:797-804);
* ``run``: the harness loop in float32 — gravity on the body, the coupler,
  the reference's semi-implicit Euler (integrator.h:20-45, damping 0,
  body-space inverse inertia = identity as the scenarios leave it), grid
  gravity and floor clamp (bench_compare_all.cpp:72-208, 215-292, 374-800);
* ``RunMetrics``: metrics.h:19-94 (max and mean |sum p_y|, energy drift,
  penetration and dwell);
* ``write_*``: the CSV files of frame_exporter.h:30-44 and of the bench's
  metrics, summary, roll and rebound writers, same names and formats;
* ``findings``: the predicates of scripts/reproduce_findings.py:58-122.

``python -m basements_b200.research --out DIR`` runs every scene with every
coupler (M0, M1, M4.5a, M4.5b, M4.5) and prints the findings. The grid
stays on the device; each step reads it back to apply the host-side grid
gravity and floor the bench applies, so the loop is a parity harness, not a
throughput path.
"""
from __future__ import annotations

import argparse
import math
import os
import sys
import time

import numpy as np

f32 = np.float32

# method names of the reference's bench -> coupler name of this package
METHODS = {"M0": "m0", "M1": "m1", "M4.5a": "m45a", "M4.5b": "m45b", "M4.5": "m45c"}


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
    # scenario_box_drop.h with box_mass = 9 (bench_compare_all.cpp:505-613)
    "box_drop_dense": dict(dx=0.1, seed_lo=(-3, 0, -3), seed_hi=(3, 2, 3), node_mass=0.01,
                           domain=((-8, -4, -8), (16, 16, 16)), center=(0.0, 0.55, 0.0),
                           half=(0.2, 0.2, 0.2), q=(1.0, 0.0, 0.0, 0.0), vel=(0, 0, 0), omg=(0, 0, 0),
                           friction=0.5, mass=9.0, shape=0, steps=720, kinematic=False),
    # scenario_foot_step.h: a thin dynamic box stamped onto a 7x3x7 patch (:374-504)
    "foot_step": dict(dx=0.1, seed_lo=(-3, 0, -3), seed_hi=(3, 2, 3), node_mass=0.01,
                      domain=((-8, -4, -8), (16, 16, 16)), center=(0.0, 0.55, 0.0),
                      half=(0.10, 0.02, 0.10), q=(1.0, 0.0, 0.0, 0.0), vel=(0, 0, 0), omg=(0, 0, 0),
                      friction=0.5, mass=1.0, shape=0, steps=480, kinematic=False),
    # benchmarks/bench_mpm_rigid_drift.cpp:37-69: the unit box over a 5x3x5 patch
    "rigid_drift": dict(dx=0.1, seed_lo=(-2, 0, -2), seed_hi=(2, 2, 2), node_mass=0.01,
                        domain=((-8, -4, -8), (16, 16, 16)), center=(0.0, 0.55, 0.0),
                        half=(0.2, 0.2, 0.2), q=(1.0, 0.0, 0.0, 0.0), vel=(0, 0, 0), omg=(0, 0, 0),
                        friction=0.5, mass=1.0, shape=0, steps=720, kinematic=False),
    # scenario_tine_drag.h: surface_y = (4 - 1 + 0.5) dx, tip 6 cm below it (:215-292)
    "tine_drag": dict(dx=0.05, seed_lo=(-2, 0, -3), seed_hi=(10, 3, 3), node_mass=0.1875,
                      domain=((-8, -4, -8), (24, 16, 16)), center=None, half=(0.005, 0.05, 0.04),
                      q=(1.0, 0.0, 0.0, 0.0), vel=(0.2, 0, 0), omg=(0, 0, 0), friction=0.55, mass=0.5,
                      shape=0, steps=480, kinematic=True),
    # scenario_rover_wheel.h, ROLL mode: cylinder about world z after a 90 deg
    # turn about x (:614-800)
    "rover_wheel": dict(dx=0.1, seed_lo=(-6, 0, -4), seed_hi=(6, 2, 4), node_mass=0.01,
                        domain=((-16, -12, -12), (32, 24, 24)), center=(0.0, 0.55, 0.0),
                        half=(0.15, 0.05, 0.15), q=_axis_angle_x(1.5707963), vel=(0, 0, 0),
                        omg=(0, 0, -10.0), friction=0.5, mass=1.0, shape=1, steps=720, kinematic=False),
}


def tine_start(dx=0.05):
    surface = f32(f32(f32(4 - 1) + f32(0.5)) * f32(dx))
    return (f32(-0.05), f32(f32(surface - f32(0.06)) + f32(0.05)), f32(0.0))


class GpuGrid:
    """A scene's seeded grid on the CUDA solver with one coupler ("m0",
    "m1", "m45a", "m45b" or "m45c")."""

    def __init__(self, bm, sc, coupler="m1"):
        self.bm = bm
        self.coupler = coupler
        self.s = bm.MPMSolver(sc["dx"], domain=sc["domain"])
        ijk = _seed_block(sc["seed_lo"], sc["seed_hi"])
        self.s.seed_grid(ijk, np.zeros((len(ijk), 3), np.float32), np.full(len(ijk), sc["node_mass"], np.float32))

    def apply(self, body, dt):
        return getattr(self.s, f"{self.coupler}_apply")(self.bm.make_collider(**body), float(dt))

    def gravity_floor(self, g, dt):
        """Grid gravity and the floor clamp on every node with mass (the
        bench's post-coupler loop); returns the nodes with mass after it:
        (ijk, velocity, mass)."""
        grid = self.s.get_grid()
        v = grid["velocity"].copy()
        act = grid["mass"] > 0
        vy = v[..., 1]
        vy[act] = vy[act] + f32(-g * dt)
        vy[act & (vy < 0)] = 0
        self.s.set_grid_velocity(v)
        idx = np.argwhere(act)
        return (idx + np.asarray(grid["origin"])).astype(np.int32), v[act], grid["mass"][act]


class RunMetrics:
    """metrics.h:19-94 in float32: per step |sum p_y|, the energy drift
    against the first step, the deepest node inside the body's box and the
    steps whose depth exceeds 0.3 of the smallest half extent."""

    def __init__(self):
        self.max_abs_p = f32(0)
        self.sum_abs_p = f32(0)
        self.max_drift = f32(0)
        self.e0 = None
        self.max_pen = f32(0)
        self.sum_pen = f32(0)
        self.dwell = 0
        self.steps = 0
        self.time_us = 0.0

    def observe(self, total_p_y, e_total, pen, min_half, step_us):
        e_total = f32(e_total)
        if self.e0 is None:
            self.e0 = e_total
        d = f32(abs(e_total - self.e0))
        drift = f32(d / abs(self.e0)) if abs(self.e0) > f32(1e-9) else d
        ap = f32(abs(f32(total_p_y)))
        self.max_abs_p = max(self.max_abs_p, ap)
        self.sum_abs_p = f32(self.sum_abs_p + ap)
        self.max_drift = max(self.max_drift, drift)
        self.max_pen = max(self.max_pen, f32(pen))
        self.sum_pen = f32(self.sum_pen + f32(pen))
        if f32(pen) > f32(f32(min_half) * f32(0.30)):
            self.dwell += 1
        self.time_us += step_us
        self.steps += 1

    def values(self):
        n = max(self.steps, 1)
        return dict(max_abs_total_p_y=float(self.max_abs_p), avg_abs_total_p_y=float(self.sum_abs_p) / n,
                    max_abs_energy_drift=float(self.max_drift), step_time_avg_us=self.time_us / n,
                    max_penetration_m=float(self.max_pen), avg_penetration_m=float(self.sum_pen) / n,
                    dwell_fraction=self.dwell / n, ratio_p_y_vs_M0=1.0)


def _rotation(q):
    w, x, y, z = (float(c) for c in q)
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


def penetration(ijk, mass, dx, center, q, half):
    """measure_penetration (metrics.h:96-127): the deepest node with mass
    inside the body's box, depth = the smallest distance to a face."""
    if len(ijk) == 0:
        return 0.0
    xn = (ijk.astype(np.float64) + 0.5) * dx
    local = (xn - np.asarray(center, np.float64)) @ _rotation(q)
    d = np.asarray(half, np.float64) - np.abs(local)
    ok = (d >= 0).all(axis=1) & (mass > 0)
    return float(d[ok].min(axis=1).max()) if ok.any() else 0.0


def run(name, grid, steps=None, record=None):
    """Runs one scene; returns per-step rows.

    dynamic scenes: [t, x, y, z, vy, p_body_y, p_grid_y, p_sum_y, KE, nodes_inside]
    (the columns of FrameExporter::log_step); tine_drag: [t, tine_x, fx, fy, fz].
    ``record`` (a dict, optional) gets "metrics" (RunMetrics values), and for
    rover_wheel the roll averages, for foot_step the rebound peaks, for
    tine_drag the draft summary.
    """
    sc = SCENES[name]
    dt, g, m = f32(1.0 / 240.0), f32(9.81), f32(sc["mass"])
    inv_m = f32(f32(1) / m)
    pos = np.array(tine_start(sc["dx"]) if sc["kinematic"] else sc["center"], np.float32)
    vel = np.array(sc["vel"], np.float32)
    omg = np.array(sc["omg"], np.float32)
    q = tuple(f32(c) for c in sc["q"])
    n_steps = sc["steps"] if steps is None else steps
    metrics = RunMetrics()
    roll = [0.0, 0.0, 0.0, 0]
    rows = []
    for i in range(n_steps):
        t0 = time.perf_counter()
        t = f32(f32(i + 1) * dt)
        if sc["kinematic"]:
            pos[0] = f32(pos[0] + f32(vel[0] * dt))
        q_step = q
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
        ijk, gv, gm = grid.gravity_floor(g, dt)
        pg = float((gv[:, 1].astype(np.float64) * gm).sum())
        pb = float(vel[1] * m)
        ke = 0.5 * float(m) * float((vel.astype(np.float64) ** 2).sum())
        rows.append([t, pos[0], pos[1], pos[2], vel[1], pb, pg, pb + pg, ke, n])
        if record is not None:
            # the bench's energy and penetration use the pose after the
            # update and the orientation the coupler saw (its collider copy)
            e_total = ke + float(m) * float(g) * float(pos[1]) + 0.5 * float(
                (gm.astype(np.float64) * (gv.astype(np.float64) ** 2).sum(1)).sum())
            pen = penetration(ijk, gm, sc["dx"], pos, q_step, sc["half"])
            metrics.observe(pb + pg, e_total, pen, min(sc["half"]), (time.perf_counter() - t0) * 1e6)
            if name == "rover_wheel" and t > f32(3.0 - 1.0):
                R = sc["half"][0]
                tip = abs(float(omg[2])) * R
                roll[0] += 0.0 if tip < 1e-6 else 1.0 - float(vel[0]) / tip
                roll[1] += float(fr[0])
                surface = (3 - 1 + 0.5) * sc["dx"]
                roll[2] += min(max(0.0, (surface + R) - float(pos[1])), 2.0 * R)
                roll[3] += 1
    rows = np.array(rows, np.float64)
    if record is not None:
        if sc["kinematic"]:
            fx, fy, n = tine_summary(rows)
            record["summary"] = dict(avg_draft_fx_n=fx, avg_vertical_fy_n=fy,
                                     specific_draught_n_per_m=fx / (2 * sc["half"][2]), samples=n)
        else:
            record["metrics"] = metrics.values()
        if name == "rover_wheel":
            k = max(roll[3], 1)
            W, b, L = 1.0 * 9.81, 2 * 0.05, 2 * 0.15
            bekker = (W / (b * L) / (0.99e3 / b + 1528e3)) ** (1.0 / 1.1)
            sink = roll[2] / k
            record["roll"] = dict(avg_slip=roll[0] / k, avg_drawbar_N=roll[1] / k, avg_sinkage_m=sink,
                                  bekker_sinkage_m=bekker, sinkage_ratio_meas_over_bekker=sink / bekker)
        if name == "foot_step":
            down, up = rebound(rows)
            e = 0.0 if down >= 0 else min(max(up / -down, 0.0), 2.0)
            record["rebound"] = dict(v_down_peak=down, v_up_peak=up, rebound_coefficient_e=e)
    return rows


def tine_summary(rows, start=0.5):
    """Average draft -Fx and vertical Fy over t > start (bench_compare_all.cpp:259-275)."""
    sel = rows[:, 0].astype(np.float32) > f32(start)
    return float(-rows[sel, 2].mean()), float(rows[sel, 3].mean()), int(sel.sum())


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


# ---- CSV writers (the reference bench's file names and formats) -------------

def write_series(path, name, rows):
    with open(path, "w") as f:
        if name == "tine_drag":
            f.write("t,tine_x,reaction_fx,reaction_fy,reaction_fz\n")
            for r in rows[::4]:  # the bench logs every 4th step
                f.write("%.4f,%.6e,%.6e,%.6e,%.6e\n" % tuple(r))
            return
        f.write("t,box_x,box_y,box_z,box_vy,p_body_y,p_grid_y,p_sum_y,KE,nodes_inside\n")
        for r in rows:
            f.write("%.6f,%.6e,%.6e,%.6e,%.6e,%.8e,%.8e,%.8e,%.6e,%d\n" % (*r[:9], int(r[9])))


def write_record(out, name, method, record):
    """The metrics / summary / roll / rebound files of one run."""
    base = os.path.join(out, f"{name}_{method}")
    if "metrics" in record:
        v = record["metrics"]
        with open(base + "_metrics.csv", "w") as f:
            f.write("method,max_abs_total_p_y,avg_abs_total_p_y,max_abs_energy_drift,step_time_avg_us,"
                    "max_penetration_m,avg_penetration_m,dwell_fraction,ratio_p_y_vs_M0\n")
            f.write("%s,%.6e,%.6e,%.6e,%.3f,%.6e,%.6e,%.4f,%.6f\n" % (
                method, v["max_abs_total_p_y"], v["avg_abs_total_p_y"], v["max_abs_energy_drift"],
                v["step_time_avg_us"], v["max_penetration_m"], v["avg_penetration_m"], v["dwell_fraction"],
                v["ratio_p_y_vs_M0"]))
    if "summary" in record:
        v = record["summary"]
        with open(base + "_summary.csv", "w") as f:
            f.write("method,avg_draft_fx_n,avg_vertical_fy_n,specific_draught_n_per_m,samples\n")
            f.write("%s,%.6e,%.6e,%.6e,%d\n" % (method, v["avg_draft_fx_n"], v["avg_vertical_fy_n"],
                                              v["specific_draught_n_per_m"], v["samples"]))
    if "roll" in record:
        v = record["roll"]
        with open(base + "_roll.csv", "w") as f:
            f.write("method,avg_slip,avg_drawbar_N,avg_sinkage_m,bekker_sinkage_m,sinkage_ratio_meas_over_bekker\n")
            f.write("%s,%.6f,%.6e,%.6e,%.6e,%.6e\n" % (method, v["avg_slip"], v["avg_drawbar_N"], v["avg_sinkage_m"],
                                                    v["bekker_sinkage_m"], v["sinkage_ratio_meas_over_bekker"]))
    if "rebound" in record:
        v = record["rebound"]
        with open(base + "_rebound.csv", "w") as f:
            f.write("method,v_down_peak,v_up_peak,rebound_coefficient_e\n")
            f.write("%s,%.6e,%.6e,%.6f\n" % (method, v["v_down_peak"], v["v_up_peak"], v["rebound_coefficient_e"]))


def run_all(out, grid_factory, methods=tuple(METHODS), scenes=("box_drop", "box_drop_dense", "foot_step",
                                                                   "tine_drag", "rover_wheel")):
    """Every scene with every method; CSVs into ``out``. ``grid_factory(sc,
    coupler)`` makes the grid adapter (``GpuGrid`` for the CUDA couplers)."""
    os.makedirs(out, exist_ok=True)
    for method in methods:
        for name in scenes:
            record = {}
            rows = run(name, grid_factory(SCENES[name], METHODS[method]), record=record)
            write_series(os.path.join(out, f"{name}_{method}.csv"), name, rows)
            write_record(out, name, method, record)


# ---- findings (scripts/reproduce_findings.py:58-122) -------------------------

def _read(out, scene, method, kind, key):
    with open(os.path.join(out, f"{scene}_{method}_{kind}.csv")) as f:
        names, vals = [line.strip().split(",") for line in f][:2]
    return float(vals[names.index(key)])


def findings(out):
    """(name, ok, message) for each of the reference's five findings."""
    res = []
    m = lambda s, meth: _read(out, s, meth, "metrics", "max_abs_total_p_y")  # noqa: E731
    r = m("box_drop", "M4.5a") / m("box_drop", "M1")
    res.append(("Finding 1   M4.5a beats M1 (box_drop)", r < 0.60, f"box_drop M4.5a/M1 = {r:.3f} (target < 0.60)"))
    r = m("box_drop_dense", "M4.5a") / m("box_drop_dense", "M1")
    res.append(("Finding 1   Mass-invariance (box_drop_dense)", r < 0.60,
                f"box_drop_dense M4.5a/M1 = {r:.3f} (target < 0.60)"))
    sa = _read(out, "rover_wheel", "M4.5a", "roll", "avg_sinkage_m")
    sb = _read(out, "rover_wheel", "M4.5b", "roll", "avg_sinkage_m")
    la = _read(out, "rover_wheel", "M4.5a", "roll", "avg_slip")
    lb = _read(out, "rover_wheel", "M4.5b", "roll", "avg_slip")
    res.append(("Finding 2   Rover-wheel layer trade-off", sa < sb and lb < la,
                f"M4.5a sinkage {sa:.3f} < M4.5b {sb:.3f}; M4.5b slip {lb:.2f} < M4.5a {la:.2f}"))
    fct = m("box_drop_dense", "M0") / m("box_drop", "M0")
    res.append(("Finding 3   M0 degrades with mass", fct > 10.0, f"M0 dense/light = {fct:.1f}x (target > 10x)"))
    pa, pb, pc = m("box_drop", "M4.5a"), m("box_drop", "M4.5b"), m("box_drop", "M4.5")
    res.append(("Finding 4   Composition is not free", pb > pa and pc > 10.0 * pa,
                f"M4.5b {pb:.3e} > M4.5a {pa:.3e}; M4.5 {pc:.3e} > 10 M4.5a"))
    es = {meth: _read(out, "foot_step", meth, "rebound", "rebound_coefficient_e")
          for meth in ("M0", "M1", "M4.5a", "M4.5b", "M4.5")}
    res.append(("Finding 5   No rebound in dry sand", all(e < 0.05 for e in es.values()),
                f"foot_step rebound e by method: {es}"))
    return res


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--out", required=True, help="directory for the CSV files")
    a = ap.parse_args(argv)
    import basements_b200 as bm
    run_all(a.out, lambda sc, coupler: GpuGrid(bm, sc, coupler))
    ok_all = True
    for name, ok, msg in findings(a.out):
        ok_all = ok_all and ok
        print(f"{'PASS' if ok else 'FAIL'}  {name}: {msg}")
    return 0 if ok_all else 1


if __name__ == "__main__":
    sys.exit(main())
