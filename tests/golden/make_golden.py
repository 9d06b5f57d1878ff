"""Generates the committed golden fixtures in tests/golden/.

Run in a container that holds the reference tree (2nugu/basements) and the
built reference harness (``make -C oracle``):

    python tests/golden/make_golden.py --ref-root <reference tree>

Every array is produced either by the reference's OWN code (oracle/_ref,
compiled from the reference headers) or read from the reference's shipped
research outputs (box_drop_M1.csv, and the M1 rows of box_drop_dense, tine_drag,
rover_wheel and foot_step, the M1 run of the rigid-drift benchmark, and the
repose-pile summary). Nothing here runs at test time; the tests
only read the .npz files, so they also run where the reference is absent.
"""
from __future__ import annotations

import argparse
import csv
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from basements_b200 import scenes  # noqa: E402


def box_drop_csv(ref_root: str):
    base = os.path.join(ref_root, "research/mpm_rigid_coupling/outputs/csv")
    with open(os.path.join(base, "box_drop_M1.csv")) as f:
        rows = list(csv.reader(f))
    cols = rows[0]
    data = np.array([[float(v) for v in r] for r in rows[1:]], np.float64)
    with open(os.path.join(base, "box_drop_M1_metrics.csv")) as f:
        m = list(csv.reader(f))
    metrics = {k: float(v) for k, v in zip(m[0][1:], m[1][1:])}
    return cols, data, metrics


def research_csv(ref_root: str, scene: str, summaries, method="M1"):
    """One scene's M1 time series and its summary rows, as the reference's
    research bench wrote them (research/mpm_rigid_coupling/bench_compare_all.cpp:
    tine_drag :215-292, foot_step :374-504, box_drop_dense :505-613,
    rover_wheel :614-800)."""
    base = os.path.join(ref_root, "research/mpm_rigid_coupling/outputs/csv")
    with open(os.path.join(base, f"{scene}_{method}.csv")) as f:
        rows = list(csv.reader(f))
    data = np.array([[float(v) for v in r] for r in rows[1:]], np.float64)
    names, values = [], []
    for summary in summaries:
        with open(os.path.join(base, f"{scene}_{method}_{summary}.csv")) as f:
            m = list(csv.reader(f))
        names += m[0][1:]
        values += [float(v) for v in m[1][1:]]
    return {f"{scene}_columns": np.array(rows[0]), f"{scene}_rows": data,
            f"{scene}_metric_names": np.array(names), f"{scene}_metric_values": np.array(values)}


def drift_dirichlet_csv(ref_root: str):
    """benchmarks/bench_mpm_rigid_drift.cpp (default --method dirichlet, M0):
    the same unit box drop; its shipped time series."""
    with open(os.path.join(ref_root, "outputs/figures/mpm_rigid_drift.csv")) as f:
        rows = list(csv.reader(f))
    return {"rigid_drift_columns": np.array(rows[0]),
            "rigid_drift_rows": np.array([[float(v) for v in r] for r in rows[1:]], np.float64)}


def drift_pic_csv(ref_root: str):
    """benchmarks/bench_mpm_rigid_drift.cpp --method pic (:24-178): a unit box
    dropped on a 5x3x5 grid patch through M1; its shipped time series."""
    with open(os.path.join(ref_root, "outputs/figures/mpm_rigid_drift_pic.csv")) as f:
        rows = list(csv.reader(f))
    return {"rigid_drift_columns": np.array(rows[0]),
            "rigid_drift_rows": np.array([[float(v) for v in r] for r in rows[1:]], np.float64)}


def repose_summary(ref_root: str):
    """research/mpm_rigid_coupling/outputs/csv/repose_pile_summary.csv
    (bench_compare_all.cpp:293-371): the settled pile of the particle run."""
    with open(os.path.join(ref_root, "research/mpm_rigid_coupling/outputs/csv/repose_pile_summary.csv")) as f:
        m = list(csv.reader(f))
    names = m[0][:-1]  # the last column is the literature range as text
    return {"metric_names": np.array(names), "metric_values": np.array([float(v) for v in m[1][:-1]])}


M1_SCENES = (("box_drop_dense", ("metrics",)), ("tine_drag", ("summary",)), ("rover_wheel", ("metrics", "roll")),
             ("foot_step", ("metrics", "rebound")))


def small_scene(seed=3, cells=(8, 4, 8), ppc=4):
    """A small sand block (1,024 particles) near the floor, dx = 1/32."""
    rng = np.random.RandomState(seed)
    dx = 1.0 / 32
    ci, cj, ck = cells
    idx = np.stack(np.meshgrid(np.arange(ci), np.arange(cj), np.arange(ck), indexing="ij"), -1).reshape(-1, 3)
    pos = ((idx[:, None, :] + np.array([4, 0, 4]) + rng.random_sample((len(idx), ppc, 3))) * dx)
    pos = pos.reshape(-1, 3).astype(np.float32)
    vel = (rng.standard_normal(pos.shape) * 0.05).astype(np.float32)
    m = np.full(len(pos), 1600.0 * dx ** 3 / ppc, np.float32)
    return dx, pos, vel, m


def run_small_scene():
    dx, pos, vel, m = small_scene()
    alpha = scenes.dp_alpha(30.0)
    s = O.CpuSolver("ref", dx)
    s.set_material(3.5e5, 0.3, 1600.0)
    s.set_plastic_alpha(alpha)
    s.add_particles(pos, vel, m)
    # phase snapshots of step 0
    s.p2g(1e-4)
    g_p2g = s.grid_nodes()
    s.grid_update(1e-4)
    g_upd = s.grid_nodes()
    s.g2p(1e-4)
    s.step(1e-4, 19)
    out = s.get_particles()
    return dict(dx=np.float32(dx), alpha=np.float32(alpha), pos0=pos, vel0=vel, mass=m,
                p2g_ijk=g_p2g["ijk"], p2g_vel=g_p2g["velocity"], p2g_force=g_p2g["force"], p2g_mass=g_p2g["mass"],
                upd_ijk=g_upd["ijk"], upd_vel=g_upd["velocity"], upd_mass=g_upd["mass"],
                pos20=out["position"], vel20=out["velocity"], F20=out["F"], C20=out["C"])


def m1_cases(n_cases=12, seed=7, coupler="m1_apply"):
    """Seeded grids (empty, tiny and normal node masses) and random box and
    cylinder poses, each through one call of the reference's coupler
    (MPMRigidCouplerPIC::apply; M4_5a/M4_5b/M4_5c::apply for coupler=
    "m45a_apply"/"m45b_apply"/"m45c_apply"; MPMRigidCoupler::apply, M0, for
    coupler="m0_apply")."""
    rng = np.random.RandomState(seed)
    out = {k: [] for k in ("dx", "seed_ijk", "seed_vel", "seed_mass", "body", "dt", "force", "torque",
                           "nodes_inside", "grid_ijk", "grid_vel", "grid_mass", "grid_active")}
    for c in range(n_cases):
        dx = float(rng.choice([0.05, 0.1, 1.0 / 32]))
        lo = rng.randint(-6, 2, size=3)
        ext = rng.randint(4, 10, size=3)
        ii = np.stack(np.meshgrid(*[np.arange(lo[a], lo[a] + ext[a]) for a in range(3)], indexing="ij"), -1)
        ijk = ii.reshape(-1, 3).astype(np.int32)
        keep = rng.random_sample(len(ijk)) < 0.8
        ijk = ijk[keep]
        mass = rng.choice([0.0, 1e-10, 1e-7, 0.01, 0.3], size=len(ijk), p=[0.05, 0.05, 0.1, 0.5, 0.3])
        mass = (mass * rng.uniform(0.5, 1.5, size=len(ijk))).astype(np.float32)
        vel = (rng.standard_normal((len(ijk), 3)) * 0.5).astype(np.float32)
        q = rng.standard_normal(4)
        q /= np.linalg.norm(q)
        centre = (lo + ext / 2.0 + rng.uniform(-1, 1, 3)) * dx
        shape = c % 2
        he = rng.uniform(1.0, 3.0, 3) * dx
        if shape == 1:
            he[2] = he[0]
        body = O.collider(centre, he, q, rng.standard_normal(3), rng.standard_normal(3) * 3, 0.5,
                          float(rng.uniform(0.1, 5.0)), shape)
        dt = float(rng.choice([1e-4, 5e-5, 1.0 / 240, 0.0]))
        s = O.CpuSolver("ref", dx)
        s.grid_seed(ijk, vel, mass)
        f, t, n = getattr(s, coupler)(body, dt)
        g = s.grid_nodes()
        out["dx"].append(dx)
        out["seed_ijk"].append(ijk)
        out["seed_vel"].append(vel)
        out["seed_mass"].append(mass)
        out["body"].append(np.array(list(body.center) + list(body.orientation) + list(body.half_extents) +
                                    list(body.linear_velocity) + list(body.angular_velocity) +
                                    [body.friction, body.mass, body.shape], np.float32))
        out["dt"].append(dt)
        out["force"].append(f)
        out["torque"].append(t)
        out["nodes_inside"].append(n)
        out["grid_ijk"].append(g["ijk"])
        out["grid_vel"].append(g["velocity"])
        out["grid_mass"].append(g["mass"])
        out["grid_active"].append(g["active"])
    flat = {}
    for k, v in out.items():
        if isinstance(v[0], np.ndarray) and v[0].ndim >= 1 and k not in ("body", "force", "torque"):
            flat[k + "_len"] = np.array([len(a) for a in v], np.int64)
            flat[k] = np.concatenate(v)
        else:
            flat[k] = np.array(v)
    return flat


def svd_cases(n=512, seed=11):
    rng = np.random.RandomState(seed)
    F = np.eye(3, dtype=np.float32)[None] + (rng.standard_normal((n, 3, 3)) * 0.3).astype(np.float32)
    F[: n // 8] = np.diag([1.5, 0.5, 1.5]).astype(np.float32)[None] + \
        (rng.standard_normal((n // 8, 3, 3)) * 1e-4).astype(np.float32)
    F[n // 8: n // 4] = np.eye(3, dtype=np.float32)  # already diagonal: every rotation skipped
    F[n // 4: n // 4 + 8] = 0.0                      # singular: unit-axis branch of U
    U, S, V = O.svd("ref", F)
    return dict(F=F, U=U, S=S, V=V)


def constitutive():
    """Single-particle cases of tests/test_mpm_constitutive.cpp and
    tests/test_mpm_stress_isolation.cpp run through the reference."""
    out = {}

    def one(F_list, positions, alpha=None):
        s = O.CpuSolver("ref", 0.1)
        s.set_material(1.0e5, 0.3, 1500.0)
        s.set_gravity((0, 0, 0))
        if alpha is not None:
            s.set_plastic_alpha(alpha)
        s.add_particles(np.array(positions, np.float32), None, np.full(len(positions), 0.01, np.float32))
        if F_list is not None:
            s.set_particle_state(0, F=np.array(F_list, np.float32))
        s.step(1.0 / 240.0)
        p = s.get_particles()
        g = s.grid_nodes()
        speed = np.linalg.norm(g["velocity"][g["active"] > 0], axis=1)
        return p, float(speed.max() if len(speed) else 0.0)

    p, sp = one(None, [(0.2, 0.2, 0.2)])
    out["zero_strain_speed"] = np.float32(sp)
    for eps in (0.005, 0.01):
        p, sp = one([np.diag([1.0, 1.0 + eps, 1.0])], [(0.2, 0.2, 0.2)])
        out[f"strain_{eps}_speed"] = np.float32(sp)
    p, _ = one([np.diag([1.5, 0.5, 1.5])], [(0.2, 0.2, 0.2)], alpha=0.6)
    out["dp_F"] = p["F"][0]
    p, _ = one([np.diag([1.0, 0.9, 1.0])] * 2, [(0.2, 0.18, 0.2), (0.2, 0.22, 0.2)])
    out["column_vel"] = p["velocity"]
    c, o = 0.3, 0.02
    pts = [(c - o, c, c), (c + o, c, c), (c, c - o, c), (c, c + o, c), (c, c, c - o), (c, c, c + o)]
    p, _ = one([np.eye(3) * 0.95] * 6, pts)
    out["hydro_vel"] = p["velocity"]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", required=True, help="root of the reference tree (2nugu/basements)")
    a = ap.parse_args()
    if not O.available("ref"):
        sys.exit("oracle/_ref/libref_mpm.so missing: run `make -C oracle` first")
    cols, data, metrics = box_drop_csv(a.ref_root)
    np.savez_compressed(os.path.join(HERE, "box_drop_M1.npz"), columns=np.array(cols), rows=data,
                        metric_names=np.array(list(metrics)), metric_values=np.array(list(metrics.values())),
                        ref_rows=O.box_drop_m1("ref"))
    scenes_m1 = {}
    for scene, summaries in M1_SCENES:
        scenes_m1.update(research_csv(a.ref_root, scene, summaries))
    scenes_m1.update(drift_pic_csv(a.ref_root))
    np.savez_compressed(os.path.join(HERE, "m1_scenes.npz"), **scenes_m1)
    np.savez_compressed(os.path.join(HERE, "repose_pile.npz"), **repose_summary(a.ref_root))
    np.savez_compressed(os.path.join(HERE, "small_scene.npz"), **run_small_scene())
    np.savez_compressed(os.path.join(HERE, "m1_cases.npz"), **m1_cases())
    np.savez_compressed(os.path.join(HERE, "m45a_cases.npz"), **m1_cases(16, 23, "m45a_apply"))
    scenes_m45a = {}
    for scene, summaries in (("box_drop", ("metrics",)),) + M1_SCENES:
        scenes_m45a.update(research_csv(a.ref_root, scene, summaries, "M4.5a"))
    np.savez_compressed(os.path.join(HERE, "m45a_scenes.npz"), **scenes_m45a)
    np.savez_compressed(os.path.join(HERE, "m0_cases.npz"), **m1_cases(16, 31, "m0_apply"))
    scenes_m0 = drift_dirichlet_csv(a.ref_root)
    for scene, summaries in (("box_drop", ("metrics",)),) + M1_SCENES:
        scenes_m0.update(research_csv(a.ref_root, scene, summaries, "M0"))
    np.savez_compressed(os.path.join(HERE, "m0_scenes.npz"), **scenes_m0)
    for coupler, method, seed in (("m45b", "M4.5b", 37), ("m45c", "M4.5", 41)):
        np.savez_compressed(os.path.join(HERE, f"{coupler}_cases.npz"), **m1_cases(16, seed, f"{coupler}_apply"))
        scenes = {}
        for scene, summaries in (("box_drop", ("metrics",)),) + M1_SCENES:
            if os.path.exists(os.path.join(a.ref_root, "research/mpm_rigid_coupling/outputs/csv",
                                           f"{scene}_{method}.csv")):
                scenes.update(research_csv(a.ref_root, scene, summaries, method))
        np.savez_compressed(os.path.join(HERE, f"{coupler}_scenes.npz"), **scenes)
    np.savez_compressed(os.path.join(HERE, "svd_cases.npz"), **svd_cases())
    np.savez_compressed(os.path.join(HERE, "constitutive.npz"), **constitutive())
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")


if __name__ == "__main__":
    main()
