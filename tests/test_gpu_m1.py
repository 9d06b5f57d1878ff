"""Parity of the CUDA M1 PIC-rigid coupler with the reference (GPU).

* per-call fixtures made by the reference's MPMRigidCouplerPIC::apply on seeded
  grids (boxes and cylinders, random poses, empty / tiny / normal node masses,
  dt = 0): grid after the call and nodes_inside exactly, force and torque to
  1e-5 relative (the reference sums in float in hash-map order, the kernel in
  double per CTA);
* the reference's grid-only research scenes (box_drop, box_drop_dense,
  foot_step, tine_drag, rover_wheel; 480-720 steps) and the rigid-drift
  benchmark's M1 run against their shipped CSVs;
* the reference's cylinder inside-test KATs, probed through the coupler;
* the M4.5a sweep and M0 Dirichlet couplers: the reference's per-call
  fixtures, the research scenes' *_M4.5a / *_M0 CSVs, the M0 unit tests, the
  Dirichlet rigid-drift output and a coupled particle scene;
* a particle scene with a cylinder through bm_solver_step_coupled against the
  reference's split phases P2G -> update_grid -> apply -> G2P.
"""
import os

import numpy as np
import pytest

import basements_b200 as bm
from basements_b200 import scenes
from oracle import oracle as O
from tests.gpu_util import POS_TOL_100, cpu_solver, dense_index, gpu_solver, max_err_dx

GOLD = os.path.join(os.path.dirname(__file__), "golden")
REF = O.reference_or_port()

pytestmark = pytest.mark.gpu


def _body_from_row(b):
    return dict(center=b[0:3], orientation=b[3:7], half_extents=b[7:10], linear_velocity=b[10:13],
                angular_velocity=b[13:16], friction=float(b[16]), mass=float(b[17]), shape=int(b[18]))


def test_m1_matches_reference_fixtures():
    d = np.load(os.path.join(GOLD, "m1_cases.npz"))
    off = {k: np.concatenate([[0], np.cumsum(d[k + "_len"])]) for k in ("seed_ijk", "grid_ijk")}
    for c in range(len(d["dx"])):
        sl = slice(off["seed_ijk"][c], off["seed_ijk"][c + 1])
        ijk = d["seed_ijk"][sl]
        lo = ijk.min(0) - 8
        hi = ijk.max(0) + 8
        s = bm.MPMSolver(float(d["dx"][c]), domain=(tuple(lo), tuple(hi - lo)))
        s.seed_grid(ijk, d["seed_vel"][sl], d["seed_mass"][sl])
        body = bm.make_collider(**_body_from_row(d["body"][c]))
        f, t, n = s.m1_apply(body, float(d["dt"][c]))
        assert n == d["nodes_inside"][c], c
        fr, tr = d["force"][c], d["torque"][c]
        scale = max(np.abs(fr).max(), 1e-30)
        assert np.abs(f - fr).max() <= 1e-5 * scale + 1e-30, (c, f, fr)
        assert np.abs(t - tr).max() <= 1e-5 * max(np.abs(tr).max(), 1e-30) + 1e-30, (c, t, tr)
        g = s.get_grid()
        gs = slice(off["grid_ijk"][c], off["grid_ijk"][c + 1])
        idx = dense_index(g, d["grid_ijk"][gs])
        assert np.array_equal(g["velocity"].reshape(-1, 3)[idx], d["grid_vel"][gs])
        assert np.array_equal(g["mass"].reshape(-1)[idx], d["grid_mass"][gs])
        # nodes of blocks the reference never allocated stay empty
        mask = np.ones(g["mass"].size, bool)
        mask[idx] = False
        assert np.all(g["mass"].reshape(-1)[mask] == 0)


@pytest.mark.parametrize("coupler", ["m45a", "m45b", "m45c", "m0"])
def test_sweep_and_dirichlet_match_reference_fixtures(coupler):
    """One call of the CUDA M4.5a sweep or M0 Dirichlet coupler on the seeded
    grids of m45a/m45b/m45c_cases.npz / m0_cases.npz (made by the reference's
    M4_5a/M4_5b/M4_5c::apply / MPMRigidCoupler::apply). nodes_inside exactly; force and
    torque to 1e-5 of their largest component (summed in double per CTA, in
    float in hash-map order by the reference). M0's node update is per node,
    so its grid is exact; M4.5a's overlap sum is taken in double on the
    device, so its grid agrees to 1e-5 relative."""
    d = np.load(os.path.join(GOLD, f"{coupler}_cases.npz"))
    off = {k: np.concatenate([[0], np.cumsum(d[k + "_len"])]) for k in ("seed_ijk", "grid_ijk")}
    for c in range(len(d["dx"])):
        sl = slice(off["seed_ijk"][c], off["seed_ijk"][c + 1])
        ijk = d["seed_ijk"][sl]
        lo = ijk.min(0) - 8
        hi = ijk.max(0) + 8
        s = bm.MPMSolver(float(d["dx"][c]), domain=(tuple(lo), tuple(hi - lo)))
        s.seed_grid(ijk, d["seed_vel"][sl], d["seed_mass"][sl])
        body = bm.make_collider(**_body_from_row(d["body"][c]))
        f, t, n = getattr(s, f"{coupler}_apply")(body, float(d["dt"][c]))
        assert n == d["nodes_inside"][c], c
        fr, tr = d["force"][c], d["torque"][c]
        assert np.abs(f - fr).max() <= 1e-5 * max(np.abs(fr).max(), 1e-30) + 1e-30, (c, f, fr)
        assert np.abs(t - tr).max() <= 1e-5 * max(np.abs(tr).max(), 1e-30) + 1e-30, (c, t, tr)
        g = s.get_grid()
        gs = slice(off["grid_ijk"][c], off["grid_ijk"][c + 1])
        idx = dense_index(g, d["grid_ijk"][gs])
        if coupler == "m0":
            assert np.array_equal(g["velocity"].reshape(-1, 3)[idx], d["grid_vel"][gs]), c
            assert np.array_equal(g["mass"].reshape(-1)[idx], d["grid_mass"][gs]), c
        else:
            np.testing.assert_allclose(g["velocity"].reshape(-1, 3)[idx], d["grid_vel"][gs], rtol=1e-5,
                                       atol=1e-6 * max(np.abs(d["grid_vel"][gs]).max(), 1.0))
            np.testing.assert_allclose(g["mass"].reshape(-1)[idx], d["grid_mass"][gs], rtol=1e-5, atol=0)
        mask = np.ones(g["mass"].size, bool)
        mask[idx] = False
        assert np.all(g["mass"].reshape(-1)[mask] == 0)


def _scene_cases():
    """(coupler, scene) pairs with a shipped CSV (no tine_drag for M4.5)."""
    out = []
    for coupler in ("m45a", "m45b", "m45c", "m0"):
        d = np.load(os.path.join(GOLD, f"{coupler}_scenes.npz"))
        out += [(coupler, s) for s in ("box_drop", "box_drop_dense", "foot_step", "tine_drag", "rover_wheel")
                if f"{s}_rows" in d.files]
    return out


@pytest.mark.parametrize("coupler,scene", _scene_cases())
def test_sweep_and_dirichlet_research_scenes_match_reference_csv(coupler, scene):
    """The grid-only research scenes with the sweep couplers or M0
    (bench_compare_all.cpp, methods "M4.5a", "M4.5b", "M4.5" and "M0"): the
    float32 harness loop of tests/m1_scene_loop.py around the CUDA coupler
    against the reference's shipped CSVs, to the bars of the M1 scenes
    (relative to the size of the positions and velocities for the M4.5
    rover, whose wheel falls 30 m through the sand)."""
    from tests import m1_scene_loop as L
    gold = np.load(os.path.join(GOLD, f"{coupler}_scenes.npz"))
    ref = gold[scene + "_rows"]
    vals = dict(zip(gold[scene + "_metric_names"], gold[scene + "_metric_values"]))
    rows = L.run(scene, L.GpuGrid(bm, L.SCENES[scene], coupler))
    if scene == "tine_drag":
        fx, fy, n = L.tine_summary(rows)
        sub = rows[::4]
        print(f"tine_drag {coupler}: max |dFx| = {np.abs(sub[:, 2] - ref[:, 2]).max():.3e} N, avg draft {fx:.6f} N "
              f"(reference {vals['avg_draft_fx_n']:.6f})")
        np.testing.assert_allclose(sub[:, 1], ref[:, 1], rtol=2e-6, atol=1e-6)
        np.testing.assert_allclose(sub[:, 2:], ref[:, 2:], rtol=1e-5, atol=1e-4)
        assert n == vals["samples"]
        assert abs(fx - vals["avg_draft_fx_n"]) <= 1e-5 * abs(vals["avg_draft_fx_n"])
        return
    e_pos = np.abs(rows[:, 1:4] - ref[:, 1:4]).max()
    e_vy = np.abs(rows[:, 4] - ref[:, 4]).max()
    max_p = np.abs(rows[:, 7]).max()
    print(f"{scene} {coupler}: max |dx| = {e_pos:.3e} m, max |dvy| = {e_vy:.3e} m/s, max |sum p_y| {max_p:.6f} "
          f"(reference {vals['max_abs_total_p_y']:.6f})")
    assert e_pos <= 2e-5 * max(1.0, np.abs(ref[:, 1:4]).max())
    assert e_vy <= 2e-4 * max(1.0, np.abs(ref[:, 4]).max())
    assert np.array_equal(rows[:, 9], ref[:, 9])
    assert abs(max_p - vals["max_abs_total_p_y"]) <= 1e-4 * vals["max_abs_total_p_y"]


def test_dirichlet_unit_tests_on_gpu():
    """tests/test_mpm_rigid_coupler.cpp:26-92 through the CUDA M0 coupler."""
    from tests import dirichlet_kats as K
    for case in K.CASES:
        s = bm.MPMSolver(0.1, domain=((-8, -8, -8), (40, 40, 40)))
        s.seed_grid(np.array([case["node"]], np.int32), np.array([case["vel"]], np.float32),
                    np.array([1.0], np.float32))
        f, t, n = s.m0_apply(bm.make_collider(**case["body"]), 1.0 / 60.0)
        g = s.get_grid()
        o = np.asarray(g["origin"])
        i, j, k = (np.array(case["node"]) - o)
        K.check(case, f, t, n, g["velocity"][i, j, k])


def test_sweep_invariants_on_gpu():
    """tests/test_mpm_rigid_sweep.cpp:70-154 (the M4.5a cases) through the
    CUDA M4.5a coupler."""
    from tests import sweep_kats as K
    for case in K.CASES:
        s = bm.MPMSolver(0.1, domain=((-8, -8, -8), (16, 16, 16)))
        if case["layers"]:
            s.seed_grid(*K.patch(case["layers"]))
        before = float(s.get_grid()["mass"].astype(np.float64).sum())
        f, t, n = s.m45a_apply(bm.make_collider(**case["body"]), case["dt"])
        after = float(s.get_grid()["mass"].astype(np.float64).sum())
        K.check(case, before, after, f, t, n)


def test_rigid_drift_dirichlet_matches_reference_csv():
    """benchmarks/bench_mpm_rigid_drift.cpp with its default method (M0): the
    unit box over a 5x3x5 patch, 720 steps, against
    outputs/figures/mpm_rigid_drift.csv (2.6e-7 from the reference rebuilt
    here, see the oracle pin)."""
    from tests import m1_scene_loop as L
    ref = np.load(os.path.join(GOLD, "m0_scenes.npz"))["rigid_drift_rows"]
    rows = L.run("rigid_drift", L.GpuGrid(bm, L.SCENES["rigid_drift"], "m0"))[:, L.DRIFT_COLUMNS]
    e_y = np.abs(rows[:, 1] - ref[:, 1]).max()
    e_vy = np.abs(rows[:, 2] - ref[:, 2]).max()
    print(f"rigid_drift M0: max |dy| = {e_y:.3e} m, max |dvy| = {e_vy:.3e} m/s")
    assert e_y <= 2e-5 and e_vy <= 2e-4
    assert np.array_equal(rows[:, 7], ref[:, 7])


@pytest.mark.parametrize("coupler", ["m45a", "m45b", "m45c", "m0"])
def test_sweep_and_dirichlet_coupled_particle_scene_match_reference_split(coupler):
    """A particle scene with a cylinder stepped by bm_solver_step_coupled with
    the M4.5a or M0 coupler, against the reference's split phases P2G ->
    update_grid -> coupler -> G2P."""
    sc = scenes.wheel_rut(n_keep=20000)
    body = sc.bodies[0]
    g = gpu_solver(sc.dx, sc.position, None, sc.mass, sc.E, sc.nu, sc.rho, sc.alpha, domain=sc.domain)
    g.set_coupler(coupler)
    c = cpu_solver(REF, sc.dx, sc.position, None, sc.mass, sc.E, sc.nu, sc.rho, sc.alpha)
    for n in range(40):
        b = body.at_time(n * sc.dt)
        gr = g.step_coupled(sc.dt, [bm.make_collider(**b.as_tuple())])[0]
        c.p2g(sc.dt)
        c.grid_update(sc.dt)
        cr = getattr(c, f"{coupler}_apply")(O.collider(**b.as_tuple()), sc.dt)
        c.g2p(sc.dt)
        assert gr[2] == cr[2]
        np.testing.assert_allclose(gr[0], cr[0], rtol=1e-3, atol=1e-3 * max(1.0, np.abs(cr[0]).max()))
    e = max_err_dx(g.get_particles()["position"], c.get_particles()["position"], sc.dx)
    print(f"coupled wheel scene with {coupler}, 40 steps: max |x_gpu - x_ref| = {e:.3e} dx")
    assert e <= POS_TOL_100
    assert g.sync() == (0, 0)


def _quat_mul(a, b):
    f = np.float32
    aw, ax, ay, az = a
    bw, bx, by, bz = b
    return (f(f(f(aw * bw) - f(ax * bx)) - f(ay * by)) - f(az * bz),
            f(f(f(aw * bx) + f(ax * bw)) + f(ay * bz)) - f(az * by),
            f(f(f(aw * by) - f(ax * bz)) + f(ay * bw)) + f(az * bx),
            f(f(f(aw * bz) + f(ax * by)) - f(ay * bx)) + f(az * bw))


def test_box_drop_scene_matches_reference_csv():
    """research/mpm_rigid_coupling/bench_compare_all.cpp:72-208, M1: the
    harness loop runs here in float32 numpy around the CUDA coupler."""
    gold = np.load(os.path.join(GOLD, "box_drop_M1.npz"))
    f = np.float32
    dx, dt, g, mass = f(0.1), f(1.0 / 240.0), f(9.81), f(1.0)
    s = bm.MPMSolver(0.1, domain=((-8, -4, -8), (16, 16, 16)))
    ijk = np.array([(i, j, k) for i in range(-3, 4) for j in range(3) for k in range(-3, 4)], np.int32)
    s.seed_grid(ijk, np.zeros((len(ijk), 3), np.float32), np.full(len(ijk), 0.01, np.float32))
    pos = np.array([0, 0.55, 0], np.float32)
    vel = np.zeros(3, np.float32)
    omg = np.zeros(3, np.float32)
    q = (f(1), f(0), f(0), f(0))
    rows = []
    for i in range(len(gold["rows"])):
        force = np.array([0, -g * mass, 0], np.float32)
        body = bm.make_collider(pos, (0.2, 0.2, 0.2), q, vel, omg, 0.5, 1.0, 0)
        fr, tq, n = s.m1_apply(body, float(dt))
        force = (force + fr).astype(np.float32)
        vel = (vel + (force * (f(1) / mass)) * dt).astype(np.float32)
        omg = (omg + tq.astype(np.float32) * dt).astype(np.float32)
        pos = (pos + vel * dt).astype(np.float32)
        dq = _quat_mul((f(0), omg[0], omg[1], omg[2]), q)
        h = f(f(0.5) * dt)
        q = tuple(f(q[a] + f(dq[a] * h)) for a in range(4))
        nrm = f(np.sqrt(f(f(f(q[0] * q[0]) + f(q[1] * q[1])) + f(q[2] * q[2])) + f(q[3] * q[3])))
        q = tuple(f(c * f(f(1) / nrm)) for c in q)
        grid = s.get_grid()
        v = grid["velocity"].copy()
        act = grid["mass"] > 0
        vy = v[..., 1]
        vy[act] = vy[act] + (-g * dt)
        vy[act & (vy < 0)] = 0
        s.set_grid_velocity(v)
        pg = (v[act] * grid["mass"][act][:, None]).astype(np.float64).sum(0)
        pb = vel * mass
        rows.append([pos[0], pos[1], pos[2], vel[1], pb[1], pg[1], pb[1] + pg[1], n])
    rows = np.array(rows)
    ref = gold["rows"]
    np.testing.assert_allclose(rows[:, 0:3], ref[:, 1:4], atol=2e-5)
    np.testing.assert_allclose(rows[:, 3], ref[:, 4], atol=2e-4)
    assert np.array_equal(rows[:, 7], ref[:, 9])
    names = list(gold["metric_names"])
    max_p = np.abs(rows[:, 6]).max()
    assert abs(max_p - gold["metric_values"][names.index("max_abs_total_p_y")]) < 1e-4 * 0.18


@pytest.mark.parametrize("scene", ["box_drop_dense", "foot_step", "tine_drag", "rover_wheel"])
def test_research_scenes_match_reference_csv(scene):
    """The other grid-only M1 research scenes (bench_compare_all.cpp:
    tine_drag :215-292, foot_step :374-504, box_drop_dense :505-613,
    rover_wheel :614-800): the
    float32 harness loop of tests/m1_scene_loop.py around the CUDA coupler,
    against the reference's shipped CSVs. The same loop around the float
    restatement reproduces those CSVs to their 7 printed digits (CPU test), so
    what is left here is the coupler's reaction sum (double per CTA against
    the reference's float sum in hash-map order) carried through the scene."""
    from tests import m1_scene_loop as L
    gold = np.load(os.path.join(GOLD, "m1_scenes.npz"))
    ref = gold[scene + "_rows"]
    vals = dict(zip(gold[scene + "_metric_names"], gold[scene + "_metric_values"]))
    rows = L.run(scene, L.GpuGrid(bm, L.SCENES[scene]))
    if scene == "tine_drag":
        fx, fy, n = L.tine_summary(rows)
        sub = rows[::4]
        print(f"tine_drag: max |dFx| = {np.abs(sub[:, 2] - ref[:, 2]).max():.3e} N, "
              f"avg draft {fx:.6f} N (reference {vals['avg_draft_fx_n']:.6f})")
        np.testing.assert_allclose(sub[:, 1], ref[:, 1], rtol=2e-6, atol=1e-6)
        np.testing.assert_allclose(sub[:, 2:], ref[:, 2:], rtol=1e-5, atol=1e-5)
        assert n == vals["samples"]
        assert abs(fx - vals["avg_draft_fx_n"]) <= 1e-5 * abs(vals["avg_draft_fx_n"])
        return
    e_pos = np.abs(rows[:, 1:4] - ref[:, 1:4]).max()
    e_vy = np.abs(rows[:, 4] - ref[:, 4]).max()
    max_p = np.abs(rows[:, 7]).max()
    print(f"{scene}: max |dx| = {e_pos:.3e} m, max |dvy| = {e_vy:.3e} m/s, first row off by 1e-5: "
          f"{L.first_divergence(rows[:, 1:4], ref[:, 1:4], 1e-5)}, max |sum p_y| {max_p:.6f} "
          f"(reference {vals['max_abs_total_p_y']:.6f})")
    assert e_pos <= 2e-5
    assert e_vy <= 2e-4
    assert np.array_equal(rows[:, 9], ref[:, 9])
    assert abs(max_p - vals["max_abs_total_p_y"]) <= 1e-4 * vals["max_abs_total_p_y"]
    if scene == "foot_step":
        down, up = L.rebound(rows)
        assert abs(down - vals["v_down_peak"]) <= 1e-4 * abs(vals["v_down_peak"]) and up == vals["v_up_peak"]


def test_rigid_drift_pic_matches_reference_csv():
    """benchmarks/bench_mpm_rigid_drift.cpp --method pic: the unit box over a
    5x3x5 patch, 720 steps, against outputs/figures/mpm_rigid_drift_pic.csv."""
    from tests import m1_scene_loop as L
    ref = np.load(os.path.join(GOLD, "m1_scenes.npz"))["rigid_drift_rows"]
    rows = L.run("rigid_drift", L.GpuGrid(bm, L.SCENES["rigid_drift"]))[:, L.DRIFT_COLUMNS]
    e_y = np.abs(rows[:, 1] - ref[:, 1]).max()
    e_vy = np.abs(rows[:, 2] - ref[:, 2]).max()
    print(f"rigid_drift: max |dy| = {e_y:.3e} m, max |dvy| = {e_vy:.3e} m/s")
    assert e_y <= 2e-5 and e_vy <= 2e-4
    assert np.array_equal(rows[:, 7], ref[:, 7])
    np.testing.assert_allclose(rows[:, 5], ref[:, 5], atol=1e-4 * np.abs(ref[:, 5]).max())


def test_cylinder_inside_kats():
    """tests/test_mpm_rigid_cylinder.cpp:37-255 through the CUDA M1: the
    inside-test cases, and the 200-probe rolling sweep entering and leaving
    once, probe for probe equal to the oracle's M1."""
    from tests import shape_kats as K
    for name, point, q, expect in K.KATS:
        assert K.probe_gpu(bm, point, q) == expect, name
    probes = K.rolling_probes()
    seq = [K.probe_gpu(bm, p, q) for p, q in probes]
    assert K.transitions(seq) == 2
    assert seq == [K.probe_oracle(O, REF, p, q) for p, q in probes]


def test_coupled_particle_scene_matches_reference_split():
    sc = scenes.wheel_rut(n_keep=20000)
    body = sc.bodies[0]
    g = gpu_solver(sc.dx, sc.position, None, sc.mass, sc.E, sc.nu, sc.rho, sc.alpha, domain=sc.domain)
    c = cpu_solver(REF, sc.dx, sc.position, None, sc.mass, sc.E, sc.nu, sc.rho, sc.alpha)
    for n in range(40):
        b = body.at_time(n * sc.dt)
        gr = g.step_coupled(sc.dt, [bm.make_collider(**b.as_tuple())])[0]
        c.p2g(sc.dt)
        c.grid_update(sc.dt)
        cr = c.m1_apply(O.collider(**b.as_tuple()), sc.dt)
        c.g2p(sc.dt)
        assert gr[2] == cr[2]
        np.testing.assert_allclose(gr[0], cr[0], rtol=1e-3, atol=1e-3 * max(1.0, np.abs(cr[0]).max()))
    e = max_err_dx(g.get_particles()["position"], c.get_particles()["position"], sc.dx)
    print(f"coupled wheel scene, 40 steps: max |x_gpu - x_ref| = {e:.3e} dx")
    assert e <= POS_TOL_100
    assert g.sync() == (0, 0)
    assert g.light_node_suspects() == 0


def test_overlapping_bodies_apply_in_order_like_the_reference():
    """Two bodies whose boxes overlap, in one bm_solver_step_coupled: the
    reference applies its couplers one after another, the second on the grid
    the first projected; the step must do the same."""
    sc = scenes.wheel_rut(n_keep=20000)
    b0 = sc.bodies[0]
    g = gpu_solver(sc.dx, sc.position, None, sc.mass, sc.E, sc.nu, sc.rho, sc.alpha, domain=sc.domain)
    c = cpu_solver(REF, sc.dx, sc.position, None, sc.mass, sc.E, sc.nu, sc.rho, sc.alpha)
    for n in range(10):
        t0 = b0.at_time(n * sc.dt).as_tuple()
        t1 = dict(t0, center=tuple(np.add(t0["center"], (1.5 * sc.dx, 0.0, 0.5 * sc.dx))),
                  linear_velocity=(0.0, -0.2, 0.0), shape=0)
        gr = g.step_coupled(sc.dt, [bm.make_collider(**t0), bm.make_collider(**t1)])
        c.p2g(sc.dt)
        c.grid_update(sc.dt)
        cr = [c.m1_apply(O.collider(**t0), sc.dt), c.m1_apply(O.collider(**t1), sc.dt)]
        c.g2p(sc.dt)
        for k in range(2):
            assert gr[k][2] == cr[k][2] > 0
            np.testing.assert_allclose(gr[k][0], cr[k][0], rtol=1e-3, atol=1e-3 * max(1.0, np.abs(cr[k][0]).max()))
    e = max_err_dx(g.get_particles()["position"], c.get_particles()["position"], sc.dx)
    print(f"two overlapping bodies, 10 steps: max |x_gpu - x_ref| = {e:.3e} dx")
    assert e <= POS_TOL_100
