"""The batched form (bm_batch_*) against the reference and the plain solver (GPU).

Scenes of uneven particle and grid counts, each with its own dt, material and
a dynamic rigid box, are stepped together by the batch. Each scene must
match the reference's own solver, coupler and rigid integrator run alone on
the CPU (oracle/_ref run_dynamic_body: P2G, update_grid, M1 on the body's
current state, TimeIntegrator, G2P), to the accuracy bar of the plain step.
"""
import dataclasses

import numpy as np
import pytest

import basements_b200 as bm
from basements_b200 import scenes
from oracle import oracle as O
from tests.gpu_util import POS_TOL_100, gpu_solver, max_err_dx

REF = O.reference_or_port()

pytestmark = pytest.mark.gpu


def small_scenes(n=6):
    sizes = [2000, 9000, 4500, 16000, 3000, 7000, 12000, 5000]
    grids = [32, 48, 32, 64, 32, 48, 64, 32]
    return [scenes.box_drop_scene(s, grid=grids[s % 8], n_particles=sizes[s % 8]) for s in range(n)]


def test_batch_matches_reference_scene_by_scene():
    scs = small_scenes(6)
    b = bm.Batch(scs)
    steps = 40
    b.step(steps)
    assert b.sync()[0] == 0
    assert b.light_node_suspects() == 0
    for i, sc in enumerate(scs):
        c = O.CpuSolver(REF, sc.dx)
        c.set_material(sc.E, sc.nu, sc.rho)
        c.set_plastic_alpha(sc.alpha)
        c.add_particles(sc.position, None, sc.mass)
        body = c.run_dynamic_body(O.collider(**sc.bodies[0].as_tuple()), sc.gravity, sc.dt, steps)
        e = max_err_dx(b.get_particles(i)["position"], c.get_particles()["position"], sc.dx)
        gb = b.get_body(i)
        print(f"scene {i}: {sc.n} particles, grid {sc.grid}: max |x_gpu - x_ref| = {e:.2e} dx, "
              f"body y {gb.center[1]:.6f} vs {body.center[1]:.6f}")
        assert e < POS_TOL_100, i
        np.testing.assert_allclose(gb.center[:], body.center[:], atol=1e-5)
        np.testing.assert_allclose(gb.linear_velocity[:], body.linear_velocity[:], atol=2e-4)
        np.testing.assert_allclose(gb.orientation[:], body.orientation[:], atol=1e-5)


def test_batch_of_one_equals_plain_solver():
    sc = scenes.sand_column(cells=(8, 6, 8))
    b = bm.Batch([sc])
    g = gpu_solver(sc.dx, sc.position, None, sc.mass, sc.E, sc.nu, sc.rho, sc.alpha)
    b.step(50)
    g.step(sc.dt, 50)
    assert max_err_dx(b.get_particles(0)["position"], g.get_particles()["position"], sc.dx) < 1e-5


def test_ragged_batch_with_empty_and_single_particle_scenes():
    """An empty scene (explicit box, no particles), a one-particle scene and a
    sand column step together, eagerly and through graph chunks: the empty
    scene stays empty and the others equal the plain solver run alone."""
    col = scenes.sand_column(cells=(8, 6, 8))
    empty = dataclasses.replace(col, name="empty", position=np.zeros((0, 3), np.float32),
                                mass=np.zeros(0, np.float32), domain=((0, 0, 0), (32, 32, 32)))
    one = dataclasses.replace(col, name="one", position=col.position[:1].copy(), mass=col.mass[:1].copy())
    steps = 2 * 16 + 7  # eager head, graph chunks, eager tail
    b = bm.Batch([empty, one, col, empty])
    b.step(steps)
    st, scene, esc = b.sync()
    assert (st, esc) == (0, 0), scene
    assert b.num_particles(0) == 0 and b.num_particles(3) == 0
    assert b.get_particles(0)["position"].shape == (0, 3)
    for i, sc in ((1, one), (2, col)):
        g = gpu_solver(sc.dx, sc.position, None, sc.mass, sc.E, sc.nu, sc.rho, sc.alpha)
        g.step(sc.dt, steps)
        e = max_err_dx(b.get_particles(i)["position"], g.get_particles()["position"], sc.dx)
        print(f"scene {i} ({sc.n} particles): max |x_batch - x_plain| = {e:.2e} dx")
        assert e < 1e-5, i


def test_graph_replay_equals_eager_steps():
    """Graph replay takes exactly the eager step sequence. FP32 atomics add in
    a different order on every run, and in a contact scene that difference
    grows with the steps (two eager runs of these scenes already differ by
    ~2e-5 dx at 50 steps), so the bar is the accuracy bar; a step missed or
    taken twice moves the falling sand by ~1e-2 dx."""
    scs = small_scenes(4)
    runs = []
    for graph in (True, False):
        b = bm.Batch(scs)
        b.set_graph(graph)
        b.step(2 * 16 + 16 + 5)  # eager head, graph chunks, eager tail
        assert b.steps_done() == 53
        runs.append([b.get_particles(i)["position"] for i in range(len(scs))])
    for i, sc in enumerate(scs):
        assert max_err_dx(runs[0][i], runs[1][i], sc.dx) < POS_TOL_100


def test_autotune_leaves_the_scenes_where_they_were():
    scs = small_scenes(3)
    a = bm.Batch(scs)
    a.step(5)
    r = a.autotune(trial_steps=8)
    assert 0 <= r["variant"] < len(bm.launch_variants()) and r["sort_interval"] in (8, 16, 32)
    assert r["ms_per_step"] > 0 and a.steps_done() == 5
    a.step(20)
    b = bm.Batch(scs)
    b.step(25)
    for i, sc in enumerate(scs):
        # atomic-order bound of a contact scene, as in the graph test above
        assert max_err_dx(a.get_particles(i)["position"], b.get_particles(i)["position"], sc.dx) < POS_TOL_100


def test_batch_reports_the_failing_scene():
    scs = small_scenes(3)
    bad = scenes.box_drop_scene(9, grid=32, n_particles=2000)
    bad.domain = ((8, 0, 8), (4, 4, 4))  # far too small: the sand leaves it
    b = bm.Batch(scs[:2] + [bad])
    b.step(3)
    st, scene, esc = b.sync()
    assert st == 4 and scene == 2 and esc > 0


def test_device_body_update_with_inverse_inertia_matches_reference():
    """The device rigid update applies a body-space inverse inertia other than
    the identity to the torque as the reference integrator does
    (integrator.h:34): a rotated box pressed into the sand column, against
    the reference run with the same tensor. The tensor moves the spin by
    ~6e-4 rad/s over these steps; the FP32-atomic order by far less."""
    inv_i = np.array([[2.0, 0.3, 0.0], [0.3, 0.5, 0.1], [0.0, 0.1, 1.3]], np.float32)
    sc = scenes.pressed_box(inv_i)
    steps = 20
    b = bm.Batch([sc])
    b.step(steps)
    assert b.sync()[0] == 0
    c = O.CpuSolver(REF, sc.dx)
    c.set_material(sc.E, sc.nu, sc.rho)
    c.set_plastic_alpha(sc.alpha)
    c.add_particles(sc.position, None, sc.mass)
    body = c.run_dynamic_body(O.collider(**sc.bodies[0].as_tuple()), sc.gravity, sc.dt, steps, inv_i)
    e = max_err_dx(b.get_particles(0)["position"], c.get_particles()["position"], sc.dx)
    gb = b.get_body(0)
    print(f"pressed box: max |x_gpu - x_ref| = {e:.2e} dx, spin {gb.angular_velocity[:]} vs {body.angular_velocity[:]}")
    assert e < POS_TOL_100
    np.testing.assert_allclose(gb.angular_velocity[:], body.angular_velocity[:], atol=2e-5)
    np.testing.assert_allclose(gb.linear_velocity[:], body.linear_velocity[:], atol=2e-4)
    np.testing.assert_allclose(gb.center[:], body.center[:], atol=1e-5)
    np.testing.assert_allclose(gb.orientation[:], body.orientation[:], atol=1e-5)


def test_device_body_with_zero_inverse_inertia_does_not_rotate():
    """A body given an all-zero inverse inertia (infinite inertia: the
    reference integrator's w += I^-1 tau dt leaves its spin alone,
    integrator.h:34) keeps its spin and orientation on the device, as in the
    reference run with the same tensor; the unset tensor still means the
    identity, which spins the same box."""
    zero = np.zeros((3, 3), np.float32)
    sc = scenes.pressed_box(zero)
    steps = 20
    b = bm.Batch([sc, scenes.pressed_box()])
    b.step(steps)
    assert b.sync()[0] == 0
    c = O.CpuSolver(REF, sc.dx)
    c.set_material(sc.E, sc.nu, sc.rho)
    c.set_plastic_alpha(sc.alpha)
    c.add_particles(sc.position, None, sc.mass)
    body = c.run_dynamic_body(O.collider(**sc.bodies[0].as_tuple()), sc.gravity, sc.dt, steps, zero)
    gb, spun = b.get_body(0), b.get_body(1)
    assert np.array_equal(gb.angular_velocity[:], sc.bodies[0].angular_velocity)
    assert np.array_equal(body.angular_velocity[:], sc.bodies[0].angular_velocity)
    np.testing.assert_allclose(gb.orientation[:], body.orientation[:], atol=1e-6)
    assert np.abs(np.array(spun.angular_velocity[:])).max() > 1e-4
    assert max_err_dx(b.get_particles(0)["position"], c.get_particles()["position"], sc.dx) < POS_TOL_100
