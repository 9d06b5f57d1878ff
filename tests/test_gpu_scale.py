"""Parity at the sizes of the benchmark's workloads (GPU).

The other GPU tests check the step on scenes of thousands to tens of
thousands of particles. These run the workloads' own generators at their
scale, each against the reference compiled from its headers (oracle/_ref)
and, where stated, the FP64 restatement:

* the wheel rut (128^3 grid, dx = 1/128, the M1 cylinder rolling through the
  bed) subsampled to 100,000 particles in the same bed and box, 100 coupled
  steps: positions within 2e-4 dx of the reference (the FP32 floor of this
  sparse contact scene: the reference's own run lies 2.8e-4 dx from FP64);
  against FP64 no further than the reference plus 1e-4 dx; grid mass equal
  to the particle mass to 1e-6;
* one batched box-drop scene at the top of that workload's range (400,000
  particles on a 96^3 grid, a dynamic box resting in the bed) stepped 100
  times in a batch beside small scenes;
* a served mix drawn from the request stream's generator (an 805k-particle
  request on a 94^3 grid with a cylinder, a 474k one on a 103^3 grid with a
  box, small ones beside them): each large request alone and in the mix,
  and against the reference.

The bodies of the batched and served scenes start pressed into the sand so
that the coupler and the device rigid update work from the first step.
"""
import dataclasses

import numpy as np
import pytest

import basements_b200 as bm
from basements_b200 import scenes
from oracle import oracle as O
from tests.gpu_util import MASS_REL_TOL, POS_TOL_100, max_err_dx

REF = O.reference_or_port()

pytestmark = pytest.mark.gpu

POS_TOL_WHEEL_100K = 2e-4  # dx, 100 coupled steps of the 100k-particle wheel rut (see the test)


def cpu_scene(kind, sc):
    c = O.CpuSolver(kind, sc.dx)
    c.set_material(sc.E, sc.nu, sc.rho)
    c.set_plastic_alpha(sc.alpha)
    c.set_gravity(sc.gravity)
    c.set_floor_friction(sc.floor_friction)
    c.add_particles(sc.position, None, sc.mass)
    return c


def pressed(sc, depth_frac=0.5):
    """The scene with its body lowered so that it reaches depth_frac of its
    half height into the bed's top surface."""
    b = sc.bodies[0]
    top = float(sc.position[:, 1].max())
    c = (b.center[0], top + b.half_extents[1] * (1.0 - depth_frac), b.center[2])
    return dataclasses.replace(sc, bodies=[dataclasses.replace(b, center=c)])


def test_wheel_rut_100k_particles_100_coupled_steps():
    sc = scenes.wheel_rut(n_keep=100_000)
    body = sc.bodies[0]
    steps = 100
    g = bm.MPMSolver(sc.dx, domain=sc.domain)
    g.set_material(sc.E, sc.nu, sc.rho)
    g.set_plastic_alpha(sc.alpha)
    g.add_particles(sc.position, None, sc.mass)
    cpus = {k: cpu_scene(k, sc) for k in (REF, "f64")}
    for i in range(steps):
        col = body.at_time(i * sc.dt).as_tuple()
        (f, _, n_in), = g.step_coupled(sc.dt, [bm.make_collider(**col)])
        for k, c in cpus.items():
            c.p2g(sc.dt)
            c.grid_update(sc.dt)
            rf, _, rn = c.m1_apply(O.collider(**col), sc.dt)
            c.g2p(sc.dt)
            if k == REF and i % 25 == 0:
                print(f"step {i}: force {f} vs {rf}, nodes inside {n_in} vs {rn}")
    assert n_in > 0
    pg = g.get_particles(("position",))["position"]
    p64 = cpus["f64"].positions_f64()
    e_ref = max_err_dx(pg, cpus[REF].get_particles()["position"], sc.dx)
    e_64 = max_err_dx(pg, p64, sc.dx)
    e_ref_64 = max_err_dx(cpus[REF].get_particles()["position"], p64, sc.dx)
    print(f"wheel rut 100k, {steps} coupled steps: max |x_gpu - x_ref| = {e_ref:.2e} dx, vs FP64 {e_64:.2e} dx; "
          f"the reference (FP32) vs FP64: {e_ref_64:.2e} dx")
    # In this sparse contact scene (0.15 particles per cell, 5 g each) FP32
    # arithmetic itself moves particles far: the reference's own run lies
    # 2.8e-4 dx from FP64 after 100 steps. Two FP32 runs that only sum the
    # P2G contributions in another order (the GPU's atomics, its regrouping
    # interval) differ by ~1e-4 dx (measured 6.9e-5 and 1.3e-4 dx with
    # regrouping every 16 and 32 steps), so the bar against the reference is
    # a fixed 2e-4 dx here, and against FP64 no further than the reference
    # plus 1e-4 dx.
    assert e_ref <= POS_TOL_WHEEL_100K
    assert e_64 <= e_ref_64 + POS_TOL_100
    assert g.sync() == (0, 0) and g.light_node_suspects() == 0
    g.p2g(sc.dt)
    grid_mass = g.get_grid()["mass"].astype(np.float64).sum()
    pm = sc.mass.astype(np.float64).sum()
    assert abs(grid_mass - pm) / pm < MASS_REL_TOL


def test_batch_with_a_400k_particle_scene_on_a_96_grid():
    big = pressed(scenes.box_drop_scene(7, grid=96, n_particles=400_000))
    small = [pressed(scenes.box_drop_scene(200 + k, grid=32, n_particles=n)) for k, n in
             enumerate((8000, 20000, 12000))]
    steps = 100
    b = bm.Batch([small[0], big] + small[1:])
    b.step(steps)
    assert b.sync()[0] == 0
    for idx, sc in ((1, big), (0, small[0])):
        c = cpu_scene(REF, sc)
        body = c.run_dynamic_body(O.collider(**sc.bodies[0].as_tuple()), sc.gravity, sc.dt, steps)
        e = max_err_dx(b.get_particles(idx)["position"], c.get_particles()["position"], sc.dx)
        gb = b.get_body(idx)
        print(f"{sc.name} ({sc.n} particles, grid {sc.grid}): {e:.2e} dx, body centre {gb.center[:]} "
              f"vs {body.center[:]}")
        assert e < POS_TOL_100
        np.testing.assert_allclose(gb.center[:], body.center[:], atol=1e-5)
        np.testing.assert_allclose(gb.linear_velocity[:], body.linear_velocity[:], atol=2e-4)
    assert b.light_node_suspects() >= 0


def test_served_mix_of_large_requests():
    large = [pressed(scenes.serve_request_scene(18)), pressed(scenes.serve_request_scene(117))]
    assert large[0].bodies[0].shape == 1 and large[1].bodies[0].shape == 0
    small = [scenes.serve_request_scene(s) for s in (0, 1, 2)]
    steps = 40
    alone = []
    for sc in large:
        srv = bm.Server()
        rid = srv.submit(sc, steps)
        assert srv.wait(rid, timeout_ms=600_000) == 0
        alone.append(srv.result(rid))
        srv.close()
    srv = bm.Server()
    first = [srv.submit(sc, steps + 20) for sc in small[:2]]
    ids = [srv.submit(sc, steps) for sc in large]
    late = [srv.submit(small[2], 30)]
    for r in first + ids + late:
        assert srv.wait(r, timeout_ms=600_000) == 0, r
    mixed = [srv.result(r) for r in ids]
    srv.close()
    for sc, a, m in zip(large, alone, mixed):
        e_mix = max_err_dx(a["position"], m["position"], sc.dx)
        c = cpu_scene(REF, sc)
        body = c.run_dynamic_body(O.collider(**sc.bodies[0].as_tuple()), sc.gravity, sc.dt, steps)
        e_ref = max_err_dx(m["position"], c.get_particles()["position"], sc.dx)
        print(f"{sc.name} ({sc.n} particles, grid {sc.grid}, shape {sc.bodies[0].shape}): alone vs mix "
              f"{e_mix:.2e} dx, vs reference {e_ref:.2e} dx")
        assert e_mix < POS_TOL_100 and e_ref < POS_TOL_100
        np.testing.assert_allclose(m["body"].center[:], body.center[:], atol=1e-5)
        np.testing.assert_allclose(a["body"].center[:], m["body"].center[:], atol=1e-5)
