"""Helpers shared by the GPU tests: run the same scene on the CUDA library and
on a CPU checker, compare in units of dx."""
import numpy as np

import basements_b200 as bm
from oracle import oracle as O

# Accuracy bars of the plain step (particle positions, units of dx).
POS_TOL_100 = 1e-4
POS_TOL_1000 = 1e-3
MASS_REL_TOL = 1e-6


def gpu_solver(dx, pos, vel=None, mass=None, E=1e5, nu=0.3, rho=1500.0, alpha=None, gravity=None,
               floor_friction=None, domain=None, margin=None):
    s = bm.MPMSolver(dx, domain=domain, margin=margin)
    s.set_material(E, nu, rho)
    if alpha is not None:
        s.set_plastic_alpha(alpha)
    if gravity is not None:
        s.set_gravity(gravity)
    if floor_friction is not None:
        s.set_floor_friction(floor_friction)
    s.add_particles(pos, vel, mass)
    return s


def cpu_solver(kind, dx, pos, vel=None, mass=None, E=1e5, nu=0.3, rho=1500.0, alpha=None, gravity=None,
               floor_friction=None):
    s = O.CpuSolver(kind, dx)
    s.set_material(E, nu, rho)
    if alpha is not None:
        s.set_plastic_alpha(alpha)
    if gravity is not None:
        s.set_gravity(gravity)
    if floor_friction is not None:
        s.set_floor_friction(floor_friction)
    s.add_particles(pos, vel, mass)
    return s


def scene_solvers(sc, kind):
    g = gpu_solver(sc.dx, sc.position, None, sc.mass, sc.E, sc.nu, sc.rho, sc.alpha, domain=sc.domain)
    c = cpu_solver(kind, sc.dx, sc.position, None, sc.mass, sc.E, sc.nu, sc.rho, sc.alpha)
    return g, c


def max_err_dx(a, b, dx):
    return float(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).max() / dx)


def dense_index(grid, ijk):
    o = grid["origin"]
    e = grid["mass"].shape
    ijk = np.asarray(ijk)
    return ((ijk[:, 0] - o[0]) * e[1] + (ijk[:, 1] - o[1])) * e[2] + (ijk[:, 2] - o[2])
