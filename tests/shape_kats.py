"""The reference's cylinder inside-test known answers
(tests/test_mpm_rigid_cylinder.cpp:37-255), probed through the M1 coupler.

``shape_inside`` (include/basements/physics/coupling/mpm_rigid_coupler.h:90-103)
is not an entry point of its own: on this path it runs inside M1, which gives
every node it finds inside the body the body's per-node mass
(mpm_rigid_coupler_pic.h:150-166). So one probe seeds a single node of mass 1
at rest, places the cylinder so that the node sits at the KAT's world point,
calls the coupler once and reads whether the node's mass grew.

The normal, AABB and overlap-fraction KATs of the same file test helpers that
only the sweep couplers (M4.5a/b) call; they are not on the M1 path.
"""
from __future__ import annotations

import math

import numpy as np

from tests.m1_scene_loop import _quat_mul

f32 = np.float32
R, L = 0.15, 0.05
DX = 0.01
PI = f32(3.14159265358979)


def axis_angle(axis, angle):
    """Quaternion::from_axis_angle (quaternion.h:36-46) in float32."""
    h = f32(f32(angle) * f32(0.5))
    s, c = f32(math.sin(float(h))), f32(math.cos(float(h)))
    return (c, f32(axis[0] * s), f32(axis[1] * s), f32(axis[2] * s))


IDENTITY = (f32(1), f32(0), f32(0), f32(0))
ROLLED = axis_angle((1, 0, 0), f32(PI * f32(0.5)))

# name, world point relative to the centre, orientation, expected inside
KATS = [
    ("UprightCenterIsInside", (0.0, 0.0, 0.0), IDENTITY, True),          # :43-49
    ("UprightOutsideRadius", (0.20, 0.0, 0.0), IDENTITY, False),         # :51-55
    ("UprightOutsideAxialClipping", (0.0, 0.10, 0.0), IDENTITY, False),  # :57-61
    ("RolledConfigInsideAtCenter", (0.0, 0.0, 0.0), ROLLED, True),       # :92-101
    ("RolledConfigOutsideAlongWorldZAxis", (0.0, 0.0, 0.20), ROLLED, False),  # :103-112
    ("RolledConfigInsideAlongWorldXAxis", (0.10, 0.0, 0.0), ROLLED, True),    # :114-122
]


def rolling_probes(n=200):
    """RollingInsideMonotone (:221-255): a point swept along world x from
    -0.25 to 0.25 while the rolled cylinder spins about its own axis."""
    base = axis_angle((1, 0, 0), f32(f32(3.14159265) * f32(0.5)))
    out = []
    for i in range(n):
        x = f32(f32(-0.25) + f32(f32(0.50) * f32(f32(i) / f32(n - 1))))
        spin = axis_angle((0, 0, 1), f32(f32(i) * f32(0.05)))
        out.append(((x, 0.0, 0.0), _quat_mul(spin, base)))
    return out


def transitions(inside_seq):
    """The reference test's state machine: OUT_LEFT -> IN -> OUT_RIGHT."""
    state, n = 0, 0
    for inside in inside_seq:
        nxt = 1 if inside else (2 if state == 1 else state)
        if nxt != state:
            state, n = nxt, n + 1
    return n


def probe_body(point, q):
    """Collider fields that put node (0,0,0), at (0.5 dx)^3, on ``point``."""
    node = f32(f32(0.5) * f32(DX))
    center = tuple(f32(node - f32(p)) for p in point)
    return dict(center=center, half_extents=(R, L, R), orientation=q, linear_velocity=(0, 0, 0),
                angular_velocity=(0, 0, 0), friction=0.5, mass=1.0, shape=1)


def probe_gpu(bm, point, q):
    s = bm.MPMSolver(DX, domain=((-8, -8, -8), (16, 16, 16)))
    s.seed_grid(np.zeros((1, 3), np.int32), np.zeros((1, 3), np.float32), np.ones(1, np.float32))
    s.m1_apply(bm.make_collider(**probe_body(point, q)), 1.0 / 240.0)
    g = s.get_grid()
    o = np.asarray(g["origin"])
    return bool(g["mass"][-o[0], -o[1], -o[2]] > 1.0)


def probe_oracle(O, kind, point, q):
    s = O.CpuSolver(kind, DX)
    s.grid_seed(np.zeros((1, 3), np.int32), np.zeros((1, 3), np.float32), np.ones(1, np.float32))
    s.m1_apply(O.collider(**probe_body(point, q)), 1.0 / 240.0)
    n = s.grid_nodes()
    at = np.nonzero((n["ijk"] == 0).all(axis=1))[0][0]
    return bool(n["mass"][at] > 1.0)
