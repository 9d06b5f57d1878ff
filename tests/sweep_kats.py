"""The reference's sweep-coupler invariants for M4.5a
(tests/test_mpm_rigid_sweep.cpp:70-154), as cases plus the checks they make,
for the oracle (CPU) and the CUDA coupler. A 5 x n x 5 patch of nodes of mass
0.01 on a dx = 0.1 grid and a 0.4 m unit box with identity orientation.

Kept: MassConservationAfterOneApplyLayerA (:70-82), EmptyGridReturnsZeroReaction
(:111-118), NormalisedMassMatchesBodyMass (:123-131), ZeroDtIsHarmless
(:135-143). The layer B and C cases test the M4.5b / M4.5 couplers."""
import numpy as np


def patch(layers, mass=0.01):
    ijk = np.array([(i, j, k) for i in range(-2, 3) for j in range(layers) for k in range(-2, 3)], np.int32)
    return ijk, np.zeros((len(ijk), 3), np.float32), np.full(len(ijk), mass, np.float32)


def box(centre=(0.0, 0.5, 0.0), mass=1.0):
    return dict(center=centre, half_extents=(0.2, 0.2, 0.2), orientation=(1.0, 0.0, 0.0, 0.0),
                linear_velocity=(0.0, 0.0, 0.0), angular_velocity=(0.0, 0.0, 0.0), friction=0.5, mass=mass,
                shape=0)


CASES = [
    dict(name="MassConservationAfterOneApplyLayerA", layers=3, body=box(), dt=1.0 / 240.0),
    dict(name="EmptyGridReturnsZeroReaction", layers=0, body=box(), dt=1.0 / 240.0),
    dict(name="NormalisedMassMatchesBodyMass", layers=4, body=box((0.0, 0.15, 0.0)), dt=1.0 / 240.0),
    dict(name="ZeroDtIsHarmless", layers=3, body=box(), dt=0.0),
]


def check(case, before, after, force, torque, nodes_inside):
    name = case["name"]
    if name in ("MassConservationAfterOneApplyLayerA", "NormalisedMassMatchesBodyMass"):
        assert abs((after - before) - case["body"]["mass"]) <= 1e-3, (name, after - before)
    elif name == "EmptyGridReturnsZeroReaction":
        assert np.linalg.norm(force) <= 1e-9 and np.linalg.norm(torque) <= 1e-9 and nodes_inside == 0, name
    elif name == "ZeroDtIsHarmless":
        assert np.linalg.norm(force) <= 1e-9 and np.linalg.norm(torque) <= 1e-9, name
