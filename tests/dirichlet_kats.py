"""The reference's M0 Dirichlet coupler unit tests
(tests/test_mpm_rigid_coupler.cpp:26-92), as data plus the checks they make,
for the oracle (CPU) and the CUDA coupler. One node of mass 1 on a dx = 0.1
grid, dt = 1/60; bodies are boxes with the test's default pose (identity
orientation, zero velocities, friction 0.5 unless set)."""
import numpy as np


def _box(center, half, friction=0.5, linear_velocity=(0.0, 0.0, 0.0)):
    return dict(center=center, half_extents=half, orientation=(1.0, 0.0, 0.0, 0.0),
                linear_velocity=linear_velocity, angular_velocity=(0.0, 0.0, 0.0), friction=friction,
                mass=1.0, shape=0)


CASES = [
    # :30-46 BasicReactionForce: upward jet just inside the bottom face
    dict(name="BasicReactionForce", node=(0, 0, 0), vel=(0.0, 5.0, 0.0),
         body=_box((0.05, 0.5, 0.05), (0.5, 0.55, 0.5))),
    # :48-59 OutsideBodyNoReaction
    dict(name="OutsideBodyNoReaction", node=(20, 20, 20), vel=(0.0, -5.0, 0.0),
         body=_box((0.0, 0.0, 0.0), (0.5, 0.5, 0.5))),
    # :61-74 TangentialFrictionTransfers
    dict(name="TangentialFrictionTransfers", node=(0, 0, 0), vel=(5.0, 0.0, 0.0),
         body=_box((0.05, 0.0, 0.05), (0.5, 0.5, 0.5), friction=1.0)),
    # :76-92 AngularReactionAtOffset
    dict(name="AngularReactionAtOffset", node=(3, 0, 0), vel=(0.0, -5.0, 0.0),
         body=_box((0.05, 0.0, 0.05), (0.5, 0.5, 0.5))),
]


def check(case, force, torque, nodes_inside, node_velocity):
    name = case["name"]
    if name == "BasicReactionForce":
        assert nodes_inside > 0 and force[1] > 0.0 and node_velocity[1] <= 1e-5, name
    elif name == "OutsideBodyNoReaction":
        assert nodes_inside == 0 and np.linalg.norm(force) <= 1e-6 and np.linalg.norm(torque) <= 1e-6, name
    elif name == "TangentialFrictionTransfers":
        assert abs(node_velocity[0]) <= 1e-4, name
    elif name == "AngularReactionAtOffset":
        assert nodes_inside > 0 and np.linalg.norm(torque) > 1e-3, name
