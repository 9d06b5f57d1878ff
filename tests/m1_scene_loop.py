"""The reference's grid-only research scenes for the tests: the scenario
registry and harness loop of basements_b200.research (which restates
research/mpm_rigid_coupling/bench_compare_all.cpp), plus an adapter that
puts the CPU oracle (reference build or float restatement) behind the same
loop. Only the tests use the oracle adapter.
"""
from __future__ import annotations

import numpy as np

from basements_b200.research import (DRIFT_COLUMNS, SCENES, GpuGrid, _quat_mul, _seed_block, f32, rebound,  # noqa: F401
                                     run, tine_start, tine_summary)


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
        return n["ijk"][sel], v, n["mass"][sel]


def first_divergence(a, b, atol):
    """First row index where |a - b| > atol in any column, or None."""
    bad = np.nonzero((np.abs(a - b) > atol).any(axis=1))[0]
    return int(bad[0]) if len(bad) else None
