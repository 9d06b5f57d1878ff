"""The reference's angle-of-repose scene (a particle run, no body):
research/mpm_rigid_coupling/bench_compare_all.cpp:293-371 with
research/mpm_rigid_coupling/scenarios/scenario_repose_pile.h.

A 7x5x7 column of 245 particles at 12.5 mm spacing collapses for 2 s at
dt = 1/960 on a dx = 25 mm grid (E = 5e5, nu = 0.3, rho = 1500, alpha = 0.55,
floor friction 0.6); ``measure_pile`` restates the reference's pile metrics
(scenario_repose_pile.h:86-171) in float32.
"""
from __future__ import annotations

import math

import numpy as np

f32 = np.float32
DX = 0.025
DT = 1.0 / 960.0
STEPS = 1920
MATERIAL = dict(E=5.0e5, nu=0.30, rho=1500.0, alpha=0.55, floor_friction=0.60)
SPACING = f32(0.0125)
BASE = (f32(0.0), f32(0.0125), f32(0.0))
NX, NY, NZ = 7, 5, 7
DOMAIN = ((-16, -4, -16), (32, 16, 32))


def column():
    """seed_repose_column (scenario_repose_pile.h:54-72): positions, masses."""
    pos = []
    for i in range(NX):
        for j in range(NY):
            for k in range(NZ):
                ox = f32(f32(f32(i) - f32(f32(NX) * f32(0.5))) + f32(0.5))
                oz = f32(f32(f32(k) - f32(f32(NZ) * f32(0.5))) + f32(0.5))
                pos.append((f32(BASE[0] + f32(ox * SPACING)), f32(BASE[1] + f32(f32(j) * SPACING)),
                            f32(BASE[2] + f32(oz * SPACING))))
    pos = np.array(pos, np.float32)
    return pos, np.full(len(pos), 2.93e-3, np.float32)


def measure_pile(pos, vel):
    """measure_pile (scenario_repose_pile.h:86-171): height, radius, slope
    angle of the binned surface, geometric angle atan(h / r), particles with
    |v| < 0.01."""
    pos = np.asarray(pos, np.float32)
    vel = np.asarray(vel, np.float32)
    speed = np.sqrt((vel.astype(np.float64) ** 2).sum(1))
    at_rest = int((speed < 0.01).sum())
    height = float(pos[:, 1].max())
    nbins = 24
    bin_dr = f32(f32(f32(1.5) * f32(f32(NX) * SPACING)) / f32(nbins))
    sy = np.full(nbins, -1.0, np.float32)
    sr = np.zeros(nbins, np.float32)
    r_outer = f32(0)
    for p in pos:
        dxh, dzh = f32(p[0] - BASE[0]), f32(p[2] - BASE[2])
        r = f32(np.sqrt(f32(f32(dxh * dxh) + f32(dzh * dzh))))
        r_outer = max(r_outer, r)
        b = int(r / bin_dr)
        if 0 <= b < nbins and p[1] > sy[b]:
            sy[b], sr[b] = p[1], r
    crest = int(np.argmax(sy))
    sel = [b for b in range(crest, nbins) if sy[b] >= 0 and sy[b] >= f32(0.005)]
    angle = 0.0
    if len(sel) >= 2:
        r_, y_ = sr[sel].astype(np.float64), sy[sel].astype(np.float64)
        n = len(sel)
        denom = n * (r_ * r_).sum() - r_.sum() ** 2
        if abs(denom) > 1e-9:
            angle = math.degrees(math.atan(abs((n * (r_ * y_).sum() - r_.sum() * y_.sum()) / denom)))
    geom = math.degrees(math.atan(height / float(r_outer))) if r_outer > 1e-6 else 0.0
    return dict(height=height, radius=float(r_outer), angle_slope=angle, angle_geom=geom, at_rest=at_rest)
