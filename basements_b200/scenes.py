"""Seeded synthetic scenes for the MLS-MPM soil step.

No public dataset is involved; every workload is generated here from a seed.

* ``sand_column``  — plain sand column collapse: 32^3 grid, dx = 1/32, cells
  [8,24) x [2,10) x [8,24) at 8 particles per cell (16,384 particles), uniform
  jitter drawn from MT19937(0) in the order x, y, z per particle with
  (i, j, k, q) lexicographic, the way ``std::uniform_real_distribution<float>``
  draws them; E = 3.5e5 Pa, nu = 0.3, rho = 1600, friction angle 30 deg,
  dt = 1e-4.
* ``wheel_rut``    — plain large rigid-wheel rut: 128^3 grid, dx = 1/128, sand
  bed of 128 x 40 x 128 cells at 8 ppc (5,242,880 candidates) subsampled
  without replacement to 2,000,000; M1 cylinder R = 0.1 m, width 0.08 m,
  5 kg, rolling about z at -2 rad/s while translating at 0.1 m/s; dt = 5e-5.
* ``scene_batch``  — uneven box-drop scenes for the batched form.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


def dp_alpha(friction_angle_deg: float) -> float:
    """alpha = sqrt(2/3) * 2 sin(phi) / (3 - sin(phi)) (mpm_solver.h:103)."""
    s = math.sin(math.radians(friction_angle_deg))
    return math.sqrt(2.0 / 3.0) * 2.0 * s / (3.0 - s)


def mt19937_uniform_f32(seed: int, n: int) -> np.ndarray:
    """n floats in [0, 1) as std::uniform_real_distribution<float>(0, 1) draws
    them from std::mt19937(seed): one 32-bit word per float, word / 2^32
    rounded to float, values that round to 1 moved to the largest float < 1."""
    rs = np.random.RandomState(seed)
    words = rs.randint(0, 2 ** 32, size=n, dtype=np.uint64).astype(np.uint32)
    u = words.astype(np.float32) / np.float32(2.0 ** 32)
    u[u >= 1.0] = np.nextafter(np.float32(1.0), np.float32(0.0))
    return u


@dataclass
class Body:
    center: tuple
    half_extents: tuple
    orientation: tuple = (1.0, 0.0, 0.0, 0.0)
    linear_velocity: tuple = (0.0, 0.0, 0.0)
    angular_velocity: tuple = (0.0, 0.0, 0.0)
    friction: float = 0.5
    mass: float = 1.0
    shape: int = 0
    kinematic: bool = True
    # body-space inverse inertia, row-major 3x3 (9 floats), applied to the
    # torque as the reference's integrator does; None: the identity the
    # reference's bodies start with
    inv_inertia: tuple | None = None

    def at_time(self, t: float) -> "Body":
        """Kinematic pose after time t (constant linear velocity; the angular
        velocity is exchanged with the grid but the pose is not rotated)."""
        c = tuple(float(self.center[a] + self.linear_velocity[a] * t) for a in range(3))
        return Body(c, self.half_extents, self.orientation, self.linear_velocity, self.angular_velocity,
                    self.friction, self.mass, self.shape, self.kinematic)

    def as_tuple(self):
        return dict(center=self.center, half_extents=self.half_extents, orientation=self.orientation,
                    linear_velocity=self.linear_velocity, angular_velocity=self.angular_velocity,
                    friction=self.friction, mass=self.mass, shape=self.shape)


@dataclass
class Scene:
    name: str
    dx: float
    grid: int
    position: np.ndarray
    mass: np.ndarray
    E: float
    nu: float
    rho: float
    alpha: float
    dt: float
    steps: int
    floor_friction: float = 0.4
    gravity: tuple = (0.0, -9.81, 0.0)
    bodies: list = field(default_factory=list)
    domain: tuple | None = None  # ((ox, oy, oz), (ex, ey, ez)) in nodes

    @property
    def n(self) -> int:
        return len(self.position)


def sand_column(cells=(16, 8, 16), offset=(8, 2, 8), ppc=8, grid=32, seed=0) -> Scene:
    dx = 1.0 / grid
    ci, cj, ck = cells
    n = ci * cj * ck * ppc
    u = mt19937_uniform_f32(seed, 3 * n).reshape(ci, cj, ck, ppc, 3)
    ii, jj, kk = np.meshgrid(np.arange(ci), np.arange(cj), np.arange(ck), indexing="ij")
    cell = np.stack([ii + offset[0], jj + offset[1], kk + offset[2]], -1).astype(np.float32)
    pos = ((cell[:, :, :, None, :] + u) * np.float32(dx)).astype(np.float32).reshape(-1, 3)
    rho = 1600.0
    m = np.float32(rho * dx ** 3 / ppc)
    return Scene("sand_column", dx, grid, pos, np.full(n, m, np.float32), 3.5e5, 0.3, rho, dp_alpha(30.0),
                 1e-4, 1000)


def pressed_box(inv_inertia=None) -> Scene:
    """The sand column with a rotated dynamic box pressed into its top
    surface, so that the coupler's torque spins the body from the first
    step (the box-drop scenes fall for hundreds of steps before contact)."""
    col = sand_column(cells=(16, 8, 16))
    q = np.array([0.95, 0.2, 0.15, 0.18])
    q = q / np.linalg.norm(q)
    body = Body(center=(0.37, 0.305, 0.38), half_extents=(0.06, 0.03, 0.045), orientation=tuple(float(v) for v in q),
                linear_velocity=(0.1, -0.4, 0.05), friction=0.5, mass=0.4, kinematic=False,
                inv_inertia=None if inv_inertia is None else tuple(float(v) for v in np.ravel(inv_inertia)))
    return Scene("pressed_box", col.dx, col.grid, col.position, col.mass, col.E, col.nu, col.rho, col.alpha, col.dt,
                 col.steps, bodies=[body])


def wheel_rut(n_keep=2_000_000, grid=128, bed_cells=(128, 40, 128), ppc=8, seed=1) -> Scene:
    dx = 1.0 / grid
    rng = np.random.default_rng(seed)
    ncand = bed_cells[0] * bed_cells[1] * bed_cells[2] * ppc
    keep = np.sort(rng.choice(ncand, size=min(n_keep, ncand), replace=False))
    cell_id = keep // ppc
    k = cell_id % bed_cells[2]
    j = (cell_id // bed_cells[2]) % bed_cells[1]
    i = cell_id // (bed_cells[2] * bed_cells[1])
    jit = rng.random((len(keep), 3), dtype=np.float32)
    pos = ((np.stack([i, j, k], -1).astype(np.float32) + jit) * np.float32(dx)).astype(np.float32)
    rho = 1600.0
    bed_vol = bed_cells[0] * bed_cells[1] * bed_cells[2] * dx ** 3
    m = np.float32(rho * bed_vol / len(keep))
    bed_top = bed_cells[1] * dx
    s45 = math.sqrt(0.5)
    wheel = Body(center=(0.3, bed_top + 0.1 - 0.01, 0.5), half_extents=(0.1, 0.04, 0.1),
                 orientation=(s45, s45, 0.0, 0.0), linear_velocity=(0.1, 0.0, 0.0),
                 angular_velocity=(0.0, 0.0, -2.0), friction=0.5, mass=5.0, shape=1, kinematic=True)
    margin = 16
    domain = ((-margin, -4, -margin), (grid + 2 * margin, bed_cells[1] + 40, grid + 2 * margin))
    return Scene("wheel_rut", dx, grid, pos, np.full(len(keep), m, np.float32), 3.5e5, 0.3, rho,
                 dp_alpha(30.0), 5e-5, 2000, bodies=[wheel], domain=domain)


def scaled_wheel_rut(n_keep: int, seed=1) -> Scene:
    """The wheel-rut scene with fewer particles kept (same bed and body)."""
    return wheel_rut(n_keep=n_keep, seed=seed)


def _sand_block(rng, G: int, N: int, ppc: int = 8):
    """A block of w x h x w cells at `ppc` jittered particles per cell, centred
    in x/z on the floor, h ~ w/2; the first N particles of it."""
    dx = 1.0 / G
    cells = max(1, N // ppc)
    w = max(2, min(G - 8, int(round((cells / 0.5) ** (1.0 / 3.0)))))
    h = max(1, int(math.ceil(cells / (w * w))))
    ncell = w * w * h
    pos = np.empty((ncell * ppc, 3), np.float32)
    ii, jj, kk = np.meshgrid(np.arange(w), np.arange(h), np.arange(w), indexing="ij")
    base = np.stack([ii + (G - w) // 2, jj, kk + (G - w) // 2], -1).reshape(-1, 3).astype(np.float32)
    jit = rng.random((ncell, ppc, 3), dtype=np.float32)
    pos[:] = ((base[:, None, :] + jit) * np.float32(dx)).reshape(-1, 3)
    return pos[:N], h


def _stable_dt(E, nu, rho, dx):
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    return min(2e-4, 0.5 * dx / math.sqrt((lam + 2 * mu) / rho))


def box_drop_scene(seed: int, grid: int | None = None, n_particles: int | None = None) -> Scene:
    """One uneven batched scene: grid side in {32,48,64,96}, particle count
    log-uniform 8k-400k at 8 ppc, friction angle U[25,40] deg, E log-uniform
    [1e5, 1e6], a dynamic box of side U[0.05, 0.2] m with a random pose dropped
    at U[0, 1] m/s."""
    rng = np.random.default_rng(1000 + seed)
    G = grid or int(rng.choice([32, 48, 64, 96]))
    N = n_particles or int(math.exp(rng.uniform(math.log(8e3), math.log(4e5))))
    dx = 1.0 / G
    ppc = 8
    pos, h = _sand_block(rng, G, N, ppc)
    rho = 1600.0
    E = float(math.exp(rng.uniform(math.log(1e5), math.log(1e6))))
    phi = float(rng.uniform(25.0, 40.0))
    side = float(rng.uniform(0.05, 0.2))
    q = rng.normal(size=4)
    q = q / np.linalg.norm(q)
    top = (h + 2) * dx
    body = Body(center=(0.5, top + side, 0.5), half_extents=(side / 2,) * 3, orientation=tuple(map(float, q)),
                linear_velocity=(0.0, -float(rng.uniform(0.0, 1.0)), 0.0), mass=float(rho * side ** 3),
                shape=0, kinematic=False)
    nu = 0.3
    dt = _stable_dt(E, nu, rho, dx)
    m = np.float32(rho * dx ** 3 / ppc)
    return Scene(f"box_drop_{seed}", dx, G, pos, np.full(len(pos), m, np.float32), E, nu, rho, dp_alpha(phi),
                 dt, 500, bodies=[body])


def serve_request_scene(seed: int) -> Scene:
    """One request of the serving stream: grid side uniform in [32, 128],
    particle count log-uniform in [10k, 1M] (capped at 8 ppc over a quarter of
    the G^3 box, so that the bed fits its grid), 100-2000 steps, friction angle
    U[25, 40] deg on the sand-column material (E = 3.5e5 Pa, nu = 0.3,
    rho = 1600 kg/m^3). With probability 1/2 a dynamic rigid body, a box or a
    cylinder with equal probability (side / diameter U[0.05, 0.2] m, random
    pose, dropped at U[0, 1] m/s), falls on the bed. The grid box spans G/2
    cells beyond the bed on each side in x and z, so that the runout of the
    sand stays inside it."""
    rng = np.random.default_rng(500_000 + seed)
    G = int(rng.integers(32, 129))
    n_cap = int(8 * 0.25 * G ** 3)
    N = min(n_cap, int(math.exp(rng.uniform(math.log(1e4), math.log(1e6)))))
    steps = int(rng.integers(100, 2001))
    dx = 1.0 / G
    pos, h = _sand_block(rng, G, N, 8)
    rho, E, nu = 1600.0, 3.5e5, 0.3
    phi = float(rng.uniform(25.0, 40.0))
    bodies = []
    if rng.random() < 0.5:
        shape = int(rng.random() < 0.5)
        side = float(rng.uniform(0.05, 0.2))
        q = rng.normal(size=4)
        q = q / np.linalg.norm(q)
        he = (side / 2, side / 2, side / 2)
        mass = rho * side ** 3 if shape == 0 else rho * math.pi * (side / 2) ** 2 * side
        bodies.append(Body(center=(0.5, (h + 2) * dx + side, 0.5), half_extents=he,
                           orientation=tuple(map(float, q)),
                           linear_velocity=(0.0, -float(rng.uniform(0.0, 1.0)), 0.0), mass=float(mass),
                           shape=shape, kinematic=False))
    m = np.float32(rho * dx ** 3 / 8)
    dom = ((-G // 2, -4, -G // 2), (2 * G, G + 8, 2 * G))
    return Scene(f"request_{seed}", dx, G, pos, np.full(len(pos), m, np.float32), E, nu, rho, dp_alpha(phi),
                 _stable_dt(E, nu, rho, dx), steps, bodies=bodies, domain=dom)


def tine_pass(grid=64, bed_cells=(64, 16, 64), ppc=4, n_waypoints=16, steps=200, dt=1e-4,
              tine_half=(0.01, 0.05, 0.025), depth=0.03, speed=1.0, jitter=2.5e-4, seed=0):
    """Differentiable tine pass: a sand bed of bed_cells at `ppc` jittered
    particles per cell (64 x 16 x 64 at 4 ppc = 262,144 particles on the
    64^3 grid), the sand-column material at a 30 deg friction angle, and a
    kinematic box tine (half extents 0.01 x 0.05 x 0.025 m, steel density)
    dragged `depth` deep through the bed along +x at `speed` m/s; its path is
    `n_waypoints` seeded control points (the straight drag plus N(0, jitter)
    per coordinate), linearly interpolated over steps*dt. Returns
    (scene, body template, waypoints (n_waypoints x 3, float32), target
    heightfield (grid x grid, float64)); the target is the bed's initial
    heightfield plus a seeded smooth bump pattern of +-2 mm."""
    rng = np.random.default_rng(3000 + seed)
    dx = 1.0 / grid
    ci, cj, ck = bed_cells
    ii, jj, kk = np.meshgrid(np.arange(ci), np.arange(cj), np.arange(ck), indexing="ij")
    base = np.stack([ii, jj, kk], -1).reshape(-1, 3).astype(np.float32)
    jit = rng.random((len(base), ppc, 3), dtype=np.float32)
    pos = ((base[:, None, :] + jit) * np.float32(dx)).reshape(-1, 3)
    rho, E, nu = 1600.0, 3.5e5, 0.3
    m = np.float32(rho * dx ** 3 / ppc)
    top = cj * dx
    hx, hy, hz = tine_half
    c0 = np.array([0.3, top - depth + hy, 0.5])
    T = steps * float(np.float32(dt))
    t = np.linspace(0.0, 1.0, n_waypoints)[:, None]
    wp = c0[None, :] + t * np.array([speed * T, 0.0, 0.0])[None, :] + rng.normal(0.0, jitter, (n_waypoints, 3))
    body = Body(center=tuple(map(float, wp[0])), half_extents=tuple(tine_half), orientation=(1.0, 0.0, 0.0, 0.0),
                linear_velocity=(0.0, 0.0, 0.0), mass=float(7850.0 * 8 * hx * hy * hz), shape=0, kinematic=True)
    h0 = heightfield(pos, grid)[0]
    ph = rng.uniform(0, 2 * math.pi, 2)
    u = (np.arange(grid) + 0.5) / grid
    bump = 0.002 * np.sin(2 * math.pi * 3 * u[:, None] + ph[0]) * np.sin(2 * math.pi * 2 * u[None, :] + ph[1])
    dom = ((-8, -4, -8), (grid + 16, int(0.6 * grid) + 8, grid + 16))
    sc = Scene(f"tine_pass_{seed}", dx, grid, pos, np.full(len(pos), m, np.float32), E, nu, rho, dp_alpha(30.0),
               float(np.float32(dt)), steps, bodies=[body], domain=dom)
    return sc, body, wp.astype(np.float32), h0 + bump


def body_on_path(body: Body, waypoints, n_steps: int, dt: float, n: int) -> Body:
    """The body of step n on the piecewise-linear waypoint path spread over
    n_steps*dt: centre on the path, linear velocity = the segment's slope
    (double arithmetic, rounded to float32 at the end, as bm_tape_forward)."""
    wp = np.asarray(waypoints, np.float32).astype(np.float64)
    dt = float(np.float32(dt))
    seg = (n_steps * dt) / (len(wp) - 1)
    tn = n * dt
    k = min(max(int(math.floor(tn / seg)), 0), len(wp) - 2)
    v = [(wp[k + 1, a] - wp[k, a]) / seg for a in range(3)]
    c = [wp[k, a] + (tn - k * seg) * v[a] for a in range(3)]
    return Body(center=tuple(float(np.float32(x)) for x in c), half_extents=body.half_extents,
                orientation=body.orientation, linear_velocity=tuple(float(np.float32(x)) for x in v),
                angular_velocity=body.angular_velocity, friction=body.friction, mass=body.mass, shape=body.shape,
                kinematic=body.kinematic)


def heightfield(pos, nbins: int):
    """Soft heightfield of particles over x, z in [0, 1): per bin b the
    weighted mean height H_b = sum_p W_bp y_p / sum_p W_bp, W the bilinear
    tent of one bin width around the bin centre (continuous in the
    positions). Returns (H, S, parts) with S the weight sums; `parts` is kept
    for heightfield_loss."""
    p = np.asarray(pos, np.float64)
    u = p[:, 0] * nbins - 0.5
    w = p[:, 2] * nbins - 0.5
    i0 = np.floor(u).astype(np.int64)
    j0 = np.floor(w).astype(np.int64)
    fu, fw = u - i0, w - j0
    S = np.zeros(nbins * nbins)
    Y = np.zeros(nbins * nbins)
    parts = []
    for di in (0, 1):
        for dj in (0, 1):
            bi, bj = i0 + di, j0 + dj
            wu = fu if di else 1.0 - fu
            wv = fw if dj else 1.0 - fw
            ok = (bi >= 0) & (bi < nbins) & (bj >= 0) & (bj < nbins)
            idx = np.where(ok, bi * nbins + bj, 0)
            wt = np.where(ok, wu * wv, 0.0)
            S += np.bincount(idx, wt, nbins * nbins)
            Y += np.bincount(idx, wt * p[:, 1], nbins * nbins)
            parts.append((idx, ok, wu, wv, 1.0 if di else -1.0, 1.0 if dj else -1.0))
    H = np.where(S > 0, Y / np.where(S > 0, S, 1.0), 0.0)
    return H.reshape(nbins, nbins), S.reshape(nbins, nbins), parts


def heightfield_loss(pos, target):
    """L = sum_b (H_b - target_b)^2 over the bins holding particles, and
    dL/d position (n x 3, float64)."""
    nbins = target.shape[0]
    H, S, parts = heightfield(pos, nbins)
    p = np.asarray(pos, np.float64)
    live = S > 0
    r = np.where(live, 2.0 * (H - target), 0.0).ravel()
    Sf = np.where(live, S, 1.0).ravel()
    Hf = H.ravel()
    L = float(np.sum(np.where(live, (H - target) ** 2, 0.0)))
    g = np.zeros_like(p)
    for idx, ok, wu, wv, su, sv in parts:
        rb = np.where(ok, r[idx] / Sf[idx], 0.0)
        dy = p[:, 1] - Hf[idx]
        g[:, 1] += rb * wu * wv
        g[:, 0] += rb * dy * su * wv * nbins
        g[:, 2] += rb * dy * wu * sv * nbins
    return L, g
