"""ctypes access to the CPU checkers (TEST INFRASTRUCTURE ONLY).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg
import this module. The product (``basements_b200``) never does.

Three libraries export the interface of ``oracle/oracle_api.h``:

* ``oracle/_ref/libref_mpm.so`` (prefix ``ref``): the reference's own
  ``MPMSolver`` / ``MPMRigidCouplerPIC`` / ``TimeIntegrator`` compiled from its
  headers by ``oracle/Makefile``;
* ``oracle/liboracle_mpm_f32.so`` and ``liboracle_mpm_f64.so`` (prefix
  ``orc``): the restatement in ``oracle/mpm_oracle.hpp`` in float and double.

``CpuSolver`` mirrors the reference ``MPMSolver`` method names
(include/basements/physics/mpm/mpm_solver.h:19-95) with numpy SoA arrays.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

LIBS = {
    "ref": os.path.join(HERE, "_ref", "libref_mpm.so"),
    "f32": os.path.join(HERE, "liboracle_mpm_f32.so"),
    "f64": os.path.join(HERE, "liboracle_mpm_f64.so"),
}
PREFIX = {"ref": "ref", "f32": "orc", "f64": "orc"}

_f = C.POINTER(C.c_float)
_i32 = C.POINTER(C.c_int32)
_u8 = C.POINTER(C.c_uint8)


class OrcCollider(C.Structure):
    _fields_ = [
        ("center", C.c_float * 3),
        ("orientation", C.c_float * 4),
        ("half_extents", C.c_float * 3),
        ("linear_velocity", C.c_float * 3),
        ("angular_velocity", C.c_float * 3),
        ("friction", C.c_float),
        ("mass", C.c_float),
        ("shape", C.c_int32),
    ]


_loaded: dict = {}


def available(kind: str) -> bool:
    return os.path.exists(LIBS[kind])


def load(kind: str):
    """Load one checker library ("ref", "f32" or "f64")."""
    if kind in _loaded:
        return _loaded[kind]
    path = LIBS[kind]
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built (run `make -C oracle`)")
    lib = C.CDLL(path)
    p = PREFIX[kind]

    def fn(name, res, *args):
        f = getattr(lib, f"{p}_{name}")
        f.restype = res
        f.argtypes = list(args)
        return f

    api = {
        "precision_bytes": fn("precision_bytes", C.c_int),
        "create": fn("create", C.c_void_p, C.c_float),
        "destroy": fn("destroy", None, C.c_void_p),
        "set_material": fn("set_material", None, C.c_void_p, C.c_float, C.c_float, C.c_float),
        "set_gravity": fn("set_gravity", None, C.c_void_p, C.c_float, C.c_float, C.c_float),
        "set_plastic_alpha": fn("set_plastic_alpha", None, C.c_void_p, C.c_float),
        "set_floor_friction": fn("set_floor_friction", None, C.c_void_p, C.c_float),
        "add_particles": fn("add_particles", None, C.c_void_p, C.c_int64, _f, _f, _f),
        "num_particles": fn("num_particles", C.c_int64, C.c_void_p),
        "set_particle_state": fn("set_particle_state", None, C.c_void_p, C.c_int64, C.c_int64, _f, _f, _f, _f),
        "get_particles": fn("get_particles", None, C.c_void_p, _f, _f, _f, _f, _f, _f),
        "get_state_f64": fn("get_state_f64", None, C.c_void_p, *([C.POINTER(C.c_double)] * 4)),
        "set_state_f64": fn("set_state_f64", None, C.c_void_p, C.c_int64, C.c_int64,
                            *([C.POINTER(C.c_double)] * 4)),
        "step": fn("step", None, C.c_void_p, C.c_float, C.c_int),
        "p2g": fn("p2g", None, C.c_void_p, C.c_float),
        "grid_update": fn("grid_update", None, C.c_void_p, C.c_float),
        "g2p": fn("g2p", None, C.c_void_p, C.c_float),
        "m1_apply": fn("m1_apply", C.c_int, C.c_void_p, C.POINTER(OrcCollider), C.c_float, _f),
        "m45a_apply": fn("m45a_apply", C.c_int, C.c_void_p, C.POINTER(OrcCollider), C.c_float, _f),
        "m0_apply": fn("m0_apply", C.c_int, C.c_void_p, C.POINTER(OrcCollider), C.c_float, _f),
        "m45b_apply": fn("m45b_apply", C.c_int, C.c_void_p, C.POINTER(OrcCollider), C.c_float, _f),
        "m45c_apply": fn("m45c_apply", C.c_int, C.c_void_p, C.POINTER(OrcCollider), C.c_float, _f),
        "grid_num_nodes": fn("grid_num_nodes", C.c_int64, C.c_void_p),
        "grid_get": fn("grid_get", C.c_int64, C.c_void_p, _i32, _f, _f, _f, _u8, C.c_int64),
        "grid_seed": fn("grid_seed", None, C.c_void_p, C.c_int64, _i32, _f, _f),
        "box_drop_m1": fn("box_drop_m1", C.c_int, _f, C.c_int),
        "svd": fn("svd", None, C.c_int64, _f, _f, _f, _f),
        "run_dynamic_body": fn("run_dynamic_body", None, C.c_void_p, C.POINTER(OrcCollider), C.c_float, C.c_float,
                               C.c_float, C.c_float, C.c_int, _f),
    }
    if hasattr(lib, f"{p}_decisions_read"):
        api["decisions_enable"] = fn("decisions_enable", None, C.c_void_p, C.c_int)
        api["decisions_read"] = fn("decisions_read", None, C.c_void_p, C.POINTER(C.c_uint64))
        api["tape_new"] = fn("tape_new", C.c_void_p)
        api["tape_free"] = fn("tape_free", None, C.c_void_p)
        api["solver_use_tape"] = fn("solver_use_tape", None, C.c_void_p, C.c_void_p, C.c_int)
        api["tape_status"] = fn("tape_status", None, C.c_void_p, C.POINTER(C.c_int64))
        api["tape_export"] = fn("tape_export", None, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                C.POINTER(C.c_int64))
        api["tape_import"] = fn("tape_import", None, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p,
                                C.c_void_p)
    _loaded[kind] = api
    return api


def _p(a):
    if a is None:
        return None
    return a.ctypes.data_as(_f)


def collider(center, half_extents, orientation=(1.0, 0.0, 0.0, 0.0), linear_velocity=(0, 0, 0),
             angular_velocity=(0, 0, 0), friction=0.5, mass=1.0, shape=0) -> OrcCollider:
    c = OrcCollider()
    c.center[:] = list(map(float, center))
    c.orientation[:] = list(map(float, orientation))
    c.half_extents[:] = list(map(float, half_extents))
    c.linear_velocity[:] = list(map(float, linear_velocity))
    c.angular_velocity[:] = list(map(float, angular_velocity))
    c.friction = float(friction)
    c.mass = float(mass)
    c.shape = int(shape)
    return c


class CpuSolver:
    """One CPU solver instance ("ref", "f32" or "f64")."""

    def __init__(self, kind: str, dx: float):
        self.kind = kind
        self.api = load(kind)
        self.h = self.api["create"](float(dx))

    def close(self):
        if self.h:
            self.api["destroy"](self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- reference MPMSolver API --------------------------------------------
    def set_material(self, E, nu, rho):
        self.api["set_material"](self.h, E, nu, rho)

    def set_gravity(self, g):
        self.api["set_gravity"](self.h, *map(float, g))

    def set_plastic_alpha(self, a):
        self.api["set_plastic_alpha"](self.h, a)

    def set_floor_friction(self, mu):
        self.api["set_floor_friction"](self.h, mu)

    def add_particles(self, pos, vel=None, mass=None):
        pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
        vel = None if vel is None else np.ascontiguousarray(vel, np.float32).reshape(-1, 3)
        mass = None if mass is None else np.ascontiguousarray(np.broadcast_to(np.float32(mass), (len(pos),)) if np.ndim(mass) == 0 else mass, np.float32)
        self.api["add_particles"](self.h, len(pos), _p(pos), _p(vel), _p(mass))

    def num_particles(self) -> int:
        return int(self.api["num_particles"](self.h))

    def set_particle_state(self, first=0, pos=None, vel=None, F=None, C_=None):
        arrs = [None if a is None else np.ascontiguousarray(a, np.float32) for a in (pos, vel, F, C_)]
        n = next(len(a.reshape(len(a), -1)) for a in arrs if a is not None)
        self.api["set_particle_state"](self.h, first, n, *[_p(a) for a in arrs])

    def get_particles(self):
        n = self.num_particles()
        out = {
            "position": np.empty((n, 3), np.float32),
            "velocity": np.empty((n, 3), np.float32),
            "F": np.empty((n, 3, 3), np.float32),
            "C": np.empty((n, 3, 3), np.float32),
            "mass": np.empty(n, np.float32),
            "volume": np.empty(n, np.float32),
        }
        self.api["get_particles"](self.h, *[_p(out[k]) for k in ("position", "velocity", "F", "C", "mass", "volume")])
        return out

    def state_f64(self):
        """x, v (n x 3) and F, C (n x 3 x 3) in the solver's own precision, as double."""
        n = self.num_particles()
        out = {"position": np.empty((n, 3)), "velocity": np.empty((n, 3)), "F": np.empty((n, 3, 3)),
               "C": np.empty((n, 3, 3))}
        dp = C.POINTER(C.c_double)
        self.api["get_state_f64"](self.h, *[out[k].ctypes.data_as(dp) for k in ("position", "velocity", "F", "C")])
        return out

    def set_state_f64(self, pos=None, vel=None, F=None, C_=None):
        """Overwrite x, v, F, C of all particles from double arrays (the f64
        solver keeps them in double; the float ones round)."""
        arrs = [None if a is None else np.ascontiguousarray(a, np.float64) for a in (pos, vel, F, C_)]
        dp = C.POINTER(C.c_double)
        self.api["set_state_f64"](self.h, 0, self.num_particles(),
                                  *[None if a is None else a.ctypes.data_as(dp) for a in arrs])

    def positions_f64(self):
        """Positions in the solver's own precision, as double."""
        return self.state_f64()["position"]

    def step(self, dt, n_steps=1):
        self.api["step"](self.h, dt, int(n_steps))

    # -- split phases (coupler contract) -----------------------------------
    def p2g(self, dt):
        self.api["p2g"](self.h, dt)

    def grid_update(self, dt):
        self.api["grid_update"](self.h, dt)

    def g2p(self, dt):
        self.api["g2p"](self.h, dt)

    def m1_apply(self, body: OrcCollider, dt):
        r = np.zeros(6, np.float32)
        n = self.api["m1_apply"](self.h, C.byref(body), dt, _p(r))
        return r[:3].copy(), r[3:].copy(), int(n)

    def m0_apply(self, body: OrcCollider, dt):
        """The M0 Dirichlet coupler (mpm_rigid_coupler.cpp:58-143)."""
        r = np.zeros(6, np.float32)
        n = self.api["m0_apply"](self.h, C.byref(body), dt, _p(r))
        return r[:3].copy(), r[3:].copy(), int(n)

    def _coupler(self, name, body, dt):
        r = np.zeros(6, np.float32)
        n = self.api[name](self.h, C.byref(body), dt, _p(r))
        return r[:3].copy(), r[3:].copy(), int(n)

    def m45b_apply(self, body: OrcCollider, dt):
        """M4.5b: M4.5a plus the friction tangent (m4_5_hybrid.h:259-275)."""
        return self._coupler("m45b_apply", body, dt)

    def m45c_apply(self, body: OrcCollider, dt):
        """M4.5 = M4_5c: M4.5b with the B-spline mass weight (m4_5_hybrid.h:282-305)."""
        return self._coupler("m45c_apply", body, dt)

    def m45a_apply(self, body: OrcCollider, dt):
        """The M4.5a two-pass sweep coupler (m4_5_hybrid.h:104-257)."""
        r = np.zeros(6, np.float32)
        n = self.api["m45a_apply"](self.h, C.byref(body), dt, _p(r))
        return r[:3].copy(), r[3:].copy(), int(n)

    def run_dynamic_body(self, body: OrcCollider, gravity, dt, n_steps, inv_inertia=None):
        """n coupled steps with a dynamic body (updated in place and returned).
        inv_inertia: body-space inverse inertia (3x3), None for the identity
        the reference's bodies start with (rigid_body.h:121-122)."""
        ii = None if inv_inertia is None else np.ascontiguousarray(np.asarray(inv_inertia, np.float32).reshape(9))
        self.api["run_dynamic_body"](self.h, C.byref(body), *map(float, gravity), float(dt), int(n_steps),
                                     None if ii is None else _p(ii))
        return body

    def decisions(self, enable=None):
        """Restatement only: with enable=True/False turns the record of the
        run's discontinuous decisions on (cleared) or off; returns the record
        so far: (svd hash, inside hash, rotations, sweeps, inside count)."""
        if enable is not None:
            self.api["decisions_enable"](self.h, 1 if enable else 0)
        out = (C.c_uint64 * 5)()
        self.api["decisions_read"](self.h, out)
        return tuple(int(v) for v in out)

    def use_tape(self, tape: "DecisionTape | None", mode: str = "off"):
        """Restatement only: record this solver's discontinuous decisions into
        `tape` ("record"), take them from it ("replay"), or detach ("off")."""
        m = {"off": 0, "record": 1, "replay": 2}[mode]
        self.api["solver_use_tape"](self.h, tape.t if tape is not None else None, m)

    def grid_nodes(self):
        """Every node of every allocated 4^3 block, as a dict keyed by (i,j,k)."""
        cap = int(self.api["grid_num_nodes"](self.h))
        ijk = np.empty((cap, 3), np.int32)
        vel = np.empty((cap, 3), np.float32)
        frc = np.empty((cap, 3), np.float32)
        mass = np.empty(cap, np.float32)
        act = np.empty(cap, np.uint8)
        n = self.api["grid_get"](self.h, ijk.ctypes.data_as(_i32), _p(vel), _p(frc), _p(mass),
                                 act.ctypes.data_as(_u8), cap)
        return {"ijk": ijk[:n], "velocity": vel[:n], "force": frc[:n], "mass": mass[:n], "active": act[:n]}

    def grid_seed(self, ijk, vel, mass):
        ijk = np.ascontiguousarray(ijk, np.int32).reshape(-1, 3)
        vel = np.ascontiguousarray(vel, np.float32).reshape(-1, 3)
        mass = np.ascontiguousarray(mass, np.float32).reshape(-1)
        self.api["grid_seed"](self.h, len(ijk), ijk.ctypes.data_as(_i32), _p(vel), _p(mass))


class DecisionTape:
    """A record of a run's SVD and coupler-inside decisions (restatement
    only), replayed by other runs so that they follow the same branch."""

    def __init__(self, kind: str):
        self.api = load(kind)
        self.t = self.api["tape_new"]()

    def status(self):
        """(SVD calls recorded, replayed, coupler calls recorded, replayed,
        replay ran past the record)."""
        out = (C.c_int64 * 4)()
        self.api["tape_status"](self.t, out)
        return int(out[0]), int(out[1]), int(out[2]), int(out[3]) & ((1 << 40) - 1), bool(out[3] >> 40)

    def export(self):
        """(SVD codes uint16, inside keys int64, offsets int64) of the record."""
        sz = (C.c_int64 * 3)()
        self.api["tape_export"](self.t, None, None, None, sz)
        svd = np.empty(sz[0], np.uint16)
        keys = np.empty(sz[2], np.int64)
        offs = np.empty(sz[1] + 1, np.int64)
        self.api["tape_export"](self.t, svd.ctypes.data, keys.ctypes.data, offs.ctypes.data, sz)
        return svd, keys, offs

    def load(self, svd, keys, offs):
        """Replace the record with arrays from export() (of either checker)."""
        svd = np.ascontiguousarray(svd, np.uint16)
        keys = np.ascontiguousarray(keys, np.int64)
        offs = np.ascontiguousarray(offs, np.int64)
        self.api["tape_import"](self.t, len(svd), svd.ctypes.data, len(offs) - 1, keys.ctypes.data, offs.ctypes.data)

    def close(self):
        if self.t:
            self.api["tape_free"](self.t)
            self.t = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def box_drop_m1(kind: str) -> np.ndarray:
    api = load(kind)
    rows = np.zeros((1000, 10), np.float32)
    n = api["box_drop_m1"](_p(rows), 1000)
    return rows[:n]


def svd(kind: str, F: np.ndarray):
    F = np.ascontiguousarray(F, np.float32).reshape(-1, 3, 3)
    n = len(F)
    U = np.empty_like(F)
    V = np.empty_like(F)
    S = np.empty((n, 3), np.float32)
    load(kind)["svd"](n, _p(F), _p(U), _p(S), _p(V))
    return U, S, V


def reference_or_port() -> str:
    """The strongest FP32 checker available: the compiled reference, else the
    float restatement (pinned bit-exact to it by tests/test_oracle_pin.py)."""
    return "ref" if available("ref") else "f32"
