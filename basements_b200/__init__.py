"""basements_b200 — B200-native MLS-MPM soil step behind the bm_* C ABI.

Python access to ``libbm_mpm.so`` through ctypes, mirroring the reference
``basements::mpm::MPMSolver`` API (include/basements/physics/mpm/mpm_solver.h:15-95)
and the coupler plug-in ``MPMRigidCouplerPIC::apply``
(include/basements/physics/coupling/mpm_rigid_coupler_pic.h:88-184). The
computation always runs in the CUDA library; if the library is missing this
module raises at import of ``lib()``; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbm_mpm.so")

BM_OK = 0
STATUS_NAMES = {
    0: "BM_OK", 1: "BM_ERR_INVALID_ARGUMENT", 2: "BM_ERR_OUT_OF_MEMORY", 3: "BM_ERR_CUDA",
    4: "BM_ERR_DOMAIN_ESCAPE", 5: "BM_ERR_NON_FINITE", 6: "BM_ERR_TIMEOUT", 7: "BM_ERR_NOT_FOUND",
    8: "BM_ERR_STATE", 9: "BM_ERR_NO_DEVICE",
}


class BMError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)} {detail}".strip())


class Domain(C.Structure):
    _fields_ = [("origin", C.c_int32 * 3), ("extent", C.c_int32 * 3)]


class Collider(C.Structure):
    """bm_collider_t: the fields of RigidColliderState (mpm_rigid_coupler.h:72-84)."""
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


class Reaction(C.Structure):
    _fields_ = [("force", C.c_float * 3), ("torque", C.c_float * 3), ("nodes_inside", C.c_int32)]


class ParticlesView(C.Structure):
    _fields_ = [(n, C.POINTER(C.c_float)) for n in ("position", "velocity", "F", "C", "mass", "volume")]


class SceneDesc(C.Structure):
    """bm_scene_desc_t: one scene of a batch."""
    _fields_ = [
        ("dx", C.c_float),
        ("has_domain", C.c_int32),
        ("domain", Domain),
        ("n_particles", C.c_int64),
        ("position", C.POINTER(C.c_float)),
        ("velocity", C.POINTER(C.c_float)),
        ("mass", C.POINTER(C.c_float)),
        ("young_modulus", C.c_float),
        ("poisson_ratio", C.c_float),
        ("bulk_density", C.c_float),
        ("plastic_alpha", C.c_float),
        ("floor_friction", C.c_float),
        ("gravity", C.c_float * 3),
        ("dt", C.c_float),
        ("has_body", C.c_int32),
        ("body", Collider),
        ("body_dynamic", C.c_int32),
        ("body_inv_inertia", C.c_float * 9),
        ("body_inv_inertia_given", C.c_int32),
    ]


class TuneResult(C.Structure):
    _fields_ = [("variant", C.c_int32), ("sort_interval", C.c_int32), ("bin_shift", C.c_int32),
                ("ms_per_step", C.c_float)]


class ServerConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_double), ("max_active", C.c_int32), ("sort_interval", C.c_int32),
                ("variant", C.c_int32)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("failed", C.c_int64),
                ("cancelled", C.c_int64), ("queued", C.c_int64), ("active", C.c_int64),
                ("iterations", C.c_int64), ("p50_latency_ms", C.c_double), ("p99_latency_ms", C.c_double),
                ("mean_latency_ms", C.c_double), ("particle_steps", C.c_double), ("busy_seconds", C.c_double),
                ("peak_bytes", C.c_double), ("admit_seconds", C.c_double), ("step_seconds", C.c_double),
                ("retire_seconds", C.c_double)]


REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED, REQ_CANCELLED = range(5)

_f = C.POINTER(C.c_float)
_i32 = C.POINTER(C.c_int32)
_u8 = C.POINTER(C.c_uint8)
_h = C.c_void_p
_st = C.c_int

_SIGS = {
    "bm_get_version": (C.c_int, []),
    "bm_debug_svd3": (_st, [C.c_int64, _f, _f, _f, _f, C.c_int32]),
    "bm_status_string": (C.c_char_p, [C.c_int]),
    "bm_last_error": (C.c_char_p, []),
    "bm_set_device": (_st, [C.c_int32]),
    "bm_solver_create": (_st, [C.c_float, C.POINTER(Domain), C.POINTER(_h)]),
    "bm_solver_destroy": (_st, [_h]),
    "bm_solver_set_domain": (_st, [_h, C.POINTER(Domain)]),
    "bm_solver_get_domain": (_st, [_h, C.POINTER(Domain)]),
    "bm_solver_set_auto_margin": (_st, [_h, C.c_int32]),
    "bm_solver_set_sort_interval": (_st, [_h, C.c_int32]),
    "bm_solver_set_math_mode": (_st, [_h, C.c_int32]),
    "bm_solver_set_launch_variant": (_st, [_h, C.c_int32]),
    "bm_launch_variant_count": (C.c_int32, []),
    "bm_launch_variant_name": (C.c_char_p, [C.c_int32]),
    "bm_solver_set_material": (_st, [_h, C.c_float, C.c_float, C.c_float]),
    "bm_solver_set_gravity": (_st, [_h, _f]),
    "bm_solver_set_plastic_alpha": (_st, [_h, C.c_float]),
    "bm_solver_set_floor_friction": (_st, [_h, C.c_float]),
    "bm_solver_add_particles": (_st, [_h, C.c_int64, _f, _f, _f]),
    "bm_solver_num_particles": (_st, [_h, C.POINTER(C.c_int64)]),
    "bm_solver_get_particles": (_st, [_h, C.POINTER(ParticlesView)]),
    "bm_solver_set_particles": (_st, [_h, C.c_int64, C.c_int64, C.POINTER(ParticlesView)]),
    "bm_solver_step": (_st, [_h, C.c_float]),
    "bm_solver_step_n": (_st, [_h, C.c_float, C.c_int32]),
    "bm_solver_p2g": (_st, [_h, C.c_float]),
    "bm_solver_grid_update": (_st, [_h, C.c_float]),
    "bm_coupler_m1_apply": (_st, [_h, C.POINTER(Collider), C.c_float, C.POINTER(Reaction)]),
    "bm_coupler_m45a_apply": (_st, [_h, C.POINTER(Collider), C.c_float, C.POINTER(Reaction)]),
    "bm_coupler_m0_apply": (_st, [_h, C.POINTER(Collider), C.c_float, C.POINTER(Reaction)]),
    "bm_coupler_m45b_apply": (_st, [_h, C.POINTER(Collider), C.c_float, C.POINTER(Reaction)]),
    "bm_coupler_m45_apply": (_st, [_h, C.POINTER(Collider), C.c_float, C.POINTER(Reaction)]),
    "bm_solver_set_coupler": (_st, [_h, C.c_int32]),
    "bm_solver_g2p": (_st, [_h, C.c_float]),
    "bm_solver_step_coupled": (_st, [_h, C.c_float, C.c_int32, C.POINTER(Collider), C.POINTER(Reaction)]),
    "bm_solver_get_reactions": (_st, [_h, C.c_int32, C.POINTER(Reaction)]),
    "bm_solver_grid_num_nodes": (_st, [_h, C.POINTER(C.c_int64)]),
    "bm_solver_get_grid": (_st, [_h, _f, _f, _f, _u8, _u8]),
    "bm_solver_seed_grid": (_st, [_h, C.c_int64, _i32, _f, _f]),
    "bm_solver_set_grid_velocity": (_st, [_h, _f]),
    "bm_solver_sync": (_st, [_h, C.POINTER(C.c_int64)]),
    "bm_solver_light_node_suspects": (_st, [_h, C.POINTER(C.c_int64)]),
    "bm_solver_stream": (_st, [_h, C.POINTER(C.c_void_p)]),
    "bm_solver_profile_enable": (_st, [_h, C.c_int32]),
    "bm_solver_profile_read": (_st, [_h, C.c_int32, C.POINTER(C.c_char_p), C.POINTER(C.c_double),
                                      C.POINTER(C.c_int64), C.POINTER(C.c_int32)]),
    "bm_solver_profile_reset": (_st, [_h]),
    "bm_batch_create": (_st, [C.c_int32, C.POINTER(SceneDesc), C.POINTER(_h)]),
    "bm_batch_destroy": (_st, [_h]),
    "bm_batch_num_scenes": (_st, [_h, C.POINTER(C.c_int32)]),
    "bm_batch_num_particles": (_st, [_h, C.c_int32, C.POINTER(C.c_int64)]),
    "bm_batch_step": (_st, [_h, C.c_int32]),
    "bm_batch_steps_done": (_st, [_h, C.POINTER(C.c_int64)]),
    "bm_batch_get_particles": (_st, [_h, C.c_int32, C.POINTER(ParticlesView)]),
    "bm_batch_get_body": (_st, [_h, C.c_int32, C.POINTER(Collider)]),
    "bm_batch_get_reaction": (_st, [_h, C.c_int32, C.POINTER(Reaction)]),
    "bm_batch_sync": (_st, [_h, C.POINTER(C.c_int32), C.POINTER(C.c_int64)]),
    "bm_batch_light_node_suspects": (_st, [_h, C.POINTER(C.c_int64)]),
    "bm_batch_set_graph": (_st, [_h, C.c_int32]),
    "bm_batch_profile_enable": (_st, [_h, C.c_int32]),
    "bm_batch_profile_read": (_st, [_h, C.c_int32, C.POINTER(C.c_char_p), C.POINTER(C.c_double),
                                    C.POINTER(C.c_int64), C.POINTER(C.c_int32)]),
    "bm_batch_profile_reset": (_st, [_h]),
    "bm_batch_set_launch": (_st, [_h, C.c_int32, C.c_int32, C.c_int32]),
    "bm_batch_autotune": (_st, [_h, C.c_int32, C.POINTER(TuneResult)]),
    "bm_batch_timer_start": (_st, [_h]),
    "bm_batch_timer_stop": (_st, [_h, C.POINTER(C.c_double)]),
    "bm_coupler_m1_apply_noalloc": (_st, [_h, C.c_int32, C.POINTER(Collider), C.c_float, C.POINTER(Reaction)]),
    "bm_tape_create": (_st, [_h, C.c_int32, C.POINTER(_h)]),
    "bm_tape_destroy": (_st, [_h]),
    "bm_tape_forward": (_st, [_h, C.c_float, C.c_int32, C.POINTER(Collider), C.c_int32, _f]),
    "bm_adjoint_backward": (_st, [_h, _f, _f, _f, _f, _f]),
    "bm_adjoint_backward_state": (_st, [_h, C.POINTER(ParticlesView), _f, C.POINTER(ParticlesView)]),
    "bm_tape_body_grad": (_st, [_h, C.c_int32, C.POINTER(C.c_double)]),
    "bm_server_create": (_st, [C.POINTER(ServerConfig), C.POINTER(_h)]),
    "bm_server_destroy": (_st, [_h]),
    "bm_server_submit": (_st, [_h, C.POINTER(SceneDesc), C.c_int32, C.POINTER(C.c_int64)]),
    "bm_server_poll": (_st, [_h, C.c_int64, C.POINTER(C.c_int32)]),
    "bm_server_wait": (_st, [_h, C.c_int64, C.c_int32]),
    "bm_server_result": (_st, [_h, C.c_int64, C.POINTER(ParticlesView), C.POINTER(Collider), C.POINTER(C.c_double)]),
    "bm_server_release": (_st, [_h, C.c_int64]),
    "bm_server_cancel": (_st, [_h, C.c_int64]),
    "bm_server_stats": (_st, [_h, C.POINTER(ServerStats)]),
    "bm_server_estimate_bytes": (_st, [C.POINTER(SceneDesc), C.POINTER(C.c_double)]),
    "bm_solver_timer_start": (_st, [_h]),
    "bm_solver_timer_stop": (_st, [_h, C.POINTER(C.c_double)]),
}

_lib = None


def lib():
    """The loaded CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m basements_b200.build`")
    L = C.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def device_svd3(F, fast_math=False):
    """The step kernels' 3x3 SVD run on the device (bm_debug_svd3) for an
    array of matrices F (n x 3 x 3): returns U, S (unsorted), V."""
    F = np.ascontiguousarray(F, np.float32).reshape(-1, 3, 3)
    U, V = np.empty_like(F), np.empty_like(F)
    S = np.empty((len(F), 3), np.float32)
    check(lib().bm_debug_svd3(len(F), _fp(F), _fp(U), _fp(S), _fp(V), 1 if fast_math else 0), "bm_debug_svd3")
    return U, S, V


def set_device(device: int):
    check(lib().bm_set_device(int(device)), "bm_set_device")


def launch_variants():
    L = lib()
    return [L.bm_launch_variant_name(i).decode() for i in range(L.bm_launch_variant_count())]


def declared_symbols():
    return list(_SIGS)


def check(status: int, where: str):
    if status != BM_OK:
        detail = lib().bm_last_error().decode(errors="replace")
        raise BMError(status, where, detail)


def _fp(a):
    return None if a is None else a.ctypes.data_as(_f)


def make_collider(center, half_extents, orientation=(1.0, 0.0, 0.0, 0.0), linear_velocity=(0, 0, 0),
                  angular_velocity=(0, 0, 0), friction=0.5, mass=1.0, shape=0) -> Collider:
    c = Collider()
    c.center[:] = [float(v) for v in center]
    c.orientation[:] = [float(v) for v in orientation]
    c.half_extents[:] = [float(v) for v in half_extents]
    c.linear_velocity[:] = [float(v) for v in linear_velocity]
    c.angular_velocity[:] = [float(v) for v in angular_velocity]
    c.friction = float(friction)
    c.mass = float(mass)
    c.shape = int(shape)
    return c


class MPMSolver:
    """Device-resident MLS-MPM solver (one CUDA stream per instance)."""

    def __init__(self, dx: float = 0.1, domain=None, margin: int | None = None):
        L = lib()
        self._h = C.c_void_p()
        d = None
        if domain is not None:
            d = Domain()
            d.origin[:] = [int(v) for v in domain[0]]
            d.extent[:] = [int(v) for v in domain[1]]
        check(L.bm_solver_create(float(dx), C.byref(d) if d is not None else None, C.byref(self._h)),
              "bm_solver_create")
        self.dx = float(dx)
        if margin is not None:
            check(L.bm_solver_set_auto_margin(self._h, int(margin)), "bm_solver_set_auto_margin")

    # -- lifetime --------------------------------------------------------------
    def close(self):
        if self._h:
            lib().bm_solver_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def set_sort_interval(self, steps: int):
        check(lib().bm_solver_set_sort_interval(self._h, int(steps)), "bm_solver_set_sort_interval")

    def set_launch_variant(self, variant: int):
        check(lib().bm_solver_set_launch_variant(self._h, int(variant)), "bm_solver_set_launch_variant")

    def set_math_mode(self, fast: bool):
        check(lib().bm_solver_set_math_mode(self._h, 1 if fast else 0), "bm_solver_set_math_mode")

    # -- MPMSolver API (mpm_solver.h:19-95) -----------------------------------
    def set_material(self, young_modulus, poisson_ratio, bulk_density):
        check(lib().bm_solver_set_material(self._h, young_modulus, poisson_ratio, bulk_density),
              "bm_solver_set_material")

    def set_gravity(self, g):
        a = np.asarray(g, np.float32)
        check(lib().bm_solver_set_gravity(self._h, _fp(a)), "bm_solver_set_gravity")

    def set_plastic_alpha(self, a):
        check(lib().bm_solver_set_plastic_alpha(self._h, a), "bm_solver_set_plastic_alpha")

    def set_floor_friction(self, mu):
        check(lib().bm_solver_set_floor_friction(self._h, mu), "bm_solver_set_floor_friction")

    def add_particles(self, position, velocity=None, mass=None):
        pos = np.ascontiguousarray(position, np.float32).reshape(-1, 3)
        vel = None if velocity is None else np.ascontiguousarray(velocity, np.float32).reshape(-1, 3)
        if mass is not None:
            mass = np.ascontiguousarray(np.broadcast_to(np.asarray(mass, np.float32), (len(pos),)))
        check(lib().bm_solver_add_particles(self._h, len(pos), _fp(pos), _fp(vel), _fp(mass)),
              "bm_solver_add_particles")

    def add_particle(self, position, velocity=(0.0, 0.0, 0.0), mass=1.0):
        self.add_particles([position], [velocity], [mass])

    def num_particles(self) -> int:
        n = C.c_int64()
        check(lib().bm_solver_num_particles(self._h, C.byref(n)), "bm_solver_num_particles")
        return n.value

    def get_particles(self, fields=("position", "velocity", "F", "C", "mass", "volume")):
        n = self.num_particles()
        shapes = {"position": (n, 3), "velocity": (n, 3), "F": (n, 3, 3), "C": (n, 3, 3), "mass": (n,),
                  "volume": (n,)}
        out = {k: np.empty(shapes[k], np.float32) for k in fields}
        v = ParticlesView()
        for k in out:
            setattr(v, k, _fp(out[k]))
        check(lib().bm_solver_get_particles(self._h, C.byref(v)), "bm_solver_get_particles")
        return out

    def set_particles(self, first=0, position=None, velocity=None, F=None, C_=None):
        arrs = {"position": position, "velocity": velocity, "F": F, "C": C_}
        arrs = {k: np.ascontiguousarray(a, np.float32) for k, a in arrs.items() if a is not None}
        n = next(len(a) for a in arrs.values())
        v = ParticlesView()
        for k, a in arrs.items():
            setattr(v, k, _fp(a))
        check(lib().bm_solver_set_particles(self._h, int(first), int(n), C.byref(v)), "bm_solver_set_particles")

    def step(self, dt, n_steps: int = 1):
        if n_steps == 1:
            check(lib().bm_solver_step(self._h, dt), "bm_solver_step")
        else:
            check(lib().bm_solver_step_n(self._h, dt, int(n_steps)), "bm_solver_step_n")

    # -- split phases + coupler plug-in ----------------------------------------
    def p2g(self, dt):
        check(lib().bm_solver_p2g(self._h, dt), "bm_solver_p2g")

    def grid_update(self, dt):
        check(lib().bm_solver_grid_update(self._h, dt), "bm_solver_grid_update")

    def g2p(self, dt):
        check(lib().bm_solver_g2p(self._h, dt), "bm_solver_g2p")

    def m1_apply(self, body: Collider, dt):
        r = Reaction()
        check(lib().bm_coupler_m1_apply(self._h, C.byref(body), dt, C.byref(r)), "bm_coupler_m1_apply")
        return np.array(r.force[:], np.float32), np.array(r.torque[:], np.float32), int(r.nodes_inside)

    def m45a_apply(self, body: Collider, dt):
        """The M4.5a two-pass sweep coupler; same contract as m1_apply."""
        r = Reaction()
        check(lib().bm_coupler_m45a_apply(self._h, C.byref(body), dt, C.byref(r)), "bm_coupler_m45a_apply")
        return np.array(r.force[:], np.float32), np.array(r.torque[:], np.float32), int(r.nodes_inside)

    def m0_apply(self, body: Collider, dt):
        """The M0 Dirichlet coupler; same contract as m1_apply."""
        r = Reaction()
        check(lib().bm_coupler_m0_apply(self._h, C.byref(body), dt, C.byref(r)), "bm_coupler_m0_apply")
        return np.array(r.force[:], np.float32), np.array(r.torque[:], np.float32), int(r.nodes_inside)

    def m45b_apply(self, body: Collider, dt):
        """The M4.5b sweep layer (M4.5a + friction tangent)."""
        r = Reaction()
        check(lib().bm_coupler_m45b_apply(self._h, C.byref(body), dt, C.byref(r)), "bm_coupler_m45b_apply")
        return np.array(r.force[:], np.float32), np.array(r.torque[:], np.float32), int(r.nodes_inside)

    def m45c_apply(self, body: Collider, dt):
        """The M4.5 sweep layer (M4_5c: M4.5b + B-spline mass weight)."""
        r = Reaction()
        check(lib().bm_coupler_m45_apply(self._h, C.byref(body), dt, C.byref(r)), "bm_coupler_m45_apply")
        return np.array(r.force[:], np.float32), np.array(r.torque[:], np.float32), int(r.nodes_inside)

    COUPLERS = {"m1": 0, "m45a": 1, "m0": 2, "m45b": 3, "m45c": 4}

    def set_coupler(self, name: str):
        """Coupler of step_coupled: "m1" (default), "m45a", "m45b", "m45c" (M4.5) or "m0"."""
        check(lib().bm_solver_set_coupler(self._h, self.COUPLERS[name]), "bm_solver_set_coupler")

    def step_coupled(self, dt, bodies, read_reactions=True):
        n = len(bodies)
        arr = (Collider * max(n, 1))(*bodies)
        out = (Reaction * max(n, 1))() if read_reactions else None
        check(lib().bm_solver_step_coupled(self._h, dt, n, arr, out if read_reactions else None),
              "bm_solver_step_coupled")
        if not read_reactions:
            return None
        return [(np.array(r.force[:], np.float32), np.array(r.torque[:], np.float32), int(r.nodes_inside))
                for r in out[:n]]

    # -- grid -------------------------------------------------------------------
    def domain(self):
        d = Domain()
        check(lib().bm_solver_get_domain(self._h, C.byref(d)), "bm_solver_get_domain")
        return tuple(d.origin), tuple(d.extent)

    def get_grid(self):
        """Dense grid over the box: dict of arrays shaped (ex, ey, ez, ...)."""
        (o, e) = self.domain()
        nn = e[0] * e[1] * e[2]
        vel = np.empty((nn, 3), np.float32)
        frc = np.empty((nn, 3), np.float32)
        mass = np.empty(nn, np.float32)
        act = np.empty(nn, np.uint8)
        bal = np.empty(nn, np.uint8)
        check(lib().bm_solver_get_grid(self._h, _fp(vel), _fp(frc), _fp(mass), act.ctypes.data_as(_u8),
                                       bal.ctypes.data_as(_u8)), "bm_solver_get_grid")
        sh = tuple(e)
        return {"origin": np.array(o), "velocity": vel.reshape(*sh, 3), "force": frc.reshape(*sh, 3),
                "mass": mass.reshape(sh), "active": act.reshape(sh), "block_allocated": bal.reshape(sh)}

    def seed_grid(self, ijk, velocity, mass):
        ijk = np.ascontiguousarray(ijk, np.int32).reshape(-1, 3)
        vel = np.ascontiguousarray(velocity, np.float32).reshape(-1, 3)
        m = np.ascontiguousarray(np.broadcast_to(np.asarray(mass, np.float32), (len(ijk),)))
        check(lib().bm_solver_seed_grid(self._h, len(ijk), ijk.ctypes.data_as(_i32), _fp(vel), _fp(m)),
              "bm_solver_seed_grid")

    def set_grid_velocity(self, velocity):
        v = np.ascontiguousarray(velocity, np.float32)
        check(lib().bm_solver_set_grid_velocity(self._h, _fp(v)), "bm_solver_set_grid_velocity")

    # -- status / profiling ----------------------------------------------------------
    def sync(self):
        """Waits for the stream; returns (status, escaped_writes) without raising."""
        esc = C.c_int64()
        st = lib().bm_solver_sync(self._h, C.byref(esc))
        return st, esc.value

    def light_node_suspects(self) -> int:
        """Nodes whose particle mass fell from >= 1e-4 to (0, 1e-6] in one step
        (the only places the fused step can depart from the reference's
        momentum-without-force rule); 0 means none so far."""
        n = C.c_int64()
        check(lib().bm_solver_light_node_suspects(self._h, C.byref(n)), "bm_solver_light_node_suspects")
        return n.value

    def profile(self, on=True):
        check(lib().bm_solver_profile_enable(self._h, 1 if on else 0), "bm_solver_profile_enable")

    def profile_reset(self):
        check(lib().bm_solver_profile_reset(self._h), "bm_solver_profile_reset")

    def timer_start(self):
        check(lib().bm_solver_timer_start(self._h), "bm_solver_timer_start")

    def timer_stop(self) -> float:
        ms = C.c_double()
        check(lib().bm_solver_timer_stop(self._h, C.byref(ms)), "bm_solver_timer_stop")
        return ms.value

    def profile_read(self):
        cap = 32
        names = (C.c_char_p * cap)()
        ms = (C.c_double * cap)()
        cnt = (C.c_int64 * cap)()
        n = C.c_int32()
        check(lib().bm_solver_profile_read(self._h, cap, names, ms, cnt, C.byref(n)), "bm_solver_profile_read")
        return {names[i].decode(): (ms[i], cnt[i]) for i in range(n.value)}


def scene_desc(scene, keep: list) -> SceneDesc:
    """bm_scene_desc_t for a basements_b200.scenes.Scene; `keep` holds the
    arrays the descriptor points to until the batch is created."""
    d = SceneDesc()
    d.dx = float(scene.dx)
    if scene.domain is not None:
        d.has_domain = 1
        d.domain.origin[:] = [int(v) for v in scene.domain[0]]
        d.domain.extent[:] = [int(v) for v in scene.domain[1]]
    pos = np.ascontiguousarray(scene.position, np.float32)
    mass = np.ascontiguousarray(scene.mass, np.float32)
    keep += [pos, mass]
    d.n_particles = len(pos)
    d.position = _fp(pos)
    d.mass = _fp(mass)
    d.young_modulus, d.poisson_ratio, d.bulk_density = float(scene.E), float(scene.nu), float(scene.rho)
    d.plastic_alpha, d.floor_friction = float(scene.alpha), float(scene.floor_friction)
    d.gravity[:] = [float(v) for v in scene.gravity]
    d.dt = float(scene.dt)
    if scene.bodies:
        b = scene.bodies[0]
        d.has_body = 1
        d.body = make_collider(**b.as_tuple())
        d.body_dynamic = 0 if b.kinematic else 1
        if b.inv_inertia is not None:
            d.body_inv_inertia[:] = [float(v) for v in b.inv_inertia]
            d.body_inv_inertia_given = 1
    return d


class Batch:
    """Many scenes stepped together (bm_batch_*)."""

    def __init__(self, scenes):
        keep = []
        descs = (SceneDesc * len(scenes))(*[scene_desc(sc, keep) for sc in scenes])
        self._h = C.c_void_p()
        check(lib().bm_batch_create(len(scenes), descs, C.byref(self._h)), "bm_batch_create")
        self.n_scenes = len(scenes)

    def close(self):
        if self._h:
            lib().bm_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n_steps=1):
        check(lib().bm_batch_step(self._h, int(n_steps)), "bm_batch_step")

    def steps_done(self):
        n = C.c_int64()
        check(lib().bm_batch_steps_done(self._h, C.byref(n)), "bm_batch_steps_done")
        return n.value

    def num_particles(self, scene):
        n = C.c_int64()
        check(lib().bm_batch_num_particles(self._h, int(scene), C.byref(n)), "bm_batch_num_particles")
        return n.value

    def get_particles(self, scene, fields=("position", "velocity", "F", "C")):
        n = self.num_particles(scene)
        shapes = {"position": (n, 3), "velocity": (n, 3), "F": (n, 3, 3), "C": (n, 3, 3), "mass": (n,),
                  "volume": (n,)}
        out = {k: np.empty(shapes[k], np.float32) for k in fields}
        v = ParticlesView()
        for k in out:
            setattr(v, k, _fp(out[k]))
        check(lib().bm_batch_get_particles(self._h, int(scene), C.byref(v)), "bm_batch_get_particles")
        return out

    def get_body(self, scene) -> Collider:
        c = Collider()
        check(lib().bm_batch_get_body(self._h, int(scene), C.byref(c)), "bm_batch_get_body")
        return c

    def get_reaction(self, scene):
        r = Reaction()
        check(lib().bm_batch_get_reaction(self._h, int(scene), C.byref(r)), "bm_batch_get_reaction")
        return np.array(r.force[:], np.float32), np.array(r.torque[:], np.float32), int(r.nodes_inside)

    def sync(self):
        bad = C.c_int32()
        esc = C.c_int64()
        st = lib().bm_batch_sync(self._h, C.byref(bad), C.byref(esc))
        return st, bad.value, esc.value

    def light_node_suspects(self) -> int:
        n = C.c_int64()
        check(lib().bm_batch_light_node_suspects(self._h, C.byref(n)), "bm_batch_light_node_suspects")
        return n.value

    def set_graph(self, on: bool):
        check(lib().bm_batch_set_graph(self._h, 1 if on else 0), "bm_batch_set_graph")

    def profile(self, on=True):
        """Per-phase CUDA-event timing (steps run eagerly while it is on)."""
        check(lib().bm_batch_profile_enable(self._h, 1 if on else 0), "bm_batch_profile_enable")

    def profile_reset(self):
        check(lib().bm_batch_profile_reset(self._h), "bm_batch_profile_reset")

    def profile_read(self):
        cap = 32
        names = (C.c_char_p * cap)()
        ms = (C.c_double * cap)()
        cnt = (C.c_int64 * cap)()
        n = C.c_int32()
        check(lib().bm_batch_profile_read(self._h, cap, names, ms, cnt, C.byref(n)), "bm_batch_profile_read")
        return {names[i].decode(): (ms[i], cnt[i]) for i in range(n.value)}

    def set_launch(self, variant, sort_interval, bin_shift=0):
        check(lib().bm_batch_set_launch(self._h, int(variant), int(sort_interval), int(bin_shift)),
              "bm_batch_set_launch")

    def autotune(self, trial_steps=16):
        r = TuneResult()
        check(lib().bm_batch_autotune(self._h, int(trial_steps), C.byref(r)), "bm_batch_autotune")
        return {"variant": r.variant, "sort_interval": r.sort_interval, "bin_shift": r.bin_shift,
                "ms_per_step": r.ms_per_step}

    def timer_start(self):
        check(lib().bm_batch_timer_start(self._h), "bm_batch_timer_start")

    def timer_stop(self) -> float:
        ms = C.c_double()
        check(lib().bm_batch_timer_stop(self._h, C.byref(ms)), "bm_batch_timer_stop")
        return ms.value


class Server:
    """Continuous-batching server (bm_server_*)."""

    def __init__(self, hbm_budget_bytes=150e9, max_active=1024, sort_interval=32, variant=-1):
        cfg = ServerConfig(float(hbm_budget_bytes), int(max_active), int(sort_interval), int(variant))
        self._h = C.c_void_p()
        check(lib().bm_server_create(C.byref(cfg), C.byref(self._h)), "bm_server_create")
        self._n = {}

    def close(self):
        if self._h:
            lib().bm_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, scene, n_steps) -> int:
        keep = []
        d = scene_desc(scene, keep)
        rid = C.c_int64()
        check(lib().bm_server_submit(self._h, C.byref(d), int(n_steps), C.byref(rid)), "bm_server_submit")
        self._n[rid.value] = scene.n
        return rid.value

    def poll(self, rid) -> int:
        st = C.c_int32()
        check(lib().bm_server_poll(self._h, int(rid), C.byref(st)), "bm_server_poll")
        return st.value

    def wait(self, rid, timeout_ms=60000) -> int:
        """Returns the bm_status_t of the wait (BM_OK, BM_ERR_TIMEOUT, ...)."""
        return lib().bm_server_wait(self._h, int(rid), int(timeout_ms))

    def result(self, rid):
        n = self._n[rid]
        out = {"position": np.empty((n, 3), np.float32), "velocity": np.empty((n, 3), np.float32),
               "F": np.empty((n, 3, 3), np.float32), "C": np.empty((n, 3, 3), np.float32)}
        v = ParticlesView()
        for k in out:
            setattr(v, k, _fp(out[k]))
        body = Collider()
        lat = C.c_double()
        check(lib().bm_server_result(self._h, int(rid), C.byref(v), C.byref(body), C.byref(lat)), "bm_server_result")
        out["body"] = body
        out["latency_ms"] = lat.value
        return out

    def release(self, rid):
        check(lib().bm_server_release(self._h, int(rid)), "bm_server_release")

    def cancel(self, rid):
        check(lib().bm_server_cancel(self._h, int(rid)), "bm_server_cancel")

    def stats(self):
        st = ServerStats()
        check(lib().bm_server_stats(self._h, C.byref(st)), "bm_server_stats")
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}


def estimate_bytes(scene) -> float:
    keep = []
    d = scene_desc(scene, keep)
    b = C.c_double()
    check(lib().bm_server_estimate_bytes(C.byref(d), C.byref(b)), "bm_server_estimate_bytes")
    return b.value


class Tape:
    """Differentiable run on a solver (bm_tape_* / bm_adjoint_backward)."""

    def __init__(self, solver: MPMSolver, checkpoint_every: int = 20):
        self.solver = solver
        self._h = C.c_void_p()
        check(lib().bm_tape_create(solver._h, int(checkpoint_every), C.byref(self._h)), "bm_tape_create")
        self.n_steps = 0
        self.n_wp = 0

    def close(self):
        if self._h:
            lib().bm_tape_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def forward(self, dt, n_steps, body: Collider | None = None, waypoints=None):
        """n_steps split steps recorded for the reverse pass; the body (if
        any) follows the piecewise-linear path through `waypoints`."""
        wp = None
        self.n_wp = 0
        if body is not None:
            wp = np.ascontiguousarray(waypoints, np.float32).reshape(-1, 3)
            self.n_wp = len(wp)
        check(lib().bm_tape_forward(self._h, float(dt), int(n_steps), C.byref(body) if body is not None else None,
                                    self.n_wp, _fp(wp) if wp is not None else None), "bm_tape_forward")
        self.n_steps = int(n_steps)

    def backward(self, dL_dx, dL_dv=None, want_x0=False, want_v0=False):
        """Returns a dict with dL_dwaypoints (when the run had a body) and,
        on request, dL_dx0 / dL_dv0."""
        n = self.solver.num_particles()
        gx = np.ascontiguousarray(dL_dx, np.float32).reshape(n, 3)
        gv = None if dL_dv is None else np.ascontiguousarray(dL_dv, np.float32).reshape(n, 3)
        out = {}
        wp = np.zeros((self.n_wp, 3), np.float32) if self.n_wp else None
        x0 = np.zeros((n, 3), np.float32) if want_x0 else None
        v0 = np.zeros((n, 3), np.float32) if want_v0 else None
        check(lib().bm_adjoint_backward(self._h, _fp(gx), _fp(gv) if gv is not None else None,
                                        _fp(wp) if wp is not None else None, _fp(x0) if x0 is not None else None,
                                        _fp(v0) if v0 is not None else None), "bm_adjoint_backward")
        if wp is not None:
            out["dL_dwaypoints"] = wp
        if x0 is not None:
            out["dL_dx0"] = x0
        if v0 is not None:
            out["dL_dv0"] = v0
        return out

    def backward_state(self, dL: dict):
        """Reverse pass for the whole state: dL maps any of position, velocity
        (n x 3), F, C (n x 3 x 3) to the loss gradient at the final state.
        Returns the gradient at the initial state for the four fields, plus
        dL_dwaypoints when the run had a body."""
        n = self.solver.num_particles()
        shapes = {"position": (n, 3), "velocity": (n, 3), "F": (n, 3, 3), "C": (n, 3, 3)}
        keep = {}
        vin = ParticlesView()
        for k, shp in shapes.items():
            if k in dL:
                keep[k] = np.ascontiguousarray(dL[k], np.float32).reshape(shp)
                setattr(vin, k, _fp(keep[k]))
        out = {k: np.zeros(shp, np.float32) for k, shp in shapes.items()}
        vout = ParticlesView()
        for k in shapes:
            setattr(vout, k, _fp(out[k]))
        wp = np.zeros((self.n_wp, 3), np.float32) if self.n_wp else None
        check(lib().bm_adjoint_backward_state(self._h, C.byref(vin), _fp(wp) if wp is not None else None,
                                              C.byref(vout)), "bm_adjoint_backward_state")
        if wp is not None:
            out["dL_dwaypoints"] = wp
        return out

    def body_grad(self):
        """dL/d(body linear velocity), dL/d(body angular velocity) per step (n_steps x 6)."""
        g = np.zeros((self.n_steps, 6), np.float64)
        check(lib().bm_tape_body_grad(self._h, self.n_steps, g.ctypes.data_as(C.POINTER(C.c_double))),
              "bm_tape_body_grad")
        return g
