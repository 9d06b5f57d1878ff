"""bm_coupler_m1_apply_noalloc against bm_coupler_m1_apply (GPU).

The allocation-free coupler entry point runs the same M1 kernels with fixed
scratch. Two solvers hold the same scene; one couples through each entry
point, on two coupled steps in a row. The second call checks that the reaction
sums restart from zero. Reactions (FP64 sums per CTA, order-dependent in the
last bits) agree to 1e-5 relative, and the grid after the call matches.
A third test checks the entry point's one property: across its calls the
device's free memory does not move. This file is collected last, so it also
runs after every other GPU test in the same process.
"""
import ctypes as C

import numpy as np
import pytest

import basements_b200 as bm
from basements_b200 import scenes
from tests.gpu_util import gpu_solver

pytestmark = pytest.mark.gpu


def _noalloc(s, bodies, dt):
    n = len(bodies)
    arr = (bm.Collider * max(n, 1))(*bodies)
    out = (bm.Reaction * max(n, 1))()
    st = bm.lib().bm_coupler_m1_apply_noalloc(s._h, n, arr, dt, out)
    return st, [(np.array(r.force[:]), np.array(r.torque[:]), int(r.nodes_inside)) for r in out[:n]]


def _free_device_bytes():
    """Free memory of the current device, from the driver (cuMemGetInfo)."""
    cuda = C.CDLL("libcuda.so.1")
    free, total = C.c_size_t(), C.c_size_t()
    assert cuda.cuMemGetInfo_v2(C.byref(free), C.byref(total)) == 0
    return free.value


def test_noalloc_coupler_allocates_no_device_memory():
    """A solver that never used the allocating coupler builds its grid (which
    allocates), then couples through the no-alloc entry point twelve times (six
    calls at each of two body poses): the device's free memory is the same before and after
    (the solver's creation already loaded the M1 code and looked up the
    scratch array)."""
    sc = scenes.wheel_rut(n_keep=20000)
    s = gpu_solver(sc.dx, sc.position, None, sc.mass, sc.E, sc.nu, sc.rho, sc.alpha, domain=sc.domain)
    s.p2g(sc.dt)
    s.grid_update(sc.dt)
    assert s.sync() == (0, 0)
    before = _free_device_bytes()
    for n in range(2):
        body = bm.make_collider(**sc.bodies[0].at_time(n * sc.dt).as_tuple())
        for _ in range(6):
            st, [(f, _t, n_in)] = _noalloc(s, [body], sc.dt)
            assert st == 0, bm.lib().bm_last_error()
            assert n_in > 0 and np.isfinite(f).all()
    assert s.sync() == (0, 0)
    assert _free_device_bytes() == before


def test_noalloc_coupler_matches_the_allocating_one_on_two_calls():
    sc = scenes.wheel_rut(n_keep=20000)
    a = gpu_solver(sc.dx, sc.position, None, sc.mass, sc.E, sc.nu, sc.rho, sc.alpha, domain=sc.domain)
    b = gpu_solver(sc.dx, sc.position, None, sc.mass, sc.E, sc.nu, sc.rho, sc.alpha, domain=sc.domain)
    for n in range(2):
        body = bm.make_collider(**sc.bodies[0].at_time(n * sc.dt).as_tuple())
        for s in (a, b):
            s.p2g(sc.dt)
            s.grid_update(sc.dt)
        fa, ta, na = a.m1_apply(body, sc.dt)
        st, [(fb, tb, nb)] = _noalloc(b, [body], sc.dt)
        assert st == 0, bm.lib().bm_last_error()
        assert na == nb and na > 0
        np.testing.assert_allclose(fb, fa, rtol=1e-5, atol=1e-5 * np.abs(fa).max())
        np.testing.assert_allclose(tb, ta, rtol=1e-5, atol=1e-5 * np.abs(ta).max())
        ga, gb = a.get_grid(), b.get_grid()
        np.testing.assert_array_equal(ga["active"], gb["active"])
        np.testing.assert_allclose(gb["velocity"], ga["velocity"], rtol=0, atol=1e-6)
        for s in (a, b):
            s.g2p(sc.dt)


def test_noalloc_coupler_limits_and_body_order():
    sc = scenes.wheel_rut(n_keep=4096)
    a = gpu_solver(sc.dx, sc.position, None, sc.mass, sc.E, sc.nu, sc.rho, sc.alpha, domain=sc.domain)
    s = gpu_solver(sc.dx, sc.position, None, sc.mass, sc.E, sc.nu, sc.rho, sc.alpha, domain=sc.domain)
    body = bm.make_collider(**sc.bodies[0].as_tuple())
    st, _ = _noalloc(s, [body], sc.dt)
    assert st == 8  # BM_ERR_STATE: no grid yet
    for x in (a, s):
        x.p2g(sc.dt)
        x.grid_update(sc.dt)
    st, _ = _noalloc(s, [body] * 65, sc.dt)
    assert st == 1 and b"64" in bm.lib().bm_last_error()
    # three copies of one body in one call are applied in order, like three
    # successive calls of the allocating entry point
    st, r = _noalloc(s, [body] * 3, sc.dt)
    assert st == 0
    for k in range(3):
        fa, ta, na = a.m1_apply(body, sc.dt)
        assert r[k][2] == na > 0
        np.testing.assert_allclose(r[k][0], fa, rtol=1e-5, atol=1e-5 * np.abs(fa).max())
    assert np.abs(r[2][0]).max() < np.abs(r[0][0]).max()
