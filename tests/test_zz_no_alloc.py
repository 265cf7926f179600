"""wq3d_ocean_sound_speed_noalloc: the sound speed evaluation for callers
that cannot allocate device memory when they need an answer (a processing
loop that reserves its GPU memory up front, code under a real-time budget).
It stages points in a fixed device array built into the library instead of
allocating.  Checked through the C ABI against wq3d_ocean_sound_speed on two
calls in a row; this file sorts last so that a run stopping at the first
failure has already run every other test.

Both entry points run the same device code built with the same flags, so
their results must agree bit for bit."""
import ctypes as C

import numpy as np
import pytest

import underseamodelinglibrary_b200 as u
from underseamodelinglibrary_b200 import _abi

pytestmark = pytest.mark.gpu


def _points(n, seed):
    rng = np.random.default_rng(seed)
    R = u.earth_radius()
    rho = R - rng.uniform(0.0, 5000.0, n)
    theta = np.full(n, u.to_radians(45.0)) + rng.uniform(-0.01, 0.01, n)
    phi = np.full(n, u.to_radians(-45.0)) + rng.uniform(-0.01, 0.01, n)
    return rho, theta, phi


def _eval(lib, fn, oc, rho, theta, phi, with_grad=True):
    n = rho.size
    c = np.empty(n)
    g = np.empty(3 * n) if with_grad else None
    rc = fn(oc.handle(), u.earth_radius(), n, _abi.as_dp(rho), _abi.as_dp(theta) if theta is not None else None,
            _abi.as_dp(phi) if phi is not None else None, _abi.as_dp(c), _abi.as_dp(g) if with_grad else None)
    _abi.check(lib, rc)
    return c, g


def _oceans():
    u.compute_earth_radius(45.0)
    munk = u.profile_munk()
    munk.flat_earth(True)
    yield "munk", u.ocean_model(u.boundary_flat(), u.boundary_flat(5000.0), munk)
    # a 3-D gridded profile (pchip in depth, linear in latitude and
    # longitude) read through the staging array's theta and phi blocks
    from underseamodelinglibrary_b200 import scenarios as S
    yield "grid3", S.gridded_ocean(np.random.default_rng(7), n_depth=12, n_lat=6, n_lng=6, n_bathy=8)


def test_noalloc_matches_allocating_entry_point_twice():
    lib = _abi.load_engine()
    n = C.c_int()
    assert lib.wq3d_device_count(C.byref(n)) == 0 and n.value > 0
    for name, oc in _oceans():
        for call, (npts, seed) in enumerate(((1000, 1), (_abi.WQ3D_NOALLOC_MAX_POINTS, 2))):
            rho, theta, phi = _points(npts, seed)
            c0, g0 = _eval(lib, lib.wq3d_ocean_sound_speed, oc, rho, theta, phi)
            c1, g1 = _eval(lib, lib.wq3d_ocean_sound_speed_noalloc, oc, rho, theta, phi)
            assert np.array_equal(c1, c0), (name, call)
            assert np.array_equal(g1, g0), (name, call)


def test_noalloc_without_angles_or_gradient():
    """theta and phi may be NULL (zero colatitude and longitude) and grad
    may be NULL; the answers equal the allocating entry point's."""
    lib = _abi.load_engine()
    u.compute_earth_radius(45.0)
    oc = u.ocean_model(u.boundary_flat(), u.boundary_flat(5000.0), u.profile_munk())
    rho, _, _ = _points(777, 5)
    for with_grad in (True, False):
        c0, g0 = _eval(lib, lib.wq3d_ocean_sound_speed, oc, rho, None, None, with_grad)
        c1, g1 = _eval(lib, lib.wq3d_ocean_sound_speed_noalloc, oc, rho, None, None, with_grad)
        assert np.array_equal(c1, c0)
        if with_grad:
            assert np.array_equal(g1, g0)


def test_noalloc_rejects_too_many_points():
    lib = _abi.load_engine()
    u.compute_earth_radius(45.0)
    oc = u.ocean_model(u.boundary_flat(), u.boundary_flat(5000.0), u.profile_munk())
    n = _abi.WQ3D_NOALLOC_MAX_POINTS + 1
    rho, theta, phi = _points(n, 3)
    c = np.empty(n)
    rc = lib.wq3d_ocean_sound_speed_noalloc(oc.handle(), u.earth_radius(), n, _abi.as_dp(rho),
                                            _abi.as_dp(theta), _abi.as_dp(phi), _abi.as_dp(c), None)
    assert rc == _abi.WQ3D_ERR_INVALID
    assert b"exceed" in lib.wq3d_last_error_string()
