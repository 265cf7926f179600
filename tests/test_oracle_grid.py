"""Pins the oracle's gridded environments (gen_grid, profile_grid,
boundary_grid) to the reference's own known-answer tests.

The 1-D and 2-D cases are types/test/datagrid_test.cc's; the grids are
evaluated through a profile_grid (sound speed = the grid value at rho) or a
boundary_grid (height = the grid value at theta, phi), the way the
propagator reads them.
"""
import ctypes as C
import math

import numpy as np
import pytest

import underseamodelinglibrary_b200 as u
from underseamodelinglibrary_b200 import _abi
from oracle_binding import load_oracle

R = 6371000.0


def quad1d(x):
    """datagrid_test.cc:106"""
    return 5.0 + 3.0 * x - 0.3 * x * x


def oracle_profile(grid, rho, theta=None, phi=None):
    """sound speed and gradient of a profile_grid at the given points"""
    lib = load_oracle()
    oc = u.ocean_model(u.boundary_flat(), u.boundary_flat(1000.0), u.profile_grid(grid))
    od = oc.descriptor()
    rho = np.ascontiguousarray(rho, dtype=np.float64)
    n = rho.size
    th = np.zeros(n) if theta is None else np.ascontiguousarray(theta, dtype=np.float64)
    ph = np.zeros(n) if phi is None else np.ascontiguousarray(phi, dtype=np.float64)
    c = np.empty(n)
    g = np.empty(3 * n)
    assert lib.oracle_sound_speed(C.byref(od), R, n, _abi.as_dp(rho), _abi.as_dp(th), _abi.as_dp(ph),
                                  _abi.as_dp(c), _abi.as_dp(g)) == 0
    return c, g.reshape(3, n).T    # SoA: all rho, then theta, then phi


def oracle_bottom(grid, theta, phi):
    """height and unit normal of a boundary_grid bottom"""
    lib = load_oracle()
    oc = u.ocean_model(u.boundary_flat(), u.boundary_grid(grid), u.profile_linear(1500.0))
    od = oc.descriptor()
    th = np.ascontiguousarray(theta, dtype=np.float64)
    ph = np.ascontiguousarray(phi, dtype=np.float64)
    n = th.size
    h = np.empty(n)
    nrm = np.empty(3 * n)
    assert lib.oracle_height(C.byref(od), 1, n, _abi.as_dp(np.zeros(n)), _abi.as_dp(th), _abi.as_dp(ph),
                             _abi.as_dp(h), _abi.as_dp(nrm)) == 0
    return h, nrm.reshape(3, n).T


def grid_1d(axis, f, kind, edge):
    g = u.data_grid([axis], [f(axis[n]) for n in range(axis.size())])
    g.interp_type(0, kind)
    g.edge_limit(0, edge)
    return g


def test_linear_1d():
    """datagrid_test.cc:116-158: linear and pchip reproduce a linear field,
    extrapolation included, within 1e-6 percent"""
    ax = u.seq_linear(1.0, 2.0, 9.0)
    xs = np.arange(0.25, 10.0001, 0.25)
    truth = 5.0 + 3.0 * xs
    for kind in (u.data_grid.LINEAR, u.data_grid.PCHIP):
        c, _ = oracle_profile(grid_1d(ax, lambda x: 5.0 + 3.0 * x, kind, False), xs)
        assert np.all(np.abs(c - truth) <= 1e-8 * np.abs(truth))


def test_quad_1d():
    """datagrid_test.cc:394-435: pchip within 1 percent of a quadratic"""
    ax = u.seq_linear(1.0, 2.0, 9.0)
    xs = np.arange(0.5, 9.5001, 0.25)
    c, _ = oracle_profile(grid_1d(ax, quad1d, u.data_grid.PCHIP, False), xs)
    assert np.all(np.abs(c - quad1d(xs)) <= 1e-2 * np.abs(quad1d(xs)))


def test_log_axis_1d():
    """datagrid_test.cc:442-482: pchip on a logarithmic axis within 2 percent"""
    ax = u.seq_log(1.0, 3.0 ** (1.0 / 3.0), 9.0)
    assert ax.size() == 7
    xs = np.arange(1.0, 9.5001, 0.25)
    c, _ = oracle_profile(grid_1d(ax, quad1d, u.data_grid.PCHIP, False), xs)
    assert np.all(np.abs(c - quad1d(xs)) <= 2e-2 * np.abs(quad1d(xs)))


def test_deriv_1d():
    """datagrid_test.cc:489-527: pchip derivative within 0.35 of the
    analytic one (edge limiting on, as data_grid defaults)"""
    ax = u.seq_linear(1.0, 2.0, 9.0)
    xs = np.arange(1.0, 9.0001, 0.25)
    _, g = oracle_profile(grid_1d(ax, quad1d, u.data_grid.PCHIP, True), xs)
    assert np.all(np.abs(g[:, 0] - (3.0 - 0.6 * xs)) < 0.35)


def test_nearest_and_edge_limit_1d():
    """gen_grid.h nearest: the closer node's value with zero derivative;
    edge_limit clamps the location to the axis ends (gen_grid.h:99-118)"""
    ax = u.seq_linear(1.0, 2.0, 9.0)
    c, g = oracle_profile(grid_1d(ax, quad1d, u.data_grid.NEAREST, True), [0.0, 1.9, 2.1, 4.0, 8.5, 12.0])
    assert np.array_equal(c, quad1d(np.array([1.0, 1.0, 3.0, 5.0, 9.0, 9.0])))
    assert np.all(g[:, 0] == 0.0)
    c, _ = oracle_profile(grid_1d(ax, quad1d, u.data_grid.LINEAR, True), [-5.0, 20.0])
    assert np.array_equal(c, quad1d(np.array([1.0, 9.0])))


def test_compute_index_3d():
    """datagrid_test.cc:41-91: row-major data with the last axis fastest;
    at the nodes a 3-D linear grid returns x + y + z exactly"""
    ax = [u.seq_linear(0.0, 100.0, 2), u.seq_linear(0.0, 10.0, 3), u.seq_linear(0.0, 1.0, 4)]
    X, Y, Z = np.meshgrid(ax[0].data, ax[1].data, ax[2].data, indexing="ij")
    g = u.data_grid(ax, X + Y + Z)
    c, _ = oracle_profile(g, X.ravel(), Y.ravel(), Z.ravel())
    assert np.array_equal(c, (X + Y + Z).ravel())


def test_fast_accuracy_2d():
    """datagrid_test.cc:617-672: 2-D pchip of x^3 y^3 on a 10x10 grid is
    within 3 percent at (0.2135, -0.3611)"""
    ax = [u.seq_linear(-0.5, 0.1, 10), u.seq_linear(-0.5, 0.1, 10)]
    x = np.arange(10) / 10.0 - 0.5
    g = u.data_grid(ax, np.outer(x ** 3, x ** 3))
    g.interp_type(0, u.data_grid.PCHIP)
    g.interp_type(1, u.data_grid.PCHIP)
    h, _ = oracle_bottom(g, [0.2135], [-0.3611])
    truth = 0.2135 ** 3 * (-0.3611) ** 3
    assert abs(h[0] - truth) <= 0.03 * abs(truth)


def test_ascii_profile_data_axis():
    """ocean/test/profile_test.cc:225-238 with ocean/ascii_profile.cc:15-63:
    a decreasing seq_data rho axis (earth radius minus depth), pchip, edge
    limited; the grid returns its data at the nodes"""
    depth = np.array([0.01, 25.45, 50.45, 100.00, 149.55, 201.36, 239.55, 400.00])
    speed = np.array([1546.50, 1547.00, 1540.60, 1522.50, 1511.20, 1504.50, 1492.70, 1490.00])
    ax = u.seq_data(R - depth)
    g = u.data_grid([ax], speed)
    g.interp_type(0, u.data_grid.PCHIP)
    c, _ = oracle_profile(g, R - depth)
    assert np.allclose(c, speed, rtol=1e-12, atol=0)
    assert abs(c[0] - 1546.50) < 1546.50 * 1e-7 and abs(c[7] - 1490.00) < 1490.0 * 1e-7
    c, _ = oracle_profile(g, R - np.array([-10.0, 1000.0]))      # beyond both ends: clamped
    assert np.allclose(c, [1546.50, 1490.00], rtol=1e-12, atol=0)
    mid, _ = oracle_profile(g, R - np.array([75.0]))
    assert 1522.50 < mid[0] < 1540.60


def test_boundary_grid_normal_is_unit_and_tilted_downslope():
    """boundary_grid.h:88-137: normal = (1, -g_theta/rho, -g_phi/(rho sin
    theta)) made unit length"""
    lat = np.radians(np.linspace(44.0, 46.0, 11))
    th_ax = u.seq_linear(math.pi / 2 - lat[-1], (lat[-1] - lat[0]) / 10, 11)
    ph_ax = u.seq_linear(math.radians(-46.0), math.radians(0.2), 11)
    depth = 1000.0 + 100.0 * np.arange(11)[None, :] * np.ones((11, 1))   # deepens with phi
    g = u.data_grid([th_ax, ph_ax], R - depth)
    th = np.full(5, th_ax[5])
    ph = np.linspace(ph_ax[1], ph_ax[8], 5)
    h, n = oracle_bottom(g, th, ph)
    assert np.allclose(np.sum(n * n, axis=1), 1.0, rtol=0, atol=1e-14)
    assert np.all(n[:, 2] > 0) and np.allclose(n[:, 1], 0.0, atol=1e-12)
    slope = 100.0 / (R * math.radians(0.2) * np.sin(th))
    assert np.allclose(n[:, 2] / n[:, 0], slope * R / h, rtol=1e-9)
