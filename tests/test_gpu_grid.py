"""Gridded environments on the GPU against the oracle: gen_grid
interpolation through profile_grid and boundary_grid point evaluations
(every axis kind, interpolation kind and edge mode), and propagation
through a 3-D profile_grid over 2-D boundary_grid bathymetry."""
import ctypes as C
import math

import numpy as np
import pytest

import underseamodelinglibrary_b200 as u
from underseamodelinglibrary_b200 import _abi
from underseamodelinglibrary_b200 import scenarios as S
from oracle_binding import OracleQueue, load_oracle
from test_gpu_parity import compare_eigenrays, compare_fronts, run_pair

pytestmark = pytest.mark.gpu

KINDS = (u.data_grid.NEAREST, u.data_grid.LINEAR, u.data_grid.PCHIP)


def _oracle_speed(oc, R, rho, th, ph):
    od = oc.descriptor()
    n = rho.size
    c = np.empty(n)
    g = np.empty(3 * n)
    assert load_oracle().oracle_sound_speed(C.byref(od), R, n, _abi.as_dp(rho), _abi.as_dp(th),
                                            _abi.as_dp(ph), _abi.as_dp(c), _abi.as_dp(g)) == 0
    return c, g.reshape(3, n)


def _oracle_height(oc, th, ph):
    od = oc.descriptor()
    n = th.size
    h = np.empty(n)
    nrm = np.empty(3 * n)
    assert load_oracle().oracle_height(C.byref(od), 1, n, _abi.as_dp(np.zeros(n)), _abi.as_dp(th),
                                       _abi.as_dp(ph), _abi.as_dp(h), _abi.as_dp(nrm)) == 0
    return h, nrm.reshape(3, n)


def _same(x, y, rtol=1e-12):
    scale = max(float(np.max(np.abs(y))), 1e-300)
    assert np.max(np.abs(x - y)) <= rtol * scale, float(np.max(np.abs(x - y)) / scale)


def _check_profile(grid, rho, th, ph):
    u.compute_earth_radius(45.0)
    R = u.earth_radius()
    oc = u.ocean_model(u.boundary_flat(), u.boundary_flat(6000.0), u.profile_grid(grid))
    c, g = oc.sound_speed(rho, th, ph)
    co, go = _oracle_speed(oc, R, rho, th, ph)
    _same(c, co)
    for k in range(3):
        _same(np.asarray(g)[k], go[k], rtol=1e-10)


def test_profile_grid_1d_axes_and_kinds(engine):
    """1-D profile_grid on increasing, decreasing, log and data axes; every
    interpolation kind; edge limiting on and off; points beyond both ends"""
    u.compute_earth_radius(45.0)
    R = u.earth_radius()
    rng = np.random.default_rng(11)
    depth = np.linspace(0.0, 5000.0, 26)
    axes = [u.seq_linear(R - 5000.0, 200.0, 26),          # increasing rho
            u.seq_linear(R, -200.0, 26),                   # decreasing rho
            u.seq_data(R - depth ** 1.3 / 5000.0 ** 0.3),  # uneven, decreasing
            u.seq_log(R - 6000.0, 1.00003, 30)]            # logarithmic
    for ax in axes:
        data = 1500.0 + 30.0 * np.sin(np.arange(ax.size()) * 0.7) + rng.normal(0.0, 2.0, ax.size())
        lo, hi = min(ax[0], ax[ax.size() - 1]), max(ax[0], ax[ax.size() - 1])
        rho = np.concatenate([np.linspace(lo - 300.0, hi + 300.0, 397), np.asarray(ax.data)])
        z = np.zeros(rho.size)
        for kind in KINDS:
            for edge in (True, False):
                g = u.data_grid([ax], data)
                g.interp_type(0, kind)
                g.edge_limit(0, edge)
                _check_profile(g, rho, z, z)


def test_profile_grid_2d_3d(engine):
    """2-D (rho, theta) and 3-D (rho, theta, phi) profile grids with mixed
    interpolation kinds, including axes too short for pchip"""
    u.compute_earth_radius(45.0)
    R = u.earth_radius()
    rng = np.random.default_rng(5)
    th0, ph0 = math.radians(44.0), math.radians(-46.0)
    rho_ax = u.seq_linear(R, -250.0, 21)
    th_ax = u.seq_linear(th0, math.radians(0.2), 11)
    ph_ax = u.seq_linear(ph0, math.radians(0.25), 9)
    short_ax = u.seq_linear(ph0, math.radians(1.0), 3)          # pchip falls back to linear
    n = 2000
    rho = R - rng.uniform(-200.0, 5400.0, n)
    th = th0 + np.radians(rng.uniform(-0.3, 2.3, n))
    ph = ph0 + np.radians(rng.uniform(-0.3, 2.3, n))
    for ndim, axes in ((2, [rho_ax, th_ax]), (3, [rho_ax, th_ax, ph_ax]), (3, [rho_ax, th_ax, short_ax])):
        shape = [a.size() for a in axes]
        data = 1500.0 + rng.normal(0.0, 5.0, shape)
        for kinds in ((2, 1, 1), (2, 2, 2), (0, 2, 1), (1, 0, 2)):
            g = u.data_grid(axes, data)
            for d in range(ndim):
                g.interp_type(d, KINDS[kinds[d]])
            g.edge_limit(ndim - 1, False)
            _check_profile(g, rho, th, ph)


def test_boundary_grid_heights_and_normals(engine):
    """1-D (theta) and 2-D (theta, phi) boundary grids: height and unit
    normal against the oracle"""
    u.compute_earth_radius(45.0)
    R = u.earth_radius()
    rng = np.random.default_rng(7)
    th0, ph0 = math.radians(44.0), math.radians(-46.0)
    th_ax = u.seq_linear(th0, math.radians(0.05), 41)
    ph_ax = u.seq_linear(ph0, math.radians(0.05), 37)
    n = 1500
    th = th0 + np.radians(rng.uniform(-0.2, 2.2, n))
    ph = ph0 + np.radians(rng.uniform(-0.2, 2.0, n))
    for axes in ([th_ax], [th_ax, ph_ax]):
        shape = [a.size() for a in axes]
        depth = S._smooth(rng.standard_normal(shape), [3.0] * len(shape))
        depth = 1000.0 + 4000.0 * (depth - depth.min()) / (depth.max() - depth.min())
        for kind in KINDS:
            g = u.data_grid(axes, R - depth)
            for d in range(len(axes)):
                g.interp_type(d, kind)
            oc = u.ocean_model(u.boundary_flat(), u.boundary_grid(g), u.profile_linear(1500.0))
            h, nrm = oc.height(1, th, ph)
            ho, no = _oracle_height(oc, th, ph)
            _same(h, ho, rtol=1e-15)
            _same(np.asarray(nrm).reshape(3, n), no, rtol=1e-12)


def test_gridded_propagation_parity(engine):
    """3-D profile_grid (Munk plus a random field) over 2-D boundary_grid
    relief with Rayleigh sand loss: eigenrays and every front field"""
    sc = S.gridded_munk(seed=3, num_de=91, num_az=13, time_max=30.0)
    q, o = run_pair(sc)
    eng = q.take_eigenrays()
    assert len(eng) > 100
    compare_eigenrays(eng, o.take_eigenrays())
    for w in ("prev", "curr", "next"):
        compare_fronts(getattr(q, w)(), getattr(o, w)(), rel=1e-9, edges=w != "next")


def test_gridded_fp32c_matches_fp64(engine):
    """the FP32 CPA screen finds the same eigenrays on the gridded ocean"""
    sc = S.gridded_munk(seed=4, num_de=91, num_az=13, time_max=20.0)
    a = S.build_queue(sc, u.wave_queue, precision=_abi.FP64)
    b = S.build_queue(sc, u.wave_queue, precision=_abi.FP32C)
    a.run(sc["time_max"])
    b.run(sc["time_max"])
    ra, rb = a.take_eigenrays(), b.take_eigenrays()
    assert len(ra) == len(rb) > 50
    for x, y in zip(ra, rb):
        assert (x.step, x.t1, x.t2, x.de_index, x.az_index) == (y.step, y.t1, y.t2, y.de_index, y.az_index)
        assert x.travel_time == y.travel_time
        assert np.array_equal(x.intensity, y.intensity)


def test_std14_parity(engine):
    """the reference's speed-study scenario (STD14 grids near Hawaii, 100
    targets on a 100 km ring) on the engine against the oracle for the
    study's 80 s, which reaches the ring (about 1300 eigenrays)"""
    sc = S.std14(num_targets=100, time_max=80.0)
    q, o = run_pair(sc)
    eng = q.take_eigenrays()
    assert len(eng) > 1000
    compare_eigenrays(eng, o.take_eigenrays())
    compare_fronts(q.curr(), o.curr(), rel=1e-9)
