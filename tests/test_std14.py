"""STD14 (studies/cmp_speed): the CDL-text loader and the netcdf_profile /
netcdf_bathy window semantics, checked on CPU against the data itself and
against the oracle's propagation."""
import math

import numpy as np

import underseamodelinglibrary_b200 as u
from underseamodelinglibrary_b200 import scenarios as S
from underseamodelinglibrary_b200.netcdf_cdl import netcdf_bathy, netcdf_profile
from oracle_binding import OracleQueue


def _npz():
    import os
    return np.load(os.path.join(os.path.dirname(u.__file__), "data", "std14.npz"))


def test_profile_window_and_axes():
    """netcdf_profile.cc:57-115: the whole 31 x 30 x 30 grid falls inside
    the study's window; rho = R - stored altitude; colatitude decreasing"""
    d = _npz()
    u.set_earth_radius(6371000.0)
    g = netcdf_profile({"time": d["p_time"], "depth": d["p_depth"], "lat": d["p_lat"], "lon": d["p_lon"],
                        "speed": d["p_speed"]}, 0.0, 16.2, 24.6, -164.4, -155.5)
    assert [a.size() for a in g.axes] == [31, 30, 30]
    assert np.array_equal(g.axes[0].data, 6371000.0 - d["p_depth"].astype(np.float64))
    lat0, latn = float(d["p_lat"][0]), float(d["p_lat"][-1])
    assert abs(g.axes[1][0] - math.radians(90.0 - lat0)) < 1e-15
    assert abs(g.axes[1].increment(0) + math.radians((latn - lat0) / 29)) < 1e-15
    assert np.array_equal(g.data, d["p_speed"][0].astype(np.float64))


def test_bathy_window():
    """netcdf_bathy.cc:67-173: the study's window keeps rows and columns
    by the file's uniform increments; values become rho = R + altitude"""
    d = _npz()
    g = netcdf_bathy({"lat": d["b_lat"], "lon": d["b_lon"], "depth": d["b_depth"]},
                     16.2, 24.6, -164.4, -155.5, 6371000.0)
    lat, lon = d["b_lat"].astype(np.float64), d["b_lon"].astype(np.float64)
    inc = (lat[-1] - lat[0]) / (lat.size - 1)
    first = max(0, int(math.floor(1e-6 + (16.2 - lat[0]) / inc)))
    last = min(lat.size - 1, int(math.floor(0.5 + (24.6 - lat[0]) / inc)))
    assert g.axes[0].size() == last - first + 1
    assert g.data.shape == (g.axes[0].size(), g.axes[1].size())
    assert np.all(g.data <= 6371000.0) and np.min(g.data) > 6371000.0 - 6000.0


def test_std14_oracle_runs():
    """the study's scenario on the oracle for 10 s with 10 targets"""
    sc = S.std14(num_targets=10, time_max=10.0)
    assert sc["az"].size() == 25 and sc["de"].size() == 181
    q = S.build_queue(sc, OracleQueue)
    q.run(sc["time_max"])
    c = q.curr()
    assert np.all(np.isfinite(c.rho))
