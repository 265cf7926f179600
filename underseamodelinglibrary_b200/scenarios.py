"""Named propagation scenarios.

* The reference's own test scenarios (waveq3d/test/*.cc), rebuilt with the
  same constructors and arguments, so a test here reads like the
  reference's test and can check the same known answers.
* The synthetic benchmark workloads ("munk_flat_181x37" and
  "linear_slope_rayleigh_1801x91"), whose shapes and value ranges are the
  published benchmark configurations of this engine; inputs are generated,
  not read from data files.

Every builder returns a dict with keys ocean, freq, pos, de, az, dt,
targets, time_max, type and the earth radius it set.
"""
import math

import numpy as np

from . import types as T
from .ocean import (attenuation_constant, boundary_flat, boundary_grid, boundary_slope,
                    data_grid, ocean_model, profile_grid, profile_linear, profile_munk,
                    reflect_loss_constant, reflect_loss_eckart, reflect_loss_rayleigh, volume_flat)
from ._abi import HYBRID_GAUSSIAN


def _pack(**kw):
    kw.setdefault("type", HYBRID_GAUSSIAN)
    kw["earth_radius"] = T.earth_radius()
    return kw


def eigenray_basic():
    """waveq3d/test/eigenray_test.cc:86-198 -- isovelocity, 3000 m flat
    bottom, direct / surface / bottom paths to one target."""
    T.compute_earth_radius(45.0)
    profile = profile_linear(1500.0, attenuation_constant(0.0))
    ocean = ocean_model(boundary_flat(), boundary_flat(3000.0), profile)
    return _pack(ocean=ocean, freq=T.seq_log(10e3, 2.0, 3), pos=T.wposition1(45.0, -45.0, -1000.0),
                 de=T.seq_linear(-60.0, 5.0, 60.0), az=T.seq_linear(-4.0, 1.0, 4.0), dt=0.1,
                 targets=T.wposition(1, 1, 45.02, -45.0, -1000.0), time_max=3.5)


def eigenray_concave():
    """eigenray_test.cc:232-332 -- target 1.2 deg away, 4 paths."""
    T.compute_earth_radius(45.0)
    profile = profile_linear(1500.0, attenuation_constant(0.0))
    ocean = ocean_model(boundary_flat(), boundary_flat(1e5), profile)
    return _pack(ocean=ocean, freq=T.seq_log(2000.0, 1.0, 1), pos=T.wposition1(45.0, -45.0, -200.0),
                 de=T.seq_linear(-1.0, 0.05, 1.0), az=T.seq_linear(-4.0, 1.0, 4.0), dt=0.1,
                 targets=T.wposition(1, 1, 46.2, -45.0, -150.0), time_max=120.0)


def eigenray_branch_pt():
    """eigenray_test.cc:428-534 -- AZ fan wrapping 0/360, targets directly
    above and below the source and on a 2226 m ring."""
    T.compute_earth_radius(0.0)
    profile = profile_linear(1500.0, attenuation_constant(0.0))
    ocean = ocean_model(boundary_flat(), boundary_flat(3000.0), profile)
    pos = T.wposition1(0.0, 0.0, -1000.0)
    num = 12
    tgt = T.wposition(num + 2, 1, 0.0, 0.0, -1000.0)
    tgt.altitude(0, 0, -1000.0 - 500)
    tgt.altitude(1, 0, -1000.0 + 500)
    angle = 2.0 * math.pi / num
    bearing = 0.0
    for n in range(2, num + 2):
        t = T.wposition1(pos, 2226.0, bearing)
        tgt.latitude(n, 0, t.latitude())
        tgt.longitude(n, 0, t.longitude())
        tgt.altitude(n, 0, t.altitude())
        bearing = bearing + angle
    return _pack(ocean=ocean, freq=T.seq_log(1000.0, 1.0, 1), pos=pos,
                 de=T.seq_linear(-90.0, 1.0, 90.0), az=T.seq_linear(0.0, 15.0, 360.0), dt=0.1,
                 targets=tgt, time_max=3.5)


def proploss_gaussian():
    """waveq3d/test/proploss_test.cc:153-248 -- ten frequencies."""
    T.compute_earth_radius(45.0)
    profile = profile_linear(1500.0, attenuation_constant(0.0))
    ocean = ocean_model(boundary_flat(), boundary_flat(3000.0), profile)
    return _pack(ocean=ocean, freq=T.seq_linear(100.0, 100.0, 1000.0),
                 pos=T.wposition1(45.0, -45.0, -1000.0), de=T.seq_linear(-90.0, 1.0, 90.0),
                 az=T.seq_linear(-5.0, 1.0, 5.0), dt=0.1,
                 targets=T.wposition(1, 1, 45.02, -45.0, -1000.0), time_max=3.5)


def refraction_munk_range():
    """waveq3d/test/refraction_test.cc:827-980 -- Munk profile with the
    flat earth correction, rays launched from the channel axis."""
    T.set_earth_radius(6371000.0)
    ssp = profile_munk()
    ssp.flat_earth(True)
    ocean = ocean_model(boundary_flat(), boundary_flat(5000.0), ssp)
    return _pack(ocean=ocean, freq=T.seq_log(10e3, 1.0, 1), pos=T.wposition1(45.0, -45.0, -1000.0),
                 de=T.seq_linear(-14.0, 1.0, 14.0), az=T.seq_linear(0.0, 0.0, 1), dt=0.1,
                 targets=None, time_max=95.0)


# analytic cycle ranges for D/E -14..14 (refraction_test.cc:836-842)
MUNK_CYCLE_RANGES = [
    64977.771509, 62686.699943, 60536.790347, 58539.834823, 56706.277890,
    55044.418981, 53559.948084, 52255.876772, 51132.827760, 50189.572079,
    49423.683193, 48832.195747, 48412.185973, 48161.238557, 48077.771909,
    48161.238557, 48412.185973, 48832.195747, 49423.683193, 50189.572079,
    51132.827760, 52255.876772, 53559.948084, 55044.418981, 56706.277890,
    58539.834823, 60536.790347, 62686.699943, 64977.771509]


def reflect_flat():
    """waveq3d/test/reflection_test.cc:168-280 -- one ray bouncing between
    the surface and a 1000 m flat bottom."""
    T.compute_earth_radius(45.0)
    ocean = ocean_model(boundary_flat(), boundary_flat(1000.0), profile_linear())
    return _pack(ocean=ocean, freq=T.seq_log(10.0, 10.0, 1), pos=T.wposition1(45.0, -45.0, 0.0),
                 de=T.seq_linear(-5.183617057, 0.0, 1), az=T.seq_linear(0.0, 0.0, 1), dt=0.1,
                 targets=None, time_max=60.0)


def reflect_slope():
    """waveq3d/test/reflection_test.cc:283-390 -- one ray at dt 1 ms
    between the surface and a bottom 1000 m deep at 45.1N sloping 1 deg,
    silt Rayleigh loss."""
    T.compute_earth_radius(45.0)
    slope_ref = T.wposition1(45.1, -45.0, 0.0)
    bottom = boundary_slope(slope_ref, 1000.0, math.radians(1.0), 0.0, reflect_loss_rayleigh("silt"))
    ocean = ocean_model(boundary_flat(), bottom, profile_linear())
    return _pack(ocean=ocean, freq=T.seq_log(10.0, 10.0, 1), pos=T.wposition1(45.0, -45.0, 0.0),
                 de=T.seq_linear(-5.175034664, 0.0, 1), az=T.seq_linear(0.0, 0.0, 1), dt=0.001,
                 targets=None, time_max=25.0)


def bounce_threshold():
    """waveq3d/test/reflection_test.cc:597-661 -- 181 x 13 fan at the
    equator, 1000 m flat bottom, max_surface 3 and max_bottom 5."""
    T.set_earth_radius(6371000.0)
    ocean = ocean_model(boundary_flat(), boundary_flat(1000.0, reflect_loss_constant(0.0)),
                        profile_linear(1500.0))
    return _pack(ocean=ocean, freq=T.seq_log(900.0, 1.0, 1), pos=T.wposition1(0.0, 0.0, -500.0),
                 de=T.seq_linear(-90.0, 1.0, 90.0), az=T.seq_linear(0.0, 30.0, 360.0), dt=0.1,
                 targets=T.wposition(1, 1, 0.01, 0.0, -500.0), time_max=10.0,
                 thresholds=dict(max_surface=3, max_bottom=5))


def eigenverb_accuracy():
    """waveq3d/test/reverb_test.cc:216-310 -- isovelocity 1500 m/s, 1000 m
    sand bottom, a volume layer at 300 m (10 m thick, -40 dB), source on
    the surface at 45N 45W, 1 kHz, D/E -80..60 step 5 x AZ -40..40 step
    10, dt 0.1 s for 3.5 s; eigenverbs only."""
    T.set_earth_radius(6371000.0)
    ocean = ocean_model(boundary_flat(), boundary_flat(1000.0, reflect_loss_rayleigh("sand")),
                        profile_linear(1500.0))
    ocean.add_volume(volume_flat(300.0, 10.0, -40.0))
    return _pack(ocean=ocean, freq=T.seq_log(1000.0, 10.0, 1), pos=T.wposition1(45.0, -45.0, 0.0),
                 de=T.seq_linear(-80.0, 5.0, 60.0), az=T.seq_linear(-40.0, 10.0, 40.1), dt=0.1,
                 targets=None, time_max=3.5, depth=1000.0, c0=1500.0)


def eigenverb_demo():
    """waveq3d/test/reverb_test.cc:334-443 -- isovelocity 1500 m/s without
    absorption, 200 m sand bottom, source on the surface, 1 kHz, 181
    tangent-spaced D/E x AZ 0..340 step 20, dt 0.1 s for 4 s, at most 2
    surface and 2 bottom bounces."""
    T.set_earth_radius(6371000.0)
    ocean = ocean_model(boundary_flat(), boundary_flat(200.0, reflect_loss_rayleigh("sand")),
                        profile_linear(1500.0, attenuation_constant(0.0)))
    return _pack(ocean=ocean, freq=T.seq_log(1000.0, 10.0, 1), pos=T.wposition1(45.0, -45.0, 0.0),
                 de=T.seq_rayfan(-90.0, 90.0, 181), az=T.seq_linear(0.0, 20.0, 359.0), dt=0.1,
                 targets=None, time_max=4.0, depth=200.0, c0=1500.0,
                 thresholds=dict(max_bottom=2, max_surface=2))


def munk_flat(num_de=181, num_az=37, n_targets=10, time_max=60.0):
    """Plain FP64 workload: Munk profile, 5000 m flat bottom with 0 dB
    loss, source 1000 m at 45N 45W, 10 Hz, tangent-spaced D/E fan from -90
    to 90 deg x AZ 0..180 deg in 5 deg steps, dt 0.1 s for 60 s, targets at
    500 m depth on a 10 x 10 lat/lon grid 0.1-0.9 deg from the source."""
    T.compute_earth_radius(45.0)
    profile = profile_munk(attmodel=attenuation_constant(0.0))
    ocean = ocean_model(boundary_flat(), boundary_flat(5000.0, reflect_loss_constant(0.0)), profile)
    lat = [45.0 + 0.1 + k * 0.8 / (n_targets - 1) for k in range(n_targets)]
    lng = [-45.0 + 0.1 + k * 0.8 / (n_targets - 1) for k in range(n_targets)]
    tgt = T.wposition.mesh(lat, lng, -500.0)
    az = T.seq_linear(0.0, 5.0, 180.0) if num_az == 37 else T.seq_linear(0.0, 180.0 / (num_az - 1), num_az)
    return _pack(ocean=ocean, freq=T.seq_log(10.0, 1.0, 1), pos=T.wposition1(45.0, -45.0, -1000.0),
                 de=T.seq_rayfan(-90.0, 90.0, num_de), az=az, dt=0.1, targets=tgt,
                 time_max=time_max, name="munk_flat_%dx%d" % (num_de, num_az))


def linear_slope_rayleigh(num_de=1801, num_az=91, n_range=32, n_depth=32, time_max=40.0):
    """Linear-gradient profile c(z) = 1500 + 0.0163 z with Thorp attenuation
    over a bottom sloping from 200 m at the source to 2000 m at 20 km north
    (boundary_slope), Rayleigh bottom (density 1.5, speed 1.1, 0.5
    dB/wavelength).  Source 50 m deep at 45N 45W, 5 log-spaced frequencies
    100 Hz - 3 kHz, tangent-spaced D/E fan x AZ 0..360 deg (wrapping), dt
    0.05 s for 40 s, targets on a range x depth grid (0.5-20 km north,
    10-2000 m)."""
    T.compute_earth_radius(45.0)
    src = T.wposition1(45.0, -45.0, -50.0)
    profile = profile_linear(1500.0, 0.0163)
    bottom = boundary_slope(src, 200.0, -math.atan(1800.0 / 20000.0), 0.0,
                            reflect_loss_rayleigh(1.5, 1.1, 0.5))
    ocean = ocean_model(boundary_flat(), bottom, profile)
    freq = T.seq_log(100.0, 30.0 ** 0.25, 5)
    ranges = np.linspace(500.0, 20000.0, n_range)
    depths = np.linspace(10.0, 2000.0, n_depth)
    tgt = T.wposition(n_range, n_depth, 0.0, 0.0, 0.0)
    for i, r in enumerate(ranges):
        p = T.wposition1(src, float(r), 0.0)
        for j, z in enumerate(depths):
            tgt.latitude(i, j, p.latitude())
            tgt.longitude(i, j, p.longitude())
            tgt.altitude(i, j, -float(z))
    az = T.seq_linear(0.0, 4.0, 360.0) if num_az == 91 else T.seq_linear(0.0, 360.0 / (num_az - 1), num_az)
    return _pack(ocean=ocean, freq=freq, pos=src, de=T.seq_rayfan(-90.0, 90.0, num_de), az=az,
                 dt=0.05, targets=tgt, time_max=time_max,
                 name="linear_slope_rayleigh_%dx%d" % (num_de, num_az))


def _smooth(field, sigmas):
    """Separable Gaussian smoothing (sigma in nodes per axis, reflecting
    edges)."""
    out = np.asarray(field, dtype=np.float64)
    for ax, sig in enumerate(sigmas):
        if sig <= 0:
            continue
        half = int(math.ceil(3.0 * sig))
        k = np.exp(-0.5 * (np.arange(-half, half + 1) / sig) ** 2)
        k /= k.sum()
        pad = [(0, 0)] * out.ndim
        pad[ax] = (half, half)
        padded = np.pad(out, pad, mode="reflect" if out.shape[ax] > half else "edge")
        out = np.apply_along_axis(lambda v: np.convolve(v, k, mode="valid"), ax, padded)
    return out


def gridded_ocean(rng, lat0=45.0, lng0=-45.0, span=2.0, n_depth=50, n_lat=20, n_lng=20,
                  n_bathy=100, ssp_std=5.0, corr_h=50e3, corr_v=300.0, depth_min=1000.0,
                  depth_max=5000.0, surface=None, bottom_loss=None):
    """Gridded environment over span x span degrees centred on (lat0, lng0):

    * profile_grid<3> on (rho, theta, phi) with n_depth nodes 0-5000 m x
      n_lat x n_lng: the Munk profile plus a Gaussian random field of
      ``ssp_std`` m/s with ``corr_h`` horizontal and ``corr_v`` vertical
      correlation lengths; pchip in depth, linear across;
    * boundary_grid<2> bottom on n_bathy x n_bathy (theta, phi) nodes:
      Gaussian-smoothed random relief scaled to depth_min..depth_max,
      linear both ways, Rayleigh sand loss (the boundary_grid default);
    * ``surface``: the ocean surface (default boundary_flat());
    * ``bottom_loss``: the bathymetry's reflection loss (default Rayleigh
      sand, the boundary_grid default).

    Inputs are seeded synthetic fields (no data files)."""
    R = T.earth_radius()
    th0 = math.radians(90.0 - (lat0 + span / 2))
    ph0 = math.radians(lng0 - span / 2)
    dz = 5000.0 / (n_depth - 1)
    rho_ax = T.seq_linear(R, -dz, n_depth)
    th_ax = T.seq_linear(th0, math.radians(span) / (n_lat - 1), n_lat)
    ph_ax = T.seq_linear(ph0, math.radians(span) / (n_lng - 1), n_lng)
    z = np.arange(n_depth) * dz
    zt = 2.0 * (z - 1300.0) / 1300.0
    munk = 1500.0 * (1.0 + 0.00737 * (zt - 1.0 + np.exp(-zt)))
    dx = R * math.radians(span) / (n_lat - 1)
    noise = _smooth(rng.standard_normal((n_depth, n_lat, n_lng)),
                    (corr_v / dz, corr_h / dx, corr_h / dx))
    noise *= ssp_std / max(noise.std(), 1e-30)
    ssp = data_grid([rho_ax, th_ax, ph_ax], munk[:, None, None] + noise)
    ssp.interp_type(0, data_grid.PCHIP)
    bt_ax = T.seq_linear(th0, math.radians(span) / (n_bathy - 1), n_bathy)
    bp_ax = T.seq_linear(ph0, math.radians(span) / (n_bathy - 1), n_bathy)
    relief = _smooth(rng.standard_normal((n_bathy, n_bathy)), (n_bathy / 12.0, n_bathy / 12.0))
    relief = (relief - relief.min()) / max(relief.max() - relief.min(), 1e-30)
    bathy = data_grid([bt_ax, bp_ax], R - (depth_min + (depth_max - depth_min) * relief))
    return ocean_model(surface if surface is not None else boundary_flat(), boundary_grid(bathy, bottom_loss),
                       profile_grid(ssp))


def random_targets(rng, src, n, max_range=100e3, depth=(10.0, 4000.0)):
    """n targets at uniform random bearing, range up to max_range and depth
    in the given interval, as a 1 x n wposition."""
    tgt = T.wposition(1, n, 0.0, 0.0, 0.0)
    for k in range(n):
        p = T.wposition1(src, float(rng.uniform(1e3, max_range)), float(rng.uniform(0.0, 2 * math.pi)))
        tgt.latitude(0, k, p.latitude())
        tgt.longitude(0, k, p.longitude())
        tgt.altitude(0, k, -float(rng.uniform(*depth)))
    return tgt


def gridded_munk(seed=1, num_de=91, num_az=13, n_targets=64, time_max=30.0, src_depth=100.0,
                 dt=0.1, freq=None, **grid_kw):
    """One instance of the batched gridded workload: gridded_ocean() around
    45N 45W, source ``src_depth`` m deep, tangent-spaced D/E fan x AZ 0..360
    deg, 64 random targets at 10-4000 m depth within 100 km."""
    T.compute_earth_radius(45.0)
    rng = np.random.default_rng(seed)
    ocean = gridded_ocean(rng, **grid_kw)
    src = T.wposition1(45.0, -45.0, -float(src_depth))
    tgt = random_targets(rng, src, n_targets)
    az = T.seq_linear(0.0, 360.0 / (num_az - 1), num_az) if num_az > 1 else T.seq_linear(0.0, 0.0, 1)
    return _pack(ocean=ocean, freq=freq or T.seq_log(1000.0, 1.0, 1), pos=src,
                 de=T.seq_rayfan(-90.0, 90.0, num_de), az=az, dt=dt, targets=tgt, time_max=time_max,
                 name="gridded_munk_%dx%d" % (num_de, num_az))


def reverb_scale(source_depth=100.0, num_de=3601, num_az=181, n_targets=4096, time_max=180.0,
                 seed=20261203, bottom_loss=None):
    """Reverberation-scale workload for one source depth: gridded_ocean()
    (random profile grid and bathymetry) with Eckart surface loss at 10 m/s
    wind, source ``source_depth`` m deep at 45N 45W, 32 log-spaced
    frequencies 100 Hz - 10 kHz with Thorp attenuation, tangent-spaced D/E
    fan x AZ 0..360 deg in 2 deg steps, dt 0.05 s, 4096 random targets
    (10-4000 m deep within 100 km).  ``bottom_loss``: the bathymetry's
    reflection loss (default Rayleigh sand)."""
    T.compute_earth_radius(45.0)
    rng = np.random.default_rng(seed)
    ocean = gridded_ocean(rng, surface=boundary_flat(0.0, reflect_loss_eckart(10.0)), bottom_loss=bottom_loss)
    src = T.wposition1(45.0, -45.0, -float(source_depth))
    tgt = random_targets(rng, src, n_targets)
    freq = T.seq_log(100.0, 100.0 ** (1.0 / 31.0), 32)
    az = T.seq_linear(0.0, 360.0 / (num_az - 1), num_az)
    return _pack(ocean=ocean, freq=freq, pos=src, de=T.seq_rayfan(-90.0, 90.0, num_de), az=az, dt=0.05,
                 targets=tgt, time_max=time_max,
                 name="reverb_scale_%dx%d_%dtgt_32f" % (num_de, num_az, n_targets))


def batched_gridded(n_instances=512, seed=20261203, num_de=(91, 1801), num_az=(1, 91),
                    time_max=(10.0, 120.0), dt=0.05, n_targets=64):
    """Batched workload of uneven instances: each has its own gridded_ocean()
    (50 x 20 x 20 profile grid of Munk plus a random field, 100 x 100
    bathymetry of 1000-5000 m), a source 10-500 m deep at 45N 45W, D/E
    and AZ counts drawn uniformly from ``num_de`` and ``num_az`` (AZ fan
    0..360 deg, which wraps from 3 rays up), time_max drawn from
    ``time_max``, and 64 random targets at 10-4000 m depth within 100 km
    (range 100 km x sqrt(U)).  Returns one scenario dict per instance."""
    T.compute_earth_radius(45.0)
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_instances):
        nde = int(rng.integers(num_de[0], num_de[1] + 1))
        naz = int(rng.integers(num_az[0], num_az[1] + 1))
        tmax = float(rng.uniform(*time_max))
        zs = float(rng.uniform(10.0, 500.0))
        ocean = gridded_ocean(rng)
        src = T.wposition1(45.0, -45.0, -zs)
        tgt = T.wposition(1, n_targets, 0.0, 0.0, 0.0)
        for j in range(n_targets):
            p = T.wposition1(src, float(100e3 * math.sqrt(rng.uniform())), float(rng.uniform(0.0, 2 * math.pi)))
            tgt.latitude(0, j, p.latitude())
            tgt.longitude(0, j, p.longitude())
            tgt.altitude(0, j, -float(rng.uniform(10.0, 4000.0)))
        az = T.seq_linear(0.0, 360.0 / (naz - 1), naz) if naz > 1 else T.seq_linear(0.0, 0.0, 1)
        out.append(_pack(ocean=ocean, freq=T.seq_log(1000.0, 1.0, 1), pos=src,
                         de=T.seq_rayfan(-90.0, 90.0, nde), az=az, dt=dt, targets=tgt, time_max=tmax,
                         name="batched_gridded_%d_of_%d" % (k, n_instances)))
    return out


def std14_ocean():
    """The STD14 environment of studies/cmp_speed/cmp_speed.cc:56-76: the
    3-D sound speed grid (netcdf_profile) and 2-D bathymetry (netcdf_bathy)
    near Hawaii over 16.2-24.6 N, 164.4-155.5 W, from the package's
    data/std14.npz (the study's CDL dumps as float32)."""
    import os
    from .netcdf_cdl import netcdf_bathy, netcdf_profile
    d = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "std14.npz"))
    prof = {"time": d["p_time"], "depth": d["p_depth"], "lat": d["p_lat"], "lon": d["p_lon"],
            "speed": d["p_speed"]}
    bathy = {"lat": d["b_lat"], "lon": d["b_lon"], "depth": d["b_depth"]}
    lat1, lat2, lng1, lng2 = 16.2, 24.6, -164.4, -155.5
    ssp = netcdf_profile(prof, 0.0, lat1, lat2, lng1, lng2)
    bottom = netcdf_bathy(bathy, lat1, lat2, lng1, lng2, T.earth_radius())
    return ocean_model(boundary_flat(), boundary_grid(bottom), profile_grid(ssp))


def std14(num_targets=100, time_max=80.0):
    """studies/cmp_speed/cmp_speed.cc:33-114 (the reference's published
    speed study): source 200 m deep at 19.52N 160.5W, 250 Hz, 181
    tangent-spaced D/E x AZ 0..360 step 15 (25 rays, wrapping), dt 0.1 s
    for 80 s, num_targets on a 100 km ring starting one bearing step from
    north.  As in the study, the ring takes the source's altitude (the
    100 m target depth it declares is overwritten) and the earth radius
    keeps its default."""
    T.set_earth_radius(6371000.0)
    ocean = std14_ocean()
    src = T.wposition1(19.52, -160.5, -200.0)
    tgt = None
    if num_targets > 0:
        tgt = T.wposition(num_targets, 1, src.latitude(), src.longitude(), 100.0)
        angle = 2.0 * math.pi / num_targets
        bearing = angle
        for n in range(num_targets):
            spot = T.wposition1(src, 100000.0, bearing)
            tgt.latitude(n, 0, spot.latitude())
            tgt.longitude(n, 0, spot.longitude())
            tgt.altitude(n, 0, spot.altitude())
            bearing += angle
    return _pack(ocean=ocean, freq=T.seq_linear(250.0, 1.0, 1), pos=src, de=T.seq_rayfan(-90.0, 90.0, 181),
                 az=T.seq_linear(0.0, 15.0, 360.0), dt=0.1, targets=tgt, time_max=time_max,
                 name="std14_%dtgt" % num_targets)


def build_queue(sc, queue_cls, **kw):
    """Constructs ``queue_cls(ocean, freq, pos, de, az, dt, targets, type)``
    and applies the scenario's threshold settings."""
    T.set_earth_radius(sc["earth_radius"])
    q = queue_cls(sc["ocean"], sc["freq"], sc["pos"], sc["de"], sc["az"], sc["dt"],
                  sc["targets"], sc["type"], **kw)
    for name, value in sc.get("thresholds", {}).items():
        getattr(q, name)(value)
    return q


def analytic_footprints(sensor_lat, sensor_lng, depth, de_values, az_values, num_freq):
    """Bottom eigenverbs of a sensor on the surface of isovelocity 1500 m/s
    water, in the shape of the reference's biverb test footprints
    (biverbs/test/biverbs_test.cc:41-77): for every (D/E, AZ) in degrees a
    footprint where the ray meets a flat bottom `depth` metres down, sized
    by the fan spacing, with power length x width / slant range^2 at every
    frequency.  Returns (wq3d_eigenverb array, power (n, num_freq)), built
    with numpy for large fans."""
    from . import _abi
    de = np.asarray(de_values, dtype=np.float64)
    az = np.asarray(az_values, dtype=np.float64)
    de_spacing = float(de[1] - de[0]) if de.size > 1 else 1.0
    az_spacing = float(az[1] - az[0]) if az.size > 1 else 1.0
    DE, AZ = np.meshgrid(de, az)            # AZ-major, as the reference's loops
    DE, AZ = DE.ravel(), AZ.ravel()
    n = DE.size
    de_rad, az_rad = np.radians(DE), np.radians(AZ)
    grazing = np.abs(de_rad)
    slant = depth / np.sin(grazing)
    horz = depth / np.tan(grazing)
    length = 0.5 * slant * math.radians(de_spacing) / np.sin(grazing)
    width = 0.5 * slant * math.radians(az_spacing) * np.cos(grazing)
    R = T.earth_radius()
    lat1, lng1 = math.radians(sensor_lat), math.radians(sensor_lng)
    rng = horz / R
    lat2 = np.arcsin(math.sin(lat1) * np.cos(rng) + math.cos(lat1) * np.sin(rng) * np.cos(az_rad))
    lng2 = lng1 + np.arctan2(np.sin(az_rad) * np.sin(rng) * math.cos(lat1),
                             np.cos(rng) - math.sin(lat1) * np.sin(lat2))
    recs = (_abi.wq3d_eigenverb * max(n, 1))()
    a = np.ctypeslib.as_array(recs)[:n]
    a["travel_time"] = slant / 1500.0
    a["length"] = length
    a["width"] = width
    pos = np.stack([np.full(n, R - depth), np.pi / 2 - lat2, lng2], axis=1)
    a["position"] = pos
    a["direction"] = az_rad
    a["grazing"] = grazing
    a["sound_speed"] = 1500.0
    a["source_de"] = de_rad
    a["source_az"] = az_rad
    a["de"] = np.round((90.0 + DE) / de_spacing - 1.0).astype(np.int32)
    a["az"] = np.round(AZ / az_spacing).astype(np.int32)
    power = np.repeat((length * width / (slant * slant))[:, None], num_freq, axis=1)
    return recs, np.ascontiguousarray(power)
