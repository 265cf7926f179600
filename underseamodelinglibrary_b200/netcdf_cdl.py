"""Gridded environments from netCDF data written as CDL text (the output
of ``ncdump``), with the reference's loader semantics:

* ``netcdf_profile`` -- netcdf/netcdf_profile.cc:28-160: a 4-D (time,
  depth, lat, lon) variable; the time slice nearest ``date``; rho axis
  ``seq_data(earth_radius - altitude)`` as stored (:57-60); the lat/lon
  window selected with the file's uniform increments (:67-115), colatitude
  axis decreasing; ``_FillValue`` to NaN, ``scale_factor`` / ``add_offset``
  applied (:145-160).  Linear interpolation with edge limits on every axis
  (data_grid defaults).
* ``netcdf_bathy`` -- netcdf/netcdf_bathy.cc:22-173: a 2-D (lat, lon)
  altitude variable over the same window rules, plus ``earth_radius`` to
  make boundary rho (:168-173).

Arrays can come from a CDL file (``read_cdl``) or from a dict of numpy
arrays with the same variable names (as saved in the package's data
files), so the loaders need no netCDF library.
"""
import math
import re

import numpy as np

from . import types as T
from .ocean import data_grid


def read_cdl(path):
    """Parses CDL text into {"dims": {name: size}, "vars": {name: dims},
    "attrs": {var: {att: value}}, "data": {name: ndarray}}."""
    text = open(path).read()
    dims, vars_, attrs, data = {}, {}, {}, {}
    sec = None
    body = text[text.index("{") + 1:text.rindex("}")]
    # split the data section values on ';'
    head, _, data_txt = body.partition("data:")
    for line in head.splitlines():
        line = line.strip()
        if not line:
            continue
        if line.startswith("dimensions:"):
            sec = "dims"
            line = line[len("dimensions:"):].strip()
            if not line:
                continue
        elif line.startswith("variables:"):
            sec = "vars"
            continue
        if sec == "dims":
            for part in line.rstrip(";").split(","):
                if "=" in part:
                    k, v = part.split("=")
                    dims[k.strip()] = int(v.strip())
        elif sec == "vars":
            m = re.match(r"(\w+):(\w+)\s*=\s*(.*?);?$", line)
            if m and not re.match(r"^(float|double|int|short|byte|char)\b", line):
                val = m.group(3).strip().rstrip(";").strip()
                if val.startswith('"'):
                    val = val.strip('"')
                else:
                    try:
                        val = float(val.rstrip("fFdDsSbBlL"))
                    except ValueError:
                        pass
                attrs.setdefault(m.group(1), {})[m.group(2)] = val
                continue
            m = re.match(r"^(float|double|int|short|byte)\s+(.*?);$", line)
            if m:
                for decl in re.findall(r"(\w+)\s*\(([^)]*)\)", m.group(2)):
                    vars_[decl[0]] = tuple(d.strip() for d in decl[1].split(","))
    for stmt in data_txt.split(";"):
        if "=" not in stmt:
            continue
        name, _, vals = stmt.partition("=")
        name = name.strip()
        if name not in vars_:
            continue
        arr = np.array([float(v) for v in vals.replace("\n", " ").split(",") if v.strip()])
        shape = tuple(dims[d] for d in vars_[name])
        data[name] = arr.reshape(shape)
    return {"dims": dims, "vars": vars_, "attrs": attrs, "data": data}


def _window(values, lo, hi, global_ok=False):
    """index range and uniform increment of a lat (or lon) window, as the
    loaders compute them (netcdf_profile.cc:90-115)"""
    v0, vn = float(values[0]), float(values[-1])
    n_max = len(values) - 1
    inc = (vn - v0) / n_max
    first = max(0, int(math.floor(1e-6 + (lo - v0) / inc)))
    last = min(n_max, int(math.floor(0.5 + (hi - v0) / inc)))
    return first, last, inc, v0


def _lon_offset(lon, west, east):
    """the +-360 degree shift of netcdf_profile.cc:67-88 for non-global data"""
    v0, vn = float(lon[0]), float(lon[-1])
    zero_to_360 = v0 < 1.0 and vn >= 359.0
    bounds_180 = v0 < -179.0 and vn > 179.0
    if zero_to_360 or bounds_180:
        raise ValueError("global longitude grids are not supported by this loader")
    offset = 0.0
    if v0 > 180.0:
        if west < 0.0:
            offset = 360.0
    elif v0 < 0.0:
        if east > 180.0:
            offset = -360.0
    return offset


def _vars(src):
    return src["data"] if isinstance(src, dict) and "data" in src else src


def netcdf_profile(src, date, south, north, west, east, earth_radius=None, names=None):
    """data_grid<3> of sound speed over (rho, theta, phi), as
    netcdf_profile(filename, date, south, north, west, east) builds it.
    ``src`` is read_cdl() output or a dict of arrays; ``names`` maps
    (time, depth, lat, lon, speed) to variable names."""
    d = _vars(src)
    nt, nd, nla, nlo, nv = names or ("time", "depth", "lat", "lon", "speed")
    R = T.earth_radius() if earth_radius is None else earth_radius
    times = np.atleast_1d(d[nt])
    ti = 0
    old = abs(date - times[0])
    for t in range(1, len(times)):
        if old > abs(date - times[t]):
            old = abs(date - times[t])
            ti = t
    alt = np.asarray(d[nd], dtype=np.float64)
    rho = T.seq_data(R - alt)
    lat, lon = np.asarray(d[nla], dtype=np.float64), np.asarray(d[nlo], dtype=np.float64)
    offset = _lon_offset(lon, west, east)
    west += offset
    east += offset
    lat_first, lat_last, inc_lat, lat0 = _window(lat, south, north)
    lon_first, lon_last, inc_lon, lon0 = _window(lon, west, east)
    th = T.seq_linear(math.radians(90.0 - (lat_first * inc_lat + lat0)), math.radians(-inc_lat),
                      lat_last - lat_first + 1)
    ph = T.seq_linear(math.radians(lon_first * inc_lon + lon0 - offset), math.radians(inc_lon),
                      lon_last - lon_first + 1)
    vals = np.asarray(d[nv], dtype=np.float64)[ti, :, lat_first:lat_last + 1, lon_first:lon_last + 1].copy()
    attrs = src.get("attrs", {}).get(nv, {}) if isinstance(src, dict) else {}
    if "_FillValue" in attrs:
        vals[vals == attrs["_FillValue"]] = np.nan
    if "scale_factor" in attrs and "add_offset" in attrs:
        vals = vals * attrs["scale_factor"] + attrs["add_offset"]
    return data_grid([rho, th, ph], vals)


def netcdf_bathy(src, south, north, west, east, earth_radius=None, names=None):
    """data_grid<2> of boundary rho over (theta, phi), as
    netcdf_bathy(filename, south, north, west, east, earth_radius) builds
    it."""
    d = _vars(src)
    nla, nlo, nz = names or ("lat", "lon", "depth")
    R = T.earth_radius() if earth_radius is None else earth_radius
    lat, lon = np.asarray(d[nla], dtype=np.float64), np.asarray(d[nlo], dtype=np.float64)
    offset = _lon_offset(lon, west, east)
    west += offset
    east += offset
    lat_first, lat_last, inc_lat, lat0 = _window(lat, south, north)
    lon_first, lon_last, inc_lon, lon0 = _window(lon, west, east)
    th = T.seq_linear(math.radians(90.0 - (lat_first * inc_lat + lat0)), math.radians(-inc_lat),
                      lat_last - lat_first + 1)
    ph = T.seq_linear(math.radians(lon_first * inc_lon + lon0 - offset), math.radians(inc_lon),
                      lon_last - lon_first + 1)
    vals = np.asarray(d[nz], dtype=np.float64)[lat_first:lat_last + 1, lon_first:lon_last + 1] + R
    return data_grid([th, ph], vals)
