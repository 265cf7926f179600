"""Host mirror of USML's sequence and geodetic position types.

These follow the reference's arithmetic exactly (Python floats are IEEE
doubles and Python never fuses a multiply-add), so a fan or a target grid
built here holds the same bits as the reference's objects:

* ``seq_linear`` -- types/seq_linear.h:30-116 (values accumulate by repeated
  addition; the increment is the constant given, not a difference)
* ``seq_log``    -- types/seq_log.h:28-115
* ``seq_rayfan`` -- types/seq_rayfan.cc:19-47 (tangent spaced D/E fan)
* ``seq_data``   -- types/seq_data.h (increments are forward differences,
  the last repeats the previous one)
* ``wposition`` / ``wposition1`` -- types/wposition.{h,cc},
  types/wposition1.cc (earth radius is the module-level global, as in the
  reference, and ``compute_earth_radius`` is the WGS-84 formula).
"""
import math

import numpy as np


def to_radians(t):
    return t * (math.pi / 180.0)


def to_degrees(t):
    return t * (180.0 / math.pi)


class seq_vector:
    """A monotonic sequence with per-element increments."""

    def __init__(self, values, increments):
        self._data = np.asarray(values, dtype=np.float64)
        self._inc = np.asarray(increments, dtype=np.float64)

    def size(self):
        return int(self._data.size)

    def __len__(self):
        return self.size()

    def __getitem__(self, i):
        return float(self._data[i])

    def __call__(self, i):
        return float(self._data[i])

    def increment(self, i):
        """seq_vector::increment clamps the index to the last element
        (seq_vector.h:140-143); its index is unsigned, so -1 clamps there
        too."""
        i = int(i)
        if i < 0 or i > self.size() - 1:
            i = self.size() - 1
        return float(self._inc[i])

    @property
    def data(self):
        return self._data

    @property
    def increments(self):
        return self._inc


class seq_linear(seq_vector):
    """seq_linear(first, increment, size|last[, first_last]).

    As in the reference's overloads, an ``int`` third argument is a size and
    a ``float`` third argument is the last value."""

    def __init__(self, first, increment, third, first_last=False):
        first = float(first)
        increment = float(increment)
        if isinstance(third, (int, np.integer)) and not isinstance(third, bool):
            size = int(third)
            inc = (float(increment) - first) / (size - 1) if first_last else increment
        else:
            last = float(third)
            inc = increment
            if increment == 0.0:
                size = 1
            else:
                size = max(1, int(math.floor(1.0 + (last + increment / 10 - first) / increment)))
        data = np.empty(size)
        v = first
        for n in range(size):
            data[n] = v
            v += inc
        super().__init__(data, np.full(size, inc))


class seq_log(seq_vector):
    """seq_log(first, increment, size|last)."""

    def __init__(self, first, increment, third):
        first = float(first)
        increment = float(increment)
        if isinstance(third, (int, np.integer)) and not isinstance(third, bool):
            size = int(third)
        else:
            last = float(third)
            if increment == 1.0:
                size = 1
            else:
                size = max(1, int(math.floor(1.0 + (math.log((last + increment / 10) / first)
                                                     / math.log(increment)))))
        data = np.empty(size)
        inc = np.zeros(size)
        v = first
        for n in range(size):
            data[n] = v
            v *= increment
            if n > 0:
                inc[n - 1] = data[n] - data[n - 1]
                inc[n] = inc[n - 1]
        super().__init__(data, inc)


class seq_data(seq_vector):
    """Arbitrary monotonic data (seq_data.h init)."""

    def __init__(self, values):
        values = np.asarray(values, dtype=np.float64)
        size = values.size
        inc = np.zeros(size)
        if size >= 2:
            left = values[1] - values[0]
            inc[0] = left
            for n in range(1, size):
                right = left
                if n < size - 1:
                    right = values[n + 1] - values[n]
                    if left * right <= 0:
                        raise ValueError("series not monotonic")
                left = right
                inc[n] = left
        super().__init__(values, inc)


class seq_rayfan(seq_data):
    """Tangent spaced fan (seq_rayfan.cc:19-47)."""

    def __init__(self, first=-90.0, last=90.0, size=181, center=0.0, spread=6.0):
        if first > last:
            first, last = last, first
        first_ang = math.atan((first - center) / spread)
        last_ang = math.atan((last - center) / spread)
        scale = (last_ang - first_ang) / float(size - 1)
        data = np.empty(size)
        for n in range(size):
            x = first_ang + scale * float(n)
            data[n] = center + math.tan(x) * spread
        super().__init__(data)


class _Earth:
    radius = 6371000.0


def earth_radius():
    return _Earth.radius


def set_earth_radius(value):
    _Earth.radius = float(value)


def compute_earth_radius(latitude):
    """wposition::compute_earth_radius (types/wposition.cc:33-42)."""
    a = 6378137.0
    f = 1.0 / 298.257223563
    e2 = f * (2.0 - f)
    sinT = math.sin(to_radians(latitude))
    w = math.sqrt(1.0 - e2 * sinT * sinT)
    rm = a * (1 - e2) / (w * w * w)
    rv = a / w
    _Earth.radius = math.sqrt(rm * rv)
    return _Earth.radius


class wposition1:
    """Single geodetic position stored as (rho, theta, phi)."""

    def __init__(self, *args):
        self.rho = 0.0
        self.theta = 0.0
        self.phi = 0.0
        if len(args) == 3 and isinstance(args[0], wposition1):
            self._from_range_bearing(*args)
        elif len(args) == 3:
            self.latitude(args[0])
            self.longitude(args[1])
            self.altitude(args[2])
        elif len(args) == 0:
            pass
        else:
            raise TypeError("wposition1(lat, lng, alt) or wposition1(pos, range, bearing)")

    def _from_range_bearing(self, location, rng, bearing):
        """wposition1.cc:23-37 (great circle range and bearing in radians)."""
        lat1 = to_radians(location.latitude())
        lng1 = to_radians(location.longitude())
        R = _Earth.radius + location.altitude()
        rng = rng / R
        lat2 = math.asin(math.sin(lat1) * math.cos(rng) + math.cos(lat1) * math.sin(rng) * math.cos(bearing))
        lng2 = lng1 + math.atan2(math.sin(bearing) * math.sin(rng) * math.cos(lat1),
                                 math.cos(rng) - math.sin(lat1) * math.sin(lat2))
        self.latitude(to_degrees(lat2))
        self.longitude(to_degrees(lng2))
        self.altitude(location.altitude())

    def latitude(self, value=None):
        if value is None:
            return 90.0 - to_degrees(self.theta)
        self.theta = to_radians(90.0 - value)

    def longitude(self, value=None):
        if value is None:
            return to_degrees(self.phi)
        self.phi = to_radians(value)

    def altitude(self, value=None):
        if value is None:
            return self.rho - _Earth.radius
        self.rho = value + _Earth.radius

    def copy(self):
        p = wposition1()
        p.rho, p.theta, p.phi = self.rho, self.theta, self.phi
        return p


class wposition:
    """Matrix of geodetic positions (rows x cols) as rho/theta/phi arrays."""

    def __init__(self, rows=1, cols=1, latitude=0.0, longitude=0.0, altitude=0.0):
        self.rho = np.full((rows, cols), altitude + _Earth.radius)
        self.theta = np.full((rows, cols), to_radians(90.0 - latitude))
        self.phi = np.full((rows, cols), to_radians(longitude))

    @classmethod
    def mesh(cls, latitudes, longitudes, altitude=0.0):
        lat = np.asarray(latitudes, dtype=np.float64)
        lng = np.asarray(longitudes, dtype=np.float64)
        p = cls(lat.size, lng.size)
        for n in range(lat.size):
            for m in range(lng.size):
                p.latitude(n, m, float(lat[n]))
                p.longitude(n, m, float(lng[m]))
                p.altitude(n, m, altitude)
        return p

    def size1(self):
        return self.rho.shape[0]

    def size2(self):
        return self.rho.shape[1]

    def latitude(self, r, c, value=None):
        if value is None:
            return 90.0 - to_degrees(float(self.theta[r, c]))
        self.theta[r, c] = to_radians(90.0 - value)

    def longitude(self, r, c, value=None):
        if value is None:
            return to_degrees(float(self.phi[r, c]))
        self.phi[r, c] = to_radians(value)

    def altitude(self, r, c, value=None):
        if value is None:
            return float(self.rho[r, c]) - _Earth.radius
        self.rho[r, c] = value + _Earth.radius

    def packed(self):
        """All rho, then all theta, then all phi (row-major), as the C ABI wants."""
        return np.ascontiguousarray(np.concatenate([self.rho.ravel(), self.theta.ravel(),
                                                    self.phi.ravel()]))
