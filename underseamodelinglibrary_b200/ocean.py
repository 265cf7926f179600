"""Host mirror of the USML ocean models that the WaveQ3D path calls.

Each class records its parameters the way the reference constructor does
(including the earth radius that boundaries bake in at construction,
ocean/boundary_flat.cc:19-21) and contributes to a ``wq3d_ocean_desc``.
The models are evaluated on the GPU by the engine; ``ocean_model`` also
exposes the engine's point evaluations for model-level checks.
"""
import ctypes as C

import numpy as np

from . import _abi
from .types import earth_radius, seq_linear, seq_log


class data_grid:
    """N-dimensional rectilinear grid (types/data_grid.h, gen_grid.h) of
    up to three axes; data is row-major with the last axis fastest.
    Interpolation defaults to linear with edge limiting on every axis
    (data_grid.h:315-316)."""
    NEAREST, LINEAR, PCHIP = _abi.INTERP_NEAREST, _abi.INTERP_LINEAR, _abi.INTERP_PCHIP

    def __init__(self, axes, data):
        self.axes = list(axes)
        self.data = np.ascontiguousarray(np.asarray(data, dtype=np.float64).reshape(
            [a.size() for a in self.axes]))
        self._interp = [_abi.INTERP_LINEAR] * len(self.axes)
        self._edge = [True] * len(self.axes)

    def interp_type(self, dim, kind):
        self._interp[dim] = int(kind)

    def edge_limit(self, dim, flag):
        self._edge[dim] = bool(flag)

    def fill(self, g, keep):
        g.ndim = len(self.axes)
        for k, a in enumerate(self.axes):
            x = np.ascontiguousarray(a.data, dtype=np.float64)
            inc = np.ascontiguousarray(a.increments, dtype=np.float64)
            keep += [x, inc]
            g.axis[k] = _abi.as_dp(x)
            g.axis_inc[k] = _abi.as_dp(inc)
            g.axis_size[k] = a.size()
            g.axis_kind[k] = (_abi.AXIS_LINEAR if isinstance(a, seq_linear)
                              else _abi.AXIS_LOG if isinstance(a, seq_log) else _abi.AXIS_DATA)
            g.interp[k] = self._interp[k]
            g.edge_limit[k] = 1 if self._edge[k] else 0
        keep.append(self.data)
        g.data = _abi.as_dp(self.data)


class attenuation_thorp:
    """ocean/attenuation_thorp.cc:14-36 (the profile default)."""
    kind = _abi.ATTEN_THORP
    coefficient = 0.0


class attenuation_constant:
    """ocean/attenuation_constant.cc:14-25: coefficient * distance * frequency."""
    kind = _abi.ATTEN_CONSTANT

    def __init__(self, coefficient):
        self.coefficient = float(coefficient)


class profile_model:
    kind = None
    params = (0.0, 0.0, 0.0, 0.0)

    def __init__(self, attmodel=None):
        self._atten = attmodel if attmodel is not None else attenuation_thorp()
        self._flat_earth = False

    def flat_earth(self, flat):
        """profile_model::flat_earth (profile_model.h:61)."""
        self._flat_earth = bool(flat)

    def attenuation(self, model):
        self._atten = model

    def fill(self, d):
        d.kind = self.kind
        for k in range(4):
            d.p[k] = self.params[k]
        d.flat_earth = 1 if self._flat_earth else 0
        d.attenuation = self._atten.kind
        d.attenuation_coef = self._atten.coefficient


class profile_linear(profile_model):
    """profile_linear(c0[, g0[, z1, g1]][, attmodel]) (profile_linear.h)."""
    kind = _abi.PROFILE_LINEAR

    def __init__(self, c0=1500.0, *args):
        att = None
        nums = []
        for a in args:
            if isinstance(a, (int, float)):
                nums.append(float(a))
            else:
                att = a
        super().__init__(att)
        if len(nums) == 0:
            self.params = (float(c0), 0.0, 0.0, 0.0)
        elif len(nums) == 1:
            self.params = (float(c0), nums[0], 0.0, nums[0])
        elif len(nums) == 3:
            self.params = (float(c0), nums[0], nums[1], nums[2])
        else:
            raise TypeError("profile_linear(c0, g0) or profile_linear(c0, g0, z1, g1)")


class profile_munk(profile_model):
    """profile_munk.h:40-60 defaults: axis 1300 m, scale 1300 m, 1500 m/s, 7.37e-3."""
    kind = _abi.PROFILE_MUNK

    def __init__(self, axis_depth=1300.0, scale=1300.0, axis_speed=1500.0,
                 epsilon=7.37e-3, attmodel=None):
        super().__init__(attmodel)
        self.params = (float(axis_depth), float(scale), float(axis_speed), float(epsilon))


class profile_catenary(profile_model):
    kind = _abi.PROFILE_CATENARY

    def __init__(self, c1, g1, z1, attmodel=None):
        super().__init__(attmodel)
        self.params = (float(c1), float(g1), float(z1), 0.0)


class profile_n2(profile_model):
    kind = _abi.PROFILE_N2

    def __init__(self, c0, g0, attmodel=None):
        super().__init__(attmodel)
        self.params = (float(c0), float(g0), 0.0, 0.0)


class profile_grid(profile_model):
    """profile_grid<N> (ocean/profile_grid.h:68-130): sound speed on a grid
    over (rho[, theta[, phi]])."""
    kind = _abi.PROFILE_GRID

    def __init__(self, grid, attmodel=None):
        super().__init__(attmodel)
        self.grid = grid

    def fill(self, d, keep=None):
        super().fill(d)
        self.grid.fill(d.grid, keep if keep is not None else [])


class reflect_loss_constant:
    """reflect_loss_constant.h:42-52."""
    kind = _abi.LOSS_CONSTANT

    def __init__(self, amplitude, phase=0.0):
        self.params = (float(amplitude), float(phase), 0.0, 0.0, 0.0)


class reflect_loss_rayleigh:
    """reflect_loss_rayleigh(density, speed, att_bottom, speed_shear, att_shear)
    as ratios to water (reflect_loss_rayleigh.cc:68-78), or a bottom type."""
    kind = _abi.LOSS_RAYLEIGH
    # Jensen et al. table 1.3 (reflect_loss_rayleigh.cc:27-39)
    TABLE = {"clay": (1.5, 1.00, 0.2, 0.00, 1.0), "silt": (1.7, 1.05, 1.0, 0.00, 1.5),
             "sand": (1.9, 1.10, 0.8, 0.00, 2.5), "gravel": (2.0, 1.20, 0.6, 0.00, 1.5),
             "moraine": (2.1, 1.30, 0.4, 0.40, 1.0), "chalk": (2.2, 1.60, 0.2, 0.67, 0.5),
             "limestone": (2.4, 2.00, 0.1, 1.00, 0.2), "basalt": (2.7, 3.50, 0.1, 1.67, 0.2)}

    def __init__(self, density, speed=None, att_bottom=0.0, speed_shear=0.0, att_shear=0.0):
        if isinstance(density, str):
            self.params = self.TABLE[density]
        else:
            self.params = (float(density), float(speed), float(att_bottom),
                           float(speed_shear), float(att_shear))


class reflect_loss_eckart:
    """reflect_loss_eckart.h:76-85."""
    kind = _abi.LOSS_ECKART

    def __init__(self, wind_speed):
        self.params = (float(wind_speed), 0.0, 0.0, 0.0, 0.0)


class scattering_model:
    """Scattering strength of an interface (ocean/scattering_model.h),
    evaluated on the GPU by the bistatic eigenverb kernels."""
    kind = None

    def __init__(self, p):
        self.p = float(p)

    def desc(self):
        d = _abi.wq3d_scattering_desc()
        d.kind = self.kind
        d.p = self.p
        return d


class scattering_constant(scattering_model):
    """scattering_constant(amplitude=-300) (ocean/scattering_constant.h):
    the same strength, in dB, at every angle and frequency."""
    kind = _abi.SCATTER_CONSTANT

    def __init__(self, amplitude=-300.0):
        super().__init__(amplitude)


class scattering_lambert(scattering_model):
    """scattering_lambert(bss=-27) (ocean/scattering_lambert.h):
    10^(bss/10) |sin(de_incident) sin(de_scattered)|."""
    kind = _abi.SCATTER_LAMBERT

    def __init__(self, bss=-27.0):
        super().__init__(bss)


class scattering_chapman(scattering_model):
    """scattering_chapman(wind_speed) (ocean/scattering_chapman.h): the
    Chapman-Harris surface scattering strength for a wind speed in m/s."""
    kind = _abi.SCATTER_CHAPMAN

    def __init__(self, wind_speed):
        super().__init__(wind_speed)


class boundary_model:
    kind = None

    def __init__(self, reflect_loss=None, scattering=None):
        self._loss = reflect_loss
        self._scattering = scattering if scattering is not None else scattering_constant()
        self._radius = earth_radius()

    def reflect_loss(self, model):
        self._loss = model

    def scattering(self, model=None):
        """boundary_model::scattering: the interface's scattering strength
        model (scattering_constant(-300 dB) unless one is given)"""
        if model is None:
            return self._scattering
        self._scattering = model

    def fill(self, d):
        d.kind = self.kind
        if self._loss is None:
            d.loss.kind = _abi.LOSS_DEFAULT
        else:
            d.loss.kind = self._loss.kind
            for k in range(5):
                d.loss.p[k] = self._loss.params[k]


class boundary_flat(boundary_model):
    """boundary_flat(depth=0, reflect_loss, scattering) (boundary_flat.cc:
    19-31)."""
    kind = _abi.BOUNDARY_FLAT

    def __init__(self, depth=0.0, reflect_loss=None, scattering=None):
        super().__init__(reflect_loss, scattering)
        self.depth = float(depth)

    def fill(self, d):
        super().fill(d)
        d.depth = self.depth


class boundary_slope(boundary_model):
    """boundary_slope(location, depth, lat_slope, lng_slope, reflect_loss)
    (boundary_slope.cc:13-24).  The reference keeps a reference to the
    caller's location; this copies it."""
    kind = _abi.BOUNDARY_SLOPE

    def __init__(self, location, depth, lat_slope, lng_slope=0.0, reflect_loss=None, scattering=None):
        super().__init__(reflect_loss, scattering)
        self.location = (location.rho, location.theta, location.phi)
        self.depth = float(depth)
        self.lat_slope = float(lat_slope)
        self.lng_slope = float(lng_slope)

    def fill(self, d):
        super().fill(d)
        d.depth = self.depth
        for k in range(3):
            d.location[k] = self.location[k]
        d.lat_slope = self.lat_slope
        d.lng_slope = self.lng_slope


class boundary_grid(boundary_model):
    """boundary_grid<N> (ocean/boundary_grid.h:40-204): boundary rho on a
    grid over theta[, phi]; Rayleigh sand loss unless one is given."""
    kind = _abi.BOUNDARY_GRID

    def __init__(self, grid, reflect_loss=None, scattering=None):
        super().__init__(reflect_loss, scattering)
        self.grid = grid

    def fill(self, d, keep=None):
        super().fill(d)
        self.grid.fill(d.grid, keep if keep is not None else [])


class volume_flat:
    """volume_flat(depth, thickness, amplitude) (ocean/volume_flat.h:32-37)
    or volume_flat(depth, thickness, scattering) (volume_flat.h:47-50): a
    scattering layer at a constant depth below mean sea level."""

    def __init__(self, depth=0.0, thickness=0.0, amplitude=-300.0):
        self.depth = float(depth)
        self.thickness = float(thickness)
        if isinstance(amplitude, scattering_model):
            self._scattering = amplitude
            self.amplitude = amplitude.p if amplitude.kind == _abi.SCATTER_CONSTANT else -300.0
        else:
            self.amplitude = float(amplitude)
            self._scattering = scattering_constant(self.amplitude)

    def scattering(self):
        return self._scattering


class ocean_model:
    """ocean_model(surface, bottom, profile) (ocean/ocean_model.h:31-60)."""

    def __init__(self, surface, bottom, profile):
        self._surface = surface
        self._bottom = bottom
        self._profile = profile
        self._volume = []
        self._handle = None
        self._lib = None

    def surface(self):
        return self._surface

    def add_volume(self, layer):
        """ocean_model::add_volume (ocean/ocean_model.h:52); layers are
        placed under the same earth radius as the boundaries."""
        if len(self._volume) >= _abi.MAX_VOLUME:
            raise ValueError("at most %d volume layers" % _abi.MAX_VOLUME)
        if self._handle is not None:
            raise RuntimeError("add volume layers before the ocean is first used")
        self._volume.append(layer)

    def num_volume(self):
        return len(self._volume)

    def scattering_model(self, interface):
        """the scattering strength model of an interface, chosen as
        ocean_model::scattering does (ocean/ocean_model.h:88-112): 0 bottom,
        1 surface, 2 + 2k and 3 + 2k the two sides of volume layer k"""
        if interface == 0:
            return self._bottom.scattering()
        if interface == 1:
            return self._surface.scattering()
        return self._volume[(int(interface) - 2) // 2].scattering()

    def volume(self, n):
        return self._volume[n]

    def bottom(self):
        return self._bottom

    def profile(self):
        return self._profile

    def descriptor(self):
        """The wq3d_ocean_desc; the arrays it points into stay alive as
        long as this ocean_model does."""
        d = _abi.wq3d_ocean_desc()
        d.earth_radius = self._bottom._radius
        self._keep = []
        for model, sub in ((self._profile, d.profile), (self._surface, d.surface), (self._bottom, d.bottom)):
            if isinstance(model, (profile_grid, boundary_grid)):
                model.fill(sub, self._keep)
            else:
                model.fill(sub)
        d.num_volume = len(self._volume)
        for k, layer in enumerate(self._volume):
            d.volume[k].depth = layer.depth
            d.volume[k].thickness = layer.thickness
            d.volume[k].amplitude = layer.amplitude
        # one construction radius serves both boundaries: build them under
        # the same wposition earth radius, as every reference caller does
        return d

    def handle(self):
        """Device-resident copy (built on first use)."""
        if self._handle is None:
            lib = _abi.load_engine()
            h = C.c_void_p()
            _abi.check(lib, lib.wq3d_ocean_create(C.byref(self.descriptor()), C.byref(h)))
            self._handle = h
            self._lib = lib
        return self._handle

    def __del__(self):
        if self._handle is not None and self._lib is not None:
            try:
                self._lib.wq3d_ocean_destroy(self._handle)
            except Exception:
                pass

    # GPU point evaluations (profile_model::sound_speed, boundary_model::height,
    # boundary_model::reflect_loss)
    def sound_speed(self, rho, theta=None, phi=None):
        rho = np.ascontiguousarray(rho, dtype=np.float64).ravel()
        n = rho.size
        theta = np.zeros(n) if theta is None else np.ascontiguousarray(theta, dtype=np.float64).ravel()
        phi = np.zeros(n) if phi is None else np.ascontiguousarray(phi, dtype=np.float64).ravel()
        c = np.empty(n)
        g = np.empty(3 * n)
        lib = _abi.load_engine()
        _abi.check(lib, lib.wq3d_ocean_sound_speed(self.handle(), earth_radius(), n, _abi.as_dp(rho),
                                                   _abi.as_dp(theta), _abi.as_dp(phi),
                                                   _abi.as_dp(c), _abi.as_dp(g)))
        return c, g.reshape(3, n)

    def height(self, which, theta, phi):
        theta = np.ascontiguousarray(theta, dtype=np.float64).ravel()
        phi = np.ascontiguousarray(phi, dtype=np.float64).ravel()
        n = theta.size
        h = np.empty(n)
        nrm = np.empty(3 * n)
        rho = np.zeros(n)
        lib = _abi.load_engine()
        _abi.check(lib, lib.wq3d_ocean_height(self.handle(), int(which), n, _abi.as_dp(rho),
                                              _abi.as_dp(theta), _abi.as_dp(phi),
                                              _abi.as_dp(h), _abi.as_dp(nrm)))
        return h, nrm.reshape(3, n)

    def attenuation(self, rho, distance, freq):
        """Absorption (dB) over ``distance`` metres at each point, as
        (n, nf) (attenuation_model::attenuation)."""
        r = np.ascontiguousarray(rho, dtype=np.float64).ravel()
        d = np.ascontiguousarray(np.broadcast_to(distance, r.shape), dtype=np.float64)
        f = np.ascontiguousarray(freq, dtype=np.float64).ravel()
        out = np.empty(r.size * f.size)
        lib = _abi.load_engine()
        _abi.check(lib, lib.wq3d_ocean_attenuation(self.handle(), earth_radius(), r.size, _abi.as_dp(r),
                                                   _abi.as_dp(d), f.size, _abi.as_dp(f), _abi.as_dp(out)))
        return out.reshape(r.size, f.size)

    def reflect_loss(self, which, grazing, freq):
        g = np.ascontiguousarray(grazing, dtype=np.float64).ravel()
        f = np.ascontiguousarray(freq, dtype=np.float64).ravel()
        n, nf = g.size, f.size
        z = np.zeros(n)
        amp = np.empty(n * nf)
        ph = np.empty(n * nf)
        lib = _abi.load_engine()
        _abi.check(lib, lib.wq3d_ocean_reflect_loss(self.handle(), int(which), n, _abi.as_dp(z),
                                                    _abi.as_dp(z), _abi.as_dp(z), _abi.as_dp(g), nf,
                                                    _abi.as_dp(f), _abi.as_dp(amp), _abi.as_dp(ph)))
        return amp.reshape(n, nf), ph.reshape(n, nf)
