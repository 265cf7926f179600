"""ctypes mirror of include/wq3d.h and the loader for the CUDA library.

The structures below must match the C declarations field for field.  The
engine library is ``libwq3d.so`` in this package directory; there is no
CPU fallback, so a missing library raises at load time.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# WQ3D_LIBRARY=checked selects the build whose kernels test every index
# they read from device data (libwq3d_checked.so, made by build.py)
LIB_PATH = os.path.join(HERE, "libwq3d_checked.so" if os.environ.get("WQ3D_LIBRARY") == "checked"
                        else "libwq3d.so")

WQ3D_OK = 0
WQ3D_ERR_INVALID = -1
WQ3D_ERR_CUDA = -2
WQ3D_ERR_NOMEM = -3
WQ3D_ERR_OVERFLOW = -4
WQ3D_ERR_TIMEOUT = -5
WQ3D_ERR_UNSUPPORTED = -6
WQ3D_ERR_NUMERIC = -7
WQ3D_ERR_ABORTED = -8
WQ3D_NOALLOC_MAX_POINTS = 16384

PROFILE_LINEAR, PROFILE_MUNK, PROFILE_CATENARY, PROFILE_N2, PROFILE_GRID = range(5)
ATTEN_THORP, ATTEN_CONSTANT = 0, 1
BOUNDARY_FLAT, BOUNDARY_SLOPE, BOUNDARY_GRID = 0, 1, 2
LOSS_DEFAULT, LOSS_CONSTANT, LOSS_RAYLEIGH, LOSS_ECKART = -1, 0, 1, 2
INTERP_NEAREST, INTERP_LINEAR, INTERP_PCHIP = -1, 0, 1
CLASSIC_RAY, HYBRID_GAUSSIAN = 0, 1
FP64, FP32C, FP32 = 0, 1, 2
REFLECT_AUTO, REFLECT_SIDE, REFLECT_INLINE = 0, 1, 2
FRONT_PAST, FRONT_PREV, FRONT_CURR, FRONT_NEXT = 0, 1, 2, 3

dp = C.POINTER(C.c_double)


AXIS_LINEAR, AXIS_LOG, AXIS_DATA = 0, 1, 2


class wq3d_grid_desc(C.Structure):
    _fields_ = [("ndim", C.c_int), ("axis", dp * 3), ("axis_inc", dp * 3),
                ("axis_size", C.c_size_t * 3), ("axis_kind", C.c_int * 3),
                ("data", dp), ("interp", C.c_int * 3), ("edge_limit", C.c_int * 3)]


class wq3d_profile_desc(C.Structure):
    _fields_ = [("kind", C.c_int), ("p", C.c_double * 4), ("flat_earth", C.c_int),
                ("attenuation", C.c_int), ("attenuation_coef", C.c_double),
                ("grid", wq3d_grid_desc)]


class wq3d_reflect_loss_desc(C.Structure):
    _fields_ = [("kind", C.c_int), ("p", C.c_double * 5)]


class wq3d_boundary_desc(C.Structure):
    _fields_ = [("kind", C.c_int), ("depth", C.c_double), ("location", C.c_double * 3),
                ("lat_slope", C.c_double), ("lng_slope", C.c_double),
                ("grid", wq3d_grid_desc), ("loss", wq3d_reflect_loss_desc)]


MAX_VOLUME = 4
VERB_BOTTOM, VERB_SURFACE, VERB_VOLUME_UPPER, VERB_VOLUME_LOWER = 0, 1, 2, 3


class wq3d_volume_desc(C.Structure):
    _fields_ = [("depth", C.c_double), ("thickness", C.c_double), ("amplitude", C.c_double)]


class wq3d_ocean_desc(C.Structure):
    _fields_ = [("earth_radius", C.c_double), ("profile", wq3d_profile_desc),
                ("surface", wq3d_boundary_desc), ("bottom", wq3d_boundary_desc),
                ("num_volume", C.c_int), ("volume", wq3d_volume_desc * MAX_VOLUME)]


class wq3d_queue_desc(C.Structure):
    _fields_ = [("freq", dp), ("num_freq", C.c_size_t), ("source", C.c_double * 3),
                ("de", dp), ("de_inc", dp), ("num_de", C.c_size_t),
                ("az", dp), ("az_inc", dp), ("num_az", C.c_size_t),
                ("time_step", C.c_double), ("targets", dp),
                ("num_targets1", C.c_size_t), ("num_targets2", C.c_size_t),
                ("spreading", C.c_int), ("precision", C.c_int),
                ("earth_radius", C.c_double), ("eigenray_capacity", C.c_size_t),
                ("device", C.c_int), ("run_id", C.c_uint64)]


class wq3d_thresholds(C.Structure):
    _fields_ = [("intensity", C.c_double), ("eigenverb", C.c_double),
                ("max_bottom", C.c_int), ("max_surface", C.c_int),
                ("max_caustic", C.c_int), ("max_upper", C.c_int), ("max_lower", C.c_int)]


class wq3d_eigenray(C.Structure):
    _fields_ = [("time", C.c_double), ("source_de", C.c_double), ("source_az", C.c_double),
                ("target_de", C.c_double), ("target_az", C.c_double),
                ("surface", C.c_int32), ("bottom", C.c_int32), ("caustic", C.c_int32),
                ("upper", C.c_int32), ("lower", C.c_int32), ("t1", C.c_int32),
                ("t2", C.c_int32), ("de", C.c_int32), ("az", C.c_int32),
                ("pad", C.c_int32), ("step", C.c_int64)]


class wq3d_reflection(C.Structure):
    _fields_ = [("time", C.c_double), ("dt", C.c_double), ("grazing", C.c_double),
                ("speed", C.c_double), ("position", C.c_double * 3),
                ("ndirection", C.c_double * 3), ("de", C.c_int32), ("az", C.c_int32),
                ("type", C.c_int32), ("pad", C.c_int32), ("step", C.c_int64)]


class wq3d_timing(C.Structure):
    _fields_ = [("ms_total", C.c_double), ("ms_advance", C.c_double), ("ms_reflect", C.c_double),
                ("ms_cpa", C.c_double), ("ms_eigenray", C.c_double), ("launches", C.c_int64)]


class wq3d_eigenverb(C.Structure):
    _fields_ = [("travel_time", C.c_double), ("length", C.c_double), ("width", C.c_double),
                ("position", C.c_double * 3), ("direction", C.c_double), ("grazing", C.c_double),
                ("sound_speed", C.c_double), ("source_de", C.c_double), ("source_az", C.c_double),
                ("de", C.c_int32), ("az", C.c_int32), ("surface", C.c_int32), ("bottom", C.c_int32),
                ("caustic", C.c_int32), ("upper", C.c_int32), ("lower", C.c_int32),
                ("interface_num", C.c_int32), ("step", C.c_int64), ("seq", C.c_int32),
                ("pad", C.c_int32)]


SCATTER_CONSTANT, SCATTER_LAMBERT, SCATTER_CHAPMAN = 0, 1, 2


class wq3d_scattering_desc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("pad", C.c_int32), ("p", C.c_double)]


class wq3d_biverb(C.Structure):
    _fields_ = [("travel_time", C.c_double), ("duration", C.c_double),
                ("source_de", C.c_double), ("source_az", C.c_double),
                ("receiver_de", C.c_double), ("receiver_az", C.c_double),
                ("de_index", C.c_int32), ("az_index", C.c_int32),
                ("source_surface", C.c_int32), ("source_bottom", C.c_int32),
                ("source_caustic", C.c_int32), ("source_upper", C.c_int32),
                ("source_lower", C.c_int32), ("receiver_surface", C.c_int32),
                ("receiver_bottom", C.c_int32), ("receiver_caustic", C.c_int32),
                ("receiver_upper", C.c_int32), ("receiver_lower", C.c_int32),
                ("source", C.c_int32), ("receiver", C.c_int32)]


ADD_EIGENRAY = C.CFUNCTYPE(None, C.c_void_p, C.c_size_t, C.c_size_t,
                           C.POINTER(wq3d_eigenray), dp, dp, C.c_size_t, C.c_uint64)
CHECK_EIGENRAYS = C.CFUNCTYPE(None, C.c_void_p, C.c_double, C.c_uint64)
REFLECT = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(wq3d_reflection))
ADD_EIGENVERB = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(wq3d_eigenverb), dp, C.c_size_t, C.c_int)


class wq3d_callbacks(C.Structure):
    _fields_ = [("add_eigenray", ADD_EIGENRAY), ("check_eigenrays", CHECK_EIGENRAYS),
                ("reflect", REFLECT), ("add_eigenverb", ADD_EIGENVERB)]


class wq3d_front_view(C.Structure):
    _fields_ = [("rho", dp), ("theta", dp), ("phi", dp), ("pos_grad", dp * 3),
                ("ndir", dp * 3), ("ndir_grad", dp * 3), ("sound_speed", dp),
                ("sound_grad", dp * 3), ("distance", dp), ("path_length", dp),
                ("attenuation", dp), ("phase", dp),
                ("surface", C.POINTER(C.c_int32)), ("bottom", C.POINTER(C.c_int32)),
                ("caustic", C.POINTER(C.c_int32)), ("upper", C.POINTER(C.c_int32)),
                ("lower", C.POINTER(C.c_int32)), ("on_edge", C.POINTER(C.c_uint8))]


# every symbol the header declares, with its ctypes signature
SIGNATURES = {
    "wq3d_ocean_create": (C.c_int, [C.POINTER(wq3d_ocean_desc), C.POINTER(C.c_void_p)]),
    "wq3d_ocean_destroy": (C.c_int, [C.c_void_p]),
    "wq3d_ocean_sound_speed": (C.c_int, [C.c_void_p, C.c_double, C.c_size_t, dp, dp, dp, dp, dp]),
    "wq3d_ocean_height": (C.c_int, [C.c_void_p, C.c_int, C.c_size_t, dp, dp, dp, dp, dp]),
    "wq3d_ocean_sound_speed_noalloc": (C.c_int, [C.c_void_p, C.c_double, C.c_size_t, dp, dp, dp, dp, dp]),
    "wq3d_queue_enable_sensitivity": (C.c_int, [C.c_void_p]),
    "wq3d_queue_sensitivities": (C.c_int, [C.c_void_p, dp, C.c_size_t, C.POINTER(C.c_size_t)]),
    "wq3d_queue_enable_adjoint": (C.c_int, [C.c_void_p, C.c_int, C.c_size_t, C.c_size_t]),
    "wq3d_set_queue_cache": (C.c_int, [C.c_size_t]),
    "wq3d_queue_adjoint_state": (C.c_int, [C.c_void_p, C.c_int, C.c_int64, C.c_int, dp, C.c_size_t]),
    "wq3d_queue_count_eigenverbs": (C.c_int, [C.c_void_p, C.c_int]),
    "wq3d_queue_eigenverb_counts": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    "wq3d_sum_eigenrays": (C.c_int, [C.c_void_p, dp, dp, C.c_size_t, dp, C.c_size_t, C.c_size_t, C.c_size_t,
                                     C.c_int, C.c_void_p, dp, dp]),
    "wq3d_queue_adjoint": (C.c_int, [C.c_void_p, C.c_void_p, dp, dp, C.c_size_t, dp, C.c_size_t, dp]),
    "wq3d_batch_run": (C.c_int, [C.POINTER(C.c_void_p), C.c_size_t, dp, C.POINTER(C.c_size_t), dp]),
    "wq3d_ocean_attenuation": (C.c_int, [C.c_void_p, C.c_double, C.c_size_t, dp, dp, C.c_size_t, dp, dp]),
    "wq3d_ocean_reflect_loss": (C.c_int, [C.c_void_p, C.c_int, C.c_size_t, dp, dp, dp, dp,
                                          C.c_size_t, dp, dp, dp]),
    "wq3d_queue_create": (C.c_int, [C.c_void_p, C.POINTER(wq3d_queue_desc), C.POINTER(C.c_void_p)]),
    "wq3d_queue_destroy": (C.c_int, [C.c_void_p]),
    "wq3d_queue_set_thresholds": (C.c_int, [C.c_void_p, C.POINTER(wq3d_thresholds)]),
    "wq3d_queue_set_callbacks": (C.c_int, [C.c_void_p, C.POINTER(wq3d_callbacks), C.c_void_p]),
    "wq3d_queue_step": (C.c_int, [C.c_void_p, C.c_size_t]),
    "wq3d_queue_run": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(C.c_size_t)]),
    "wq3d_queue_time": (C.c_int, [C.c_void_p, dp]),
    "wq3d_queue_source": (C.c_int, [C.c_void_p, dp]),
    "wq3d_queue_steps": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "wq3d_queue_get_front": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(wq3d_front_view)]),
    "wq3d_queue_take_eigenrays": (C.c_int, [C.c_void_p, C.POINTER(wq3d_eigenray), dp, dp,
                                            C.c_size_t, C.POINTER(C.c_size_t)]),
    "wq3d_queue_abort": (C.c_int, [C.c_void_p]),
    "wq3d_queue_timing": (C.c_int, [C.c_void_p, C.POINTER(wq3d_timing), C.c_int]),
    "wq3d_queue_set_timing": (C.c_int, [C.c_void_p, C.c_int]),
    "wq3d_queue_set_reflect_schedule": (C.c_int, [C.c_void_p, C.c_int]),
    "wq3d_queue_reflect_schedule": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "wq3d_biverbs": (C.c_int, [C.POINTER(wq3d_eigenverb), dp, C.c_size_t, C.POINTER(wq3d_eigenverb), dp,
                               C.c_size_t, dp, C.c_size_t, C.POINTER(wq3d_scattering_desc), C.c_double,
                               C.c_double, C.c_double, C.POINTER(wq3d_biverb), dp, C.c_size_t,
                               C.POINTER(C.c_size_t)]),
    "wq3d_last_error_string": (C.c_char_p, []),
    "wq3d_abi_version": (C.c_int, []),
    "wq3d_device_count": (C.c_int, [C.POINTER(C.c_int)]),
}


class EngineError(RuntimeError):
    """Raised when a wq3d_* call returns a negative status."""

    def __init__(self, code, msg):
        super().__init__("wq3d error %d: %s" % (code, msg))
        self.code = code


_lib = None


def bind(lib, signatures=SIGNATURES):
    for name, (res, args) in signatures.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def load_engine(path=None):
    """Loads libwq3d.so (built by build.py).  Raises if it is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError("the CUDA engine library %s is not built; run "
                           "underseamodelinglibrary_b200/build.py" % p)
    lib = bind(C.CDLL(p))
    if lib.wq3d_abi_version() != 1:
        raise RuntimeError("libwq3d ABI version mismatch")
    if path is None:
        _lib = lib
    return lib


def check(lib, rc, errfn="wq3d_last_error_string"):
    if rc != WQ3D_OK:
        msg = getattr(lib, errfn)()
        raise EngineError(rc, msg.decode() if msg else "")
    return rc


def as_dp(arr):
    return arr.ctypes.data_as(dp) if arr is not None else None
