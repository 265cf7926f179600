"""Test-only ctypes binding of the CPU oracle (oracle/liboracle_wq3d.so).

``OracleQueue`` takes the same reference-style arguments as
``underseamodelinglibrary_b200.wave_queue`` and runs the CPU restatement of
the reference path, so a test can build one scenario and compare the two.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from underseamodelinglibrary_b200 import _abi
from underseamodelinglibrary_b200.waveq3d import (eigenray_model, make_queue_desc,
                                                  wave_front_view)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "liboracle_wq3d.so")

dp = _abi.dp
SIGS = {
    "oracle_queue_create": (C.c_int, [C.POINTER(_abi.wq3d_ocean_desc), C.POINTER(_abi.wq3d_queue_desc),
                                      C.POINTER(C.c_void_p)]),
    "oracle_queue_destroy": (C.c_int, [C.c_void_p]),
    "oracle_queue_set_thresholds": (C.c_int, [C.c_void_p, C.POINTER(_abi.wq3d_thresholds)]),
    "oracle_queue_set_reflections": (C.c_int, [C.c_void_p, C.c_int]),
    "oracle_queue_set_eigenverbs": (C.c_int, [C.c_void_p, C.c_int]),
    "oracle_queue_take_eigenverbs": (C.c_int, [C.c_void_p, C.POINTER(_abi.wq3d_eigenverb), dp, C.c_size_t,
                                               C.POINTER(C.c_size_t)]),
    "oracle_queue_step": (C.c_int, [C.c_void_p, C.c_size_t]),
    "oracle_queue_run": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(C.c_size_t)]),
    "oracle_queue_time": (C.c_int, [C.c_void_p, dp]),
    "oracle_queue_source": (C.c_int, [C.c_void_p, dp]),
    "oracle_queue_get_front": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(_abi.wq3d_front_view)]),
    "oracle_queue_take_eigenrays": (C.c_int, [C.c_void_p, C.POINTER(_abi.wq3d_eigenray), dp, dp,
                                              C.c_size_t, C.POINTER(C.c_size_t)]),
    "oracle_queue_take_reflections": (C.c_int, [C.c_void_p, C.POINTER(_abi.wq3d_reflection),
                                                C.c_size_t, C.POINTER(C.c_size_t)]),
    "oracle_sound_speed": (C.c_int, [C.POINTER(_abi.wq3d_ocean_desc), C.c_double, C.c_size_t,
                                     dp, dp, dp, dp, dp]),
    "oracle_height": (C.c_int, [C.POINTER(_abi.wq3d_ocean_desc), C.c_int, C.c_size_t, dp, dp, dp, dp, dp]),
    "oracle_reflect_loss": (C.c_int, [C.POINTER(_abi.wq3d_ocean_desc), C.c_int, C.c_size_t, dp,
                                      C.c_size_t, dp, dp, dp]),
    "oracle_attenuation": (C.c_int, [C.POINTER(_abi.wq3d_ocean_desc), C.c_double, C.c_size_t, dp, dp,
                                     C.c_size_t, dp, dp]),
    "oracle_biverbs": _abi.SIGNATURES["wq3d_biverbs"],
    "oracle_last_error_string": (C.c_char_p, []),
}

ORACLE_OPCOUNT_LIB = os.path.join(ORACLE_DIR, "liboracle_opcount.so")
_libs = {}


def load_oracle(opcount=False):
    """the oracle library, or with opcount its operation-counting build
    (oracle/opcount.cpp), which adds oracle_opcount_read / _reset"""
    path = ORACLE_OPCOUNT_LIB if opcount else ORACLE_LIB
    if path not in _libs:
        if opcount or not os.path.exists(path):
            subprocess.check_call(["make", "-s", "-C", ORACLE_DIR] + (["opcount"] if opcount else []))
        lib = _abi.bind(C.CDLL(path), SIGS)
        if opcount:
            lib.oracle_opcount_read.restype = C.c_int
            lib.oracle_opcount_read.argtypes = [C.POINTER(C.c_uint64)]
            lib.oracle_opcount_reset.restype = C.c_int
            lib.oracle_opcount_reset.argtypes = []
        _libs[path] = lib
    return _libs[path]


def _check(rc):
    if rc != 0:
        raise _abi.EngineError(rc, load_oracle().oracle_last_error_string().decode())


class OracleQueue:
    def __init__(self, ocean, freq, pos, de, az, time_step, target_pos=None,
                 type=_abi.HYBRID_GAUSSIAN, reflections=False, eigenverbs=False, opcount=False):
        lib = load_oracle(opcount)
        self._lib = lib
        self._freq, self._de, self._az = freq, de, az
        d, self._keep = make_queue_desc(freq, pos, de, az, time_step, target_pos, type)
        self._od = ocean.descriptor()
        h = C.c_void_p()
        _check(lib.oracle_queue_create(C.byref(self._od), C.byref(d), C.byref(h)))
        self._q = h
        if reflections:
            lib.oracle_queue_set_reflections(h, 1)
        if eigenverbs:
            lib.oracle_queue_set_eigenverbs(h, 1)

    def __del__(self):
        if getattr(self, "_q", None) is not None:
            self._lib.oracle_queue_destroy(self._q)
            self._q = None

    def set_thresholds(self, intensity=300.0, max_bottom=999, max_surface=999, max_caustic=999,
                       max_upper=999, max_lower=999, eigenverb=300.0):
        self._thresh = dict(intensity=intensity, max_bottom=max_bottom, max_surface=max_surface,
                            max_caustic=max_caustic, max_upper=max_upper, max_lower=max_lower,
                            eigenverb=eigenverb)
        t = _abi.wq3d_thresholds(intensity, eigenverb, max_bottom, max_surface, max_caustic,
                                 max_upper, max_lower)
        _check(self._lib.oracle_queue_set_thresholds(self._q, C.byref(t)))

    def _set_one(self, name, value):
        kw = dict(getattr(self, "_thresh", {}))
        kw[name] = value
        self.set_thresholds(**kw)

    def max_bottom(self, v):
        self._set_one("max_bottom", int(v))

    def max_surface(self, v):
        self._set_one("max_surface", int(v))

    def max_caustic(self, v):
        self._set_one("max_caustic", int(v))

    def step(self, n=1):
        _check(self._lib.oracle_queue_step(self._q, int(n)))

    def run(self, time_max):
        n = C.c_size_t()
        _check(self._lib.oracle_queue_run(self._q, float(time_max), C.byref(n)))
        return n.value

    def time(self):
        t = C.c_double()
        self._lib.oracle_queue_time(self._q, C.byref(t))
        return t.value

    def source_pos(self):
        s = (C.c_double * 3)()
        self._lib.oracle_queue_source(self._q, s)
        return tuple(s)

    def _front(self, which):
        return wave_front_view(self._lib.oracle_queue_get_front, self._q, which, self._de.size(),
                               self._az.size(), self._freq.size(), check=_check)

    def past(self):
        return self._front(_abi.FRONT_PAST)

    def prev(self):
        return self._front(_abi.FRONT_PREV)

    def curr(self):
        return self._front(_abi.FRONT_CURR)

    def next(self):
        return self._front(_abi.FRONT_NEXT)

    def take_eigenrays(self):
        n = C.c_size_t()
        _check(self._lib.oracle_queue_take_eigenrays(self._q, None, None, None, 0, C.byref(n)))
        cnt = n.value
        nf = self._freq.size()
        recs = (_abi.wq3d_eigenray * max(cnt, 1))()
        inten = np.empty(max(cnt, 1) * nf)
        phase = np.empty(max(cnt, 1) * nf)
        _check(self._lib.oracle_queue_take_eigenrays(self._q, recs, _abi.as_dp(inten), _abi.as_dp(phase),
                                                     cnt, C.byref(n)))
        return [eigenray_model.from_record(recs[i], inten[i * nf:(i + 1) * nf],
                                           phase[i * nf:(i + 1) * nf], self._freq) for i in range(cnt)]

    def eigenverb_threshold(self, value):
        self._set_one("eigenverb", abs(float(value)))

    def take_eigenverbs(self):
        """eigenverbs in the order a listener would have received them"""
        from underseamodelinglibrary_b200.eigenverbs import eigenverb_model
        n = C.c_size_t()
        _check(self._lib.oracle_queue_take_eigenverbs(self._q, None, None, 0, C.byref(n)))
        cnt = n.value
        nf = self._freq.size()
        recs = (_abi.wq3d_eigenverb * max(cnt, 1))()
        power = np.empty(max(cnt, 1) * nf)
        _check(self._lib.oracle_queue_take_eigenverbs(self._q, recs, _abi.as_dp(power), cnt, C.byref(n)))
        return [eigenverb_model.from_record(recs[i], power[i * nf:(i + 1) * nf], self._freq)
                for i in range(cnt)]

    def take_reflections(self):
        n = C.c_size_t()
        _check(self._lib.oracle_queue_take_reflections(self._q, None, 0, C.byref(n)))
        recs = (_abi.wq3d_reflection * max(n.value, 1))()
        _check(self._lib.oracle_queue_take_reflections(self._q, recs, n.value, C.byref(n)))
        return [recs[i] for i in range(n.value)]
