"""The C ABI: every symbol include/wq3d.h declares is exported by the
library, and the ctypes mirror matches the C struct layouts (checked
against a probe compiled from the header with gcc).  No GPU calls."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from underseamodelinglibrary_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "wq3d.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(wq3d_[a-z0-9_]+)\s*\(", text)
    return sorted(set(n for n in names if not n.endswith("_t")))


def test_library_exports_every_declared_symbol():
    lib = _abi.load_engine()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the ctypes signature table covers them all
    assert set(names) <= set(_abi.SIGNATURES), set(names) - set(_abi.SIGNATURES)


STRUCTS = ["wq3d_grid_desc", "wq3d_profile_desc", "wq3d_reflect_loss_desc", "wq3d_boundary_desc",
           "wq3d_ocean_desc", "wq3d_queue_desc", "wq3d_thresholds", "wq3d_eigenray",
           "wq3d_reflection", "wq3d_callbacks", "wq3d_front_view", "wq3d_eigenverb",
           "wq3d_scattering_desc", "wq3d_biverb", "wq3d_timing"]


def test_struct_layouts_match_header():
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "%s"' % HEADER, "int main(void){"]
    for s in STRUCTS:
        lines.append('printf("%s %%zu\\n", sizeof(%s));' % (s, s))
        for f, _ in getattr(_abi, s)._fields_:
            lines.append('printf("%s.%s %%zu\\n", offsetof(%s, %s));' % (s, f, s, f))
    lines.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "probe.c")
        exe = os.path.join(d, "probe")
        open(src, "w").write("\n".join(lines))
        subprocess.check_call(["gcc", "-std=c99", "-o", exe, src])
        out = subprocess.check_output([exe]).decode().split("\n")
    got = dict(l.split() for l in out if l.strip())
    for s in STRUCTS:
        cls = getattr(_abi, s)
        assert int(got[s]) == C.sizeof(cls), s
        for f, _ in cls._fields_:
            assert int(got["%s.%s" % (s, f)]) == getattr(cls, f).offset, (s, f)


def test_abi_version_and_error_string():
    lib = _abi.load_engine()
    assert lib.wq3d_abi_version() == 1
    assert isinstance(lib.wq3d_last_error_string(), bytes)


def test_invalid_arguments_are_reported_not_crashed():
    """null pointers return WQ3D_ERR_INVALID without touching a device"""
    lib = _abi.load_engine()
    assert lib.wq3d_ocean_create(None, None) == _abi.WQ3D_ERR_INVALID
    assert lib.wq3d_queue_create(None, None, None) == _abi.WQ3D_ERR_INVALID
    assert lib.wq3d_queue_step(None, 1) == _abi.WQ3D_ERR_INVALID
    assert b"null" in lib.wq3d_last_error_string()


def test_unsupported_ocean_kinds_are_rejected():
    lib = _abi.load_engine()
    d = _abi.wq3d_ocean_desc()
    d.earth_radius = 6371000.0
    d.profile.kind = 99
    h = C.c_void_p()
    assert lib.wq3d_ocean_create(C.byref(d), C.byref(h)) == _abi.WQ3D_ERR_UNSUPPORTED
