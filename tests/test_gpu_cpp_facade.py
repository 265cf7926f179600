"""The C++ drop-in header (underseamodelinglibrary_b200/cpp/usml_b200.hpp):
the reference's eigenray_basic test written against it, compiled with g++
and linked to libwq3d.so, must reproduce the reference's known answers."""
import os
import subprocess

import pytest

from underseamodelinglibrary_b200 import _abi

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build_cpp(tmp_path, name):
    """compiles tests/cpp/<name>.cpp against the header and libwq3d.so"""
    lib_dir = os.path.dirname(_abi.LIB_PATH)
    exe = str(tmp_path / name)
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "cpp", name + ".cpp"),
                           "-L", lib_dir, "-lwq3d", "-Wl,-rpath," + lib_dir, "-o", exe])
    return exe


def test_cpp_eigenray_basic(tmp_path, engine):
    out = subprocess.run([build_cpp(tmp_path, "eigenray_basic_cpp")], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.count("ray ") == 3


def test_cpp_eigenverb_accuracy(tmp_path, engine):
    """reverb_test.cc:216-310 through the C++ header: volume layer added
    after construction, eigenverb listener, analytic bottom footprints"""
    out = subprocess.run([build_cpp(tmp_path, "eigenverb_accuracy_cpp")], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "interfaces 4" in out.stdout


def test_cpp_run_batch(tmp_path, engine):
    """wave_queue::run_batch through the C++ header: two sources batched,
    each equal to its solo run bit for bit"""
    out = subprocess.run([build_cpp(tmp_path, "batch_cpp")], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "batch equals solo" in out.stdout


def test_cpp_reflection_listener(tmp_path, engine):
    """reflection_test.cc:168-280 through the C++ header: a
    reflection_listener hears every bounce, the same as the oracle's, and a
    removed listener hears no more; the queue's accessors read back"""
    import math
    import re

    from oracle_binding import OracleQueue
    from underseamodelinglibrary_b200 import scenarios as S

    out = subprocess.run([build_cpp(tmp_path, "reflect_cpp")], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "reflections ok" in out.stdout
    got = [(int(m[0]), float(m[1]), float(m[2]))
           for m in re.findall(r"type (\d+) time ([-\d.]+) grazing ([-\d.]+)", out.stdout)]
    sc = S.reflect_flat()
    o = S.build_queue(sc, OracleQueue, reflections=True)
    o.run(sc["time_max"])
    ref = o.take_reflections()
    assert len(got) == len(ref) >= 7
    for (t, time, graz), r in zip(got, ref):
        assert t == r.type
        assert abs(time - r.time) < 2e-9
        assert abs(graz - math.degrees(r.grazing)) < 2e-6


def test_cpp_biverb_generator(tmp_path, engine):
    """biverbs_test.cc:41-158 through the C++ header: biverb_generator over
    the 80 analytic footprints, 109 biverbs ordered by travel time, every
    footprint overlapping itself"""
    out = subprocess.run([build_cpp(tmp_path, "biverbs_cpp")], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "biverbs ok" in out.stdout and "biverbs 109" in out.stdout
