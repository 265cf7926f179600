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


def _write_grid(fh, grid):
    import struct

    import numpy as np
    from underseamodelinglibrary_b200 import types as T
    fh.write(struct.pack("<i", len(grid.axes)))
    for a in grid.axes:
        kind = (_abi.AXIS_LINEAR if isinstance(a, T.seq_linear) else
                _abi.AXIS_LOG if isinstance(a, T.seq_log) else _abi.AXIS_DATA)
        x = np.ascontiguousarray(a.data, dtype=np.float64)
        inc = np.ascontiguousarray(a.increments, dtype=np.float64)
        fh.write(struct.pack("<ii", kind, x.size))
        fh.write(x.tobytes())
        fh.write(inc.tobytes())
    for v in grid._interp:
        fh.write(struct.pack("<i", int(v)))
    for v in grid._edge:
        fh.write(struct.pack("<i", 1 if v else 0))
    fh.write(np.ascontiguousarray(grid.data, dtype=np.float64).tobytes())


def test_cpp_std14_gridded(tmp_path, engine):
    """The reference's speed study (studies/cmp_speed/cmp_speed.cc:33-114)
    through the C++ header: STD14 profile_grid and boundary_grid built from
    data_grid objects, 20 targets on the 100 km ring, 80 s; every eigenray
    equals the oracle's (per target, in order: travel time within 1 us, TL
    within 0.1 dB, angles within 0.01 deg, counts equal), and curr() reads
    the front back."""
    import struct

    import numpy as np
    from oracle_binding import OracleQueue
    from underseamodelinglibrary_b200 import scenarios as S
    sc = S.std14(num_targets=20, time_max=80.0)
    ocean = sc["ocean"]
    path = str(tmp_path / "std14.bin")
    with open(path, "wb") as fh:
        fh.write(struct.pack("<d", sc["earth_radius"]))
        _write_grid(fh, ocean._profile.grid)
        _write_grid(fh, ocean.bottom().grid)
        p = sc["pos"]
        fh.write(struct.pack("<dddd", p.latitude(), p.longitude(), p.altitude(), sc["time_max"]))
        tg = sc["targets"]
        fh.write(struct.pack("<i", tg.size1() * tg.size2()))
        for i in range(tg.size1()):
            fh.write(struct.pack("<ddd", tg.latitude(i, 0), tg.longitude(i, 0), tg.altitude(i, 0)))
    out = subprocess.run([build_cpp(tmp_path, "std14_cpp"), path], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    got = {}
    for line in out.stdout.splitlines():
        f = line.split()
        if f[0] == "ray":
            got.setdefault(int(f[1]), []).append([float(x) for x in f[2:8]] + [int(x) for x in f[8:11]])
    o = S.build_queue(sc, OracleQueue)
    o.run(sc["time_max"])
    want = {}
    for r in o.take_eigenrays():
        want.setdefault(r.t1, []).append([r.travel_time, r.intensity[0], r.source_de, r.source_az,
                                          r.target_de, r.target_az, r.surface, r.bottom, r.caustic])
    assert sum(len(v) for v in want.values()) > 200
    assert set(got) == set(want)
    for t in want:
        assert len(got[t]) == len(want[t]), t
        for a, b in zip(got[t], want[t]):
            assert abs(a[0] - b[0]) < 1e-6 and abs(a[1] - b[1]) < 0.1, (t, a, b)
            assert max(abs(a[k] - b[k]) for k in (2, 3, 4, 5)) < 0.01, (t, a, b)
            assert a[6:] == b[6:], (t, a, b)
    fronts = [line for line in out.stdout.splitlines() if line.startswith("front")]
    assert fronts and all(float(line.split()[2]) > 6.3e6 for line in fronts)
