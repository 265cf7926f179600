"""The C++ drop-in header (underseamodelinglibrary_b200/cpp/usml_b200.hpp):
the reference's eigenray_basic test written against it, compiled with g++
and linked to libwq3d.so, must reproduce the reference's known answers."""
import os
import subprocess

import pytest

from underseamodelinglibrary_b200 import _abi

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpp_eigenray_basic(tmp_path, engine):
    lib_dir = os.path.dirname(_abi.LIB_PATH)
    exe = str(tmp_path / "eigenray_basic_cpp")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "cpp", "eigenray_basic_cpp.cpp"),
                           "-L", lib_dir, "-lwq3d", "-Wl,-rpath," + lib_dir, "-o", exe])
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.count("ray ") == 3
