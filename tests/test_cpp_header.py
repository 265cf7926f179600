"""The C++ drop-in header compiles and links against libwq3d.so (no GPU
needed to build; the programs run in the GPU tests)."""
import os
import subprocess

import pytest

from underseamodelinglibrary_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("name", ["eigenray_basic_cpp", "eigenverb_accuracy_cpp", "batch_cpp", "reflect_cpp",
                                  "biverbs_cpp"])
def test_cpp_program_builds(tmp_path, name):
    if not os.path.exists(_abi.LIB_PATH):
        pytest.skip("libwq3d.so not built")
    lib_dir = os.path.dirname(_abi.LIB_PATH)
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "cpp", name + ".cpp"),
                           "-L", lib_dir, "-lwq3d", "-Wl,-rpath," + lib_dir, "-o", str(tmp_path / name)])
