"""Build recipe for the in-tree CUDA library ``libwq3d.so`` (sm_100a).

The library is compiled with nvcc straight from ``csrc/`` into this package
directory, so it travels with the source tree.  ``--fmad=false`` keeps every
FP64 add and multiply rounding separately, as the reference's C++ does.
"""
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libwq3d.so")
# the same library with WQ3D_CHECKED=1: every index a kernel reads from
# device data is tested before use (a failure is reported, never a trap)
CHECKED_LIB = os.path.join(HERE, "libwq3d_checked.so")
SOURCES = ["wq3d_api.cu", "wq3d_kernels.cu", "wq3d_noalloc.cu", "wq3d_biverbs.cu", "wq3d_sum.cu"]
# (object name, source, extra flags): wq3d_kernels.cu is compiled a second
# time for the ray-stepping kernels of oceans without gridded models
OBJECTS = [(f, f, []) for f in SOURCES] + [
    ("wq3d_kernels_analytic.cu", "wq3d_kernels.cu",
     ["-DWQ3D_WITH_GRID=0", "-DWQ3D_KERNEL_NS=analytic", "-DWQ3D_STEP_KERNELS_ONLY=1"]),
]
HEADERS = ["wq3d_engine.cuh", "wq3d_models.cuh", "wq3d_dual.cuh", "wq3d_adjoint.cuh"]

NVCC_FLAGS = [
    "-std=c++17", "-O3", "--fmad=false", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
]


def nvcc():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def stale():
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "wq3d.h"))
    for lib in (LIB, CHECKED_LIB):
        if not os.path.exists(lib):
            return True
        t = os.path.getmtime(lib)
        if any(os.path.getmtime(d) > t for d in deps):
            return True
    return False


def build(force=False, verbose=False):
    """Compiles each source to an object for both libraries in parallel,
    then links them."""
    if not force and not stale():
        return LIB
    with tempfile.TemporaryDirectory(prefix="wq3d_build_") as tmp:
        procs = []
        objs = {LIB: [], CHECKED_LIB: []}
        for lib, flags in ((LIB, []), (CHECKED_LIB, ["-DWQ3D_CHECKED=1"])):
            for name, f, extra in OBJECTS:
                obj = os.path.join(tmp, os.path.basename(lib) + "." + name + ".o")
                cmd = [nvcc()] + NVCC_FLAGS + extra + flags + ["-I", os.path.join(ROOT, "include"), "-c",
                                                               os.path.join(CSRC, f), "-o", obj]
                if verbose:
                    print(" ".join(cmd), file=sys.stderr)
                procs.append((cmd, subprocess.Popen(cmd)))
                objs[lib].append(obj)
        failed = [cmd for cmd, p in procs if p.wait() != 0]
        if failed:
            raise subprocess.CalledProcessError(1, failed[0])
        for lib, lib_objs in objs.items():
            link = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", lib + ".tmp"] + lib_objs
            if verbose:
                print(" ".join(link), file=sys.stderr)
            subprocess.check_call(link)
    for lib in objs:
        os.replace(lib + ".tmp", lib)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
