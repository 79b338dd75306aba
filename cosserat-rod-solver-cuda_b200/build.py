"""Build the engine in-tree.

1. libropesim_b200.so: the sm_100a kernels, the C++ driver and the extern "C" boundary
   (include/ropesim_b200.h), compiled by nvcc for `-gencode arch=compute_100a,code=sm_100a`
   only, IEEE division / square root (no fast math; the frame step's rotor norms alone use
   rsqrtf), no compiler FMA contraction (the fused multiply-adds are written out in the
   sources), static CUDA runtime.
2. ropesim/_ropesim*.so: the pybind11 module (RopeSim, RopeBatch, CudaView) linked against (1)
   with an $ORIGIN rpath, so the package directory is self-contained.
3. The checked build: the same sources with -DROPESIM_CHECKED (every kernel index the topology
   or the data could push out of range is tested; the first failure is recorded, nothing traps)
   as libropesim_b200_checked.so and ropesim/_ropesim_checked*.so, for the bounds tests.

Usage: python cosserat-rod-solver-cuda_b200/build.py [--force] [-v]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
PKG = os.path.join(HERE, "ropesim")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["rs_frame.cu", "rs_plain.cu", "rs_adjoint.cu", "rs_adjoint_plain.cu", "rs_ropegrid.cu", "rs_sdfbake.cu"]
CPP_SOURCES = ["rs_batch.cpp", "rs_capi.cpp"]
HEADERS = ["rs_types.h", "rs_device.cuh", "rs_substep.cuh", "rs_adjoint.cuh", "rs_kernels.h", "rs_batch.h"]


def lib_path(checked: bool = False) -> str:
    return os.path.join(PKG, "libropesim_b200_checked.so" if checked else "libropesim_b200.so")


def ext_path(checked: bool = False) -> str:
    return os.path.join(PKG, ("_ropesim_checked" if checked else "_ropesim") + (sysconfig.get_config_var("EXT_SUFFIX") or ".so"))


def _nvcc() -> str:
    cand = [os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"]
    for c in cand:
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found: the engine needs the CUDA toolkit to build")


def _stale(out: str, deps) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _build_one(checked: bool, force: bool, verbose: bool) -> str:
    nvcc = _nvcc()
    objdir = os.path.join(HERE, "_build_checked" if checked else "_build")
    os.makedirs(objdir, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "ropesim_b200.h")]
    common = ["-std=c++17", "-O3", "-I", CSRC, "-I", INCLUDE, "-Xcompiler", "-fPIC,-fvisibility=hidden,-ffp-contract=off"]
    if checked:
        common.append("-DROPESIM_CHECKED")
    objs = []
    for src in CU_SOURCES + CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(objdir, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            # -fmad=false: the sources spell out every fused multiply-add (fmaf), so each kernel
            # instantiation rounds identically whatever its block size or surface variant
            extra = ARCH + ["-lineinfo", "-fmad=false", "-Xptxas", "-v"] if src.endswith(".cu") else ARCH
            cmd = [nvcc] + common + extra + ["-c", s, "-o", o]
            if src.endswith(".cu") and not verbose:
                cmd.remove("-Xptxas"); cmd.remove("-v")
            _run(cmd, verbose)
    lib = lib_path(checked)
    if force or _stale(lib, objs):
        _run([nvcc] + ARCH + ["-shared", "-cudart", "static", "-o", lib + ".tmp"] + objs, verbose)
        os.replace(lib + ".tmp", lib)

    import pybind11

    ext = ext_path(checked)
    src = os.path.join(CSRC, "rs_pybind.cpp")
    if force or _stale(ext, [src, lib, os.path.join(INCLUDE, "ropesim_b200.h")]):
        cxx = os.environ.get("CXX", "g++")
        name = "ropesim_b200_checked" if checked else "ropesim_b200"
        cmd = [cxx, "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden",
               "-I", sysconfig.get_paths()["include"], "-I", pybind11.get_include(), "-I", INCLUDE,
               src, "-o", ext + ".tmp", "-L", PKG, "-l" + name, "-Wl,-rpath,$ORIGIN"]
        if checked:
            cmd.insert(1, "-DRS_MODULE_NAME=_ropesim_checked")
        _run(cmd, verbose)
        os.replace(ext + ".tmp", ext)
    return ext


def build(force: bool = False, verbose: bool = False, checked: bool = True) -> str:
    """The engine (libropesim_b200.so + ropesim._ropesim) and, unless checked=False, its checked
    build (libropesim_b200_checked.so + ropesim._ropesim_checked)."""
    ext = _build_one(False, force, verbose)
    if checked:
        _build_one(True, force, verbose)
    return ext


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
