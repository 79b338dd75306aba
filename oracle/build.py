"""Build recipe for the CPU test oracle (TEST INFRASTRUCTURE ONLY).

Compiles oracle/_oracle.cpp (pybind11 binding of rs_oracle.hpp, rs_adjoint.hpp and
rs_sdfbake_oracle.hpp) into an in-tree
extension module with the host compiler. No fast-math: the restatement keeps IEEE
float/double arithmetic. The reference itself is not built here: it needs GLM, which
is not present in this image.
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))


def ext_path() -> str:
    suffix = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    return os.path.join(HERE, "_oracle" + suffix)


def build(force: bool = False, verbose: bool = False) -> str:
    import pybind11

    out = ext_path()
    srcs = [os.path.join(HERE, "_oracle.cpp"), os.path.join(HERE, "rs_oracle.hpp"), os.path.join(HERE, "rs_opcount.hpp"),
            os.path.join(HERE, "rs_adjoint.hpp"), os.path.join(HERE, "rs_sdfbake_oracle.hpp")]
    if not force and os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(s) for s in srcs):
        return out
    cmd = [
        os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden",
        "-fno-fast-math", "-pthread",
        "-I", sysconfig.get_paths()["include"], "-I", pybind11.get_include(),
        srcs[0], "-o", out + ".tmp",
    ]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(out + ".tmp", out)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
