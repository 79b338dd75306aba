"""The C-ABI library: it loads, exports every entry point include/ropesim_b200.h declares, and
reports errors through status codes (no compute calls here: this runs without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ropesim_b200.h")
LIB = os.path.join(ROOT, "cosserat-rod-solver-cuda_b200", "ropesim", "libropesim_b200.so")


def declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"RS_API\s+[\w\s\*]+?\b(rs_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared()
    assert "rs_batch_create" in names and "rs_batch_step_program" in names and "rs_last_error_string" in names
    assert len(names) >= 40


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB), "build the engine first (cosserat-rod-solver-cuda_b200/build.py)"
    lib = ctypes.CDLL(LIB)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"


def test_status_codes_without_device_work():
    lib = ctypes.CDLL(LIB)
    lib.rs_last_error_string.restype = ctypes.c_char_p
    lib.rs_version.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.rs_version()
    # a null handle is an invalid argument (RS_EINVAL = 1), with a message
    assert lib.rs_batch_set_num_itr(None, 4) == 1
    assert b"null" in lib.rs_last_error_string()
    # argument validation happens before any device work
    out = ctypes.c_void_p()
    verts = (ctypes.c_int * 1)(2)
    pos = (ctypes.c_float * 6)(0, 0, 0, 0, 0, 1)
    rc = lib.rs_batch_create(ctypes.byref(out), 1, verts, pos, None, ctypes.c_float(0.1), ctypes.c_float(500.0),
                             ctypes.c_float(1e-6), ctypes.c_float(1e-3), 8, 0, 0, ctypes.c_float(1e-4), ctypes.c_float(8e-4))
    assert rc == 1 and b"3 vertices" in lib.rs_last_error_string()


def test_python_package_imports_and_fails_loudly_without_gpu():
    import numpy as np

    import ropesim

    try:
        import torch

        cuda = torch.cuda.is_available()
    except ImportError:
        cuda = False
    assert hasattr(ropesim, "RopeBatch") and hasattr(ropesim, "RopeSim")
    with pytest.raises(ValueError):
        ropesim.RopeSim(num_verts=2)
    if not cuda:
        with pytest.raises(RuntimeError):
            ropesim.RopeSim(num_verts=8, dir=np.array([1, 0, 0], np.float32))


def test_bake_entry_point_validates_before_device_work():
    """rs_sdf_bake refuses bad meshes and lattices with RS_EINVAL before touching the device."""
    import numpy as np

    lib = ctypes.CDLL(LIB)
    lib.rs_last_error_string.restype = ctypes.c_char_p
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32)
    f = np.array([[0, 1, 2], [0, 1, 7]], np.int32)  # index 7 is out of range
    org = np.zeros(3, np.float32)
    out = np.zeros(8, np.float32)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    F = ctypes.c_float
    rc = lib.rs_sdf_bake(P(v), 4, P(f), 2, P(org), ctypes.c_double(0.5), 2, 2, 2, F(0.0), F(0.0), P(out), 0, None, None)
    assert rc == 1 and b"out of range" in lib.rs_last_error_string()
    f[1, 2] = 3
    rc = lib.rs_sdf_bake(P(v), 4, P(f), 2, P(org), ctypes.c_double(-1.0), 2, 2, 2, F(0.0), F(0.0), P(out), 0, None, None)
    assert rc == 1 and b"spacing" in lib.rs_last_error_string()
    rc = lib.rs_sdf_bake(P(v), 4, P(f), 2, P(org), ctypes.c_double(0.5), 2, 2, 8000, F(0.0), F(0.0), P(out), 0, None, None)
    assert rc == 1 and b"along z" in lib.rs_last_error_string()
    rc = lib.rs_sdf_bake(P(v), 4, P(f), 2, P(org), ctypes.c_double(0.5), 2, 2, 2, F(-1.0), F(0.0), P(out), 0, None, None)
    assert rc == 1 and b"thickness" in lib.rs_last_error_string()
