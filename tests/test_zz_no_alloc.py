"""The allocation-free frame step (rs_batch_step_program_static_scratch).

Some callers cannot allocate device memory once they are running: engines that reserve the
GPU's memory for their own allocator, control loops whose memory is fixed at start-up, and
runtimes that forbid allocation after initialisation. For them the library keeps the rope-rope
candidate lists in a static device array instead of a buffer of the handle. This test drives two
identical batches in rope-rope contact through the C-ABI, one with the regular entry point
(rs_batch_step_program) and one with the allocation-free one, for two frames in a row. Both run
the same kernel on the same inputs and bins, so the positions must agree bit for bit (well within
the 1e-5 m parity tolerance of the other GPU tests). The device's free memory must not change
across the second allocation-free call (the first call on a device may load the kernel module),
and the call reports its frame time when timing is on. A batch larger than the static array is
refused with a clear error.
"""
import ctypes
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "cosserat-rod-solver-cuda_b200", "ropesim", "libropesim_b200.so")
F = ctypes.c_float
TOL = 1e-5


def lib():
    L = ctypes.CDLL(LIB)
    L.rs_last_error_string.restype = ctypes.c_char_p
    return L


def ok(L, rc):
    assert rc == 0, L.rs_last_error_string().decode()


def make(L, ropes=4, verts=24, group=None):
    """Ropes hanging 1.5 cm apart in one rope-rope contact group (or groups of `group` ropes)."""
    pos = np.zeros((ropes, verts, 3), np.float32)
    for r in range(ropes):
        pos[r, :, 0] = 0.015 * r
        pos[r, :, 2] = 1.0 - 0.02 * np.arange(verts)
        pos[r, 1:, 1] = 1e-4 * (r + 1) * np.sin(np.arange(1, verts))
    pos = np.ascontiguousarray(pos.reshape(-1, 3))
    h = ctypes.c_void_p()
    nv = (ctypes.c_int * ropes)(*([verts] * ropes))
    ok(L, L.rs_batch_create(ctypes.byref(h), ropes, nv, pos.ctypes.data_as(ctypes.c_void_p), None, F(0.117),
                            F(11473.0), F(4.48e-3), F(1 / 6000), 8, 0, 0, F(2e-4), F(1.6e-3)))
    ok(L, L.rs_batch_set_autotune(h, 0))
    ok(L, L.rs_batch_set_gravity(h, (F * 3)(0.0, 0.0, -9.81)))
    ok(L, L.rs_batch_set_param(h, 3, F(0.0)))   # damping
    ok(L, L.rs_batch_set_param(h, 0, F(0.5)))   # drag
    R = 0.00635
    ok(L, L.rs_batch_set_rope_contact(h, 1, F(0.9 * R), F(0.2 * R), F(0.025), F(0.4), F(1e7), F(1.2), group or ropes))
    return h, pos.reshape(ropes, verts, 3)


def download(L, h, n):
    p = np.empty((n, 3), np.float32)
    ok(L, L.rs_batch_download(h, p.ctypes.data_as(ctypes.c_void_p), None, None))
    return p.astype(np.float64)


def test_static_scratch_step_matches_regular_step():
    import torch

    assert torch.cuda.is_available()
    L = lib()
    a, pos = make(L)
    b, _ = make(L)
    ok(L, L.rs_batch_set_timing(b, 1))
    ropes, verts = pos.shape[:2]
    roots = pos[:, 0].copy()
    sway = (np.arange(ropes) % 2 - 0.5)[:, None] * np.array([0.0, 0.02, 0.0], np.float32)
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())
    for f in range(2):  # two calls in a row: the second reuses the static array
        p0 = torch.tensor(roots + sway * np.sin(f / 3), device="cuda", dtype=torch.float32)
        p1 = torch.tensor(roots + sway * np.sin((f + 1) / 3), device="cuda", dtype=torch.float32)
        v0 = ((p1 - p0) * 60).contiguous()
        torch.cuda.synchronize()
        ok(L, L.rs_batch_step_program(a, ptr(p0), ptr(v0), ptr(p1), None, None, F(1 / 60), 50, 0))
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        ok(L, L.rs_batch_step_program_static_scratch(b, ptr(p0), ptr(v0), ptr(p1), None, None, F(1 / 60), 50))
        free1 = torch.cuda.mem_get_info()[0]
        ms = ctypes.c_double(0.0)
        ok(L, L.rs_batch_last_frame_ms(b, ctypes.byref(ms)))
        xa, xb = download(L, a, ropes * verts), download(L, b, ropes * verts)
        d = np.max(np.linalg.norm(xa - xb, axis=1))
        moved = np.max(np.linalg.norm(xa - pos.reshape(-1, 3), axis=1))
        print(f"\n  frame {f}: regular vs allocation-free step {d:.2e} m (ropes moved up to {moved:.3f} m), "
              f"free device memory {free0} -> {free1} B, frame kernel {ms.value:.3f} ms")
        assert np.isfinite(xb).all() and moved > 1e-4
        assert d <= TOL and np.array_equal(xa.astype(np.float32).view(np.uint32), xb.astype(np.float32).view(np.uint32))
        assert ms.value > 0.0
        if f == 1:
            assert free1 == free0, "the allocation-free step changed the device's free memory"
    for h in (a, b):
        ok(L, L.rs_batch_destroy(h))


def test_static_scratch_rejects_batches_beyond_capacity():
    L = lib()
    big, _ = make(L, ropes=205, verts=40, group=5)  # 8200 vertices > 8192
    z = np.zeros((205, 3), np.float32)
    import torch

    t = torch.as_tensor(z, device="cuda")
    p = ctypes.c_void_p(t.data_ptr())
    rc = L.rs_batch_step_program_static_scratch(big, p, p, p, None, None, F(1 / 60), 2)
    assert rc == 1
    assert b"8192" in L.rs_last_error_string()
    ok(L, L.rs_batch_destroy(big))
