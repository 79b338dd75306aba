"""Shared helpers for the test suite.

Backends: "oracle" is the FP64 CPU restatement (oracle/, test infrastructure) and runs
everywhere; "cuda" is the product (ropesim package, persistent sm_100a kernel) and is marked
`gpu`. Physics tests are parametrized over both, so the reference's known-answer checks
(tests/test_statics.py, test_dynamics.py, test_contact.py, ... of the reference) pin the
oracle on the CPU and check the product on the GPU.

Conventions follow the reference suite (tests/conftest.py of DeformX/Cosserat-Rod-Solver-CUDA):
density = rho [kg/m], k_stretch = EA [N], k_bend = EI [N*m^2]; make_rope() zeroes drag and
damping unless overridden; H is the control frame.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "cosserat-rod-solver-cuda_b200")
ORACLE = os.path.join(ROOT, "oracle")
for p in (PKG, ORACLE, os.path.dirname(os.path.abspath(__file__))):
    if p not in sys.path:
        sys.path.insert(0, p)

G = 9.8
H = 1.0 / 60.0


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the product kernels")
    config.addinivalue_line("markers", "slow: long-running")


BACKENDS = ["oracle", pytest.param("cuda", marks=pytest.mark.gpu)]


def rope_sim_class(backend):
    if backend == "oracle":
        import ropesim_oracle

        return ropesim_oracle.RopeSim
    import ropesim

    return ropesim.RopeSim


def rope_batch_class(backend):
    if backend == "oracle":
        import ropesim_oracle

        return ropesim_oracle.RopeBatch
    import ropesim

    return ropesim.RopeBatch


def make_rope(backend="oracle", n=33, seg=0.02, direction=(0.0, -1.0, 0.0), density=0.1, EA=500.0, EI=1e-6,
              max_h=1.0 / 3000.0, drag=0.0, damping=0.0, **kw):
    cls = rope_sim_class(backend)
    r = cls(num_verts=n, seg_len=seg, dir=np.asarray(direction, np.float32), density=density, k_stretch=EA,
            k_bend=EI, max_h=max_h, **kw)
    r.set_gravity(np.array([0.0, -G, 0.0], np.float32))
    r.drag = drag
    r.damping = damping
    return r


def rope_length(r):
    return float(np.sum(np.asarray(r.rest_lengths(), np.float64)))


def masses(r):
    inv = np.asarray(r.inv_masses(), dtype=np.float64)
    m = np.zeros_like(inv)
    nz = inv > 0
    m[nz] = 1.0 / inv[nz]
    return m


def segment_strains(r):
    p = np.asarray(r.positions(), dtype=np.float64)
    lens = np.linalg.norm(np.diff(p, axis=0), axis=1)
    rest = np.asarray(r.rest_lengths(), dtype=np.float64)
    return (lens - rest) / rest


def settle(r, t=3.0, drag=3.0):
    old = r.drag
    r.drag = drag
    for _ in range(int(round(t / H))):
        r.advance(H)
    r.drag = old


def drive(r, traj, t_end, rate=60.0):
    h = 1.0 / rate
    tips = []
    for k in range(int(round(t_end * rate))):
        t = k * h
        p0 = np.asarray(traj(t), np.float64)
        p1 = np.asarray(traj(t + h), np.float64)
        r.set_root(p0.astype(np.float32), ((p1 - p0) * rate).astype(np.float32))
        r.advance(h)
        tips.append(np.asarray(r.positions(), np.float64)[-1])
    return np.array(tips)


def energy_scalar(r, EA, y_ref=0.0):
    p = np.asarray(r.positions(), dtype=np.float64)
    v = np.asarray(r.velocities(), dtype=np.float64)
    m = masses(r)
    ke = 0.5 * np.sum(m * np.sum(v * v, axis=1))
    pe = G * np.sum(m * (p[:, 1] - y_ref))
    rest = np.asarray(r.rest_lengths(), dtype=np.float64)
    eps = segment_strains(r)
    return ke + pe + 0.5 * EA * np.sum(eps * eps * rest)


def quat_rotate(q, v):
    q = np.asarray(q, dtype=np.float64)
    v = np.asarray(v, dtype=np.float64)
    u, w = q[:3], q[3]
    return v + 2.0 * np.cross(u, np.cross(u, v) + w * v)


def axis_angle_quat(axis, angle):
    axis = np.asarray(axis, dtype=np.float64)
    axis = axis / np.linalg.norm(axis)
    s = np.sin(angle / 2.0)
    return np.array([axis[0] * s, axis[1] * s, axis[2] * s, np.cos(angle / 2.0)])


def has_cuda():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
