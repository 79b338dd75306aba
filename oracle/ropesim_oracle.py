"""TEST INFRASTRUCTURE ONLY: the CPU oracle behind the ropesim API shape.

`RopeSim` and `RopeBatch` here take the same constructor arguments and methods as the
product's (and the reference's) classes, but run the CPU restatement in rs_oracle.hpp on
host numpy arrays: `precision="f64"` (the parity target) or `"f32"` (the float
instantiation, used to measure the fp32-vs-fp64 spread and as the timed CPU baseline).

Reference API followed: csrc/bindings.cpp:185-582 (RopeSim) and :735-1210 (RopeBatch) of
DeformX/Cosserat-Rod-Solver-CUDA. Only tests/, __graft_entry__.smoke() and bench.py's CPU
legs import this module.
"""
from __future__ import annotations

import importlib
import os
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))


def _ext():
    if _HERE not in sys.path:
        sys.path.insert(0, _HERE)
    try:
        return importlib.import_module("_oracle")
    except ImportError:
        from build import build  # type: ignore
        build()
        return importlib.import_module("_oracle")


def _sim_class(precision):
    """f64: the parity target; f32: the float instantiation; ops: double precision with every
    floating-point operation tallied (_oracle.op_tally), for algorithmic FLOP counts."""
    m = _ext()
    return {"f64": m.Sim64, "f32": m.Sim32, "ops": m.SimOps}[precision]


def _f32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def _unit_rows(planes):
    planes = np.asarray(planes, np.float32).reshape(-1, 4)
    out = np.zeros_like(planes)
    for i, row in enumerate(planes):
        n = row[:3]
        l = np.float32(np.sqrt(np.float32(n[0] * n[0] + n[1] * n[1] + n[2] * n[2])))
        if not (l > 0) or not np.isfinite(l) or not np.isfinite(row[3]):
            raise ValueError("plane rows need a finite, nonzero normal and a finite offset")
        out[i, :3] = n / l
        out[i, 3] = row[3] / l
    return out


class _Common:
    """Knobs shared by both classes (bindings.cpp:535-579)."""

    def __init__(self, sim, max_h):
        self._s = sim
        self._max_h = np.float32(max_h)

    drag = property(lambda self: self._s.drag, lambda self, v: setattr(self._s, "drag", float(v)))
    drag_quad = property(lambda self: self._s.drag_quad, lambda self, v: setattr(self._s, "drag_quad", float(v)))
    drag_quad_t = property(lambda self: self._s.drag_quad_t, lambda self, v: setattr(self._s, "drag_quad_t", float(v)))
    damping = property(lambda self: self._s.damping, lambda self, v: setattr(self._s, "damping", float(v)))
    accel_ratio = property(lambda self: self._s.accel_ratio, lambda self, v: setattr(self._s, "accel_ratio", float(v)))
    num_itr = property(lambda self: self._s.num_itr, lambda self, v: setattr(self._s, "num_itr", int(v)))
    time = property(lambda self: self._s.time)
    last_error = property(lambda self: self._s.last_error)
    last_warning = property(lambda self: self._s.last_warning)

    @property
    def max_h(self):
        return self._s.max_h

    @max_h.setter
    def max_h(self, v):
        if not v > 0:
            raise ValueError("max_h must be > 0")
        self._s.max_h = float(v)

    @property
    def gravity(self):
        return np.asarray(self._s.gravity, np.float32)

    def set_gravity(self, g):
        self._s.gravity = [float(x) for x in np.asarray(g, np.float32).reshape(3)]

    def set_contact(self, radius, mu_s=0.5, mu_k=None, v_slip=1e-3, kappa=2.0):
        mu_k = mu_s if mu_k is None else mu_k
        if not (radius > 0 and kappa > 0 and mu_s >= 0 and mu_k >= 0 and v_slip > 0):
            raise ValueError("surface contact needs radius > 0, kappa > 0, mu_s >= 0, mu_k >= 0, v_slip > 0")
        self._s.set_contact(radius, mu_s, mu_k, v_slip, kappa)
        self._material = (radius, mu_s, mu_k)

    def set_planes(self, planes, radius=0.0, mu_s=0.5, mu_k=None, v_slip=1e-3, kappa=2.0):
        planes = np.asarray(planes, np.float32)
        if planes.ndim != 2 or planes.shape[1] != 4 or planes.shape[0] > 8:
            raise ValueError("planes must be [P<=8, 4] rows")
        rows = _unit_rows(planes)
        if len(rows):
            self.set_contact(radius, mu_s, mu_k, v_slip, kappa)
        self._s.set_planes(rows)

    def enable_contact_forces(self, on=True):
        self._s.enable_forces(bool(on))
        self._forces = bool(on)

    def _add_mesh(self, values, origin, spacing, pos, quat, mu_s, mu_k, rows):
        rad, ms0, mk0 = getattr(self, "_material", (0.0, 0.0, 0.0))
        if not rad > 0:
            raise ValueError("set the contact material first")
        ms = ms0 if mu_s is None else float(mu_s)
        mk = (mk0 if mu_s is None else ms) if mu_k is None else float(mu_k)
        return self._s.add_mesh(_f32(values), _f32(origin).reshape(3), float(spacing), ms, mk,
                                _f32(pos).reshape(-1), _f32(quat).reshape(-1), rows)

    def set_mesh_friction(self, index, mu_s, mu_k=None):
        self._s.set_mesh_friction(int(index), float(mu_s), float(mu_s if mu_k is None else mu_k))

    def clear_meshes(self):
        self._s.clear_meshes()


class RopeSim(_Common):
    """Single rope with a host-driven root, bindings.cpp:185-582."""

    def __init__(self, num_verts, seg_len=0.02, dir=(1.0, 0.0, 0.0), density=0.1, k_stretch=500.0, k_bend=1e-6,
                 max_h=1.0 / 3000.0, num_itr=8, fix_root_orientation=False, collisions=False, precision="f64"):
        if num_verts < 3:
            raise ValueError("num_verts must be >= 3")
        d = np.asarray(dir, np.float32).reshape(3)
        dl = np.float32(np.sqrt(np.float32(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])))
        if not dl > 0:
            raise ValueError("dir must be nonzero")
        d = d / dl
        seg = np.float32(seg_len)
        pos = np.stack([np.float32(i) * seg * d for i in range(num_verts)]).astype(np.float32)
        pins = np.zeros(num_verts, np.uint8)
        pins[0] = 1
        if collisions:
            dead_r, dead_b = 1e-4, 8e-4
        else:
            dead_r, dead_b = np.float32(0.01) * seg, np.float32(0.08) * seg
        sim = _sim_class(precision)(pos, np.array([0, num_verts], np.int32), pins, density, k_stretch, k_bend, max_h,
                                    num_itr, fix_root_orientation, False, False, float(dead_r), float(dead_b))
        super().__init__(sim, max_h)
        self._n = num_verts
        self._fix = fix_root_orientation
        if collisions:
            sim.set_rope_contact(True, 1e-4, 8e-4, 1e-5, 0.1, 5.0, 1.2, 1)
        self.collisions_enabled = bool(collisions)

    num_verts = property(lambda self: self._n)
    fixed_root_orientation = property(lambda self: self._fix)

    def advance(self, dt, substeps=0):
        if substeps < 0:
            raise ValueError("substeps must be >= 0")
        if not dt > 0:
            return
        self._s.advance(float(dt), int(substeps))

    def reset(self):
        self._s.reset_all()

    def set_root(self, pos, vel, q=None):
        qq = None
        if q is not None:
            if not self._fix:
                raise ValueError("set_root(q=...) requires fix_root_orientation=True")
            qq = np.asarray(q, np.float32).reshape(4)
            l = np.float32(np.sqrt(np.float32(np.dot(qq, qq))))
            if not (np.isfinite(l) and l > 1e-6):
                raise ValueError("q must be finite with nonzero norm")
            qq = (qq / l).astype(np.float32)
        self._s.set_root(0, _f32(pos).reshape(3), _f32(vel).reshape(3), qq)

    def positions(self):
        return self._s.positions()

    def velocities(self):
        return self._s.velocities()

    def quaternions(self):
        return self._s.quaternions()

    def inv_masses(self):
        return self._s.inv_masses()

    def rest_lengths(self):
        return self._s.rest_lengths()[:-1]

    def set_velocities(self, v):
        self._s.set_velocities(_f32(v).reshape(-1))

    def set_stretch_stiffnesses(self, ea):
        ea = np.asarray(ea, np.float32)
        if ea.shape != (self._n - 1,) or not (np.isfinite(ea).all() and (ea > 0).all()):
            raise ValueError("expected length n-1 array of finite EA values > 0")
        for i, v in enumerate(ea):
            self._s.set_vertex_ea(i, float(v))

    def set_bend_stiffnesses(self, ei):
        ei = np.asarray(ei, np.float32)
        if ei.shape != (self._n - 1,) or not (np.isfinite(ei).all() and (ei > 0).all()):
            raise ValueError("expected length n-1 array of finite EI values > 0")
        for i, v in enumerate(ei):
            self._s.set_vertex_ei(i, float(v))

    def unpin_root(self):
        self._s.unpin_root()

    def add_mesh(self, values, origin, spacing, pos=(0, 0, 0), quat=(0, 0, 0, 1), mu_s=None, mu_k=None):
        return self._add_mesh(values, origin, spacing, pos, quat, mu_s, mu_k, 1)

    def set_mesh_pose(self, index, pos, quat, teleport=False):
        self._s.set_targets(int(index), _f32(pos).reshape(-1), _f32(quat).reshape(-1), 1, None, bool(teleport))

    def contact_forces(self):
        return self._s.contact_forces()

    def mesh_wrenches(self):
        w = self._s.wrenches().reshape(-1, 2, 3)[: self._s.num_meshes]
        return w.reshape(-1, 6)


class RopeBatch(_Common):
    """N ropes in one solver, bindings.cpp:735-1210, on host arrays. `rope_verts` (a list of
    per-rope vertex counts) extends it to uneven ropes via `from_ropes`."""

    def __init__(self, num_envs, verts_per_rope, root_pos, seg_len=0.02, dir=(0.0, 0.0, -1.0), density=0.1,
                 k_stretch=500.0, k_bend=1e-6, max_h=1.0 / 3000.0, num_itr=8, fix_root_orientation=True,
                 deterministic=False, precision="f64"):
        root_pos = np.asarray(root_pos, np.float32).reshape(num_envs, 3)
        d = np.asarray(dir, np.float32).reshape(3)
        d = d / np.float32(np.sqrt(np.float32(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])))
        seg = np.float32(seg_len)
        pos = np.zeros((num_envs, verts_per_rope, 3), np.float32)
        for v in range(verts_per_rope):
            pos[:, v] = root_pos + np.float32(v) * seg * d
        pins = np.zeros((num_envs, verts_per_rope), np.uint8)
        pins[:, 0] = 1
        self._build(pos.reshape(-1, 3), [verts_per_rope] * num_envs, pins.reshape(-1), density, k_stretch, k_bend, max_h,
                    num_itr, fix_root_orientation, False, seg, precision)

    @classmethod
    def from_positions(cls, positions, density, k_stretch, k_bend, max_h, num_itr, fix_root_orientation=False,
                       pinned=None, straight_rest=False, deterministic=False, precision="f64"):
        p = np.asarray(positions, np.float32)
        N, V = p.shape[0], p.shape[1]
        pins = np.zeros((N, V), np.uint8)
        if pinned is None:
            pins[:, 0] = 1
        else:
            pm = np.asarray(pinned, bool)
            pins[:] = np.broadcast_to(pm, (N, V))
        self = cls.__new__(cls)
        self._build(p.reshape(-1, 3), [V] * N, pins.reshape(-1), density, k_stretch, k_bend, max_h, num_itr,
                    fix_root_orientation, straight_rest, None, precision)
        return self

    @classmethod
    def from_ropes(cls, ropes, density, k_stretch, k_bend, max_h, num_itr, fix_root_orientation=False, pinned=None,
                   straight_rest=False, precision="f64"):
        """Uneven ropes: `ropes` is a list of [V_r, 3] arrays; `pinned` a list of [V_r] masks."""
        verts = [len(r) for r in ropes]
        pos = np.concatenate([np.asarray(r, np.float32) for r in ropes])
        if pinned is None:
            pins = np.concatenate([np.eye(1, v, 0, dtype=np.uint8)[0] for v in verts])
        else:
            pins = np.concatenate([np.asarray(m, np.uint8) for m in pinned])
        self = cls.__new__(cls)
        self._build(pos, verts, pins, density, k_stretch, k_bend, max_h, num_itr, fix_root_orientation, straight_rest,
                    None, precision)
        return self

    def _build(self, pos, verts, pins, density, ks, kb, max_h, num_itr, fix_root, straight_rest, seg, precision):
        starts = np.concatenate([[0], np.cumsum(verts)]).astype(np.int32)
        if seg is None:  # batch.cu:367-373: dead radii from the shortest given segment
            mins = np.float32(1e30)
            for r in range(len(verts)):
                a = pos[starts[r]:starts[r + 1]]
                dd = np.diff(a, axis=0).astype(np.float32)
                lens = np.sqrt((dd * dd).sum(1, dtype=np.float32)).astype(np.float32)
                mins = min(mins, np.float32(lens.min()))
            seg = mins
        sim = _sim_class(precision)(np.ascontiguousarray(pos, np.float32), starts, np.ascontiguousarray(pins, np.uint8),
                                    density, ks, kb, max_h, num_itr, fix_root, straight_rest, True,
                                    float(np.float32(0.01) * np.float32(seg)), float(np.float32(0.08) * np.float32(seg)))
        _Common.__init__(self, sim, max_h)
        self._verts = list(verts)
        self._starts = starts
        self._fix = fix_root
        self.stepped = False

    num_envs = property(lambda self: len(self._verts))
    verts_per_rope = property(lambda self: self._verts[0])
    fixed_root_orientation = property(lambda self: self._fix)

    def _shape(self, a, k):
        if len(set(self._verts)) == 1:
            return a.reshape(len(self._verts), self._verts[0], k)
        return a

    def positions(self):
        return self._shape(self._s.positions(), 3)

    def velocities(self):
        return self._shape(self._s.velocities(), 3)

    def quaternions(self):
        return self._shape(self._s.quaternions(), 4)

    def inv_masses(self):
        return self._shape(self._s.inv_masses(), 1)[..., 0] if len(set(self._verts)) == 1 else self._s.inv_masses()

    def step(self, root_pos, root_vel, dt, substeps, root_q=None, root_pos_end=None, root_q_end=None):
        self.stepped = True
        if root_pos_end is None:
            self._s.step_legacy(_f32(root_pos).reshape(-1), _f32(root_vel).reshape(-1),
                                None if root_q is None else _f32(root_q).reshape(-1), float(dt), int(substeps))
        else:
            self._s.step_program(_f32(root_pos).reshape(-1), _f32(root_vel).reshape(-1), _f32(root_pos_end).reshape(-1),
                                 None if root_q is None else _f32(root_q).reshape(-1),
                                 None if root_q_end is None else _f32(root_q_end).reshape(-1), float(dt), int(substeps))

    def step_free(self, dt, substeps):
        self.stepped = True
        self._s.step_free(float(dt), int(substeps))

    def reset_envs(self, ids):
        self._s.reset_ropes(np.ascontiguousarray(ids, np.int32))

    def set_velocities(self, v):
        self._s.set_velocities(_f32(v).reshape(-1))

    def set_rope_contact(self, enabled, radius=0.0, barrier=0.0, k_collision=0.0, mu=0.0, k_friction=0.0,
                         detection_scaler=1.2, group_ropes=1):
        if enabled and 2 * self._s.min_seg_len < 2 * radius + barrier:
            raise ValueError("rope contact needs 2 * radius + barrier <= 2 * shortest segment")
        self._s.set_rope_contact(bool(enabled), radius, barrier, k_collision, mu, k_friction, detection_scaler,
                                 int(group_ropes))

    def _per_vertex(self, arr, ncols):
        """Per-rope rows of a per-vertex array: [V] (one profile for every rope) or [N, V] for
        uniform batches, or a flat caller-order [total_verts] array for uneven ropes."""
        arr = np.asarray(arr, np.float32)
        N = len(self._verts)
        uniform = len(set(self._verts)) == 1
        out = []
        for r in range(N):
            if not uniform:
                row = arr[self._starts[r]:self._starts[r + 1]]
            else:
                row = arr if arr.ndim == 1 else arr[r]
            out.append(row[:ncols(r)])
        return out

    def set_masses(self, m):
        if self.stepped:
            raise ValueError("set_masses is only legal before the first step")
        for r, row in enumerate(self._per_vertex(m, lambda r: self._verts[r])):
            for v, val in enumerate(row):
                self._s.set_vertex_mass(int(self._starts[r] + v), float(val))

    def set_stretch_stiffnesses(self, ea):
        if self.stepped:
            raise ValueError("set_stretch_stiffnesses is only legal before the first step")
        for r, row in enumerate(self._per_vertex(ea, lambda r: self._verts[r] - 1)):
            for v, val in enumerate(row):
                self._s.set_vertex_ea(int(self._starts[r] + v), float(val))

    def set_bend_stiffnesses(self, ei):
        if self.stepped:
            raise ValueError("set_bend_stiffnesses is only legal before the first step")
        for r, row in enumerate(self._per_vertex(ei, lambda r: self._verts[r] - 1)):
            for v, val in enumerate(row):
                self._s.set_vertex_ei(int(self._starts[r] + v), float(val))

    def add_mesh(self, values, origin, spacing, pos=(0, 0, 0), quat=(0, 0, 0, 1), mu_s=None, mu_k=None):
        rows = 1 if np.asarray(pos).ndim == 1 else len(self._verts)
        return self._add_mesh(values, origin, spacing, pos, quat, mu_s, mu_k, rows)

    def set_mesh_poses(self, index, pos, quat, teleport=False):
        rows = 1 if np.asarray(pos).ndim == 1 else len(self._verts)
        tele_all = isinstance(teleport, (bool, np.bool_)) and bool(teleport)
        tele = None if isinstance(teleport, (bool, np.bool_)) else np.asarray(teleport, np.uint8)
        self._s.set_targets(int(index), _f32(pos).reshape(-1), _f32(quat).reshape(-1), rows, tele, tele_all)

    def set_mesh_poses_all(self, pos, quat, teleport=False):
        tele_all = isinstance(teleport, (bool, np.bool_)) and bool(teleport)
        tele = None if isinstance(teleport, (bool, np.bool_)) else np.asarray(teleport, np.uint8)
        self._s.set_targets(-1, _f32(pos).reshape(-1), _f32(quat).reshape(-1), 0, tele, tele_all)

    def contact_forces(self):
        return self._shape(self._s.contact_forces(), 3)

    def mesh_wrenches(self):
        M = self._s.num_meshes
        w = self._s.wrenches().reshape(len(self._verts), 64, 6)
        return w[:, :M]
