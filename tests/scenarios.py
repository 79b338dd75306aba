"""Seeded parity scenarios shared by the parity tests, the golden-fixture generator and smoke().

Each scenario takes a backend module exposing RopeSim / RopeBatch (the product `ropesim` or the
oracle `ropesim_oracle`) plus a per-frame callback, builds the same scene and returns the
per-frame caller-order positions. Device inputs go through torch tensors for the product and
numpy arrays for the oracle (`to_dev`).

Scenes restate the benchmark configurations at sizes the FP64 oracle finishes in seconds:
  c1        one RopeSim rope, 33 verts (config 1 exactly: 60 frames x 51 substeps)
  program   RopeBatch.from_positions, 64-vertex jittered ropes, config-2 parameters,
            plane z = 0, second-order root program (config 2 at reduced N and frames)
  uneven    RopeBatch.from_ropes, V in [16, 256], per-rope EA/EI, per-vertex mass +-20%,
            2 planes, sphere/box/capsule meshes with random per-env poses every frame,
            contact-force readout (config 3 at reduced N and frames)
  legacy    constant-velocity roots with clamped root frames (RopeBatch.step legacy path)
  planes_only  uneven ropes (16..64 verts) swinging onto one or several planes, no meshes,
            contact-force readout
"""
from __future__ import annotations

import numpy as np

G = 9.81


def c1(mod, frames=60, to_dev=None, precision=None, literal=False):
    """Config 1. The rope is built from the origin along -z (RopeSim has no root argument).
    literal=True calls set_root((0, 0, 1), (0.1, 0, 0)) as the configuration reads, which moves
    only vertex 0 and stretches the first segment from 3 cm to ~1 m: a violent snap whose
    trajectory is chaotic (fp32 and fp64 runs of the same algorithm part by metres within a
    frame). literal=False is the well-posed equivalent: the same rope hanging from its root,
    the root moving at 0.1 m/s (the scene translated by -1 m in z)."""
    kw = {} if precision is None else {"precision": precision}
    r = mod.RopeSim(33, 0.03, np.array([0, 0, -1], np.float32), 0.1, 500.0, 1e-4, 1.0 / 3000.0, 8, **kw)
    r.set_gravity(np.array([0, 0, -G], np.float32))
    r.drag = 0.2
    r.damping = 0.0
    r.set_root(np.array([0, 0, 1.0 if literal else 0.0], np.float32), np.array([0.1, 0, 0], np.float32))
    out = []
    for _ in range(frames):
        r.advance(1.0 / 60.0)
        out.append(np.asarray(r.positions(), np.float64).copy())
    return np.stack(out)


def c2_positions(N, V, seed):
    rng = np.random.default_rng(seed)
    roots = np.stack([rng.uniform(-0.5, 0.5, N), rng.uniform(-0.5, 0.5, N), rng.uniform(1.4, 2.4, N)], 1)
    pos = np.zeros((N, V, 3), np.float32)
    for v in range(V):
        pos[:, v] = roots + np.array([0, 0, -0.02 * v])
    pos[:, 1:] += rng.normal(0, 1e-3, (N, V - 1, 3))
    return pos.astype(np.float32), roots.astype(np.float32)


def program(mod, N=8, V=64, frames=20, S=100, seed=1, to_dev=None, precision=None, views=None, v_std=0.5, p_std=0.05,
            tweak=None):
    """Config 2's workload (64-vertex jittered ropes hanging clear of the plane z = 0, program
    roots with v0 ~ N(0, v_std), p1 = p0 + N(0, p_std)) at reduced N and frames."""
    kw = {} if precision is None else {"precision": precision}
    pos, roots = c2_positions(N, V, seed)
    b = mod.RopeBatch.from_positions(pos, 0.117, 11473.0, 4.48e-3, 1.0 / 6000.0, 8, deterministic=True, **kw)
    b.set_gravity(np.array([0, 0, -G], np.float32))
    b.damping = 0.0
    b.drag = 0.0
    b.set_planes(np.array([[0, 0, 1, 0]], np.float32), radius=0.00635)
    if tweak:
        tweak(b)
    rng = np.random.default_rng(seed + 100)
    p0 = roots.copy()
    out = []
    for _ in range(frames):
        v0 = rng.normal(0, v_std, (N, 3)).astype(np.float32)
        p1 = (p0 + rng.normal(0, p_std, (N, 3))).astype(np.float32)
        b.step(to_dev(p0), to_dev(v0), 1.0 / 60.0, S, root_pos_end=to_dev(p1))
        out.append(views(b) if views else np.asarray(b.positions(), np.float64).copy())
        p0 = p1
    return np.stack(out)


def uneven_ropes(R, seed, lo=16, hi=256, spacing=0.5):
    """R ropes of U{lo..hi} vertices at 1 cm, tilted 25 degrees from vertical, roots on a grid of
    `spacing` m, each rope's lowest vertex 2 cm above the floor z = 0."""
    rng = np.random.default_rng(seed)
    verts = rng.integers(lo, hi + 1, R)
    g = int(np.ceil(np.sqrt(R)))
    ropes = []
    tilt = np.deg2rad(25.0)
    for r in range(R):
        az = rng.uniform(0, 2 * np.pi)
        d = np.array([np.sin(tilt) * np.cos(az), np.sin(tilt) * np.sin(az), -np.cos(tilt)])
        L = 0.01 * (verts[r] - 1)
        root = np.array([(r % g) * spacing, (r // g) * spacing, 0.02 + L * np.cos(tilt)])
        jitter = rng.normal(0, 3e-4, (verts[r], 3)) * (np.arange(verts[r]) > 0)[:, None]
        ropes.append((root + np.outer(np.arange(verts[r]) * 0.01, d) + jitter).astype(np.float32))
    return ropes


def mesh_grids(sdf_mod, spacing=0.02):
    """Sphere, box and capsule lattices (object frame), float32."""
    s = sdf_mod.from_function(sdf_mod.sdf_sphere(0.08), [-0.14] * 3, [0.14] * 3, spacing)
    b = sdf_mod.from_function(sdf_mod.sdf_box([0.08, 0.06, 0.05], round=0.01), [-0.14] * 3, [0.14] * 3, spacing)
    c = sdf_mod.from_function(sdf_mod.sdf_capsule(0.05, 0.08, axis=0), [-0.2, -0.12, -0.12], [0.2, 0.12, 0.12], spacing)
    return [s, b, c]


def random_poses(rng, R, M):
    pos = np.stack([rng.uniform(-0.2, 0.2, (R, M)), rng.uniform(-0.2, 0.2, (R, M)), rng.uniform(0.0, 0.6, (R, M))], -1)
    q = rng.normal(0, 1, (R, M, 4))
    q /= np.linalg.norm(q, axis=-1, keepdims=True)
    return pos.astype(np.float32), q.astype(np.float32)


def walk_poses(rng, pos, q, step=0.004, ang=0.02):
    """One frame of a random rigid walk: pos += N(0, step), q <- exp(N(0, ang)) q."""
    pos = (pos + rng.normal(0, step, pos.shape)).astype(np.float32)
    w = rng.normal(0, ang, pos.shape)
    th = np.linalg.norm(w, axis=-1, keepdims=True)
    ax = w / np.maximum(th, 1e-12)
    dq = np.concatenate([ax * np.sin(th / 2), np.cos(th / 2)], -1)
    x1, y1, z1, w1 = np.moveaxis(dq, -1, 0)
    x2, y2, z2, w2 = np.moveaxis(q.astype(np.float64), -1, 0)
    qn = np.stack([w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2, w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2,
                   w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2, w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2], -1)
    qn /= np.linalg.norm(qn, axis=-1, keepdims=True)
    return pos, qn.astype(np.float32)


def uneven(mod, sdf_mod, R=6, frames=10, S=50, seed=3, to_dev=None, precision=None, forces=True, tweak=None):
    """Config 3's workload at reduced size: uneven ropes, per-rope EA/EI, per-vertex masses,
    two planes, three meshes teleported to random per-env poses and then walked randomly."""
    kw = {} if precision is None else {"precision": precision}
    ropes = uneven_ropes(R, seed)
    b = mod.RopeBatch.from_ropes(ropes, 0.117, 11473.0, 4.48e-3, 1.0 / 3000.0, 8, **kw)
    rng = np.random.default_rng(seed + 7)
    total = sum(len(r) for r in ropes)
    ea = np.exp(rng.uniform(np.log(1e2), np.log(1e4), R))
    ei = np.exp(rng.uniform(np.log(1e-5), np.log(1e-2), R))
    ea_v = np.concatenate([np.full(len(r), ea[i]) for i, r in enumerate(ropes)]).astype(np.float32)
    ei_v = np.concatenate([np.full(len(r), ei[i]) for i, r in enumerate(ropes)]).astype(np.float32)
    lens = [len(r) for r in ropes]
    m_v = []
    for i, r in enumerate(ropes):
        seg = np.linalg.norm(np.diff(r.astype(np.float64), axis=0), axis=1)
        m = np.zeros(len(r))
        m[:-1] += 0.5 * 0.117 * seg
        m[1:] += 0.5 * 0.117 * seg
        m_v.append(m * rng.uniform(0.8, 1.2, len(r)))
    m_v = np.concatenate(m_v).astype(np.float32)
    b.set_stretch_stiffnesses(ea_v)
    b.set_bend_stiffnesses(ei_v)
    b.set_masses(m_v)
    b.set_gravity(np.array([0, 0, -G], np.float32))
    b.damping = 0.0
    b.drag = 0.1
    b.set_planes(np.array([[0, 0, 1, 0], [0.3, 0, 1, -0.05]], np.float32), radius=0.005, mu_s=0.5, mu_k=0.4)
    grids = mesh_grids(sdf_mod)
    for g in grids:
        p, q = random_poses(rng, 1, 1)
        b.add_mesh(*g.as_args(), pos=p[0, 0], quat=q[0, 0])
    if forces:
        b.enable_contact_forces(True)
    if tweak:
        tweak(b)
    out, fo, wr = [], [], []
    M = len(grids)
    # meshes start next to each rope (offsets from its root along its length), random frames
    p, q = random_poses(rng, R, M)
    for r, rope in enumerate(ropes):
        L = 0.01 * (len(rope) - 1)
        for m, frac in enumerate((0.35, 0.65, 0.85)[:M]):
            p[r, m] = rope[0] + np.array([0.12 * np.cos(2.1 * m), 0.12 * np.sin(2.1 * m), -frac * L])
    for f in range(frames):
        if f > 0:
            p, q = walk_poses(rng, p, q)
        b.set_mesh_poses_all(p, q, teleport=(f == 0))
        b.step_free(1.0 / 60.0, S)
        out.append(np.asarray(_flat_positions(b), np.float64).copy())
        if forces:
            fo.append(np.asarray(b.contact_forces(), np.float64).reshape(total, 3).copy())
            wr.append(np.asarray(b.mesh_wrenches(), np.float64).copy())
    return np.stack(out), (np.stack(fo) if forces else None), (np.stack(wr) if forces else None), lens


def planes_only(mod, planes, R=6, frames=10, S=50, seed=11, to_dev=None, precision=None, tweak=None):
    """Uneven ropes (16..64 vertices, roots held, 25 degrees from vertical, lowest vertex 2 cm up)
    swinging onto `planes` alone (no meshes), contact-force readout on: the plane-only kernel
    with one plane or with several."""
    kw = {} if precision is None else {"precision": precision}
    ropes = uneven_ropes(R, seed, lo=16, hi=64)
    b = mod.RopeBatch.from_ropes(ropes, 0.117, 11473.0, 4.48e-3, 1.0 / 3000.0, 8, **kw)
    total = sum(len(r) for r in ropes)
    b.set_gravity(np.array([0, 0, -G], np.float32))
    b.damping = 0.0
    b.drag = 0.1
    b.set_planes(np.asarray(planes, np.float32), radius=0.005, mu_s=0.5, mu_k=0.4)
    b.enable_contact_forces(True)
    if tweak:
        tweak(b)
    out, fo = [], []
    for _ in range(frames):
        b.step_free(1.0 / 60.0, S)
        out.append(np.asarray(_flat_positions(b), np.float64).copy())
        fo.append(np.asarray(b.contact_forces(), np.float64).reshape(total, 3).copy())
    return np.stack(out), np.stack(fo)


# ---------------------------------------------------------------- the benchmarked scenes
# The exact seeded inputs bench.py times, shared with the parity tests that replay samples of
# them rope by rope through the oracle (ropes are independent, so a rope's trajectory does not
# depend on which other ropes share the launch).

BENCH_H, BENCH_ITERS, BENCH_S, BENCH_DT = 1.0 / 6000.0, 8, 100, 1.0 / 60.0


def bench_c2_inputs(n_ropes, frames, seed, V=64):
    """Config 2: 64-vertex jittered ropes hanging clear of z = 0 and their root programs
    (v0 ~ N(0, 0.5) m/s, p1 = p0 + N(0, 0.05) m, next p0 = p1) for `frames` frames."""
    pos, roots = c2_positions(n_ropes, V, seed)
    rng = np.random.default_rng(seed + 1000)
    p0 = np.empty((frames, n_ropes, 3), np.float32)
    v0 = rng.normal(0, 0.5, (frames, n_ropes, 3)).astype(np.float32)
    p1 = np.empty_like(p0)
    cur = roots.copy()
    for f in range(frames):
        p0[f] = cur
        p1[f] = (cur + rng.normal(0, 0.05, (n_ropes, 3))).astype(np.float32)
        cur = p1[f]
    return pos, p0, v0, p1


def bench_c2_configure(b):
    """Config 2's solver settings (damping 0 and drag 0.2 set explicitly, plane z = 0)."""
    b.set_gravity(np.array([0, 0, -G], np.float32))
    b.damping = 0.0
    b.drag = 0.2
    b.set_planes(np.array([[0, 0, 1, 0]], np.float32), radius=0.00635)


def bench_c3_scene(sdf_mod, n_ropes, seed=3):
    """Config 3: n_ropes uneven ropes, V ~ U{16..256} at 2 cm, EA log-U[1e2, 1e4] and
    EI log-U[1e-5, 1e-2] per rope, per-vertex masses x U[0.8, 1.2]; eight 64^3 float32 lattices
    (sphere, box, capsule closed forms). Returns (ropes, verts, ea_v, ei_v, m_v, grids)."""
    rng = np.random.default_rng(seed)
    verts = rng.integers(16, 257, n_ropes)
    g = int(np.ceil(np.sqrt(n_ropes)))
    ropes = []
    for r in range(n_ropes):
        L = 0.02 * (verts[r] - 1)
        root = np.array([(r % g) * 0.7, (r // g) * 0.7, 0.06 + 0.97 * L])
        tilt = np.deg2rad(rng.uniform(5, 20))
        az = rng.uniform(0, 2 * np.pi)
        d = np.array([np.sin(tilt) * np.cos(az), np.sin(tilt) * np.sin(az), -np.cos(tilt)])
        pts = root + np.outer(np.arange(verts[r]) * 0.02, d)
        pts[1:] += rng.normal(0, 1e-3, (verts[r] - 1, 3))
        ropes.append(pts.astype(np.float32))
    ea = np.exp(rng.uniform(np.log(1e2), np.log(1e4), n_ropes))
    ei = np.exp(rng.uniform(np.log(1e-5), np.log(1e-2), n_ropes))
    ea_v = np.concatenate([np.full(v, ea[i]) for i, v in enumerate(verts)]).astype(np.float32)
    ei_v = np.concatenate([np.full(v, ei[i]) for i, v in enumerate(verts)]).astype(np.float32)
    m_v = []
    for rope in ropes:
        seg = np.linalg.norm(np.diff(rope.astype(np.float64), axis=0), axis=1)
        m = np.zeros(len(rope))
        m[:-1] += 0.5 * 0.117 * seg
        m[1:] += 0.5 * 0.117 * seg
        m_v.append(m * rng.uniform(0.8, 1.2, len(rope)))
    m_v = np.concatenate(m_v).astype(np.float32)
    n64 = (0.4) / 63.0
    grids = [sdf_mod.from_function(sdf_mod.sdf_sphere(0.12), [-0.2] * 3, [0.2] * 3, n64),
             sdf_mod.from_function(sdf_mod.sdf_box([0.12, 0.08, 0.06], round=0.01), [-0.2] * 3, [0.2] * 3, n64),
             sdf_mod.from_function(sdf_mod.sdf_capsule(0.06, 0.12, axis=0), [-0.2] * 3, [0.2] * 3, n64)]
    grids = [grids[i % 3] for i in range(8)]
    return ropes, verts, ea_v, ei_v, m_v, grids


def bench_c3_build(mod, scene, sel=None, **kw):
    """A RopeBatch (product or oracle module) of the config-3 scene, or of the ropes `sel` of it
    (same per-vertex EA, EI and masses): two planes, the eight lattices, damping 0, drag 0.2."""
    ropes, verts, ea_v, ei_v, m_v, grids = scene
    if sel is not None:
        starts = np.concatenate([[0], np.cumsum(verts)])
        idx = np.concatenate([np.arange(starts[r], starts[r + 1]) for r in sel])
        ropes = [ropes[r] for r in sel]
        ea_v, ei_v, m_v = ea_v[idx], ei_v[idx], m_v[idx]
    b = mod.RopeBatch.from_ropes(ropes, 0.117, 1000.0, 1e-3, BENCH_H, BENCH_ITERS, **kw)
    lens = {len(r) for r in ropes}
    if len(lens) == 1:  # ropes of one length make a uniform batch: per-segment [N, V-1], per-vertex [N, V]
        Vr = lens.pop()
        ea_v, ei_v, m_v = (x.reshape(-1, Vr) for x in (ea_v, ei_v, m_v))
        ea_v, ei_v = ea_v[:, :-1], ei_v[:, :-1]
    b.set_stretch_stiffnesses(np.ascontiguousarray(ea_v))
    b.set_bend_stiffnesses(np.ascontiguousarray(ei_v))
    b.set_masses(np.ascontiguousarray(m_v))
    b.set_gravity(np.array([0, 0, -G], np.float32))
    b.damping = 0.0
    b.drag = 0.2
    b.set_planes(np.array([[0, 0, 1, 0], [0.05, 0.0, 1.0, -0.02]], np.float32), radius=0.005, mu_s=0.5, mu_k=0.4)
    for gd in grids:
        b.add_mesh(*gd.as_args())
    return b


def bench_c3_inputs(scene, frames, seed=17, M=8):
    """Per-frame mesh poses (per env: next to its rope along its length, then a random rigid walk)
    and root programs (v0 ~ N(0, 0.1), p1 = p0 + N(0, 0.01)) of config 3: pos [F, R, M, 3],
    quat [F, R, M, 4], p0 / v0 / p1 [F, R, 3], all float32. Frame 0's poses teleport."""
    ropes = scene[0]
    R = len(ropes)
    rng = np.random.default_rng(seed)
    p = np.zeros((R, M, 3), np.float32)
    for r, rope in enumerate(ropes):
        L = 0.02 * (len(rope) - 1)
        for m in range(M):
            p[r, m] = rope[0] + np.array([0.25 * np.cos(0.8 * m), 0.25 * np.sin(0.8 * m), -(0.15 + 0.1 * m) * L])
    q = np.zeros((R, M, 4), np.float32)
    q[..., 3] = 1.0
    PP = np.empty((frames, R, M, 3), np.float32)
    QQ = np.empty((frames, R, M, 4), np.float32)
    for f in range(frames):
        PP[f], QQ[f] = p, q
        p, q = walk_poses(rng, p, q, step=0.003, ang=0.02)
    roots = np.stack([r[0] for r in ropes]).astype(np.float32)
    p0 = np.empty((frames, R, 3), np.float32)
    v0 = np.empty_like(p0)
    p1 = np.empty_like(p0)
    cur = roots.copy()
    for f in range(frames):
        p0[f] = cur
        v0[f] = rng.normal(0, 0.1, (R, 3)).astype(np.float32)
        p1[f] = (cur + rng.normal(0, 0.01, (R, 3))).astype(np.float32)
        cur = p1[f]
    return PP, QQ, p0, v0, p1


def _flat_positions(b):
    p = b.positions()
    try:
        import torch

        if hasattr(p, "__cuda_array_interface__"):
            return torch.as_tensor(p).cpu().numpy().reshape(-1, 3)
    except ImportError:
        pass
    return np.asarray(p).reshape(-1, 3)


def legacy(mod, N=4, V=16, frames=30, S=50, to_dev=None, precision=None):
    kw = {} if precision is None else {"precision": precision}
    roots = np.zeros((N, 3), np.float32)
    roots[:, 0] = np.arange(N) * 1.0
    b = mod.RopeBatch(N, V, roots, 0.02, np.array([1, 0, 0], np.float32), 0.05, 2000.0, 0.4, 1.0 / 3000.0, 8,
                      fix_root_orientation=True, **kw)
    b.set_gravity(np.array([0, -9.8, 0], np.float32))
    b.damping = 0.0
    b.drag = 1.0
    out = []
    for k in range(frames):
        th = np.deg2rad(30.0) * (k + 1) / frames * (1 + np.arange(N)) / N
        q = np.zeros((N, 4), np.float32)
        q[:, 2] = np.sin(th / 2)
        q[:, 3] = np.cos(th / 2)
        vel = np.zeros((N, 3), np.float32)
        vel[:, 1] = 0.05 * np.sin(k / 5.0)
        p = roots + vel * (k / 60.0)
        b.step(to_dev(p), to_dev(vel), 1.0 / 60.0, S, root_q=to_dev(q))
        out.append(np.asarray(_flat_positions(b), np.float64).copy())
    return np.stack(out)
