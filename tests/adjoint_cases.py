"""Scenes and oracle-side trajectory gradients shared by the adjoint tests (test infrastructure).

The loss is the differentiable workload's: mean squared distance of every rope's tip to a seeded
target curve, summed over control frames. Oracle gradients chain the FP64 hand-written adjoint
(oracle/rs_adjoint.hpp) frame by frame, with the frame-start states as checkpoints.
"""
from __future__ import annotations

import numpy as np

import ropesim_oracle as ro


# Materials: (segment length, density, EA, EI). "c1": the single-rope configuration's rope
# (3 cm segments, 0.1 kg/m, EA 500 N, EI 1e-4 N m^2), which the differentiable workload uses;
# "c2": the batched configuration's stiff rope (2 cm, 0.117 kg/m, EA 11473 N, EI 4.48e-3 N m^2).
MATERIALS = {"c1": (0.03, 0.1, 500.0, 1e-4), "c2": (0.02, 0.117, 11473.0, 4.48e-3)}


def mesh_setup(pos):
    """A static mesh under every rope's tip: a 0.2 x 0.2 x 0.1 m box lattice (64^3, edges rounded
    by 1 cm), its flat top 2 mm above the tip (the tip sits inside the 5 mm contact band, so the
    contact stays on, as with the plane scenes), rotated 0.6 rad about z. Returns (lattice args,
    positions [R, 3], rotors [R, 4])."""
    from ropesim import sdf

    R = pos.shape[0]
    g = sdf.from_function(sdf.sdf_box([0.1, 0.1, 0.05], round=0.01), [-0.14] * 3, [0.14] * 3, 0.28 / 63)
    tips = pos[:, -1].astype(np.float64)
    mp = np.stack([tips[r] + np.array([0.01 * ((r % 3) - 1), 0.0, 0.002 - 0.05]) for r in range(R)]).astype(np.float32)
    quat = np.tile(np.array([0, 0, np.sin(0.3), np.cos(0.3)], np.float32), (R, 1))
    return g.as_args(), mp, quat


def scene(R=8, V=16, seed=0, plane=True, damping=0.0, drag_quad=0.0, num_itr=8, precision="f64", material="c2",
          clearance=0.004, mesh=False, free=False):
    """R hanging ropes of V vertices, tips `clearance` above a plane at z = 0 (when `plane`), or
    resting on a static mesh (when `mesh`, see mesh_setup). `free`: no vertex pinned."""
    seg, density, ea, ei = MATERIALS[material]
    rng = np.random.default_rng(seed)
    pos = np.zeros((R, V, 3), np.float32)
    for r in range(R):
        pos[r, :, 0] = 0.15 * (r % 4)
        pos[r, :, 1] = 0.15 * (r // 4)
        pos[r, :, 2] = seg * (V - 1) + clearance - seg * np.arange(V)
        pos[r, 1:, :2] += rng.normal(0, 1e-3, (V - 1, 2)).astype(np.float32)
    pins = np.zeros(V, bool) if free else None
    b = ro.RopeBatch.from_positions(pos, density, ea, ei, 1 / 6000, num_itr, pinned=pins, precision=precision)
    b.set_gravity((0.0, 0.0, -9.81))
    b.damping = damping
    b.drag = 0.2
    b.drag_quad = drag_quad
    b.drag_quad_t = 0.5 * drag_quad
    if plane:
        b.set_planes([[0.0, 0.0, 1.0, 0.0]], radius=0.00635, mu_s=0.5, mu_k=0.3)
    if mesh:  # frictionless: with friction the FP32 gradient of this resting contact is ill-conditioned
        args, mp, quat = mesh_setup(pos)
        b.set_contact(0.005, mu_s=0.0, mu_k=0.0)
        b.add_mesh(*args, pos=mp, quat=quat, mu_s=0.0, mu_k=0.0)
    return b, pos


def programs(pos, F, seed=1, v_std=0.3, p_std=0.02):
    """Per-frame root programs (p0, v0, p1) [F, R, 3] chaining p0 = previous p1 (float32 values)."""
    rng = np.random.default_rng(seed)
    R = pos.shape[0]
    p0 = pos[:, 0].astype(np.float32)
    out = []
    for _ in range(F):
        v0 = rng.normal(0, v_std, (R, 3)).astype(np.float32)
        p1 = (p0 + rng.normal(0, p_std, (R, 3))).astype(np.float32)
        out.append((p0.copy(), v0, p1))
        p0 = p1
    return [np.stack([o[k] for o in out]) for k in range(3)]


def targets(pos, F, seed=2):
    """Seeded target curve of each rope's tip, [F, R, 3]."""
    rng = np.random.default_rng(seed)
    R = pos.shape[0]
    base = pos[:, -1].astype(np.float64)
    t = np.arange(1, F + 1)[:, None, None] / F
    amp = rng.normal(0, 0.05, (1, R, 3))
    return base[None] + amp * np.sin(2 * np.pi * t)


def oracle_loss_and_grad(b, progs, tgt, dt, S, V, w_end=None):
    """FP64 loss and its gradients through the oracle's adjoint, frame by frame. `w_end` =
    (Wx, Wv) [n, 3] adds sum(Wx * x_F + Wv * v_F) of the final state to the loss.
    Returns (loss, dict) with g_pos/g_vel/g_lvel/g_q of the initial state, g_ea/g_ei/g_mass per
    vertex and g_p0/g_v0/g_p1 [F, R, 3]."""
    s = b._s
    free = progs is None or (not isinstance(progs[0], np.ndarray) and progs[0] is None)
    if free:  # free frames: progs = (None, None, None) or None, with F = len(tgt)
        F, R = len(tgt), tgt.shape[1]
    else:
        P0, V0, P1 = progs
        F, R = P0.shape[:2]
    n = s.n
    starts = []
    loss = 0.0
    tips = []
    for f in range(F):
        starts.append(s.get_state())
        if free:
            s.step_free(dt, S)
        else:
            s.step_program_rows(np.concatenate([P0[f].ravel(), V0[f].ravel(), P1[f].ravel()]).astype(np.float64), dt, S)
        x = s.get_state()[0].reshape(R, V, 3)
        tips.append(x[:, -1])
        loss += ((x[:, -1] - tgt[f]) ** 2).sum(-1).mean()
    ks, rho, w = s.get_params()
    l = s.rest_lengths()
    gx, gv, glv, gq = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros((n, 3)), np.zeros((n, 4))
    if w_end is not None:
        xF, vF = s.get_state()[:2]
        loss += float((w_end[0] * xF).sum() + (w_end[1] * vF).sum())
        gx += w_end[0]
        gv += w_end[1]
    gks, grho, gw = np.zeros(n), np.zeros(n), np.zeros(n)
    gP = [np.zeros((F, R, 3)) for _ in range(3)]
    end = s.get_state()
    for f in range(F - 1, -1, -1):
        gx.reshape(R, V, 3)[:, -1] += 2.0 * (tips[f] - tgt[f]) / R
        s.set_state(*starts[f])
        prog = None if free else np.concatenate([P0[f].ravel(), V0[f].ravel(), P1[f].ravel()]).astype(np.float64)
        g = s.frame_backward(prog, dt, S, gx, gv, glv, gq)
        gx, gv, glv, gq = g["x"], g["v"], g["lv"], g["q"]
        gks += g["ks"]; grho += g["rho"]; gw += g["w"]
        if not free:
            gP[0][f], gP[1][f], gP[2][f] = g["P0"], g["V0"], g["P1"]
    s.set_state(*end)
    return loss, {
        "g_pos": gx, "g_vel": gv, "g_lvel": glv, "g_q": gq,
        "g_ea": gks * l, "g_ei": grho * 4.0 / l, "g_mass": -w * w * gw,
        "g_p0": gP[0], "g_v0": gP[1], "g_p1": gP[2],
    }


def rel(a, b):
    """Norm-wise relative difference |a - b| / |b|."""
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def rope_crossing(V=10, seed=0, num_itr=4, gap=0.005, static_bar=False, damping=0.1, precision="f64", backend="oracle",
                  pairs=1, floor=None):
    """Two ropes of the "c1" material in one rope-rope contact group, crossing at right angles:
    rope 0 along x at z = 0 with both ends pinned (every vertex pinned when `static_bar`), rope 1
    along y, `gap` above it (centre to centre), pinned at its root. Contact radius 2 mm, barrier
    2 mm: the barrier acts while the centre lines are 4 to 6 mm apart. `backend` "cuda" builds
    the same scene on the GPU batch. `pairs` > 1 repeats the crossing along x (pair p shifted by
    p x (V + 4) x 3 cm, clear of the others), all ropes in one contact group. `floor` = z makes
    every vertex free (no pins) and adds the plane z = floor with contact radius 2 mm."""
    seg, density, ea, ei = MATERIALS["c1"]
    rng = np.random.default_rng(seed)
    r0 = np.zeros((V, 3))
    r0[:, 0] = seg * (np.arange(V) - (V - 1) / 2)
    r1 = np.zeros((V, 3))
    r1[:, 0] = 0.004
    r1[:, 1] = seg * (np.arange(V) - 3.0)
    r1[:, 2] = gap
    r1[1:] += rng.normal(0, 3e-4, (V - 1, 3))
    pin0 = np.zeros(V, bool)
    pin0[0] = pin0[-1] = True
    if static_bar:
        pin0[:] = True
    pin1 = np.zeros(V, bool)
    pin1[0] = True
    if floor is not None:
        pin0[:] = False
        pin1[:] = False
    ropes, pins = [], []
    for k in range(pairs):
        shift = np.array([k * (V + 4) * seg, 0.0, 0.0])
        ropes += [r0 + shift, r1 + shift]
        pins += [pin0, pin1]
    pos = np.stack(ropes).astype(np.float32)
    if backend == "cuda":
        import ropesim

        b = ropesim.RopeBatch.from_ropes(list(pos), density, ea, ei, 1 / 6000, num_itr, pinned=pins)
    else:
        b = ro.RopeBatch.from_ropes(list(pos), density, ea, ei, 1 / 6000, num_itr, pinned=pins, precision=precision)
    b.set_gravity(np.array([0.0, 0.0, -9.81], np.float32))
    b.damping = damping
    b.drag = 0.2
    b.set_rope_contact(True, radius=0.002, barrier=0.002, k_collision=0.025, mu=0.1, k_friction=1e7,
                       group_ropes=2 * pairs)
    if floor is not None:
        b.set_planes(np.array([[0.0, 0.0, 1.0, floor]], np.float32), radius=0.002, mu_s=0.5, mu_k=0.3)
    return b, pos
