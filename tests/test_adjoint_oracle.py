"""Pins the FP64 hand-written adjoint of the oracle (oracle/rs_adjoint.hpp) on the CPU.

The reference has no gradients, so the adjoint has no reference parity; it is pinned by
  (1) an FP64 torch-autograd restatement of the same update (oracle/torch_rods.py), whose
      forward is first checked against the oracle's, and
  (2) FP64 central finite differences of the oracle's forward (directional derivatives).
The CUDA adjoint is then checked against this adjoint on the GPU (test_gpu_adjoint.py).
Tolerances: forward 1e-9 m (both FP64); adjoint vs autograd 1e-7 relative (both exact gradients
of the same FP64 update, differing only by rounding); adjoint vs finite differences 1e-5 of the
directional derivative plus 1e-7 of |g| |u| plus 1e-14 (Richardson-extrapolated central
differences: truncation and rounding of the quotient; the loss is O(1e-2)).
"""
import numpy as np
import pytest
import torch

import adjoint_cases as ac
import torch_rods as tr

F32 = lambda x: float(np.float32(x))


def _setup(R=3, V=8, I=4, seed=1):
    b, pos = ac.scene(R=R, V=V, seed=seed, plane=True, damping=0.1, drag_quad=1.0, num_itr=I)
    # planes at z = 0 with the tips 4 mm above: contact with friction is active during the frames
    return b, pos


def _cfg(b, dt, S, last_h, I):
    return tr.Config(h=F32(F32(dt) / np.float32(S)), last_h=last_h, num_itr=I, gravity=(0.0, 0.0, F32(-9.81)),
                     damping=F32(0.1), drag=F32(0.2), drag_quad=F32(1.0), drag_quad_t=F32(0.5), accel=1.0,
                     planes=[(0.0, 0.0, 1.0, 0.0)], c_radius=F32(0.00635), mu_s=F32(0.5), mu_k=F32(0.3),
                     v_slip=F32(1e-3), kappa=2.0)


def _torch_inputs(b, R, V):
    s = b._s
    x, v, lv, q, h, _ = s.get_state()  # the frame's prepare() makes the current h its lastH
    ks, rho, w = s.get_params()
    rr = s.rest_rotations()
    nr = np.linalg.norm(rr, axis=1, keepdims=True)
    rq = np.where(nr > 0, rr / np.where(nr > 0, nr, 1), 0.0)
    T = lambda a, *sh: torch.tensor(np.asarray(a).reshape(R, V, *sh), dtype=torch.float64, requires_grad=True)
    st = [T(x, 3), T(v, 3), T(lv, 3), T(q, 4)]
    par = [T(ks), T(rho), T(w)]
    return st, par, torch.tensor(rq.reshape(R, V, 4)), torch.tensor(s.rest_lengths().reshape(R, V)), h


def test_torch_restatement_matches_oracle_forward():
    R, V, I, S, dt = 3, 8, 4, 10, 1 / 600
    b, pos = _setup(R, V, I)
    s = b._s
    P0, V0, P1 = ac.programs(pos, 2, v_std=0.5, p_std=0.01)
    st, par, rq, l, last_h = _torch_inputs(b, R, V)
    state = [t.detach() for t in st]
    for f in range(2):
        cfg = _cfg(b, dt, S, last_h, I)
        pg = [torch.tensor(a[f], dtype=torch.float64) for a in (P0, V0, P1)]
        state = tr.frame(state, [t.detach() for t in par], rq, l, cfg, F32(dt), S, prog=pg)
        s.step_program_rows(np.concatenate([P0[f].ravel(), V0[f].ravel(), P1[f].ravel()]).astype(np.float64), dt, S)
        last_h = cfg.h
        ox = s.get_state()
        for a, o in zip(state, ox[:4]):
            assert np.abs(a.numpy().reshape(o.shape) - o).max() < 1e-9


def test_oracle_adjoint_matches_torch_autograd():
    R, V, I, S, dt = 3, 8, 4, 10, 1 / 600
    b, pos = _setup(R, V, I)
    s = b._s
    P0, V0, P1 = ac.programs(pos, 1, v_std=0.5, p_std=0.01)
    st0 = s.get_state()
    st, par, rq, l, last_h = _torch_inputs(b, R, V)
    pg = [torch.tensor(a[0], dtype=torch.float64, requires_grad=True) for a in (P0, V0, P1)]
    out = tr.frame(st, par, rq, l, _cfg(b, dt, S, last_h, I), F32(dt), S, prog=pg)
    rng = np.random.default_rng(5)
    W = [rng.standard_normal(tuple(o.shape)) for o in out]
    sum((torch.tensor(wi) * o).sum() for wi, o in zip(W, out)).backward()
    s.set_state(*st0)
    prog = np.concatenate([P0[0].ravel(), V0[0].ravel(), P1[0].ravel()]).astype(np.float64)
    g = s.frame_backward(prog, dt, S, *[wi.reshape(-1, wi.shape[-1]) for wi in W])
    w = s.get_params()[2]
    for name, t in [("x", st[0]), ("v", st[1]), ("lv", st[2]), ("q", st[3]), ("ks", par[0]), ("rho", par[1]),
                    ("w", par[2]), ("P0", pg[0]), ("V0", pg[1]), ("P1", pg[2])]:
        a, o = t.grad.numpy().ravel(), g[name].ravel()
        if name == "w":  # pinned vertices: not a parameter (invMass stays 0)
            a, o = a[w != 0], o[w != 0]
        assert ac.rel(o, a) < 1e-7, name


def test_oracle_adjoint_matches_finite_differences():
    R, V, I, S, dt, F = 4, 8, 4, 20, 1 / 300, 3
    b, pos = _setup(R, V, I, seed=3)
    s = b._s
    progs = ac.programs(pos, F + 1, v_std=0.3, p_std=0.01)
    # one frame first, so no clamp of the initial guess sits exactly at its kink (v = lv = 0)
    s.step_program_rows(np.concatenate([a[0].ravel() for a in progs]).astype(np.float64), dt, S)
    progs = [a[1:] for a in progs]
    tgt = ac.targets(pos, F)
    st0 = s.get_state()
    par0 = s.get_params()
    # tip-trajectory loss plus a seeded linear term on the final state, so that every input
    # (V0 included: the root reaches P1 at the frame end whatever V0 is) has an O(1) effect
    wr = np.random.default_rng(7)
    w_end = (1e-2 * wr.standard_normal((R * V, 3)), 1e-3 * wr.standard_normal((R * V, 3)))
    L0, g = ac.oracle_loss_and_grad(b, progs, tgt, dt, S, V, w_end=w_end)
    l = s.rest_lengths()

    def loss(progs_, st_, par_):
        s.set_state(*st_)
        s.set_params(*par_)
        P0, V0, P1 = progs_
        val = 0.0
        for f in range(F):
            s.step_program_rows(np.concatenate([P0[f].ravel(), V0[f].ravel(), P1[f].ravel()]).astype(np.float64), dt, S)
            x = s.get_state()[0].reshape(R, V, 3)
            val += ((x[:, -1] - tgt[f]) ** 2).sum(-1).mean()
        xF, vF = s.get_state()[:2]
        return val + float((w_end[0] * xF).sum() + (w_end[1] * vF).sum())

    rng = np.random.default_rng(11)
    w = par0[2]
    free = w != 0
    seg = np.ones(R * V, bool)
    seg[V - 1::V] = False
    cases = []
    for k, name in enumerate(("g_p0", "g_v0", "g_p1")):
        u = rng.standard_normal(progs[k].shape)
        cases.append((name, u, lambda e, u=u, k=k: loss([p + (e * u if j == k else 0) for j, p in enumerate(progs)], st0, par0), 1e-4))
    # steps sized to each input's effect: initial velocities and frames barely reach the loss
    # (the implicit substeps absorb them), so their differences need larger steps to rise above
    # the rounding of the loss
    for k, name, eps in ((0, "g_pos", 1e-5), (1, "g_vel", 1e-2), (2, "g_lvel", 1e-2), (3, "g_q", 1e-3)):
        u = rng.standard_normal(st0[k].shape)
        if name == "g_pos":
            u[::V] = 0  # the program overwrites the roots
        cases.append((name, u, lambda e, u=u, k=k: loss(progs, [a + e * u if j == k else a for j, a in enumerate(st0)], par0), eps))
    # parameters in the API's units: EA = ks / l, EI = rho l / 4, mass = 1 / w
    ea0, ei0 = par0[0] / l, par0[1] * l / 4
    m0 = np.where(free, 1 / np.where(free, w, 1), 0)
    u = rng.standard_normal(R * V) * seg * ea0
    cases.append(("g_ea", u, lambda e, u=u: loss(progs, st0, [(ea0 + e * u) * l, par0[1], w]), 1e-4))
    u = rng.standard_normal(R * V) * seg * ei0
    cases.append(("g_ei", u, lambda e, u=u: loss(progs, st0, [par0[0], (ei0 + e * u) * 4 / l, w]), 1e-3))
    u = rng.standard_normal(R * V) * free * m0
    cases.append(("g_mass", u, lambda e, u=u: loss(progs, st0, [par0[0], par0[1], np.where(free, 1 / np.where(free, m0 + e * u, 1), 0)]), 1e-4))
    for name, u, fn, eps in cases:
        d1 = (fn(eps) - fn(-eps)) / (2 * eps)
        d2 = (fn(eps / 2) - fn(-eps / 2)) / eps
        fd = (4 * d2 - d1) / 3  # Richardson: O(eps^4) truncation
        ad = float((g[name] * u.reshape(g[name].shape)).sum())
        scale = np.linalg.norm(g[name]) * np.linalg.norm(u)  # bound of the directional derivative
        assert abs(ad - fd) <= 1e-5 * abs(fd) + 1e-7 * scale + 1e-14, (name, ad, fd, scale)


def test_oracle_adjoint_with_mesh_contact_matches_finite_differences():
    """Mesh (SDF) contact differentiated: three config-1 ropes whose tips rest on a static
    r = 0.3 m sphere lattice (64^3), rotated about z; contact carries force during the frames."""
    from ropesim import sdf

    R, V, I, S, dt, F = 3, 8, 4, 20, 1 / 300, 2
    b, pos = ac.scene(R=R, V=V, seed=3, plane=False, material="c1", num_itr=I, clearance=0.0)
    g = sdf.from_function(sdf.sdf_sphere(0.3), [-0.32] * 3, [0.32] * 3, 0.64 / 63)
    b.set_contact(0.005, mu_s=0.5, mu_k=0.3)
    tips = pos[:, -1].astype(np.float64)
    mp = np.stack([tips[r] + np.array([0.0, 0.002 * (r - 1), -0.3045]) for r in range(R)]).astype(np.float32)
    quat = np.tile(np.array([0, 0, np.sin(0.3), np.cos(0.3)], np.float32), (R, 1))
    b.add_mesh(*g.as_args(), pos=mp, quat=quat, mu_s=0.5, mu_k=0.3)
    s = b._s
    progs = ac.programs(pos, F + 1, v_std=0.02, p_std=0.002)
    s.step_program_rows(np.concatenate([a[0].ravel() for a in progs]).astype(np.float64), dt, S)
    progs = [a[1:] for a in progs]
    tgt = ac.targets(pos, F)
    st0, par0 = s.get_state(), s.get_params()
    wr = np.random.default_rng(7)
    w_end = (1e-2 * wr.standard_normal((R * V, 3)), 1e-3 * wr.standard_normal((R * V, 3)))
    L0, gr = ac.oracle_loss_and_grad(b, progs, tgt, dt, S, V, w_end=w_end)

    def loss(progs_, st_, par_, forces=False):
        s.set_state(*st_)
        s.set_params(*par_)
        s.enable_forces(forces)
        P0, V0, P1 = progs_
        val, fsum = 0.0, 0.0
        for f in range(F):
            s.step_program_rows(np.concatenate([P0[f].ravel(), V0[f].ravel(), P1[f].ravel()]).astype(np.float64), dt, S)
            x = s.get_state()[0].reshape(R, V, 3)
            val += ((x[:, -1] - tgt[f]) ** 2).sum(-1).mean()
            if forces:
                fsum += float(np.linalg.norm(s.contact_forces(), axis=1).sum())
        s.enable_forces(False)
        xF, vF = s.get_state()[:2]
        return (val + float((w_end[0] * xF).sum() + (w_end[1] * vF).sum())), fsum

    assert loss(progs, st0, par0, forces=True)[1] > 0.1  # the meshes push on the ropes
    rng = np.random.default_rng(11)
    l = s.rest_lengths()
    w = par0[2]
    free = w != 0
    ea0 = par0[0] / l
    m0 = np.where(free, 1 / np.where(free, w, 1), 0)
    seg = np.ones(R * V, bool)
    seg[V - 1::V] = False
    cases = []
    for k, name in enumerate(("g_p0", "g_v0", "g_p1")):
        u = rng.standard_normal(progs[k].shape)
        cases.append((name, u, lambda e, u=u, k=k: loss([p + (e * u if j == k else 0) for j, p in enumerate(progs)], st0, par0)[0], 1e-6))
    for k, name, eps in ((0, "g_pos", 1e-6), (1, "g_vel", 1e-4), (3, "g_q", 1e-4)):
        u = rng.standard_normal(st0[k].shape)
        if name == "g_pos":
            u[::V] = 0
        cases.append((name, u, lambda e, u=u, k=k: loss(progs, [a + e * u if j == k else a for j, a in enumerate(st0)], par0)[0], eps))
    u = rng.standard_normal(R * V) * seg * ea0
    cases.append(("g_ea", u, lambda e, u=u: loss(progs, st0, [(ea0 + e * u) * l, par0[1], w])[0], 1e-5))
    u = rng.standard_normal(R * V) * free * m0
    cases.append(("g_mass", u, lambda e, u=u: loss(progs, st0, [par0[0], par0[1], np.where(free, 1 / np.where(free, m0 + e * u, 1), 0)])[0], 1e-5))
    for name, u, fn, eps in cases:
        d1 = (fn(eps) - fn(-eps)) / (2 * eps)
        d2 = (fn(eps / 2) - fn(-eps / 2)) / eps
        fd = (4 * d2 - d1) / 3
        ad = float((gr[name] * u.reshape(gr[name].shape)).sum())
        scale = np.linalg.norm(gr[name]) * np.linalg.norm(u)
        assert abs(ad - fd) <= 1e-5 * abs(fd) + 1e-7 * scale + 1e-14, (name, ad, fd, scale)


@pytest.mark.parametrize("case", ["resting_crossing", "falling_onto_bar"])
def test_oracle_adjoint_with_rope_contact_matches_finite_differences(case):
    """Rope-rope contact differentiated: the barrier, its damping and friction, the closest-point
    parameters (u, v) of each candidate pair and the step limit with the limit's own dependence on
    the substep-start state (padding and candidate distances). "resting_crossing": rope 1 rests on
    rope 0 inside the barrier band (stretch damping 0.1); "falling_onto_bar": rope 1 drops 2 cm
    onto a fully pinned rope at h = 1/60, so the step limit clips steps, by both of its bounds."""
    R, V = 2, 10
    # difference steps: the resting scene's small orientation gradient needs larger steps to rise
    # above rounding; the falling scene's clipped steps need smaller ones to stay off their kinks
    if case == "resting_crossing":
        b, pos = ac.rope_crossing(V=V)
        dt, S, F, es = 1 / 300, 20, 3, 1.0
    else:
        b, pos = ac.rope_crossing(V=V, gap=0.02, static_bar=True, damping=0.0)
        dt, S, F, es = 1 / 30, 2, 3, 0.01
    s = b._s
    progs = ac.programs(pos, F + 1, v_std=0.3 if case != "resting_crossing" else 0.05,
                        p_std=0.01 if case != "resting_crossing" else 0.001)
    s.step_program_rows(np.concatenate([a[0].ravel() for a in progs]).astype(np.float64), dt, S)
    progs = [a[1:] for a in progs]
    tgt = ac.targets(pos, F)
    st0, par0 = s.get_state(), s.get_params()
    wr = np.random.default_rng(7)
    w_end = (1e-2 * wr.standard_normal((R * V, 3)), 1e-3 * wr.standard_normal((R * V, 3)))
    L0, gr = ac.oracle_loss_and_grad(b, progs, tgt, dt, S, V, w_end=w_end)

    def loss(progs_, st_, par_):
        s.set_state(*st_)
        s.set_params(*par_)
        P0, V0, P1 = progs_
        val = 0.0
        for f in range(F):
            s.step_program_rows(np.concatenate([P0[f].ravel(), V0[f].ravel(), P1[f].ravel()]).astype(np.float64), dt, S)
            x = s.get_state()[0].reshape(R, V, 3)
            val += ((x[:, -1] - tgt[f]) ** 2).sum(-1).mean()
        xF, vF = s.get_state()[:2]
        return val + float((w_end[0] * xF).sum() + (w_end[1] * vF).sum())

    s.rope_contact_counts()
    loss(progs, st0, par0)
    terms, limited = s.rope_contact_counts()
    assert terms > 0  # barrier terms act during the differentiated frames
    if case == "falling_onto_bar":
        assert limited > 0  # and the step limit clips steps
    rng = np.random.default_rng(11)
    l = s.rest_lengths()
    w = par0[2]
    free = w != 0
    ea0 = par0[0] / l
    m0 = np.where(free, 1 / np.where(free, w, 1), 0)
    seg = np.ones(R * V, bool)
    seg[V - 1::V] = False
    cases = []
    for k, name in enumerate(("g_p0", "g_v0", "g_p1")):
        u = rng.standard_normal(progs[k].shape)
        cases.append((name, u, lambda e, u=u, k=k: loss([p + (e * u if j == k else 0) for j, p in enumerate(progs)], st0, par0), 1e-6 * es))
    for k, name, eps in ((0, "g_pos", 1e-6 * es), (1, "g_vel", 1e-4 * es), (3, "g_q", 1e-4 * es)):
        u = rng.standard_normal(st0[k].shape)
        if name == "g_pos":
            u[::V] = 0
        cases.append((name, u, lambda e, u=u, k=k: loss(progs, [a + e * u if j == k else a for j, a in enumerate(st0)], par0), eps))
    u = rng.standard_normal(R * V) * seg * ea0
    cases.append(("g_ea", u, lambda e, u=u: loss(progs, st0, [(ea0 + e * u) * l, par0[1], w]), 1e-5 * es))
    u = rng.standard_normal(R * V) * free * m0
    cases.append(("g_mass", u, lambda e, u=u: loss(progs, st0, [par0[0], par0[1], np.where(free, 1 / np.where(free, m0 + e * u, 1), 0)]), 1e-3 * es))
    for name, u, fn, eps in cases:
        d1 = (fn(eps) - fn(-eps)) / (2 * eps)
        d2 = (fn(eps / 2) - fn(-eps / 2)) / eps
        fd = (4 * d2 - d1) / 3
        ad = float((gr[name] * u.reshape(gr[name].shape)).sum())
        scale = np.linalg.norm(gr[name]) * np.linalg.norm(u)
        assert abs(ad - fd) <= 1e-5 * abs(fd) + 1e-7 * scale + 1e-14, (name, ad, fd, scale)
