"""TEST INFRASTRUCTURE ONLY: an FP64 torch restatement of the program-driven substep, used as the
reference gradient (torch autograd) for the hand-written adjoints (the oracle's rs_adjoint.hpp and
the CUDA adjoint kernel).

It restates, for ropes of equal length V held as [R, V, ...] tensors, the same deterministic update
as rs_oracle.hpp (which is pinned by the reference's known-answer tests):
  root program           csrc/batch.cu:122-159
  inertial prediction    sim/iteration.cu:34-68 (acceleration-projected gravity)
  position step          sim/cosserat.cu:37-88,198-209 (inertia, plane contact + friction, stretch, damping)
  plane contact          sim/contact.cuh:27-46,141-163
  frame step             sim/cosserat.cu:242-272 (SNAPSHOT ordering)
  velocity / drag        sim/iteration.cu:85-112
Branch decisions (contact active, friction regime, sign choices, clamps) are taken from the
forward values, so autograd differentiates the same active set as the hand-written adjoints.
Rope-rope and mesh contact are not restated here.

Only tests/ import this module.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import torch

DT = torch.float64


def qmul(a, b):
    av, aw = a[..., :3], a[..., 3:]
    bv, bw = b[..., :3], b[..., 3:]
    v = bv * aw + av * bw + torch.cross(av, bv, dim=-1)
    w = aw * bw - (av * bv).sum(-1, keepdim=True)
    return torch.cat([v, w], -1)


def conj(a):
    return torch.cat([-a[..., :3], a[..., 3:]], -1)


def tangent(q):
    x, y, z, w = q.unbind(-1)
    return torch.stack([w * w + x * x - y * y - z * z, 2 * (x * y + w * z), 2 * (x * z - w * y)], -1)


def _safe_norm(v):
    n2 = (v * v).sum(-1)
    pos = n2 > 0
    return torch.where(pos, torch.sqrt(torch.where(pos, n2, torch.ones_like(n2))), torch.zeros_like(n2))


@dataclass
class Config:
    h: float
    last_h: float
    num_itr: int
    gravity: tuple = (0.0, 0.0, -9.81)
    damping: float = 0.0
    drag: float = 0.2
    drag_quad: float = 0.0
    drag_quad_t: float = 0.0
    accel: float = 1.0
    fix_root: bool = False
    planes: list = field(default_factory=list)   # rows (nx, ny, nz, offset), unit normals
    c_radius: float = 0.0
    mu_s: float = 0.5
    mu_k: float = 0.5
    v_slip: float = 1e-3
    kappa: float = 2.0


def _position(x, y, d, q, ks, w, l, cfg: Config):
    R, V = x.shape[:2]
    h = cfg.h
    free = w != 0
    ws = torch.where(free, w, torch.ones_like(w))
    a = 1.0 / (ws * h * h)
    damp = cfg.damping / h
    F = (y - d) * a[..., None]
    Hs = a.clone()
    eye = torch.eye(3, dtype=DT)
    Hc = torch.zeros(R, V, 3, 3, dtype=DT)
    kap = cfg.kappa / h
    kc = kap * kap / ws
    for row in cfg.planes:
        n = torch.tensor(row[:3], dtype=DT)
        gap = ((x * n).sum(-1) - row[3]) + (d * n).sum(-1) - cfg.c_radius
        active = (gap < 0) & free
        N = -kc * gap
        ut = d - n * (d * n).sum(-1, keepdim=True)
        ul = _safe_norm(ut)
        vt = ul / h
        eps = cfg.v_slip
        static = vt <= eps
        kt_s = cfg.mu_s * N / (eps * h)
        sw = 1.0 - torch.clamp(vt / eps - 1.0, max=1.0)
        mu = sw * cfg.mu_s + (1.0 - sw) * cfg.mu_k
        kt_d = mu * N / torch.where(ul > 0, ul, torch.ones_like(ul))
        kt = torch.where(static, kt_s, kt_d)
        f = n * N[..., None] - ut * kt[..., None]
        nn = torch.outer(n, n)
        Hp = kc[..., None, None] * nn - kt[..., None, None] * (nn - eye)
        F = F + torch.where(active[..., None], f, torch.zeros_like(f))
        Hc = Hc + torch.where(active[..., None, None], Hp, torch.zeros_like(Hp))
    invl = 1.0 / l[:, :-1]
    c = ((x[:, 1:] - x[:, :-1]) + (d[:, 1:] - d[:, :-1])) * invl[..., None] - tangent(q[:, :-1])
    kk = ks[:, :-1] * invl
    dd = kk * invl
    own = c * kk[..., None] - d[:, :-1] * (damp * dd)[..., None]
    nxt = -c * kk[..., None] - d[:, 1:] * (damp * dd)[..., None]
    z3 = torch.zeros(R, 1, 3, dtype=DT)
    F = F + torch.cat([own, z3], 1) + torch.cat([z3, nxt], 1)
    ddh = dd * (1.0 + damp)
    z1 = torch.zeros(R, 1, dtype=DT)
    Hs = Hs + torch.cat([ddh, z1], 1) + torch.cat([z1, ddh], 1)
    H = Hs[..., None, None] * eye + Hc
    delta = cfg.accel * torch.linalg.solve(H, F[..., None])[..., 0]
    return torch.where(free[..., None], d + delta, d)


def _frame(x, dn, q, ks, r, l, cfg: Config):
    R, V = x.shape[:2]
    u = ((x[:, 1:] - x[:, :-1]) + (dn[:, 1:] - dn[:, :-1])) / l[:, :-1, None]
    vv = u * (-2.0 * ks[:, :-1, None])
    # segment-pair sign tests D_j = <q_j^-1 q_{j+1}, r_j>, j = 0 .. V-3
    with torch.no_grad():
        D = (qmul(conj(q[:, :V - 2]), q[:, 1:V - 1]) * r[:, :V - 2]).sum(-1)
        sgn = torch.where(D > 0, torch.ones_like(D), -torch.ones_like(D))[..., None]
    z4 = torch.zeros(R, 1, 4, dtype=DT)
    b_prev = torch.cat([z4, qmul(q[:, :V - 2], r[:, :V - 2]) * sgn], 1)          # vertices 1 .. V-2
    # next-orientation term of vertex i: q_{i+1} r_i^*, sign <q_i^-1 q_{i+1}, r_i> (i = 0 .. V-3)
    b_next = torch.cat([qmul(q[:, 1:V - 1], conj(r[:, :V - 2])) * sgn, z4], 1)
    b = b_prev + b_next
    lam = _safe_norm(vv) + _safe_norm(b)
    V4 = torch.cat([vv, torch.zeros(R, V - 1, 1, dtype=DT)], -1)
    e1 = torch.tensor([1.0, 0.0, 0.0, 0.0], dtype=DT).expand(R, V - 1, 4)
    z = qmul(qmul(V4, b), e1) + b * lam[..., None]
    qn = z / _safe_norm(z)[..., None]
    upd = torch.ones(R, V - 1, dtype=torch.bool)
    if cfg.fix_root:
        upd[:, 0] = False
    head = torch.where(upd[..., None], qn, q[:, :V - 1])
    return torch.cat([head, q[:, V - 1:]], 1)


def substep(state, params, rq, l, cfg: Config, prog=None, s=0, dt=None):
    """One substep. state = (x, v, lv, q), params = (ks, rho, w); rq = unit rest rotors [R, V, 4],
    l = rest lengths [R, V]; prog = (P0, V0, P1) [R, 3] each for a program-driven frame."""
    x, v, lv, q = state
    ks, rho, w = params
    h = cfg.h
    if prog is not None:
        P0, V0, P1 = prog
        A = ((P1 - P0) - V0 * dt) * (2.0 / (dt * dt))
        tau = s * h
        xr = P0 + V0 * tau + A * (0.5 * tau * tau)
        vr = V0 + A * (tau + 0.5 * h)
        x = torch.cat([xr[:, None], x[:, 1:]], 1)
        v = torch.cat([vr[:, None], v[:, 1:]], 1)
    free = w != 0
    g = torch.tensor(cfg.gravity, dtype=DT)
    g2 = float((g * g).sum())
    d = v * h
    y = d + g * (h * h)
    if g2 > 0:
        acc = (v - lv) / cfg.last_h
        sg = torch.clamp((acc * g).sum(-1) / g2, 0.0, 1.0)
        d = torch.where(free[..., None], d + g * (h * h) * sg[..., None], d)
    r = rq * rho[..., None]
    for _ in range(cfg.num_itr):
        d = _position(x, y, d, q, ks, w, l, cfg)
        q = _frame(x, d, q, ks, r, l, cfg)
    vel = d / h
    if cfg.drag_quad > 0:
        t = tangent(torch.cat([q[:, :-1], q[:, -2:-1]], 1))  # the last vertex uses the previous frame
        tv = (t * vel).sum(-1, keepdim=True)
        vt = t * tv
        vn = vel - vt
        vn = vn / (1.0 + cfg.drag_quad * _safe_norm(vn)[..., None] * h)
        vt = vt / (1.0 + cfg.drag_quad_t * _safe_norm(vt)[..., None] * h)
        vel = vn + vt
    vel = vel * (1.0 - cfg.drag * h)
    v_out = torch.where(free[..., None], vel, v)
    return x + d, v_out, v, q


def frame(state, params, rq, l, cfg: Config, dt, S, prog=None):
    for s in range(S):
        state = substep(state, params, rq, l, cfg, prog, s, dt)
    return state
