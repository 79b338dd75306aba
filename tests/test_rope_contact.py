"""Rope-rope contact (YarnBall's barrier/friction/step-limit model on per-group brute-force
candidates), ported from the reference's tests/test_contact.py:153-222 and
tests/test_equivalence.py:25-34, on both backends; plus GPU parity of the CTA-resident path,
the plain engine (groups larger than one CTA) and the candidate-overflow error.

Rope: 21 vertices x 5 cm, rho 0.117, EA 11473, EI 4.48e-3, radius 6.35 mm, h = 1/6000, 16 itr;
rope-rope radius 0.9 R, barrier 0.2 R, k_collision 0.025, k_friction 1e7.
"""
import numpy as np
import pytest

import scenarios as S
from conftest import BACKENDS, make_rope, rope_batch_class

NV, SEG, RHO, EA, EI = 21, 0.05, 0.117, 11473.0, 4.48e-3
R = 0.00635
H, ITR, G = 1.0 / 6000.0, 16, 9.81
PEN0 = G * H * H / 4.0
RR = dict(radius=0.9 * R, barrier=0.2 * R, k_collision=0.025, k_friction=1e7)


def dev_fn(backend):
    if backend == "oracle":
        return lambda a: np.ascontiguousarray(a, np.float32)
    import torch

    return lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32), device="cuda")


def host(x):
    if hasattr(x, "__cuda_array_interface__"):
        import torch

        return torch.as_tensor(x).cpu().numpy()
    return np.asarray(x)


def seg_dist(p0, p1, q0, q1):
    d1, d2, r = p1 - p0, q1 - q0, p0 - q0
    a, e, f = (d1 * d1).sum(-1), (d2 * d2).sum(-1), (d2 * r).sum(-1)
    c, bb = (d1 * r).sum(-1), (d1 * d2).sum(-1)
    den = a * e - bb * bb
    s = np.where(den > 1e-12, np.clip((bb * f - c * e) / np.maximum(den, 1e-12), 0, 1), 0.0)
    tt = (bb * s + f) / np.maximum(e, 1e-12)
    s = np.where(tt < 0, np.clip(-c / np.maximum(a, 1e-12), 0, 1), np.where(tt > 1, np.clip((bb - c) / np.maximum(a, 1e-12), 0, 1), s))
    tt = np.clip(tt, 0, 1)
    return np.linalg.norm(p0 + d1 * s[..., None] - (q0 + d2 * tt[..., None]), axis=-1)


def batch(backend, roots, dir3=(0.0, 0.0, -1.0)):
    b = rope_batch_class(backend)(num_envs=len(roots), verts_per_rope=NV, root_pos=np.asarray(roots, np.float32),
                                  seg_len=SEG, dir=np.asarray(dir3, np.float32), density=RHO, k_stretch=EA, k_bend=EI,
                                  max_h=H, num_itr=ITR, fix_root_orientation=False)
    b.damping = 0.0
    b.drag = 0.0
    b.set_gravity(np.array([0.0, 0.0, -G], np.float32))
    return b


@pytest.mark.parametrize("backend", BACKENDS)
def test_rope_rope_no_passthrough(backend):
    """Rope B's root circles rope A: they wind around each other but never interpenetrate."""
    to = dev_fn(backend)
    b = batch(backend, [[0.0, 0.0, 1.1], [0.08, 0.0, 1.1]])
    b.set_rope_contact(True, RR["radius"], RR["barrier"], RR["k_collision"], 0.4, RR["k_friction"], 1.2, 2)
    w = 2 * np.pi * 0.5
    closest = np.inf
    for f in range(90):
        t0, t1 = f / 60, (f + 1) / 60
        pa = np.array([0.0, 0.0, 1.1])
        p0 = np.stack([pa, [0.08 * np.cos(w * t0), 0.08 * np.sin(w * t0), 1.1]]).astype(np.float32)
        p1 = np.stack([pa, [0.08 * np.cos(w * t1), 0.08 * np.sin(w * t1), 1.1]]).astype(np.float32)
        b.step(to(p0), to((p1 - p0) * 60), 1 / 60, 100, root_pos_end=to(p1))
        P = host(b.positions()).astype(np.float64)
        closest = min(closest, seg_dist(P[0, :-1, None], P[0, 1:, None], P[1, None, :-1], P[1, None, 1:]).min())
    print(f"\n  closest centreline distance {closest * 1e3:.2f} mm (contact at 12.7 mm)")
    assert closest > 2 * RR["radius"]


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("mu,expect_slide", [(0.5, False), (0.2, True)])
def test_rope_on_rope_coulomb(backend, mu, expect_slide):
    """Rope B lies on rope A on a 20 deg slope; A grips the floor. B obeys Coulomb with mu."""
    th = np.radians(20.0)
    zA = R - PEN0 * np.cos(th)
    zB = zA + 2 * RR["radius"] + 0.97 * RR["barrier"]
    pos = np.zeros((2, NV, 3), np.float32)
    pos[:, :, 0] = np.arange(NV) * SEG
    pos[0, :, 2], pos[1, :, 2] = zA, zB
    b = rope_batch_class(backend).from_positions(pos, RHO, EA, EI, H, ITR, pinned=np.zeros(NV, bool))
    b.damping = 0.0
    b.drag = 0.0
    b.set_planes(np.array([[0.0, 0.0, 1.0, 0.0]], np.float32), radius=R, mu_s=1.0)
    b.set_rope_contact(True, RR["radius"], RR["barrier"], RR["k_collision"], mu, RR["k_friction"], 1.2, 2)
    b.set_gravity(np.array([G * np.sin(th), 0.0, -G * np.cos(th)], np.float32))
    m = 1.0 / np.asarray(b.inv_masses(), np.float64)
    ts, vB = [], []
    for f in range(36):
        b.step_free(1 / 120, 50)
        V = host(b.velocities()).astype(np.float64)
        ts.append((f + 1) / 120)
        vB.append((m[1][:, None] * V[1]).sum(0)[0] / m[1].sum())
    ts, vB = np.array(ts), np.array(vB)
    a = np.polyfit(ts[ts > 0.05], vB[ts > 0.05], 1)[0]
    if expect_slide:
        assert a == pytest.approx(G * (np.sin(th) - mu * np.cos(th)), rel=0.02)
    else:
        assert abs(a) < 2e-3


@pytest.mark.parametrize("backend", BACKENDS)
def test_rope_contact_groups_isolate_envs(backend):
    """Two envs at the same spot do not see each other (group = 1 rope)."""
    to = dev_fn(backend)

    def run(n):
        b = batch(backend, [[0.0, 0.0, 1.1]] * n)
        b.set_rope_contact(True, RR["radius"], RR["barrier"], RR["k_collision"], 0.4, RR["k_friction"], 1.2, 1)
        for f in range(30):
            p = np.array([[0.0, 0.0, 1.1]] * n, np.float32)
            v = np.zeros((n, 3), np.float32)
            p1 = p.copy()
            if n == 2:
                t0, t1 = f / 60, (f + 1) / 60
                p1[1, 0] = 0.3 * np.sin(6 * t1)
                p[1, 0] = 0.3 * np.sin(6 * t0)
                v[1, 0] = (p1[1, 0] - p[1, 0]) * 60
            b.step(to(p), to(v), 1 / 60, 100, root_pos_end=to(p1))
        return host(b.positions())[0]

    out1, out2 = run(1), run(2)
    assert np.isfinite(out2).all()
    assert np.array_equal(out1, out2)


@pytest.mark.parametrize("backend", BACKENDS)
def test_collisions_on_off_equivalent_when_contact_free(backend):
    """RopeSim(collisions=True) = self contact; contact-free it matches collisions=False."""
    tips = {}
    for col in (False, True):
        r = make_rope(backend, n=25, direction=(0, -1, 0), collisions=col)
        tt = []
        for k in range(90):
            t = k / 60
            p0 = np.array([0.03 * np.sin(2 * np.pi * 0.5 * t), 0, 0], np.float32)
            p1 = np.array([0.03 * np.sin(2 * np.pi * 0.5 * (t + 1 / 60)), 0, 0], np.float32)
            r.set_root(p0, (p1 - p0) * 60)
            r.advance(1 / 60)
            tt.append(np.asarray(r.positions(), np.float64)[-1])
        tips[col] = np.array(tt)
        assert r.last_error == 0
    d = np.max(np.linalg.norm(tips[False] - tips[True], axis=1))
    assert d < 0.01 * 24 * 0.02


# ---------------------------------------------------------------- GPU parity
def contact_pile(mod, to_dev, precision=None, ropes=4, verts=24, frames=6, group=None, engine=None):
    """Ropes hanging side by side 1.5 cm apart, roots swept across each other: dense rope-rope
    contact within one group."""
    kw = {} if precision is None else {"precision": precision}
    pos = np.zeros((ropes, verts, 3), np.float32)
    for r in range(ropes):
        pos[r, :, 0] = 0.015 * r
        pos[r, :, 2] = 1.0 - 0.02 * np.arange(verts)
        pos[r, 1:, 1] = 1e-4 * (r + 1) * np.sin(np.arange(1, verts))
    b = mod.RopeBatch.from_positions(pos, RHO, EA, EI, H, 8, **kw)
    if engine:
        b.set_engine(engine)
    b.damping = 0.0
    b.drag = 0.5
    b.set_gravity(np.array([0.0, 0.0, -G], np.float32))
    b.set_rope_contact(True, RR["radius"], RR["barrier"], RR["k_collision"], 0.4, RR["k_friction"], 1.2, group or ropes)
    out = []
    roots = pos[:, 0].copy()
    for f in range(frames):
        p0 = roots + np.array([0.0, 0.02 * np.sin(f / 3), 0.0], np.float32) * (np.arange(ropes) % 2 - 0.5)[:, None]
        p1 = roots + np.array([0.0, 0.02 * np.sin((f + 1) / 3), 0.0], np.float32) * (np.arange(ropes) % 2 - 0.5)[:, None]
        b.step(to_dev(p0.astype(np.float32)), to_dev(((p1 - p0) * 60).astype(np.float32)), 1 / 60, 50,
               root_pos_end=to_dev(p1.astype(np.float32)))
        out.append(host(b.positions()).reshape(-1, 3).astype(np.float64))
    return np.stack(out)


def _dev(a, b):
    return float(np.max(np.linalg.norm(a - b, axis=-1)))


@pytest.mark.gpu
def test_rope_contact_parity_cta_resident():
    import ropesim
    import ropesim_oracle

    hostf = dev_fn("oracle")
    g = contact_pile(ropesim, dev_fn("cuda"))
    o = contact_pile(ropesim_oracle, hostf, precision="f64")
    o32 = contact_pile(ropesim_oracle, hostf, precision="f32")
    d, d32 = _dev(g, o), _dev(o32, o)
    print(f"\n  rope-rope pile (4x24, one group, 6 frames): gpu-f64 {d:.2e} m, f32-f64 {d32:.2e} m, first frame "
          f"{_dev(g[0], o[0]):.2e} m")
    assert _dev(g[0], o[0]) <= max(1e-5, 4 * _dev(o32[0], o[0]))
    assert d <= 4.0 * d32 + 1e-6


@pytest.mark.gpu
def test_rope_contact_plain_engine_matches():
    import ropesim

    to = dev_fn("cuda")
    g = contact_pile(ropesim, to)
    p = contact_pile(ropesim, to, engine="plain")
    print(f"\n  rope-rope pile, persistent vs plain: {_dev(g, p):.2e} m")
    assert _dev(g[0], p[0]) <= 1e-5


@pytest.mark.gpu
def test_rope_contact_group_larger_than_cta():
    """A 1,200-vertex contact group cannot be CTA-resident: frames run on the plain engine and
    still match the oracle within its FP32 noise floor."""
    import ropesim
    import ropesim_oracle

    hostf = dev_fn("oracle")
    kw = dict(ropes=50, verts=24, frames=2)
    g = contact_pile(ropesim, dev_fn("cuda"), **kw)
    o = contact_pile(ropesim_oracle, hostf, precision="f64", **kw)
    o32 = contact_pile(ropesim_oracle, hostf, precision="f32", **kw)
    d, d32 = _dev(g, o), _dev(o32, o)
    print(f"\n  1200-vertex group (plain engine): gpu-f64 {d:.2e} m, f32-f64 {d32:.2e} m")
    assert d <= max(1e-5, 4.0 * d32 + 1e-6)


@pytest.mark.gpu
def test_candidate_overflow_raises():
    """More than 128 candidates for one segment is a solver error (batch.cu:46, YarnBall.cu:318-321)."""
    import ropesim

    n = 140
    pos = np.zeros((n, 4, 3), np.float32)
    pos[:, :, 2] = 1.0 - 0.01 * np.arange(4)
    pos[:, :, 0] = 1e-4 * np.arange(n)[:, None]
    b = ropesim.RopeBatch.from_positions(pos, RHO, EA, EI, H, 4, pinned=np.ones(4, bool))
    b.set_rope_contact(True, 0.004, 0.001, 0.025, 0.4, 1e7, 1.2, n)
    with pytest.raises(RuntimeError, match="MAX_COLLISIONS"):
        b.step_free(1 / 60, 2)
    assert b.last_error == 1


@pytest.mark.gpu
def test_candidate_overflow_raises_in_grid_broad_phase():
    """The same error from a contact group larger than one CTA (300 x 4 = 1,200 vertices), whose
    detection runs through the grid broad phase: a segment with more than 128 candidates falls
    back to the brute force, which keeps the first 128 and raises."""
    import ropesim

    n = 300
    pos = np.zeros((n, 4, 3), np.float32)
    pos[:, :, 2] = 1.0 - 0.01 * np.arange(4)
    pos[:, :, 0] = 1e-4 * np.arange(n)[:, None]
    b = ropesim.RopeBatch.from_positions(pos, RHO, EA, EI, H, 4, pinned=np.ones(4, bool))
    b.set_rope_contact(True, 0.004, 0.001, 0.025, 0.4, 1e7, 1.2, n)
    with pytest.raises(RuntimeError, match="MAX_COLLISIONS"):
        b.step_free(1 / 60, 2)
    assert b.last_error == 1
