"""The CUDA adjoint (rs_batch_backward behind ropesim.grad) against the FP64 oracle adjoint.

Workload: the differentiable configuration's check size, 8 ropes x 16 vertices of the
config-1 rope (3 cm segments, density 0.1, EA 500, EI 1e-4, 8 iterations), program roots,
5 control frames x 100 substeps of 1/6000 s, loss = mean squared distance of the rope tips to
a seeded target curve summed over frames. Gradients with respect to the root programs
(p0, v0, p1 of every frame), EA, EI, per-vertex mass and the initial state. Scenes: free ropes,
ropes resting on a plane, damped ropes with quadratic drag, ropes resting on a static SDF mesh
(a box lattice whose flat top holds the tips in contact, frictionless: with mesh friction the
FP32 and FP64 gradients of this resting contact already differ by 2e-3 .. 1e-2, so FP32 cannot
be checked there; curved mesh contact with friction is checked against FP64 finite differences
on the CPU, test_adjoint_oracle.py).

The oracle adjoint is pinned on the CPU by FP64 finite differences and by FP64 torch autograd
(test_adjoint_oracle.py); here the GPU's FP32 gradients are compared with it. Tolerance, per
gradient group (norm-wise relative): 1e-4, or 4x the deviation of the oracle's own FP32
adjoint from FP64 when that FP32 noise floor is larger (an FP32 gradient linearises the FP32
trajectory, which itself deviates from the FP64 one, and the bin size the autotuner picks
changes the adjoint's rounding). A direct check against FP64 central finite differences of the
oracle's forward along seeded directions uses the same rule, the floor taken as the larger of
the FP32 oracle's error along the direction and over the gradient group.

Scenes whose FP64 loss is itself ill-conditioned are not usable here: with the stiff config-2
rope (EA 11473 N on 2 cm segments) and no damping, 8 Jacobi sweeps leave the stiffest stretch
mode unconverged, and FP64 finite differences of the tip loss with respect to the initial
positions disagree with each other by 10% across step sizes.
"""
import numpy as np
import pytest

import adjoint_cases as ac

pytestmark = pytest.mark.gpu

R, V, F, S, DT = 8, 16, 5, 100, 1.0 / 60.0
GROUPS = ["g_p0", "g_v0", "g_p1", "g_ea", "g_ei", "g_mass", "g_pos", "g_vel", "g_lvel", "g_q"]
SCENES = {
    "free": (dict(plane=False), dict(v_std=0.3, p_std=0.02)),
    "resting_on_plane": (dict(plane=True, clearance=-0.002), dict(v_std=0.05, p_std=0.01)),
    "damped_quadratic_drag": (dict(plane=False, damping=0.01, drag_quad=2.0), dict(v_std=0.3, p_std=0.02)),
    "resting_on_mesh": (dict(plane=False, mesh=True, clearance=0.0), dict(v_std=0.05, p_std=0.01)),
}


def _gpu_batch(pos, plane=True, damping=0.0, drag_quad=0.0, material="c1", clearance=None, mesh=False, engine=None):
    import ropesim

    _, density, ea, ei = ac.MATERIALS[material]
    b = ropesim.RopeBatch.from_positions(pos, density, ea, ei, 1 / 6000, 8)
    b.set_gravity(np.array([0.0, 0.0, -9.81], np.float32))
    b.damping = damping
    b.drag = 0.2
    b.drag_quad = drag_quad
    b.drag_quad_t = 0.5 * drag_quad
    if plane:
        b.set_planes(np.array([[0.0, 0.0, 1.0, 0.0]], np.float32), radius=0.00635, mu_s=0.5, mu_k=0.3)
    if mesh:
        args, mp, quat = ac.mesh_setup(pos)
        b.set_contact(0.005, mu_s=0.0, mu_k=0.0)
        b.add_mesh(*args, pos=mp, quat=quat, mu_s=0.0, mu_k=0.0)
    if engine:
        b.set_engine(engine)
    return b


def _gpu_loss_and_grad(pos, progs, tgt, tape=True, **kw):
    import torch

    import ropesim.grad as rg

    b = _gpu_batch(pos, **kw)
    st = [t.clone().requires_grad_() for t in rg.state(b)]
    par = [t.clone().requires_grad_() for t in rg.parameters(b)]
    P = [torch.tensor(a, device="cuda", requires_grad=True) for a in progs]
    tg = torch.tensor(tgt, device="cuda", dtype=torch.float32)
    cur = st
    loss = 0.0
    for f in range(F):
        cur = rg.frame(b, cur, par, P[0][f], P[1][f], P[2][f], DT, S, tape=tape)
        tip = cur[0].view(R, V, 3)[:, -1]
        loss = loss + ((tip - tg[f]) ** 2).sum(-1).mean()
    loss.backward()
    g = {"g_p0": P[0].grad, "g_v0": P[1].grad, "g_p1": P[2].grad, "g_ea": par[0].grad, "g_ei": par[1].grad,
         "g_mass": par[2].grad, "g_pos": st[0].grad, "g_vel": st[1].grad, "g_lvel": st[2].grad, "g_q": st[3].grad}
    return float(loss.detach()), {k: v.detach().cpu().numpy().astype(np.float64) for k, v in g.items()}, b


@pytest.mark.parametrize("engine", ["persistent", "persistent_iterates", "plain"])
@pytest.mark.parametrize("kind", list(SCENES))
def test_adjoint_matches_fp64_oracle(kind, engine):
    """Both engines: the CTA-resident adjoint kernel after persistent frames (recomputing the
    iterates, or reading them from the forward's iterate tape), the per-launch adjoint
    (rs_adjoint_plain.cu) after plain-engine frames."""
    kw, pk = SCENES[kind]
    kw = dict(material="c1", **kw)
    ob, pos = ac.scene(R=R, V=V, **kw)
    progs = ac.programs(pos, F, **pk)
    tgt = ac.targets(pos, F)
    L64, g64 = ac.oracle_loss_and_grad(ob, progs, tgt, DT, S, V)
    ob32, _ = ac.scene(R=R, V=V, precision="f32", **kw)
    _, g32 = ac.oracle_loss_and_grad(ob32, progs, tgt, DT, S, V)
    tape = "iterates" if engine == "persistent_iterates" else True
    L, g, _ = _gpu_loss_and_grad(pos, progs, tgt, tape=tape, engine="plain" if engine == "plain" else None, **kw)
    print(f"\n  [{kind}, {engine}] loss gpu {L:.8e} fp64 {L64:.8e}")
    assert abs(L - L64) <= 1e-4 * abs(L64)
    for k in GROUPS:
        e_gpu = ac.rel(g[k], g64[k])
        e_32 = ac.rel(g32[k], g64[k])
        print(f"  {k:7s} |g| {np.linalg.norm(g64[k]):.3e}  gpu-vs-fp64 {e_gpu:.2e}  fp32-oracle-vs-fp64 {e_32:.2e}")
        assert np.isfinite(g[k]).all()
        assert e_gpu <= max(1e-4, 4 * e_32), k


def test_adjoint_matches_fp64_finite_differences():
    kw = dict(material="c1", plane=False)
    ob, pos = ac.scene(R=R, V=V, **kw)
    progs = ac.programs(pos, F, v_std=0.3, p_std=0.02)
    tgt = ac.targets(pos, F)
    _, g, _ = _gpu_loss_and_grad(pos, progs, tgt, **kw)
    ob32, _ = ac.scene(R=R, V=V, precision="f32", **kw)
    _, g32 = ac.oracle_loss_and_grad(ob32, progs, tgt, DT, S, V)
    s = ob._s
    st0, par0 = s.get_state(), s.get_params()  # the start state, before any stepping
    _, g64 = ac.oracle_loss_and_grad(ob, progs, tgt, DT, S, V)
    l = s.rest_lengths()
    seg = np.ones(R * V, bool)
    seg[V - 1::V] = False

    def loss(pr, par):
        s.set_state(*st0)
        s.set_params(*par)
        val = 0.0
        for f in range(F):
            s.step_program_rows(np.concatenate([pr[0][f].ravel(), pr[1][f].ravel(), pr[2][f].ravel()]).astype(np.float64), DT, S)
            x = s.get_state()[0].reshape(R, V, 3)
            val += ((x[:, -1] - tgt[f]) ** 2).sum(-1).mean()
        return val

    rng = np.random.default_rng(3)
    progs64 = [a.astype(np.float64) for a in progs]
    ea0, ei0 = par0[0] / l, par0[1] * l / 4
    cases = []
    # p0 moves the root's position at the frame start (a jump from the previous frame's end), so
    # the loss is sharply curved along it: its differences need a 1e-6 step
    for k, name, eps in ((0, "g_p0", 1e-6), (1, "g_v0", 1e-4), (2, "g_p1", 1e-4)):
        u = rng.standard_normal(progs64[k].shape)
        cases.append((name, u, lambda e, u=u, k=k: loss([p + e * u if j == k else p for j, p in enumerate(progs64)], par0), eps))
    u = rng.standard_normal(R * V) * seg * ea0
    cases.append(("g_ea", u, lambda e, u=u: loss(progs64, [(ea0 + e * u) * l, par0[1], par0[2]]), 1e-4))
    u = rng.standard_normal(R * V) * seg * ei0
    cases.append(("g_ei", u, lambda e, u=u: loss(progs64, [par0[0], (ei0 + e * u) * 4 / l, par0[2]]), 1e-3))
    for name, u, fn, eps in cases:
        d1 = (fn(eps) - fn(-eps)) / (2 * eps)
        d2 = (fn(eps / 2) - fn(-eps / 2)) / eps
        fd = (4 * d2 - d1) / 3
        ad = float((g[name] * u.reshape(g[name].shape)).sum())
        a32 = float((g32[name] * u.reshape(g32[name].shape)).sum())
        # FP32 noise floor: the FP32 oracle's error along u and over the whole group
        floor = max(abs(a32 - fd) / abs(fd), ac.rel(g32[name], g64[name]))
        print(f"\n  {name}: gpu {ad:+.8e} fd64 {fd:+.8e} rel {abs(ad - fd) / abs(fd):.2e} (fp32 oracle {floor:.2e})")
        assert floor < 1e-2, name  # the rule must not be vacuous
        assert abs(ad - fd) <= max(1e-4, 4 * floor) * abs(fd), name


def test_taped_and_replayed_backward_agree():
    """The backward from the forward's own tape equals the one that replays the frame, bitwise. The
    one that reads the forward's iterates (tape="iterates") instead of recomputing them linearises
    the same trajectory; the adjoint kernel's recomputation matches the frame kernel's iterates only
    to FP32 rounding (two kernels, two instruction schedules), so these agree to the scene's FP32
    noise (it is checked against the FP64 oracle in test_adjoint_matches_fp64_oracle)."""
    kw = dict(material="c1", plane=True, clearance=-0.002)
    _, pos = ac.scene(R=R, V=V, **kw)
    progs = ac.programs(pos, 3, v_std=0.05, p_std=0.01)
    tgt = ac.targets(pos, 3)
    global F
    F0, F = F, 3
    try:
        La, ga, _ = _gpu_loss_and_grad(pos, progs, tgt, tape=True, **kw)
        Lb, gb, _ = _gpu_loss_and_grad(pos, progs, tgt, tape=False, **kw)
        Lc, gc, _ = _gpu_loss_and_grad(pos, progs, tgt, tape="iterates", **kw)
    finally:
        F = F0
    assert La == Lb == Lc
    for k in GROUPS:
        assert np.array_equal(ga[k], gb[k]), k
        print(f"  {k:7s} iterate tape vs recomputed: {ac.rel(gc[k], ga[k]):.2e}")
        assert np.isfinite(gc[k]).all()


def test_differentiable_frame_forward_is_the_step():
    """rg.frame advances like RopeBatch.step (same kernel; state and parameters round-tripped)."""
    import torch

    import ropesim.grad as rg

    _, pos = ac.scene(R=R, V=V, plane=True, material="c1")
    progs = ac.programs(pos, 2)
    a = _gpu_batch(pos)
    b = _gpu_batch(pos)
    st = rg.state(b)
    par = rg.parameters(b)
    for f in range(2):
        p0, v0, p1 = (torch.tensor(x[f], device="cuda") for x in progs)
        a.step(p0, v0, DT, S, root_pos_end=p1)
        with torch.no_grad():
            st = rg.frame(b, st, par, p0, v0, p1, DT, S)
        xa = torch.as_tensor(a.positions()).reshape(-1, 3)
        # EA, EI and mass round-trip through EA l, 4 EI / l and 1 / m (a rounding each)
        assert float((xa - st[0]).abs().max()) <= 1e-5


def test_adjoint_refuses_moving_meshes():
    """Mesh poses are differentiated as constants: a frame with pending mesh targets (a mesh
    that moves during it) is refused, by the taped step or the backward."""
    import torch

    import ropesim.grad as rg

    _, pos = ac.scene(R=R, V=V, plane=False, material="c1")
    progs = ac.programs(pos, 1)
    b = _gpu_batch(pos, plane=False, mesh=True)
    _, mp, quat = ac.mesh_setup(pos)
    b.set_mesh_poses(0, mp + np.float32(0.01), quat)
    st = [t.requires_grad_() for t in rg.state(b)]
    par = rg.parameters(b)
    p0, v0, p1 = (torch.tensor(x[0], device="cuda") for x in progs)
    with pytest.raises(ValueError, match="static meshes"):
        out = rg.frame(b, st, par, p0, v0, p1, DT, 10)
        out[0].sum().backward()


@pytest.mark.parametrize("engine", ["persistent", "plain"])
def test_free_frames_adjoint_matches_fp64_oracle(engine):
    """Free frames (no root program: p0 = v0 = p1 = None): unpinned ropes thrown with seeded
    vertex velocities N(0, 0.3) m/s; gradients w.r.t. EA, EI, mass and the initial state."""
    import torch

    import ropesim
    import ropesim.grad as rg

    kw = dict(material="c1", plane=False, free=True)
    ob, pos = ac.scene(R=R, V=V, **kw)
    vel0 = np.random.default_rng(4).normal(0, 0.3, (R * V, 3))
    tgt = ac.targets(pos, F)
    res = {}
    for prec in ("f64", "f32"):
        o, _ = ac.scene(R=R, V=V, precision=prec, **kw)
        st = list(o._s.get_state())
        st[1] = vel0.copy()
        o._s.set_state(*st)
        res[prec] = ac.oracle_loss_and_grad(o, None, tgt, DT, S, V)
    (L64, g64), (_, g32) = res["f64"], res["f32"]
    _, density, ea, ei = ac.MATERIALS["c1"]
    b = ropesim.RopeBatch.from_positions(pos, density, ea, ei, 1 / 6000, 8, pinned=np.zeros(V, bool))
    b.set_gravity(np.array([0.0, 0.0, -9.81], np.float32))
    b.damping = 0.0
    b.drag = 0.2
    if engine == "plain":
        b.set_engine("plain")
    st = [t.clone() for t in rg.state(b)]
    st[1] = torch.tensor(vel0, device="cuda", dtype=torch.float32)
    st = [t.requires_grad_() for t in st]
    par = [t.clone().requires_grad_() for t in rg.parameters(b)]
    tg = torch.tensor(tgt, device="cuda", dtype=torch.float32)
    cur, loss = st, 0.0
    for f in range(F):
        cur = rg.frame(b, cur, par, None, None, None, DT, S)
        loss = loss + ((cur[0].view(R, V, 3)[:, -1] - tg[f]) ** 2).sum(-1).mean()
    loss.backward()
    g = {"g_ea": par[0].grad, "g_ei": par[1].grad, "g_mass": par[2].grad, "g_pos": st[0].grad, "g_vel": st[1].grad,
         "g_lvel": st[2].grad, "g_q": st[3].grad}
    L = float(loss.detach())
    print(f"\n  [free frames, {engine}] loss gpu {L:.8e} fp64 {L64:.8e}")
    assert abs(L - L64) <= 1e-4 * abs(L64)
    for k, v in g.items():
        gk = v.detach().cpu().numpy().astype(np.float64)
        e_gpu, e_32 = ac.rel(gk, g64[k]), ac.rel(g32[k], g64[k])
        print(f"  {k:7s} |g| {np.linalg.norm(g64[k]):.3e}  gpu-vs-fp64 {e_gpu:.2e}  fp32-oracle-vs-fp64 {e_32:.2e}")
        assert np.isfinite(gk).all()
        assert e_gpu <= max(1e-4, 4 * e_32), k


# Rope-rope contact scenes (tests/adjoint_cases.rope_crossing; the oracle adjoint is pinned on
# them by FP64 finite differences in test_adjoint_oracle.py): (scene, dt, substeps, frames,
# program spread). "resting_crossing": rope 1 settles on rope 0 inside the barrier band (192
# active pair terms); "clipped_crossing": rope 1 starts 7 mm above rope 0 and steps of h = 1/60
# are clipped by the step limit (51 of them, at the padding bound) while 40 pair terms act. The
# limit's other bound (a candidate's distance) binds only in scenes whose FP64 gradient itself
# moves by 0.3% .. 100% when the start state moves by 1e-8 m (e.g. a rope dropped onto a pinned
# one), where FP32 cannot be compared; it is pinned by FP64 finite differences on the CPU. The
# loss adds a seeded linear term of the final state to the tip loss (rope 0's tip is pinned).
# The pair shares of the other segment are summed with shared-memory atomics, so these
# gradients are reproducible to rounding, not bitwise.
ROPE_SCENES = {
    "resting_crossing": (dict(damping=0.0), 1 / 300, 20, 3, dict(v_std=0.05, p_std=0.001)),
    "clipped_crossing": (dict(gap=0.007, damping=0.0), 1 / 60, 1, 4, dict(v_std=0.3, p_std=0.01)),
}


@pytest.mark.parametrize("engine", ["persistent", "plain", "oversize_group"])
@pytest.mark.parametrize("kind", list(ROPE_SCENES))
def test_rope_contact_adjoint_matches_fp64_oracle(kind, engine):
    """Rope-rope contact through the CTA-resident adjoint (persistent), the per-launch adjoint
    after plain frames (plain), and the per-launch adjoint that a contact group larger than one
    CTA takes by itself (oversize_group: ten crossings of 52-vertex ropes in one group of
    20 ropes, 1040 vertices)."""
    import torch

    import ropesim.grad as rg

    kw, dt, S_, F_, pk = ROPE_SCENES[kind]
    Rr, Vr = 2, 10
    if engine == "oversize_group":
        Vr = 52
        kw = dict(kw, pairs=10)
        Rr = 20
    ob, pos = ac.rope_crossing(V=Vr, **kw)
    progs = ac.programs(pos, F_, **pk)
    tgt = ac.targets(pos, F_)
    wr = np.random.default_rng(7)
    w_end = (1e-2 * wr.standard_normal((Rr * Vr, 3)), 1e-3 * wr.standard_normal((Rr * Vr, 3)))
    L64, g64 = ac.oracle_loss_and_grad(ob, progs, tgt, dt, S_, Vr, w_end=w_end)
    ob32, _ = ac.rope_crossing(V=Vr, precision="f32", **kw)
    L32, g32 = ac.oracle_loss_and_grad(ob32, progs, tgt, dt, S_, Vr, w_end=w_end)
    b, _ = ac.rope_crossing(V=Vr, backend="cuda", **kw)
    if engine == "plain":
        b.set_engine("plain")
    st = [t.clone().requires_grad_() for t in rg.state(b)]
    par = [t.clone().requires_grad_() for t in rg.parameters(b)]
    P = [torch.tensor(a, device="cuda", requires_grad=True) for a in progs]
    tg = torch.tensor(tgt, device="cuda", dtype=torch.float32)
    cur, loss = st, 0.0
    for f in range(F_):
        cur = rg.frame(b, cur, par, P[0][f], P[1][f], P[2][f], dt, S_)
        tip = cur[0].view(Rr, Vr, 3)[:, -1]
        loss = loss + ((tip - tg[f]) ** 2).sum(-1).mean()
    Wx, Wv = (torch.tensor(w, device="cuda", dtype=torch.float32) for w in w_end)
    loss = loss + (Wx * cur[0]).sum() + (Wv * cur[1]).sum()
    loss.backward()
    g = {"g_p0": P[0].grad, "g_v0": P[1].grad, "g_p1": P[2].grad, "g_ea": par[0].grad, "g_ei": par[1].grad,
         "g_mass": par[2].grad, "g_pos": st[0].grad, "g_vel": st[1].grad, "g_lvel": st[2].grad, "g_q": st[3].grad}
    g = {k: v.detach().cpu().numpy().astype(np.float64) for k, v in g.items()}
    L = float(loss.detach())
    print(f"\n  [{kind}, {engine}] loss gpu {L:.8e} fp64 {L64:.8e} fp32-oracle {L32:.8e}")
    assert abs(L - L64) <= max(1e-4 * abs(L64), 4 * abs(L32 - L64))
    for k in GROUPS:
        if np.linalg.norm(g64[k]) == 0.0:  # one substep: v0 cancels from the root's velocity exactly
            assert np.abs(g[k]).max() <= 1e-6 * np.linalg.norm(g64["g_p1"]), k
            continue
        e_gpu = ac.rel(g[k], g64[k])
        e_32 = ac.rel(g32[k], g64[k])
        print(f"  {k:7s} |g| {np.linalg.norm(g64[k]):.3e}  gpu-vs-fp64 {e_gpu:.2e}  fp32-oracle-vs-fp64 {e_32:.2e}")
        assert np.isfinite(g[k]).all()
        assert e_gpu <= max(1e-4, 4 * e_32), k
