"""The reference's RopeBatch contract suites (tests/test_batch.py, test_rest_shape.py and
test_deterministic_sweeps.py of the reference) restated over both backends: the single-rope
RopeSim (itself checked by the physics suites) is the oracle of a batch env.

Contract: root commands arrive as contiguous float32 CUDA tensors; observations are device
buffers shared zero-copy through __cuda_array_interface__, refreshed in place after every step
and reset, and writes into them do not reach solver state; invalid inputs raise ValueError;
envs never talk to each other; reset_envs restores the listed envs exactly and leaves the others
bitwise untouched; the second-order program lands the root exactly on its end pose; the rest
shape is the given geometry unless straight_rest; fresh objects replay bitwise.
"""
import numpy as np
import pytest

from backends import P, Q, Vel, dev, host, module
from conftest import BACKENDS, G, H, make_rope

F32 = np.float32


def batch(backend, N=4, V=25, seg=0.02, roots=None, direction=(0, -1, 0), fix_root_orientation=False, drag=0.0, **kw):
    if roots is None:
        roots = np.zeros((N, 3), F32)
        roots[:, 0] = np.arange(N) * 1.5  # envs far apart
    args = dict(density=0.1, k_stretch=500.0, k_bend=1e-6, max_h=1.0 / 3000.0, num_itr=8)
    args.update(kw)
    b = module(backend).RopeBatch(N, V, roots.astype(F32), seg, np.asarray(direction, F32), args["density"],
                                  args["k_stretch"], args["k_bend"], args["max_h"], args["num_itr"],
                                  fix_root_orientation=fix_root_orientation)
    b.set_gravity(np.array([0.0, -G, 0.0], F32))
    b.drag = drag
    b.damping = 0.0
    return b, roots.astype(F32)


def wobble(t):
    return np.array([0.06 * np.sin(2 * np.pi * 0.7 * t), 0.02 * np.sin(2 * np.pi * 1.3 * t), 0.0])


def drive_batch_and_rope(backend, T=1.0, N=3, V=25):
    """Every env and a single RopeSim through the same root motion (per env offset by its root)."""
    b, roots = batch(backend, N=N, V=V)
    s = make_rope(backend, n=V, seg=0.02, direction=(0, -1, 0))  # root at the origin = env 0
    for k in range(int(round(T / H))):
        p0, p1 = wobble(k * H), wobble(k * H + H)
        vel = (p1 - p0) / H
        b.step(dev(backend, roots + p0), dev(backend, np.tile(vel, (N, 1))), H, 50)
        s.set_root(p0.astype(F32), vel.astype(F32))
        s.advance(H, substeps=50)
    return b, s, roots


@pytest.mark.parametrize("backend", BACKENDS)
def test_env0_is_the_single_rope(backend):
    b, s, _ = drive_batch_and_rope(backend)
    assert np.max(np.linalg.norm(P(b)[0] - host(s.positions()), axis=1)) < 1e-6


@pytest.mark.parametrize("backend", BACKENDS)
def test_envs_agree_up_to_their_root_translation(backend):
    b, _, roots = drive_batch_and_rope(backend)
    rel = P(b) - roots[:, None, :]
    for e in range(1, rel.shape[0]):
        assert np.max(np.linalg.norm(rel[e] - rel[0], axis=1)) < 1e-5


@pytest.mark.parametrize("backend", BACKENDS)
def test_a_whipped_env_does_not_touch_its_neighbour(backend):
    b, roots = batch(backend, N=2, V=25)
    for k in range(60):
        t = k * H
        pos, vel = roots.copy(), np.zeros((2, 3), F32)
        pos[1, 0] += 0.3 * np.sin(6 * np.pi * t)
        vel[1, 0] = (0.3 * np.sin(6 * np.pi * (t + H)) - 0.3 * np.sin(6 * np.pi * t)) / H
        b.step(dev(backend, pos), dev(backend, vel), H, 50)
    ref, _ = batch(backend, N=1, V=25, roots=roots[:1])
    for _ in range(60):
        ref.step(dev(backend, roots[:1]), dev(backend, np.zeros((1, 3))), H, 50)
    assert np.max(np.linalg.norm(P(b)[0] - P(ref)[0], axis=1)) < 1e-6


@pytest.mark.parametrize("backend", BACKENDS)
def test_partial_reset_envs(backend):
    b, roots = batch(backend, N=4, V=25)
    init = P(b).copy()
    vel = dev(backend, np.tile([0.2, 0, 0], (4, 1)))
    for k in range(30):
        b.step(dev(backend, roots + np.array([0.2 * (k * H), 0, 0], F32)), vel, H, 50)
    before = P(b).copy()
    b.reset_envs(np.array([1, 3], np.int32))
    after, v_after = P(b), Vel(b)
    np.testing.assert_allclose(after[[1, 3]], init[[1, 3]], atol=1e-6)
    np.testing.assert_allclose(v_after[[1, 3]], 0.0, atol=1e-7)
    np.testing.assert_array_equal(after[[0, 2]], before[[0, 2]])
    b.step(dev(backend, after[:, 0, :]), dev(backend, np.zeros((4, 3))), H, 50)
    assert np.isfinite(P(b)).all() and b.last_error == 0


@pytest.mark.gpu
def test_views_are_zero_copy_and_write_safe():
    """positions() is the device buffer itself (same pointer, refreshed by step); the quaternion
    view is a gathered copy, so vandalising it does not reach solver state."""
    import torch

    b, _ = batch("cuda", N=2, V=10)
    view = b.positions()
    t = torch.as_tensor(view)
    assert t.is_cuda and t.dtype == torch.float32 and tuple(t.shape) == (2, 10, 3)
    assert t.data_ptr() == view.ptr
    t0 = t.clone()
    b.step(dev("cuda", P(b)[:, 0, :]), dev("cuda", np.full((2, 3), 0.1)), H, 50)
    assert not torch.equal(t, t0)
    q = torch.as_tensor(b.quaternions())
    assert q.data_ptr() != 0 and tuple(q.shape) == (2, 10, 4)
    q.add_(99.0)
    b.gather()
    assert torch.all(torch.as_tensor(b.quaternions()) < 50.0)
    n = torch.linalg.vector_norm(q[:, :-1, :], dim=-1)
    assert torch.allclose(n, torch.ones_like(n), atol=1e-5)
    # the pointer stays the same across steps and resets
    b.reset_envs(np.array([0], np.int32))
    assert b.positions().ptr == view.ptr


@pytest.mark.gpu
def test_step_inputs_are_validated():
    import torch

    import ropesim

    b, roots = batch("cuda", N=2, V=10)
    ok_pos, ok_vel = dev("cuda", roots), dev("cuda", np.zeros((2, 3)))
    with pytest.raises(ValueError):
        b.step(torch.zeros(2, 3), ok_vel, H, 50)  # host tensor
    with pytest.raises(ValueError):
        b.step(dev("cuda", np.zeros((3, 3))), ok_vel, H, 50)  # wrong rows
    with pytest.raises(ValueError):
        b.step(torch.zeros(2, 3, device="cuda", dtype=torch.float64), ok_vel, H, 50)
    with pytest.raises(ValueError):
        b.step(torch.zeros(2, 6, device="cuda")[:, ::2], ok_vel, H, 50)  # non-contiguous
    with pytest.raises(ValueError):
        b.step(ok_pos, ok_vel, H, 0)
    with pytest.raises(ValueError):
        b.step(ok_pos, ok_vel, H, 50, root_q=torch.zeros(2, 4, device="cuda"))  # q without fixed roots
    with pytest.raises(ValueError):
        b.reset_envs(np.array([5], np.int32))
    with pytest.raises(ValueError):
        ropesim.RopeBatch(1, 4, np.zeros((1, 3), F32), k_bend=0.0)


@pytest.mark.parametrize("backend", BACKENDS)
def test_program_lands_exactly_on_its_end_pose(backend):
    """The last substep samples the program at tau = dt (position) and SLERP t = 1 (frame): the
    root lands on root_pos_end and root_q_end; its velocity is the last substep's midpoint
    sample v0 + a (dt - h/2)."""
    b, roots = batch(backend, N=3, V=10, fix_root_orientation=True)
    p1 = roots + np.array([0.04, -0.02, 0.03], F32)
    v0 = np.tile(np.array([0.5, 0.2, -0.1], F32), (3, 1))
    th = np.deg2rad([10.0, 20.0, 30.0])
    q0 = np.zeros((3, 4), F32)
    q0[:, 3] = 1.0
    q1 = np.zeros((3, 4), F32)
    q1[:, 2], q1[:, 3] = np.sin(th / 2), np.cos(th / 2)
    b.step(dev(backend, roots), dev(backend, v0), H, 50, root_q=dev(backend, q0), root_pos_end=dev(backend, p1),
           root_q_end=dev(backend, q1))
    np.testing.assert_allclose(P(b)[:, 0, :], p1, atol=2e-6)
    np.testing.assert_allclose(Q(b)[:, 0, :], q1, atol=1e-5)
    a = 2.0 * ((p1 - roots) - v0 * H) / H ** 2
    np.testing.assert_allclose(Vel(b)[:, 0, :], v0 + a * (H - (H / 50) / 2), rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("backend", BACKENDS)
def test_program_with_zero_acceleration_is_constant_velocity(backend):
    traj = lambda t: np.array([0.05 * np.sin(1.6 * np.pi * t), 0.0, 0.0])
    out = {}
    for mode in ("legacy", "program"):
        b, roots = batch(backend, N=1, V=25, drag=0.5)
        for k in range(60):
            p0 = (roots + traj(k * H)).astype(F32)
            p1 = (roots + traj(k * H + H)).astype(F32)
            v0 = (p1 - p0) / H
            if mode == "legacy":
                b.step(dev(backend, p0), dev(backend, v0), H, 50)
            else:
                b.step(dev(backend, p0), dev(backend, v0), H, 50, root_pos_end=dev(backend, p1))
        out[mode] = P(b)[0]
    assert np.max(np.linalg.norm(out["legacy"] - out["program"], axis=1)) < 1e-5


@pytest.mark.parametrize("backend", BACKENDS)
def test_program_tracks_better_than_constant_velocity(backend):
    """With the analytic start velocity, 60 Hz program driving tracks a 120 Hz run at the same
    substep h = 1/3000 better than 60 Hz constant-velocity driving (RMS over the whole rope)."""
    Rr, w = 0.06, 3 * np.pi
    p_of = lambda t: np.array([Rr * (np.cos(w * t) - 1.0), Rr * np.sin(w * t), 0.0])
    v_of = lambda t: np.array([-Rr * w * np.sin(w * t), Rr * w * np.cos(w * t), 0.0])

    def run(rate, substeps, mode):
        b, roots = batch(backend, N=1, V=25, drag=0.5)
        dt = 1.0 / rate
        every = int(rate // 60)
        snaps = []
        for k in range(int(1.5 * rate)):
            p0 = (roots + p_of(k * dt)).astype(F32)
            p1 = (roots + p_of(k * dt + dt)).astype(F32)
            if mode == "program":
                b.step(dev(backend, p0), dev(backend, v_of(k * dt)[None]), dt, substeps, root_pos_end=dev(backend, p1))
            else:
                b.step(dev(backend, p0), dev(backend, (p1 - p0) / dt), dt, substeps)
            if (k + 1) % every == 0:
                snaps.append(P(b)[0])
        return np.array(snaps)

    ref = run(120.0, 25, "program")
    d_prog = np.sqrt(np.mean(np.sum((run(60.0, 50, "program") - ref) ** 2, axis=-1)))
    d_leg = np.sqrt(np.mean(np.sum((run(60.0, 50, "legacy") - ref) ** 2, axis=-1)))
    assert d_prog < d_leg


@pytest.mark.parametrize("backend", BACKENDS)
def test_slerped_frames_do_not_add_strain(backend):
    """A clamped root turned 90 degrees over 0.5 s: SLERPed frames stress the rod no more than
    frames stepped once per frame (both near the FP32 noise floor at this rate)."""

    def peak_strain(slerped):
        b, roots = batch(backend, N=1, V=16, direction=(1, 0, 0), fix_root_orientation=True, k_stretch=2000.0,
                         k_bend=0.4, density=0.05)
        b.drag = 1.0
        zeros = dev(backend, np.zeros((1, 3)))
        worst, q_prev = 0.0, np.array([[0, 0, 0, 1]], F32)
        for k in range(30):
            th = np.deg2rad(90.0) * (k + 1) / 30
            q = np.array([[0, 0, np.sin(th / 2), np.cos(th / 2)]], F32)
            if slerped:
                b.step(dev(backend, roots), zeros, H, 50, root_q=dev(backend, q_prev), root_pos_end=dev(backend, roots),
                       root_q_end=dev(backend, q))
            else:
                b.step(dev(backend, roots), zeros, H, 50, root_q=dev(backend, q))
            q_prev = q
            lens = np.linalg.norm(np.diff(P(b)[0], axis=0), axis=1)
            worst = max(worst, float(np.max(np.abs(lens - 0.02) / 0.02)))
        return worst

    s_slerp, s_step = peak_strain(True), peak_strain(False)
    assert s_slerp <= max(s_step * 1.5, 5e-3)
    assert s_slerp < 0.10


@pytest.mark.parametrize("backend", BACKENDS)
def test_commanded_root_frames_hold(backend):
    b, roots = batch(backend, N=3, V=16, direction=(1, 0, 0), fix_root_orientation=True, k_stretch=2000.0, k_bend=0.4,
                     density=0.05)
    b.drag = 1.0
    th = np.deg2rad([5.0, 15.0, 25.0])
    q = np.zeros((3, 4), F32)
    q[:, 2], q[:, 3] = np.sin(th / 2), np.cos(th / 2)
    for _ in range(120):
        b.step(dev(backend, roots), dev(backend, np.zeros((3, 3))), H, 50, root_q=dev(backend, q))
    np.testing.assert_allclose(Q(b)[:, 0, :], q, atol=1e-5)
    assert np.isfinite(P(b)).all()


# ------------------------------------------------------------------------------ rest shape


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("straight", [False, True])
def test_rest_shape_is_the_given_geometry_unless_straight(backend, straight):
    """A right-angle fold (10 segments down, 10 along +x, 5 cm each) without gravity: as the rest
    shape it stays folded; with straight_rest the fold is strain and the rope unfolds."""
    V, L = 21, 0.05
    pos = np.zeros((2, V, 3), F32)
    for v in range(V):
        pos[:, v] = (0.0, 0.0, -v * L) if v <= 10 else ((v - 10) * L, 0.0, -10 * L)
    b = module(backend).RopeBatch.from_positions(pos, 0.1, 500.0, 1e-2, 1 / 3000, 8, straight_rest=straight)
    b.set_gravity(np.zeros(3, F32))
    b.drag = 1.0
    root, zero = dev(backend, pos[:, 0]), dev(backend, np.zeros((2, 3)))
    for _ in range(360):
        b.step(root, zero, 1 / 60, 50)
    p = P(b)
    end = np.linalg.norm(p[:, -1] - p[:, 0], axis=-1)
    full = (V - 1) * L
    if straight:
        assert np.all(end > 0.9 * full), end
    else:
        assert np.all(end < 0.8 * full), end


# ------------------------------------------------------------------------------ replay


@pytest.mark.gpu
@pytest.mark.parametrize("strings,vertices,iterations", [(1, 3, 3), (1, 63, 3), (1, 64, 3), (1, 127, 3), (1, 128, 3),
                                                         (6, 124, 3), (6, 124, 24)])
def test_fresh_objects_replay_bitwise(strings, vertices, iterations):
    """Moving, endpoint-pinned strings: two fresh batches fed the same commands agree bit for bit
    at every frame (positions, velocities, frames), whatever the rope length against the CTA."""
    dt, substeps = 1 / 480, 32
    u = np.linspace(0, 1, vertices, dtype=F32)
    init = np.zeros((strings, vertices, 3), F32)
    init[:, :, 0] = 0.64 * u
    init[:, :, 1] = np.arange(strings)[:, None] * 0.009
    init[:, :, 2] = (0.002 + 0.001 * np.arange(strings)[:, None]) * np.sin(u * np.pi)
    pins = np.zeros(init.shape[:2], bool)
    pins[:, [0, -1]] = True
    roots = init[:, 0].copy()
    program = []
    for step in range(16):
        start, end = roots.copy(), roots.copy()
        start[:, 0] -= 1e-5 * step
        end[:, 0] -= 1e-5 * (step + 1)
        program.append(tuple(dev("cuda", x) for x in (start, (end - start) / dt, end)))

    def run():
        import ropesim

        b = ropesim.RopeBatch.from_positions(init, 0.005, 7500.0, 1e-7, dt / substeps, iterations, pinned=pins,
                                             straight_rest=True, deterministic=True)
        b.set_gravity(np.array([0, 0, -9.81], F32))
        b.damping = 0.0
        b.drag = 20.0
        states = []
        for start, vel, end in program:
            b.step(start, vel, dt, substeps, root_pos_end=end)
            st = tuple(host(f()).astype(F32) for f in (b.positions, b.velocities, b.quaternions))
            assert all(np.isfinite(a).all() for a in st)
            states.append(st)
        return states

    first, second = run(), run()
    assert not np.array_equal(first[-1][0][:, 1:-1], init[:, 1:-1])
    for a, c in zip(first, second):
        for x, y in zip(a, c):
            np.testing.assert_array_equal(x.view(np.uint32), y.view(np.uint32))
