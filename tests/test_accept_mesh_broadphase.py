"""Many meshes per sim: the reference's broad-phase acceptance suite (tests/test_mesh_broadphase.py
of the reference) restated over both backends: the per-vertex candidate list rebuilt every
substep from world boxes, the 64-mesh capacity, the fall-back to scanning every mesh past 8
candidates, per-mesh friction, poses from CUDA tensors and the device views of the readout.
Same rope as the mesh-contact suite (21 x 5 cm, h = 1/6000 s, 16 itr).
"""
import numpy as np
import pytest

from backends import P, Vel, host, module
from conftest import BACKENDS

NV, SEG, RHO, EA, EI = 21, 0.05, 0.117, 11473.0, 4.48e-3
R = 0.00635
H, ITR, G = 1.0 / 6000.0, 16, 9.81
KAPPA, VSLIP = 2.0, 1e-3
PEN0 = G * H * H / KAPPA ** 2
DT, SUB = 1 / 60, 100
Q0 = np.array([0, 0, 0, 1], np.float32)


def slab(spacing=1 / 128, lo=(-0.3125, -0.6, -0.1875), hi=(1.3125, 0.6, 0.1875)):
    from ropesim import sdf

    return sdf.from_function(sdf.sdf_box((3.0, 3.0, 0.125), (0, 0, -0.125)), lo, hi, spacing)


def ropes(backend, pos, pinned=None, mu_s=0.5, mu_k=None, drag=0.0):
    pos = np.asarray(pos, np.float32)
    pin = np.zeros(pos.shape[:2], bool) if pinned is None else pinned
    b = module(backend).RopeBatch.from_positions(pos, RHO, EA, EI, H, ITR, pinned=pin)
    b.damping = 0.0
    b.drag = drag
    b.set_gravity(np.array([0, 0, -G], np.float32))
    b.set_contact(radius=R, mu_s=mu_s, mu_k=mu_k, v_slip=VSLIP, kappa=KAPPA)
    return b


def rows(n, z=0.02, y=0.0):
    pos = np.zeros((n, NV, 3))
    pos[:, :, 0] = np.arange(NV) * SEG
    pos[:, :, 1] = y
    pos[:, :, 2] = z
    return pos


def cuda(a, dtype=None):
    import torch

    return torch.as_tensor(np.ascontiguousarray(a), device="cuda") if dtype is None else \
        torch.as_tensor(np.ascontiguousarray(a), device="cuda", dtype=dtype)


# ------------------------------------------------------------------------------ broad phase / cap


@pytest.mark.parametrize("backend", BACKENDS)
def test_far_meshes_never_enter(backend):
    """24 meshes, the rope's floor is mesh 20 and the other 23 sit 5 m away: the sink is the
    one-mesh value and the result is bitwise the one-mesh run (far meshes never become
    candidates)."""
    g = slab()

    def run(many):
        b = ropes(backend, rows(1), drag=0.1)
        if many:
            for m in range(24):
                b.add_mesh(*g.as_args(), pos=np.array([0, 0, -0.02] if m == 20 else [5.0 + m, 5.0, -0.02], np.float32))
        else:
            b.add_mesh(*g.as_args(), pos=np.array([0, 0, -0.02], np.float32))
        for _ in range(60):
            b.step_free(DT, SUB)
        return P(b)

    one, many = run(False), run(True)
    assert one[0, :, 2].min() == pytest.approx(-0.02 + R - PEN0, abs=3e-8)
    assert np.array_equal(one, many)


@pytest.mark.parametrize("backend", BACKENDS)
def test_more_than_eight_candidates_scan_every_mesh(backend):
    """Coincident floors share the weight: two give PEN0 / 2; ten (more than the 8 candidate
    slots, so the vertex scans every mesh) give PEN0 / 10."""
    g = slab()

    def sink(n):
        b = ropes(backend, rows(1), drag=0.1)
        for _ in range(n):
            b.add_mesh(*g.as_args(), pos=np.array([0, 0, -0.02], np.float32))
        for _ in range(60):
            b.step_free(DT, SUB)
        return -0.02 + R - P(b)[0, :, 2].min()

    assert sink(2) == pytest.approx(PEN0 / 2, rel=0.05)
    assert sink(10) == pytest.approx(PEN0 / 10, rel=0.1)


@pytest.mark.gpu
def test_mesh_slot_63_and_per_env_wrenches():
    """The 64th mesh (slot 63) holds both envs' ropes; a 65th is refused; the wrench rows of the
    63 far meshes stay exactly zero; the view equals the host readout; packed all-mesh pose
    updates move env 1's floor."""
    g = slab(spacing=1 / 32)
    pos = rows(2, z=R - PEN0)
    pos[1, :, 1] = 2.0
    b = ropes("cuda", pos)
    tr = np.zeros((2, 64, 3), np.float32)
    tr[:, :63, 0] = 5.0
    tr[1, 63, 1] = 2.0
    quats = np.tile(Q0, (2, 64, 1))
    for m in range(64):
        assert b.add_mesh(*g.as_args(), pos=tr[:, m], quat=quats[:, m]) == m
    with pytest.raises(ValueError):
        b.add_mesh(*g.as_args(), pos=np.array([0, 0, -40.0], np.float32))
    b.enable_contact_forces()
    for _ in range(20):
        b.step_free(DT, SUB)
    W = host(b.mesh_wrenches())
    np.testing.assert_array_equal(W[:, :63], 0.0)
    mass = (1.0 / host(b.inv_masses())).sum(axis=1)
    np.testing.assert_allclose(W[:, 63, 2], -mass * G, rtol=2e-3)
    np.testing.assert_array_equal(host(b.mesh_wrenches_view()), W)
    for i in range(10):
        tr[1, 63, 2] = (i + 1) * 0.001
        b.set_mesh_poses_all(tr, quats)
        b.step_free(DT, SUB)
    np.testing.assert_allclose(P(b)[0, :, 2], R - PEN0, atol=1e-6)
    np.testing.assert_allclose(P(b)[1, :, 2], R - PEN0 + 0.01, atol=5e-5)
    W = host(b.mesh_wrenches())
    np.testing.assert_array_equal(W[:, :63], 0.0)
    assert np.all(W[:, 63, 2] < 0)


@pytest.mark.parametrize("backend", BACKENDS)
def test_mesh_arrives_lifts_the_tail_and_leaves(backend):
    """A slab far below a hanging rope rises (fast while far, then 0.2 m/s), lifts the tail 5 cm,
    and goes back down: the broad phase admits it on arrival and drops it after; the tail rests
    on it while there and hangs free before and after. The hanging rope carries a 0.1 mm lateral
    imperfection: lifted by its tail, a perfectly straight vertical rope is an unstable but exact
    equilibrium that deterministic sweeps keep (the tail then stays 1.5 mm into the contact band,
    held by the rope's axial stiffness); the reference's racing sweeps break the symmetry
    themselves."""
    pos = np.stack([np.zeros(NV), np.zeros(NV), 0.55 - np.arange(NV) * SEG], -1)
    pos[1:, 0] += 1e-4 * np.sin(np.arange(1, NV))
    pin = np.zeros((1, NV), bool)
    pin[:, 0] = True
    b = ropes(backend, pos[None], pinned=pin, drag=0.5)
    b.add_mesh(*slab().as_args(), pos=np.array([0, 0, -3.0], np.float32))
    for _ in range(60):
        b.step_free(DT, SUB)
    assert P(b)[0, -1, 2] == pytest.approx(-0.45, abs=1e-3)

    def top(i):
        return -3.0 + 2.4 * min(1.0, i / 30) if i <= 30 else min(-0.4, -0.6 + 0.2 * (i - 30) * DT)

    for i in range(1, 150):
        b.set_mesh_poses(0, np.array([0, 0, top(i)], np.float32), Q0)
        b.step_free(DT, SUB)
    z = P(b)[0, :, 2].min()
    assert -0.4 + R - PEN0 - 1e-5 < z < -0.4 + R + 2e-4
    for i in range(1, 150):
        b.set_mesh_poses(0, np.array([0, 0, max(-3.0, -0.4 - 2.6 * i / 60)], np.float32), Q0)
        b.step_free(DT, SUB)
    assert P(b)[0, -1, 2] == pytest.approx(-0.45, abs=5e-3)


# ------------------------------------------------------------------------------ per-mesh friction


@pytest.mark.parametrize("backend", BACKENDS)
def test_friction_is_per_mesh(backend):
    """Two 20-degree slabs in one sim: mu 0.5 holds (tan 20 = 0.36), mu 0.1 lets the rope slide;
    set_mesh_friction changes it later; an out-of-range index is refused (product)."""
    th = np.deg2rad(20.0)
    qy = np.array([0.0, np.sin(-th / 2), 0.0, np.cos(-th / 2)], np.float32)
    Rm = np.array([[np.cos(th), 0, np.sin(th)], [0, 1, 0], [-np.sin(th), 0, np.cos(th)]])
    base = rows(1, z=0.0)[0] @ Rm + np.array([0, 0, R + 0.002])
    pos = np.stack([base + [0, 0.5, 0], base + [0, -0.5, 0]])
    b = ropes(backend, pos, mu_s=0.5)
    g = slab()
    b.add_mesh(*g.as_args(), pos=np.array([[0, 0.5, 0], [0, 0.5, 0]], np.float32), quat=np.tile(qy, (2, 1)))
    b.add_mesh(*g.as_args(), pos=np.array([[0, -0.5, 0], [0, -0.5, 0]], np.float32), quat=np.tile(qy, (2, 1)), mu_s=0.1)
    for _ in range(90):
        b.step_free(DT, SUB)
    p = P(b)
    assert np.abs(p[0] - pos[0]).max() < 2e-3
    assert p[1, :, 0].mean() - pos[1, :, 0].mean() < -0.3
    b.set_mesh_friction(1, 0.5)
    if backend == "cuda":
        with pytest.raises(ValueError):
            b.set_mesh_friction(5, 0.5)


# ------------------------------------------------------------------------------ device poses / views


@pytest.mark.gpu
def test_cuda_pose_targets_match_the_host_path():
    """set_mesh_poses from CUDA tensors (pos [N, 3], quat [N, 4], teleport [N] bool) gives the
    host path's trajectory (bitwise here: the sweeps are deterministic)."""
    import torch

    v = 0.2

    def run(on_device):
        b = ropes("cuda", rows(2), mu_s=0.5)
        b.add_mesh(*slab().as_args(), pos=np.array([0, 0, -0.02], np.float32))
        for _ in range(30):
            b.step_free(DT, SUB)
        for i in range(60):
            p = np.array([[v * (i + 1) * DT, 0, -0.02]] * 2, np.float32)
            q = np.tile(Q0, (2, 1))
            t = np.array([False, i == 10])  # env 1 teleports once
            if on_device:
                b.set_mesh_poses(0, cuda(p), cuda(q), cuda(t, torch.bool))
            else:
                b.set_mesh_poses(0, p, q, t)
            b.step_free(DT, SUB)
        return P(b)

    a, c = run(False), run(True)
    assert np.array_equal(a, c)
    assert np.allclose(a[0, :, 0] - rows(1)[0, :, 0], v * 1.0 - v * v / (2 * 0.5 * G), atol=1.5e-3)


@pytest.mark.gpu
def test_cuda_pose_target_validation():
    import torch

    b = ropes("cuda", rows(2))
    b.add_mesh(*slab(spacing=1 / 32).as_args())
    p = torch.zeros((2, 3), device="cuda")
    q = torch.tensor([[0, 0, 0, 1.0]] * 2, device="cuda")
    b.set_mesh_poses(0, p, q)
    b.set_mesh_poses(0, p, q, teleport=True)
    with pytest.raises(ValueError):
        b.set_mesh_poses(0, p, np.zeros((2, 4), np.float32))  # host and device rows mixed
    b.set_mesh_poses(0, p, q, teleport=np.array([True, False]))  # host flags with device poses
    with pytest.raises(ValueError):
        b.set_mesh_poses(0, p.double(), q)
    with pytest.raises(ValueError):
        b.set_mesh_poses(0, torch.zeros((3, 3), device="cuda"), q)


@pytest.mark.gpu
def test_force_views_match_the_readouts():
    """contact_forces_view / mesh_wrenches_view are the device buffers behind the host readouts:
    [N, V, 3] and [N, 64, 6], equal to contact_forces() / mesh_wrenches(), unused rows zero."""
    b = ropes("cuda", rows(2, z=-0.02 + R - PEN0))
    b.add_mesh(*slab().as_args(), pos=np.array([0, 0, -0.02], np.float32))
    b.enable_contact_forces()
    for _ in range(30):
        b.step_free(DT, SUB)
    W, F = host(b.mesh_wrenches()), host(b.contact_forces())
    Wv, Fv = host(b.mesh_wrenches_view()), host(b.contact_forces_view())
    assert Wv.shape == (2, 64, 6) and Fv.shape == (2, NV, 3)
    assert np.array_equal(Wv[:, 0], W[:, 0]) and np.array_equal(Fv, F)
    assert np.abs(Wv[:, 1:]).max() == 0.0
    M = (1.0 / host(b.inv_masses())[0]).sum()
    assert np.allclose(W[:, 0, 2], -M * G, rtol=2e-3)


@pytest.mark.gpu
def test_all_mesh_poses_in_one_call_match_per_mesh_calls():
    """set_mesh_poses_all(pos [N, M, 3], quat [N, M, 4], teleport) == M calls of set_mesh_poses,
    from host arrays and from CUDA tensors; M must equal the mesh count."""
    import torch

    v = 0.2

    def run(mode):
        b = ropes("cuda", rows(2), mu_s=0.5)
        g = slab()
        b.add_mesh(*g.as_args(), pos=np.array([0, 0, -0.02], np.float32))
        b.add_mesh(*g.as_args(), pos=np.array([0, 0, -3.0], np.float32))
        for _ in range(20):
            b.step_free(DT, SUB)
        for i in range(30):
            Pm = np.zeros((2, 2, 3), np.float32)
            Pm[:, 0] = [v * (i + 1) * DT, 0, -0.02]
            Pm[:, 1] = [0, 0, -3.0]
            Qm = np.tile(Q0, (2, 2, 1))
            if mode == "per":
                for m in range(2):
                    b.set_mesh_poses(m, Pm[:, m], Qm[:, m])
            elif mode == "host":
                b.set_mesh_poses_all(Pm, Qm)
            else:
                b.set_mesh_poses_all(cuda(Pm), cuda(Qm), torch.zeros(2, dtype=torch.bool, device="cuda"))
            b.step_free(DT, SUB)
        return P(b)

    a, h, d = run("per"), run("host"), run("cuda")
    assert np.array_equal(a, h) and np.array_equal(a, d)
    assert np.allclose(a[0, :, 0] - rows(1)[0, :, 0], v * 0.5 - v * v / (2 * 0.5 * G), atol=1.5e-3)
    b = ropes("cuda", rows(2))
    b.add_mesh(*slab(spacing=1 / 32).as_args())
    with pytest.raises(ValueError):
        b.set_mesh_poses_all(np.zeros((2, 2, 3), np.float32), np.zeros((2, 2, 4), np.float32))


# ------------------------------------------------------------------------------ pending targets


@pytest.mark.parametrize("backend", BACKENDS)
def test_add_mesh_keeps_pending_targets(backend):
    """add_mesh after set_mesh_poses does not turn the other mesh's pending target into a
    teleport: the rope rides the 1 cm lift instead of being ejected."""

    def run(add_between):
        b = ropes(backend, rows(1), drag=0.1)
        b.add_mesh(*slab().as_args(), pos=np.array([0, 0, -0.02], np.float32))
        for _ in range(30):
            b.step_free(DT, SUB)
        b.set_mesh_poses(0, np.array([0, 0, -0.01], np.float32), Q0)
        if add_between:
            b.add_mesh(*slab(spacing=1 / 32).as_args(), pos=np.array([0, 0, -5.0], np.float32))
        b.step_free(DT, SUB)
        return np.abs(Vel(b)[0, :, 2]).max()

    assert run(False) < 0.7 and run(True) < 0.7


@pytest.mark.parametrize("backend", BACKENDS)
def test_advance_zero_keeps_the_target_pending(backend):
    """RopeSim.advance(0) runs nothing and does not commit a pending mesh target."""
    r = module(backend).RopeSim(num_verts=NV, seg_len=SEG, dir=np.array([1.0, 0, 0], np.float32), density=RHO,
                                k_stretch=EA, k_bend=EI, max_h=H, num_itr=ITR)
    r.damping = 0.0
    r.drag = 0.1
    r.set_gravity(np.array([0, 0, -G], np.float32))
    r.set_contact(radius=R, mu_s=0.5, v_slip=VSLIP, kappa=KAPPA)
    r.unpin_root()
    r.add_mesh(*slab().as_args(), pos=np.array([0, 0, -0.02], np.float32))
    for _ in range(30):
        r.advance(DT, substeps=SUB)
    r.set_mesh_pose(0, np.array([0, 0, -0.01], np.float32), Q0)
    r.advance(0.0, substeps=SUB)
    r.advance(DT, substeps=SUB)
    assert np.abs(host(r.velocities())[:, 2]).max() < 0.7


@pytest.mark.parametrize("backend", BACKENDS)
def test_fast_mesh_is_caught_by_the_broad_phase(backend):
    """A slab arriving at 6 m/s (10 cm per frame, 1 mm per substep) from far below a rope resting
    on a plane is admitted in time (the padding includes the mesh's own travel) and lifts it."""
    b = ropes(backend, rows(1, z=0.3 + R - PEN0), drag=0.3)
    b.set_planes(np.array([[0, 0, 1.0, 0.3]], np.float32), radius=R)
    b.add_mesh(*slab().as_args(), pos=np.array([0, 0, -6.0], np.float32))
    for _ in range(10):
        b.step_free(DT, SUB)
    for i in range(80):
        b.set_mesh_poses(0, np.array([0, 0, min(0.31, -6.0 + 6.0 * (i + 1) * DT)], np.float32), Q0)
        b.step_free(DT, SUB)
    for _ in range(60):
        b.step_free(DT, SUB)
    assert P(b)[0, :, 2].min() == pytest.approx(0.31 + R - PEN0, abs=5e-5)
