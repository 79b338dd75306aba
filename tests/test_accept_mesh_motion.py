"""Kinematic (moving) meshes and the contact-force readout: the reference's mesh-motion acceptance
suite (tests/test_mesh_motion.py of the reference) restated over both backends.

A pose given to set_mesh_pose(s) is the pose at the END of the next step: the mesh moves there
over the substeps at constant linear and angular velocity, and friction acts on the rope's motion
relative to the moving surface; teleport=True replaces the pose at once. enable_contact_forces()
averages, per step, the force every surface applied to each vertex and the wrench the rope
applied to each mesh. Same rope as the mesh-contact suite (21 x 5 cm, h = 1/6000 s, 16 itr).
"""
import numpy as np
import pytest

from backends import P, Vel, dev, host, module
from conftest import BACKENDS

NV, SEG, RHO, EA, EI = 21, 0.05, 0.117, 11473.0, 4.48e-3
R = 0.00635
H, ITR, G = 1.0 / 6000.0, 16, 9.81
KAPPA, VSLIP = 2.0, 1e-3
PEN0 = G * H * H / KAPPA ** 2
DT, SUB = 1 / 60, 100
Q0 = np.array([0, 0, 0, 1], np.float32)


def slab(spacing=1 / 128, lo=(-0.3125, -0.6, -0.1875), hi=(1.3125, 0.6, 0.1875)):
    """A slab whose top face is the object plane z = 0 (object origin on the face)."""
    from ropesim import sdf

    return sdf.from_function(sdf.sdf_box((3.0, 3.0, 0.125), (0, 0, -0.125)), lo, hi, spacing)


def single_rope(backend, mu_s=0.5, mu_k=None):
    r = module(backend).RopeSim(num_verts=NV, seg_len=SEG, dir=np.array([1.0, 0, 0], np.float32), density=RHO,
                                k_stretch=EA, k_bend=EI, max_h=H, num_itr=ITR)
    r.damping = 0.0
    r.drag = 0.0
    r.set_gravity(np.array([0, 0, -G], np.float32))
    r.set_contact(radius=R, mu_s=mu_s, mu_k=mu_k, v_slip=VSLIP, kappa=KAPPA)
    r.unpin_root()
    return r


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


def quat_z(a):
    return np.array([0.0, 0.0, np.sin(a / 2), np.cos(a / 2)], np.float32)


# ------------------------------------------------------------------------------ interpolation


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("w", [0.01, 0.1])
def test_rising_floor_carries_the_rope_without_a_kick(backend, w):
    """A floor raised w per second (a pose per frame): the rope rides at w and keeps the resting
    sink PEN0 (at constant velocity the inertial term vanishes). A pose jump at the frame
    boundary instead would be an impact (0.67 m/s at 1 cm/s)."""
    r = single_rope(backend)
    r.add_mesh(*slab().as_args(), pos=np.array([0, 0, -0.02], np.float32))
    for _ in range(60):
        r.advance(DT, substeps=SUB)
    vmax, z = 0.0, -0.02
    for i in range(60):
        z = -0.02 + w * (i + 1) * DT
        r.set_mesh_pose(0, np.array([0, 0, z], np.float32), Q0)
        r.advance(DT, substeps=SUB)
        vmax = max(vmax, np.abs(host(r.velocities())).max())
    v, p = host(r.velocities()), host(r.positions())
    assert vmax < 1.3 * w + 1e-3
    assert np.allclose(v[:, 2], w, atol=0.02 * w + 1e-4)
    assert p[:, 2].min() == pytest.approx(z + R - PEN0, abs=2e-6)
    assert p[:, 2].max() == pytest.approx(z + R - PEN0, abs=2e-6)


@pytest.mark.parametrize("backend", BACKENDS)
def test_conveyor_carries_the_rope_only_with_friction(backend):
    """A slab translating at 0.2 m/s under a resting rope: with friction the rope goes along after
    slipping until it catches up (lag v^2 / (2 mu g) = 4.1 mm), without friction it stays."""
    v = 0.2
    out = {}
    for mu in (0.5, 0.0):
        b = ropes(backend, rows(1), mu_s=mu)
        b.add_mesh(*slab().as_args(), pos=np.array([0, 0, -0.02], np.float32))
        for _ in range(30):
            b.step_free(DT, SUB)
        x0 = P(b)[0].copy()
        for i in range(60):
            b.set_mesh_poses(0, np.array([v * (i + 1) * DT, 0, -0.02], np.float32), Q0)
            b.step_free(DT, SUB)
        out[mu] = (P(b)[0] - x0, Vel(b)[0])
    d, vel = out[0.5]
    assert np.allclose(vel[:, 0], v, atol=0.01 * v)
    assert np.allclose(d[:, 0], v * 1.0 - v * v / (2 * 0.5 * G), atol=1.5e-3)
    assert np.abs(d[:, 1:]).max() < 1e-4
    d, vel = out[0.0]
    assert np.abs(vel).max() < 1e-3
    assert np.abs(d).max() < 1e-3


@pytest.mark.parametrize("backend", BACKENDS)
def test_turntable_turns_the_rope(backend):
    """A slab spun about world z up to 0.5 rad/s (ramped over 0.5 s, so the rope never slips)
    under a rope offset from the axis: the rope follows the rigid rotation, its velocity
    omega x r (the surface velocity includes the angular part; the pose rotor per substep)."""
    om = 0.5
    b = ropes(backend, rows(1, y=0.3), mu_s=0.5)
    b.add_mesh(*slab(lo=(-0.3125, -0.3125, -0.1875), hi=(1.3125, 0.6, 0.1875)).as_args(),
               pos=np.array([0, 0, -0.02], np.float32))
    for _ in range(30):
        b.step_free(DT, SUB)
    x0 = P(b)[0].copy()
    th = 0.0
    for i in range(90):
        t1 = (i + 1) * DT
        th = om * (t1 * t1 if t1 < 0.5 else t1 - 0.25)
        b.set_mesh_poses(0, np.array([0, 0, -0.02], np.float32), quat_z(th))
        b.step_free(DT, SUB)
    c, s = np.cos(th), np.sin(th)
    expect = x0 @ np.array([[c, s, 0], [-s, c, 0], [0, 0, 1]])
    p, vel = P(b)[0], Vel(b)[0]
    assert np.abs(p - expect).max() < 3e-3
    assert np.allclose(vel[:, 0], -om * p[:, 1], atol=0.02 * om)
    assert np.allclose(vel[:, 1], om * p[:, 0], atol=0.02 * om)


@pytest.mark.parametrize("backend", BACKENDS)
def test_incline_slab_carries_the_rope_uphill(backend):
    """A 20-degree slab (posed) moving up its slope at 0.1 m/s with mu 0.5 > tan 20: the rope
    rides along at the slab's velocity (friction acts on the motion relative to the surface),
    after a start-up lag v^2 / 2a plus the creep the regularised law needs on the slope."""
    th = np.deg2rad(20.0)
    qy = np.array([0.0, np.sin(-th / 2), 0.0, np.cos(-th / 2)], np.float32)
    up = np.array([np.cos(th), 0.0, np.sin(th)])
    Rm = np.array([[np.cos(th), 0, np.sin(th)], [0, 1, 0], [-np.sin(th), 0, np.cos(th)]])
    pos = rows(1, z=0.0)[0] @ Rm + np.array([0, 0, R + 0.002])
    b = ropes(backend, pos[None], mu_s=0.5)
    b.add_mesh(*slab().as_args(), pos=np.zeros(3, np.float32), quat=qy)
    for _ in range(60):
        b.step_free(DT, SUB)
    p0 = P(b)[0].copy()
    v = 0.1
    for i in range(60):
        b.set_mesh_poses(0, (v * (i + 1) * DT * up).astype(np.float32), qy)
        b.step_free(DT, SUB)
    assert np.allclose(Vel(b)[0], v * up, atol=0.02 * v)
    lag = v * v / (2 * G * (0.5 * np.cos(th) - np.sin(th))) + VSLIP * np.tan(th) / 0.5
    d = P(b)[0] - p0
    assert np.allclose(d @ up, v - lag, atol=1.5e-3)
    assert np.abs(d @ np.array([-np.sin(th), 0.0, np.cos(th)])).max() < 2e-4


@pytest.mark.parametrize("backend", BACKENDS)
def test_step_path_interpolates_the_floor(backend):
    """RopeBatch.step (roots driven): a rope on a floor, root pinned at the resting height; floor
    and root rise together at 5 cm/s. The rope rides at that speed (no kick, sink PEN0) and
    translates rigidly."""
    z0 = -0.2
    pos = rows(1, z=z0 + R - PEN0)
    pin = np.zeros((1, NV), bool)
    pin[:, 0] = True
    b = ropes(backend, pos, pinned=pin)
    b.add_mesh(*slab().as_args(), pos=np.array([0, 0, z0], np.float32))
    root = pos[:, 0].astype(np.float32)
    zero = dev(backend, np.zeros((1, 3)))
    for _ in range(60):
        b.step(dev(backend, root), zero, DT, SUB)
    p0 = P(b)[0].copy()
    w, vmax = 0.05, 0.0
    wv = dev(backend, np.array([[0, 0, w]]))
    for i in range(60):
        z = z0 + w * (i + 1) * DT
        b.set_mesh_poses(0, np.array([0, 0, z], np.float32), Q0)
        b.step(dev(backend, root + np.array([0, 0, w * i * DT], np.float32)), wv, DT, SUB)
        vmax = max(vmax, np.abs(Vel(b)[0, 1:]).max())
    assert vmax < 1.3 * w
    assert P(b)[0, 1:, 2].min() == pytest.approx(z + R - PEN0, abs=2e-6)
    assert np.allclose(P(b)[0] - p0, [0, 0, w * 1.0], atol=1e-4)


@pytest.mark.parametrize("backend", BACKENDS)
def test_teleport_is_an_impact_interpolation_is_not(backend):
    """Both floors go up 1 cm in one frame; env 0 teleports (an impact: ejected at ~0.8 cm / h),
    env 1 interpolates (the floor moves at 0.6 m/s for a frame and the rope rides it)."""
    b = ropes(backend, rows(2))
    p = np.array([[0, 0, -0.02], [0, 0, -0.02]], np.float32)
    q = np.tile(Q0, (2, 1))
    b.add_mesh(*slab().as_args(), pos=p, quat=q)
    for _ in range(60):
        b.step_free(DT, SUB)
    p[:, 2] += 0.01
    b.set_mesh_poses(0, p, q, teleport=np.array([True, False]))
    b.step_free(DT, SUB)
    v = Vel(b)
    assert np.abs(v[0, :, 2]).max() > 10.0
    assert np.abs(v[1, :, 2]).max() < 1.0
    for _ in range(90):
        b.step_free(DT, SUB)
    assert P(b)[1, :, 2].min() == pytest.approx(-0.01 + R - PEN0, abs=3e-8)
    assert P(b)[0, :, 2].min() > 1.0  # still flying


@pytest.mark.parametrize("backend", BACKENDS)
def test_target_equal_to_the_pose_is_inert(backend):
    """set_mesh_poses with the pose the mesh already has leaves every step bitwise unchanged."""

    def run(call):
        b = ropes(backend, rows(1), drag=0.1)
        b.add_mesh(*slab().as_args(), pos=np.array([0, 0, -0.02], np.float32))
        for _ in range(30):
            if call:
                b.set_mesh_poses(0, np.array([0, 0, -0.02], np.float32), Q0)
            b.step_free(DT, SUB)
        return P(b)

    assert np.array_equal(run(False), run(True))


# ------------------------------------------------------------------------------ readout


@pytest.mark.parametrize("backend", BACKENDS)
def test_resting_rope_wrench_is_its_weight_at_the_centre_of_mass(backend):
    """A rope resting on a slab: the wrench on the mesh is the rope's weight applied at its centre
    of mass (torque about the mesh origin r_cm x F), and the per-vertex forces sum to +M g; on a
    plane instead the per-vertex readout still sees it, with no mesh wrench rows."""
    r = single_rope(backend)
    r.add_mesh(*slab().as_args(), pos=np.array([0, 0, -0.02], np.float32))
    r.enable_contact_forces()
    for _ in range(90):
        r.advance(DT, substeps=SUB)
    m = 1.0 / host(r.inv_masses())
    M = m.sum()
    x_cm = (m * host(r.positions())[:, 0]).sum() / M
    W = host(r.mesh_wrenches())
    assert W.shape == (1, 6)
    assert np.allclose(W[0, :3], [0, 0, -M * G], atol=2e-3 * M * G)
    assert np.allclose(W[0, 3:], [0, M * G * x_cm, 0], atol=2e-3 * M * G * x_cm)
    F = host(r.contact_forces())
    assert F.shape == (NV, 3)
    assert np.allclose(F.sum(0), [0, 0, M * G], atol=2e-3 * M * G)
    assert (F[:, 2] > 0).all()
    r2 = single_rope(backend)
    r2.set_planes(np.array([[0, 0, 1, -0.02]], np.float32), radius=R)
    r2.enable_contact_forces()
    for _ in range(90):
        r2.advance(DT, substeps=SUB)
    assert np.allclose(host(r2.contact_forces()).sum(0), [0, 0, M * G], atol=2e-3 * M * G)
    assert host(r2.mesh_wrenches()).shape == (0, 6)
    if backend == "cuda":
        r2.enable_contact_forces(False)
        with pytest.raises(ValueError):
            r2.contact_forces()


@pytest.mark.parametrize("backend", BACKENDS)
def test_belt_under_a_held_rope_sees_kinetic_friction(backend):
    """Root pinned (RopeBatch.step), a slab sliding away from the root at 0.2 m/s under the taut,
    still rope (slip >> v_slip): the wrench on the slab is the weight of the free vertices plus
    the sliding friction mu_k N against the belt's motion; the per-vertex forces are its
    reaction."""
    mu_k = 0.3
    pos = rows(1, z=-0.02 + R - PEN0)
    pin = np.zeros((1, NV), bool)
    pin[:, 0] = True
    b = ropes(backend, pos, pinned=pin, mu_s=0.5, mu_k=mu_k)
    b.add_mesh(*slab(lo=(-0.6, -0.6, -0.1875), hi=(1.3125, 0.6, 0.1875)).as_args(),
               pos=np.array([-0.25, 0, -0.02], np.float32))
    b.enable_contact_forces()
    root, zero = dev(backend, pos[:, 0]), dev(backend, np.zeros((1, 3)))
    for _ in range(60):
        b.step(root, zero, DT, SUB)
    v = 0.2
    for i in range(60):
        b.set_mesh_poses(0, np.array([-0.25 + v * (i + 1) * DT, 0, -0.02], np.float32), Q0)
        b.step(root, zero, DT, SUB)
    inv = host(b.inv_masses()).reshape(-1)
    Mf = (1.0 / inv[inv > 0]).sum()
    W = host(b.mesh_wrenches())
    assert W.shape == (1, 1, 6)
    assert W[0, 0, 2] == pytest.approx(-Mf * G, rel=0.02)
    assert W[0, 0, 0] == pytest.approx(mu_k * W[0, 0, 2], rel=0.01)
    assert abs(W[0, 0, 1]) < 1e-3 * Mf * G
    F = host(b.contact_forces()).reshape(1, NV, 3)
    assert F[0, 0].tolist() == [0, 0, 0]
    assert np.allclose(F[0].sum(0), -W[0, 0, :3], rtol=1e-5, atol=1e-6)
    assert np.abs(Vel(b)[0]).max() < 2e-3


@pytest.mark.gpu
def test_teleport_flag_validation():
    """teleport as a per-env mask must have one entry per env; a mask or a bool both work."""
    b = ropes("cuda", rows(2))
    b.add_mesh(*slab().as_args())
    with pytest.raises(ValueError):
        b.set_mesh_poses(0, np.zeros(3, np.float32), Q0, teleport=np.array([True]))
    b.set_mesh_poses(0, np.zeros(3, np.float32), Q0, teleport=np.array([True, False]))
    b.set_mesh_poses(0, np.zeros(3, np.float32), Q0, teleport=True)
