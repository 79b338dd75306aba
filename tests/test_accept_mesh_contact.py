"""Rope-mesh contact through signed-distance lattices: the reference's mesh-contact acceptance
suite (tests/test_mesh_contact.py of the reference) restated over both backends: the FP64 oracle
on the CPU and the product on the GPU.

Known answers: on a box's top face the lattice is exactly the plane z, so the mesh path must
reproduce the plane path; a posed box is an incline (Coulomb stick / slide at g (sin - mu cos));
a rope over a cylinder holds iff the capstan ratio exp(mu pi) exceeds the load ratio; drapes over
a sphere and into a bowl never enter the surface; a thin wall stops an 8 m/s rope; per-env poses
keep envs independent; a mesh the rope never reaches is bitwise inert.

Rope: 21 vertices x 5 cm, rho 0.117 kg/m, EA 11473 N, EI 4.48e-3 N m^2, contact radius 6.35 mm,
h = 1/6000 s, 16 iterations, kappa = 2 (the reference's rope_A fit).
"""
import numpy as np
import pytest

from backends import P, Vel, dev, host, module
from conftest import BACKENDS

NV, SEG, RHO, EA, EI = 21, 0.05, 0.117, 11473.0, 4.48e-3
R = 0.00635
H, ITR, G = 1.0 / 6000.0, 16, 9.81
KAPPA, VSLIP = 2.0, 1e-3
PEN0 = G * H * H / KAPPA ** 2  # resting sink under the full weight: k = m (kappa/h)^2, pen = m g / k


def sdf():
    from ropesim import sdf as s

    return s


def rot_y(angle):
    """(quaternion (x, y, z, w), 3x3 matrix) of a rotation by `angle` about +y."""
    c, s = np.cos(angle), np.sin(angle)
    return (np.array([0.0, np.sin(angle / 2), 0.0, np.cos(angle / 2)], np.float32),
            np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]]))


def floor_lattice(spacing=1 / 128, x_hi=1.3125):
    """A box (half extents 3 x 1 x 0.125 m) whose top face is the object plane z = 0, the object
    origin on that face (the rest gap is tens of float32 steps of a centimetre-scale coordinate,
    so the frame origin has to sit near the surface); the lattice covers only the reachable part
    of the face, with float32-exact nodes."""
    s = sdf()
    return s.from_function(s.sdf_box((3.0, 1.0, 0.125), (0, 0, -0.125)), (-0.3125, -0.3125, -0.1875),
                           (x_hi, 0.3125, 0.1875), spacing)


def single_rope(backend, gravity=(0, 0, -G), mu_s=0.5, mu_k=None, num_itr=ITR, pinned=False):
    r = module(backend).RopeSim(num_verts=NV, seg_len=SEG, dir=np.array([1.0, 0, 0], np.float32), density=RHO,
                                k_stretch=EA, k_bend=EI, max_h=H, num_itr=num_itr)
    r.damping = 0.0
    r.drag = 0.0
    r.set_gravity(np.asarray(gravity, np.float32))
    r.set_contact(radius=R, mu_s=mu_s, mu_k=mu_k, v_slip=VSLIP, kappa=KAPPA)
    if not pinned:
        r.unpin_root()
    return r


def ropes_from(backend, pos, pinned=None, gravity=(0, 0, -G), mu_s=0.5, mu_k=None, drag=0.0):
    """A RopeBatch of explicit shapes [N, V, 3], every vertex free unless `pinned`."""
    pos = np.asarray(pos, np.float32)
    pin = np.zeros(pos.shape[:2], bool) if pinned is None else pinned
    b = module(backend).RopeBatch.from_positions(pos, RHO, EA, EI, H, ITR, pinned=pin)
    b.damping = 0.0
    b.drag = drag
    b.set_gravity(np.asarray(gravity, np.float32))
    b.set_contact(radius=R, mu_s=mu_s, mu_k=mu_k, v_slip=VSLIP, kappa=KAPPA)
    return b


def straight_rows(n, z, y_step=0.0):
    pos = np.zeros((n, NV, 3))
    pos[:, :, 0] = np.arange(NV) * SEG
    pos[:, :, 1] = y_step * np.arange(n)[:, None]
    pos[:, :, 2] = z
    return pos


# ------------------------------------------------------------------------------ floors


@pytest.mark.parametrize("backend", BACKENDS)
def test_box_top_face_is_the_plane(backend):
    """Resting on the box's top face (SDF = z there) gives the plane's answer: the penalty forces
    carry the weight, the sink is PEN0, and the two paths agree to rounding."""
    g = floor_lattice()
    w = -1 / 128  # the surface at z = w (float32-exact): the rope drops 1.5 mm and rests
    finals = []
    for mesh in (False, True):
        r = single_rope(backend)
        if mesh:
            r.add_mesh(*g.as_args(), pos=np.array([0, 0, w], np.float32))
        else:
            r.set_planes(np.array([[0.0, 0.0, 1.0, w]], np.float32), radius=R, mu_s=0.5, v_slip=VSLIP, kappa=KAPPA)
        for _ in range(60):
            r.advance(1 / 60, substeps=100)
        p = host(r.positions())
        m = 1.0 / host(r.inv_masses())
        pen = np.maximum(-(p[:, 2] - w - R), 0.0)
        assert (m * (KAPPA / H) ** 2 * pen).sum() / (m.sum() * G) == pytest.approx(1.0, abs=5e-3)
        assert pen.max() == pytest.approx(PEN0, rel=0.05)
        assert np.abs(host(r.velocities())).max() < 1e-3
        finals.append(p)
    assert np.abs(finals[0] - finals[1]).max() < 1e-6


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("mu,slides", [(0.5, False), (0.2, True)])
def test_posed_box_is_a_coulomb_incline(backend, mu, slides):
    """The box posed 20 degrees about y: its top face is an incline under vertical gravity. The
    rope sticks for mu 0.5 > tan 20 and slides at g (sin - mu cos) for mu 0.2."""
    th = np.radians(20.0)
    normal = np.array([np.sin(th), 0.0, np.cos(th)])
    down = np.array([np.cos(th), 0.0, -np.sin(th)])
    g = floor_lattice(x_hi=2.6875)  # the sliding rope travels ~1.3 m along the face
    q, Rm = rot_y(th)
    s = np.arange(NV) * SEG
    pos = s[:, None] * down[None] + (R - PEN0 * np.cos(th)) * normal[None]
    b = ropes_from(backend, pos[None], mu_s=mu, mu_k=mu)
    b.add_mesh(*g.as_args(), pos=(Rm @ np.zeros(3)).astype(np.float32), quat=q)
    m = 1.0 / host(b.inv_masses()).reshape(-1)
    t, vt = [], []
    for f in range(72):
        b.step_free(1 / 60, 100)
        t.append((f + 1) / 60)
        vt.append((m[:, None] * Vel(b).reshape(-1, 3)).sum(0) @ down / m.sum())
    t, vt = np.array(t), np.array(vt)
    accel = np.polyfit(t[t > 0.3], vt[t > 0.3], 1)[0]
    if slides:
        assert accel == pytest.approx(G * (np.sin(th) - mu * np.cos(th)), rel=0.01)
    else:
        assert abs(accel) < 1e-3 and abs(vt[-1]) < 2e-3  # creep of the regularised friction only
    p = P(b).reshape(-1, 3)
    assert np.abs(p[:, 1]).max() < 1e-3
    assert (p @ normal).min() > R - 3 * PEN0 - 1e-6


# ------------------------------------------------------------------------------ capstan


def capstan_shape(L1, rc, zc):
    """Vertices up side 1 (x = -rc), over the top of a cylinder (axis y at height zc), down side 2."""
    s = np.arange(NV) * SEG
    arc = np.pi * rc
    out = np.zeros((NV, 3))
    for i, si in enumerate(s):
        if si < L1:
            out[i] = (-rc, 0.0, zc - (L1 - si))
        elif si < L1 + arc:
            phi = np.pi - (si - L1) / rc
            out[i] = (rc * np.cos(phi), 0.0, zc + rc * np.sin(phi))
        else:
            out[i] = (rc, 0.0, zc - (si - L1 - arc))
    return out


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("mu,holds", [(0.5, True), (0.05, False)])
def test_capstan_holds_or_slips(backend, mu, holds):
    """Hanging lengths 1 : 2 over a cylinder: holds iff 2 <= exp(mu pi) (4.8 at mu 0.5; 1.17 at
    mu 0.05, which slips: the heavy side runs down)."""
    rcyl, zc = 0.10, 0.5
    rc = rcyl + R - PEN0
    L1 = (1.0 - np.pi * rc) / 3
    s = sdf()
    g = s.from_function(s.sdf_cylinder(rcyl, axis=1), (-0.2, -0.1, -0.2), (0.2, 0.1, 0.2), 0.004)
    start = capstan_shape(L1, rc, zc)
    b = ropes_from(backend, start[None], mu_s=mu, mu_k=mu)
    b.add_mesh(*g.as_args(), pos=np.array([0, 0, zc], np.float32))
    for _ in range(60 if holds else 18):
        b.step_free(1 / 60, 100)
    p = P(b).reshape(-1, 3)
    assert np.isfinite(p).all()
    moved = np.linalg.norm(p - start, axis=1).max()
    assert np.hypot(p[:, 0], p[:, 2] - zc).min() > rcyl + R - 1e-3  # never inside the cylinder
    if holds:
        assert moved < 0.01
    else:
        assert moved > 0.03 and p[-1, 2] < start[-1, 2] - 0.03


# ------------------------------------------------------------------------------ shapes


@pytest.mark.parametrize("backend", BACKENDS)
def test_drape_over_sphere(backend):
    """Dropped over a 25 cm sphere (larger than the rope's bending length (EI / rho g)^(1/3)
    = 16 cm) the rope drapes, never enters, stays centred, both ends below the centre."""
    rs, c = 0.25, np.array([0.5, 0.0, 0.4])
    s = sdf()
    g = s.from_function(s.sdf_sphere(rs), (-0.35, -0.35, -0.35), (0.35, 0.35, 0.35), 0.005)
    pos = straight_rows(1, c[2] + rs + R + 0.02)
    b = ropes_from(backend, pos, drag=2.0)  # strong air damping: the stiff rope rocks for a while
    b.add_mesh(*g.as_args(), pos=c.astype(np.float32))
    for _ in range(240):
        b.step_free(1 / 60, 100)
    p = P(b).reshape(-1, 3)
    assert np.isfinite(p).all()
    d = np.linalg.norm(p - c, axis=1) - rs
    assert d.min() > R - 1e-3
    assert (d < R + 2e-3).sum() >= 10
    assert abs(p[:, 0].mean() - c[0]) < 0.05
    assert p[[0, -1], 2].max() < c[2]
    assert np.abs(Vel(b)).max() < 0.05


@pytest.mark.parametrize("backend", BACKENDS)
def test_bowl_keeps_the_rope_inside(backend):
    """Dropped into a 0.6 m spherical bowl (mu 0.1) the rope stays inside, in its lower half,
    centred on the axis, at rest."""
    rb, c = 0.6, np.array([0.5, 0.0, 0.6])
    s = sdf()
    g = s.from_function(s.sdf_bowl(rb), (-0.65, -0.65, -0.65), (0.65, 0.65, 0.65), 0.01)
    pos = straight_rows(1, c[2])
    assert (rb - np.linalg.norm(pos[0] - c, axis=1)).min() > R + 0.05
    b = ropes_from(backend, pos, drag=0.3, mu_s=0.1)
    b.add_mesh(*g.as_args(), pos=c.astype(np.float32))
    for _ in range(300):
        b.step_free(1 / 60, 100)
    p = P(b).reshape(-1, 3)
    assert np.isfinite(p).all()
    assert (rb - np.linalg.norm(p - c, axis=1)).min() > R - 1e-3
    assert p[:, 2].max() < c[2] - rb / 2
    assert np.linalg.norm(p[:, :2].mean(0) - c[:2]) < 0.05
    assert np.abs(Vel(b)).max() < 0.05


@pytest.mark.parametrize("backend", BACKENDS)
def test_thin_wall_stops_a_fast_rope(backend):
    """A 5 mm wall stops a rope flying at 8 m/s without gravity (1.5 mm dynamic penetration
    allowed) and the rope bounces back."""
    s = sdf()
    g = s.from_function(s.sdf_box((0.0025, 0.6, 0.6)), (-0.06, -0.65, -0.65), (0.06, 0.65, 0.65), 0.0025)
    pos = np.zeros((1, NV, 3))
    pos[0, :, 1] = np.arange(NV) * SEG - 0.5
    pos[0, :, 0] = 0.3
    b = ropes_from(backend, pos, gravity=(0, 0, 0))
    b.add_mesh(*g.as_args(), pos=np.array([0.5, 0, 0], np.float32))
    v = np.zeros((1, NV, 3), np.float32)
    v[0, :, 0] = 8.0
    b.set_velocities(v)
    xmax = 0.0
    for _ in range(30):
        b.step_free(1 / 120, 50)
        xmax = max(xmax, P(b)[..., 0].max())
    p = P(b).reshape(-1, 3)
    assert np.isfinite(p).all()
    assert xmax < 0.5 - 0.0025 - R + 1.5e-3
    assert p[:, 0].max() < 0.49


# ------------------------------------------------------------------------------ envs and API


@pytest.mark.parametrize("backend", BACKENDS)
def test_env_zero_alone_or_beside_other_envs(backend):
    """Per-env poses: env 0's result is bitwise the same alone or beside envs whose floors sit
    elsewhere."""
    g = floor_lattice()

    def env0(n):
        pos = straight_rows(n, 0.2, y_step=3.0)
        b = ropes_from(backend, pos, drag=0.1)
        p = np.zeros((n, 3), np.float32)
        p[:, 1] = 3.0 * np.arange(n)
        p[:, 2] = -0.01 * np.arange(n)
        q = np.tile(np.array([0, 0, 0, 1], np.float32), (n, 1))
        b.add_mesh(*g.as_args(), pos=p, quat=q)
        for _ in range(30):
            b.step_free(1 / 60, 100)
        return P(b)[0]

    one = env0(1)
    assert (one[:, 2] < 0.05).all()  # it reached the floor
    assert np.array_equal(one, env0(4))


@pytest.mark.gpu
def test_mesh_api_validation_and_inert_meshes():
    """add_mesh validates before any state change (material set, 3-D values, spacing > 0, finite
    values, unit-able quaternion, 64 meshes at most); a mesh the rope never reaches, and a mesh
    added then cleared, leave the trajectory bitwise unchanged."""
    import ropesim

    g = floor_lattice(spacing=0.05)
    r = ropesim.RopeSim(num_verts=NV, seg_len=SEG, dir=np.array([1.0, 0, 0], np.float32), density=RHO, k_stretch=EA,
                        k_bend=EI, max_h=H, num_itr=ITR)
    with pytest.raises(ValueError):
        r.add_mesh(*g.as_args())  # no contact material yet
    r.set_contact(radius=R)
    with pytest.raises(ValueError):
        r.add_mesh(g.values[0], g.origin, g.spacing)
    with pytest.raises(ValueError):
        r.add_mesh(g.values, g.origin, 0.0)
    bad = g.values.copy()
    bad[0, 0, 0] = np.nan
    with pytest.raises(ValueError):
        r.add_mesh(bad, g.origin, g.spacing)
    with pytest.raises(ValueError):
        r.add_mesh(*g.as_args(), quat=np.zeros(4, np.float32))
    far = np.array([0, 0, -50.0], np.float32)
    for i in range(64):
        assert r.add_mesh(*g.as_args(), pos=far) == i
    with pytest.raises(ValueError):
        r.add_mesh(*g.as_args())
    with pytest.raises(ValueError):
        r.set_mesh_pose(64, np.zeros(3, np.float32), np.array([0, 0, 0, 1], np.float32))

    def swing(setup):
        rr = ropesim.RopeSim(num_verts=NV, seg_len=SEG, dir=np.array([1.0, 0, 0], np.float32), density=RHO,
                             k_stretch=EA, k_bend=EI, max_h=H, num_itr=8)
        rr.damping = 0.0
        rr.set_contact(radius=R)
        setup(rr)
        for f in range(30):
            t = f / 60
            rr.set_root(np.array([0.1 * np.sin(4 * t), 0.0, 0.0], np.float32),
                        np.array([0.4 * np.cos(4 * t), 0.0, 0.0], np.float32))
            rr.advance(1 / 60, substeps=100)
        return np.asarray(rr.positions())

    ref = swing(lambda rr: None)
    assert np.array_equal(ref, swing(lambda rr: rr.add_mesh(*g.as_args(), pos=far)))

    def add_then_clear(rr):
        rr.add_mesh(*g.as_args(), pos=np.array([0, 0, -0.1 - R + 0.002], np.float32))
        rr.clear_meshes()

    assert np.array_equal(ref, swing(add_then_clear))


# ------------------------------------------------------------------------------ convex edges


def drag_over_slab_edge(backend, round_r, T=3.0, fps=120):
    """Rope on a 60 cm high slab (edges rounded by round_r), root driven +x at 0.4 m/s over the
    far edge while the tail hangs over the near edge. Returns (peak strain, min vertex phi)."""
    TH = 0.6
    s = sdf()
    box = s.sdf_box((0.5, 0.4, 0.05), (0, 0, -0.05), round=round_r)
    g = s.from_function(box, (-0.65, -0.55, -0.25), (0.65, 0.55, 0.15), 0.005)
    pos = np.zeros((1, NV, 3), np.float32)
    pos[0, :, 0] = -0.2 - np.arange(NV) * SEG
    pos[0, :, 2] = TH + R + 0.002
    pin = np.zeros((1, NV), bool)
    pin[0, 0] = True
    b = ropes_from(backend, pos, pinned=pin, mu_s=0.3, mu_k=0.3, drag=0.03)
    b.add_mesh(*g.as_args(), pos=np.array([0, 0, TH], np.float32))
    strain, phimin = 0.0, np.inf
    x_at = lambda t: -0.2 + 0.4 * max(0.0, min(t - 0.5, 3.0))
    for f in range(int(T * fps)):
        p0 = np.array([[x_at(f / fps), 0.0, TH + R + 0.002]], np.float32)
        p1 = np.array([[x_at((f + 1) / fps), 0.0, TH + R + 0.002]], np.float32)
        b.step(dev(backend, p0), dev(backend, (p1 - p0) * fps), 1 / fps, 100 * 60 // fps, root_pos_end=dev(backend, p1))
        p = P(b)[0]
        strain = max(strain, np.linalg.norm(np.diff(p, axis=0), axis=1).max() / SEG - 1)
        phimin = min(phimin, box(p - np.array([0, 0, TH])).min())
    assert np.isfinite(p).all()
    return strain, phimin


@pytest.mark.parametrize("backend", BACKENDS)
def test_rounded_edge_slides_sharp_edge_snags(backend):
    """Contact acts at vertices, so a sharp 90-degree edge is below the rope's resolution: dragged
    over it from slightly below, the rope snags (friction holds a vertex on the side face while
    the tension runs away). Rounded by 2 cm (about half a segment) the edge lets it slide."""
    s_round, phi_round = drag_over_slab_edge(backend, 0.02)
    assert s_round < 0.02 and phi_round > R - 1e-3
    s_sharp, _ = drag_over_slab_edge(backend, 0.0)
    assert s_sharp > 0.3


# ------------------------------------------------------------------------------ precision and poses


@pytest.mark.parametrize("backend", BACKENDS)
def test_wall_far_from_origin_rests_like_the_plane(backend):
    """A wall at world x = 1 m (one float32 step of the position there is 1.75 rest sinks): the
    pose transform keeps pos and dx apart, so the rope rests as on the plane instead of chattering
    by one ulp per substep."""
    s = sdf()
    g = s.from_function(s.sdf_box((0.125, 3.0, 2.0), (0.125, 0, 0)), (-0.1875, -0.3125, -0.3125),
                        (0.1875, 0.3125, 1.3125), 1 / 128)
    X0 = 1.0
    finals = []
    for mesh in (False, True):
        pos = np.zeros((1, NV, 3), np.float32)
        pos[0, :, 0] = X0 - R - 2e-3
        pos[0, :, 2] = 0.1 + np.arange(NV) * SEG
        phi, inside = g.sample(pos[0] - np.array([X0, 0, 0]))
        assert inside.all() and (phi > R).all()  # the scene starts in the lattice, outside the wall
        b = ropes_from(backend, pos, gravity=(G, 0, 0))
        if mesh:
            b.add_mesh(*g.as_args(), pos=np.array([X0, 0, 0], np.float32))
        else:
            b.set_planes(np.array([[-1.0, 0.0, 0.0, -X0]], np.float32), radius=R, mu_s=0.5, v_slip=VSLIP, kappa=KAPPA)
        for _ in range(60):
            b.step_free(1 / 60, 100)
        finals.append(P(b)[0])
        assert np.abs(Vel(b)).max() < 1e-3
    assert np.abs(finals[0] - finals[1]).max() < 1e-6


@pytest.mark.parametrize("backend", BACKENDS)
def test_per_env_floor_heights_and_pose_update(backend):
    """Four envs with floors at different heights through per-env poses: each rope rests at its
    floor + R - PEN0; set_mesh_poses then lowers every floor by 2 cm and the ropes follow."""
    g = floor_lattice()
    n = 4
    b = ropes_from(backend, straight_rows(n, 0.05), drag=0.3)
    zf = -0.02 * np.arange(n)
    p = np.zeros((n, 3), np.float32)
    p[:, 2] = zf
    q = np.tile(np.array([0, 0, 0, 1], np.float32), (n, 1))
    b.add_mesh(*g.as_args(), pos=p, quat=q)
    for _ in range(90):
        b.step_free(1 / 60, 100)
    pos = P(b)
    for e in range(n):
        assert pos[e, :, 2].min() == pytest.approx(zf[e] + R - PEN0, abs=3e-8)
    p[:, 2] -= 0.02
    b.set_mesh_poses(0, p, q)
    for _ in range(90):
        b.step_free(1 / 60, 100)
    pos = P(b)
    for e in range(n):
        assert pos[e, :, 2].min() == pytest.approx(zf[e] - 0.02 + R - PEN0, abs=3e-8)


@pytest.mark.parametrize("backend", BACKENDS)
def test_empty_planes_keep_the_mesh_material(backend):
    """set_planes([]) switches the planes off and leaves the contact material a mesh uses."""
    g = floor_lattice()
    r = single_rope(backend)
    r.add_mesh(*g.as_args(), pos=np.array([0, 0, -1 / 128], np.float32))
    r.set_planes(np.zeros((0, 4), np.float32))
    for _ in range(60):
        r.advance(1 / 60, substeps=100)
    assert host(r.positions())[:, 2].min() == pytest.approx(-1 / 128 + R - PEN0, abs=3e-8)


def test_lattice_sample_matches_the_closed_form():
    """SdfGrid.sample reproduces the lattice interpolation (exact on the box's planar faces) and
    reports points outside the lattice as nan / not inside."""
    g = floor_lattice()
    pts = np.array([[0.5, 0.0, 0.02], [0.5, 0.1, -0.03], [0.5, 0.0, 0.5], [2.0, 0.0, 0.0]])
    phi, inside = g.sample(pts)
    assert inside.tolist() == [True, True, False, False]
    s = sdf()
    assert np.allclose(phi[:2], s.sdf_box((3.0, 1.0, 0.125), (0, 0, -0.125))(pts[:2]), atol=1e-6)
    assert np.isnan(phi[2:]).all()
