"""Known-answer physics, ported from the reference's analytic suite and run on both backends.

On the CPU this pins the oracle (the reference has no golden vectors: its tests are its
known answers); on the GPU the same checks run through the product kernels.
Reference sources: tests/test_statics.py:15-161, tests/test_dynamics.py:22-90,
tests/test_drag_quad.py:56-100, tests/test_contact.py:55-105, tests/test_api.py:9-130.
"""
import numpy as np
import pytest

from conftest import (BACKENDS, G, H, axis_angle_quat, energy_scalar, make_rope, masses, quat_rotate, rope_length,
                      segment_strains, settle)

Z1 = 2.404825557695773  # first zero of Bessel J0 (hanging-chain mode)


@pytest.mark.parametrize("backend", BACKENDS)
def test_vertical_hang_equilibrium(backend):
    r = make_rope(backend, n=33, direction=(0, -1, 0))
    settle(r, t=3.0, drag=3.0)
    p = np.asarray(r.positions(), dtype=np.float64)
    L = rope_length(r)
    assert np.max(np.abs(p[:, 0])) < 1e-3 * L
    assert np.max(np.abs(p[:, 2])) < 1e-3 * L
    assert np.all(np.diff(p[:, 1]) < 0)
    v = np.asarray(r.velocities(), dtype=np.float64)
    assert np.max(np.linalg.norm(v, axis=1)) < 5e-3
    assert np.all(segment_strains(r) > 0)


@pytest.mark.parametrize("backend", BACKENDS)
def test_hang_elongation_matches_EA_theory(backend):
    """Discrete-exact: elongation_i = (g * mass below i) * l_i / EA (test_statics.py:31-47)."""
    n, seg, rho, EA = 51, 0.02, 0.1, 500.0
    r = make_rope(backend, n=n, seg=seg, density=rho, EA=EA, direction=(0, -1, 0))
    settle(r, t=4.0, drag=3.0)
    m = masses(r)
    rest = np.asarray(r.rest_lengths(), dtype=np.float64)
    tension = G * np.array([np.sum(m[i + 1:]) for i in range(n - 1)])
    dL_theory = np.sum(tension * rest / EA)
    p = np.asarray(r.positions(), dtype=np.float64)
    dL = np.sum(np.linalg.norm(np.diff(p, axis=0), axis=1)) - np.sum(rest)
    assert dL == pytest.approx(dL_theory, rel=0.02)


@pytest.mark.parametrize("backend", BACKENDS)
def test_horizontal_release_settles_vertical(backend):
    r = make_rope(backend, n=33, direction=(1, 0, 0))
    settle(r, t=6.0, drag=2.0)
    p = np.asarray(r.positions(), dtype=np.float64)
    L = rope_length(r)
    assert abs(p[-1, 0]) < 0.02 * L
    assert abs(p[-1, 2]) < 0.02 * L
    assert p[-1, 1] == pytest.approx(-L, rel=0.02)


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("EI", [0.4, 0.8])
def test_cantilever_droop_vs_beam_theory(backend, EI):
    """delta_tip = w L^4 / (8 EI) within the reference's measured band (test_statics.py:60-85)."""
    n, seg, rho, EA = 26, 0.02, 0.1, 2000.0
    L = (n - 1) * seg
    r = make_rope(backend, n=n, seg=seg, density=rho, EA=EA, EI=EI, direction=(1, 0, 0), fix_root_orientation=True)
    settle(r, t=4.0, drag=2.0)
    delta = -np.asarray(r.positions(), dtype=np.float64)[-1, 1]
    ratio = delta / (rho * G * L ** 4 / (8.0 * EI))
    assert np.isfinite(delta)
    assert 0.80 < ratio < 1.05, f"ratio {ratio:.3f}"


@pytest.mark.parametrize("backend", BACKENDS)
def test_clamped_root_holds_rod_against_gravity(backend):
    th = np.deg2rad(30.0)
    d = (np.cos(th), np.sin(th), 0.0)
    n, seg = 16, 0.02
    L = (n - 1) * seg
    r = make_rope(backend, n=n, seg=seg, density=0.05, EA=2000.0, EI=0.4, direction=d, fix_root_orientation=True)
    settle(r, t=4.0, drag=2.0)
    p = np.asarray(r.positions(), dtype=np.float64)
    dirs = np.diff(p, axis=0)
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    angles = np.rad2deg(np.arccos(np.clip(dirs @ np.asarray(d), -1.0, 1.0)))
    assert angles[0] < 3.0
    assert np.max(angles) < 8.0
    assert p[-1, 1] > 0.8 * L * np.sin(th)
    pivot = make_rope(backend, n=n, seg=seg, density=0.05, EA=2000.0, EI=0.4, direction=d, fix_root_orientation=False)
    settle(pivot, t=4.0, drag=2.0)
    assert float(np.asarray(pivot.positions(), dtype=np.float64)[-1, 1]) < 0.0


@pytest.mark.parametrize("backend", BACKENDS)
def test_clamped_root_steers_rod_smoothly(backend):
    th0, th1 = np.deg2rad(30.0), np.deg2rad(40.0)
    d0 = (np.cos(th0), np.sin(th0), 0.0)
    r = make_rope(backend, n=16, seg=0.02, density=0.05, EA=2000.0, EI=0.4, direction=d0, fix_root_orientation=True)
    r.drag = 1.0
    ramp, hold = 90, 150
    for k in range(ramp + hold):
        th = th0 + (th1 - th0) * min(1.0, (k + 1) / ramp)
        r.set_root(np.zeros(3, np.float32), np.zeros(3, np.float32), q=axis_angle_quat([0, 0, 1], th).astype(np.float32))
        r.advance(H)
    q = axis_angle_quat([0, 0, 1], th1)
    np.testing.assert_allclose(np.asarray(r.quaternions(), dtype=np.float64)[0], q, atol=1e-5)
    p = np.asarray(r.positions(), dtype=np.float64)
    dirs = np.diff(p, axis=0)
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    angles = np.rad2deg(np.arccos(np.clip(dirs @ quat_rotate(q, [1.0, 0, 0]), -1.0, 1.0)))
    assert angles[0] < 3.0
    assert np.max(angles) < 10.0
    assert np.max(np.abs(segment_strains(r))) < 0.02


@pytest.mark.parametrize("backend", BACKENDS)
def test_hanging_chain_pendulum_period(backend):
    """T = (4 pi / z1) sqrt(L / g) within 5% (test_dynamics.py:22-38)."""
    n, seg = 33, 0.02
    L = (n - 1) * seg
    theta = np.deg2rad(2.0)
    r = make_rope(backend, n=n, seg=seg, direction=(np.sin(theta), -np.cos(theta), 0))
    ts, xs = [], []
    for k in range(int(round(6.0 / H))):
        r.advance(H)
        ts.append((k + 1) * H)
        xs.append(float(np.asarray(r.positions())[-1, 0]))
    ts, xs = np.array(ts), np.array(xs)
    s = np.sign(xs)
    idx = np.where(np.diff(s) != 0)[0]
    tc = ts[idx] - xs[idx] * (ts[idx + 1] - ts[idx]) / (xs[idx + 1] - xs[idx])
    assert len(tc) >= 5
    T = 2.0 * np.mean(np.diff(tc))
    assert T == pytest.approx((4.0 * np.pi / Z1) * np.sqrt(L / G), rel=0.05)


@pytest.mark.parametrize("backend", BACKENDS)
def test_energy_no_gain_horizontal_release(backend):
    n, seg, EA = 33, 0.02, 500.0
    r = make_rope(backend, n=n, seg=seg, EA=EA, direction=(1, 0, 0))
    E0 = energy_scalar(r, EA)
    m = masses(r)
    E_scale = G * np.sum(m * np.arange(n) * seg)
    E = []
    for _ in range(int(round(3.5 / H))):
        r.advance(H)
        E.append(energy_scalar(r, EA))
    E = np.array(E)
    assert (np.max(E) - E0) / E_scale < 0.02
    assert 1.0 + (E[-1] - E0) / E_scale > 0.08
    assert np.isfinite(E).all()


@pytest.mark.parametrize("backend", BACKENDS)
def test_gravity_mirror_symmetry(backend):
    n, seg, theta = 25, 0.02, np.deg2rad(3.0)
    tips = {}
    for s in (+1, -1):
        r = make_rope(backend, n=n, seg=seg, direction=(s * np.sin(theta), -np.cos(theta), 0))
        xs = []
        for _ in range(int(round(2.0 / H))):
            r.advance(H)
            xs.append(float(np.asarray(r.positions())[-1, 0]))
        tips[s] = np.array(xs)
    assert np.max(np.abs(tips[+1] + tips[-1])) < 5e-3 * (n - 1) * seg


# ---------------------------------------------------------------- quadratic drag (test_drag_quad.py)
def _free_decay(backend, kn, kt, v0, max_h=1.0 / 3000.0):
    r = make_rope(backend, n=33, seg=0.02, direction=(1.0, 0.0, 0.0), density=0.1, EA=1.0, EI=1e-6, max_h=max_h)
    r.set_gravity(np.zeros(3, np.float32))
    r.drag_quad = kn
    r.drag_quad_t = kt
    r.set_velocities(np.tile(np.asarray(v0, np.float32), (33, 1)))
    for _ in range(3):
        r.advance(H)
    return np.asarray(r.velocities(), dtype=np.float64)


@pytest.mark.parametrize("backend", BACKENDS)
def test_quadratic_drag_normal_decay(backend):
    v = _free_decay(backend, 0.5, 0.0, (0.0, 10.0, 0.0))
    expected = 10.0 / (1.0 + 0.5 * 10.0 * 3 * H)
    assert np.allclose(v[16:, 1], expected, rtol=1e-2)
    assert np.max(np.abs(v[16:, [0, 2]])) < 0.05


@pytest.mark.parametrize("backend", BACKENDS)
def test_quadratic_drag_axial_undamped(backend):
    v = _free_decay(backend, 0.5, 0.0, (10.0, 0.0, 0.0))
    assert np.allclose(v[16:, 0], 10.0, rtol=2e-3)


@pytest.mark.parametrize("backend", BACKENDS)
def test_quadratic_drag_substep_invariance(backend):
    vys = [np.mean(_free_decay(backend, 0.5, 0.0, (0.0, 10.0, 0.0), max_h=mh)[16:, 1]) for mh in (1 / 1500, 1 / 6000)]
    assert abs(vys[0] - vys[1]) / vys[1] < 5e-3


# ---------------------------------------------------------------- plane contact (test_contact.py)
NV, SEG, RHO, EA_C, EI_C = 21, 0.05, 0.117, 11473.0, 4.48e-3
R_C = 0.00635
H_C, ITR_C, G_C = 1.0 / 6000.0, 16, 9.81
KAPPA, VSLIP = 2.0, 1e-3
PEN0 = G_C * H_C * H_C / KAPPA ** 2


def _free_rope(backend, gravity, plane_w, mu_s, mu_k):
    from conftest import rope_sim_class

    r = rope_sim_class(backend)(num_verts=NV, seg_len=SEG, dir=np.array([1.0, 0, 0], np.float32), density=RHO,
                                k_stretch=EA_C, k_bend=EI_C, max_h=H_C, num_itr=ITR_C)
    r.damping = 0.0
    r.drag = 0.0
    r.set_gravity(np.asarray(gravity, np.float32))
    r.set_planes(np.array([[0.0, 0.0, 1.0, plane_w]], np.float32), radius=R_C, mu_s=mu_s, mu_k=mu_k, v_slip=VSLIP,
                 kappa=KAPPA)
    r.unpin_root()
    return r


def _com_vx(r, m):
    return (m[:, None] * np.asarray(r.velocities(), np.float64)).sum(0)[0] / m.sum()


@pytest.mark.parametrize("backend", BACKENDS)
def test_plane_rest_support_equals_weight(backend):
    w = -(R_C + 5e-4)
    r = _free_rope(backend, (0, 0, -G_C), w, 0.5, 0.5)
    m = 1.0 / np.asarray(r.inv_masses(), np.float64)
    for _ in range(60):
        r.advance(1 / 60, substeps=100)
    pen = np.maximum(-(np.asarray(r.positions(), np.float64)[:, 2] - w - R_C), 0)
    k = m * (KAPPA / H_C) ** 2
    assert (k * pen).sum() / (m.sum() * G_C) == pytest.approx(1.0, abs=5e-3)
    assert pen.max() == pytest.approx(PEN0, rel=0.05)
    assert np.abs(np.asarray(r.velocities())).max() < 1e-3


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("mu,slide", [(0.5, False), (0.2, True)])
def test_plane_incline_coulomb(backend, mu, slide):
    th = np.radians(20.0)
    r = _free_rope(backend, (G_C * np.sin(th), 0, -G_C * np.cos(th)), -(R_C - PEN0 * np.cos(th)), mu, mu)
    m = 1.0 / np.asarray(r.inv_masses(), np.float64)
    ts, vx = [], []
    for f in range(72):
        r.advance(1 / 60, substeps=100)
        ts.append((f + 1) / 60)
        vx.append(_com_vx(r, m))
    ts, vx = np.array(ts), np.array(vx)
    a = np.polyfit(ts[ts > 0.3], vx[ts > 0.3], 1)[0]
    if slide:
        assert a == pytest.approx(G_C * (np.sin(th) - mu * np.cos(th)), rel=0.01)
    else:
        assert abs(a) < 1e-3 and abs(vx[-1]) < 2e-3


# ---------------------------------------------------------------- API-level known answers (test_api.py)
@pytest.mark.parametrize("backend", BACKENDS)
def test_constructor_geometry_and_masses(backend):
    n, seg = 17, 0.03
    d = np.array([1.0, 2.0, -0.5])
    r = make_rope(backend, n=n, seg=seg, direction=d)
    p = np.asarray(r.positions(), dtype=np.float64)
    np.testing.assert_allclose(p, np.outer(np.arange(n) * seg, d / np.linalg.norm(d)), atol=1e-6)
    np.testing.assert_allclose(r.rest_lengths(), seg, rtol=1e-5)
    r2 = make_rope(backend, n=9, seg=0.02, density=0.1)
    inv = np.asarray(r2.inv_masses(), dtype=np.float64)
    assert inv[0] == 0.0
    np.testing.assert_allclose(inv[1:-1], 1.0 / (0.1 * 0.02), rtol=1e-5)
    np.testing.assert_allclose(inv[-1], 1.0 / (0.1 * 0.02 / 2), rtol=1e-5)


@pytest.mark.parametrize("backend", BACKENDS)
def test_advance_explicit_substeps_root_sweep(backend):
    r = make_rope(backend, n=8, direction=(0, -1, 0))
    v = np.array([0.12, 0.0, 0.0])
    r.set_root(np.zeros(3, np.float32), v.astype(np.float32))
    r.advance(H, substeps=50)
    np.testing.assert_allclose(np.asarray(r.positions(), dtype=np.float64)[0], v * H, atol=1e-6)


@pytest.mark.parametrize("backend", BACKENDS)
def test_initial_quaternions_identity_along_x(backend):
    r = make_rope(backend, n=8, direction=(1, 0, 0))
    q = np.asarray(r.quaternions(), dtype=np.float64)[:-1]
    np.testing.assert_allclose(q, np.array([0, 0, 0, 1.0]) * np.ones((7, 1)), atol=1e-6)


@pytest.mark.parametrize("backend", BACKENDS)
def test_reset_restores_initial_state(backend):
    r = make_rope(backend, direction=(1, 0, 0))
    p0 = np.array(r.positions())
    q0 = np.array(r.quaternions())
    for _ in range(30):
        r.advance(H)
    assert not np.allclose(np.array(r.positions()), p0, atol=1e-4)
    r.reset()
    np.testing.assert_allclose(np.array(r.positions()), p0, atol=1e-7)
    np.testing.assert_allclose(np.array(r.quaternions()), q0, atol=1e-7)
    np.testing.assert_allclose(np.array(r.velocities()), 0.0, atol=1e-7)
    assert r.time == pytest.approx(0.0)


def test_substep_count_float_ceil():
    """advance(1/60) at max_h = 1/3000 runs 51 substeps (float ceil, step.cpp:37-42)."""
    import math

    dt, mh = np.float32(1 / 60), np.float32(1 / 3000)
    assert math.ceil(np.float32(dt / mh)) == 51
