"""The reference's API-contract and root-driving acceptance suites (tests/test_api.py and
tests/test_driving.py of the reference) restated over both backends; the geometry, mass,
explicit-substep and reset checks already live in test_physics.py.

API: invalid constructor arguments and stiffness arrays raise ValueError before any state change;
fine discretisations run; the root quaternion is normalised on write and refused on a free root;
knobs round-trip; shapes and dtypes; an undriven root stays pinned; a reset rope evolves like a
fresh one. Driving (set_root(pos, vel) then advance(H): the root sweeps linearly over the
frame): the sweep is exact and continuous, 60 Hz control tracks 240 Hz, a root swung near the
chain's first mode pumps energy in, and aggressive whipping stays stable.
"""
import numpy as np
import pytest

from conftest import BACKENDS, H, make_rope, masses, rope_length, rope_sim_class, segment_strains

F32 = np.float32


def drive(r, traj, t_end, rate=60.0, every=1):
    """Per frame: set_root(traj(t), (traj(t + 1/rate) - traj(t)) * rate), advance(1/rate).
    Returns the tips [frames / every, 3]."""
    h = 1.0 / rate
    tips = []
    for k in range(int(round(t_end * rate))):
        p0, p1 = np.asarray(traj(k * h), np.float64), np.asarray(traj(k * h + h), np.float64)
        r.set_root(p0.astype(F32), ((p1 - p0) * rate).astype(F32))
        r.advance(h)
        if (k + 1) % every == 0:
            tips.append(np.asarray(r.positions(), np.float64)[-1])
    return np.array(tips)


# ------------------------------------------------------------------------------ construction


@pytest.mark.gpu
def test_invalid_constructor_arguments_raise():
    import ropesim

    for kw in (dict(num_verts=2), dict(num_verts=8, seg_len=0.0), dict(num_verts=8, dir=np.zeros(3, F32)),
               dict(num_verts=8, density=0.0), dict(num_verts=8, max_h=0.0),
               # k_bend = 0 zeroes the rest rotors and the frame solve normalises a zero vector
               dict(num_verts=8, k_bend=0.0)):
        with pytest.raises(ValueError):
            ropesim.RopeSim(**kw)
    with pytest.raises(ValueError, match="5e-4"):
        ropesim.RopeSim(num_verts=8, seg_len=4e-4, collisions=True)


@pytest.mark.parametrize("backend", BACKENDS)
def test_stiffness_arrays_are_validated(backend):
    r = make_rope(backend, n=8)
    for bad in (np.zeros(7, F32), np.full(7, np.nan, F32)):
        with pytest.raises(ValueError):
            r.set_bend_stiffnesses(bad)
        with pytest.raises(ValueError):
            r.set_stretch_stiffnesses(bad)
    r.set_bend_stiffnesses(np.full(7, 1e-4, F32))  # still usable after the refused calls
    r.set_stretch_stiffnesses(np.full(7, 500.0, F32))
    for _ in range(10):
        r.advance(H)
    assert np.isfinite(np.asarray(r.positions())).all()


@pytest.mark.parametrize("backend", BACKENDS)
def test_fine_discretisation_runs(backend):
    """0.4 mm segments (below the yarn-scale radius floor of 5e-4 m): with collisions off the
    dead radius and barrier scale with the segment length, so construction succeeds and runs."""
    r = make_rope(backend, n=101, seg=0.0004, drag=1.0)
    for _ in range(30):
        r.advance(H)
    assert np.isfinite(np.asarray(r.positions())).all()


@pytest.mark.parametrize("backend", BACKENDS)
def test_root_quaternion_is_normalised_and_guarded(backend):
    r = make_rope(backend, n=8, fix_root_orientation=True)
    r.set_root(np.zeros(3, F32), np.zeros(3, F32), q=np.array([0, 0, 0, 2.0], F32))
    np.testing.assert_allclose(np.asarray(r.quaternions())[0], [0, 0, 0, 1.0], atol=1e-6)
    with pytest.raises(ValueError):
        r.set_root(np.zeros(3, F32), np.zeros(3, F32), q=np.zeros(4, F32))
    free = make_rope(backend, n=8)  # q on a free pivot would act only as a transient impulse
    with pytest.raises(ValueError):
        free.set_root(np.zeros(3, F32), np.zeros(3, F32), q=np.array([0, 0, 0, 1], F32))


@pytest.mark.parametrize("backend", BACKENDS)
def test_knobs_round_trip_and_shapes(backend):
    r = make_rope(backend, n=12)
    r.drag, r.damping, r.num_itr, r.accel_ratio, r.max_h = 0.25, 1e-5, 4, 0.9, 1e-3
    r.set_gravity(np.array([0.1, -9.0, 0.2], F32))
    assert r.drag == pytest.approx(0.25) and r.damping == pytest.approx(1e-5)
    assert r.num_itr == 4 and r.accel_ratio == pytest.approx(0.9) and r.max_h == pytest.approx(1e-3)
    np.testing.assert_allclose(r.gravity, [0.1, -9.0, 0.2], rtol=1e-6)
    assert r.last_error == 0 and r.last_warning == 0
    shapes = {"positions": (12, 3), "velocities": (12, 3), "quaternions": (12, 4), "inv_masses": (12,),
              "rest_lengths": (11,)}
    for name, shape in shapes.items():
        a = getattr(r, name)()
        assert a.shape == shape
    if backend == "cuda":
        assert r.positions().dtype == np.float32 and r.num_verts == 12
        old = r.max_h
        r.advance(H, substeps=50)
        assert r.max_h == pytest.approx(old)  # explicit substeps leave max_h as it was
        with pytest.raises(ValueError):
            r.advance(H, substeps=-1)


@pytest.mark.parametrize("backend", BACKENDS)
def test_undriven_root_stays_pinned(backend):
    r = make_rope(backend, direction=(1, 0, 0))
    for _ in range(30):
        r.advance(H)
    p = np.asarray(r.positions(), np.float64)
    np.testing.assert_allclose(p[0], 0.0, atol=1e-7)
    assert p[-1, 1] < -0.01


@pytest.mark.parametrize("backend", BACKENDS)
def test_reset_rope_evolves_like_a_fresh_one(backend):
    """No hidden state survives reset(): with deterministic sweeps a reset rope replays a fresh
    rope's trajectory bit for bit (the reference bounds it by its racing sweeps' chaos floor)."""

    def drop(pre_frames):
        r = make_rope(backend, direction=(1, 0, 0), drag=0.5)
        if pre_frames:
            for _ in range(pre_frames):
                r.advance(H)
            r.reset()
        for _ in range(30):
            r.advance(H)
        return np.asarray(r.positions(), np.float64)

    assert np.array_equal(drop(0), drop(60))


@pytest.mark.parametrize("backend", BACKENDS)
def test_collisions_flag_runs(backend):
    r = make_rope(backend, collisions=True, drag=0.5)
    for _ in range(30):
        r.advance(H)
    assert np.isfinite(np.asarray(r.positions())).all()
    assert r.collisions_enabled and r.last_error == 0


# ------------------------------------------------------------------------------ root driving


@pytest.mark.parametrize("backend", BACKENDS)
def test_root_sweep_is_exact(backend):
    r = make_rope(backend, n=25, direction=(0, -1, 0))
    v = np.array([0.10, 0.0, 0.05])
    r.set_root(np.zeros(3, F32), v.astype(F32))
    r.advance(H)
    np.testing.assert_allclose(np.asarray(r.positions(), np.float64)[0], v * H, atol=1e-5)
    for k in range(1, 10):  # a continuous piecewise-linear trajectory over many frames
        r.set_root((v * k * H).astype(F32), v.astype(F32))
        r.advance(H)
    np.testing.assert_allclose(np.asarray(r.positions(), np.float64)[0], v * 10 * H, atol=1e-4)


@pytest.mark.parametrize("backend", BACKENDS)
def test_driven_root_has_no_teleports(backend):
    """Where a frame's sweep ends is where the next command starts."""
    traj = lambda t: np.array([0.1 * np.sin(2 * np.pi * t), 0.0, 0.0])
    r = make_rope(backend, n=25, direction=(0, -1, 0))
    jump = 0.0
    for k in range(60):
        p_cmd = traj(k * H)
        if k:
            jump = max(jump, float(np.linalg.norm(p_cmd - np.asarray(r.positions(), np.float64)[0])))
        r.set_root(p_cmd.astype(F32), ((traj(k * H + H) - p_cmd) / H).astype(F32))
        r.advance(H)
    assert jump < 1e-4


@pytest.mark.parametrize("backend", BACKENDS)
def test_60hz_control_tracks_240hz(backend):
    circle = lambda t: np.array([0.05 * np.cos(np.pi * t) - 0.05, 0.0, 0.05 * np.sin(np.pi * t)])
    tips = {}
    for rate in (60.0, 240.0):
        r = make_rope(backend, n=25, drag=0.5)
        tips[rate] = drive(r, circle, 2.0, rate, every=int(rate // 60))
    L = 24 * 0.02
    assert np.sqrt(np.mean(np.sum((tips[60.0] - tips[240.0]) ** 2, axis=1))) < 0.03 * L


@pytest.mark.parametrize("backend", BACKENDS)
def test_swung_root_pumps_energy_in(backend):
    """A root swung near the hanging chain's first mode (omega_1 = 2.405/2 sqrt(g/L)) pumps the
    rope far above the still-hanging rope's residual (stretch-ringing) energy."""

    def ke(r):
        v = np.asarray(r.velocities(), np.float64)
        return 0.5 * float(np.sum(masses(r) * np.sum(v * v, axis=1)))

    still = make_rope(backend, n=25, direction=(0, -1, 0))
    for _ in range(int(round(2.0 / H))):
        still.advance(H)
    L = 24 * 0.02
    f = 0.9 / ((4 * np.pi / 2.404826) * np.sqrt(L / 9.8))
    swung = make_rope(backend, n=25, direction=(0, -1, 0))
    drive(swung, lambda t: np.array([0.15 * np.sin(2 * np.pi * f * t), 0.0, 0.0]), 2.0)
    assert ke(swung) > 50.0 * max(ke(still), 1e-12)
    assert ke(swung) > 1e-4


@pytest.mark.parametrize("backend", BACKENDS)
def test_whipping_stays_stable(backend):
    r = make_rope(backend, n=33, direction=(0, -1, 0), EA=500.0)
    drive(r, lambda t: np.array([0.3 * np.sin(4 * np.pi * t), 0.1 * np.sin(8 * np.pi * t), 0.0]), 2.0)
    p = np.asarray(r.positions(), np.float64)
    assert np.isfinite(p).all()
    assert np.max(np.abs(segment_strains(r))) < 0.25
    assert np.max(np.linalg.norm(p - p[0], axis=1)) < 2.0 * rope_length(r)
    assert r.last_error == 0
