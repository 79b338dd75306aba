"""The two engines compute the same substep: the persistent frame kernel (one launch per
control frame) and the per-substep-launch plain path (the reference's launch structure) call
the same per-vertex routines (rs_substep.cuh). nvcc may contract a*b+c into FMAs differently in
the two kernels, so they agree to rounding rather than bitwise: on a well-conditioned scene to
5e-6 m after 10 frames (measured 1.4e-6 m; each lands within 1e-5 m of the FP64 oracle), and through the
contact-rich uneven scene (meshes teleported against the ropes) within the FP32 noise floor
measured by the oracle (~5e-5 m after 2 frames; bound 2e-4 m)."""
import numpy as np
import pytest

import scenarios as S

pytestmark = pytest.mark.gpu


def to_dev(a):
    import torch

    return torch.as_tensor(np.ascontiguousarray(a, np.float32), device="cuda")


def test_plain_engine_matches_persistent_program():
    import torch

    import ropesim

    def run(engine):
        pos, roots = S.c2_positions(6, 64, 21)
        b = ropesim.RopeBatch.from_positions(pos, 0.117, 11473.0, 4.48e-3, 1 / 6000, 8)
        b.set_engine(engine)
        b.set_gravity(np.array([0, 0, -9.81], np.float32))
        b.damping = 0.0
        b.drag_quad = 0.09
        b.drag_quad_t = 0.01
        b.set_planes(np.array([[0, 0, 1, 0]], np.float32), radius=0.00635)
        rng = np.random.default_rng(3)
        p0 = roots.copy()
        for _ in range(10):
            v0 = rng.normal(0, 0.05, (6, 3)).astype(np.float32)
            p1 = (p0 + rng.normal(0, 0.005, (6, 3))).astype(np.float32)
            b.step(to_dev(p0), to_dev(v0), 1 / 60, 100, root_pos_end=to_dev(p1))
            p0 = p1
        return [torch.as_tensor(f()).cpu().numpy().astype(np.float64) for f in (b.positions, b.velocities, b.quaternions)]

    a, p = run("persistent"), run("plain")
    dp = np.abs(a[0] - p[0]).max()
    print(f"\n  persistent vs plain after 10 frames: positions {dp:.2e} m, frames {np.abs(a[2] - p[2]).max():.2e}")
    assert dp <= 5e-6
    np.testing.assert_allclose(a[2], p[2], atol=1e-4)
    np.testing.assert_allclose(a[1], p[1], atol=2e-2)  # velocity = dx / h amplifies position rounding by 6000


def test_plain_engine_matches_persistent_meshes():
    import ropesim
    from ropesim import sdf

    class Plain:
        RopeSim = ropesim.RopeSim

        class RopeBatch:
            @staticmethod
            def from_ropes(*a, **k):
                b = ropesim.RopeBatch.from_ropes(*a, **k)
                b.set_engine("plain")
                return b

    g, gf, gw, _ = S.uneven(ropesim, sdf, to_dev=to_dev, frames=2)
    p, pf, pw, _ = S.uneven(Plain, sdf, to_dev=to_dev, frames=2)
    d = np.max(np.linalg.norm(g - p, axis=-1))
    print(f"\n  persistent vs plain, uneven ropes in plane + mesh contact, 2 frames: {d:.2e} m")
    assert d <= 2e-4
    assert np.abs(gf - pf).max() <= 1e-2 * max(1.0, np.abs(gf).max())
    np.testing.assert_allclose(gw, pw, rtol=1e-2, atol=1e-2 * max(1.0, np.abs(gw).max()))


def test_plain_engine_matches_oracle():
    import torch

    import ropesim
    import ropesim_oracle

    class Plain:
        class RopeBatch:
            @staticmethod
            def from_positions(*a, **k):
                b = ropesim.RopeBatch.from_positions(*a, **k)
                b.set_engine("plain")
                return b

    views = lambda b: torch.as_tensor(b.positions()).cpu().numpy().astype(np.float64)
    g = S.program(Plain, to_dev=to_dev, views=views, v_std=0.05, p_std=0.005, N=4, frames=10)
    o = S.program(ropesim_oracle, to_dev=lambda a: np.asarray(a, np.float32), precision="f64", v_std=0.05, p_std=0.005,
                  N=4, frames=10)
    d = np.max(np.linalg.norm(g - o, axis=-1))
    print(f"\n  plain engine vs FP64 oracle (gentle program, 4x64, 10 frames): {d:.2e} m")
    assert d <= 1e-5
