"""The sweep ordering: this engine's Jacobi sweeps against the reference's default in-place ones.

`deterministic=False`, the reference's default, runs the frame sweep in place (SNAPSHOT=false,
cosserat.cu:252-268: threads read neighbour rotors while others overwrite them, in warp-schedule
order) and writes each displacement in place (cosserat.cu:198-223, racing only across CUDA
blocks). The product always runs the deterministic (snapshot, Jacobi) ordering. The oracle's
`inplace_frames` switch runs the frame sweep as a vertex-order Gauss-Seidel pass, one
deterministic realisation of the in-place sweep, so the difference can be measured:

  * a rope settling under gravity: both orderings reach the same rest shape (the sweeps share
    their fixed points); measured <= 2.2e-7 m apart over 3 s;
  * gentle program driving (config 2's program with v0 ~ N(0, 0.05)): 1e-6 ... 1.5e-5 m apart per
    frame, about 4x the FP32 rounding floor;
  * config 2's whipping (v0 ~ N(0, 0.5)): the orderings part like two chaotic runs, 1e-5 m after
    one frame, 1e-3 m after twelve, centimetres after sixteen.

A caller relying on the default therefore sees trajectories within the ordering's own spread
(which the reference's racing sweeps also have from run to run), not a different equilibrium.
"""
import numpy as np
import pytest

import scenarios as S

F32 = np.float32


def _oracle_program(inplace, precision, v_std, p_std, frames):
    import ropesim_oracle as ro

    tweak = (lambda b: setattr(b._s, "inplace_frames", True)) if inplace else None
    r = S.program(ro, N=4, frames=frames, to_dev=lambda a: np.asarray(a, F32), precision=precision, v_std=v_std,
                  p_std=p_std, tweak=tweak)
    return r.reshape(frames, -1, 3)


def _per_frame(a, b):
    return np.linalg.norm(a - b, axis=-1).max(-1)


def test_orderings_share_the_rest_shape():
    import ropesim_oracle as ro

    def settle(inplace, frames=180):
        pos, roots = S.c2_positions(4, 64, 1)
        b = ro.RopeBatch.from_positions(pos, 0.117, 11473.0, 4.48e-3, 1 / 6000, 8, deterministic=True, precision="f64")
        b.set_gravity(np.array([0, 0, -9.8], F32))
        b.damping = 0.0
        b.drag = 2.0
        b._s.inplace_frames = inplace
        out = []
        for _ in range(frames):
            b.step(roots, np.zeros_like(roots), 1 / 60, 100)
            out.append(np.asarray(b.positions(), np.float64).reshape(-1, 3).copy())
        return np.stack(out)

    d = _per_frame(settle(False), settle(True))
    print(f"\n  settling: Jacobi vs in-place max {d.max():.2e} m, last frame {d[-1]:.2e} m")
    assert d.max() < 1e-6


def test_inplace_frames_differ_measurably_but_little():
    frames = 20
    j64 = _oracle_program(False, "f64", 0.05, 0.005, frames)
    i64 = _oracle_program(True, "f64", 0.05, 0.005, frames)
    j32 = _oracle_program(False, "f32", 0.05, 0.005, frames)
    d, floor = _per_frame(i64, j64), _per_frame(j32, j64)
    print(f"\n  gentle driving: Jacobi vs in-place max {d.max():.2e} m, FP32 floor {floor.max():.2e} m")
    assert d.max() < 1e-4                  # the same trajectory within 0.1 mm
    assert d.max() > 2.0 * floor.max()     # and a real difference, above rounding


@pytest.mark.gpu
def test_product_runs_the_jacobi_ordering():
    """Config 2's whipping for twelve frames: the GPU tracks the FP64 Jacobi oracle at FP32
    rounding and is told apart from the in-place ordering by more than four times that."""
    import torch

    import ropesim

    frames = 12
    to_dev = lambda a: torch.as_tensor(np.ascontiguousarray(a, F32), device="cuda")
    views = lambda b: torch.as_tensor(b.positions()).cpu().numpy().astype(np.float64)
    g = S.program(ropesim, N=4, frames=frames, to_dev=to_dev, views=views).reshape(frames, -1, 3)
    j64 = _oracle_program(False, "f64", 0.5, 0.05, frames)
    i64 = _oracle_program(True, "f64", 0.5, 0.05, frames)
    dj, di = _per_frame(g, j64), _per_frame(g, i64)
    print(f"\n  whipping, 12 frames: GPU vs Jacobi max {dj.max():.2e} m, GPU vs in-place max {di.max():.2e} m")
    assert dj.max() < 0.25 * di.max()
