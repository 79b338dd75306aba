"""The checked build (libropesim_b200_checked.so through ropesim._ropesim_checked, compiled with
-DROPESIM_CHECKED): the frame and adjoint kernels test every neighbour (t +- 1), candidate list,
contact-group, pose-cache, lattice-node, block-bound and caller index they use and record the
first failed check in the status word instead of trapping. On the small parity scenes - program
driving over a plane, uneven ropes against planes and teleported / walking meshes with the
readout on, a CTA-resident rope-rope contact group, and one differentiable frame forward and
backward - no check may fail, and the results must be those of the regular build (the checks add
no arithmetic: within 1e-6 m, and the regular build's own parity bounds against the oracle).
"""
import numpy as np
import pytest

import scenarios as S

pytestmark = pytest.mark.gpu


class Checked:
    """The checked module behind the ropesim API shape."""

    def __init__(self):
        from ropesim import _ropesim_checked as m

        self.RopeSim, self.RopeBatch = m.RopeSim, m.RopeBatch


def to_dev(a):
    import torch

    return torch.as_tensor(np.ascontiguousarray(a, np.float32), device="cuda")


def views(b):
    import torch

    return torch.as_tensor(b.positions()).cpu().numpy().astype(np.float64)


def record(holder):
    """A scenario hook that keeps the batch (to query its checks after the run)."""
    return lambda b: holder.append(b)


def assert_clean(batches):
    for b in batches:
        code, checked = b.bounds_check()
        assert checked, "the checked module is not the checked build"
        assert code == 0, f"bounds check {code} failed"


def test_checked_program_scene():
    import ropesim
    import ropesim_oracle

    kept = []
    c = S.program(Checked(), N=4, frames=5, to_dev=to_dev, views=views, v_std=0.05, p_std=0.005, tweak=record(kept))
    r = S.program(ropesim, N=4, frames=5, to_dev=to_dev, views=views, v_std=0.05, p_std=0.005)
    o = S.program(ropesim_oracle, N=4, frames=5, to_dev=lambda a: np.asarray(a, np.float32), precision="f64",
                  v_std=0.05, p_std=0.005)
    assert_clean(kept)
    assert np.abs(c - r).max() <= 1e-6
    assert np.max(np.linalg.norm(c - o, axis=-1)) <= 1e-5


def test_checked_uneven_mesh_scene():
    import ropesim
    from ropesim import sdf

    kept = []
    c, cf, cw, _ = S.uneven(Checked(), sdf, to_dev=to_dev, frames=3, tweak=record(kept))
    r, rf, rw, _ = S.uneven(ropesim, sdf, to_dev=to_dev, frames=3)
    assert_clean(kept)
    assert np.abs(cw).max() > 0.0  # the readout saw contact
    assert np.abs(c - r).max() <= 1e-6
    assert np.abs(cf - rf).max() <= 1e-6 * max(1.0, np.abs(rf).max())


def test_checked_rope_contact_group():
    import ropesim

    def run(mod):
        R, V = 4, 24
        pos = np.zeros((R, V, 3), np.float32)
        for r in range(R):
            pos[r, :, 0] = 0.015 * r
            pos[r, :, 2] = 1.0 - 0.02 * np.arange(V)
            pos[r, 1:, 1] = 1e-4 * (r + 1) * np.sin(np.arange(1, V))
        b = mod.RopeBatch.from_positions(pos, 0.117, 11473.0, 4.48e-3, 1 / 6000, 8)
        b.set_gravity(np.array([0, 0, -9.81], np.float32))
        b.damping = 0.0
        b.drag = 0.5
        rad = 0.00635
        b.set_rope_contact(True, 0.9 * rad, 0.2 * rad, 0.025, 0.4, 1e7, 1.2, R)
        roots = pos[:, 0].copy()
        sway = (np.arange(R) % 2 - 0.5)[:, None] * np.array([0.0, 0.02, 0.0], np.float32)
        for f in range(3):
            p0, p1 = roots + sway * np.sin(f / 3), roots + sway * np.sin((f + 1) / 3)
            b.step(to_dev(p0), to_dev((p1 - p0) * 60), 1 / 60, 50, root_pos_end=to_dev(p1))
        return b, views(b)

    bc, c = run(Checked())
    _, r = run(ropesim)
    assert_clean([bc])
    assert np.abs(c - r).max() <= 1e-6


def test_checked_adjoint_frame():
    import torch

    import adjoint_cases as ac
    import ropesim
    import ropesim.grad as rg

    R, V, F = 4, 16, 2
    _, pos = ac.scene(R=R, V=V, plane=True, material="c1")
    progs = ac.programs(pos, F, v_std=0.3, p_std=0.02)
    tgt = torch.tensor(ac.targets(pos, F), device="cuda", dtype=torch.float32)
    _, dens, ea0, ei0 = ac.MATERIALS["c1"]

    def grads(mod):
        b = mod.RopeBatch.from_positions(pos, dens, ea0, ei0, 1 / 6000, 8)
        b.set_gravity(np.array([0.0, 0.0, -9.81], np.float32))
        b.damping = 0.0
        b.drag = 0.2
        b.set_planes(np.array([[0.0, 0.0, 1.0, 0.0]], np.float32), radius=0.00635, mu_s=0.5, mu_k=0.3)
        st = [t.clone().requires_grad_() for t in rg.state(b)]
        par = [t.clone().requires_grad_() for t in rg.parameters(b)]
        P = [torch.tensor(a, device="cuda", requires_grad=True) for a in progs]
        cur, loss = st, 0.0
        for f in range(F):
            cur = rg.frame(b, cur, par, P[0][f], P[1][f], P[2][f], 1 / 60, 100)
            loss = loss + ((cur[0].view(R, V, 3)[:, -1] - tgt[f]) ** 2).sum(-1).mean()
        loss.backward()
        return b, [t.grad.detach().cpu().numpy() for t in P + par]

    bc, gc = grads(Checked())
    _, gr = grads(ropesim)
    assert_clean([bc])
    for x, y in zip(gc, gr):
        assert ac.rel(x, y) <= 1e-5
