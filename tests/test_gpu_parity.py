"""Parity of the CUDA product against the FP64 oracle (and its FP32 instantiation).

Bounds, stated per scene (the target tolerance is 1e-5 m of vertex deviation over 60 control frames):
  * well-posed scenes (the 33-vertex hanging rope, gentle program driving, clamped legacy roots):
    max |x_gpu - x_f64| <= 1e-5 m over every frame;
  * chaotic scenes (the 4096 x 64 whipping workload, uneven ropes in mesh/plane
    contact): rounding is amplified by the dynamics itself (the FP32 and FP64 oracles part by
    mm), so the bound is the FP32 noise floor: the GPU may deviate from FP64 by at most
    4x the FP32 oracle's own deviation + 1e-6 m, and by <= 1e-5 m after the first frame.
"""
import numpy as np
import pytest

import scenarios as S

pytestmark = pytest.mark.gpu

TOL = 1e-5


@pytest.fixture(scope="module")
def mods():
    import torch

    import ropesim
    import ropesim_oracle

    assert torch.cuda.is_available()
    return ropesim, ropesim_oracle


def to_dev(a):
    import torch

    return torch.as_tensor(np.ascontiguousarray(a, np.float32), device="cuda")


def host(a):
    return np.asarray(a, np.float32)


def views(b):
    import torch

    return torch.as_tensor(b.positions()).cpu().numpy().astype(np.float64)


def dev(a, b):
    return float(np.max(np.linalg.norm(np.asarray(a, np.float64) - np.asarray(b, np.float64), axis=-1)))


def test_c1_hanging_rope_parity(mods):
    rs, orc = mods
    g = S.c1(rs)
    o64 = S.c1(orc, precision="f64")
    o32 = S.c1(orc, precision="f32")
    d, d32 = dev(g, o64), dev(o32, o64)
    print(f"\n  config 1 (33 verts, 60 frames x 51 substeps): gpu-f64 {d:.2e} m, f32-f64 {d32:.2e} m, gpu-f32 {dev(g, o32):.2e} m")
    assert d <= TOL


def test_c1_literal_snap_is_finite(mods):
    """The literal config-1 start (set_root to (0,0,1) on a rope built from the origin) is a
    violent snap: reported, bounded only by finiteness and the rope staying attached."""
    rs, orc = mods
    g = S.c1(rs, literal=True)
    o64 = S.c1(orc, precision="f64", literal=True)
    print(f"\n  literal config 1: gpu-f64 {dev(g, o64):.2e} m (chaotic start)")
    assert np.isfinite(g).all()
    np.testing.assert_allclose(g[-1, 0], [0.1, 0.0, 1.0], atol=1e-5)


def test_program_gentle_parity(mods):
    rs, orc = mods
    g = S.program(rs, to_dev=to_dev, views=views, v_std=0.05, p_std=0.005)
    o64 = S.program(orc, to_dev=host, precision="f64", v_std=0.05, p_std=0.005)
    d = dev(g, o64)
    print(f"\n  program (gentle), 8x64, 20 frames x 100 substeps: gpu-f64 {d:.2e} m")
    assert d <= TOL


def test_legacy_clamped_roots_parity(mods):
    rs, orc = mods
    g = S.legacy(rs, to_dev=to_dev)
    o64 = S.legacy(orc, to_dev=host, precision="f64")
    d = dev(g, o64)
    print(f"\n  legacy clamped roots: gpu-f64 {d:.2e} m")
    assert d <= TOL


def test_program_config2_noise_floor(mods):
    rs, orc = mods
    kw = dict(N=4, frames=20)
    g = S.program(rs, to_dev=to_dev, views=views, **kw)
    o64 = S.program(orc, to_dev=host, precision="f64", **kw)
    o32 = S.program(orc, to_dev=host, precision="f32", **kw)
    d, d32 = dev(g, o64), dev(o32, o64)
    print(f"\n  config-2 whipping (4x64, 20 frames): gpu-f64 {d:.2e} m, f32-f64 {d32:.2e} m; first frame {dev(g[0], o64[0]):.2e} m")
    assert dev(g[0], o64[0]) <= TOL
    assert d <= 4.0 * d32 + 1e-6


def test_uneven_mesh_contact_noise_floor(mods):
    """Uneven ropes teleport-hit by meshes in the first frame: contact-rich from the start, so
    positions and the force/wrench readout are held to the FP32 noise floor of the oracle."""
    rs, orc = mods
    from ropesim import sdf

    g, gf, gw, _ = S.uneven(rs, sdf, to_dev=to_dev)
    o, of, ow, _ = S.uneven(orc, sdf, to_dev=host, precision="f64")
    o32, of32, ow32, _ = S.uneven(orc, sdf, to_dev=host, precision="f32")
    d, d32 = dev(g, o), dev(o32, o)
    print(f"\n  uneven ropes + planes + meshes (6 ropes, 10 frames): gpu-f64 {d:.2e} m, f32-f64 {d32:.2e} m, "
          f"first frame {dev(g[0], o[0]):.2e} m (f32 {dev(o32[0], o[0]):.2e}); |F| max {np.abs(of).max():.1f} N, "
          f"force dev gpu {np.abs(gf - of).max():.3f} N (f32 {np.abs(of32 - of).max():.3f}), "
          f"wrench dev gpu {np.abs(gw - ow).max():.3f} (f32 {np.abs(ow32 - ow).max():.3f})")
    assert dev(g[0], o[0]) <= 4.0 * dev(o32[0], o[0]) + 1e-6
    assert d <= 4.0 * d32 + 1e-6
    assert np.abs(gf[0] - of[0]).max() <= 4.0 * np.abs(of32[0] - of[0]).max() + 1e-3
    assert np.abs(gw[0] - ow[0]).max() <= 4.0 * np.abs(ow32[0] - ow[0]).max() + 1e-3
    assert np.abs(ow).max() > 0.0 and np.abs(of).max() > 0.0  # the readout saw contact


@pytest.mark.parametrize("planes", [[[0, 0, 1, 0.02]], [[0, 0, 1, 0], [0.3, 0, 1, -0.05], [-0.2, 0.1, 1, -0.03]]],
                         ids=["one-plane", "three-planes"])
def test_plane_only_contact_noise_floor(mods, planes):
    """Plane-only scenes: the sweep flags the lanes near a plane and redoes their terms with
    contact after the exchange (single plane as straight-line code, several in a loop). Positions
    and the contact-force readout are held to the FP32 noise floor of the oracle."""
    rs, orc = mods
    g, gf = S.planes_only(rs, planes)
    o, of = S.planes_only(orc, planes, precision="f64")
    o32, of32 = S.planes_only(orc, planes, precision="f32")
    d, d32 = dev(g, o), dev(o32, o)
    touching = int((np.linalg.norm(of, axis=-1) > 0).sum())
    print(f"\n  {len(planes)} plane(s), 6 uneven ropes, 10 frames: gpu-f64 {d:.2e} m, f32-f64 {d32:.2e} m, "
          f"first frame {dev(g[0], o[0]):.2e} m; vertex-frames in contact {touching}, |F| max {np.abs(of).max():.2f} N, "
          f"force dev gpu {np.abs(gf - of).max():.4f} N (f32 {np.abs(of32 - of).max():.4f})")
    assert touching > 0
    assert dev(g[0], o[0]) <= 4.0 * dev(o32[0], o[0]) + 1e-6
    assert d <= 4.0 * d32 + 1e-6
    assert np.abs(gf[0] - of[0]).max() <= 4.0 * np.abs(of32[0] - of[0]).max() + 1e-3


def test_bitwise_replay_and_block_invariance(mods):
    """Fresh objects replay bitwise, and the packed layout (bin size) does not change a single
    bit: every rope's arithmetic is independent of which CTA owns it."""
    rs, _ = mods
    import torch

    def run(block):
        pos, roots = S.c2_positions(12, 40, 5)
        b = rs.RopeBatch.from_positions(pos, 0.117, 11473.0, 4.48e-3, 1 / 6000, 8)
        if block:
            b.set_block(block)
        b.set_gravity(np.array([0, 0, -9.81], np.float32))
        b.damping = 0.0
        b.set_planes(np.array([[0, 0, 1, 0]], np.float32), radius=0.00635)
        rng = np.random.default_rng(9)
        p0 = roots.copy()
        for _ in range(5):
            v0 = rng.normal(0, 0.5, (12, 3)).astype(np.float32)
            p1 = (p0 + rng.normal(0, 0.05, (12, 3))).astype(np.float32)
            b.step(to_dev(p0), to_dev(v0), 1 / 60, 100, root_pos_end=to_dev(p1))
            p0 = p1
        return tuple(torch.as_tensor(f()).cpu().numpy() for f in (b.positions, b.velocities, b.quaternions)), b.layout()

    ref, lay = run(0)
    again, _ = run(0)
    for x, y in zip(ref, again):
        np.testing.assert_array_equal(x.view(np.uint32), y.view(np.uint32))
    for block in (64, 128, 256, 512):
        other, l2 = run(block)
        assert l2[0] == block
        for x, y in zip(ref, other):
            np.testing.assert_array_equal(x.view(np.uint32), y.view(np.uint32))


def test_exact_culling_is_bitwise_inert(mods):
    """The persistent kernel's early outs (the per-substep surface slack, the lattices' contact
    boxes and block bounds) only skip evaluations whose gap is >= 0: with them off (every plane
    and every candidate lattice evaluated at every iteration, as the reference does) positions,
    contact forces and mesh wrenches are the same bit for bit, on plane-only scenes (one plane
    and three), the uneven scene with teleported and walking meshes, and config-2 ropes. (Mesh
    wrenches are summed with float atomics across warps, so their last bits follow the order in
    which warps arrive.)"""
    rs, _ = mods
    from ropesim import sdf

    off = lambda b: b.set_culling(False)
    for planes in ([[0, 0, 1, 0.02]], [[0, 0, 1, 0], [0.3, 0, 1, -0.05], [-0.2, 0.1, 1, -0.03]]):
        a, af = S.planes_only(rs, planes, frames=4)
        b, bf = S.planes_only(rs, planes, frames=4, tweak=off)
        np.testing.assert_array_equal(a.view(np.uint64), b.view(np.uint64))
        np.testing.assert_array_equal(af.view(np.uint64), bf.view(np.uint64))
    g, gf, gw, _ = S.uneven(rs, sdf, to_dev=to_dev, frames=4)
    h, hf, hw, _ = S.uneven(rs, sdf, to_dev=to_dev, frames=4, tweak=off)
    assert np.abs(gw).max() > 0.0
    for x, y in ((g, h), (gf, hf)):
        np.testing.assert_array_equal(x.view(np.uint64), y.view(np.uint64))
    np.testing.assert_allclose(gw, hw, rtol=1e-5, atol=1e-6)  # float atomics: summation order
    c = S.program(rs, N=6, frames=4, to_dev=to_dev, views=views)
    d = S.program(rs, N=6, frames=4, to_dev=to_dev, views=views, tweak=off)
    np.testing.assert_array_equal(c.view(np.uint64), d.view(np.uint64))


def test_work_queue_schedule_is_bitwise_inert(mods):
    """Bins taken from the work queue in longest-first order of the previous frame's times, or one
    CTA per bin in packing order: the same bits, on config-2 ropes and the uneven mesh scene (the
    order changes from the second frame on, once bin times have been measured)."""
    rs, _ = mods
    from ropesim import sdf

    grid = lambda b: b.set_work_queue(False)
    a = S.program(rs, N=12, frames=4, to_dev=to_dev, views=views)
    b = S.program(rs, N=12, frames=4, to_dev=to_dev, views=views, tweak=grid)
    np.testing.assert_array_equal(a.view(np.uint64), b.view(np.uint64))
    g, gf, gw, _ = S.uneven(rs, sdf, to_dev=to_dev, frames=4)
    h, hf, hw, _ = S.uneven(rs, sdf, to_dev=to_dev, frames=4, tweak=grid)
    for x, y in ((g, h), (gf, hf)):
        np.testing.assert_array_equal(x.view(np.uint64), y.view(np.uint64))
    np.testing.assert_allclose(gw, hw, rtol=1e-5, atol=1e-6)  # float atomics: summation order
