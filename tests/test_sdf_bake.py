"""Mesh baking (ropesim.sdf.bake_mesh): signed-distance lattices of triangle meshes.

The reference bakes with Warp (ropesim/sdf.py:96-167); its tests give known answers
(tests/test_mesh_contact.py:233-250 and tests/test_isaac_bridge_geometry.py of the reference):
a tessellated sphere agrees with the analytic sphere up to tessellation, primitive meshes with
their closed forms up to interpolation, overlapping closed parts make a solid union, an open mesh
becomes a two-sided shell, rounding moves the surface outward, and a rope lands the same on the
baked sphere as on its closed form. Those answers pin the FP64 oracle (oracle/rs_sdfbake_oracle.hpp)
on the CPU and check the GPU bake; the GPU bake is also compared node by node with the oracle.
"""
import ctypes
import os

import numpy as np
import pytest

import meshes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def oracle_bake(v, f, spacing, margin, thickness=0.0, round=0.0):
    """The oracle on the lattice bake_mesh would choose (same box rule as sdf.py:135-138)."""
    import _oracle
    from ropesim import sdf

    v = np.asarray(v, np.float32)
    pad = margin + 0.5 * thickness + round
    origin, dims = sdf._lattice(v.min(0) - pad, v.max(0) + pad, spacing)
    phi, dist, wind = _oracle.bake_sdf(v, np.asarray(f, np.int32), origin, float(spacing), list(dims), thickness, round)
    return sdf.SdfGrid(phi.astype(np.float32), origin, float(spacing)), phi, dist, wind


def product_bake(v, f, spacing, margin, thickness=0.0, round=0.0):
    from ropesim import sdf

    return sdf.bake_mesh(v, f, spacing, margin, thickness=thickness, round=round)


BAKES = {"oracle": lambda *a, **k: oracle_bake(*a, **k)[0],
         "cuda": product_bake}
BACKENDS = ["oracle", pytest.param("cuda", marks=pytest.mark.gpu)]


def check_closed_form(grid, phi_ref, pts, tol):
    phi, inside = grid.sample(pts)
    assert inside.all()
    err = np.abs(phi - phi_ref(pts))
    assert err.max() < tol, err.max()


# ----------------------------------------------------------------------------- known answers

@pytest.mark.parametrize("backend", BACKENDS)
def test_icosphere_matches_analytic_sphere(backend):
    """test_mesh_contact.py:233-241: icosphere (4 subdivisions, r 0.15 m) within 5e-4 of the
    analytic distance at every node (tessellation only); the oracle at 2 cm, the GPU at 5 mm."""
    from ropesim import sdf

    rs = 0.15
    v, f = meshes.icosphere(4, rs)
    g = BAKES[backend](v, f, 0.02 if backend == "oracle" else 0.005, 0.1)
    ana = np.linalg.norm(g.nodes().reshape(-1, 3).astype(np.float64), axis=1) - rs
    assert np.abs(g.values.reshape(-1) - ana).max() < 5e-4
    assert (g.values < 0).sum() > 0 and (g.values > 0).sum() > 0
    assert isinstance(g, sdf.SdfGrid)


@pytest.mark.parametrize("backend", BACKENDS)
def test_box_mesh_bakes_to_the_box_sdf(backend):
    """test_isaac_bridge_geometry.py:19-25: 12-triangle box, 1 cm cells, 2000 points."""
    from ropesim import sdf

    v, f = meshes.box_mesh((0.2, 0.2, 0.1))
    assert sdf.is_closed(f)
    g = BAKES[backend](v, f, 0.01, 0.05)
    pts = np.random.default_rng(0).uniform(-0.22, 0.22, (2000, 3)) * np.array([1, 1, 0.55])
    check_closed_form(g, sdf.sdf_box((0.2, 0.2, 0.1)), pts, 5e-3)


@pytest.mark.parametrize("backend", BACKENDS)
def test_sphere_and_cylinder_meshes(backend):
    """test_isaac_bridge_geometry.py:28-39: 24-segment sphere and cylinders along each axis."""
    from ropesim import sdf

    v, f = meshes.uv_sphere(0.1)
    assert sdf.is_closed(f)
    g = BAKES[backend](v, f, 0.005, 0.03)
    check_closed_form(g, sdf.sdf_sphere(0.1), np.random.default_rng(1).uniform(-0.12, 0.12, (2000, 3)), 3e-3)
    for axis in range(3):
        v, f = meshes.cylinder_mesh(0.05, 0.3, axis)
        assert sdf.is_closed(f)
        g = BAKES[backend](v, f, 0.005, 0.03)
        keep = [d for d in range(3) if d != axis]
        pts = np.random.default_rng(2).uniform(-0.06, 0.06, (2000, 3))
        pts[:, axis] *= 0.5
        check_closed_form(g, lambda p: np.linalg.norm(p[:, keep], axis=1) - 0.05, pts, 3e-3)


@pytest.mark.parametrize("backend", BACKENDS)
def test_capsule_is_a_union_of_closed_parts(backend):
    """test_isaac_bridge_geometry.py:42-47: cylinder + two spheres, overlapping, bake as a solid."""
    from ropesim import sdf

    v, f = meshes.capsule_mesh(0.05, 0.3, 2)
    assert sdf.is_closed(f)
    g = BAKES[backend](v, f, 0.005, 0.03)
    phi, _ = g.sample(np.array([[0, 0, 0.0], [0, 0, 0.19], [0, 0, 0.21], [0.049, 0, 0.0], [0, 0.07, 0.0]]))
    assert phi[0] < -0.045 and phi[1] < -0.005 and phi[2] > 0.005 and abs(phi[3]) < 2e-3 and abs(phi[4] - 0.02) < 2e-3


@pytest.mark.parametrize("backend", BACKENDS)
def test_open_mesh_bakes_as_a_shell(backend):
    """test_isaac_bridge_geometry.py:50-58: a box without its top face, thickness 2 cells."""
    from ropesim import sdf

    v, f = meshes.box_mesh((0.2, 0.2, 0.1))
    top = [i for i, t in enumerate(f) if all(v[k, 2] > 0 for k in t)]
    f = np.delete(f, top, axis=0)
    assert not sdf.is_closed(f)
    g = BAKES[backend](v, f, 0.01, 0.05, thickness=0.02)
    phi, _ = g.sample(np.array([[0, 0, 0.0], [0, 0, -0.1], [0, 0, 0.1]]))
    assert phi[0] > 0.05 and abs(phi[1] + 0.01) < 3e-3
    assert phi[2] > 0.05


@pytest.mark.parametrize("backend", BACKENDS)
def test_rounding_fattens_the_shape(backend):
    """test_isaac_bridge_geometry.py:61-66."""
    v, f = meshes.box_mesh((0.2, 0.2, 0.1))
    g = BAKES[backend](v, f, 0.01, 0.05, round=0.02)
    phi, _ = g.sample(np.array([[0, 0, 0.11], [0, 0, 0.13], [0.2, 0.2, 0.1]]))
    assert abs(phi[0] + 0.01) < 2e-3 and abs(phi[1] - 0.01) < 2e-3
    assert phi[2] < 0.0


def test_bake_mesh_validates_before_any_device_work():
    """sdf.py:120-140: ValueError for a non-mesh, bad indices, an open mesh without thickness,
    a too-thin shell and negative rounding (checked on the host, so this runs without a GPU)."""
    from ropesim import sdf

    v, f = meshes.box_mesh((0.2, 0.2, 0.1))
    with pytest.raises(ValueError, match="triangle mesh"):
        sdf.bake_mesh(v[:2], f[:0], 0.01, 0.05)
    with pytest.raises(ValueError, match="out of range"):
        sdf.bake_mesh(v, f + 8, 0.01, 0.05)
    vu, fu = meshes.unweld(v, f)
    assert not sdf.is_closed(fu)
    with pytest.raises(ValueError, match="open mesh"):
        sdf.bake_mesh(vu, fu, 0.01, 0.05)
    with pytest.raises(ValueError, match="thickness"):
        sdf.bake_mesh(vu, fu, 0.01, 0.05, thickness=0.015)
    with pytest.raises(ValueError, match="round"):
        sdf.bake_mesh(v, f, 0.01, 0.05, round=-1.0)


def test_oracle_distance_and_winding_are_exact_on_a_box():
    """The oracle on the box: at nodes inside, the distance is the smallest face distance; the
    winding number is 1 inside and 0 outside to rounding."""
    v, f = meshes.box_mesh((0.2, 0.2, 0.1))
    g, phi, dist, wind = oracle_bake(v, f, 0.02, 0.05)
    p = g.nodes().astype(np.float64)
    d = np.abs(p) - np.array([0.2, 0.2, 0.1])
    inside = (d < 0).all(-1)
    assert np.allclose(dist[inside], -d.max(-1)[inside], atol=1e-12)
    assert np.allclose(wind[inside], 1.0, atol=1e-9) and np.allclose(wind[(d > 1e-9).any(-1)], 0.0, atol=1e-9)


# ----------------------------------------------------------------------------- GPU vs oracle

def _gpu_vs_oracle(v, f, spacing, margin, thickness=0.0, round=0.0):
    g = product_bake(v, f, spacing, margin, thickness=thickness, round=round)
    o, phi, dist, wind = oracle_bake(v, f, spacing, margin, thickness=thickness, round=round)
    assert g.values.shape == o.values.shape and np.array_equal(g.origin, o.origin)
    err = np.abs(g.values.astype(np.float64) - phi)
    # FP32 distances at coordinates up to ~0.4 m: a few float32 steps
    assert err.max() < 2e-6, err.max()
    if thickness == 0.0:
        clear = dist > 1e-5
        assert np.array_equal(g.values[clear] + np.float32(round) < 0, np.abs(wind[clear]) > 0.5)
    return g


@pytest.mark.gpu
def test_gpu_bake_matches_oracle_node_by_node():
    v, f = meshes.icosphere(4, 0.15)  # 5120 triangles in 160 culling tiles
    _gpu_vs_oracle(v, f, 0.013, 0.07)
    v, f = meshes.capsule_mesh(0.05, 0.3, 1)  # overlapping parts: winding number 2 inside the overlaps
    _gpu_vs_oracle(v, f, 0.007, 0.03)
    v, f = meshes.box_mesh((0.2, 0.2, 0.1))
    _gpu_vs_oracle(v, f, 0.011, 0.05, round=0.02)
    f_open = f[:-2]
    _gpu_vs_oracle(v, f_open, 0.011, 0.05, thickness=0.025)


@pytest.mark.gpu
def test_gpu_bake_drops_zero_area_triangles_and_keeps_winding_free():
    """Degenerate triangles (repeated vertices) change nothing; reversed winding gives the same
    lattice (the sign follows the winding number's magnitude)."""
    from ropesim import sdf

    v, f = meshes.icosphere(2, 0.1)
    g0 = sdf.bake_mesh(v, f, 0.01, 0.03)
    # the closedness check refuses the degenerate extras, so they go to the kernel directly
    from ropesim._ropesim import bake_sdf

    fd = np.concatenate([f, np.array([[0, 0, 1], [5, 5, 5]], np.int32)])
    vals = bake_sdf(v, fd, g0.origin, g0.spacing, list(g0.shape), 0.0, 0.0)
    assert np.array_equal(vals, g0.values)
    gr = sdf.bake_mesh(v, f[:, ::-1].copy(), 0.01, 0.03)
    assert np.array_equal(gr.values < 0, g0.values < 0)
    assert np.abs(gr.values - g0.values).max() < 1e-6


@pytest.mark.gpu
def test_gpu_sign_falls_back_to_solid_angles_on_an_open_mesh():
    """Signed bake of an open box (no top face) straight through the kernel: rows whose line
    crossings do not cancel take the solid-angle winding number; signs match the oracle's
    wherever the winding number is not within 1e-3 of 1/2."""
    from ropesim import sdf
    from ropesim._ropesim import bake_sdf

    v, f = meshes.box_mesh((0.2, 0.2, 0.1))
    top = [i for i, t in enumerate(f) if all(v[k, 2] > 0 for k in t)]
    f = np.delete(f, top, axis=0)
    origin, dims = sdf._lattice(v.min(0) - 0.05, v.max(0) + 0.05, 0.013)
    vals, n_dist, n_cross, n_solid = bake_sdf(v, f, origin, 0.013, list(dims), 0.0, 0.0, counters=True)
    import _oracle

    phi, dist, wind = _oracle.bake_sdf(v, f, origin, 0.013, list(dims), 0.0, 0.0)
    assert n_solid > 0 and n_cross > 0 and n_dist > 0
    assert np.abs(np.abs(vals) - dist).max() < 2e-6
    sure = (dist > 1e-5) & (np.abs(np.abs(wind) - 0.5) > 1e-3)
    assert np.array_equal(vals[sure] < 0, np.abs(wind[sure]) > 0.5)


@pytest.mark.gpu
def test_rope_lands_the_same_on_baked_and_closed_form_sphere():
    """test_mesh_contact.py:242-250: a free rope dropped on the baked icosphere and on the closed
    form sampled on the same lattice ends within 3 mm after 120 frames."""
    import torch

    import ropesim
    from ropesim import sdf

    NV, SEG, RHO, EA, EI, R = 21, 0.05, 0.117, 11473.0, 4.48e-3, 0.00635
    H, ITR, G = 1.0 / 6000.0, 16, 9.81
    rs, c = 0.15, np.array([0.5, 0.0, 0.3])
    v, f = meshes.icosphere(4, rs)
    baked = sdf.bake_mesh(v, f, spacing=0.005, margin=0.1)
    outs = []
    hi = baked.origin + baked.spacing * (np.array(baked.shape) - 1)
    for grid in (sdf.from_function(sdf.sdf_sphere(rs), baked.origin, hi, baked.spacing), baked):
        pos = np.zeros((1, NV, 3))
        pos[0, :, 0] = np.arange(NV) * SEG
        pos[0, :, 2] = c[2] + rs + R + 0.02
        b = ropesim.RopeBatch.from_positions(pos.astype(np.float32), RHO, EA, EI, H, ITR, pinned=np.zeros((1, NV), bool))
        b.damping = 0.0
        b.drag = 0.3
        b.set_gravity(np.array([0.0, 0.0, -G]))
        b.set_contact(radius=R, mu_s=0.5, mu_k=None, v_slip=1e-3, kappa=2.0)
        b.add_mesh(*grid.as_args(), pos=c.astype(np.float32))
        for _ in range(120):
            b.step_free(1 / 60, 100)
        outs.append(torch.as_tensor(b.positions()).cpu().numpy()[0])
    assert np.isfinite(outs[1]).all()
    assert np.abs(outs[0] - outs[1]).max() < 3e-3


@pytest.mark.gpu
def test_bake_through_the_c_abi_with_device_output():
    """rs_sdf_bake with a device output buffer (queued on a stream) equals the host-output call
    bitwise; the evaluation counters show the culling at work."""
    import torch

    from ropesim import sdf

    lib = ctypes.CDLL(os.path.join(ROOT, "cosserat-rod-solver-cuda_b200", "ropesim", "libropesim_b200.so"))
    v, f = meshes.icosphere(3, 0.12)
    ref = sdf.bake_mesh(v, f, 0.008, 0.05)
    nx, ny, nz = ref.shape
    out = torch.full((nx, ny, nz), float("nan"), dtype=torch.float32, device="cuda")
    cnt = (ctypes.c_ulonglong * 4)()
    s = torch.cuda.Stream()
    vp = np.ascontiguousarray(v, np.float32)
    fp = np.ascontiguousarray(f, np.int32)
    org = np.ascontiguousarray(ref.origin, np.float32)
    torch.cuda.synchronize()
    rc = lib.rs_sdf_bake(vp.ctypes.data_as(ctypes.c_void_p), len(v), fp.ctypes.data_as(ctypes.c_void_p), len(f),
                         org.ctypes.data_as(ctypes.c_void_p), ctypes.c_double(ref.spacing), nx, ny, nz, ctypes.c_float(0.0),
                         ctypes.c_float(0.0), ctypes.c_void_p(out.data_ptr()), 1, ctypes.c_void_p(s.cuda_stream), cnt)
    assert rc == 0
    s.synchronize()
    assert np.array_equal(out.cpu().numpy(), ref.values)
    nodes = nx * ny * nz
    assert 0 < cnt[0] < 0.75 * nodes * len(f)  # distances culled by the tile bounds
    assert 0 < cnt[1] < nx * ny * len(f)  # crossing tests: at most one pass over the triangles per row
    assert cnt[2] == 0  # a closed mesh: every row's crossings cancel, no solid-angle fallback
    assert cnt[3] > 0  # the kernels' device time in ns
