"""Signed-distance lattices for rod-mesh contact.

A lattice stores phi (negative inside) at nodes origin + (i, j, k) * spacing of the object's own
frame, values[i, j, k] in C order. `RopeSim/RopeBatch.add_mesh(*grid.as_args())` uploads it.
Contact acts where phi < rope radius, so the lattice must extend beyond the surface by at least
the rope radius plus a few cells; outside the lattice there is no contact.

The lattice rule of the reference's helpers is kept so that a shape sampled here is the same
grid the reference would build (ropesim/sdf.py:61-85 of DeformX/Cosserat-Rod-Solver-CUDA):
origin = lo rounded to float32, nodes per axis = max(ceil((hi - lo) / spacing) + 1, 2).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

__all__ = ["SdfGrid", "from_function", "sdf_box", "sdf_sphere", "sdf_cylinder", "sdf_bowl", "sdf_capsule",
           "bake_mesh", "is_closed"]


@dataclass
class SdfGrid:
    values: np.ndarray   # float32 [nx, ny, nz]
    origin: np.ndarray   # float32 [3]
    spacing: float

    @property
    def shape(self):
        return tuple(self.values.shape)

    def axes(self):
        """Node coordinates along x, y, z (float64)."""
        return [float(self.origin[d]) + self.spacing * np.arange(self.values.shape[d], dtype=np.float64) for d in range(3)]

    def nodes(self):
        """Node coordinates [nx, ny, nz, 3] (float32, object frame)."""
        x, y, z = self.axes()
        g = np.empty(self.values.shape + (3,), np.float32)
        g[..., 0] = x[:, None, None]
        g[..., 1] = y[None, :, None]
        g[..., 2] = z[None, None, :]
        return g

    def as_args(self):
        return self.values, self.origin, float(self.spacing)

    def sample(self, points):
        """Host check of a scene: the solver's trilinear interpolant (float64) at object-frame
        points [M, 3] and the mask of points inside the lattice (phi is nan outside, where the
        solver applies no contact)."""
        p = np.asarray(points, np.float64).reshape(-1, 3)
        u = (p - self.origin.astype(np.float64)) / float(self.spacing)
        hi = np.asarray(self.values.shape, np.float64) - 1.0
        inside = np.all(u >= 0.0, axis=1) & np.all(u < hi, axis=1)
        phi = np.full(p.shape[0], np.nan)
        if not inside.any():
            return phi, inside
        ui = u[inside]
        cell = np.floor(ui).astype(np.int64)
        t = ui - cell
        v = self.values
        acc = np.zeros(ui.shape[0])
        for corner in range(8):
            bx, by, bz = corner & 1, (corner >> 1) & 1, (corner >> 2) & 1
            w = (t[:, 0] if bx else 1.0 - t[:, 0]) * (t[:, 1] if by else 1.0 - t[:, 1]) * (t[:, 2] if bz else 1.0 - t[:, 2])
            acc += w * v[cell[:, 0] + bx, cell[:, 1] + by, cell[:, 2] + bz].astype(np.float64)
        phi[inside] = acc
        return phi, inside


def _lattice(lo, hi, spacing):
    lo64 = np.asarray(lo, np.float64).reshape(3)
    hi64 = np.asarray(hi, np.float64).reshape(3)
    dims = np.maximum(np.ceil((hi64 - lo64) / float(spacing)).astype(np.int64) + 1, 2)
    return lo64.astype(np.float32), tuple(int(d) for d in dims)


def from_function(phi, lo, hi, spacing, max_nodes_per_block=1 << 21):
    """Sample a vectorised signed distance phi(points [M, 3] float64) -> [M] on the box [lo, hi]
    (x-slab blocks of at most `max_nodes_per_block` nodes)."""
    origin, dims = _lattice(lo, hi, spacing)
    g = SdfGrid(np.empty(dims, np.float32), origin, float(spacing))
    x, y, z = g.axes()
    plane = dims[1] * dims[2]
    step = max(1, max_nodes_per_block // plane)
    yy, zz = np.meshgrid(y, z, indexing="ij")
    yz = np.stack([yy.ravel(), zz.ravel()], axis=1)
    for i0 in range(0, dims[0], step):
        i1 = min(dims[0], i0 + step)
        pts = np.empty(((i1 - i0) * plane, 3))
        pts[:, 0] = np.repeat(x[i0:i1], plane)
        pts[:, 1:] = np.tile(yz, (i1 - i0, 1))
        g.values[i0:i1] = np.asarray(phi(pts), np.float32).reshape(i1 - i0, dims[1], dims[2])
    return g


# ---- closed-form shapes in the object frame ------------------------------------------------
def sdf_box(half, centre=(0.0, 0.0, 0.0), round=0.0):
    """Axis-aligned box of half extents `half` about `centre`, edges rounded with radius
    `round` (outer size unchanged). Exact outside and inside."""
    h = np.asarray(half, np.float64).reshape(3) - float(round)
    if np.any(h < 0):
        raise ValueError("round must not exceed the smallest half extent")
    c = np.asarray(centre, np.float64).reshape(3)
    r = float(round)

    def phi(p):
        q = np.abs(np.asarray(p, np.float64) - c) - h
        outside = np.sqrt(np.sum(np.square(np.clip(q, 0.0, None)), axis=1))
        inside = np.minimum(np.max(q, axis=1), 0.0)
        return outside + inside - r
    return phi


def sdf_sphere(radius, centre=(0.0, 0.0, 0.0)):
    c = np.asarray(centre, np.float64).reshape(3)
    r = float(radius)
    return lambda p: np.sqrt(np.sum(np.square(np.asarray(p, np.float64) - c), axis=1)) - r


def sdf_cylinder(radius, axis=2):
    """Infinite cylinder of `radius` along coordinate `axis`."""
    others = [a for a in range(3) if a != axis]
    r = float(radius)
    return lambda p: np.sqrt(np.sum(np.square(np.asarray(p, np.float64)[:, others]), axis=1)) - r


def sdf_bowl(radius, centre=(0.0, 0.0, 0.0)):
    """Spherical cavity: negative outside the sphere, the rope lives inside it."""
    s = sdf_sphere(radius, centre)
    return lambda p: -s(p)


def sdf_capsule(radius, half_length, axis=2, centre=(0.0, 0.0, 0.0)):
    """Capsule: the points within `radius` of the segment centre +- half_length * e_axis."""
    c = np.asarray(centre, np.float64).reshape(3)
    r, hl = float(radius), float(half_length)

    def phi(p):
        d = np.asarray(p, np.float64) - c
        t = np.clip(d[:, axis], -hl, hl)
        d = d.copy()
        d[:, axis] -= t
        return np.sqrt(np.sum(np.square(d), axis=1)) - r
    return phi


def is_closed(triangles):
    """True when every undirected edge belongs to exactly two triangles (closed, manifold)."""
    t = np.asarray(triangles, np.int64).reshape(-1, 3)
    if t.size == 0:
        return False
    e = np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]])
    e.sort(axis=1)
    if e.min() < 0:
        raise ValueError("triangle indices must be >= 0")
    key = e[:, 0] * (int(e[:, 1].max()) + 1) + e[:, 1]  # one integer per undirected edge
    _, counts = np.unique(key, return_counts=True)
    return bool(np.all(counts == 2))


def bake_mesh(vertices, triangles, spacing, margin, thickness=0.0, round=0.0, device=None):
    """Distance lattice of a triangle mesh on its padded bounding box, baked on the GPU
    (the reference's bake_mesh, ropesim/sdf.py:96-156, which needs Warp; here the library's own
    sm_100a kernels, no Warp).

    vertices [V, 3], triangles [T, 3], any winding. thickness == 0: the SIGNED distance, negative
    inside (generalized winding number of magnitude > 1/2); the mesh must be closed (every edge
    shared by exactly two triangles; weld unwelded exports first). thickness > 0: a two-sided
    shell, |distance| - thickness / 2, for open meshes (sheets, heightfields); thickness must be
    >= 2 * spacing so that both faces keep a gradient. round > 0 offsets the surface outward
    (phi - round), rounding convex edges by that radius. margin pads the box beyond the shell and
    rounding on every side (use >= rope radius + a few cells). `device` is accepted for the
    reference's signature; the current CUDA device bakes.
    """
    from ._ropesim import bake_sdf

    vertices = np.asarray(vertices, np.float32).reshape(-1, 3)
    triangles = np.asarray(triangles, np.int32).reshape(-1, 3)
    if len(vertices) < 3 or len(triangles) < 1:
        raise ValueError("bake_mesh needs a triangle mesh")
    if triangles.min() < 0 or triangles.max() >= len(vertices):
        raise ValueError("triangle indices out of range")
    if thickness > 0:
        if thickness < 2 * spacing:
            raise ValueError("thickness must be >= 2 * spacing (one cell on each side of the mid-surface)")
    elif not is_closed(triangles):
        raise ValueError("open mesh (an edge is not shared by exactly two triangles): a signed distance has no "
                         "inside. Weld a watertight but unwelded export first, or pass thickness >= 2 * spacing "
                         "to bake a two-sided shell")
    if round < 0:
        raise ValueError("round must be >= 0")
    pad = margin + 0.5 * thickness + round
    lo, hi = vertices.min(0) - pad, vertices.max(0) + pad
    origin, dims = _lattice(lo, hi, spacing)
    values = bake_sdf(vertices, triangles, origin, float(spacing), list(dims), float(thickness), float(round))
    if not np.isfinite(values).all():
        raise ValueError("bake_mesh produced non-finite distances")
    return SdfGrid(values, origin, float(spacing))
