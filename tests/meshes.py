"""Triangle meshes for the bake tests and the bake benchmark (outward, counter-clockwise faces).

The reference's bake tests take their meshes from trimesh (icosphere) and from the Kit-free
tessellation helpers of ropesim/isaac_bridge.py (box, sphere, cylinder, capsule); neither is
available here, so these are written from the geometry: a subdivided icosahedron projected on
the sphere, a 12-triangle box, latitude/longitude spheres and capped cylinders.
"""
from __future__ import annotations

import numpy as np


def icosphere(subdivisions: int, radius: float):
    """Icosahedron whose faces are split in four `subdivisions` times, vertices on the sphere."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]
    verts = [np.array(p, np.float64) / np.linalg.norm(p) for p in v]
    faces = list(f)
    for _ in range(subdivisions):
        mid = {}

        def midpoint(a, b):
            key = (min(a, b), max(a, b))
            if key not in mid:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                mid[key] = len(verts) - 1
            return mid[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = midpoint(a, b), midpoint(b, c), midpoint(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return (np.array(verts) * radius).astype(np.float32), np.array(faces, np.int32)


def box_mesh(half):
    """Axis-aligned box of half extents `half` centred at the origin: 8 vertices, 12 triangles."""
    hx, hy, hz = (float(h) for h in half)
    v = np.array([[sx * hx, sy * hy, sz * hz] for sx in (-1, 1) for sy in (-1, 1) for sz in (-1, 1)], np.float32)
    # vertex index = 4 * (x > 0) + 2 * (y > 0) + (z > 0)
    quads = [(0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)]
    f = []
    for a, b, c, d in quads:
        f += [(a, b, c), (a, c, d)]
    return v, np.array(f, np.int32)


def uv_sphere(radius: float, segments: int = 24, rings: int = 12, centre=(0.0, 0.0, 0.0)):
    """Latitude/longitude sphere: two poles, `rings - 1` latitude circles of `segments` vertices."""
    c = np.asarray(centre, np.float64)
    v = [c + (0.0, 0.0, radius)]
    for r in range(1, rings):
        th = np.pi * r / rings
        for s in range(segments):
            ph = 2 * np.pi * s / segments
            v.append(c + radius * np.array([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)]))
    v.append(c + (0.0, 0.0, -radius))
    south = len(v) - 1
    f = []
    ring = lambda r, s: 1 + (r - 1) * segments + (s % segments)
    for s in range(segments):
        f.append((0, ring(1, s), ring(1, s + 1)))
        f.append((south, ring(rings - 1, s + 1), ring(rings - 1, s)))
    for r in range(1, rings - 1):
        for s in range(segments):
            a, b, cc, d = ring(r, s), ring(r + 1, s), ring(r + 1, s + 1), ring(r, s + 1)
            f += [(a, b, cc), (a, cc, d)]
    return np.array(v, np.float32), np.array(f, np.int32)


def cylinder_mesh(radius: float, length: float, axis: int = 2, segments: int = 24):
    """Closed cylinder of `radius` and `length` along coordinate `axis`, centred at the origin,
    its caps fanned from a centre vertex."""
    h = 0.5 * length
    v = [(0.0, 0.0, -h), (0.0, 0.0, h)]
    for z in (-h, h):
        for s in range(segments):
            ph = 2 * np.pi * s / segments
            v.append((radius * np.cos(ph), radius * np.sin(ph), z))
    lo = lambda s: 2 + (s % segments)
    hi = lambda s: 2 + segments + (s % segments)
    f = []
    for s in range(segments):
        f.append((0, lo(s + 1), lo(s)))
        f.append((1, hi(s), hi(s + 1)))
        f += [(lo(s), lo(s + 1), hi(s + 1)), (lo(s), hi(s + 1), hi(s))]
    v = np.array(v, np.float64)
    out = np.empty_like(v)  # cyclic relabelling (keeps the orientation): local z -> axis
    out[:, axis] = v[:, 2]
    out[:, (axis + 1) % 3] = v[:, 0]
    out[:, (axis + 2) % 3] = v[:, 1]
    return out.astype(np.float32), np.array(f, np.int32)


def capsule_mesh(radius: float, length: float, axis: int = 2, segments: int = 24):
    """A cylinder and two end spheres: three overlapping closed components."""
    parts = [cylinder_mesh(radius, length, axis, segments)]
    for sgn in (-1.0, 1.0):
        c = [0.0, 0.0, 0.0]
        c[axis] = sgn * 0.5 * length
        parts.append(uv_sphere(radius, segments, segments // 2, c))
    vs, fs, off = [], [], 0
    for v, f in parts:
        vs.append(v)
        fs.append(f + off)
        off += len(v)
    return np.concatenate(vs), np.concatenate(fs)


def unweld(vertices, triangles):
    """One vertex copy per triangle corner (how many exporters write meshes)."""
    return vertices[triangles.reshape(-1)], np.arange(triangles.size, dtype=np.int32).reshape(-1, 3)
