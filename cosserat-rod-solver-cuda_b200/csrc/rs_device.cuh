// rs_device.cuh -- device arithmetic of the substep: vectors, rotors, the symmetric 3x3
// local solve, the surface contact law and the trilinear SDF sample.
//
// Every function keeps the operation order of the reference routine it cites so that a
// single-precision run tracks the reference within rounding (IEEE div/sqrt, no fast math), with
// two exceptions on the contact path: the lattice normal is normalised by rsqrt_nr (about 1 ulp)
// and the contact law forms its slip ratio with one division instead of two.
//
// The engine is compiled with -fmad=false: the compiler fuses nothing, and every fused
// multiply-add is written out here (fmaf, one rounding). A sum of products is evaluated as
// an fmaf chain from its first term, e.g. dot = fma(z, z', fma(y, y', x x')). Every kernel
// instantiation (block size, surface variant) therefore does the same arithmetic, and a rope's
// result does not depend on the launch configuration that stepped it.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "rs_types.h"

namespace rsd {

// Checked builds: record the first failed check (rs_types.h, CHK_*) in status[3].
__device__ __forceinline__ void check_fail(int* status, int code) {
    if (status) atomicCAS(status + 3, 0, code);
}

struct f3 {
    float x, y, z;
};
__device__ __forceinline__ f3 mk3(float x, float y, float z) { return f3{x, y, z}; }
__device__ __forceinline__ f3 zero3() { return f3{0.f, 0.f, 0.f}; }
__device__ __forceinline__ f3 operator+(f3 a, f3 b) { return f3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ f3 operator-(f3 a, f3 b) { return f3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ f3 operator-(f3 a) { return f3{-a.x, -a.y, -a.z}; }
__device__ __forceinline__ f3 operator*(f3 a, float s) { return f3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ f3 operator*(float s, f3 a) { return f3{s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ f3 operator/(f3 a, float s) { return f3{a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ f3& operator+=(f3& a, f3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
__device__ __forceinline__ f3& operator-=(f3& a, f3 b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; return a; }
__device__ __forceinline__ f3& operator*=(f3& a, float s) { a.x *= s; a.y *= s; a.z *= s; return a; }
__device__ __forceinline__ float dot(f3 a, f3 b) { return fmaf(a.z, b.z, fmaf(a.y, b.y, a.x * b.x)); }
// a * s + b, fused per component
__device__ __forceinline__ f3 fma3(f3 a, float s, f3 b) { return f3{fmaf(a.x, s, b.x), fmaf(a.y, s, b.y), fmaf(a.z, s, b.z)}; }
__device__ __forceinline__ f3 cross(f3 a, f3 b) {
    return f3{fmaf(a.y, b.z, -(a.z * b.y)), fmaf(a.z, b.x, -(a.x * b.z)), fmaf(a.x, b.y, -(a.y * b.x))};
}
// Reciprocal square root: rsqrtf (within 2 ulp) and one Newton step, within about 1 ulp.
__device__ __forceinline__ float rsqrt_nr(float x) {
    const float y = rsqrtf(x);
    return fmaf(0.5f * y, fmaf(-x * y, y, 1.f), y);
}
// c + a x b and c + a.b, accumulated into c by fused multiply-adds
__device__ __forceinline__ f3 cross_add(f3 a, f3 b, f3 c) {
    return f3{fmaf(a.y, b.z, fmaf(-a.z, b.y, c.x)), fmaf(a.z, b.x, fmaf(-a.x, b.z, c.y)),
              fmaf(a.x, b.y, fmaf(-a.y, b.x, c.z))};
}
__device__ __forceinline__ float dot_add(f3 a, f3 b, float c) { return fmaf(a.z, b.z, fmaf(a.y, b.y, fmaf(a.x, b.x, c))); }
__device__ __forceinline__ float len(f3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ f3 lerp3(f3 a, f3 b, float t) { return fma3(b, t, a * (1.f - t)); }
__device__ __forceinline__ f3 xyz(float4 v) { return f3{v.x, v.y, v.z}; }
__device__ __forceinline__ float4 f4(f3 v, float w) { return make_float4(v.x, v.y, v.z, w); }

// Rotor (x, y, z = bivector part, w = scalar) products, Rotor.h:96-105 and :185-188.
__device__ __forceinline__ float4 qmul(float4 a, float4 b) {
    const f3 av = xyz(a), bv = xyz(b);
    const f3 v = fma3(av, b.w, fma3(bv, a.w, cross(av, bv)));
    return make_float4(v.x, v.y, v.z, fmaf(a.w, b.w, -dot(av, bv)));
}
__device__ __forceinline__ float4 qconj(float4 a) { return make_float4(-a.x, -a.y, -a.z, a.w); }
__device__ __forceinline__ float dot4(float4 a, float4 b) {
    return fmaf(a.w, b.w, fmaf(a.z, b.z, fmaf(a.y, b.y, a.x * b.x)));
}
__device__ __forceinline__ float4 scale4(float4 a, float s) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }
__device__ __forceinline__ float4 add4(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
__device__ __forceinline__ float4 sub4(float4 a, float4 b) { return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
// a * s + c, fused per component
__device__ __forceinline__ float4 fma4(float4 a, float s, float4 c) {
    return make_float4(fmaf(a.x, s, c.x), fmaf(a.y, s, c.y), fmaf(a.z, s, c.z), fmaf(a.w, s, c.w));
}
// c + vec(a b): the vector part of a rotor product, accumulated into c
__device__ __forceinline__ f3 qmul_vec_add(float4 a, float4 b, f3 c) {
    const f3 av = mk3(a.x, a.y, a.z), bv = mk3(b.x, b.y, b.z);
    return fma3(av, b.w, fma3(bv, a.w, cross_add(av, bv, c)));
}
__device__ __forceinline__ float4 normalize4(float4 a) { return scale4(a, 1.f / sqrtf(dot4(a, a))); }
__device__ __forceinline__ f3 qrot(float4 q, f3 v) {
    const f3 qv = xyz(q);
    const f3 a = fma3(v, q.w, cross(qv, v));
    const float c = dot(v, qv);
    return fma3(qv, c, fma3(a, q.w, cross(qv, a)));
}
// q * e1, the tangent of the segment frame: qrot(q, e1) with the zero terms of e1 dropped
// (a = (w, z, -y), c = x; exact, as multiplying by 1 and adding 0 are).
__device__ __forceinline__ f3 qtangent(float4 q) {
    const f3 qv = xyz(q);
    const f3 a = mk3(q.w, q.z, -q.y);
    return fma3(qv, q.x, fma3(a, q.w, cross(qv, a)));
}
// (v, 0) * b for a pure vector v: the rotor product with the zero scalar's terms dropped.
__device__ __forceinline__ float4 qmul_pure(f3 v, float4 b) {
    const f3 bv = xyz(b);
    const f3 r = fma3(v, b.w, cross(v, bv));
    return make_float4(r.x, r.y, r.z, -dot(v, bv));
}
// c * (1, 0, 0, 0): a signed permutation of c's components.
__device__ __forceinline__ float4 qmul_e1(float4 c) { return make_float4(c.w, c.z, -c.y, -c.x); }

// Symmetric 3x3: diag (xx, yy, zz), upper (xy, xz, yz).
struct sym3 {
    float xx, yy, zz, xy, xz, yz;
};
__device__ __forceinline__ sym3 sym_diag(float d) { return sym3{d, d, d, 0.f, 0.f, 0.f}; }
__device__ __forceinline__ sym3 sym_zero() { return sym3{0.f, 0.f, 0.f, 0.f, 0.f, 0.f}; }
__device__ __forceinline__ void sym_add(sym3& a, const sym3& b) {
    a.xx += b.xx; a.yy += b.yy; a.zz += b.zz; a.xy += b.xy; a.xz += b.xz; a.yz += b.yz;
}
__device__ __forceinline__ void sym_add_scaled_outer(sym3& a, f3 n, float s) {  // a += (n n^T) * s
    a.xx = fmaf(n.x * n.x, s, a.xx); a.yy = fmaf(n.y * n.y, s, a.yy); a.zz = fmaf(n.z * n.z, s, a.zz);
    a.xy = fmaf(n.x * n.y, s, a.xy); a.xz = fmaf(n.x * n.z, s, a.xz); a.yz = fmaf(n.y * n.z, s, a.yz);
}
// a -= (n n^T - I) * s
__device__ __forceinline__ void sym_sub_scaled_outer_minus_I(sym3& a, f3 n, float s) {
    a.xx = fmaf(-fmaf(n.x, n.x, -1.f), s, a.xx); a.yy = fmaf(-fmaf(n.y, n.y, -1.f), s, a.yy);
    a.zz = fmaf(-fmaf(n.z, n.z, -1.f), s, a.zz);
    a.xy = fmaf(-(n.x * n.y), s, a.xy); a.xz = fmaf(-(n.x * n.z), s, a.xz); a.yz = fmaf(-(n.y * n.z), s, a.yz);
}
// x = H^-1 f through the adjugate of the symmetric matrix (cofactor expansion).
__device__ __forceinline__ f3 sym_solve(const sym3& H, f3 f) {
    const float c00 = fmaf(H.yy, H.zz, -(H.yz * H.yz)), c01 = fmaf(H.xz, H.yz, -(H.xy * H.zz));
    const float c02 = fmaf(H.xy, H.yz, -(H.xz * H.yy)), c11 = fmaf(H.xx, H.zz, -(H.xz * H.xz));
    const float c12 = fmaf(H.xy, H.xz, -(H.xx * H.yz)), c22 = fmaf(H.xx, H.yy, -(H.xy * H.xy));
    const float idet = 1.f / dot(mk3(H.xx, H.xy, H.xz), mk3(c00, c01, c02));
    return f3{dot(mk3(c00, c01, c02), f) * idet, dot(mk3(c01, c11, c12), f) * idet, dot(mk3(c02, c12, c22), f) * idet};
}

// Closest points of segments a0a1 / b0b1 as (u, v), Common.h:327-345.
__device__ __forceinline__ void seg_closest(f3 a0, f3 a1, f3 b0, f3 b1, float& u, float& v) {
    const f3 A0 = a1 - a0, A1 = b1 - b0;
    const float a = dot(A0, A0), b = dot(A0, A1), c = dot(A1, A1);
    const f3 diff = b0 - a0;
    v = (b * dot(A0, diff) - a * dot(A1, diff)) / (a * c - b * b);
    if (!isfinite(v)) v = 0.5f;
    v = fminf(fmaxf(v, 0.f), 1.f);
    u = fminf(fmaxf(dot(lerp3(b0, b1, v) - a0, A0) / a, 0.f), 1.f);
    v = fminf(fmaxf(dot(lerp3(a0, a1, u) - b0, A1) / c, 0.f), 1.f);
}

// One surface contact at a vertex: penalty k (|gap| along n) + regularised Coulomb friction
// on the tangential displacement d (relative to the surface), contact.cuh:27-46.
__device__ __forceinline__ void surface_contact(f3 n, float gap, f3 d, float k, float h, float muS, float muK,
                                                float vslip, f3& f, sym3& H) {
    const float N = -k * gap;
    f = fma3(n, N, f);
    sym_add_scaled_outer(H, n, k);
    const f3 ut = fma3(n, -dot(n, d), d);
    const float ul = len(ut);
    // the slip speed over the regularisation speed, (ul / h) / vslip, as one division by the
    // slip length vslip h (which the static branch divides by as well)
    const float w = vslip * h;
    const float xr = ul / w;
    float kt;
    if (xr <= 1.f) kt = muS * N / w;
    else {
        const float s = 1.f - fminf(1.f, xr - 1.f);
        kt = fmaf(s, muS, (1.f - s) * muK) * N / ul;
    }
    f = fma3(ut, -kt, f);
    sym_sub_scaled_outer_minus_I(H, n, kt);
}

// Trilinear phi and its exact gradient at object-frame point p, contact.cuh:57-76, in three parts
// (the contact test finds the cell once for its block bound and its sample): the cell of p (false
// outside the lattice and on its upper faces), the cell's eight nodes, the interpolation.
__device__ __forceinline__ bool sdf_cell(const rs::GridDesc& g, f3 p, int& i, int& j, int& k) {
    const f3 u = (p - mk3(g.ox, g.oy, g.oz)) * g.invH;
    if (!(u.x >= 0.f && u.y >= 0.f && u.z >= 0.f && u.x < float(g.nx - 1) && u.y < float(g.ny - 1) &&
          u.z < float(g.nz - 1)))
        return false;
    i = (int)u.x; j = (int)u.y; k = (int)u.z;
    if (rs::kChecked && !(i >= 0 && j >= 0 && k >= 0 && i <= g.nx - 2 && j <= g.ny - 2 && k <= g.nz - 2)) {
        check_fail(g.status, rs::CHK_LATTICE);
        return false;
    }
    return true;
}
struct CellNodes {
    float c000, c001, c010, c011, c100, c101, c110, c111;
};
__device__ __forceinline__ CellNodes sdf_nodes(const rs::GridDesc& g, int i, int j, int k) {
    const int sy = g.nz, sx = g.ny * g.nz;
    const float* c = g.v + (size_t)i * sx + (size_t)j * sy + k;
    return CellNodes{__ldg(c), __ldg(c + 1), __ldg(c + sy), __ldg(c + sy + 1),
                     __ldg(c + sx), __ldg(c + sx + 1), __ldg(c + sx + sy), __ldg(c + sx + sy + 1)};
}
__device__ __forceinline__ void sdf_interp(const rs::GridDesc& g, f3 p, int i, int j, int k, const CellNodes& n,
                                           float& phi, f3& grad) {
    const f3 o = mk3(g.ox, g.oy, g.oz);
    const f3 fr = (p - fma3(mk3(float(i), float(j), float(k)), g.h, o)) * g.invH;
    const float fx = fminf(fmaxf(fr.x, 0.f), 1.f), fy = fminf(fmaxf(fr.y, 0.f), 1.f), fz = fminf(fmaxf(fr.z, 0.f), 1.f);
    const float dx00 = n.c100 - n.c000, dx01 = n.c101 - n.c001, dx10 = n.c110 - n.c010, dx11 = n.c111 - n.c011;
    const float c00 = fmaf(fx, dx00, n.c000), c01 = fmaf(fx, dx01, n.c001), c10 = fmaf(fx, dx10, n.c010),
                c11 = fmaf(fx, dx11, n.c011);
    const float dy0 = c10 - c00, dy1 = c11 - c01;
    const float c0 = fmaf(fy, dy0, c00), c1 = fmaf(fy, dy1, c01);
    phi = fmaf(fz, c1 - c0, c0);
    const float gx0 = fmaf(fy, dx10 - dx00, dx00), gx1 = fmaf(fy, dx11 - dx01, dx01);
    grad = mk3(fmaf(fz, gx1 - gx0, gx0), fmaf(fz, dy1 - dy0, dy0), c1 - c0) * g.invH;
}
__device__ __forceinline__ bool sdf_sample(const rs::GridDesc& g, f3 p, float& phi, f3& grad) {
    int i, j, k;
    if (!sdf_cell(g, p, i, j, k)) return false;
    sdf_interp(g, p, i, j, k, sdf_nodes(g, i, j, k), phi, grad);
    return true;
}

// Pose cache entry accessors (rs::Pose is 5 float4).
struct PoseV {
    f3 pos, vel, om, lo, hi;
    float4 q;
};
__device__ __forceinline__ PoseV load_pose(const float4* e) {
    const float4 a = e[0], b = e[1], c = e[2], d = e[3], f = e[4];
    PoseV P;
    P.pos = mk3(a.x, a.y, a.z);
    P.vel = mk3(a.w, c.x, c.y);
    P.q = b;
    P.om = mk3(c.z, c.w, d.x);
    P.lo = mk3(d.y, d.z, d.w);
    P.hi = mk3(f.x, f.y, f.z);
    return P;
}
__device__ __forceinline__ void store_pose(float4* e, f3 pos, float4 q, f3 vel, f3 om, f3 lo, f3 hi) {
    e[0] = make_float4(pos.x, pos.y, pos.z, vel.x);
    e[1] = q;
    e[2] = make_float4(vel.y, vel.z, om.x, om.y);
    e[3] = make_float4(om.z, lo.x, lo.y, lo.z);
    e[4] = make_float4(hi.x, hi.y, hi.z, 0.f);
}

// World AABB of the lattice box [lo_o, hi_o] under (pos, q), contact.cuh:79-87.
__device__ __forceinline__ void world_box(f3 lo_o, f3 hi_o, f3 pos, float4 q, f3& lo, f3& hi) {
    lo = mk3(INFINITY, INFINITY, INFINITY);
    hi = mk3(-INFINITY, -INFINITY, -INFINITY);
#pragma unroll
    for (int c = 0; c < 8; c++) {
        const f3 corner = mk3((c & 1) ? hi_o.x : lo_o.x, (c & 2) ? hi_o.y : lo_o.y, (c & 4) ? hi_o.z : lo_o.z);
        const f3 w = qrot(q, corner) + pos;
        lo = mk3(fminf(lo.x, w.x), fminf(lo.y, w.y), fminf(lo.z, w.z));
        hi = mk3(fmaxf(hi.x, w.x), fmaxf(hi.y, w.y), fmaxf(hi.z, w.z));
    }
}

// Exact early out: the trilinear field inside a lattice block is at least the block's smallest
// node value, so a block whose bound clears the radius (by more than the rounding of the
// interpolation, 1e-5) cannot produce gap < 0. The bound of the block holding cell (i, j, k);
// false (no bound: the sample decides) when a checked build finds the index out of range.
// `btab`: the CTA's shared-memory copy of the bound tables (nullptr: read them from L2).
__device__ __forceinline__ bool sdf_block_bound(const rs::GridDesc& g, const float* btab, int i, int j, int k,
                                                float& bound) {
    const int bi = i / rs::kSdfBlock, bj = j / rs::kSdfBlock, bk = k / rs::kSdfBlock;
    const int idx = (bi * g.by + bj) * g.bz + bk;
    if (rs::kChecked && !(bi >= 0 && bj >= 0 && bk >= 0 && bj < g.by && bk < g.bz && idx < g.bcount)) {
        check_fail(g.status, rs::CHK_BLOCK);
        return false;
    }
    bound = btab ? btab[g.boff + idx] : __ldg(g.bmin + idx);
    return true;
}

// How far the probe (pos - P.pos) + d of a vertex can move (|d|) before it could touch lattice g
// at radius R, from its position at d = 0 (the rotation into the lattice preserves |d|):
//  - outside the lattice: the distance back into it (no contact outside, sdf_sample);
//  - inside: (phi(0) - R) / L, since phi(d) >= phi(0) - L |d| (GridDesc::lip_inv).
// Margins (1e-4 relative, 1e-6 m outside, 1e-5 m on phi) cover the FP32 evaluation of both the
// probe and phi, so a probe with |d| below the slack has gap >= 0 in sdf_contact_at. A negative
// slack means "may touch at any |d|".
__device__ __forceinline__ float sdf_slack(const rs::GridDesc& g, const PoseV& P, f3 pos, float R) {
    const f3 po = qrot(qconj(P.q), pos - P.pos);
    const f3 u = (po - mk3(g.ox, g.oy, g.oz)) * g.invH;
    const f3 ex = mk3(fmaxf(fmaxf(-u.x, u.x - float(g.nx - 1)), 0.f), fmaxf(fmaxf(-u.y, u.y - float(g.ny - 1)), 0.f),
                      fmaxf(fmaxf(-u.z, u.z - float(g.nz - 1)), 0.f));
    const float e2 = dot(ex, ex);
    if (e2 > 0.f) return sqrtf(e2) * g.h * 0.9999f - 1e-6f;
    float phi;
    f3 gr;
    if (!sdf_sample(g, po, phi, gr)) return -1.f;  // on the lattice's upper faces: evaluate every iteration
    return (phi - R - 1e-5f) * g.lip_inv * 0.9999f;
}

// Contact of a vertex with one posed lattice at probe (pos - P.pos) + d, contact.cuh:94-110.
__device__ __forceinline__ bool sdf_contact_at(const rs::GridDesc& g, const PoseV& P, f3 pos, f3 d, float h, float R,
                                               bool moving, bool skip, const float* btab, f3& n, float& gap, f3& dRel) {
    float phi;
    f3 gr;
    const f3 po = qrot(qconj(P.q), (pos - P.pos) + d);
    int i, j, k;
    if (!sdf_cell(g, po, i, j, k)) return false;  // the cell once, for the block bound and the sample
    float bound = 0.f;
    if (skip && sdf_block_bound(g, btab, i, j, k, bound) && bound - R > 1e-5f) return false;
    sdf_interp(g, po, i, j, k, sdf_nodes(g, i, j, k), phi, gr);
    gap = phi - R;
    if (gap >= 0.f) return false;
    const float g2 = dot(gr, gr);
    if (!(g2 > 0.f)) return false;
    // the unit normal by the reciprocal square root with one Newton step (within about 1 ulp),
    // not a square root and three divisions: this sits on the critical path of every lane in
    // contact, which its CTA waits for at the next barrier
    n = qrot(P.q, gr * rsqrt_nr(g2));
    dRel = d;
    if (moving) dRel = fma3(P.vel + cross(P.om, pos - P.pos), -h, dRel);
    return true;
}

}  // namespace rsd
