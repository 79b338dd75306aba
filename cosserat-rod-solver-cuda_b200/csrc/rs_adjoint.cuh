// rs_adjoint.cuh -- device pieces of the frame adjoint shared by the CTA-resident adjoint kernel
// (rs_adjoint.cu) and the per-launch adjoint for contact groups larger than one CTA
// (rs_adjoint_plain.cu): reverse of the contact laws, of the SDF sample, of the closest points
// and of the rope-rope barrier/friction term and step limit.
#pragma once

#include <cuda_runtime.h>

#include "rs_device.cuh"
#include "rs_substep.cuh"
#include "rs_types.h"

namespace rs {
namespace {

using namespace rsd;


__device__ __forceinline__ float4 zero4() { return make_float4(0.f, 0.f, 0.f, 0.f); }
__device__ __forceinline__ f3 ld3(const float* a, int u) { return mk3(a[3 * u], a[3 * u + 1], a[3 * u + 2]); }
__device__ __forceinline__ void st3(float* a, int u, f3 v) { a[3 * u] = v.x; a[3 * u + 1] = v.y; a[3 * u + 2] = v.z; }

// Transposed Jacobian of the tangent t(q) = q e_x q*.
// The factor 2 is applied to tb first (exact: a power of two), each component is an fmaf chain.
__device__ __forceinline__ float4 tangent_vjp(float4 q, f3 tb) {
    const f3 t2 = tb * 2.f;
    return make_float4(fmaf(q.z, t2.z, fmaf(q.y, t2.y, q.x * t2.x)), fmaf(-q.w, t2.z, fmaf(q.x, t2.y, -q.y * t2.x)),
                       fmaf(q.x, t2.z, fmaf(q.w, t2.y, -q.z * t2.x)), fmaf(-q.y, t2.z, fmaf(q.z, t2.y, q.w * t2.x)));
}

// Contact law (contact.cuh:27-46) reversed: f += n N - ut kt, H += k nnᵀ - kt (nnᵀ - I), with
// N = -k gap and ut = d - n (n.d). Given F̄ and H̄ = -e δᵀ: adds to d̄, returns the adjoints of
// the gap, of the penalty stiffness k and of the normal n.
__device__ __forceinline__ void surface_contact_bwd(f3 n, float gap, f3 d, float k, float h, float muS, float muK,
                                                    float eps, f3 Fb, f3 e, f3 del, f3& db, float& gapb, float& kb,
                                                    f3& nb) {
    const float nHn = -dot(n, e) * dot(n, del), trHb = -dot(e, del);
    const float N = -k * gap;
    const f3 ut = d - n * dot(n, d);
    const float ul = len(ut);
    const float w = eps * h, x = ul / w;  // the forward's slip ratio (surface_contact)
    float Nb = dot(n, Fb);
    kb = nHn;
    float kt, mu = 0.f, xr = 0.f;
    if (x <= 1.f) kt = muS * N / w;
    else {
        xr = x - 1.f;
        const float sw = 1.f - fminf(1.f, xr);
        mu = sw * muS + (1.f - sw) * muK;
        kt = mu * N / ul;
    }
    f3 utb = Fb * (-kt);
    const float ktb = -dot(ut, Fb) - (nHn - trHb);
    if (x <= 1.f) Nb += ktb * muS / w;
    else {
        Nb += ktb * mu / ul;
        float ulb = -ktb * mu * N / (ul * ul);
        if (xr < 1.f) ulb -= ktb * (muS - muK) * N / ul / w;
        utb += ut * (ulb / ul);
    }
    db += utb - n * dot(n, utb);
    kb += -gap * Nb;
    gapb = -k * Nb;
    // normal: f's n N, ut's -n (n.d), H's (k - kt) nnᵀ with (H̄ + H̄ᵀ) n = -e (δ.n) - δ (e.n)
    nb = Fb * N - utb * dot(n, d) - d * dot(utb, n) + (e * (-dot(del, n)) - del * dot(e, n)) * (k - kt);
}

// Trilinear sample (contact.cuh:57-76) with the field's Hessian in lattice-fraction coordinates
// (zero diagonal): hxy, hxz, hyz of d²φ / df_a df_b.
__device__ __forceinline__ bool sdf_sample_hess(const GridDesc& g, f3 p, float& phi, f3& grad, float& hxy, float& hxz,
                                                float& hyz) {
    if (!sdf_sample(g, p, phi, grad)) return false;
    const f3 o = mk3(g.ox, g.oy, g.oz);
    const f3 u = (p - o) * g.invH;
    const int i = (int)u.x, j = (int)u.y, k = (int)u.z;
    const f3 fr = (p - (o + mk3(float(i), float(j), float(k)) * g.h)) * g.invH;
    const float fx = fminf(fmaxf(fr.x, 0.f), 1.f), fy = fminf(fmaxf(fr.y, 0.f), 1.f), fz = fminf(fmaxf(fr.z, 0.f), 1.f);
    const int sy = g.nz, sx = g.ny * g.nz;
    const float* c = g.v + (size_t)i * sx + (size_t)j * sy + k;
    const float c000 = __ldg(c), c001 = __ldg(c + 1), c010 = __ldg(c + sy), c011 = __ldg(c + sy + 1);
    const float c100 = __ldg(c + sx), c101 = __ldg(c + sx + 1), c110 = __ldg(c + sx + sy), c111 = __ldg(c + sx + sy + 1);
    const float dx00 = c100 - c000, dx01 = c101 - c001, dx10 = c110 - c010, dx11 = c111 - c011;
    const float D = (dx11 - dx01) - (dx10 - dx00);
    hxy = (dx10 - dx00) + fz * D;
    hxz = (dx01 - dx00) + fy * D;
    hyz = ((c011 - c001) + fx * (dx11 - dx01)) - ((c010 - c000) + fx * (dx10 - dx00));
    return true;
}

// Mesh contacts of one vertex reversed (static poses; contact.cuh:94-110, then the contact law):
// p_o = R(q)ᵀ((x - P) + d), gap = φ(p_o) - r, n = R(q) ∇φ / |∇φ|. Adds to d̄ and x̄, returns the
// adjoint of the penalty stiffness.
__device__ __forceinline__ float mesh_contact_bwd(const FrameArgs& a, const float4* cache, uint64_t cand, f3 x, f3 d,
                                                  float kc, float h, f3 Fb, f3 e, f3 del, f3& db, f3& xb) {
    float kbs = 0.f;
    for (uint64_t mm = cand; mm; mm &= mm - 1ull) {
        const int m = __ffsll((long long)mm) - 1;
        const PoseV P = load_pose(cache + m * kPoseF4);
        const GridDesc& G = a.grids[m];
        const f3 po = qrot(qconj(P.q), (x - P.pos) + d);
        float phi, hxy, hxz, hyz;
        f3 gr;
        if (!sdf_sample_hess(G, po, phi, gr, hxy, hxz, hyz)) continue;
        const float gap = phi - a.c_radius;
        if (gap >= 0.f) continue;
        const float g2 = dot(gr, gr);
        if (!(g2 > 0.f)) continue;
        const float il = rsqrt_nr(g2);  // the forward's normalisation (sdf_contact_at)
        const f3 gh = gr * il;
        const f3 nrm = qrot(P.q, gh);
        float gapb, kb;
        f3 nb;
        surface_contact_bwd(nrm, gap, d, kc, h, G.muS, G.muK, a.c_vslip, Fb, e, del, db, gapb, kb, nb);
        kbs += kb;
        const f3 ghb = qrot(qconj(P.q), nb);
        const f3 grb = (ghb - gh * dot(gh, ghb)) * il;
        const float inv2 = G.invH * G.invH;
        const f3 pob = gr * gapb + mk3(hxy * grb.y + hxz * grb.z, hxy * grb.x + hyz * grb.z, hxz * grb.x + hyz * grb.y) * inv2;
        const f3 wv = qrot(P.q, pob);
        xb += wv;
        db += wv;
    }
    return kbs;
}

// seg_closest (Common.h:327-345, with a0 = 0) reversed: given the adjoints of the returned
// (u, v), adds those of a1 = A, b0 = B0, b1 = B1. Each clamp passes its adjoint inside [0, 1],
// ends included; the fallback for parallel segments (a non-finite first v) is a constant.
__device__ __forceinline__ void seg_closest_bwd(f3 A, f3 B0, f3 B1, float ub, float vb, f3& Ab, f3& B0b, f3& B1b) {
    const f3 E = B1 - B0;
    const float a = dot(A, A), b = dot(A, E), c = dot(E, E);
    const float AB0 = dot(A, B0), EB0 = dot(E, B0);
    const float Den = a * c - b * b, t0 = (b * AB0 - a * EB0) / Den;
    const bool fin = isfinite(t0);
    const float v0 = fin ? t0 : 0.5f;
    const float v0c = fminf(fmaxf(v0, 0.f), 1.f);
    const f3 Bv = lerp3(B0, B1, v0c);
    const float tu = dot(Bv, A) / a;
    const float u = fminf(fmaxf(tu, 0.f), 1.f);
    const f3 Au = lerp3(zero3(), A, u) - B0;
    const float tv = dot(Au, E) / c;
    f3 Ea = zero3(), Aa = zero3(), B0a = zero3();  // adjoints in the (A, B0, E = B1 - B0) parametrisation
    if (tv >= 0.f && tv <= 1.f) {
        const float Nb = vb / c;
        ub += Nb * dot(A, E);
        Aa += E * (Nb * u);
        B0a -= E * Nb;
        Ea += Au * Nb + E * (-2.f * vb * tv / c);
    }
    if (tu >= 0.f && tu <= 1.f) {
        const float Mb = ub / a;
        const f3 Bvb = A * Mb;
        B0a += Bvb;
        Ea += Bvb * v0c;
        Aa += Bv * Mb + A * (-2.f * ub * tu / a);
        if (fin && v0 >= 0.f && v0 <= 1.f) {
            const float t0b = dot(Bvb, E);
            const float Numb = t0b / Den, Denb = -t0b * t0 / Den;
            const float bb = Numb * AB0 - 2.f * b * Denb, aa = -Numb * EB0 + Denb * c, cc = Denb * a;
            const float AB0b = Numb * b, EB0b = -Numb * a;
            Aa += E * bb + A * (2.f * aa) + B0 * AB0b;
            Ea += A * bb + E * (2.f * cc) + B0 * EB0b;
            B0a += A * AB0b + E * EB0b;
        }
    }
    Ab += Aa;
    B1b += Ea;
    B0b += B0a - Ea;
}

// One rope-rope candidate reversed (cosserat.cu:99-157). Segment (x0, x1) with iterates
// (d0, d1) against segment (y0, y1) with iterates (e0, e1): the term adds f, H to the segment's
// first vertex with weight wa = 1 - u and f2, H2 to its second with weight wb = u. Given F̄ and
// H̄ = -e δᵀ of both (Fa, ea, la; Fc, ec, lc), adds the adjoints of the eight inputs. Barrier:
// s = (|n| - 2r) / b clamped below at 1e-3, force ff and stiffness dH of the log barrier; friction
// f1 = min(kf, μ ff / |uu|) along the tangential slip uu.
struct PairGrad {
    f3 x0, x1, y0, y1, d0, d1, e0, e1;
};
__device__ __forceinline__ void collision_bwd(const FrameArgs& a, float damp, f3 x0, f3 x1, f3 y0, f3 y1, f3 d0, f3 d1,
                                              f3 e0, f3 e1, f3 Fa, f3 ea, f3 la, f3 Fc, f3 ec, f3 lc, PairGrad& o) {
    const f3 A = (x1 - x0) + (d1 - d0), B0 = (y0 - x0) + (e0 - d0), B1 = (y1 - x0) + (e1 - d0);
    float u, v;
    seg_closest(zero3(), A, B0, B1, u, v);
    const f3 dpos = lerp3(x0, x1, u) - lerp3(y0, y1, v);
    const f3 ddpos = lerp3(d0, d1, u) - lerp3(e0, e1, v);
    const f3 raw = dpos + ddpos;
    const float dist = len(raw);
    if (!(dist > 0.f)) return;
    const f3 nr = raw * (1.f / dist);
    const float wb = u, wa = 1.f - u;
    const float invb = 1.f / a.rc_barrier, kCol = a.rc_kcol * invb;
    const float sr = (dist - 2.f * a.rc_radius) * invb;
    if (sr > 1.f) return;
    const float sd = fmaxf(sr, 1e-3f);
    const float invd = 1.f / sd, logd = logf(sd);
    const float dH = (-3.f + (2.f + invd) * invd - 2.f * logd) * kCol * invb;
    const float ff = -(1.f - sd) * (sd - 1.f + 2.f * sd * logd) * invd * kCol;
    const float Ga = dot(Fa, nr), Gc = dot(Fc, nr), nd0 = dot(nr, d0), nd1 = dot(nr, d1);
    const float nHa = -dot(nr, ea) * dot(nr, la), nHc = -dot(nr, ec) * dot(nr, lc);
    const float trA = -dot(ea, la), trC = -dot(ec, lc);
    // (H̄ + H̄ᵀ) n for H̄ = -e δᵀ
    const f3 symS = (ea * (-dot(la, nr)) - la * dot(ea, nr)) * (wa * wa) + (ec * (-dot(lc, nr)) - lc * dot(ec, nr)) * (wb * wb);
    const float nHs = wa * wa * nHa + wb * wb * nHc, trS = wa * wa * trA + wb * wb * trC;
    const float dp = 1.f + damp;
    float ffb = Ga * wa + Gc * wb;
    const float dHb = -damp * (Ga * wa * wa * nd0 + Gc * wb * wb * nd1) + dp * nHs;
    float wab = Ga * ff - 2.f * damp * dH * wa * Ga * nd0 + 2.f * wa * dp * dH * nHa;
    float wbb = Gc * ff - 2.f * damp * dH * wb * Gc * nd1 + 2.f * wb * dp * dH * nHc;
    f3 nb = Fa * (ff * wa - damp * dH * wa * wa * nd0) + Fc * (ff * wb - damp * dH * wb * wb * nd1) +
            d0 * (-damp * dH * wa * wa * Ga) + d1 * (-damp * dH * wb * wb * Gc) + symS * (dp * dH);
    f3 d0b = nr * (-damp * dH * wa * wa * Ga), d1b = nr * (-damp * dH * wb * wb * Gc);
    f3 ddb = zero3();  // adjoint of ddpos
    const f3 uu = ddpos - nr * dot(nr, ddpos);
    const float ul = len(uu);
    if (ul > 0.f) {
        const float ratio = a.rc_mu * ff / ul;
        const float f1 = fminf(a.rc_kfric, ratio);
        const f3 Fu = Fa * wa + Fc * wb;
        const float f1b = -dot(uu, Fu) - (nHs - trS);
        wab += -f1 * dot(uu, Fa) - 2.f * wa * f1 * (nHa - trA);
        wbb += -f1 * dot(uu, Fc) - 2.f * wb * f1 * (nHc - trC);
        nb -= symS * f1;
        f3 uub = Fu * (-f1);
        if (!(a.rc_kfric < ratio)) {  // f1 = μ ff / |uu|
            ffb += f1b * a.rc_mu / ul;
            uub += uu * (-f1b * ratio / (ul * ul));
        }
        ddb += uub - nr * dot(nr, uub);
        nb -= uub * dot(nr, ddpos) + ddpos * dot(nr, uub);
    }
    float ub = wbb - wab, distb = 0.f;
    if (sr >= 1e-3f) {
        const float pm = 1.f - sd, qv = sd - 1.f + 2.f * sd * logd;
        const float ffp = -kCol * ((-qv + pm * (3.f + 2.f * logd)) * invd - pm * qv * invd * invd);
        const float dHp = -2.f * (invd * invd + invd * invd * invd + invd) * kCol * invb;
        distb = (ffb * ffp + dHb * dHp) * invb;
    }
    const f3 rawb = (nb - nr * dot(nr, nb)) * (1.f / dist) + nr * distb;
    ddb += rawb;
    o.x0 += rawb * wa;
    o.x1 += rawb * wb;
    o.y0 -= rawb * (1.f - v);
    o.y1 -= rawb * v;
    ub += dot(rawb, x1 - x0) + dot(ddb, d1 - d0);
    const float vbv = -dot(rawb, y1 - y0) - dot(ddb, e1 - e0);
    d0b += ddb * wa;
    d1b += ddb * wb;
    o.e0 -= ddb * (1.f - v);
    o.e1 -= ddb * v;
    f3 Ab = zero3(), B0b = zero3(), B1b = zero3();
    seg_closest_bwd(A, B0, B1, ub, vbv, Ab, B0b, B1b);
    o.x1 += Ab;
    d1b += Ab;
    o.y0 += B0b;
    o.e0 += B0b;
    o.y1 += B1b;
    o.e1 += B1b;
    const f3 sb = Ab + B0b + B1b;
    o.x0 -= sb;
    d0b -= sb;
    o.d0 += d0b;
    o.d1 += d1b;
}

// Step limit of segment t reversed (recomputeStepLimitKernel, collision.cu:103-136): the limit is
// the least of padding - detection radius (padding = scaled radius + |y|, y = v h + g h²) and
// 0.45 x each listed candidate's distance at the substep start; its adjoint goes to the argument
// that attained it (the first on ties, as the forward's running minimum). Returns the adjoint of
// y (padding branch) and adds the position adjoints (candidate branch).
__device__ __forceinline__ f3 step_limit_bwd(const FrameArgs& a, int dv, int ncol, const float4* X, f3 p, f3 p1, float pad,
                                             f3 y, float limb, f3& xb0, f3& xb1, int& jo, f3& xbj0, f3& xbj1) {
    jo = -1;
    const f3 a1 = p1 - p;
    float best = pad - a.det_radius;
    int arg = -1;
    for (int cc = 0; cc < ncol; cc++) {
        const int j = a.cols[(size_t)cc * a.n + dv];
        const float val = step_limit_of(p, a1, xyz(X[j]), xyz(X[j + 1]));
        if (val < best) { best = val; arg = j; }
    }
    if (arg < 0) {
        const float ly = len(y);
        return ly > 0.f ? y * (limb / ly) : zero3();
    }
    const f3 b0 = xyz(X[arg]) - p, b1 = xyz(X[arg + 1]) - p;
    float u, v;
    seg_closest(zero3(), a1, b0, b1, u, v);
    const f3 nn = a1 * u - lerp3(b0, b1, v);
    const float l = len(nn);
    if (!(l > 0.f)) return zero3();
    const f3 nnb = nn * ((1.f - 0.1f) * 0.5f * limb / l);
    f3 Ab = nnb * u, B0b = nnb * (-(1.f - v)), B1b = nnb * (-v);
    seg_closest_bwd(a1, b0, b1, dot(nnb, a1), -dot(nnb, b1 - b0), Ab, B0b, B1b);
    xb1 += Ab;
    xb0 -= Ab + B0b + B1b;
    jo = arg;
    xbj0 = B0b;
    xbj1 = B1b;
    return zero3();
}

__device__ __forceinline__ void atomic_add3(float4* p, f3 v) {
    atomicAdd(&p->x, v.x);
    atomicAdd(&p->y, v.y);
    atomicAdd(&p->z, v.z);
}

}  // namespace
}  // namespace rs
