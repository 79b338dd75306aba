// rs_adjoint_plain.cu -- the frame adjoint as a sequence of per-vertex launches over HBM arrays,
// for batches whose rope-rope contact groups do not fit one CTA and for the plain engine.
//
// The arithmetic is the CTA-resident adjoint kernel's (rs_adjoint.cu), split where that kernel
// waits at a barrier; a launch boundary is a grid-wide barrier, so the rope-rope pairs of one
// contact group may span any number of CTAs. Per substep, from the tape:
//   init, detect                        the substep's start state, candidate lists, step limits
//   num_itr x (position, frame)         the iterates d^k, q^k into HBM (the plain engine's sweep)
//   end                                 velocity and drag reversed
//   num_itr x (rev_frame, rev_position, rev_stretch)
//                                       frame step reversed (+ collision Hessians at d^k); the
//                                       position step's local solve, contacts and step limit
//                                       reversed; stretch and rope-rope pairs reversed, the other
//                                       segment's shares added with float atomics
//   limit, start                        step limits, inertial prediction and root program reversed
// Vertex-local adjoint state (x̄, v̄, q̄, parameter adjoints) lives in HBM between launches.
#include "rs_adjoint.cuh"
#include "rs_kernels.h"

namespace rs {

namespace {

constexpr int kPosBlock = 128;     // position recompute: 127 owned vertices + the previous halo vertex
constexpr int kOwned = kPosBlock - 1;
constexpr int kOwnedRope = kPosBlock / 2 - 1;  // rope-rope recompute: two threads per vertex
constexpr int kBlock = 128;

__device__ __forceinline__ const float4* static_poses(const FrameArgs& a, int env) {
    return reinterpret_cast<const float4*>(a.poses + (size_t)env * kMaxSdf);
}

__device__ __forceinline__ void add3(float4* p, f3 v) {
    const float4 o = *p;
    *p = make_float4(o.x + v.x, o.y + v.y, o.z + v.z, o.w);
}

// Adjoints of the frame-end state into the accumulators; the pair-share arrays start at zero.
__global__ void padj_load_kernel(const FrameArgs* __restrict__ pa, const AdjArgs g, PlainAdjBufs b, int n) {
    const FrameArgs& a = *pa;
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const int u = a.topo[d].z;
    b.gx[d] = f4(g.g_pos ? ld3(g.g_pos, u) : zero3(), 0.f);
    b.gv[d] = f4(g.g_vel ? ld3(g.g_vel, u) : zero3(), 0.f);
    b.gl[d] = f4(g.g_lvel ? ld3(g.g_lvel, u) : zero3(), 0.f);
    b.gq[d] = g.g_q ? reinterpret_cast<const float4*>(g.g_q)[u] : zero4();
    b.gp0[d] = zero4();
    b.gv0[d] = zero4();
    b.gp1[d] = zero4();
    b.cd[d] = zero4();
    b.cd[n + d] = zero4();
    b.cx[d] = zero4();
}

// The substep's start state (after its root program) from the tape; inertial prediction.
__global__ void padj_init_kernel(const FrameArgs* __restrict__ pa, const AdjArgs g, PlainAdjBufs b, int n, int s) {
    const FrameArgs& a = *pa;
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const float im = a.pos[d].w;
    const float4* tp = g.tape + (size_t)s * 4 * n + a.topo[d].z;
    const float4 t0 = tp[0], t1 = tp[n];
    const f3 p = xyz(t0), v = xyz(t1), lvin = xyz(tp[2 * (size_t)n]);
    const f3 gv = mk3(a.gx, a.gy, a.gz);
    f3 dx, y;
    init_vertex(v, lvin, im, a.h, a.last_h, gv, dot(gv, gv), dx, y);
    b.x[d] = f4(p, im);
    b.ld[d] = f4(dx, 1.f);
    b.lq[d] = tp[3 * (size_t)n];
    b.y[d] = f4(y, 0.f);
    b.cand[d] = (uint64_t)(uint32_t)__float_as_int(t0.w) | ((uint64_t)(uint32_t)__float_as_int(t1.w) << 32);
    if (a.rope_contact) a.pad[d] = a.sdet_radius + len(y);
}

// Rope-rope detection and step limit of segment d over its contact group (the frame kernels').
__global__ void padj_detect_kernel(const FrameArgs* __restrict__ pa, PlainAdjBufs b, int n) {
    const FrameArgs& a = *pa;
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    if (!(a.topo[d].x & F_NEXT)) {
        a.ncols[d] = 0;
        a.maxstep[d] = INFINITY;
        return;
    }
    const int4 gr = a.grp[d];
    float lim;
    const int cnt = detect_group(
        a, d, d, gr.x, gr.y, gr.z, gr.w, xyz(b.x[d]), xyz(b.x[d + 1]), [&](int j) { return a.pad[j]; },
        [&](int j) { return a.topo[j].x; }, [&](int j) { return xyz(b.x[j]); }, lim);
    a.ncols[d] = cnt < kMaxCols ? cnt : kMaxCols;
    a.maxstep[d] = lim;
}

// Position step k recomputed (SNAPSHOT): d^{k+1} and the step limit's scale into ld[k+1].
template <int SURF, bool ROPE>
__global__ void __launch_bounds__(kPosBlock) padj_position_kernel(const FrameArgs* __restrict__ pa, PlainAdjBufs b, int n,
                                                                  int k) {
    const FrameArgs& a = *pa;
    __shared__ float4 sfa[kPosBlock], sfb[kPosBlock];
    __shared__ float sfc[kPosBlock];
    const int lt = threadIdx.x;
    const int d = blockIdx.x * kOwned + lt - 1;
    const bool valid = d >= 0 && d < n;
    const float4* Dk = b.ld + (size_t)k * n;
    uint32_t fl = 0;
    f3 f = zero3(), f2 = zero3(), dx = zero3();
    sym3 H = sym_zero(), H2 = sym_zero();
    float im = 0.f;
    bool touched = false;
    if (valid) {
        const int4 tp = a.topo[d];
        fl = (uint32_t)tp.x;
        const float4 P = b.x[d];
        im = P.w;
        const VConst c = vertex_constants(a, im, a.vel[d].w, a.lvel[d].w);
        const bool hasNext = fl & F_NEXT;
        dx = xyz(Dk[d]);
        const f3 p1 = hasNext ? xyz(b.x[d + 1]) : zero3();
        const f3 p1dx = hasNext ? xyz(Dk[d + 1]) : zero3();
        const float4* cache = (SURF == SURF_MESHES) ? static_poses(a, tp.w) : nullptr;
        const uint64_t cand = (SURF == SURF_MESHES) ? b.cand[d] : 0ull;
        const float damp = a.damping / a.h;
        touched = position_terms<SURF>(a, cache, cand, c, hasNext, xyz(P), p1, dx, p1dx, xyz(b.y[d]),
                                       b.lq[(size_t)k * n + d], damp, f, H, f2, H2);
        if constexpr (ROPE)
            collision_sectors(a, hasNext ? a.ncols[d] : 0, d, b.x, Dk, damp, xyz(P), p1, dx, p1dx, f, f2, H, H2);
    }
    sfa[lt] = f4(f2, H2.xx);
    sfb[lt] = make_float4(H2.yy, H2.zz, H2.xy, H2.xz);
    sfc[lt] = H2.yz;
    __syncthreads();
    if (!valid || lt == 0) return;  // the halo vertex belongs to the previous block
    if (fl & F_PREV) {
        const float4 fa = sfa[lt - 1], fb = sfb[lt - 1];
        f += xyz(fa);
        H.xx += fa.w; H.yy += fb.x; H.zz += fb.y; H.xy += fb.z; H.xz += fb.w; H.yz += sfc[lt - 1];
    }
    float sc = 1.f;
    if constexpr (ROPE) {
        const float lim = (fl & F_PREV) ? fminf(a.maxstep[d], a.maxstep[d - 1]) : a.maxstep[d];
        sc = position_solve_limited(dx, f, H, a.accel, im, lim);
    } else {
        position_solve(dx, f, H, a.accel, im, !touched);
    }
    b.ld[(size_t)(k + 1) * n + d] = f4(dx, sc);
}

// Position step k recomputed with rope-rope terms, two threads per vertex: the reference's two
// candidate sectors (even candidates joining the own terms, odd ones a partial added after them,
// cosserat.cu:99-182) on their own threads, the same sums in the same order as
// collision_sectors().
template <int SURF>
__global__ void __launch_bounds__(kPosBlock) padj_position_rope_kernel(const FrameArgs* __restrict__ pa, PlainAdjBufs b,
                                                                       int n, int k) {
    const FrameArgs& a = *pa;
    constexpr int V = kPosBlock / 2;
    __shared__ float4 so[V][5];  // sector 1: fo, f2o, Ho, H2o
    __shared__ float4 sfa[V], sfb[V];
    __shared__ float sfc[V];
    const int lt = threadIdx.x, lv = lt >> 1, sec = lt & 1;
    const int d = blockIdx.x * kOwnedRope + lv - 1;
    const bool valid = d >= 0 && d < n;
    const float4* Dk = b.ld + (size_t)k * n;
    uint32_t fl = 0;
    f3 f = zero3(), f2 = zero3(), dx = zero3();
    sym3 H = sym_zero(), H2 = sym_zero();
    float im = 0.f;
    int nc = 0;
    if (valid) {
        const int4 tp = a.topo[d];
        fl = (uint32_t)tp.x;
        const float4 P = b.x[d];
        im = P.w;
        const bool hasNext = fl & F_NEXT;
        dx = xyz(Dk[d]);
        const f3 p1 = hasNext ? xyz(b.x[d + 1]) : zero3();
        const f3 p1dx = hasNext ? xyz(Dk[d + 1]) : zero3();
        const float damp = a.damping / a.h;
        nc = hasNext ? a.ncols[d] : 0;
        if (sec == 0) {
            const VConst c = vertex_constants(a, im, a.vel[d].w, a.lvel[d].w);
            const float4* cache = (SURF == SURF_MESHES) ? static_poses(a, tp.w) : nullptr;
            const uint64_t cand = (SURF == SURF_MESHES) ? b.cand[d] : 0ull;
            position_terms<SURF>(a, cache, cand, c, hasNext, xyz(P), p1, dx, p1dx, xyz(b.y[d]), b.lq[(size_t)k * n + d],
                                 damp, f, H, f2, H2);
        }
        for (int cc = sec; cc < nc; cc += 2) {
            const int j = a.cols[(size_t)cc * n + d];
            collision_term(a, damp, xyz(P), p1, dx, p1dx, xyz(b.x[j]), xyz(b.x[j + 1]), xyz(Dk[j]), xyz(Dk[j + 1]), f, f2,
                           H, H2);
        }
        if (sec == 1) {
            so[lv][0] = f4(f, f2.x);
            so[lv][1] = make_float4(f2.y, f2.z, H.xx, H.yy);
            so[lv][2] = make_float4(H.zz, H.xy, H.xz, H.yz);
            so[lv][3] = make_float4(H2.xx, H2.yy, H2.zz, H2.xy);
            so[lv][4] = make_float4(H2.xz, H2.yz, 0.f, 0.f);
        }
    }
    __syncthreads();
    if (sec == 0) {
        if (valid && nc > 1) {
            const float4 o0 = so[lv][0], o1 = so[lv][1], o2 = so[lv][2], o3 = so[lv][3], o4 = so[lv][4];
            f += xyz(o0);
            f2 += mk3(o0.w, o1.x, o1.y);
            sym_add(H, sym3{o1.z, o1.w, o2.x, o2.y, o2.z, o2.w});
            sym_add(H2, sym3{o3.x, o3.y, o3.z, o3.w, o4.x, o4.y});
        }
        sfa[lv] = f4(f2, H2.xx);
        sfb[lv] = make_float4(H2.yy, H2.zz, H2.xy, H2.xz);
        sfc[lv] = H2.yz;
    }
    __syncthreads();
    if (sec != 0 || !valid || lv == 0) return;  // the halo vertex belongs to the previous block
    if (fl & F_PREV) {
        const float4 fa = sfa[lv - 1], fb = sfb[lv - 1];
        f += xyz(fa);
        H.xx += fa.w; H.yy += fb.x; H.zz += fb.y; H.xy += fb.z; H.xz += fb.w; H.yz += sfc[lv - 1];
    }
    const float lim = (fl & F_PREV) ? fminf(a.maxstep[d], a.maxstep[d - 1]) : a.maxstep[d];
    const float sc = position_solve_limited(dx, f, H, a.accel, im, lim);
    b.ld[(size_t)(k + 1) * n + d] = f4(dx, sc);
}

// Frame step k recomputed: q^{k+1} into lq[k+1].
__global__ void padj_frame_kernel(const FrameArgs* __restrict__ pa, PlainAdjBufs b, int n, int k) {
    const FrameArgs& a = *pa;
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const float4* Lk = b.lq + (size_t)k * n;
    const float4* Dn = b.ld + (size_t)(k + 1) * n;
    const uint32_t fl = (uint32_t)a.topo[d].x;
    float4 q = Lk[d];
    if (!(fl & F_FIX_ORIENT) && (fl & F_NEXT)) {
        const f3 seg = (xyz(b.x[d + 1]) - xyz(b.x[d])) + (xyz(Dn[d + 1]) - xyz(Dn[d]));
        const bool hp = fl & F_PREV, hn = fl & F_NEXT_ORIENT;
        q = frame_update(q, seg, 1.f / a.vel[d].w, a.lvel[d].w, hp, hp ? Lk[d - 1] : q, hp ? a.qrest[d - 1] : q, hn,
                         hn ? Lk[d + 1] : q, a.qrest[d]);
    }
    b.lq[(size_t)(k + 1) * n + d] = q;
}

// End of substep reversed: x' = x + d, v' = drag(d / h), lv' = v.
__global__ void padj_end_kernel(const FrameArgs* __restrict__ pa, PlainAdjBufs b, int n) {
    const FrameArgs& a = *pa;
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const uint32_t fl = (uint32_t)a.topo[d].x;
    const int I = a.iters;
    const float im = a.pos[d].w, h = a.h, invH = 1.f / h;
    const f3 vb = xyz(b.gv[d]);
    float4 qb = b.gq[d];
    f3 db = xyz(b.gx[d]);
    f3 vbn = xyz(b.gl[d]);
    float4 qpart = zero4();
    if (im != 0.f) {
        const f3 ob = vb * (1.f - a.drag * h);
        f3 vbar = ob;
        if (a.drag_quad > 0.f) {
            const bool hasNext = fl & F_NEXT;
            const float4 tq = b.lq[(size_t)I * n + (hasNext ? d : d - 1)];
            const f3 tg = qtangent(tq);
            const f3 vv = xyz(b.ld[(size_t)I * n + d]) * invH;
            const float tv = dot(tg, vv);
            const f3 vt = tg * tv, vn = vv - vt;
            const float ln = len(vn), Dn = 1.f + a.drag_quad * ln * h;
            const float lt = len(vt), Dt = 1.f + a.drag_quad_t * lt * h;
            f3 vnb = ob / Dn;
            if (ln > 0.f) vnb -= vn * (a.drag_quad * h * dot(vn, ob) / (ln * Dn * Dn));
            f3 vtb = ob / Dt;
            if (lt > 0.f) vtb -= vt * (a.drag_quad_t * h * dot(vt, ob) / (lt * Dt * Dt));
            vbar = vnb;
            vtb -= vnb;
            const float tvb = dot(vtb, tg);
            vbar += tg * tvb;
            const float4 qg = tangent_vjp(tq, vtb * tv + vv * tvb);
            if (hasNext) qb = add4(qb, qg);
            else qpart = qg;
        }
        db += vbar * invH;
    } else {
        vbn += vb;  // a pinned vertex keeps its driven velocity
    }
    b.gq[d] = qb;
    b.qp[d] = qpart;
    b.td[d] = f4(db, 0.f);
    b.tn[d] = f4(vbn, 0.f);
    b.ty[d] = zero4();
    b.ms[d] = make_float2(0.f, 0.f);
}

// Frame step k reversed, q^{k+1}_t = normalize(vv b e1 + (|vv| + |b|) b); and the segment's
// collision Hessians at d^k (the position reverse needs H again).
template <bool ROPE>
__global__ void padj_rev_frame_kernel(const FrameArgs* __restrict__ pa, PlainAdjBufs b, int n, int k, int first) {
    const FrameArgs& a = *pa;
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const uint32_t fl = (uint32_t)a.topo[d].x;
    const bool hasNext = fl & F_NEXT, hasPrev = fl & F_PREV, nextOrient = fl & F_NEXT_ORIENT;
    const bool upd = hasNext && !(fl & F_FIX_ORIENT);
    const float4* Lq = b.lq + (size_t)k * n;
    const float4* Dn = b.ld + (size_t)(k + 1) * n;
    float4 qb = b.gq[d];
    if (first && a.drag_quad > 0.f && hasNext) qb = add4(qb, b.qp[d + 1]);
    float4 own = qb, toL = zero4(), toR = zero4();
    f3 su = zero3();
    if (upd) {
        own = zero4();
        const float ks = a.lvel[d].w, invl = 1.f / a.vel[d].w;
        const f3 p = xyz(b.x[d]), p1 = xyz(b.x[d + 1]);
        const f3 u = ((p1 - p) + (xyz(Dn[d + 1]) - xyz(Dn[d]))) * invl;
        const f3 vv = u * (-2.f * ks);
        const float4 q0 = Lq[d];
        float4 bq = zero4(), qp = zero4(), qn = zero4(), rp = zero4(), rn = zero4();
        float sp = 0.f, sn = 0.f;
        if (hasPrev) {
            qp = Lq[d - 1]; rp = a.qrest[d - 1];
            const float4 pr = qmul(qp, rp);
            sp = dot4(q0, pr) > 0.f ? 1.f : -1.f;
            bq = scale4(pr, sp);
        }
        if (nextOrient) {
            qn = Lq[d + 1]; rn = a.qrest[d];
            const float4 nx = qmul(qn, qconj(rn));
            sn = dot4(q0, nx) > 0.f ? 1.f : -1.f;
            bq = add4(bq, scale4(nx, sn));
        }
        float ilvv, ilb, lambda;  // the forward's z (frame_z), so the reverse linearises what ran
        const float4 z = frame_z(vv, bq, ilvv, ilb, lambda);
        const float izl = rsqrt_nr(dot4(z, z));
        const float4 qo = scale4(z, izl);
        const float4 zb = scale4(add4(qb, scale4(qo, -dot4(qo, qb))), izl);
        float4 bb = scale4(zb, lambda);
        const float lamb = dot4(zb, bq);
        f3 vvb = vv * (lamb * ilvv);
        bb = add4(bb, scale4(bq, lamb * ilb));
        const float4 Ab = scale4(qmul_e1(zb), -1.f);
        vvb += xyz(qmul(Ab, qconj(bq)));
        bb = add4(bb, scale4(qmul_pure(vv, Ab), -1.f));
        float4 gx = b.gx[d], gv = b.gv[d], gl = b.gl[d];
        gx.w += -2.f * dot(u, vvb);
        su = vvb * (-2.f * ks * invl);
        if (hasPrev) {
            toL = qmul(scale4(bb, sp), qconj(rp));
            gl.w += dot4(toL, qp) / sqrtf(dot4(rp, rp));
        }
        if (nextOrient) {
            toR = qmul(scale4(bb, sn), rn);
            gv.w += dot4(toR, qn) / sqrtf(dot4(rn, rn));
        }
        b.gx[d] = gx;
        b.gv[d] = gv;
        b.gl[d] = gl;
    }
    b.ea[d] = toL;
    b.eb[d] = toR;
    b.ec[d] = f4(su, 0.f);
    b.gq[d] = own;
    if constexpr (ROPE) {
        sym3 HcA = sym_zero(), HcB = sym_zero();
        if (hasNext) {
            const float4* Dk = b.ld + (size_t)k * n;
            f3 fd = zero3(), f2d = zero3();
            collision_sectors(a, a.ncols[d], d, b.x, Dk, a.damping / a.h, xyz(b.x[d]), xyz(b.x[d + 1]), xyz(Dk[d]),
                              xyz(Dk[d + 1]), fd, f2d, HcA, HcB);
        }
        b.ha0[d] = make_float4(HcA.xx, HcA.yy, HcA.zz, HcA.xy);
        b.ha1[d] = make_float4(HcA.xz, HcA.yz, 0.f, 0.f);
        b.hb0[d] = make_float4(HcB.xx, HcB.yy, HcB.zz, HcB.xy);
        b.hb1[d] = make_float4(HcB.xz, HcB.yz, 0.f, 0.f);
    }
}

// Position step k reversed: d^{k+1}_t = limit(d^k_t + a H_t^-1 F_t). Gathers the frame step's
// shares first (rotor and segment adjoints of the neighbours, the pairs' d̄ shares of step k+1).
template <int SURF, bool ROPE>
__global__ void padj_rev_position_kernel(const FrameArgs* __restrict__ pa, PlainAdjBufs b, int n, int k) {
    const FrameArgs& a = *pa;
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const int4 tp = a.topo[d];
    const uint32_t fl = (uint32_t)tp.x;
    const bool hasNext = fl & F_NEXT, hasPrev = fl & F_PREV;
    float4 qb = b.gq[d];
    if (hasPrev) qb = add4(qb, b.eb[d - 1]);
    if (hasNext) qb = add4(qb, b.ea[d + 1]);
    b.gq[d] = qb;
    f3 dd = -xyz(b.ec[d]);
    if (hasPrev) dd += xyz(b.ec[d - 1]);
    float4 gx = b.gx[d];
    f3 db = xyz(b.td[d]) + dd;
    f3 xb = xyz(gx) + dd;
    if constexpr (ROPE) {
        float4* cd = b.cd + (size_t)((k + 1) & 1) * n + d;
        db += xyz(*cd);
        *cd = zero4();
    }
    const float im = b.x[d].w, h = a.h;
    const f3 p = xyz(b.x[d]);
    const f3 dk = xyz(b.ld[(size_t)k * n + d]);
    const float4 zn4 = b.ld[(size_t)(k + 1) * n + d];
    f3 dn = db;
    f3 Fb = zero3(), e = zero3(), yb = xyz(b.ty[d]);
    float trH = 0.f;
    if (im != 0.f) {
        const float damp = a.damping / h;
        const VConst c = vertex_constants(a, im, a.vel[d].w, a.lvel[d].w);
        const float4* cache = (SURF == SURF_MESHES) ? static_poses(a, tp.w) : nullptr;
        const uint64_t cand = (SURF == SURF_MESHES) ? b.cand[d] : 0ull;
        sym3 H = sym_diag(c.Hd);
        bool touched = false;
        if constexpr (SURF != SURF_NONE) {
            f3 fdummy = zero3();
            touched = surfaces<SURF>(a, cache, cand, p, dk, c.kc, h, fdummy, H, nullptr, nullptr);
        }
        if (hasNext) {
            const float s = c.ks * c.invl * c.invl * (1.f + damp);
            H.xx += s; H.yy += s; H.zz += s;
        }
        if (hasPrev) {
            const float ilp = 1.f / a.vel[d - 1].w;
            const float s = a.lvel[d - 1].w * ilp * ilp * (1.f + damp);
            H.xx += s; H.yy += s; H.zz += s;
        }
        f3 gb = db;
        f3 zk = xyz(zn4);
        if constexpr (ROPE) {
            const float4 a0 = b.ha0[d], a1 = b.ha1[d];
            H.xx += a0.x; H.yy += a0.y; H.zz += a0.z; H.xy += a0.w; H.xz += a1.x; H.yz += a1.y;
            if (hasPrev) {
                const float4 h0 = b.hb0[d - 1], h1 = b.hb1[d - 1];
                H.xx += h0.x; H.yy += h0.y; H.zz += h0.z; H.xy += h0.w; H.xz += h1.x; H.yz += h1.y;
            }
            touched = true;
            if (zn4.w < 1.f) {  // the step limit clipped this step
                const float l = len(zk);
                const f3 zh = zk * (1.f / l);
                const float zg = dot(zh, gb);
                float2 ms = b.ms[d];
                if (hasPrev && a.maxstep[d - 1] < a.maxstep[d]) ms.y += zg;
                else ms.x += zg;
                b.ms[d] = ms;
                gb = (gb - zh * zg) * zn4.w;
                zk = zk * (1.f / zn4.w);
            }
            dn = gb;
        }
        e = touched ? sym_solve(H, gb) : gb * (1.f / H.xx);
        const f3 del = zk - dk;
        Fb = e * a.accel;
        trH = -dot(e, del);
        yb += Fb * c.fm;
        dn -= Fb * c.fm;
        float wsum = (dot(xyz(b.y[d]) - dk, Fb) + trH) * (-c.fm / im);
        if constexpr (SURF != SURF_NONE) {
            for (int pl = 0; pl < a.num_planes; pl++) {
                const float4 P = a.planes[pl];
                const f3 nrm = mk3(P.x, P.y, P.z);
                const float gap = (dot(nrm, p) - P.w) + dot(nrm, dk) - a.c_radius;
                if (gap >= 0.f) continue;
                float gapb, kb;
                f3 nb;
                surface_contact_bwd(nrm, gap, dk, c.kc, h, a.c_mu_s, a.c_mu_k, a.c_vslip, Fb, e, del, dn, gapb, kb, nb);
                dn += nrm * gapb;
                xb += nrm * gapb;
                wsum += kb * (-c.kc / im);
            }
        }
        if constexpr (SURF == SURF_MESHES)
            wsum += mesh_contact_bwd(a, cache, cand, p, dk, c.kc, h, Fb, e, del, dn, xb) * (-c.kc / im);
        float4 gv0 = b.gv0[d];
        gv0.w += wsum;
        b.gv0[d] = gv0;
    }
    b.ef[d] = f4(Fb, trH);
    b.ee[d] = f4(e, 0.f);
    b.td[d] = f4(dn, 0.f);
    b.ty[d] = f4(yb, 0.f);
    b.gx[d] = f4(xb, gx.w);
}

// Stretch terms and the segment's rope-rope pairs reversed (position step k); the pairs' shares
// of the other segment's vertices and of vertex t+1 go by atomics to cd (parity k) and cx.
template <bool ROPE>
__global__ void padj_rev_stretch_kernel(const FrameArgs* __restrict__ pa, PlainAdjBufs b, int n, int k) {
    const FrameArgs& a = *pa;
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const uint32_t fl = (uint32_t)a.topo[d].x;
    const bool hasNext = fl & F_NEXT, hasPrev = fl & F_PREV;
    const float damp = a.damping / a.h;
    const float4* Dk = b.ld + (size_t)k * n;
    const float4* Dn = b.ld + (size_t)(k + 1) * n;
    const float4 ef = b.ef[d];
    const f3 Fb = xyz(ef);
    float4 gx = b.gx[d];
    f3 dn = xyz(b.td[d]), xb = xyz(gx);
    float4 qb = b.gq[d];
    const f3 dk = xyz(Dk[d]);
    if (hasNext) {
        const float ks = a.lvel[d].w, invl = 1.f / a.vel[d].w;
        const f3 p = xyz(b.x[d]), p1 = xyz(b.x[d + 1]);
        const f3 dkn = xyz(Dk[d + 1]);
        const float4 qk = b.lq[(size_t)k * n + d];
        const f3 cc = ((p1 - p) + (dkn - dk)) * invl - qtangent(qk);
        const float4 Fn4 = b.ef[d + 1];
        const f3 Fn = xyz(Fn4);
        const float kk = ks * invl, dd = kk * invl;
        const f3 dF = Fb - Fn;
        const f3 cb = dF * kk;
        gx.w += dot(cc, dF) * invl + (-damp * (dot(dk, Fb) + dot(dkn, Fn)) + (1.f + damp) * (ef.w + Fn4.w)) * invl * invl;
        qb = add4(qb, scale4(tangent_vjp(qk, cb), -1.f));
        dn -= cb * invl;
        xb -= cb * invl;
        dn -= Fb * (damp * dd);
        if constexpr (ROPE) {
            const int ncol = a.ncols[d];
            if (ncol > 0) {
                const float4 zo4 = Dn[d], zn4 = Dn[d + 1];
                const f3 la = xyz(zo4) * (1.f / zo4.w) - dk;
                const f3 lc = xyz(zn4) * (1.f / zn4.w) - dkn;
                const f3 ea = xyz(b.ee[d]), ec = xyz(b.ee[d + 1]);
                float4* cdk = b.cd + (size_t)(k & 1) * n;
                PairGrad acc{};
                for (int q2 = 0; q2 < ncol; q2++) {
                    const int j = a.cols[(size_t)q2 * n + d];
                    PairGrad o{};
                    collision_bwd(a, damp, p, p1, xyz(b.x[j]), xyz(b.x[j + 1]), dk, dkn, xyz(Dk[j]), xyz(Dk[j + 1]), Fb, ea,
                                  la, Fn, ec, lc, o);
                    acc.x0 += o.x0; acc.d0 += o.d0; acc.x1 += o.x1; acc.d1 += o.d1;
                    atomic_add3(cdk + j, o.e0);
                    atomic_add3(cdk + j + 1, o.e1);
                    atomic_add3(b.cx + j, o.y0);
                    atomic_add3(b.cx + j + 1, o.y1);
                }
                dn += acc.d0;
                xb += acc.x0;
                atomic_add3(cdk + d + 1, acc.d1);
                atomic_add3(b.cx + d + 1, acc.x1);
            }
        }
    }
    if (hasPrev) {
        const float ilp = 1.f / a.vel[d - 1].w;
        const float kkp = a.lvel[d - 1].w * ilp, ddp = kkp * ilp;
        const f3 cbp = (xyz(b.ef[d - 1]) - Fb) * kkp;
        dn += cbp * ilp;
        xb += cbp * ilp;
        dn -= Fb * (damp * ddp);
    }
    b.td[d] = f4(dn, 0.f);
    b.gx[d] = f4(xb, gx.w);
    b.gq[d] = qb;
}

// Step limits reversed (their adjoints from this vertex and from vertex t+1), with the pairs'
// d̄ shares of position step 0.
__global__ void padj_limit_kernel(const FrameArgs* __restrict__ pa, PlainAdjBufs b, int n) {
    const FrameArgs& a = *pa;
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const uint32_t fl = (uint32_t)a.topo[d].x;
    const bool hasNext = fl & F_NEXT;
    float4* cd = b.cd + d;
    const float4 td = b.td[d];
    b.td[d] = f4(xyz(td) + xyz(*cd), 0.f);
    *cd = zero4();
    float msb = b.ms[d].x;
    if (hasNext) msb += b.ms[d + 1].y;
    if (hasNext && msb != 0.f) {
        const f3 p = xyz(b.x[d]);
        f3 xb = xyz(b.gx[d]), xb1 = zero3(), xj0 = zero3(), xj1 = zero3();
        int jo;
        const f3 ybl = step_limit_bwd(a, d, a.ncols[d], b.x, p, xyz(b.x[d + 1]), a.pad[d], xyz(b.y[d]), msb, xb, xb1, jo,
                                      xj0, xj1);
        add3(&b.tn[d], ybl * a.h);  // y = v h + g h²
        b.gx[d] = f4(xb, b.gx[d].w);
        atomic_add3(b.cx + d + 1, xb1);
        if (jo >= 0) {
            atomic_add3(b.cx + jo, xj0);
            atomic_add3(b.cx + jo + 1, xj1);
        }
    }
}

// Inertial prediction and root program reversed; the substep's start-state adjoints become the
// previous substep's end-state adjoints.
template <bool ROPE>
__global__ void padj_start_kernel(const FrameArgs* __restrict__ pa, const AdjArgs g, PlainAdjBufs b, int n, int s) {
    const FrameArgs& a = *pa;
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const int4 tp = a.topo[d];
    const uint32_t fl = (uint32_t)tp.x;
    const float im = a.pos[d].w, h = a.h;
    float4 gx = b.gx[d];
    f3 xb = xyz(gx);
    if constexpr (ROPE) {
        xb += xyz(b.cx[d]);
        b.cx[d] = zero4();
    }
    const f3 db = xyz(b.td[d]), yb = xyz(b.ty[d]);
    f3 vbn = xyz(b.tn[d]), lvbn = zero3();
    float4 qb = b.gq[d];
    if (im != 0.f) {
        vbn += (db + yb) * h;
        const f3 gv = mk3(a.gx, a.gy, a.gz);
        const float g2 = dot(gv, gv);
        if (g2 > 0.f) {
            const float4* t = g.tape + (size_t)s * 4 * n + tp.z;
            const f3 acc = (xyz(t[n]) - xyz(t[2 * (size_t)n])) / a.last_h;
            const float raw = dot(acc, gv) / g2;
            if (raw >= 0.f && raw <= 1.f) {  // inclusive at the clamp's ends (as torch.clamp)
                const float sb = dot(gv * (h * h), db);
                const f3 gs = gv * (sb / (a.last_h * g2));
                vbn += gs;
                lvbn -= gs;
            }
        }
    } else {
        vbn += db * h;
    }
    if ((fl & F_ROOT) && a.root_mode == ROOT_PROGRAM) {
        const float dt = a.dt, tau = float(s) * h, th = tau + 0.5f * h, idt2 = 2.f / (dt * dt);
        const float xa = 0.5f * tau * tau * idt2;
        add3(&b.gp0[d], xb * (1.f - xa) + vbn * (-th * idt2));
        add3(&b.gv0[d], xb * (tau - xa * dt) + vbn * (1.f - th * idt2 * dt));
        add3(&b.gp1[d], xb * xa + vbn * (th * idt2));
        xb = zero3();
        vbn = zero3();
        if (a.has_q0) qb = zero4();
    }
    b.gx[d] = f4(xb, gx.w);
    b.gv[d] = f4(vbn, b.gv[d].w);
    b.gl[d] = f4(lvbn, b.gl[d].w);
    b.gq[d] = qb;
}

// Outputs in caller order; segment t's bending adjoint also has vertex t+1's share.
__global__ void padj_out_kernel(const FrameArgs* __restrict__ pa, const AdjArgs g, PlainAdjBufs b, int n) {
    const FrameArgs& a = *pa;
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const int4 tp = a.topo[d];
    const uint32_t fl = (uint32_t)tp.x;
    const bool hasNext = fl & F_NEXT;
    const int u = tp.z;
    const float im = a.pos[d].w, lr = a.vel[d].w;
    const float4 gx = b.gx[d], gv = b.gv[d], gl = b.gl[d];
    st3(g.o_pos, u, xyz(gx));
    st3(g.o_vel, u, xyz(gv));
    st3(g.o_lvel, u, xyz(gl));
    reinterpret_cast<float4*>(g.o_q)[u] = b.gq[d];
    const float rho = gv.w + (hasNext ? b.gl[d + 1].w : 0.f);
    if (g.o_ea) g.o_ea[u] = hasNext ? gx.w * lr : 0.f;
    if (g.o_ei) g.o_ei[u] = hasNext ? rho * 4.f / lr : 0.f;
    if (g.o_mass) g.o_mass[u] = (im != 0.f) ? -im * im * b.gv0[d].w : 0.f;
    if ((fl & F_ROOT) && a.root_mode == ROOT_PROGRAM) {
        if (g.o_p0) st3(g.o_p0, tp.w, xyz(b.gp0[d]));
        if (g.o_v0) st3(g.o_v0, tp.w, xyz(b.gv0[d]));
        if (g.o_p1) st3(g.o_p1, tp.w, xyz(b.gp1[d]));
    }
}

inline int blocks_of(int n, int t) { return (n + t - 1) / t; }

template <int SURF, bool ROPE>
void run_adjoint_plain(const FrameArgs* pa, const AdjArgs& g, const PlainAdjBufs& b, int n, int iters, int substeps,
                       const RopeGrid* grid, cudaStream_t st) {
    const int nb = blocks_of(n, kBlock);
    padj_load_kernel<<<nb, kBlock, 0, st>>>(pa, g, b, n);
    for (int s = substeps - 1; s >= 0; s--) {
        padj_init_kernel<<<nb, kBlock, 0, st>>>(pa, g, b, n, s);
        if (ROPE && grid) rope_grid_detect(pa, b.x, *grid, n, false, st);
        else if (ROPE) padj_detect_kernel<<<nb, kBlock, 0, st>>>(pa, b, n);
        for (int k = 0; k < iters; k++) {
            if constexpr (ROPE) padj_position_rope_kernel<SURF><<<blocks_of(n, kOwnedRope), kPosBlock, 0, st>>>(pa, b, n, k);
            else padj_position_kernel<SURF, ROPE><<<blocks_of(n, kOwned), kPosBlock, 0, st>>>(pa, b, n, k);
            padj_frame_kernel<<<nb, kBlock, 0, st>>>(pa, b, n, k);
        }
        padj_end_kernel<<<nb, kBlock, 0, st>>>(pa, b, n);
        for (int k = iters - 1; k >= 0; k--) {
            padj_rev_frame_kernel<ROPE><<<nb, kBlock, 0, st>>>(pa, b, n, k, k == iters - 1 ? 1 : 0);
            padj_rev_position_kernel<SURF, ROPE><<<nb, kBlock, 0, st>>>(pa, b, n, k);
            padj_rev_stretch_kernel<ROPE><<<nb, kBlock, 0, st>>>(pa, b, n, k);
        }
        if (ROPE) padj_limit_kernel<<<nb, kBlock, 0, st>>>(pa, b, n);
        padj_start_kernel<ROPE><<<nb, kBlock, 0, st>>>(pa, g, b, n, s);
    }
    padj_out_kernel<<<nb, kBlock, 0, st>>>(pa, g, b, n);
}

template <bool ROPE>
void run_adjoint_plain_s(const FrameArgs* pa, const AdjArgs& g, const PlainAdjBufs& b, int n, int iters, int substeps,
                         int surf, const RopeGrid* grid, cudaStream_t st) {
    if (surf == SURF_MESHES) run_adjoint_plain<SURF_MESHES, ROPE>(pa, g, b, n, iters, substeps, grid, st);
    else if (surf == SURF_PLANES) run_adjoint_plain<SURF_PLANES, ROPE>(pa, g, b, n, iters, substeps, grid, st);
    else run_adjoint_plain<SURF_NONE, ROPE>(pa, g, b, n, iters, substeps, grid, st);
}

}  // namespace

size_t adjoint_plain_words(int n, int iters) { return (size_t)n * (size_t)(2 * (iters + 1) + 27); }

PlainAdjBufs adjoint_plain_carve(float4* base, int n, int iters) {
    PlainAdjBufs b{};
    float4* p = base;
    auto take = [&](size_t count) { float4* r = p; p += count; return r; };
    const size_t N = (size_t)n;
    b.ld = take((iters + 1) * N);
    b.lq = take((iters + 1) * N);
    b.x = take(N); b.y = take(N);
    b.cand = reinterpret_cast<uint64_t*>(take((N + 1) / 2));
    b.gx = take(N); b.gv = take(N); b.gl = take(N); b.gq = take(N);
    b.gp0 = take(N); b.gv0 = take(N); b.gp1 = take(N);
    b.td = take(N); b.tn = take(N); b.ty = take(N);
    b.ms = reinterpret_cast<float2*>(take((N + 1) / 2));
    b.ea = take(N); b.eb = take(N); b.ec = take(N);
    b.ha0 = take(N); b.ha1 = take(N); b.hb0 = take(N); b.hb1 = take(N);
    b.ef = take(N); b.ee = take(N);
    b.cd = take(2 * N);
    b.cx = take(N);
    b.qp = take(N);
    return b;
}

cudaError_t launch_adjoint_plain(const FrameArgs* pa, const AdjArgs& g, const PlainAdjBufs& b, int n, int iters,
                                 int substeps, int surf, bool rope, const RopeGrid* grid, cudaStream_t st) {
    if (rope) run_adjoint_plain_s<true>(pa, g, b, n, iters, substeps, surf, grid, st);
    else run_adjoint_plain_s<false>(pa, g, b, n, iters, substeps, surf, grid, st);
    return cudaGetLastError();
}

}  // namespace rs
