// rs_substep.cuh -- the per-vertex pieces of one substep, shared by the persistent frame kernel
// (rs_frame.cu) and the per-substep-launch plain path (rs_plain.cu), so both engines run the
// same arithmetic in the same order.
//
// Reference routines restated (deterministic ordering):
//   root_program / root_set   csrc/batch.cu:90-159
//   compute_pose              sim/iteration.cu:12-33, sim/contact.cuh:79-87
//   init_vertex               sim/iteration.cu:34-68
//   position_terms            sim/cosserat.cu:37-159 (inertia, surfaces, stretch)
//   position_solve            sim/cosserat.cu:198-217
//   frame_update              sim/cosserat.cu:242-272
//   end_velocity              sim/iteration.cu:85-112
//   build_candidates          sim/contact.cuh:121-136
#pragma once

#include "rs_device.cuh"
#include "rs_types.h"

namespace rs {

using namespace rsd;

// Surface-contact variants of the kernels: none, planes only, planes + SDF meshes.
enum : int { SURF_NONE = 0, SURF_PLANES = 1, SURF_MESHES = 2 };
constexpr int kPoseF4 = 5;  // float4 per cached pose

__device__ __forceinline__ uint64_t all_meshes(int n) { return n >= 64 ? ~0ull : ((1ull << n) - 1ull); }

// Checked builds: the load-time checks of one vertex at bin-local index t (caller index uidx, its
// rope's slot lrope among the bin's ropes, its rope's caller index env; nsdf meshes in the pose
// cache). Flags whose neighbour reads would leave the bin are cleared, an out-of-range rope slot
// is replaced by 0; returns false when the caller or rope index is out of range (the kernel then
// drops the vertex: no reads or writes through those indices).
__device__ __forceinline__ bool checked_vertex(const FrameArgs& a, const Bin& bin, int t, int uidx, uint32_t& fl,
                                               int& lrope, int& env, int nsdf) {
    if ((fl & (F_NEXT | F_NEXT_ORIENT)) && t + 1 >= bin.vcount) {
        check_fail(a.status, CHK_NEXT);
        fl &= ~(F_NEXT | F_NEXT_ORIENT);
    }
    if (((fl & F_PREV) || !(fl & F_NEXT)) && t < 1) {  // the rope's last vertex reads t - 1 as well
        check_fail(a.status, CHK_PREV);
        fl &= ~F_PREV;
    }
    if (nsdf > 0 && !(lrope >= 0 && lrope < bin.rcount && (lrope + 1) * nsdf <= a.pose_cache)) {
        check_fail(a.status, CHK_POSE);
        lrope = 0;
    }
    if (!(uidx >= 0 && uidx < a.n && env >= 0 && env < a.num_ropes)) {
        check_fail(a.status, CHK_CALLER);
        fl = 0;
        env = 0;
        return false;
    }
    return true;
}

// Shortest-arc SLERP with an nlerp fallback above dot 0.9995, batch.cu:106-114.
__device__ __forceinline__ float4 slerp4(float4 a, float4 b, float t) {
    float d = dot4(a, b);
    if (d < 0.f) { b = scale4(b, -1.f); d = -d; }
    if (d > 0.9995f) return normalize4(add4(scale4(a, 1.f - t), scale4(b, t)));
    const float th = acosf(fminf(d, 1.f));
    const float s = sinf(th);
    return add4(scale4(a, sinf((1.f - t) * th) / s), scale4(b, sinf(t * th) / s));
}
__device__ __forceinline__ float4 unit_or_identity(const float* q) {
    float4 a = make_float4(q[0], q[1], q[2], q[3]);
    const float l = dot4(a, a);
    return (l > 0.f) ? scale4(a, rsqrtf(l)) : make_float4(0.f, 0.f, 0.f, 1.f);
}

// Root program of substep s of S (row = p0, v0, p1, q0, q1): quadratic position at tau = s h,
// velocity at the substep midpoint, SLERPed frame at (s + 1) / S, batch.cu:122-159.
__device__ __forceinline__ void root_program(const FrameArgs& a, const float* row, int s, int S, float h, f3& p, f3& v,
                                             float4& q) {
    const f3 P0 = mk3(__ldg(row), __ldg(row + 1), __ldg(row + 2));
    const f3 V0 = mk3(__ldg(row + 3), __ldg(row + 4), __ldg(row + 5));
    const f3 P1 = mk3(__ldg(row + 6), __ldg(row + 7), __ldg(row + 8));
    const f3 A = 2.f / (a.dt * a.dt) * ((P1 - P0) - V0 * a.dt);
    const float tau = float(s) * h;
    p = P0 + V0 * tau + 0.5f * tau * tau * A;
    v = V0 + (tau + 0.5f * h) * A;
    if (a.has_q0) {
        const float4 qa = unit_or_identity(row + 9);
        float4 qq = a.has_q1 ? slerp4(qa, unit_or_identity(row + 13), float(s + 1) / float(S)) : qa;
        const float l2 = dot4(qq, qq);
        q = (l2 > 0.f) ? scale4(qq, rsqrtf(l2)) : make_float4(0.f, 0.f, 0.f, 1.f);
    }
}
// Constant-velocity root of a frame (row = p, v, -, q), batch.cu:90-104.
__device__ __forceinline__ void root_set(const FrameArgs& a, const float* row, f3& p, f3& v, float4& q) {
    p = mk3(row[0], row[1], row[2]);
    v = mk3(row[3], row[4], row[5]);
    if (a.has_q0) q = unit_or_identity(row + 9);
}

// Kinematics of (env en, mesh m) at the end of substep s of S: constant linear and angular
// velocity over the frame (position, rotor, velocity, angular velocity).
__device__ __forceinline__ void pose_kinematics(const FrameArgs& a, int en, int m, int s, int S, float h, f3& Pp, float4& Pq,
                                                f3& Pv, f3& Pw) {
    const Motion M = a.motion[(size_t)en * kMaxSdf + m];
    const float al = float(s + 1) / float(S);
    const float invDt = 1.f / (float(S) * h);
    const f3 p0 = mk3(M.p0x, M.p0y, M.p0z), dp = mk3(M.dpx, M.dpy, M.dpz), rot = mk3(M.rx, M.ry, M.rz);
    const float4 q0 = make_float4(M.qx, M.qy, M.qz, M.qw);
    const float th = len(rot);
    if (th > 0.f || dp.x != 0.f || dp.y != 0.f || dp.z != 0.f) {
        Pp = p0 + al * dp;
        float4 dq = make_float4(0.f, 0.f, 0.f, 1.f);
        if (th > 0.f) {
            const f3 ax = rot / th;
            const float hr = (al * th) * 0.5f;
            const float sn = sinf(hr);
            dq = make_float4(sn * ax.x, sn * ax.y, sn * ax.z, cosf(hr));
        }
        Pq = normalize4(qmul(dq, q0));
        Pv = dp * invDt;
        Pw = rot * invDt;
    } else {  // a target equal to the current pose: exactly the static pose
        Pp = p0; Pq = q0; Pv = zero3(); Pw = zero3();
    }
}

// Lattice box [lo_o, hi_o] of grid gd in the object frame.
__device__ __forceinline__ void lattice_box(const GridDesc& gd, f3& lo_o, f3& hi_o) {
    lo_o = mk3(gd.ox, gd.oy, gd.oz);
    hi_o = lo_o + mk3(float(gd.nx - 1), float(gd.ny - 1), float(gd.nz - 1)) * gd.h;
}

// The broad phase's padding for a mesh's own travel over one substep (contact.cuh:121-136),
// once per pose instead of once per vertex; static poses keep 0.
__device__ __forceinline__ float travel_pad(const FrameArgs& a, f3 Pv, f3 Pw, f3 lo, f3 hi) {
    return a.sdf_moving ? a.h * (len(Pv) + len(Pw) * 0.5f * len(hi - lo)) : 0.f;
}

// Pose of (env en, mesh m) at the end of substep s of S with the world AABB of the lattice;
// 5 float4 at `out`.
__device__ __forceinline__ void compute_pose(const FrameArgs& a, int en, int m, int s, int S, float h, float4* out) {
    f3 Pp, Pv, Pw;
    float4 Pq;
    pose_kinematics(a, en, m, s, S, h, Pp, Pq, Pv, Pw);
    f3 lo_o, hi_o, lo, hi;
    lattice_box(a.grids[m], lo_o, hi_o);
    world_box(lo_o, hi_o, Pp, Pq, lo, hi);
    store_pose(out, Pp, Pq, Pv, Pw, lo, hi);
    out[4].w = travel_pad(a, Pv, Pw, lo, hi);
}

// Surfaces (planes, then candidate meshes in ascending index) at one probe point,
// contact.cuh:141-163; with `wr` != nullptr it is the readout (contact.cuh:172-204): mesh
// forces are added to *facc and their wrenches to wr[m * 6 ...]. Returns whether any contact
// term was added (H then stops being a multiple of the identity).
// `tbox` (persistent kernel): per mesh the world AABB of its contact box (GridDesc::tlo/thi at
// this substep's pose), an exact early out before the probe is rotated into the lattice.
template <int SURF>
__device__ __forceinline__ bool surfaces(const FrameArgs& a, const float4* cache, uint64_t cand, f3 pos, f3 d, float k,
                                         float h, f3& f, sym3& H, float* wr, f3* facc, const float* btab = nullptr,
                                         const float4* tbox = nullptr) {
    bool touched = false;
    if (a.num_planes == 1) {
        // the common single plane as straight-line code: the runtime-bounded loop below costs a
        // frame of 4096 64-vertex ropes 4% (it keeps the gap test from being scheduled with its
        // neighbours)
        const float4 P = a.planes[0];
        const f3 n = mk3(P.x, P.y, P.z);
        const float gap = (dot(n, pos) - P.w) + dot(n, d) - a.c_radius;
        if (gap < 0.f) {
            surface_contact(n, gap, d, k, h, a.c_mu_s, a.c_mu_k, a.c_vslip, f, H);
            touched = true;
        }
    } else {
        for (int pl = 0; pl < a.num_planes; pl++) {
            const float4 P = a.planes[pl];
            const f3 n = mk3(P.x, P.y, P.z);
            const float gap = (dot(n, pos) - P.w) + dot(n, d) - a.c_radius;
            if (gap >= 0.f) continue;
            surface_contact(n, gap, d, k, h, a.c_mu_s, a.c_mu_k, a.c_vslip, f, H);
            touched = true;
        }
    }
    if constexpr (SURF == SURF_MESHES) {
    for (uint64_t mm = cand; mm; mm &= mm - 1ull) {
        const int m = __ffsll((long long)mm) - 1;
        const PoseV P = load_pose(cache + m * kPoseF4);  // loaded with the contact box, not after its test
        if (tbox) {
            const float4 lo = tbox[2 * m], hi = tbox[2 * m + 1];
            const f3 pr = pos + d;
            if (!(pr.x >= lo.x && pr.x <= hi.x && pr.y >= lo.y && pr.y <= hi.y && pr.z >= lo.z && pr.z <= hi.z)) continue;
        }
        f3 n, dRel;
        float gap;
        if (!sdf_contact_at(a.grids[m], P, pos, d, h, a.c_radius, a.sdf_moving != 0, a.sdf_skip != 0, btab, n, gap, dRel))
            continue;
        touched = true;
        if (wr) {
            f3 fm = zero3();
            sym3 Hs = sym_zero();
            surface_contact(n, gap, dRel, k, h, a.grids[m].muS, a.grids[m].muK, a.c_vslip, fm, Hs);
            *facc += fm;
            const f3 r = (pos - P.pos) + d - n * a.c_radius;
            const f3 tq = cross(r, -fm);
            float* w = wr + m * 6;
            atomicAdd(w + 0, -fm.x); atomicAdd(w + 1, -fm.y); atomicAdd(w + 2, -fm.z);
            atomicAdd(w + 3, tq.x); atomicAdd(w + 4, tq.y); atomicAdd(w + 5, tq.z);
        } else {
            surface_contact(n, gap, dRel, k, h, a.grids[m].muS, a.grids[m].muK, a.c_vslip, f, H);
        }
    }
    }
    return touched;
}

// The smallest sdf_slack over a vertex's candidate meshes at this substep's poses, from the
// probe `pos` (the persistent kernel passes the position plus the substep's initial guess d0):
// while the iterate d satisfies |d - d0| < slack, surfaces() finds no mesh contact (the mesh terms
// are then skipped without rotating the probe into any lattice).
__device__ __forceinline__ float mesh_slack(const FrameArgs& a, const float4* cache, uint64_t cand, f3 pos) {
    float s = INFINITY;
    for (uint64_t mm = cand; mm; mm &= mm - 1ull) {
        const int m = __ffsll((long long)mm) - 1;
        if (a.grids[m].never) continue;
        s = fminf(s, sdf_slack(a.grids[m], load_pose(cache + m * kPoseF4), pos, a.c_radius));
    }
    return s;
}

// How far a vertex's iterate may move from the probe `pos` (the persistent kernel passes the
// position plus the substep's initial guess d0) before it could reach a plane's contact band:
// gap(d) = (n.x - w) + n.d - R >= (n.pos - w - R) - |d - d0| for a unit normal n and
// pos = x + d0, less a 1 mm margin that covers any difference in evaluating the gap expression
// for coordinates up to ~10 km. INFINITY without planes.
__device__ __forceinline__ float plane_slack(const FrameArgs& a, f3 pos) {
    float s = INFINITY;
    for (int pl = 0; pl < a.num_planes; pl++) {
        const float4 P = a.planes[pl];
        s = fminf(s, ((dot(mk3(P.x, P.y, P.z), pos) - P.w) - a.c_radius) - 1e-3f);
    }
    return s;
}

// World AABB of a lattice's contact box under the pose (pos, q); an empty box when the lattice
// can never reach the contact radius.
__device__ __forceinline__ void contact_box(const GridDesc& g, f3 pos, float4 q, float4* out) {
    if (g.never) {
        out[0] = make_float4(INFINITY, INFINITY, INFINITY, 0.f);
        out[1] = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.f);
        return;
    }
    f3 lo, hi;
    world_box(mk3(g.tlo[0], g.tlo[1], g.tlo[2]), mk3(g.thi[0], g.thi[1], g.thi[2]), pos, q, lo, hi);
    out[0] = f4(lo, 0.f);
    out[1] = f4(hi, 0.f);
}

// Inertial target y and initial guess dx from the substep's start velocity, iteration.cu:34-68.
__device__ __forceinline__ void init_vertex(f3 vel0, f3 lv_old, float im, float h, float last_h, f3 g, float g2, f3& dx,
                                            f3& y) {
    dx = vel0 * h;
    y = fma3(g, h * h, dx);
    if (im != 0.f && g2 > 0.f) {
        const f3 acc = (vel0 - lv_old) / last_h;
        const float sg = fminf(fmaxf(dot(acc, g) / g2, 0.f), 1.f);
        dx = fma3(g, h * h * sg, dx);
    }
}

// Per-vertex constants of a frame.
struct VConst {
    float im, invl, ks, Hd, fm, kc;
};
__device__ __forceinline__ VConst vertex_constants(const FrameArgs& a, float im, float lr, float ks) {
    VConst c;
    c.im = im;
    c.invl = 1.f / lr;
    c.ks = ks;
    c.Hd = 1.f / (im * a.h * a.h);
    c.fm = 1.f / (a.h * a.h * im);
    const float kap = a.c_kappa / a.h;
    c.kc = kap * kap / im;
    return c;
}

// Position-step terms of vertex i, cosserat.cu:37-88: own force f / Hessian H (inertia, then
// surfaces, then the stretch of segment i) and the segment's share f2 / H2 on vertex i + 1.
// Returns whether a surface contact touched H (otherwise H is a multiple of the identity).
template <int SURF>
__device__ __forceinline__ bool position_terms(const FrameArgs& a, const float4* cache, uint64_t cand, const VConst& c,
                                               bool hasNext, f3 p, f3 p1, f3 dx, f3 p1dx, f3 y, float4 q, float damp,
                                               f3& f, sym3& H, f3& f2, sym3& H2, const float* btab = nullptr,
                                               const float4* tbox = nullptr) {
    f = (y - dx) * c.fm;
    H = sym_diag(c.Hd);
    bool touched = false;
    if (SURF != SURF_NONE && c.im != 0.f)
        touched = surfaces<SURF>(a, cache, cand, p, dx, c.kc, a.h, f, H, nullptr, nullptr, btab, tbox);
    f2 = zero3();
    H2 = sym_zero();
    {  // without a next vertex the zero stiffness makes every term 0 (no branch for interior vertices)
        const float il = hasNext ? c.invl : 0.f;
        const f3 cc = fma3((p1 - p) + (p1dx - dx), il, -qtangent(q));
        const float k = hasNext ? c.ks * c.invl : 0.f;
        float dd = k * il;
        f = fma3(dx, -(damp * dd), fma3(cc, k, f));
        f2 = fma3(p1dx, -(damp * dd), cc * (-k));
        dd *= 1.f + damp;
        H.xx += dd; H.yy += dd; H.zz += dd;
        H2.xx += dd; H2.yy += dd; H2.zz += dd;
    }
    return touched;
}

// One rope-rope candidate of segment (p, p1) with iterates (d, p1d) against the segment
// (b0, b1) with iterates (db0, db1): IPC log barrier at 2 r + barrier with its damping terms
// and a friction spring capped at mu * |f_n|, cosserat.cu:99-157.
__device__ __forceinline__ void collision_term(const FrameArgs& a, float damp, f3 p, f3 p1, f3 d, f3 p1d, f3 b0, f3 b1,
                                               f3 db0, f3 db1, f3& f, f3& f2, sym3& H, sym3& H2) {
    float u, v;
    seg_closest(zero3(), (p1 - p) + (p1d - d), (b0 - p) + (db0 - d), (b1 - p) + (db1 - d), u, v);
    const f3 dpos = lerp3(p, p1, u) - lerp3(b0, b1, v);
    const f3 ddpos = lerp3(d, p1d, u) - lerp3(db0, db1, v);
    f3 nrm = dpos + ddpos;
    float dist = len(nrm);
    if (!(dist > 0.f)) return;  // coincident centrelines: no normal
    nrm *= 1.f / dist;
    const float wa = 1.f - u, wb = u;
    const float invb = 1.f / a.rc_barrier;
    const float kCol = a.rc_kcol * invb;
    dist = dist - 2.f * a.rc_radius;
    dist *= invb;
    if (dist > 1.f) return;  // not touching
    dist = fmaxf(dist, 1e-3f);
    const float invd = 1.f / dist;
    const float logd = logf(dist);
    float dH = (-3.f + (2.f + invd) * invd - 2.f * logd) * kCol * invb;
    const float ff = -(1.f - dist) * (dist - 1.f + 2.f * dist * logd) * invd * kCol;
    f = fma3(nrm, fmaf(ff, wa, -(damp * dH * wa * wa * dot(nrm, d))), f);
    f2 = fma3(nrm, fmaf(ff, wb, -(damp * dH * wb * wb * dot(nrm, p1d))), f2);
    dH *= 1.f + damp;
    sym_add_scaled_outer(H, nrm, dH * wa * wa);
    sym_add_scaled_outer(H2, nrm, dH * wb * wb);
    const f3 uu = fma3(nrm, -dot(nrm, ddpos), ddpos);
    const float ul = len(uu);
    if (ul > 0.f) {
        const float f1 = fminf(a.rc_kfric, a.rc_mu * ff / ul);
        f = fma3(uu, -(f1 * wa), f);
        sym_sub_scaled_outer_minus_I(H, nrm, wa * wa * f1);
        f2 = fma3(uu, -(f1 * wb), f2);
        sym_sub_scaled_outer_minus_I(H2, nrm, wb * wb * f1);
    }
}

// Candidate test of segment pair (i, j) at the substep start, batch.cu:33-45: closest distance
// of the centrelines below the sum of the padded detection radii.
__device__ __forceinline__ bool rope_pair_candidate(f3 a0, f3 a1, float ri, f3 pj0, f3 pj1, float rj) {
    const f3 b0 = pj0 - a0, b1 = pj1 - a0;
    float u, v;
    seg_closest(zero3(), a1, b0, b1, u, v);
    const f3 dd = a1 * u - lerp3(b0, b1, v);
    const float r = ri + rj;
    return dot(dd, dd) < r * r;
}

// Step-limit contribution of one candidate, collision.cu:124-134: 0.45 x the distance.
__device__ __forceinline__ float step_limit_of(f3 a0, f3 a1, f3 pj0, f3 pj1) {
    const f3 b0 = pj0 - a0, b1 = pj1 - a0;
    float u, v;
    seg_closest(zero3(), a1, b0, b1, u, v);
    const f3 nn = a1 * u - lerp3(b0, b1, v);
    return ((1.f - 0.1f) * 0.5f) * len(nn);
}

// Local solve dx += accel * H^-1 f of a free vertex, cosserat.cu:206-209. Without contact
// terms (`diag`) H is a multiple of the identity and the solve is one division.
__device__ __forceinline__ void position_solve(f3& dx, f3 f, const sym3& H, float accel, float im, bool diag) {
    if (im != 0.f) dx = diag ? fma3(f, accel / H.xx, dx) : fma3(sym_solve(H, f), accel, dx);
}
// The same with the step limit of rope-rope contact, cosserat.cu:211-214. Returns the limit's
// scale lim / |dx| (1 when the step is not limited).
__device__ __forceinline__ float position_solve_limited(f3& dx, f3 f, const sym3& H, float accel, float im, float lim) {
    float sc = 1.f;
    if (im != 0.f) {
        dx = fma3(sym_solve(H, f), accel, dx);
        const float l = len(dx);
        if (l > lim && l > 0.f) {
            sc = lim / l;
            dx *= sc;
        }
    }
    return sc;
}

// Rope-rope detection of segment t over its CTA-resident contact group [g0, g1) (CTA-local
// indices; [r0, r1) is t's own rope, whose segments within two of t are skipped), ascending j,
// capped at kMaxCols: writes the candidate list to cols[c * n + dv] and the segment's step limit
// (padding - detection radius, and 0.45 x each listed candidate's distance), batch.cu:19-49 and
// collision.cu:103-136. pad(j), flg(j) and pos(j) read the group's padded radii, flags and
// substep-start positions. Returns the number of candidates found (the list keeps kMaxCols).
//
// Before the closest-point test each pair passes a conservative early out: the centre lines of
// segments with midpoints m_t, m_j and half-lengths h_t, h_j are at least |m_t - m_j| - h_t - h_j
// apart, so a pair with |m_t - m_j| > (h_t + h_j + r) (1 + 1e-4) + 1e-6 m (r the sum of the padded
// radii) cannot pass the test, whose FP32 distance errs by far less than that margin at these
// separations. The candidate lists are those of the plain brute force, pair for pair.
// The pair test of detect_group (segment (p, p + a1) with midpoint mt, half-length ht and padded
// radius ri against segment (pj0, pj1) with radius rj), shared with the grid broad phase.
__device__ __forceinline__ bool pair_accepts(f3 p, f3 a1, f3 mt, float ht, float ri, f3 pj0, f3 pj1, float rj) {
    const f3 dm = (pj0 + pj1) * 0.5f - mt;
    const float reach = (ht + 0.5f * len(pj1 - pj0) + ri + rj) * 1.0001f + 1e-6f;
    if (dot(dm, dm) > reach * reach) return false;
    return rope_pair_candidate(p, a1, ri, pj0, pj1, rj);
}

template <class Pad, class Flg, class Pos>
__device__ __forceinline__ int detect_group(const FrameArgs& a, int t, int dv, int g0, int g1, int r0, int r1, f3 p, f3 p1,
                                           Pad pad, Flg flg, Pos pos, float& lim) {
    const f3 a1 = p1 - p;
    const float ri = fmaxf(pad(t), pad(t + 1));
    const f3 mt = p + a1 * 0.5f;
    const float ht = 0.5f * len(a1);
    lim = pad(t) - a.det_radius;
    int cnt = 0;
    for (int j = g0; j < g1; j++) {
        if (!(flg(j) & F_NEXT)) continue;
        if (j >= r0 && j < r1 && abs(j - t) <= 2) continue;
        const f3 pj0 = pos(j), pj1 = pos(j + 1);
        const float rj = fmaxf(pad(j), pad(j + 1));
        if (pair_accepts(p, a1, mt, ht, ri, pj0, pj1, rj)) {
            if (cnt < kMaxCols) {
                a.cols[(size_t)cnt * a.n + dv] = j;
                lim = fminf(lim, step_limit_of(p, a1, pj0, pj1));
            }
            cnt++;
        }
    }
    return cnt;
}

// Rope-rope terms of segment t over its ncol candidates, positions P and iterates D of the
// CTA's vertices: even candidates join the own terms, odd ones a second partial added after them
// (the reference's two sectors, cosserat.cu:99-182).
__device__ __forceinline__ void collision_sectors(const FrameArgs& a, int ncol, int dv, const float4* P, const float4* D,
                                                  float damp, f3 p, f3 p1, f3 dx, f3 p1dx, f3& f, f3& f2, sym3& H,
                                                  sym3& H2, int nloc = 0x7fffffff) {
    if (ncol <= 0) return;
    f3 fo = zero3(), f2o = zero3();
    sym3 Ho = sym_zero(), H2o = sym_zero();
    for (int cc = 0; cc < ncol; cc++) {
        const int j = a.cols[(size_t)cc * a.n + dv];
        if (kChecked && !(j >= 0 && j + 1 < nloc)) {  // nloc: the vertices P and D hold
            check_fail(a.status, CHK_CANDIDATE);
            continue;
        }
        const f3 b0 = xyz(P[j]), b1 = xyz(P[j + 1]);
        const f3 db0 = xyz(D[j]), db1 = xyz(D[j + 1]);
        if (cc & 1) collision_term(a, damp, p, p1, dx, p1dx, b0, b1, db0, db1, fo, f2o, Ho, H2o);
        else collision_term(a, damp, p, p1, dx, p1dx, b0, b1, db0, db1, f, f2, H, H2);
    }
    if (ncol > 1) { f += fo; f2 += f2o; sym_add(H, Ho); sym_add(H2, H2o); }
}

// The frame step's unnormalised rotor z = vv b e1 + (|vv| + |b|) b, with lambda = |vv| + |b| and
// the reciprocal norms 1/|vv|, 1/|b| (0 for a zero vector) the reverse needs. The norms use the
// hardware reciprocal square root: z is normalised right after, so their rounding (within 2 ulp)
// only tilts the blend of its two terms.
__device__ __forceinline__ float4 frame_z(f3 vv, float4 b, float& ilvv, float& ilb, float& lambda) {
    const float v2 = dot(vv, vv), b2 = dot4(b, b);
    ilvv = v2 > 0.f ? rsqrtf(v2) : 0.f;
    ilb = b2 > 0.f ? rsqrtf(b2) : 0.f;
    lambda = fmaf(v2, ilvv, b2 * ilb);
    const float4 m = qmul_e1(qmul_pure(vv, b));
    return make_float4(fmaf(b.x, lambda, m.x), fmaf(b.y, lambda, m.y), fmaf(b.z, lambda, m.z), fmaf(b.w, lambda, m.w));
}

// The frame step's two sign tests (each +1 or -1) as one exact small float, 2 snv + spv, for the
// iterate tape; decoded by frame_signs_decode.
__device__ __forceinline__ float frame_signs_encode(float spv, float snv) { return fmaf(2.f, snv, spv); }
__device__ __forceinline__ void frame_signs_decode(float code, float& spv, float& snv) {
    snv = code > 0.f ? 1.f : -1.f;
    spv = fmaf(-2.f, snv, code);
}

// Frame step of segment i, cosserat.cu:242-272: vv = -2 k ((p1 - p) + (p1dx - dx)) / l, b from
// the neighbours' frames and rest rotations, q = normalize(vv b e1 + (|vv| + |b|) b). The
// reference's sign tests dot((q_{i-1}^-1 q_i), r_{i-1}) and dot((q_i^-1 q_{i+1}), r_i) equal
// dot(q_i, q_{i-1} r_{i-1}) and dot(q_i, q_{i+1} r_i^*) (Re(xy) = Re(yx) for quaternions), so
// they reuse the products b needs.
// Both neighbour products are evaluated whatever the flags (the caller passes valid rotors for a
// missing neighbour) and the missing terms are selected away: interior vertices, all but two per
// rope, take no branch. The normalisation multiplies by rsqrt_nr (IEEE sqrt and division cost
// twice the instructions and a branch each; a frame of 4096 64-vertex ropes 2.75 -> 2.35 ms with
// the rest of this step's diet).
__device__ __forceinline__ float4 frame_update(float4 q, f3 seg, float invl, float ks, bool hasPrev, float4 qprev,
                                               float4 qrprev, bool hasNextOrient, float4 qnext, float4 qrown,
                                               float4& b_out, float& signs) {
    const f3 vv = (seg * invl) * (-2.f * ks);
    const float4 pr = qmul(qprev, qrprev);
    const float4 nx = qmul(qnext, qconj(qrown));
    const float spv = dot4(q, pr) > 0.f ? 1.f : -1.f, snv = dot4(q, nx) > 0.f ? 1.f : -1.f;
    const float4 prs = scale4(pr, spv);
    const float4 nxs = scale4(nx, snv);
    float4 b = hasPrev ? prs : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 bn = add4(b, nxs);
    b = hasNextOrient ? bn : b;
    b_out = b;
    signs = frame_signs_encode(spv, snv);
    float ilvv, ilb, lambda;
    const float4 z = frame_z(vv, b, ilvv, ilb, lambda);
    return scale4(z, rsqrt_nr(dot4(z, z)));
}
__device__ __forceinline__ float4 frame_update(float4 q, f3 seg, float invl, float ks, bool hasPrev, float4 qprev,
                                               float4 qrprev, bool hasNextOrient, float4 qnext, float4 qrown) {
    float4 b;
    float signs;
    return frame_update(q, seg, invl, ks, hasPrev, qprev, qrprev, hasNextOrient, qnext, qrown, b, signs);
}

// New velocity of a free vertex: dx / h, quadratic drag split by the segment tangent `tg`
// (exact frozen-direction solution), then linear drag, iteration.cu:87-112.
__device__ __forceinline__ f3 end_velocity(const FrameArgs& a, f3 dx, float invH, f3 tg) {
    f3 vv = dx * invH;
    const float kn = a.drag_quad;
    if (kn > 0.f) {
        const f3 vt = tg * dot(tg, vv);
        f3 vn = vv - vt;
        vn = vn / fmaf(kn * len(vn), a.h, 1.f);
        const f3 vt2 = vt / fmaf(a.drag_quad_t * len(vt), a.h, 1.f);
        vv = vn + vt2;
    }
    return vv * (1.f - a.drag * a.h);
}

// Broad phase for the next substep: meshes of this env whose padded world AABB holds p
// (pad = 2 |dx| + 2 cm + the mesh's own travel); more than kMaxCand = every mesh.
__device__ __forceinline__ uint64_t build_candidates(const FrameArgs& a, const float4* cache, int nsdf, f3 p, f3 dx) {
    const float pad = 2.f * len(dx) + 0.02f;
    uint64_t mask = 0ull;
    int cnt = 0;
    for (int m = 0; m < nsdf; m++) {
        const float4 e3 = cache[m * kPoseF4 + 3], e4 = cache[m * kPoseF4 + 4];  // (.., lo), (hi, travel pad)
        const float pm = pad + e4.w;
        if (p.x >= e3.y - pm && p.x <= e4.x + pm && p.y >= e3.z - pm && p.y <= e4.y + pm && p.z >= e3.w - pm &&
            p.z <= e4.z + pm) {
            mask |= 1ull << m;
            cnt++;
        }
    }
    return cnt <= kMaxCand ? mask : all_meshes(nsdf);
}

}  // namespace rs
