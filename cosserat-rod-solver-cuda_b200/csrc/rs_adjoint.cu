// rs_adjoint.cu -- reverse-mode adjoint of one control frame (the differentiable path) and the
// state / parameter transfer kernels it needs.
//
// The reference has no gradients. What is differentiated is the deterministic (Jacobi) substep
// the frame kernel runs: root program (batch.cu:122-159), inertial prediction with the
// acceleration-projected gravity (iteration.cu:34-68), num_itr x (position step with inertia,
// plane contact + friction, stretch and damping, cosserat.cu:37-88,198-209; frame step,
// cosserat.cu:242-272), velocity with linear and quadratic drag (iteration.cu:85-112). Every
// iteration is reversed (not only the converged state); branches that switch terms (contact
// active, friction regime, frame-step signs, clamps) are held where the forward pass took them.
//
// Data flow of one frame's backward (Batch::backward_program):
//   1. the state after each substep's root program is taped [S][4][n] (x, v, lv, q; caller
//      order, so the tape outlives a repacking of the bins) in HBM: by the forward step itself
//      when the caller kept a tape, else by a replay of the frame from its start state;
//   2. adjoint_kernel (one CTA per bin, one thread per vertex, like the forward) walks the
//      substeps backwards: it recomputes the substep's iterates d^k, q^k into shared memory
//      from the tape, then reverses end -> frame/position steps -> init -> root program.
// Per reverse iteration two CTA barriers: the frame step's neighbour rotor/segment adjoints,
// then the position step's force adjoints. Cross-vertex contributions are gathered by the
// receiving vertex, so no atomics are used and the result is deterministic.
//
// Reverse of the local solve d' = d + a H^-1 F (H symmetric): F̄ = a H^-1 ḡ, H̄ = -(H^-1 ḡ) δᵀ,
// δ = d' - d. Quaternion products c = a b reverse as ā = c̄ b*, b̄ = a* c̄.
#include <cuda_runtime.h>

#include "rs_adjoint.cuh"
#include "rs_kernels.h"

using namespace rsd;

namespace rs {

namespace {

// 16-byte asynchronous copies global -> shared (cp.async, no L1 allocation) and their completion.
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
    const unsigned dst = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Shared memory of the adjoint kernel, in float4 units (BLOCK = bin size, I = iterations):
//   X, QR, KC, EA, EB, EC, EF   one slot per vertex each
//   with rope-rope contact, seven more: RP (padding, step limit, flags, limit adjoint handed to
//   the previous vertex), EE (e = H⁻¹ z̄), HB0/HB1 (the segment's collision Hessian share of its
//   second vertex), CD[2] (d̄ contributions of other segments' pairs, by iteration parity), CX
//   (their x̄ contributions, per substep)
//   LD [I+1][BLOCK]   displacement iterates d^k (.w: the step limit's scale, 1 when not limited)
//   LQ [I+1][BLOCK]   frame iterates q^k
// 64-thread bins at 8 iterations: 25.6 KB, 8 CTAs per SM with <= 128 registers; with rope
// contact 32.8 KB and 4 CTAs per SM with <= 255 registers (the pair reverse's working set).
template <int BLOCK, int SURF, bool ROPE>
__global__ void __launch_bounds__(BLOCK, ROPE ? (BLOCK >= 256 ? 1 : 256 / BLOCK) : 512 / BLOCK)
    adjoint_kernel(const FrameArgs a, const AdjArgs g) {
    extern __shared__ float4 smem[];
    const int I = a.iters;
    float4* X = smem;
    float4* QR = X + BLOCK;
    float4* KC = QR + BLOCK;   // (kStretch, 1 / lRest, invMass, -)
    float4* EA = KC + BLOCK;
    float4* EB = EA + BLOCK;
    float4* EC = EB + BLOCK;
    float4* EF = EC + BLOCK;
    float4* RP = EF + BLOCK;
    float4* EE = RP + BLOCK;
    float4* HB0 = EE + BLOCK;
    float4* HB1 = HB0 + BLOCK;
    float4* CD = HB1 + BLOCK;  // [2][BLOCK]
    float4* CX = CD + 2 * BLOCK;
    float4* LD = ROPE ? CX + BLOCK : RP;
    float4* LQ = LD + (size_t)(I + 1) * BLOCK;
    float4* PC = LQ + (size_t)(I + 1) * BLOCK;  // static mesh poses of the bin's ropes [rope][mesh]

    const Bin bin = a.bins[blockIdx.x];
    const int t = threadIdx.x;
    bool act = t < bin.vcount;
    const int dv = bin.vstart + t;
    if constexpr (kChecked)
        if (act && !(bin.vstart >= 0 && bin.vcount <= BLOCK && dv < a.n)) {
            check_fail(a.status, CHK_BIN);
            act = false;
        }
    uint32_t fl = 0;
    int uidx = 0, env = 0, lrope = 0;
    float im = 0.f, lr = 1.f, ks = 0.f;
    QR[t] = make_float4(0.f, 0.f, 0.f, 1.f);
    const int nsdf = (SURF == SURF_MESHES) ? a.num_sdf : 0;
    if constexpr (SURF == SURF_MESHES) {
        for (int e = t; e < bin.rcount * nsdf; e += BLOCK) {
            const int r = e / nsdf, m = e % nsdf;
            const float4* src = reinterpret_cast<const float4*>(a.poses + (size_t)a.ropes[bin.rstart + r].user * kMaxSdf + m);
#pragma unroll
            for (int k = 0; k < kPoseF4; k++) PC[e * kPoseF4 + k] = src[k];
        }
    }
    if (act) {
        const int4 tp = a.topo[dv];
        fl = (uint32_t)tp.x; lrope = tp.y; uidx = tp.z; env = tp.w;
        im = a.pos[dv].w; lr = a.vel[dv].w; ks = a.lvel[dv].w;
        QR[t] = a.qrest[dv];
        if constexpr (kChecked)
            if (!checked_vertex(a, bin, t, uidx, fl, lrope, env, nsdf)) {
                act = false;
                uidx = 0;
            }
    }
    const bool hasNext = fl & F_NEXT, hasPrev = fl & F_PREV, nextOrient = fl & F_NEXT_ORIENT;
    const bool upd = hasNext && !(fl & F_FIX_ORIENT);
    const bool driven = (fl & F_ROOT) && a.root_mode == ROOT_PROGRAM;
    const VConst c = vertex_constants(a, im, lr, ks);
    const float4 qr_own = QR[t];
    const float irho = hasNext ? 1.f / sqrtf(dot4(qr_own, qr_own)) : 0.f;  // 1 / |qRest| of segment t
    KC[t] = make_float4(ks, c.invl, im, irho);
    // rope-rope contact group and rope of this vertex (CTA-local indices)
    int g0 = 0, g1 = 0, r0 = 0, r1 = 0;
    if constexpr (ROPE) {
        CD[t] = zero4();
        CD[BLOCK + t] = zero4();
        CX[t] = zero4();
        if (act) {
            const int4 gr = a.grp[dv];
            g0 = gr.x - bin.vstart; g1 = gr.y - bin.vstart; r0 = gr.z - bin.vstart; r1 = gr.w - bin.vstart;
            if constexpr (kChecked)
                if (!(0 <= g0 && g0 <= r0 && r0 <= t && t < r1 && r1 <= g1 && g1 <= bin.vcount)) {
                    check_fail(a.status, CHK_GROUP);
                    g0 = g1 = r0 = r1 = t;  // no candidates
                }
        }
    }
    const float h = a.h, invH = 1.f / h;
    const float damp = a.damping / h;
    // Without contact terms H is (m / h^2 + k_t / l_t + k_{t-1} / l_{t-1}) I at every iteration of the
    // frame (the forward's hoisted diagonal): its reciprocal and the mass-weight scales are formed once,
    // in the order the reverse position step builds H.
    __syncthreads();  // the neighbours' KC
    float ihxx = 0.f, wscale = 0.f, kscale = 0.f;
    if (im != 0.f) {
        float hxx = c.Hd;
        if (hasNext) hxx += ks * c.invl * c.invl * (1.f + damp);
        if (hasPrev) {
            const float4 kp = KC[t - 1];
            hxx += kp.x * kp.y * kp.y * (1.f + damp);
        }
        ihxx = 1.f / hxx;
        wscale = -c.fm / im;
        kscale = -c.kc / im;
    }
    const f3 gv = mk3(a.gx, a.gy, a.gz);
    const float g2 = dot(gv, gv);
    const int S = a.substeps;
    const size_t n = (size_t)a.n;
    // Constant over the frame: the neighbour slots (a missing neighbour reads the own slot), the
    // frame step's -2k and -2k/l, the stretch reverse's 1/l, k/l and k/l² of the own segment (zero
    // without one) and k/l² of the previous segment, and the damping shares of both.
    const int tp = hasPrev ? t - 1 : t, tn = nextOrient ? t + 1 : t, tn1 = hasNext ? t + 1 : t;
    const float m2ks = -2.f * ks, m2ksil = m2ks * c.invl;
    const float ilo = hasNext ? c.invl : 0.f, ilo2 = ilo * ilo;
    const float kko = ks * ilo, ddo = kko * ilo;
    // (the mesh variant reads the previous segment's from KC where they are used: held in
    // registers they make its lattice path spill)
    auto prev_seg = [&](float& dd, float& ir) {
        const float4 kp = KC[tp];
        const float ilp = hasPrev ? kp.y : 0.f;
        dd = (kp.x * ilp) * ilp;
        ir = kp.w;
    };
    float ddp = 0.f, irho_p = 0.f;
    if constexpr (SURF != SURF_MESHES) prev_seg(ddp, irho_p);
    // The iterate tape also holds each frame step's blend rotor b and its sign tests: b of the next
    // reverse iteration is loaded one iteration ahead (only this vertex reads it). The mesh variant
    // recomputes them instead (the prefetched rotor's registers would make its lattice path spill).
    const bool tb = !ROPE && SURF != SURF_MESHES && g.itape != nullptr;
    const float4* btape = tb ? g.itape + 2 * (size_t)I * n + uidx : nullptr;  // + (s * 3I + k) * n
    float4 bnx = zero4();
    if (tb && act) bnx = __ldcs(btape + ((size_t)(S - 1) * 3 * I + (I - 1)) * n);

    // adjoints of the frame-end state
    f3 xb = zero3(), vb = zero3(), lvb = zero3();
    float4 qb = zero4();
    if (act) {
        if (g.g_pos) xb = ld3(g.g_pos, uidx);
        if (g.g_vel) vb = ld3(g.g_vel, uidx);
        if (g.g_lvel) lvb = ld3(g.g_lvel, uidx);
        if (g.g_q) qb = reinterpret_cast<const float4*>(g.g_q)[uidx];
    }
    f3 P0b = zero3(), V0b = zero3(), P1b = zero3();
    float ksb = 0.f, rhob = 0.f, rhobp = 0.f, wb = 0.f;

    for (int s = S - 1; s >= 0; s--) {
        // ---- the substep's start state (after its root program) from the tape
        f3 p = zero3(), v = zero3(), lvin = zero3();
        float4 q = make_float4(0.f, 0.f, 0.f, 1.f);
        uint64_t cand = 0ull;  // the forward's broad-phase mask of this substep (tape .w lanes)
        if (act) {
            float4 t0, t1, t2, t3;
            if (!ROPE && g.itape && s < S - 1) {  // copied into this thread's slots during substep s + 1
                cp_async_wait_all();
                t0 = X[t]; t1 = EA[t]; t2 = EB[t]; t3 = EC[t];
            } else {
                const float4* ts = g.tape + (size_t)s * 4 * n + uidx;
                t0 = __ldcs(ts); t1 = __ldcs(ts + n); t2 = __ldcs(ts + 2 * n); t3 = __ldcs(ts + 3 * n);
            }
            p = xyz(t0); v = xyz(t1); lvin = xyz(t2); q = t3;
            cand = (uint64_t)(uint32_t)__float_as_int(t0.w) | ((uint64_t)(uint32_t)__float_as_int(t1.w) << 32);
            if constexpr (kChecked)
                if (cand & ~all_meshes(nsdf)) {  // the tape's mask names a mesh the pose cache does not hold
                    check_fail(a.status, CHK_POSE);
                    cand &= all_meshes(nsdf);
                }
        }
        const float4* mycache = PC + (size_t)lrope * nsdf * kPoseF4;
        f3 dx, y;
        init_vertex(v, lvin, im, h, a.last_h, gv, g2, dx, y);
        X[t] = f4(p, 0.f);
        LD[t] = f4(dx, 1.f);
        LQ[t] = q;
        if constexpr (ROPE) RP[t] = make_float4(a.sdet_radius + len(y), INFINITY, __int_as_float((int)fl), 0.f);
        __syncthreads();
        const f3 p1 = hasNext ? xyz(X[t + 1]) : zero3();
        const f3 p1mp = p1 - p;

        // ---- rope-rope detection and step limit (the frame kernel's, from the same inputs)
        int ncol = 0;
        float lim = INFINITY;
        if constexpr (ROPE) {
            if (hasNext) {
                const int cnt = detect_group(
                    a, t, dv, g0, g1, r0, r1, p, p1, [&](int j) { return RP[j].x; },
                    [&](int j) { return __float_as_int(RP[j].z); }, [&](int j) { return xyz(X[j]); }, lim);
                ncol = cnt < kMaxCols ? cnt : kMaxCols;
            }
            RP[t].y = lim;
        }

        // ---- the iterates: from the forward's iterate tape, or recomputed (the frame kernel's
        // arithmetic). Levels 1..I of the tape arrive by asynchronous copies: the last substep's
        // here, every other substep's during the reverse of the substep after it, each level into
        // its slot as soon as that reverse is done with it.
        if (!ROPE && g.itape) {
            if (s == S - 1 && act) {
                for (int k = 0; k < I; k++) {
                    cp_async16(LD + (size_t)(k + 1) * BLOCK + t, g.itape + (size_t)(s * 3 * I + k) * n + uidx);
                    cp_async16(LQ + (size_t)(k + 1) * BLOCK + t, g.itape + (size_t)(s * 3 * I + I + k) * n + uidx);
                }
                cp_async_commit();
            }
            cp_async_wait_all();
            dx = xyz(LD[(size_t)I * BLOCK + t]);
            q = LQ[(size_t)I * BLOCK + t];
        } else {
            for (int k = 0; k < I; k++) {
                f3 f, f2;
                sym3 H, H2;
                const float4* Dk = LD + (size_t)k * BLOCK;
                const f3 p1dx = hasNext ? xyz(Dk[t + 1]) : zero3();
                const bool touched =
                    position_terms<SURF>(a, mycache, cand, c, hasNext, p, p1, dx, p1dx, y, q, damp, f, H, f2, H2);
                if constexpr (ROPE)
                    collision_sectors(a, ncol, dv, X, Dk, damp, p, p1, dx, p1dx, f, f2, H, H2, bin.vcount);
                // without rope contact H2 is dd I (position_terms): one float4 carries the exchange
                EA[t] = f4(f2, H2.xx);
                if constexpr (ROPE) {
                    EB[t] = make_float4(H2.yy, H2.zz, H2.xy, H2.xz);
                    EC[t].x = H2.yz;
                }
                __syncthreads();
                if (hasPrev) {
                    const float4 fa = EA[t - 1];
                    f += xyz(fa);
                    if constexpr (ROPE) {
                        const float4 fb = EB[t - 1];
                        H.xx += fa.w; H.yy += fb.x; H.zz += fb.y; H.xy += fb.z; H.xz += fb.w; H.yz += EC[t - 1].x;
                    } else {
                        H.xx += fa.w; H.yy += fa.w; H.zz += fa.w;
                    }
                }
                float sc = 1.f;
                if constexpr (ROPE)
                    sc = position_solve_limited(dx, f, H, a.accel, im, hasPrev ? fminf(lim, RP[t - 1].y) : lim);
                else position_solve(dx, f, H, a.accel, im, !touched);
                LD[(size_t)(k + 1) * BLOCK + t] = f4(dx, sc);
                __syncthreads();
                if (upd) {
                    const f3 seg = (p1 - p) + (xyz(LD[(size_t)(k + 1) * BLOCK + t + 1]) - dx);
                    const float4* Lk = LQ + (size_t)k * BLOCK;
                    q = frame_update(q, seg, c.invl, ks, hasPrev, hasPrev ? Lk[t - 1] : q, hasPrev ? QR[t - 1] : q,
                                     nextOrient, nextOrient ? Lk[t + 1] : q, QR[t]);
                }
                LQ[(size_t)(k + 1) * BLOCK + t] = q;
            }
        }
        // prefetched levels were complete before the barrier after the start state (every thread
        // waited for its copies there); otherwise the levels just written need one
        if (ROPE || !g.itape || s == S - 1) __syncthreads();

        // ---- end of substep reversed: x' = x + d, v' = drag(d / h), lv' = v
        f3 db = xb;
        f3 vbn = lvb, lvbn = zero3(), yb = zero3();
        float4 qpart = zero4();   // quadratic-drag share on the previous vertex's frame (rope ends)
        if (im != 0.f) {
            const f3 ob = vb * (1.f - a.drag * h);
            f3 vbar = ob;
            if (a.drag_quad > 0.f) {
                const float4 tq = hasNext ? q : LQ[(size_t)I * BLOCK + ((kChecked && t == 0) ? 0 : t - 1)];
                const f3 tg = qtangent(tq);
                const f3 vv = dx * invH;
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
        if (a.drag_quad > 0.f) {
            EF[t] = qpart;
            __syncthreads();
            if (hasNext) qb = add4(qb, EF[t + 1]);
        }
        float msb = 0.f, msbp = 0.f;  // step-limit adjoints of this segment's limit and the previous one's

        // ---- iterations reversed
        for (int k = I - 1; k >= 0; k--) {
            const float4* Lq = LQ + (size_t)k * BLOCK;
            const float4* Dk = LD + (size_t)k * BLOCK;
            const float4* Dn = LD + (size_t)(k + 1) * BLOCK;
            const float4* Dq = LQ + (size_t)(k + 1) * BLOCK;
            // frame step k: q^{k+1}_t = normalize(vv b e1 + (|vv| + |b|) b)
            float4 own = qb, toL = zero4(), toR = zero4();
            f3 su = zero3();
            const float4 bk = bnx;
            if (tb && act && (k > 0 || s > 0))
                bnx = __ldcs(btape + ((size_t)(k > 0 ? s : s - 1) * 3 * I + (k > 0 ? k - 1 : I - 1)) * n);
            if (upd) {
                own = zero4();
                const f3 u = (p1mp + (xyz(Dn[t + 1]) - xyz(Dn[t]))) * c.invl;
                const f3 vv = u * m2ks;
                const float4 qp = Lq[tp], rp = QR[tp];
                const float4 qn = Lq[tn], rn = QR[t];
                float spv, snv;
                float4 b;
                if (tb) {  // the forward's b and sign tests, from the iterate tape
                    frame_signs_decode(Dn[t].w, spv, snv);
                    b = bk;
                } else {   // both neighbour products, the missing ones selected away (as frame_update)
                    const float4 q0 = Lq[t];
                    const float4 pr = qmul(qp, rp), nx = qmul(qn, qconj(rn));
                    spv = dot4(q0, pr) > 0.f ? 1.f : -1.f;
                    snv = dot4(q0, nx) > 0.f ? 1.f : -1.f;
                    b = hasPrev ? scale4(pr, spv) : zero4();
                    const float4 bn = add4(b, scale4(nx, snv));
                    b = nextOrient ? bn : b;
                }
                const float sp = hasPrev ? spv : 0.f, sn = nextOrient ? snv : 0.f;
                float ilvv, ilb, lambda;  // the forward's z (frame_z), so the reverse linearises what ran
                const float4 z = frame_z(vv, b, ilvv, ilb, lambda);
                const float izl = rsqrt_nr(dot4(z, z));
                const float4 qo = Dq[t];  // q^{k+1} = z / |z|, as the forward stored it
                const float4 zb = scale4(fma4(qo, -dot4(qo, qb), qb), izl);
                const float lamb = dot4(zb, b);
                f3 vvb = vv * (lamb * ilvv);
                float4 bb = fma4(b, lamb * ilb, scale4(zb, lambda));
                const float4 Ab = scale4(qmul_e1(zb), -1.f);   // z = A e1  ->  Ā = z̄ e1* = -(z̄ e1)
                vvb = qmul_vec_add(Ab, qconj(b), vvb);           // A = (vv, 0) b: vv̄ += vec(Ā b*)
                {                                                // b̄ += (vv, 0)* Ā = -(vv, 0) Ā
                    const f3 Av = xyz(Ab);
                    const f3 r = fma3(vv, -Ab.w, cross_add(Av, vv, xyz(bb)));
                    bb = make_float4(r.x, r.y, r.z, dot_add(vv, Av, bb.w));
                }
                ksb = fmaf(-2.f, dot(u, vvb), ksb);
                su = vvb * m2ksil;
                // b = sp q_{t-1} r_{t-1} + sn q_{t+1} r_t^*: the rotor adjoints b̄ r^(*) also give the
                // rest-rotor magnitude adjoints, <q^* b̄, r> = <b̄ r^*, q> and <(q^* b̄)^*, r> = <b̄ r, q>
                toL = qmul(scale4(bb, sp), qconj(rp));  // zero without the neighbour (sp, sn = 0)
                if constexpr (SURF == SURF_MESHES) prev_seg(ddp, irho_p);
                rhobp = fmaf(dot4(toL, qp), irho_p, rhobp);
                toR = qmul(scale4(bb, sn), rn);
                rhob = fmaf(dot4(toR, qn), irho, rhob);
            }
            EA[t] = toL;
            EB[t] = toR;
            EC[t] = f4(su, 0.f);
            // the segment's collision Hessians at d^k: its first vertex's share stays here, the
            // second's goes to vertex t+1
            sym3 HcA = sym_zero();
            if constexpr (ROPE) {
                f3 fd = zero3(), f2d = zero3();
                sym3 HcB = sym_zero();
                if (hasNext)
                    collision_sectors(a, ncol, dv, X, Dk, damp, p, p1, xyz(Dk[t]), xyz(Dk[t + 1]), fd, f2d, HcA, HcB,
                                      bin.vcount);
                HB0[t] = make_float4(HcB.xx, HcB.yy, HcB.zz, HcB.xy);
                HB1[t] = make_float4(HcB.xz, HcB.yz, 0.f, 0.f);
            }
            __syncthreads();
            {
                const float4 ebp = EB[tp], ean = EA[tn1];
                const float4 q1 = add4(own, ebp);
                qb = hasPrev ? q1 : own;
                const float4 q2 = add4(qb, ean);
                qb = hasNext ? q2 : qb;
                const f3 dp = -su + xyz(EC[tp]);
                const f3 dd = hasPrev ? dp : -su;
                db += dd;
                xb += dd;
            }
            if constexpr (ROPE) {  // pair contributions to d̄^{k+1} from the reverse of position step k+1
                float4* cd = CD + ((k + 1) & 1) * BLOCK + t;
                db += xyz(*cd);
                *cd = zero4();
            }

            // position step k: d^{k+1}_t = limit(d^k_t + a H_t^-1 F_t)
            const f3 dk = xyz(Dk[t]);
            f3 dn = db;
            f3 Fb = zero3(), e = zero3(), del = zero3();
            float trH = 0.f;
            if (im != 0.f) {
                sym3 H = sym_diag(c.Hd);
                bool touched = false;
                if constexpr (SURF != SURF_NONE) {
                    f3 fdummy = zero3();
                    touched = surfaces<SURF>(a, mycache, cand, p, dk, c.kc, h, fdummy, H, nullptr, nullptr);
                }
                if (SURF != SURF_NONE || ROPE) {  // H beyond its diagonal only where contact can touch it
                    if (hasNext) {
                        const float dd = ks * c.invl * c.invl * (1.f + damp);
                        H.xx += dd; H.yy += dd; H.zz += dd;
                    }
                    if (hasPrev) {
                        const float4 kp = KC[t - 1];
                        const float dd = kp.x * kp.y * kp.y * (1.f + damp);
                        H.xx += dd; H.yy += dd; H.zz += dd;
                    }
                }
                f3 gb = db;
                f3 zk = xyz(Dn[t]);  // the solve's result before the step limit
                if constexpr (ROPE) {
                    sym_add(H, HcA);
                    if (hasPrev) {
                        const float4 h0 = HB0[t - 1], h1 = HB1[t - 1];
                        H.xx += h0.x; H.yy += h0.y; H.zz += h0.z; H.xy += h0.w; H.xz += h1.x; H.yz += h1.y;
                    }
                    touched = true;
                    // d' = z lim / |z| when |z| > lim (cosserat.cu:211-214): z̄ = (lim/|z|)(I - ẑẑᵀ) d̄',
                    // and ẑ.d̄' is the adjoint of the limit, min(own, previous segment's)
                    const float sc = Dn[t].w;
                    if (sc < 1.f) {
                        const float l = len(zk);
                        const f3 zh = zk * (1.f / l);
                        const float zg = dot(zh, gb);
                        if (hasPrev && RP[t - 1].y < lim) msbp += zg;
                        else msb += zg;
                        gb = (gb - zh * zg) * sc;
                        zk = zk * (1.f / sc);
                    }
                    dn = gb;
                }
                e = touched ? sym_solve(H, gb) : gb * ihxx;
                del = zk - dk;
                Fb = e * a.accel;
                trH = -dot(e, del);
                yb = fma3(Fb, c.fm, yb);
                dn = fma3(Fb, -c.fm, dn);
                float wsum = dot_add(y - dk, Fb, trH) * wscale;
                if constexpr (SURF != SURF_NONE) {
                    for (int pl = 0; pl < a.num_planes; pl++) {
                        const float4 P = a.planes[pl];
                        const f3 nrm = mk3(P.x, P.y, P.z);
                        const float gap = (dot(nrm, p) - P.w) + dot(nrm, dk) - a.c_radius;
                        if (gap >= 0.f) continue;
                        float gapb, kb;
                        f3 nb;
                        surface_contact_bwd(nrm, gap, dk, c.kc, h, a.c_mu_s, a.c_mu_k, a.c_vslip, Fb, e, del, dn, gapb,
                                            kb, nb);
                        dn += nrm * gapb;
                        xb += nrm * gapb;
                        wsum += kb * kscale;
                    }
                }
                if constexpr (SURF == SURF_MESHES)
                    wsum += mesh_contact_bwd(a, mycache, cand, p, dk, c.kc, h, Fb, e, del, dn, xb) * kscale;
                wb += wsum;
            }
            // segment t's residual c = ((x1 - x) + (d1 - d)) / l - t(q), read before the barrier:
            // after it a neighbour may already be writing the next substep's iterates
            const float4 qk = Lq[t];
            const f3 dkn = hasNext ? xyz(Dk[t + 1]) : zero3();
            const f3 cc = hasNext ? fma3(p1mp + (dkn - dk), c.invl, -qtangent(qk)) : zero3();
            EF[t] = f4(Fb, trH);
            if constexpr (ROPE) EE[t] = f4(e, 0.f);
            __syncthreads();
            // level k+1 is read by no one any more: fetch the previous substep's into its slot;
            // after the last reverse iteration the exchange slots X, EA, EB, EC are free as well
            // and take the previous substep's start state
            if (!ROPE && g.itape && s > 0 && act) {
                cp_async16(LD + (size_t)(k + 1) * BLOCK + t, g.itape + (size_t)((s - 1) * 3 * I + k) * n + uidx);
                cp_async16(LQ + (size_t)(k + 1) * BLOCK + t, g.itape + (size_t)((s - 1) * 3 * I + I + k) * n + uidx);
                if (k == 0) {
                    const float4* ts = g.tape + (size_t)(s - 1) * 4 * n + uidx;
                    cp_async16(X + t, ts);
                    cp_async16(EA + t, ts + n);
                    cp_async16(EB + t, ts + 2 * n);
                    cp_async16(EC + t, ts + 3 * n);
                }
                cp_async_commit();
            }
            if constexpr (!ROPE) {
                // the stretch terms of segments t and t-1 reversed, without branches: a missing
                // segment contributes with zero stiffness (its reads stay in the CTA's own slot)
                const float4 Fn4 = EF[tn1];
                const f3 Fn = xyz(Fn4);
                const f3 dF = Fb - Fn;
                const float sx = fmaf(-damp, dot_add(dkn, Fn, dot(dk, Fb)), (1.f + damp) * (trH + Fn4.w));
                ksb = fmaf(sx, ilo2, fmaf(dot(cc, dF), ilo, ksb));
                qb = sub4(qb, tangent_vjp(qk, dF * kko));
                dn = fma3(dF, -ddo, dn);
                xb = fma3(dF, -ddo, xb);
                if constexpr (SURF == SURF_MESHES) prev_seg(ddp, irho_p);
                const f3 dFp = xyz(EF[tp]) - Fb;
                dn = fma3(dFp, ddp, dn);
                xb = fma3(dFp, ddp, xb);
                dn = fma3(Fb, -(damp * ddo + damp * ddp), dn);
            } else {
                if (hasNext) {
                    const float4 Fn4 = EF[t + 1];
                    const f3 Fn = xyz(Fn4);
                    const float kk = ks * c.invl, dd = kk * c.invl;
                    const f3 dF = Fb - Fn;
                    const f3 cb = dF * kk;
                    ksb += dot(cc, dF) * c.invl +
                           (-damp * (dot(dk, Fb) + dot(dkn, Fn)) + (1.f + damp) * (trH + Fn4.w)) * c.invl * c.invl;
                    qb = add4(qb, scale4(tangent_vjp(qk, cb), -1.f));
                    dn -= cb * c.invl;
                    xb -= cb * c.invl;
                    dn -= Fb * (damp * dd);
                    if constexpr (ROPE) {
                        if (ncol > 0) {  // the segment's pairs reversed; other vertices' shares by shared-memory atomics
                            const float4 zn4 = Dn[t + 1];
                            const f3 lc = xyz(zn4) * (1.f / zn4.w) - dkn;
                            const f3 ec = xyz(EE[t + 1]);
                            PairGrad acc{};
                            float4* cdk = CD + (k & 1) * BLOCK;
                            for (int q2 = 0; q2 < ncol; q2++) {
                                const int j = a.cols[(size_t)q2 * n + dv];
                                PairGrad o{};
                                collision_bwd(a, damp, p, p1, xyz(X[j]), xyz(X[j + 1]), dk, dkn, xyz(Dk[j]), xyz(Dk[j + 1]),
                                              Fb, e, del, Fn, ec, lc, o);
                                acc.x0 += o.x0; acc.d0 += o.d0; acc.x1 += o.x1; acc.d1 += o.d1;
                                atomic_add3(cdk + j, o.e0);
                                atomic_add3(cdk + j + 1, o.e1);
                                atomic_add3(CX + j, o.y0);
                                atomic_add3(CX + j + 1, o.y1);
                            }
                            dn += acc.d0;
                            xb += acc.x0;
                            atomic_add3(cdk + t + 1, acc.d1);
                            atomic_add3(CX + t + 1, acc.x1);
                        }
                    }
                }
                if (hasPrev) {
                    const float4 kp = KC[t - 1];
                    const float kkp = kp.x * kp.y, ddp = kkp * kp.y;
                    const f3 cbp = (xyz(EF[t - 1]) - Fb) * kkp;
                    dn += cbp * kp.y;
                    xb += cbp * kp.y;
                    dn -= Fb * (damp * ddp);
                }
            }
            db = dn;
        }

        if constexpr (ROPE) {
            // step-limit adjoints: the previous segment's share, then the limits reversed (the
            // limit of segment t rests on the substep-start positions and the padding of y)
            RP[t].w = msbp;
            __syncthreads();
            db += xyz(CD[t]);  // pair contributions to d̄^0
            CD[t] = zero4();
            if (hasNext) msb += RP[t + 1].w;
            if (hasNext && msb != 0.f) {
                f3 xb1 = zero3(), xj0 = zero3(), xj1 = zero3();
                int jo;
                const f3 ybl = step_limit_bwd(a, dv, ncol, X, p, p1, RP[t].x, y, msb, xb, xb1, jo, xj0, xj1);
                vbn += ybl * h;  // y = v h + g h²
                atomic_add3(CX + t + 1, xb1);
                if (jo >= 0) {
                    atomic_add3(CX + jo, xj0);
                    atomic_add3(CX + jo + 1, xj1);
                }
            }
            __syncthreads();
            xb += xyz(CX[t]);
            CX[t] = zero4();
        }

        // ---- inertial prediction reversed: d^0 = v h + g h² s(v, lv), y = v h + g h²
        if (im != 0.f) {
            vbn += (db + yb) * h;
            if (g2 > 0.f) {
                const f3 acc = (v - lvin) / a.last_h;
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
        // ---- root program reversed: x = P0 + V0 tau + A tau²/2, v = V0 + A (tau + h/2)
        if (driven) {
            const float dt = a.dt, tau = float(s) * h, th = tau + 0.5f * h, idt2 = 2.f / (dt * dt);
            const float xa = 0.5f * tau * tau * idt2;
            P0b += xb * (1.f - xa) + vbn * (-th * idt2);
            V0b += xb * (tau - xa * dt) + vbn * (1.f - th * idt2 * dt);
            P1b += xb * xa + vbn * (th * idt2);
            xb = zero3();
            vbn = zero3();
            if (a.has_q0) qb = zero4();
        }
        vb = vbn;
        lvb = lvbn;
    }

    // ---- outputs (caller order); segment t's bending adjoint also has vertex t+1's share
    EA[t] = make_float4(rhobp, 0.f, 0.f, 0.f);
    __syncthreads();
    if (act) {
        st3(g.o_pos, uidx, xb);
        st3(g.o_vel, uidx, vb);
        st3(g.o_lvel, uidx, lvb);
        reinterpret_cast<float4*>(g.o_q)[uidx] = qb;
        const float rho = rhob + (hasNext ? EA[t + 1].x : 0.f);
        if (g.o_ea) g.o_ea[uidx] = hasNext ? ksb * lr : 0.f;        // kStretch = EA lRest
        if (g.o_ei) g.o_ei[uidx] = hasNext ? rho * 4.f / lr : 0.f;  // |qRest| = 4 EI / lRest
        if (g.o_mass) g.o_mass[uidx] = (im != 0.f) ? -im * im * wb : 0.f;
        if (driven) {
            if (g.o_p0) st3(g.o_p0, env, P0b);
            if (g.o_v0) st3(g.o_v0, env, V0b);
            if (g.o_p1) st3(g.o_p1, env, P1b);
        }
    }
}

template <int BLOCK, int SURF, bool ROPE>
cudaError_t launch_adjoint_t(const FrameArgs& a, const AdjArgs& g, int num_bins, cudaStream_t s) {
    auto k = adjoint_kernel<BLOCK, SURF, ROPE>;
    const size_t bytes = adjoint_smem_bytes(BLOCK, a.iters, ROPE) +
                         (SURF == SURF_MESHES ? (size_t)a.pose_cache * kPoseF4 * sizeof(float4) : 0);
    if (bytes > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e != cudaSuccess) return e;
    }
    k<<<num_bins, BLOCK, bytes, s>>>(a, g);
    return cudaGetLastError();
}
template <int BLOCK, bool ROPE>
cudaError_t launch_adjoint_r(const FrameArgs& a, const AdjArgs& g, int num_bins, cudaStream_t s) {
    if (a.num_sdf > 0) return launch_adjoint_t<BLOCK, SURF_MESHES, ROPE>(a, g, num_bins, s);
    if (a.num_planes > 0) return launch_adjoint_t<BLOCK, SURF_PLANES, ROPE>(a, g, num_bins, s);
    return launch_adjoint_t<BLOCK, SURF_NONE, ROPE>(a, g, num_bins, s);
}
template <int BLOCK>
cudaError_t launch_adjoint_b(const FrameArgs& a, const AdjArgs& g, int num_bins, cudaStream_t s) {
    return a.rope_contact ? launch_adjoint_r<BLOCK, true>(a, g, num_bins, s) : launch_adjoint_r<BLOCK, false>(a, g, num_bins, s);
}

// Caller-order state (pos / vel / lvel [n,3], q [n,4]) into device order, keeping the
// per-vertex constants stored in the .w lanes (invMass, lRest, kStretch) of `cst_*`.
__global__ void state_in_kernel(const int4* topo, const float* pos, const float* vel, const float* lvel, const float* q,
                                const float4* cst_pos, const float4* cst_vel, const float4* cst_lvel, float4* o_pos,
                                float4* o_vel, float4* o_lvel, float4* o_q, int n) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const int u = topo[d].z;
    if (pos) o_pos[d] = f4(ld3(pos, u), cst_pos[d].w);
    if (vel) o_vel[d] = f4(ld3(vel, u), cst_vel[d].w);
    if (lvel) o_lvel[d] = f4(ld3(lvel, u), cst_lvel[d].w);
    if (q) o_q[d] = reinterpret_cast<const float4*>(q)[u];
}
__global__ void state_out_kernel(const int4* topo, const float4* pos, const float4* vel, const float4* lvel,
                                 const float4* q, float* o_pos, float* o_vel, float* o_lvel, float* o_q, int n) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const int u = topo[d].z;
    if (o_pos) st3(o_pos, u, xyz(pos[d]));
    if (o_vel) st3(o_vel, u, xyz(vel[d]));
    if (o_lvel) st3(o_lvel, u, xyz(lvel[d]));
    if (o_q) reinterpret_cast<float4*>(o_q)[u] = q[d];
}
// Per-vertex parameters in caller order: EA (kStretch = EA lRest), EI (qRest = its unit direction
// scaled by 4 EI / lRest, so that setting the same EI twice gives the same rotor) on vertices
// that own a segment, mass (invMass = 1 / mass) on free vertices.
__global__ void params_in_kernel(const int4* topo, const float* ea, const float* ei, const float* mass, float4* pos,
                                 const float4* vel, float4* lvel, float4* qrest, const float4* qdir, int n) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const int4 tp = topo[d];
    const int u = tp.z;
    const bool seg = (tp.x & F_NEXT) != 0;
    const float lr = vel[d].w;
    if (ea && seg) lvel[d].w = ea[u] * lr;
    if (ei && seg) qrest[d] = scale4(qdir[d], 4.f * ei[u] / lr);
    if (mass && pos[d].w != 0.f) pos[d].w = 1.f / mass[u];
}
__global__ void params_out_kernel(const int4* topo, const float4* pos, const float4* vel, const float4* lvel,
                                  const float4* qrest, float* ea, float* ei, float* mass, int n) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const int4 tp = topo[d];
    const int u = tp.z;
    const bool seg = (tp.x & F_NEXT) != 0;
    const float lr = vel[d].w;
    if (ea) ea[u] = seg ? lvel[d].w / lr : 0.f;
    if (ei) ei[u] = seg ? sqrtf(dot4(qrest[d], qrest[d])) * lr * 0.25f : 0.f;
    if (mass) mass[u] = pos[d].w != 0.f ? 1.f / pos[d].w : 0.f;
}

}  // namespace

size_t adjoint_smem_bytes(int block, int iters, bool rope) {
    return sizeof(float4) * (size_t)block * (size_t)(2 * iters + 9 + (rope ? 7 : 0));
}

cudaError_t launch_adjoint(const FrameArgs& a, const AdjArgs& g, int block, int num_bins, cudaStream_t s) {
    switch (block) {
        case 64: return launch_adjoint_b<64>(a, g, num_bins, s);
        case 128: return launch_adjoint_b<128>(a, g, num_bins, s);
        case 256: return launch_adjoint_b<256>(a, g, num_bins, s);
        case 512: return launch_adjoint_b<512>(a, g, num_bins, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_state_in(const int4* topo, const float* pos, const float* vel, const float* lvel, const float* q,
                            const float4* cst_pos, const float4* cst_vel, const float4* cst_lvel, float4* o_pos,
                            float4* o_vel, float4* o_lvel, float4* o_q, int n, cudaStream_t s) {
    state_in_kernel<<<(n + 255) / 256, 256, 0, s>>>(topo, pos, vel, lvel, q, cst_pos, cst_vel, cst_lvel, o_pos, o_vel,
                                                     o_lvel, o_q, n);
    return cudaGetLastError();
}
cudaError_t launch_state_out(const int4* topo, const float4* pos, const float4* vel, const float4* lvel, const float4* q,
                             float* o_pos, float* o_vel, float* o_lvel, float* o_q, int n, cudaStream_t s) {
    state_out_kernel<<<(n + 255) / 256, 256, 0, s>>>(topo, pos, vel, lvel, q, o_pos, o_vel, o_lvel, o_q, n);
    return cudaGetLastError();
}
cudaError_t launch_params_in(const int4* topo, const float* ea, const float* ei, const float* mass, float4* pos,
                             const float4* vel, float4* lvel, float4* qrest, const float4* qdir, int n, cudaStream_t s) {
    params_in_kernel<<<(n + 255) / 256, 256, 0, s>>>(topo, ea, ei, mass, pos, vel, lvel, qrest, qdir, n);
    return cudaGetLastError();
}
cudaError_t launch_params_out(const int4* topo, const float4* pos, const float4* vel, const float4* lvel,
                              const float4* qrest, float* ea, float* ei, float* mass, int n, cudaStream_t s) {
    params_out_kernel<<<(n + 255) / 256, 256, 0, s>>>(topo, pos, vel, lvel, qrest, ea, ei, mass, n);
    return cudaGetLastError();
}

}  // namespace rs
