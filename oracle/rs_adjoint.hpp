// rs_adjoint.hpp -- TEST INFRASTRUCTURE ONLY. Hand-written reverse-mode adjoint of one control
// frame of rso::Sim<T> (rs_oracle.hpp), the FP64 checker of the CUDA adjoint kernel. It is
// itself pinned on the CPU by FP64 central finite differences of Sim<double> and by an FP64
// torch-autograd restatement of the same update (oracle/torch_rods.py).
//
// The reference has no gradients; the update differentiated here is the deterministic
// (SNAPSHOT) substep it runs (iteration.cu:34-129, cosserat.cu:23-273, contact.cuh:27-46,
// batch.cu:122-159). The adjoint is exact for the discrete update: every iteration of the
// local solve and every frame step is reversed, not only the converged state. Branches that
// switch terms on and off (contact active, friction regime, sign choices of the frame step,
// clamps) are held at the branch the forward pass took ("differentiated through the active set").
//
// Per substep, given the adjoints of the end state (x', v', lv', q'):
//   end     x' = x + d^I, v' = drag(d^I / h), lv' = v            -> x̄, d̄^I, v̄, q̄^I
//   k = I-1 .. 0:
//     frame    q^{k+1}_i = normalize(vv b e1 + (|vv| + |b|) b)    -> q̄^k (neighbours), d̄^{k+1}, x̄, k̄s, ρ̄
//     position d^{k+1}_i = d^k_i + a H_i^-1 F_i                   -> d̄^k, x̄, ȳ, q̄^k (tangents), k̄s, w̄
//       with F̄ = a H^-1 ḡ and H̄ = -(H^-1 ḡ) δᵀ, δ = d^{k+1} - d^k (H is symmetric)
//   init    d^0 = v h + g h² s(v, lv), y = v h + g h²            -> v̄, l̄v
//   program x_root, v_root = P(P0, V0, P1; s)                     -> P̄0, V̄0, P̄1
// Quaternion products c = a b reverse as ā = c̄ b*, b̄ = a* c̄ (left and right multiplication
// are transposed by conjugation). Contributions that cross vertices are gathered per vertex,
// the same decomposition the CUDA kernel uses.
#pragma once

#include "rs_oracle.hpp"

namespace rso {

template <class T> inline Q4<T> qc(const Q4<T>& a) { return Q4<T>(-a.x, -a.y, -a.z, a.w); }

// Transposed Jacobian of the tangent t(q) = q e_x q*:  q̄ = J_t(q)ᵀ t̄.
template <class T> inline Q4<T> tangent_vjp(const Q4<T>& q, const V3<T>& tb) {
    return Q4<T>(T(2) * (q.x * tb.x + q.y * tb.y + q.z * tb.z), T(2) * (-q.y * tb.x + q.x * tb.y - q.w * tb.z),
                 T(2) * (-q.z * tb.x + q.w * tb.y + q.x * tb.z), T(2) * (q.w * tb.x + q.z * tb.y - q.y * tb.z));
}

// Adjoints of a frame's start state, of its root program and of the per-vertex parameters.
// Parameters: ks = kStretch (EA l), rho = |qRest| (4 EI / l), w = invMass.
template <class T> struct FrameGrad {
    std::vector<V3<T>> x, v, lv;
    std::vector<Q4<T>> q;
    std::vector<V3<T>> P0, V0, P1;
    std::vector<T> ks, rho, w;
    void init(int n, int R) {
        x.assign(n, V3<T>()); v.assign(n, V3<T>()); lv.assign(n, V3<T>()); q.assign(n, Q4<T>(0, 0, 0, 0));
        P0.assign(R, V3<T>()); V0.assign(R, V3<T>()); P1.assign(R, V3<T>());
        ks.assign(n, T(0)); rho.assign(n, T(0)); w.assign(n, T(0));
    }
};

template <class T> class FrameAdjoint {
public:
    explicit FrameAdjoint(Sim<T>& sim) : s(sim) {}

    // Reverse one frame. On entry the Sim holds the frame's START state (pos, vel, lastVel, q,
    // h and lastH as left by the previous frame) and g.x/v/lv/q hold the adjoints of its END
    // state; on return g.x/v/lv/q hold the adjoints of the start state, g.P0/V0/P1 those of the
    // program rows (zero when prog == nullptr: a free frame) and g.ks/rho/w have been ADDED to.
    // The Sim is left at the frame's end state. prog is [p0 (3R), v0 (3R), p1 (3R)].
    void frame_backward(const T* prog, bool has_q0, const float* q0, const float* q1, float dt, int S, FrameGrad<T>& g) {
        if (s.pendingSet) throw std::invalid_argument("oracle adjoint: only static meshes are differentiated");
        const int n = s.n;
        s.sdf_begin_step();
        s.prepare(T(dt / (float)S));
        // forward replay: substep-start states
        std::vector<State> st(S);
        for (int k = 0; k < S; k++) {
            st[k].save(s);
            if (prog) s.apply_root_program(prog, q0, q1, k, S, dt);
            s.substep(k, S);
        }
        State end;
        end.save(s);
        // reverse
        for (int k = S - 1; k >= 0; k--) {
            st[k].load(s);
            substep_backward(k, S, dt, prog, has_q0 && prog != nullptr, q0, q1, g);
        }
        end.load(s);
        s.finish(dt);
        s.sdf_end_step(S);
        (void)n;
    }

private:
    Sim<T>& s;
    std::vector<T> msb;  // adjoints of the substep's step limits (maxStep)
    struct State {
        std::vector<V3<T>> pos, vel, lastVel;
        std::vector<Q4<T>> q;
        std::vector<int> numCand;              // broad-phase candidate lists of the substep
        std::vector<std::vector<int>> cand;
        void save(const Sim<T>& m) {
            pos = m.pos; vel = m.vel; lastVel = m.lastVel; q = m.q; numCand = m.numCand; cand = m.cand;
        }
        void load(Sim<T>& m) const {
            m.pos = pos; m.vel = vel; m.lastVel = lastVel; m.q = q; m.numCand = numCand; m.cand = cand;
        }
    };

    bool has(int i, uint32_t f) const { return (s.flags[i] & f) != 0; }

    // Contact reverse (contact.cuh:27-46): f += n N - ut kt, H += k nnᵀ - kt (nnᵀ - I), with
    // N = -k gap and ut = d - n (n.d). Given F̄ and H̄ = -e δᵀ, adds to d̄ and returns the adjoints
    // of the gap, of the penalty stiffness k and of the normal n.
    void surface_contact_bwd(const V3<T>& nrm, T gap, const V3<T>& d, T k, T muS, T muK, const V3<T>& Fb,
                             const V3<T>& e, const V3<T>& delta, V3<T>& db, T& gapb, T& kb, V3<T>& nb) const {
        const T nHn = -dot(nrm, e) * dot(nrm, delta), trHb = -dot(e, delta);
        const T eps = s.cVSlip, h = s.h;
        const T N = -k * gap;
        const V3<T> ut = d - nrm * dot(nrm, d);
        const T ul = len(ut);
        const T vt = ul / h;
        T Nb = dot(nrm, Fb);
        kb = nHn;
        T kt;
        T mu = 0, xr = 0;
        if (vt <= eps) kt = muS * N / (eps * h);
        else {
            xr = vt / eps - T(1);
            const T sw = T(1) - std::min(T(1), xr);
            mu = sw * muS + (T(1) - sw) * muK;
            kt = mu * N / ul;
        }
        V3<T> utb = Fb * (-kt);
        const T ktb = -dot(ut, Fb) - (nHn - trHb);
        if (vt <= eps) Nb += ktb * muS / (eps * h);
        else {
            Nb += ktb * mu / ul;
            T ulb = -ktb * mu * N / (ul * ul);
            if (xr < T(1)) ulb += ktb * (muS - muK) * N / ul * (T(-1) / (eps * h));
            utb += ut * (ulb / ul);
        }
        db += utb - nrm * dot(nrm, utb);
        kb += -gap * Nb;
        gapb = -k * Nb;
        // normal: f's n N, ut's -n (n.d), H's (k - kt) nnᵀ with (H̄ + H̄ᵀ) n = -e (δ.n) - δ (e.n)
        nb = Fb * N - utb * dot(nrm, d) - d * dot(utb, nrm) +
             (e * (-dot(delta, nrm)) - delta * dot(e, nrm)) * (k - kt);
    }
    // Trilinear sample with the field's Hessian in lattice-fraction coordinates (zero diagonal):
    // hxy, hxz, hyz of d²φ/df_a df_b, contact.cuh:57-76.
    static bool sdf_sample_hess(const typename Sim<T>::Grid& g, const V3<T>& p, T& phi, V3<T>& grad, T& hxy, T& hxz,
                                T& hyz) {
        if (!Sim<T>::sdf_sample(g, p, phi, grad)) return false;
        const V3<T> u = (p - g.origin) * g.inv;
        const int i = (int)u.x, j = (int)u.y, k = (int)u.z;
        const V3<T> fr = (p - (g.origin + V3<T>(T(i), T(j), T(k)) * g.sp)) * g.inv;
        const T fy = std::min(std::max(fr.y, T(0)), T(1)), fz = std::min(std::max(fr.z, T(0)), T(1));
        const T fx = std::min(std::max(fr.x, T(0)), T(1));
        const size_t sy = (size_t)g.nz, sx = (size_t)g.ny * g.nz;
        const float* c = g.v.data() + (size_t)i * sx + (size_t)j * sy + k;
        const T c000 = c[0], c001 = c[1], c010 = c[sy], c011 = c[sy + 1];
        const T c100 = c[sx], c101 = c[sx + 1], c110 = c[sx + sy], c111 = c[sx + sy + 1];
        const T dx00 = c100 - c000, dx01 = c101 - c001, dx10 = c110 - c010, dx11 = c111 - c011;
        const T D = (dx11 - dx01) - (dx10 - dx00);
        hxy = (dx10 - dx00) + fz * D;
        hxz = (dx01 - dx00) + fy * D;
        const T dy0 = (c010 - c000) + fx * (dx10 - dx00), dy1 = (c011 - c001) + fx * (dx11 - dx01);
        hyz = dy1 - dy0;
        return true;
    }
    // Mesh contact of vertex i reversed (contact.cuh:94-110 then the contact law): adds to d̄, x̄
    // and returns the stiffness adjoint. p_o = R(q)ᵀ((x - P) + d); n = R(q) ∇φ/|∇φ|; gap = φ - r;
    // dRel = d - h (v_P + ω × (x - P)) for a moving mesh.
    T mesh_contact_bwd(int i, const V3<T>& x, const V3<T>& d, T kc, const V3<T>& Fb, const V3<T>& e, const V3<T>& delta,
                       V3<T>& db, V3<T>& xb) const {
        T kbs = 0;
        const int cnt = s.cand_count(i);
        for (int c = 0; c < cnt; c++) {
            const int m = s.cand_at(i, c);
            const auto& P = s.poses[(size_t)s.env[i] * kMaxSdf + m];
            const auto& G = s.grids[m];
            const V3<T> po = qrot(P.q.inv(), (x - P.pos) + d);
            T phi, hxy, hxz, hyz;
            V3<T> gr;
            if (!sdf_sample_hess(G, po, phi, gr, hxy, hxz, hyz)) continue;
            const T gap = phi - s.cR;
            if (gap >= 0) continue;
            const T gl = len(gr);
            if (!(gl > 0)) continue;
            const V3<T> gh = gr / gl;
            const V3<T> nrm = qrot(P.q, gh);
            V3<T> dRel = d;
            if (s.sdfMoving) dRel -= (P.vel + cross(P.omega, x - P.pos)) * s.h;
            V3<T> dRelb, nb;
            T gapb, kb = 0;
            surface_contact_bwd(nrm, gap, dRel, kc, G.muS, G.muK, Fb, e, delta, dRelb, gapb, kb, nb);
            kbs += kb;
            db += dRelb;
            if (s.sdfMoving) xb += cross(P.omega, dRelb) * s.h;
            // n = R(q) ĝ: the object-frame gradient's adjoint
            const V3<T> ghb = qrot(P.q.inv(), nb);
            const V3<T> grb = (ghb - gh * dot(gh, ghb)) / gl;
            // φ and ∇φ (= G inv) at p_o: d φ/dp_o = ∇φ, d ∇φ/dp_o = inv² Hf
            const T inv2 = G.inv * G.inv;
            const V3<T> pob = gr * gapb + V3<T>(hxy * grb.y + hxz * grb.z, hxy * grb.x + hyz * grb.z,
                                                 hxz * grb.x + hyz * grb.y) * inv2;
            const V3<T> wb = qrot(P.q, pob);
            xb += wb;
            db += wb;
        }
        return kbs;
    }

    void substep_backward(int sub, int S, float dtf, const T* prog, bool q0set, const float* q0, const float* q1,
                          FrameGrad<T>& g) {
        const int n = s.n, I = s.numItr;
        // -- recompute the substep, keeping the iterates
        if (prog) s.apply_root_program(prog, q0, q1, sub, S, dtf);
        s.stage_poses(sub, S);
        const std::vector<V3<T>> x = s.pos, vin = s.vel, lvin = s.lastVel;
        s.init_itr();
        if (s.ropeContact) s.brute_detect();
        if (s.useStepLimit) s.step_limit();
        const std::vector<V3<T>> y = s.vel;  // the inertial target of free vertices
        std::vector<std::vector<V3<T>>> d(I + 1), z(I + 1);
        std::vector<std::vector<Q4<T>>> qk(I + 1);
        d[0] = s.dx;
        qk[0] = s.q;
        for (int it = 0; it < I; it++) {
            s.position_sweep();
            z[it + 1] = s.dxRaw;
            s.frame_sweep();
            d[it + 1] = s.dx;
            qk[it + 1] = s.q;
        }
        msb.assign(n, T(0));
        const T h = s.h, damp = s.damping / h, accel = s.accel;
        std::vector<V3<T>> db(n), xb(n), yb(n), vb(n), lvb(n);
        std::vector<Q4<T>> qb(n);
        // -- end: x' = x + d, v' = drag(d / h) for free vertices, lv' = v_in
        for (int i = 0; i < n; i++) {
            xb[i] = g.x[i];
            db[i] = g.x[i];
            qb[i] = g.q[i];
            vb[i] = g.lv[i];
            lvb[i] = V3<T>();
        }
        for (int i = 0; i < n; i++) {
            if (s.invMass[i] != 0) {
                const V3<T> ob = g.v[i] * (T(1) - s.drag * h);
                V3<T> vbar = ob;
                if (s.dragQuad > 0) {
                    const int ti = has(i, F_NEXT) ? i : i - 1;
                    const Q4<T>& tq = qk[I][ti];
                    const V3<T> t = qtangent(tq);
                    const V3<T> v = d[I][i] / h;
                    const T tv = dot(t, v);
                    const V3<T> vt = t * tv, vn = v - vt;
                    const T ln = len(vn), Dn = T(1) + s.dragQuad * ln * h;
                    const T lt = len(vt), Dt = T(1) + s.dragQuadT * lt * h;
                    V3<T> vnb = ob / Dn;
                    if (ln > 0) vnb -= vn * (s.dragQuad * h * dot(vn, ob) / (ln * Dn * Dn));
                    V3<T> vtb = ob / Dt;
                    if (lt > 0) vtb -= vt * (s.dragQuadT * h * dot(vt, ob) / (lt * Dt * Dt));
                    vbar = vnb;
                    vtb -= vnb;
                    const T tvb = dot(vtb, t);
                    vbar += t * tvb;
                    const V3<T> tb = vtb * tv + v * tvb;
                    qb[ti] += tangent_vjp(tq, tb);
                }
                db[i] += vbar / h;
            } else {
                vb[i] += g.v[i];  // a pinned vertex keeps its (driven) velocity
            }
        }
        // -- iterations in reverse
        for (int it = I - 1; it >= 0; it--) {
            frame_reverse(x, d[it + 1], qk[it], qb, db, xb, g);
            position_reverse(x, y, d[it], s.useStepLimit ? z[it + 1] : d[it + 1], qk[it], damp, accel, db, qb, xb, yb, g);
        }
        if (s.useStepLimit) step_limit_reverse(x, vin, xb, vb);
        // -- init: d^0 = v h + g h² s, y = v h + g h²
        const V3<T> grav = s.gravity;
        const T g2 = len2(grav);
        for (int i = 0; i < n; i++) {
            if (s.invMass[i] != 0) {
                vb[i] += (db[i] + yb[i]) * h;
                if (g2 > 0) {
                    const V3<T> acc = (vin[i] - lvin[i]) / s.lastH;
                    const T raw = dot(acc, grav) / g2;
                    if (raw >= 0 && raw <= 1) {  // inclusive at the clamp's ends (as torch.clamp)
                        const T sb = dot(grav * (h * h), db[i]);
                        const V3<T> gs = grav * (sb / (s.lastH * g2));
                        vb[i] += gs;
                        lvb[i] -= gs;
                    }
                }
            } else {
                vb[i] += db[i] * h;
            }
        }
        // -- root program: x = P0 + V0 tau + A tau²/2, v = V0 + A (tau + h/2),
        //    A = ((P1 - P0) - V0 dt) 2 / dt²; the program overwrites the root's incoming state
        if (prog) {
            const T dt = T(dtf), tau = T(sub) * h, th = tau + T(0.5) * h, idt2 = T(2) / (dt * dt);
            const T xa = T(0.5) * tau * tau * idt2;  // d x / d P1
            for (int r = 0; r < s.R; r++) {
                const int root = s.start[r];
                const V3<T> X = xb[root], Vv = vb[root];
                g.P0[r] += X * (T(1) - xa) + Vv * (-th * idt2);
                g.V0[r] += X * (tau - xa * dt) + Vv * (T(1) - th * idt2 * dt);
                g.P1[r] += X * xa + Vv * (th * idt2);
                xb[root] = V3<T>();
                vb[root] = V3<T>();
                if (q0set) qb[root] = Q4<T>(0, 0, 0, 0);
            }
        }
        g.x = xb; g.v = vb; g.lv = lvb; g.q = qb;
    }

    // Frame step k reversed: qb holds q̄^{k+1} on entry and q̄^k on return; db gains the
    // d^{k+1} contributions, xb the position ones.
    void frame_reverse(const std::vector<V3<T>>& x, const std::vector<V3<T>>& dn, const std::vector<Q4<T>>& qo,
                       std::vector<Q4<T>>& qb, std::vector<V3<T>>& db, std::vector<V3<T>>& xb, FrameGrad<T>& g) {
        const int n = s.n;
        const Q4<T> e1(1, 0, 0, 0);
        std::vector<Q4<T>> own(n), toL(n, Q4<T>(0, 0, 0, 0)), toR(n, Q4<T>(0, 0, 0, 0));
        std::vector<V3<T>> su(n);
        for (int i = 0; i < n; i++) {
            if (has(i, F_FIX_ORIENT) || !has(i, F_NEXT)) { own[i] = qb[i]; continue; }
            own[i] = Q4<T>(0, 0, 0, 0);
            const T l = s.lRest[i], ks = s.kStretch[i];
            const V3<T> u = ((x[i + 1] - x[i]) + (dn[i + 1] - dn[i])) / l;
            const V3<T> vv = u * (T(-2) * ks);
            const Q4<T> q0 = qo[i];
            Q4<T> b(0, 0, 0, 0);
            T sp = 0, sn = 0;
            if (has(i, F_PREV)) {
                const Q4<T> qr = s.qRest[i - 1], qq = qo[i - 1];
                sp = dot4(qmul(qq.inv(), q0), qr) > 0 ? T(1) : T(-1);
                b += qmul(qq, qr) * sp;
            }
            if (has(i, F_NEXT_ORIENT)) {
                const Q4<T> qr = s.qRest[i], qq = qo[i + 1];
                sn = dot4(qmul(q0.inv(), qq), qr) > 0 ? T(1) : T(-1);
                b += qmul(qq, qr.inv()) * sn;
            }
            const T lvv = len(vv), lb = len4(b), lambda = lvv + lb;
            const Q4<T> V(vv, T(0));
            const Q4<T> A = qmul(V, b);
            const Q4<T> z = qmul(A, e1) + b * lambda;
            const T zl = len4(z);
            const Q4<T> qn = z * (T(1) / zl);
            const Q4<T> qbn = qb[i];
            const Q4<T> zb = (qbn - qn * dot4(qn, qbn)) * (T(1) / zl);
            Q4<T> bb = zb * lambda;
            const T lamb = dot4(zb, b);
            V3<T> vvb = lvv > 0 ? vv * (lamb / lvv) : V3<T>();
            if (lb > 0) bb += b * (lamb / lb);
            const Q4<T> Ab = qmul(zb, qc(e1));
            vvb += qmul(Ab, qc(b)).vec();
            bb += qmul(qc(V), Ab);
            const V3<T> ub = vvb * (T(-2) * ks);
            g.ks[i] += T(-2) * dot(u, vvb);
            if (has(i, F_PREV)) {
                const Q4<T> bq = bb * sp, qr = s.qRest[i - 1];
                toL[i] = qmul(bq, qc(qr));
                g.rho[i - 1] += dot4(qmul(qc(qo[i - 1]), bq), qr) / len4(qr);
            }
            if (has(i, F_NEXT_ORIENT)) {
                const Q4<T> bq = bb * sn, qr = s.qRest[i];
                toR[i] = qmul(bq, qr);
                g.rho[i] += dot4(qc(qmul(qc(qo[i + 1]), bq)), qr) / len4(qr);
            }
            su[i] = ub / l;
        }
        for (int i = 0; i < n; i++) {
            Q4<T> a = own[i];
            if (i > 0) a += toR[i - 1];
            if (i + 1 < n) a += toL[i + 1];
            qb[i] = a;
            V3<T> dv = V3<T>() - su[i];
            if (i > 0) dv += su[i - 1];
            db[i] += dv;
            xb[i] += dv;
        }
    }

    // seg_closest (Common.h:327-345, with a0 = 0) reversed: given the adjoints of the returned
    // (u, v), adds those of a1 = A, b0 = B0, b1 = B1. Each clamp passes its adjoint inside [0, 1],
    // ends included; the fallback for parallel segments (a non-finite first v) is a constant.
    static void seg_closest_bwd(const V3<T>& A, const V3<T>& B0, const V3<T>& B1, T ub, T vb, V3<T>& Ab, V3<T>& B0b,
                                V3<T>& B1b) {
        const V3<T> E = B1 - B0;
        const T a = len2(A), b = dot(A, E), c = len2(E);
        const T AB0 = dot(A, B0), EB0 = dot(E, B0);
        const T Den = a * c - b * b, t0 = (b * AB0 - a * EB0) / Den;
        const bool fin = m_isfinite(t0);
        const T v0 = fin ? t0 : T(0.5);
        const bool p0 = fin && v0 >= 0 && v0 <= 1;
        const T v0c = std::min(std::max(v0, T(0)), T(1));
        const V3<T> Bv = lerp(B0, B1, v0c);
        const T tu = dot(Bv, A) / a;
        const bool pu = tu >= 0 && tu <= 1;
        const T u = std::min(std::max(tu, T(0)), T(1));
        const V3<T> Au = lerp(V3<T>(), A, u) - B0;
        const T tv = dot(Au, E) / c;
        V3<T> Ea, Aa, B0a;  // adjoints in the (A, B0, E = B1 - B0) parametrisation
        if (tv >= 0 && tv <= 1) {
            const T Nb = vb / c;
            ub += Nb * dot(A, E);
            Aa += E * (Nb * u);
            B0a -= E * Nb;
            Ea += Au * Nb + E * (T(-2) * vb * tv / c);
        }
        if (pu) {
            const T Mb = ub / a;
            const V3<T> Bvb = A * Mb;
            B0a += Bvb;
            Ea += Bvb * v0c;
            Aa += Bv * Mb + A * (T(-2) * ub * tu / a);
            if (p0) {
                const T t0b = dot(Bvb, E);
                const T Numb = t0b / Den, Denb = -t0b * t0 / Den;
                const T bb = Numb * AB0 - T(2) * b * Denb, aa = -Numb * EB0 + Denb * c, cc = Denb * a;
                const T AB0b = Numb * b, EB0b = -Numb * a;
                Aa += E * bb + A * (T(2) * aa) + B0 * AB0b;
                Ea += A * bb + E * (T(2) * cc) + B0 * EB0b;
                B0a += A * AB0b + E * EB0b;
            }
        }
        Ab += Aa;
        B1b += Ea;
        B0b += B0a - Ea;
    }
    // Collision Hessians of every segment's candidates at iterate d^k: Ha to vertex i, Hb to i+1.
    void collision_hessians(const std::vector<V3<T>>& dk, T damp, std::vector<S3<T>>& Ha, std::vector<S3<T>>& Hb) const {
        const int n = s.n;
        Ha.assign(n, S3<T>());
        Hb.assign(n, S3<T>());
        const std::vector<V3<T>> keep = s.dx;
        s.dx = dk;
        const T invb = T(1) / s.barrier, rad2 = T(2) * s.radius, kCol = s.kCollision * invb;
        for (int i = 0; i < n; i++) {
            if (!has(i, F_NEXT)) continue;
            V3<T> f, f2;
            for (int c = 0; c < s.numCols[i]; c++)
                s.collision_term(i, s.cols[i][c], s.lastPos[i + 1], dk[i + 1], dk[i], invb, rad2, kCol, damp, f, f2, Ha[i], Hb[i]);
        }
        s.dx = keep;
    }
    // One rope-rope candidate reversed (cosserat.cu:99-157). Segment i's term with candidate o adds
    // f, H to vertex i with weight wa = 1 - u and f2, H2 to vertex i+1 with weight wb = u; given F̄
    // and H̄ = -e δᵀ of both vertices (Fa, ea, la for i; Fc, ec, lc for i+1), adds d̄ and x̄ of the
    // four vertices i, i+1, o, o+1. Barrier: s = (|n| - 2r)/b clamped below at 1e-3, ff and dH of
    // the log barrier; friction f1 = min(kf, μ ff / |uu|) along the tangential slip uu.
    void collision_bwd(int i, int o, const std::vector<V3<T>>& x, const std::vector<V3<T>>& dk, T damp, const V3<T>& Fa,
                       const V3<T>& ea, const V3<T>& la, const V3<T>& Fc, const V3<T>& ec, const V3<T>& lc,
                       std::vector<V3<T>>& db, std::vector<V3<T>>& xb) const {
        const T invb = T(1) / s.barrier, rad2 = T(2) * s.radius, kCol = s.kCollision * invb;
        const V3<T> xi = x[i], x1 = x[i + 1], xo0 = x[o], xo1 = x[o + 1];
        const V3<T> di = dk[i], d1 = dk[i + 1], do0 = dk[o], do1 = dk[o + 1];
        const V3<T> A = (x1 - xi) + (d1 - di), B0 = (xo0 - xi) + (do0 - di), B1 = (xo1 - xi) + (do1 - di);
        T u, v;
        seg_closest(V3<T>(), A, B0, B1, u, v);
        const V3<T> dpos = lerp(xi, x1, u) - lerp(xo0, xo1, v);
        const V3<T> ddpos = lerp(di, d1, u) - lerp(do0, do1, v);
        const V3<T> raw = dpos + ddpos;
        const T dist = len(raw);
        if (!(dist > 0)) return;
        const V3<T> nr = raw * (T(1) / dist);
        const T wb = u, wa = T(1) - u;
        const T sr = (dist - rad2) * invb;
        if (sr > 1) return;
        const T sd = std::max(sr, T(1e-3));
        const T invd = T(1) / sd, logd = m_log(sd);
        const T dH = (T(-3) + (T(2) + invd) * invd - T(2) * logd) * kCol * invb;
        const T ff = -(T(1) - sd) * (sd - T(1) + T(2) * sd * logd) * invd * kCol;
        const T Ga = dot(Fa, nr), Gc = dot(Fc, nr), ndi = dot(nr, di), nd1 = dot(nr, d1);
        const T nHa = -dot(nr, ea) * dot(nr, la), nHc = -dot(nr, ec) * dot(nr, lc);
        const T trA = -dot(ea, la), trC = -dot(ec, lc);
        // (H̄ + H̄ᵀ) n for H̄ = -e δᵀ
        const V3<T> symA = ea * (-dot(la, nr)) - la * dot(ea, nr), symC = ec * (-dot(lc, nr)) - lc * dot(ec, nr);
        const V3<T> symS = symA * (wa * wa) + symC * (wb * wb);
        const T nHs = wa * wa * nHa + wb * wb * nHc, trS = wa * wa * trA + wb * wb * trC;
        T ffb = Ga * wa + Gc * wb;
        const T dHb = -damp * (Ga * wa * wa * ndi + Gc * wb * wb * nd1) + (T(1) + damp) * nHs;
        T wab = Ga * ff - T(2) * damp * dH * wa * Ga * ndi + T(2) * wa * (T(1) + damp) * dH * nHa;
        T wbb = Gc * ff - T(2) * damp * dH * wb * Gc * nd1 + T(2) * wb * (T(1) + damp) * dH * nHc;
        V3<T> nb = Fa * (ff * wa - damp * dH * wa * wa * ndi) + Fc * (ff * wb - damp * dH * wb * wb * nd1) +
                   di * (-damp * dH * wa * wa * Ga) + d1 * (-damp * dH * wb * wb * Gc) + symS * ((T(1) + damp) * dH);
        V3<T> dib = nr * (-damp * dH * wa * wa * Ga), d1b = nr * (-damp * dH * wb * wb * Gc);
        V3<T> ddb;  // adjoint of ddpos
        const V3<T> uu = ddpos - nr * dot(nr, ddpos);
        const T ul = len(uu);
        if (ul > 0) {
            const T ratio = s.fricMu * ff / ul;
            const T f1 = std::min(s.kFriction, ratio);
            const V3<T> Fu = Fa * wa + Fc * wb;
            const T f1b = -dot(uu, Fu) - (nHs - trS);
            wab += -f1 * dot(uu, Fa) - T(2) * wa * f1 * (nHa - trA);
            wbb += -f1 * dot(uu, Fc) - T(2) * wb * f1 * (nHc - trC);
            nb -= symS * f1;
            V3<T> uub = Fu * (-f1);
            if (!(s.kFriction < ratio)) {  // f1 = μ ff / |uu|
                ffb += f1b * s.fricMu / ul;
                uub += uu * (-f1b * ratio / (ul * ul));
            }
            ddb += uub - nr * dot(nr, uub);
            nb -= uub * dot(nr, ddpos) + ddpos * dot(nr, uub);
        }
        T ub = wbb - wab, distb = 0;
        if (sr >= T(1e-3)) {
            const T p = T(1) - sd, qv = sd - T(1) + T(2) * sd * logd;
            const T ffp = -kCol * ((-qv + p * (T(3) + T(2) * logd)) * invd - p * qv * invd * invd);
            const T dHp = T(-2) * (invd * invd + invd * invd * invd + invd) * kCol * invb;
            distb = (ffb * ffp + dHb * dHp) * invb;
        }
        const V3<T> rawb = (nb - nr * dot(nr, nb)) * (T(1) / dist) + nr * distb;
        ddb += rawb;
        xb[i] += rawb * wa;
        xb[i + 1] += rawb * wb;
        xb[o] -= rawb * (T(1) - v);
        xb[o + 1] -= rawb * v;
        ub += dot(rawb, x1 - xi) + dot(ddb, d1 - di);
        const T vb = -dot(rawb, xo1 - xo0) - dot(ddb, do1 - do0);
        dib += ddb * wa;
        d1b += ddb * wb;
        db[o] -= ddb * (T(1) - v);
        db[o + 1] -= ddb * v;
        V3<T> Ab, B0b, B1b;
        seg_closest_bwd(A, B0, B1, ub, vb, Ab, B0b, B1b);
        xb[i + 1] += Ab;
        d1b += Ab;
        xb[o] += B0b;
        db[o] += B0b;
        xb[o + 1] += B1b;
        db[o + 1] += B1b;
        const V3<T> sb = Ab + B0b + B1b;
        xb[i] -= sb;
        dib -= sb;
        db[i] += dib;
        db[i + 1] += d1b;
    }
    // Step limits reversed (recomputeStepLimitKernel, collision.cu:103-136): maxStep[i] is the
    // least of padding[i] - detRadius, padding = scaledDetRadius + |v h + g h²| (initItr), and
    // 0.45 times each candidate's closest distance at the substep start; its adjoint goes to the
    // argument that attained it (the first, on ties, as the forward's running minimum).
    void step_limit_reverse(const std::vector<V3<T>>& x, const std::vector<V3<T>>& vin, std::vector<V3<T>>& xb,
                            std::vector<V3<T>>& vb) const {
        const T h = s.h, fac = T((1 - 0.1f) * 0.5f);
        for (int i = 0; i < s.n; i++) {
            if (msb[i] == 0 || !has(i, F_NEXT)) continue;
            const V3<T> a0 = x[i], a1 = x[i + 1] - a0;
            T best = s.padding[i] - s.detRadius;
            int arg = -1;
            for (int c = 0; c < s.numCols[i]; c++) {
                const int o = s.cols[i][c];
                const V3<T> b0 = x[o] - a0, b1 = x[o + 1] - a0;
                T u, v;
                seg_closest(V3<T>(), a1, b0, b1, u, v);
                const T val = fac * len(a1 * u - lerp(b0, b1, v));
                if (val < best) { best = val; arg = c; }
            }
            if (arg < 0) {
                const V3<T> y = vin[i] * h + s.gravity * (h * h);
                const T ly = len(y);
                if (ly > 0) vb[i] += y * (msb[i] * h / ly);
                continue;
            }
            const int o = s.cols[i][arg];
            const V3<T> b0 = x[o] - a0, b1 = x[o + 1] - a0;
            T u, v;
            seg_closest(V3<T>(), a1, b0, b1, u, v);
            const V3<T> nn = a1 * u - lerp(b0, b1, v);
            const T l = len(nn);
            if (!(l > 0)) continue;
            const V3<T> nnb = nn * (fac * msb[i] / l);
            V3<T> Ab = nnb * u, B0b = nnb * (-(T(1) - v)), B1b = nnb * (-v);
            seg_closest_bwd(a1, b0, b1, dot(nnb, a1), -dot(nnb, b1 - b0), Ab, B0b, B1b);
            xb[i + 1] += Ab;
            xb[o] += B0b;
            xb[o + 1] += B1b;
            xb[i] -= Ab + B0b + B1b;
        }
    }
    // Position step k reversed: db holds d̄^{k+1} on entry and d̄^k on return.
    void position_reverse(const std::vector<V3<T>>& x, const std::vector<V3<T>>& y, const std::vector<V3<T>>& dk,
                          const std::vector<V3<T>>& dn, const std::vector<Q4<T>>& qo, T damp, T accel,
                          std::vector<V3<T>>& db, std::vector<Q4<T>>& qb, std::vector<V3<T>>& xb, std::vector<V3<T>>& yb,
                          FrameGrad<T>& g) {
        const int n = s.n;
        const T h = s.h;
        std::vector<V3<T>> Fb(n), dnew(n), sc(n);
        std::vector<T> trH(n, T(0));
        std::vector<V3<T>> ev(n), lv(n);  // e = H⁻¹ z̄ and δ = z - d^k per vertex (H̄ = -e δᵀ)
        std::vector<S3<T>> HcA, HcB;
        if (s.ropeContact) collision_hessians(dk, damp, HcA, HcB);
        for (int i = 0; i < n; i++) {
            dnew[i] = db[i];
            const T w = s.invMass[i];
            if (w == 0) continue;
            const T a = T(1) / (w * h * h);
            S3<T> H(a);
            const bool surf = s.numPlanes > 0 || !s.grids.empty();
            const T kap = s.cKappa / h, kc = kap * kap / w;
            if (surf) {
                V3<T> fdummy;
                s.surfaces_at(i, x[i], dk[i], kc, fdummy, H);
            }
            if (has(i, F_NEXT)) H.add_diag(s.kStretch[i] / s.lRest[i] / s.lRest[i] * (T(1) + damp));
            if (has(i, F_PREV)) H.add_diag(s.kStretch[i - 1] / s.lRest[i - 1] / s.lRest[i - 1] * (T(1) + damp));
            if (s.ropeContact) {
                H += HcA[i];
                if (has(i, F_PREV)) H += HcB[i - 1];
            }
            // step limit d' = z lim / |z| when |z| > lim (cosserat.cu:204-208): z̄ = (lim/|z|)(I - ẑẑᵀ) d̄',
            // and the limit's adjoint ẑ.d̄' goes to the maxStep entry that set it
            V3<T> gb = db[i];
            if (s.useStepLimit) {
                T lim = s.maxStep[i];
                int arg = i;
                if (has(i, F_PREV) && s.maxStep[i - 1] < lim) { lim = s.maxStep[i - 1]; arg = i - 1; }
                const T l = len(dn[i]);
                if (l > lim && l > 0) {
                    const V3<T> zh = dn[i] * (T(1) / l);
                    const T zg = dot(zh, gb);
                    msb[arg] += zg;
                    gb = (gb - zh * zg) * (lim / l);
                }
            }
            dnew[i] = gb;
            const V3<T> e = sym_solve(H, gb);
            const V3<T> delta = dn[i] - dk[i];
            ev[i] = e;
            lv[i] = delta;
            Fb[i] = e * accel;
            trH[i] = -dot(e, delta);
            yb[i] += Fb[i] * a;
            dnew[i] -= Fb[i] * a;
            T wb = (dot(y[i] - dk[i], Fb[i]) + trH[i]) * (-a / w);
            if (surf) {
                for (int pl = 0; pl < s.numPlanes; pl++) {
                    const V3<T> nrm(s.planes[pl][0], s.planes[pl][1], s.planes[pl][2]);
                    const T gap = (dot(nrm, x[i]) - s.planes[pl][3]) + dot(nrm, dk[i]) - s.cR;
                    if (gap >= 0) continue;
                    T gapb, kb;
                    V3<T> nb;
                    surface_contact_bwd(nrm, gap, dk[i], kc, s.cMuS, s.cMuK, Fb[i], e, delta, dnew[i], gapb, kb, nb);
                    dnew[i] += nrm * gapb;
                    xb[i] += nrm * gapb;
                    wb += kb * (-kc / w);
                }
                if (!s.grids.empty()) wb += mesh_contact_bwd(i, x[i], dk[i], kc, Fb[i], e, delta, dnew[i], xb[i]) * (-kc / w);
            }
            g.w[i] += wb;
        }
        if (s.ropeContact) {
            for (int j = 0; j < n; j++) {
                if (!has(j, F_NEXT)) continue;
                for (int c = 0; c < s.numCols[j]; c++)
                    collision_bwd(j, s.cols[j][c], x, dk, damp, Fb[j], ev[j], lv[j], Fb[j + 1], ev[j + 1], lv[j + 1], dnew, xb);
            }
        }
        for (int j = 0; j < n; j++) {
            if (!has(j, F_NEXT)) continue;
            const T l = s.lRest[j], invl = T(1) / l;
            const V3<T> c = ((x[j + 1] - x[j]) + (dk[j + 1] - dk[j])) * invl - qtangent(qo[j]);
            const T kk = s.kStretch[j] * invl, dd = kk * invl;
            const V3<T> dF = Fb[j] - Fb[j + 1];
            const V3<T> cb = dF * kk;
            const T kb = dot(c, dF);
            const T ddb = -damp * (dot(dk[j], Fb[j]) + dot(dk[j + 1], Fb[j + 1])) + (T(1) + damp) * (trH[j] + trH[j + 1]);
            g.ks[j] += kb * invl + ddb * invl * invl;
            qb[j] += tangent_vjp(qo[j], cb) * T(-1);
            sc[j] = cb * invl;
            dnew[j] -= Fb[j] * (damp * dd);
            dnew[j + 1] -= Fb[j + 1] * (damp * dd);
        }
        for (int i = 0; i < n; i++) {
            V3<T> dv = V3<T>() - sc[i];
            if (i > 0) dv += sc[i - 1];
            dnew[i] += dv;
            xb[i] += dv;
        }
        db = dnew;
    }
};

}  // namespace rso
