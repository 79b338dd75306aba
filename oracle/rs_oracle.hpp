// rs_oracle.hpp -- TEST INFRASTRUCTURE ONLY. CPU restatement of the Stable Cosserat Rods
// substep that ropesim's RopeSim / RopeBatch run (DeformX/Cosserat-Rod-Solver-CUDA, which
// vendors YarnBall). It is the checker for the CUDA product path and is never linked into it:
// only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs use it.
//
// Ordering: the reference's `deterministic=True` (SNAPSHOT) sweeps, i.e. per iteration
//   dx_{k+1} = PositionStep(dx_k, q_k)       (Jacobi over the previous iterate)
//   q_{k+1}  = FrameStep(dx_{k+1}, q_k)      (Jacobi over a frame snapshot)
// which is well defined and independent of any CTA partition.
//
// Parity pin: the reference cannot be built here (GLM is absent), so this restatement is
// pinned by the reference's own known-answer tests (hanging elongation, cantilever droop,
// pendulum period, Coulomb incline, rest support = weight, program endpoint, ...), ported
// to run against it on the CPU (tests/test_physics.py, tests/test_accept_*.py, the oracle
// backend of each parametrized test). Golden fixtures generated from it live in tests/golden/.
//
// Reference files followed (paths within the reference project):
//   third_party/yarnball/KittenEngine/YarnBall/YarnBall.cu:11-61,112-259,261-272   setup
//   third_party/yarnball/KittenEngine/YarnBall/sim/iteration.cu:10-129            initItr/endItr
//   third_party/yarnball/KittenEngine/YarnBall/sim/cosserat.cu:23-273              sweeps
//   third_party/yarnball/KittenEngine/YarnBall/sim/contact.cuh:27-204              surfaces
//   third_party/yarnball/KittenEngine/YarnBall/sim/collision.cu:103-136            step limit
//   third_party/yarnball/KittenEngine/YarnBall/sim/step.cpp:37-57                  advance
//   csrc/batch.cu:19-49,90-159,178-276,288-413                                     batch driver
//   csrc/sdf.cu:25-92,137-270                                                      mesh poses
//   third_party/yarnball/KittenEngine/KittenEngine/includes/modules/Rotor.h:57-188 rotor algebra
//   third_party/yarnball/KittenEngine/KittenEngine/includes/modules/Common.h:327-345 seg-seg
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

namespace rso {

// ---------------------------------------------------------------- math dispatch
// Unqualified calls after `using std::...` let the op-counting scalar (rs_opcount.hpp) stand in
// for float / double without touching the restatement.
template <class T> inline T m_sqrt(T x) { using std::sqrt; return sqrt(x); }
template <class T> inline T m_log(T x) { using std::log; return log(x); }
template <class T> inline T m_sin(T x) { using std::sin; return sin(x); }
template <class T> inline T m_cos(T x) { using std::cos; return cos(x); }
template <class T> inline T m_acos(T x) { using std::acos; return acos(x); }
template <class T> inline T m_atan2(T y, T x) { using std::atan2; return atan2(y, x); }
template <class T> inline bool m_isfinite(T x) { using std::isfinite; return isfinite(x); }

// ---------------------------------------------------------------- small linear algebra
template <class T> struct V3 {
    T x, y, z;
    V3() : x(0), y(0), z(0) {}
    V3(T a, T b, T c) : x(a), y(b), z(c) {}
    explicit V3(T a) : x(a), y(a), z(a) {}
    V3 operator+(const V3& o) const { return V3(x + o.x, y + o.y, z + o.z); }
    V3 operator-(const V3& o) const { return V3(x - o.x, y - o.y, z - o.z); }
    V3 operator-() const { return V3(-x, -y, -z); }
    V3 operator*(T s) const { return V3(x * s, y * s, z * s); }
    V3 operator/(T s) const { return V3(x / s, y / s, z / s); }
    V3& operator+=(const V3& o) { x += o.x; y += o.y; z += o.z; return *this; }
    V3& operator-=(const V3& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
    V3& operator*=(T s) { x *= s; y *= s; z *= s; return *this; }
    V3& operator/=(T s) { x /= s; y /= s; z /= s; return *this; }
    bool operator==(const V3& o) const { return x == o.x && y == o.y && z == o.z; }
};
template <class T> inline V3<T> operator*(T s, const V3<T>& v) { return V3<T>(s * v.x, s * v.y, s * v.z); }
template <class T> inline T dot(const V3<T>& a, const V3<T>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> inline V3<T> cross(const V3<T>& a, const V3<T>& b) {
    return V3<T>(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <class T> inline T len2(const V3<T>& a) { return dot(a, a); }
template <class T> inline T len(const V3<T>& a) { return m_sqrt(dot(a, a)); }
template <class T> inline V3<T> vmin(const V3<T>& a, const V3<T>& b) {
    return V3<T>(std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z));
}
template <class T> inline V3<T> vmax(const V3<T>& a, const V3<T>& b) {
    return V3<T>(std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z));
}
template <class T> inline V3<T> lerp(const V3<T>& a, const V3<T>& b, T t) { return a * (T(1) - t) + b * t; }

// Quaternion in rotor layout (x, y, z = bivector part, w = scalar), Rotor.h:11-20.
template <class T> struct Q4 {
    T x, y, z, w;
    Q4() : x(0), y(0), z(0), w(1) {}
    Q4(T a, T b, T c, T d) : x(a), y(b), z(c), w(d) {}
    Q4(const V3<T>& v, T s) : x(v.x), y(v.y), z(v.z), w(s) {}
    V3<T> vec() const { return V3<T>(x, y, z); }
    Q4 operator+(const Q4& o) const { return Q4(x + o.x, y + o.y, z + o.z, w + o.w); }
    Q4 operator-(const Q4& o) const { return Q4(x - o.x, y - o.y, z - o.z, w - o.w); }
    Q4 operator*(T s) const { return Q4(x * s, y * s, z * s, w * s); }
    Q4& operator+=(const Q4& o) { x += o.x; y += o.y; z += o.z; w += o.w; return *this; }
    Q4 inv() const { return Q4(-x, -y, -z, w); }  // Rotor.h:87-89 (unit rotors)
};
template <class T> inline Q4<T> operator*(T s, const Q4<T>& q) { return q * s; }
template <class T> inline T dot4(const Q4<T>& a, const Q4<T>& b) { return (a.x * b.x + a.y * b.y) + (a.z * b.z + a.w * b.w); }
template <class T> inline T len4(const Q4<T>& a) { return m_sqrt(dot4(a, a)); }
template <class T> inline Q4<T> normalize4(const Q4<T>& a) { return a * (T(1) / m_sqrt(dot4(a, a))); }
// Rotor product, Rotor.h:185-188.
template <class T> inline Q4<T> qmul(const Q4<T>& a, const Q4<T>& b) {
    const V3<T> av = a.vec(), bv = b.vec();
    return Q4<T>(bv * a.w + av * b.w + cross(av, bv), a.w * b.w - dot(av, bv));
}
// Rotation of a vector, Rotor.h:96-105.
template <class T> inline V3<T> qrot(const Q4<T>& q, const V3<T>& v) {
    const V3<T> qv = q.vec();
    const V3<T> a = v * q.w + cross(qv, v);
    const T c = dot(v, qv);
    return a * q.w + cross(qv, a) + qv * c;
}
// q * (1, 0, 0): the segment tangent of a frame.
template <class T> inline V3<T> qtangent(const Q4<T>& q) { return qrot(q, V3<T>(T(1), T(0), T(0))); }
// Rotor::fromTo, Rotor.h:57-64 (only reached for non-antiparallel targets here).
template <class T> inline Q4<T> q_from_to(const V3<T>& from, const V3<T>& to) {
    V3<T> h = (from + to) * T(0.5);
    const T l = len2(h);
    if (l > 0) h *= T(1) / m_sqrt(l);
    else h = V3<T>(T(0), T(1), T(0));
    return Q4<T>(cross(from, h), dot(from, h));
}
// Rotor::angleAxis, Rotor.h:23-26.
template <class T> inline Q4<T> q_angle_axis(T rad, const V3<T>& axis) {
    rad *= T(0.5);
    return Q4<T>(axis * m_sin(rad), m_cos(rad));
}

// Symmetric 3x3 stored as diag (xx, yy, zz) and upper (xy, xz, yz), SymMat.h:8-113 layout.
template <class T> struct S3 {
    T a[6];
    S3() { for (int i = 0; i < 6; i++) a[i] = 0; }
    explicit S3(T d) { a[0] = a[1] = a[2] = d; a[3] = a[4] = a[5] = 0; }
    S3 operator+(const S3& o) const { S3 r; for (int i = 0; i < 6; i++) r.a[i] = a[i] + o.a[i]; return r; }
    S3 operator*(T s) const { S3 r; for (int i = 0; i < 6; i++) r.a[i] = a[i] * s; return r; }
    S3& operator+=(const S3& o) { for (int i = 0; i < 6; i++) a[i] += o.a[i]; return *this; }
    S3& operator-=(const S3& o) { for (int i = 0; i < 6; i++) a[i] -= o.a[i]; return *this; }
    void add_diag(T d) { a[0] += d; a[1] += d; a[2] += d; }
    static S3 outer(const V3<T>& v) {
        S3 m;
        m.a[0] = v.x * v.x; m.a[1] = v.y * v.y; m.a[2] = v.z * v.z;
        m.a[3] = v.x * v.y; m.a[4] = v.x * v.z; m.a[5] = v.y * v.z;
        return m;
    }
};
// x = H^-1 f by the adjugate of the symmetric matrix (written from the cofactor expansion).
template <class T> inline V3<T> sym_solve(const S3<T>& H, const V3<T>& f) {
    const T xx = H.a[0], yy = H.a[1], zz = H.a[2], xy = H.a[3], xz = H.a[4], yz = H.a[5];
    const T c00 = yy * zz - yz * yz, c01 = xz * yz - xy * zz, c02 = xy * yz - xz * yy;
    const T c11 = xx * zz - xz * xz, c12 = xy * xz - xx * yz, c22 = xx * yy - xy * xy;
    const T idet = T(1) / (xx * c00 + xy * c01 + xz * c02);
    return V3<T>((c00 * f.x + c01 * f.y + c02 * f.z) * idet,
                 (c01 * f.x + c11 * f.y + c12 * f.z) * idet,
                 (c02 * f.x + c12 * f.y + c22 * f.z) * idet);
}

// Closest points between segments a0a1 and b0b1 as (u, v) parameters, Common.h:327-345.
template <class T> inline void seg_closest(const V3<T>& a0, const V3<T>& a1, const V3<T>& b0, const V3<T>& b1, T& u, T& v) {
    const V3<T> A0 = a1 - a0, A1 = b1 - b0;
    const T a = len2(A0), b = dot(A0, A1), c = len2(A1);
    const V3<T> diff = b0 - a0;
    v = (b * dot(A0, diff) - a * dot(A1, diff)) / (a * c - b * b);
    if (!m_isfinite(v)) v = T(0.5);
    v = std::min(std::max(v, T(0)), T(1));
    u = std::min(std::max(dot(lerp(b0, b1, v) - a0, A0) / a, T(0)), T(1));
    v = std::min(std::max(dot(lerp(a0, a1, u) - b0, A1) / c, T(0)), T(1));
}

// ---------------------------------------------------------------- flags (YarnBall.h:52-58)
enum : uint32_t { F_PREV = 1, F_NEXT = 2, F_NEXT_ORIENT = 4, F_FIX_ORIENT = 8 };
enum { ERR_NONE = 0, ERR_MAX_COLLISIONS = 1, WARN_INTERPENETRATION = 2 };
constexpr int kMaxSdf = 64, kMaxCand = 8, kMaxCols = 128;

// ---------------------------------------------------------------- the simulated batch
template <class T> class Sim {
public:
    // ---- per-vertex state, flat order = rope order (rope r owns [start[r], start[r+1]))
    int n = 0, R = 0;
    std::vector<int> start;        // rope offsets, size R+1
    std::vector<int> env;          // per-vertex env index (meshes): rope index, or 0 for RopeSim
    std::vector<int> ropeOf;       // per-vertex rope index
    int numEnvs = 1;
    std::vector<V3<T>> pos, vel, lastVel, dx, dxNext, lastPos;
    std::vector<V3<T>> dxRaw;      // each iterate before the step limit (read by the adjoint)
    mutable long long nCollisionTerms = 0, nLimitedSteps = 0;  // forward counters (tests assert coverage)
    std::vector<Q4<T>> q, qPrev, qRest;
    std::vector<T> invMass, lRest, kStretch, padding, maxStep;
    std::vector<uint32_t> flags;
    std::vector<T> initInvMass;
    std::vector<V3<T>> initPos;
    std::vector<Q4<T>> initQ;

    // ---- solver knobs (YarnBall.cu:11-61 defaults)
    V3<T> gravity = V3<T>(T(0), T(-9.8), T(0));
    T h = T(1e-3), lastH = T(1e-3), time = 0;
    float maxH = 1e-3f;          // kept in float: the substep count is a float ceil (step.cpp:40)
    int numItr = 8;
    T damping = T(1e-6), drag = T(0.2), dragQuad = 0, dragQuadT = 0, accel = 1;
    // plane/mesh contact material (YarnBall.h:128-134)
    int numPlanes = 0;
    T planes[8][4] = {};
    T cR = 0, cKappa = 2, cMuS = 0, cMuK = 0, cVSlip = T(1e-3);
    // rope-rope contact (YarnBall.h:175-192)
    T radius = T(1e-4), barrier = T(8e-4), kCollision = T(1e-5), fricMu = T(0.1), kFriction = 5, detScaler = T(1.2);
    T detRadius = 0, scaledDetRadius = 0, minSegLen = 0, maxSegLen = 0;
    bool ropeContact = false, useStepLimit = false;
    bool inplaceFrames = false;  // frame sweep in place (frame_sweep)
    int groupRopes = 1;
    std::vector<int> numCols;             // per segment
    std::vector<std::vector<int>> cols;   // per segment candidate list (ascending j)
    int lastError = 0, lastWarning = 0, pendingError = 0, pendingWarning = 0;

    // ---- meshes (sdf.h / sdf.cu)
    struct Grid { std::vector<float> v; int nx, ny, nz; V3<T> origin; T sp, inv; T muS, muK; V3<T> boxLo, boxHi; };
    struct Pose { V3<T> pos; Q4<T> q; V3<T> vel, omega, lo, hi; };
    struct Pose7 { V3<T> pos; Q4<T> q; };
    struct Motion { V3<T> p0; Q4<T> q0; V3<T> dp, rot; };
    std::vector<Grid> grids;
    std::vector<Pose7> cur, tgt;          // [numEnvs * kMaxSdf]
    std::vector<uint8_t> tele;
    std::vector<Motion> motion;
    std::vector<Pose> poses;
    bool pendingSet = false, moving = false, sdfMoving = false, forcesOn = false;
    std::vector<int> numCand;             // per vertex; -1 = every mesh
    std::vector<std::vector<int>> cand;
    std::vector<V3<T>> contactForce;      // per vertex
    std::vector<V3<T>> wrench;            // [numEnvs * kMaxSdf * 2]

    // ------------------------------------------------------------------ construction
    // positions: float32 [n, 3] in rope order; pinned: [n] (nonzero = kinematic);
    // starts: [R + 1]; per_rope_env: env = rope index (RopeBatch) or 0 (RopeSim).
    Sim(const float* positions, const int* starts, int numRopes, const uint8_t* pinned, float density,
        float kStretchIn, float kBendIn, float max_h, int num_itr, bool fixRootOrientation, bool straightRest,
        bool perRopeEnv, float deadRadius, float deadBarrier) {
        R = numRopes;
        start.assign(starts, starts + R + 1);
        n = start[R];
        if (n < 3) throw std::invalid_argument("Too little vertices");
        resize_all();
        for (int r = 0; r < R; r++)
            for (int i = start[r]; i < start[r + 1]; i++) { ropeOf[i] = r; env[i] = perRopeEnv ? r : 0; }
        numEnvs = perRopeEnv ? R : 1;
        // Sim ctor defaults, YarnBall.cu:52-60
        for (int i = 0; i < n; i++) {
            pos[i] = V3<T>(T(positions[3 * i]), T(positions[3 * i + 1]), T(positions[3 * i + 2]));
            invMass[i] = 1; lRest[i] = 1; kStretch[i] = 100;
            qRest[i] = Q4<T>(0, 0, 0, 5);
            flags[i] = F_NEXT;
        }
        flags[n - 1] = 0;
        // RopeBatch ctor, batch.cu:344-361: rope ends, pins, clamped roots
        for (int r = 0; r < R; r++) {
            flags[start[r + 1] - 1] = 0;
            for (int i = start[r]; i < start[r + 1]; i++)
                if (pinned[i]) invMass[i] = 0;
            if (fixRootOrientation) flags[start[r]] |= F_FIX_ORIENT;
        }
        radius = T(deadRadius);
        barrier = T(deadBarrier);
        configure(T(density));
        if (straightRest)
            for (int r = 0; r < R; r++)
                for (int i = start[r]; i + 1 < start[r + 1]; i++) qRest[i] = Q4<T>(0, 0, 0, 1);
        set_k_stretch(T(kStretchIn));
        set_k_bend(T(kBendIn));
        maxH = max_h;
        h = T(max_h);
        numItr = num_itr;
        initPos = pos;
        initQ = q;
        cur.assign((size_t)numEnvs * kMaxSdf, Pose7{V3<T>(), Q4<T>()});
        tgt = cur;
        tele.assign((size_t)numEnvs * kMaxSdf, 0);
        motion.assign((size_t)numEnvs * kMaxSdf, Motion{});
        poses.assign((size_t)numEnvs * kMaxSdf, Pose{});
        wrench.assign((size_t)numEnvs * kMaxSdf * 2, V3<T>());
    }

    void resize_all() {
        ropeOf.assign(n, 0); env.assign(n, 0);
        pos.assign(n, V3<T>()); vel.assign(n, V3<T>()); lastVel.assign(n, V3<T>());
        dx.assign(n, V3<T>()); dxNext.assign(n, V3<T>()); dxRaw.assign(n, V3<T>()); lastPos.assign(n, V3<T>());
        q.assign(n, Q4<T>()); qPrev.assign(n, Q4<T>()); qRest.assign(n, Q4<T>());
        invMass.assign(n, T(1)); lRest.assign(n, T(1)); kStretch.assign(n, T(100));
        padding.assign(n, T(0)); maxStep.assign(n, std::numeric_limits<T>::infinity());
        flags.assign(n, 0u);
        numCols.assign(n, 0); cols.assign(n, std::vector<int>());
        numCand.assign(n, -1); cand.assign(n, std::vector<int>());
        contactForce.assign(n, V3<T>());
    }

    // Sim::configure, YarnBall.cu:112-182: lumped masses, min-twist frames, rest rotations.
    // The frame transport runs over the whole flat array, so a rope's initial frames start
    // from the previous rope's last frame (as in the reference).
    void configure(T density) {
        maxSegLen = 0;
        minSegLen = std::numeric_limits<T>::max();
        initInvMass.assign(n, T(0));
        Q4<T> lastQ;
        for (int i = 0; i < n; i++) {
            if (i < n - 1) {
                const bool hasNext = flags[i] & F_NEXT;
                flags[i + 1] = hasNext ? (flags[i + 1] | F_PREV) : (flags[i + 1] & ~F_PREV);
                const bool hasNextNext = hasNext && (flags[i + 1] & F_NEXT);
                flags[i] = hasNextNext ? (flags[i] | F_NEXT_ORIENT) : (flags[i] & ~F_NEXT_ORIENT);
                if (!hasNext) flags[i] |= F_FIX_ORIENT;
            }
            if (!(flags[i] & F_PREV) && !(flags[i] & F_NEXT))
                throw std::invalid_argument("Dangling segment. Yarns must be atleast 2 segments long");
            lRest[i] = T(1) / T(n);
            T mass = 0;
            if (flags[i] & F_PREV) mass += lRest[i - 1];
            if (flags[i] & F_NEXT) {
                const V3<T> seg0 = pos[i + 1] - pos[i];
                lRest[i] = len(seg0);
                if (lRest[i] == 0 || !m_isfinite(lRest[i])) throw std::invalid_argument("0 length segment");
                const V3<T> sd = seg0 * (T(1) / m_sqrt(len2(seg0)));
                const Q4<T> qq = (sd.x < T(-0.999999)) ? Q4<T>(0, 0, 1, 0) : q_from_to(V3<T>(1, 0, 0), sd);
                Q4<T> t = qmul(qq.inv(), lastQ);
                const Q4<T> tw(t.x, 0, 0, t.w);
                t = (dot4(tw, tw) > T(1e-12)) ? normalize4(tw) : Q4<T>(0, 0, 0, 1);
                lastQ = qmul(qq, t);
                mass += lRest[i];
                maxSegLen = std::max(maxSegLen, lRest[i]);
                minSegLen = std::min(minSegLen, lRest[i]);
            }
            q[i] = lastQ;
            mass *= T(0.5) * density;
            invMass[i] = (mass != 0) ? invMass[i] * (T(1) / mass) : T(0);
            initInvMass[i] = invMass[i];
        }
        for (int i = 0; i < n - 1; i++) qRest[i] = qmul(q[i].inv(), q[i + 1]) * len4(qRest[i]);
    }
    // Sim::setKStretch / setKBend, YarnBall.cu:237-259.
    void set_k_stretch(T k) { for (int i = 0; i < n; i++) kStretch[i] = k * lRest[i]; }
    void set_k_bend(T k) {
        k *= 4;
        for (int i = 0; i < n; i++) qRest[i] = normalize4(qRest[i]) * (k / lRest[i]);
    }
    // Per-vertex setters, bindings.cpp:1121-1201 (values are already validated by the caller).
    void set_vertex_ea(int i, T ea) { kStretch[i] = ea * lRest[i]; }
    void set_vertex_ei(int i, T ei) { qRest[i] = normalize4(qRest[i]) * (T(4) * ei / lRest[i]); }
    void set_vertex_mass(int i, T m) { if (invMass[i] != 0) invMass[i] = T(1) / m; }

    // ------------------------------------------------------------------ contact material
    void set_contact(T r, T muS, T muK, T vslip, T kappa) { cR = r; cMuS = muS; cMuK = muK; cVSlip = vslip; cKappa = kappa; }
    void set_planes(int P, const float* rows) {  // rows already normalized by the caller
        numPlanes = P;
        for (int p = 0; p < P; p++) for (int k = 0; k < 4; k++) planes[p][k] = T(rows[4 * p + k]);
    }
    void set_rope_contact(bool on, T r, T b, T kc, T mu, T kf, T scaler, int groups) {
        if (on) {
            radius = r; barrier = b; kCollision = kc; fricMu = mu; kFriction = kf; detScaler = scaler;
            groupRopes = groups > 0 ? groups : 1;
        } else {
            std::fill(numCols.begin(), numCols.end(), 0);
        }
        ropeContact = on;
        useStepLimit = on;
    }

    // ------------------------------------------------------------------ meshes (sdf.cu)
    int add_mesh(const float* values, int nx, int ny, int nz, const float* origin, float spacing, float muS, float muK,
                 const float* p, const float* qq, int rows) {
        if ((int)grids.size() >= kMaxSdf) throw std::invalid_argument("at most 64 meshes per sim");
        Grid g;
        g.v.assign(values, values + (size_t)nx * ny * nz);
        g.nx = nx; g.ny = ny; g.nz = nz;
        g.origin = V3<T>(T(origin[0]), T(origin[1]), T(origin[2]));
        g.sp = T(spacing); g.inv = T(1.f / spacing);
        g.muS = T(muS); g.muK = T(muK);
        g.boxLo = g.origin;
        g.boxHi = g.origin + V3<T>(T(nx - 1), T(ny - 1), T(nz - 1)) * g.sp;
        grids.push_back(g);
        const int idx = (int)grids.size() - 1;
        const bool pending = pendingSet;
        set_targets(idx, p, qq, rows, nullptr, true);
        for (int e = 0; e < numEnvs; e++) commit_slot((size_t)e * kMaxSdf + idx, idx);
        pendingSet = pending;
        return idx;
    }
    void set_mesh_friction(int idx, T muS, T muK) { grids.at(idx).muS = muS; grids.at(idx).muK = muK; }
    // scatterTargetsK, sdf.cu:37-51 (index < 0: a dense [numEnvs, M] block).
    void set_targets(int index, const float* p, const float* qq, int rows, const uint8_t* teleFlags, bool teleAll) {
        const int M = (int)grids.size();
        const int per = index < 0 ? M : 1;
        for (int i = 0; i < numEnvs * per; i++) {
            const int e = i / per, m = index < 0 ? i % per : index;
            const int r = index < 0 ? i : (rows == 1 ? 0 : e);
            Q4<T> qv(T(qq[4 * r]), T(qq[4 * r + 1]), T(qq[4 * r + 2]), T(qq[4 * r + 3]));
            const T l = len4(qv);
            qv = l > 0 ? qv * (T(1) / l) : Q4<T>(0, 0, 0, 1);
            const size_t slot = (size_t)e * kMaxSdf + m;
            tgt[slot].pos = V3<T>(T(p[3 * r]), T(p[3 * r + 1]), T(p[3 * r + 2]));
            tgt[slot].q = qv;
            tele[slot] = teleAll ? 1 : (teleFlags ? teleFlags[e] : 0);
        }
        pendingSet = true;
    }
    void clear_meshes() { grids.clear(); pendingSet = false; moving = false; }
    void enable_forces(bool on) { forcesOn = on; }

    // World AABB of the lattice box under a pose, contact.cuh:79-87.
    static void world_box(const V3<T>& lo_o, const V3<T>& hi_o, const V3<T>& p, const Q4<T>& qq, V3<T>& lo, V3<T>& hi) {
        const T inf = std::numeric_limits<T>::infinity();
        lo = V3<T>(inf); hi = V3<T>(-inf);
        for (int c = 0; c < 8; c++) {
            const V3<T> corner((c & 1) ? hi_o.x : lo_o.x, (c & 2) ? hi_o.y : lo_o.y, (c & 4) ? hi_o.z : lo_o.z);
            const V3<T> w = qrot(qq, corner) + p;
            lo = vmin(lo, w); hi = vmax(hi, w);
        }
    }
    void commit_slot(size_t i, int m) {  // sdf.cu:67-81
        cur[i] = tgt[i];
        tele[i] = 0;
        Pose P;
        P.pos = cur[i].pos; P.q = cur[i].q; P.vel = V3<T>(); P.omega = V3<T>();
        world_box(grids[m].boxLo, grids[m].boxHi, P.pos, P.q, P.lo, P.hi);
        poses[i] = P;
    }
    // Rotation vector taking q0 to q1 (world frame, shortest arc), sdf.cu:25-33.
    static V3<T> rotvec(const Q4<T>& q0, const Q4<T>& q1) {
        const V3<T> a(q1.x, q1.y, q1.z), b(-q0.x, -q0.y, -q0.z);
        V3<T> v = b * q1.w + a * q0.w + cross(a, b);
        T w = q1.w * q0.w - dot(a, b);
        if (w < 0) { v = -v; w = -w; }
        const T s = len(v);
        if (!(s > T(1e-9))) return V3<T>();
        return v * (T(2) * m_atan2(s, w) / s);
    }
    // SdfStore::begin_step, sdf.cu:217-232.
    void sdf_begin_step() {
        if (pendingSet) {
            for (size_t i = 0; i < cur.size(); i++) {
                if (tele[i]) { cur[i] = tgt[i]; tele[i] = 0; }
                motion[i].p0 = cur[i].pos;
                motion[i].q0 = cur[i].q;
                motion[i].dp = tgt[i].pos - cur[i].pos;
                motion[i].rot = rotvec(cur[i].q, tgt[i].q);
            }
            sdfMoving = true;
            moving = true;
        } else {
            sdfMoving = false;
        }
        if (!grids.empty()) std::fill(numCand.begin(), numCand.end(), -1);
        if (forcesOn) {
            std::fill(contactForce.begin(), contactForce.end(), V3<T>());
            std::fill(wrench.begin(), wrench.end(), V3<T>());
        }
    }
    // SdfStore::end_step, sdf.cu:239-253.
    void sdf_end_step(int substeps) {
        const int S = substeps > 0 ? substeps : 1;
        if (moving) {
            for (int e = 0; e < numEnvs; e++)
                for (int m = 0; m < (int)grids.size(); m++) commit_slot((size_t)e * kMaxSdf + m, m);
            moving = false;
            pendingSet = false;
        }
        if (forcesOn) {
            const T k = T(1.f / (float)S);
            for (auto& f : contactForce) f *= k;
            for (auto& w : wrench) w *= k;
        }
    }
    // Pose of substep `sub` of `nSub` (constant velocity over the frame), iteration.cu:12-33.
    void stage_poses(int sub, int nSub) {
        if (!sdfMoving) return;
        for (int e = 0; e < numEnvs; e++)
            for (int m = 0; m < (int)grids.size(); m++) {
                const size_t i = (size_t)e * kMaxSdf + m;
                const Motion& M = motion[i];
                const T a = T(sub + 1) / T(nSub);
                const T invDt = T(1) / (T(nSub) * h);
                Pose P;
                const T th = len(M.rot);
                if (th > 0 || !(M.dp == V3<T>())) {
                    P.pos = M.p0 + M.dp * a;
                    const Q4<T> dq = th > 0 ? q_angle_axis(a * th, M.rot / th) : Q4<T>();
                    P.q = normalize4(qmul(dq, M.q0));
                    P.vel = M.dp * invDt;
                    P.omega = M.rot * invDt;
                } else {
                    P.pos = M.p0; P.q = M.q0; P.vel = V3<T>(); P.omega = V3<T>();
                }
                world_box(grids[m].boxLo, grids[m].boxHi, P.pos, P.q, P.lo, P.hi);
                poses[i] = P;
            }
    }

    // ------------------------------------------------------------------ surface contact
    // One contact: penalty + regularised Coulomb friction, contact.cuh:27-46.
    void surface_contact(const V3<T>& nrm, T gap, const V3<T>& d, T k, T muS, T muK, V3<T>& f, S3<T>& H) const {
        const T eps = cVSlip;
        const T N = -k * gap;
        f += nrm * N;
        S3<T> nn = S3<T>::outer(nrm);
        H += nn * k;
        const V3<T> ut = d - nrm * dot(nrm, d);
        const T ul = len(ut);
        const T vt = ul / h;
        T kt;
        if (vt <= eps) kt = muS * N / (eps * h);
        else {
            const T s = T(1) - std::min(T(1), vt / eps - T(1));
            kt = (s * muS + (T(1) - s) * muK) * N / ul;
        }
        f -= ut * kt;
        nn.add_diag(T(-1));
        H -= nn * kt;
    }
    // Trilinear sample with the analytic gradient, contact.cuh:57-76.
    static bool sdf_sample(const Grid& g, const V3<T>& p, T& phi, V3<T>& grad) {
        const V3<T> u = (p - g.origin) * g.inv;
        if (!(u.x >= 0 && u.y >= 0 && u.z >= 0 && u.x < T(g.nx - 1) && u.y < T(g.ny - 1) && u.z < T(g.nz - 1))) return false;
        const int i = (int)u.x, j = (int)u.y, k = (int)u.z;
        const V3<T> fr = (p - (g.origin + V3<T>(T(i), T(j), T(k)) * g.sp)) * g.inv;
        const T fx = std::min(std::max(fr.x, T(0)), T(1)), fy = std::min(std::max(fr.y, T(0)), T(1)),
                fz = std::min(std::max(fr.z, T(0)), T(1));
        const size_t sy = (size_t)g.nz, sx = (size_t)g.ny * g.nz;
        const float* c = g.v.data() + (size_t)i * sx + (size_t)j * sy + k;
        const T c000 = c[0], c001 = c[1], c010 = c[sy], c011 = c[sy + 1];
        const T c100 = c[sx], c101 = c[sx + 1], c110 = c[sx + sy], c111 = c[sx + sy + 1];
        const T dx00 = c100 - c000, dx01 = c101 - c001, dx10 = c110 - c010, dx11 = c111 - c011;
        const T c00 = c000 + fx * dx00, c01 = c001 + fx * dx01, c10 = c010 + fx * dx10, c11 = c011 + fx * dx11;
        const T dy0 = c10 - c00, dy1 = c11 - c01;
        const T c0 = c00 + fy * dy0, c1 = c01 + fy * dy1;
        phi = c0 + fz * (c1 - c0);
        const T gx0 = dx00 + fy * (dx10 - dx00), gx1 = dx01 + fy * (dx11 - dx01);
        grad = V3<T>(gx0 + fz * (gx1 - gx0), dy0 + fz * (dy1 - dy0), c1 - c0) * g.inv;
        return true;
    }
    // contact.cuh:94-110.
    bool sdf_contact_at(const Pose& P, int m, const V3<T>& p, const V3<T>& d, V3<T>& nrm, T& gap, V3<T>& dRel) const {
        T phi;
        V3<T> g;
        if (!sdf_sample(grids[m], qrot(P.q.inv(), (p - P.pos) + d), phi, g)) return false;
        gap = phi - cR;
        if (gap >= 0) return false;
        const T gl = len(g);
        if (!(gl > 0)) return false;
        nrm = qrot(P.q, g / gl);
        dRel = d;
        if (sdfMoving) dRel -= (P.vel + cross(P.omega, p - P.pos)) * h;
        return true;
    }
    int cand_count(int i) const { return numCand[i] < 0 ? (int)grids.size() : numCand[i]; }
    int cand_at(int i, int c) const { return numCand[i] < 0 ? c : cand[i][c]; }
    // surfacesAt, contact.cuh:141-163.
    void surfaces_at(int i, const V3<T>& p, const V3<T>& d, T k, V3<T>& f, S3<T>& H) const {
        for (int pl = 0; pl < numPlanes; pl++) {
            const V3<T> nrm(planes[pl][0], planes[pl][1], planes[pl][2]);
            const T gap = (dot(nrm, p) - planes[pl][3]) + dot(nrm, d) - cR;
            if (gap >= 0) continue;
            surface_contact(nrm, gap, d, k, cMuS, cMuK, f, H);
        }
        if (!grids.empty()) {
            const int cnt = cand_count(i);
            for (int c = 0; c < cnt; c++) {
                const int m = cand_at(i, c);
                const Pose& P = poses[(size_t)env[i] * kMaxSdf + m];
                V3<T> nrm, dRel;
                T gap;
                if (!sdf_contact_at(P, m, p, d, nrm, gap, dRel)) continue;
                surface_contact(nrm, gap, dRel, k, grids[m].muS, grids[m].muK, f, H);
            }
        }
    }
    // surfaceReadout, contact.cuh:172-204 (sums are sequential here: deterministic).
    void surface_readout(int i, const V3<T>& p, const V3<T>& d, T k) {
        V3<T> fv;
        S3<T> Hs;
        for (int pl = 0; pl < numPlanes; pl++) {
            const V3<T> nrm(planes[pl][0], planes[pl][1], planes[pl][2]);
            const T gap = (dot(nrm, p) - planes[pl][3]) + dot(nrm, d) - cR;
            if (gap >= 0) continue;
            surface_contact(nrm, gap, d, k, cMuS, cMuK, fv, Hs);
        }
        if (!grids.empty()) {
            const int cnt = cand_count(i);
            for (int c = 0; c < cnt; c++) {
                const int m = cand_at(i, c);
                const size_t slot = (size_t)env[i] * kMaxSdf + m;
                const Pose& P = poses[slot];
                V3<T> nrm, dRel;
                T gap;
                if (!sdf_contact_at(P, m, p, d, nrm, gap, dRel)) continue;
                V3<T> fm;
                surface_contact(nrm, gap, dRel, k, grids[m].muS, grids[m].muK, fm, Hs);
                fv += fm;
                const V3<T> r = (p - P.pos) + d - nrm * cR;
                const V3<T> tq = cross(r, -fm);
                wrench[slot * 2] += -fm;
                wrench[slot * 2 + 1] += tq;
            }
        }
        contactForce[i] += fv;
    }
    // sdfBuildCandidates, contact.cuh:121-136.
    void build_candidates(int i, const V3<T>& p, T pad) {
        int cnt = 0;
        cand[i].clear();
        for (int m = 0; m < (int)grids.size(); m++) {
            const Pose& P = poses[(size_t)env[i] * kMaxSdf + m];
            const T pm = pad + (sdfMoving ? h * (len(P.vel) + len(P.omega) * T(0.5) * len(P.hi - P.lo)) : T(0));
            if (p.x >= P.lo.x - pm && p.x <= P.hi.x + pm && p.y >= P.lo.y - pm && p.y <= P.hi.y + pm &&
                p.z >= P.lo.z - pm && p.z <= P.hi.z + pm) {
                if (cnt < kMaxCand) cand[i].push_back(m);
                cnt++;
            }
        }
        numCand[i] = cnt <= kMaxCand ? cnt : -1;
    }

    // ------------------------------------------------------------------ rope-rope detection
    // Per-group brute force in ascending j, batch.cu:19-49. Groups = groupRopes consecutive ropes.
    void brute_detect() {
        for (int i = 0; i < n; i++) {
            cols[i].clear();
            numCols[i] = 0;
            if (!(flags[i] & F_NEXT)) continue;
            const int g = ropeOf[i] / groupRopes;
            const int r0 = g * groupRopes, r1 = std::min(R, r0 + groupRopes);
            const int g0 = start[r0], g1 = start[r1];
            const V3<T> a0 = lastPos[i], a1 = lastPos[i + 1] - a0;
            const T ri = std::max(padding[i], padding[i + 1]);
            int cnt = 0;
            for (int j = g0; j < g1; j++) {
                if (!(flags[j] & F_NEXT)) continue;
                if (ropeOf[j] == ropeOf[i] && std::abs(j - i) <= 2) continue;
                const V3<T> b0 = lastPos[j] - a0, b1 = lastPos[j + 1] - a0;
                T u, v;
                seg_closest(V3<T>(), a1, b0, b1, u, v);
                const V3<T> dd = a1 * u - lerp(b0, b1, v);
                const T r = ri + std::max(padding[j], padding[j + 1]);
                if (len2(dd) < r * r) {
                    if (cnt < kMaxCols) cols[i].push_back(j);
                    cnt++;
                }
            }
            if (cnt > kMaxCols) pendingError = ERR_MAX_COLLISIONS;
            numCols[i] = std::min(cnt, kMaxCols);
        }
    }
    // recomputeStepLimitKernel, collision.cu:103-136.
    void step_limit() {
        for (int i = 0; i < n; i++) {
            T minDist = std::numeric_limits<T>::infinity();
            if (flags[i] & F_NEXT) {
                const V3<T> a0 = lastPos[i], a1 = lastPos[i + 1] - a0;
                minDist = padding[i] - detRadius;
                for (int c = 0; c < numCols[i]; c++) {
                    const int o = cols[i][c];
                    const V3<T> b0 = lastPos[o] - a0, b1 = lastPos[o + 1] - a0;
                    T u, v;
                    seg_closest(V3<T>(), a1, b0, b1, u, v);
                    const V3<T> nn = a1 * u - lerp(b0, b1, v);
                    minDist = std::min(minDist, T((1 - 0.1f) * 0.5f) * len(nn));
                }
            }
            maxStep[i] = minDist;
        }
    }

    // ------------------------------------------------------------------ substep pieces
    // initItr, iteration.cu:34-68 (the pose part is stage_poses).
    void init_itr() {
        for (int i = 0; i < n; i++) {
            const V3<T> v = vel[i];
            V3<T> d = v * h;
            const V3<T> lv = lastVel[i];
            lastVel[i] = v;
            T pad = scaledDetRadius;
            const V3<T> y = d + gravity * (h * h);
            pad += len(y);
            if (invMass[i] != 0) {
                vel[i] = y;  // vel holds the inertial target y during the iterations
                const T g2 = len2(gravity);
                if (g2 > 0) {
                    const V3<T> a = (v - lv) / lastH;
                    const T s = std::min(std::max(dot(a, gravity) / g2, T(0)), T(1));
                    d += gravity * (h * h * s);
                }
            }
            padding[i] = pad;
            dx[i] = d;
            lastPos[i] = pos[i];
        }
    }
    // cosseratItr<LIMIT, SNAPSHOT=true>, cosserat.cu:23-225; accumulation order kept:
    // inertia, surfaces, own stretch, collisions (even entries, then odd entries), then the
    // previous segment's (f2, H2).
    void position_sweep() {
        const T damp = damping / h;
        std::vector<V3<T>> F2(n);
        std::vector<S3<T>> H2v(n);
        std::vector<V3<T>> F(n);
        std::vector<S3<T>> Hv(n);
        for (int i = 0; i < n; i++) {
            const V3<T> d = dx[i];
            S3<T> H(T(1) / (invMass[i] * h * h));
            V3<T> f = (vel[i] - d) * (T(1) / (h * h * invMass[i]));
            if ((numPlanes > 0 || !grids.empty()) && invMass[i] != 0) {
                const T kap = cKappa / h;
                surfaces_at(i, pos[i], d, kap * kap / invMass[i], f, H);
            }
            V3<T> f2;
            S3<T> H2;
            V3<T> fS, f2S;      // odd collision entries ("sector 1")
            S3<T> HS, H2S;
            if (flags[i] & F_NEXT) {
                const V3<T> p1 = lastPos[i + 1], p1d = dx[i + 1];
                const T invl = T(1) / lRest[i];
                const V3<T> c = ((p1 - pos[i]) + (p1d - d)) * invl - qtangent(q[i]);
                const T k = kStretch[i] * invl;
                T dd = k * invl;
                f += c * k - d * (damp * dd);
                f2 += c * (-k) - p1d * (damp * dd);
                dd *= T(1) + damp;
                H.add_diag(dd);
                H2.add_diag(dd);
                if (ropeContact) {
                    const T invb = T(1) / barrier, rad2 = T(2) * radius, kCol = kCollision * invb;
                    for (int sidx = 0; sidx < 2; sidx++) {
                        V3<T>& fa = sidx ? fS : f;
                        V3<T>& fb = sidx ? f2S : f2;
                        S3<T>& Ha = sidx ? HS : H;
                        S3<T>& Hb = sidx ? H2S : H2;
                        for (int cc = sidx; cc < numCols[i]; cc += 2)
                            collision_term(i, cols[i][cc], p1, p1d, d, invb, rad2, kCol, damp, fa, fb, Ha, Hb);
                    }
                }
            }
            f += fS; f2 += f2S; H += HS; H2 += H2S;
            F[i] = f; Hv[i] = H; F2[i] = f2; H2v[i] = H2;
        }
        for (int i = 0; i < n; i++) {
            V3<T> f = F[i];
            S3<T> H = Hv[i];
            V3<T> d = dx[i];
            T lim = useStepLimit ? maxStep[i] : std::numeric_limits<T>::infinity();
            if (flags[i] & F_PREV) {
                if (useStepLimit) lim = std::min(lim, maxStep[i - 1]);
                f += F2[i - 1];
                H += H2v[i - 1];
            }
            if (invMass[i] != 0) {
                d += sym_solve(H, f) * accel;
                dxRaw[i] = d;
                if (useStepLimit) {
                    const T l = len(d);
                    if (l > lim && l > 0) {
                        d *= lim / l;
                        nLimitedSteps++;
                    }
                }
            }
            dxNext[i] = d;
            qPrev[i] = q[i];
        }
    }
    // One rope-rope candidate of segment i: IPC log barrier + friction, cosserat.cu:99-157.
    void collision_term(int i, int o, const V3<T>& p1, const V3<T>& p1d, const V3<T>& d, T invb, T rad2, T kCol, T damp,
                        V3<T>& f, V3<T>& f2, S3<T>& H, S3<T>& H2) const {
        const V3<T> b0 = lastPos[o], b1 = lastPos[o + 1], db0 = dx[o], db1 = dx[o + 1];
        T u, v;
        seg_closest(V3<T>(), (p1 - pos[i]) + (p1d - d), (b0 - pos[i]) + (db0 - d), (b1 - pos[i]) + (db1 - d), u, v);
        const V3<T> dpos = lerp(pos[i], p1, u) - lerp(b0, b1, v);
        const V3<T> ddpos = lerp(d, p1d, u) - lerp(db0, db1, v);
        V3<T> nrm = dpos + ddpos;
        T dist = len(nrm);
        if (!(dist > 0)) return;
        nrm *= T(1) / dist;
        const T wb = u, wa = T(1) - u;  // weights of the segment's two vertices
        dist = (dist - rad2) * invb;
        if (dist > 1) return;
        dist = std::max(dist, T(1e-3));
        nCollisionTerms++;
        const T invd = T(1) / dist, logd = m_log(dist);
        T dH = (T(-3) + (T(2) + invd) * invd - T(2) * logd) * kCol * invb;
        const T ff = -(T(1) - dist) * (dist - T(1) + T(2) * dist * logd) * invd * kCol;
        f += nrm * (ff * wa - damp * dH * wa * wa * dot(nrm, d));
        f2 += nrm * (ff * wb - damp * dH * wb * wb * dot(nrm, p1d));
        dH *= T(1) + damp;
        S3<T> op = S3<T>::outer(nrm);
        H += op * (dH * wa * wa);
        H2 += op * (dH * wb * wb);
        const V3<T> uu = ddpos - nrm * dot(nrm, ddpos);
        const T ul = len(uu);
        if (ul > 0) {
            const T f1 = std::min(kFriction, fricMu * ff / ul);
            op.add_diag(T(-1));
            f -= uu * (f1 * wa);
            H -= op * (wa * wa * f1);
            f2 -= uu * (f1 * wb);
            H2 -= op * (wb * wb * f1);
        }
    }
    // quaternionLambdaItr<SNAPSHOT=true>, cosserat.cu:227-273. With inplaceFrames the sweep reads
    // the rotors it has already updated (SNAPSHOT=false, cosserat.cu:252-268, reads d_qs while
    // threads write it): a vertex-order Gauss-Seidel pass, one deterministic realisation of the
    // reference's default racing sweep (there the order is the warp schedule), kept so that the
    // difference between the two orderings can be measured.
    void frame_sweep() {
        const std::vector<Q4<T>>& qs = inplaceFrames ? q : qPrev;
        for (int i = 0; i < n; i++) {
            dx[i] = dxNext[i];
            if ((flags[i] & F_FIX_ORIENT) || !(flags[i] & F_NEXT)) continue;
            const V3<T> d = dxNext[i], p1 = pos[i + 1], p1d = dxNext[i + 1];
            V3<T> vv = ((p1 - pos[i]) + (p1d - d)) / lRest[i];
            vv *= T(-2) * kStretch[i];
            Q4<T> b(0, 0, 0, 0);
            const Q4<T> q0 = qPrev[i];
            if (flags[i] & F_PREV) {
                const Q4<T> qr = qRest[i - 1], qq = qs[i - 1];
                const T s = dot4(qmul(qq.inv(), q0), qr) > 0 ? T(1) : T(-1);
                b += qmul(qq, qr) * s;
            }
            if (flags[i] & F_NEXT_ORIENT) {
                const Q4<T> qr = qRest[i], qq = qs[i + 1];
                const T s = dot4(qmul(q0.inv(), qq), qr) > 0 ? T(1) : T(-1);
                b += qmul(qq, qr.inv()) * s;
            }
            const T lambda = len(vv) + len4(b);
            const Q4<T> m = qmul(qmul(Q4<T>(vv, T(0)), b), Q4<T>(1, 0, 0, 0));
            q[i] = normalize4(m + b * lambda);
        }
    }
    // endItr, iteration.cu:77-129.
    void end_itr() {
        const T invH = T(1) / h;
        for (int i = 0; i < n; i++) {
            const V3<T> d = dx[i];
            if (invMass[i] != 0) {
                V3<T> v = d * invH;
                if (dragQuad > 0) {
                    const V3<T> t = (flags[i] & F_NEXT) ? qtangent(q[i]) : qtangent(q[i - 1]);
                    const V3<T> vt = t * dot(t, v);
                    V3<T> vn = v - vt;
                    vn /= T(1) + dragQuad * len(vn) * h;
                    V3<T> vtt = vt / (T(1) + dragQuadT * len(vt) * h);
                    v = vn + vtt;
                }
                vel[i] = v * (T(1) - drag * h);
                if (forcesOn && (numPlanes > 0 || !grids.empty())) {
                    const T kap = cKappa / h;
                    surface_readout(i, pos[i], d, kap * kap / invMass[i]);
                }
            }
            pos[i] += d;
            if (!grids.empty()) {
                if (invMass[i] != 0) build_candidates(i, pos[i], T(2) * len(d) + T(0.02));
                else numCand[i] = 0;
            }
        }
    }
    void substep(int sub, int nSub) {
        stage_poses(sub, nSub);
        init_itr();
        if (ropeContact) brute_detect();
        if (useStepLimit) step_limit();
        for (int it = 0; it < numItr; it++) { position_sweep(); frame_sweep(); }
        end_itr();
    }

    // ------------------------------------------------------------------ frame drivers
    // uploadMeta's derived radii and its validity check, YarnBall.cu:261-272.
    void prepare(T hNew) {
        lastH = h;
        h = hNew;
        detRadius = radius + T(0.5) * barrier;
        scaledDetRadius = detRadius * detScaler;
        if (T(2) * minSegLen < T(2) * radius + barrier)
            throw std::invalid_argument("Use thinner yarn or use longer segments");
    }
    void finish(float dt) {
        time += T(dt);
        if (pendingError) { lastError = pendingError; const int e = pendingError; pendingError = 0;
                            if (e == ERR_MAX_COLLISIONS) throw std::runtime_error("MAX_COLLISIONS_PER_SEGMENT exceeded"); }
        if (pendingWarning) { lastWarning = pendingWarning; pendingWarning = 0; }
    }
    // Sim::advance with the float ceil of the substep count, step.cpp:37-57.
    static int ceil_steps(float dt, float mh) {
        int s = (int)std::ceil(dt / mh);
        return s < 1 ? 1 : s;
    }
    template <class P>
    void run_substeps(int steps, float dt, const P* prog, const float* q0, const float* q1) {
        for (int s = 0; s < steps; s++) {
            if (prog) apply_root_program(prog, q0, q1, s, steps, dt);
            substep(s, steps);
        }
    }
    // RopeSim.advance(dt, substeps), bindings.cpp:274-295.
    void advance(float dt, int substeps) {
        if (!(dt > 0)) return;
        sdf_begin_step();
        const float mh = substeps > 0 ? (dt / (float)substeps) * 1.000001f : maxH;
        const int steps = ceil_steps(dt, mh);
        prepare(T(dt / (float)steps));
        run_substeps<float>(steps, dt, nullptr, nullptr, nullptr);
        finish(dt);
        sdf_end_step(substeps > 0 ? substeps : steps);
    }
    // RopeBatch.step (legacy constant-velocity roots), batch.cu:90-104,288-319.
    void step_legacy(const float* p, const float* v, const float* qq, float dt, int substeps) {
        for (int r = 0; r < R; r++) {
            const int root = start[r];
            pos[root] = V3<T>(T(p[3 * r]), T(p[3 * r + 1]), T(p[3 * r + 2]));
            vel[root] = V3<T>(T(v[3 * r]), T(v[3 * r + 1]), T(v[3 * r + 2]));
            if (qq) {
                Q4<T> a(T(qq[4 * r]), T(qq[4 * r + 1]), T(qq[4 * r + 2]), T(qq[4 * r + 3]));
                const T l2 = dot4(a, a);
                q[root] = l2 > 0 ? a * (T(1) / m_sqrt(l2)) : Q4<T>(0, 0, 0, 1);
            }
        }
        sdf_begin_step();
        if (ropeContact) {
            prepare(T(dt / (float)substeps));
            run_substeps<float>(substeps, dt, nullptr, nullptr, nullptr);
            finish(dt);
        } else {
            const float mh = (dt / (float)substeps) * 1.000001f;
            const int steps = ceil_steps(dt, mh);
            prepare(T(dt / (float)steps));
            run_substeps<float>(steps, dt, nullptr, nullptr, nullptr);
            finish(dt);
        }
        sdf_end_step(substeps);
    }
    // Shortest-arc SLERP with an nlerp fallback, batch.cu:106-114.
    static Q4<T> slerp(Q4<T> a, Q4<T> b, T t) {
        T d = dot4(a, b);
        if (d < 0) { b = b * T(-1); d = -d; }
        if (d > T(0.9995)) return normalize4(a * (T(1) - t) + b * t);
        const T th = m_acos(std::min(d, T(1)));
        const T s = m_sin(th);
        return a * (m_sin((T(1) - t) * th) / s) + b * (m_sin(t * th) / s);
    }
    static Q4<T> unit_or_identity(const float* qq, int r) {
        Q4<T> a(T(qq[4 * r]), T(qq[4 * r + 1]), T(qq[4 * r + 2]), T(qq[4 * r + 3]));
        const T l = dot4(a, a);
        return l > 0 ? a * (T(1) / m_sqrt(l)) : Q4<T>(0, 0, 0, 1);
    }
    // applyRootProgramK, batch.cu:122-159. prog = [p0 (3R), v0 (3R), p1 (3R)] (float rows as the
    // API passes them, or rows in T for finite differences of the program).
    template <class P>
    void apply_root_program(const P* prog, const float* q0, const float* q1, int s, int S, float dtf) {
        const T dt = T(dtf);
        for (int r = 0; r < R; r++) {
            const int root = start[r];
            const V3<T> P0(T(prog[3 * r]), T(prog[3 * r + 1]), T(prog[3 * r + 2]));
            const V3<T> V0(T(prog[3 * R + 3 * r]), T(prog[3 * R + 3 * r + 1]), T(prog[3 * R + 3 * r + 2]));
            const V3<T> P1(T(prog[6 * R + 3 * r]), T(prog[6 * R + 3 * r + 1]), T(prog[6 * R + 3 * r + 2]));
            const V3<T> A = ((P1 - P0) - V0 * dt) * (T(2) / (dt * dt));
            const T tau = T(s) * h;
            pos[root] = P0 + V0 * tau + A * (T(0.5) * tau * tau);
            vel[root] = V0 + A * (tau + T(0.5) * h);
            if (q0) {
                const Q4<T> qa = unit_or_identity(q0, r);
                Q4<T> qv = q1 ? slerp(qa, unit_or_identity(q1, r), T(s + 1) / T(S)) : qa;
                const T l2 = dot4(qv, qv);
                q[root] = l2 > 0 ? qv * (T(1) / m_sqrt(l2)) : Q4<T>(0, 0, 0, 1);
            }
        }
    }
    // RopeBatch::step_program, batch.cu:321-363.
    void step_program(const float* p0, const float* v0, const float* p1, const float* q0, const float* q1, float dt,
                      int substeps) {
        std::vector<float> prog((size_t)9 * R);
        std::memcpy(prog.data(), p0, sizeof(float) * 3 * R);
        std::memcpy(prog.data() + 3 * R, v0, sizeof(float) * 3 * R);
        std::memcpy(prog.data() + 6 * R, p1, sizeof(float) * 3 * R);
        sdf_begin_step();
        prepare(T(dt / (float)substeps));
        run_substeps(substeps, dt, prog.data(), q0, q1);
        finish(dt);
        sdf_end_step(substeps);
    }
    // The same frame with program rows in T (finite differences with respect to the program).
    void step_program_rows(const T* prog, float dt, int substeps) {
        sdf_begin_step();
        prepare(T(dt / (float)substeps));
        run_substeps(substeps, dt, prog, nullptr, nullptr);
        finish(dt);
        sdf_end_step(substeps);
    }
    // RopeBatch::step_free, batch.cu:388-398.
    void step_free(float dt, int substeps) {
        sdf_begin_step();
        prepare(T(dt / (float)substeps));
        run_substeps<float>(substeps, dt, nullptr, nullptr, nullptr);
        finish(dt);
        sdf_end_step(substeps);
    }
    // resetEnvsK, batch.cu:178-189 (here by rope index).
    void reset_ropes(const int* ids, int count) {
        for (int c = 0; c < count; c++)
            for (int i = start[ids[c]]; i < start[ids[c] + 1]; i++) {
                pos[i] = initPos[i]; q[i] = initQ[i]; vel[i] = V3<T>(); lastVel[i] = V3<T>();
            }
    }
    // RopeSim::reset, bindings.cpp:303-316.
    void reset_all() {
        for (int i = 0; i < n; i++) { pos[i] = initPos[i]; q[i] = initQ[i]; vel[i] = V3<T>(); lastVel[i] = V3<T>(); }
        time = 0;
        h = T(maxH);
        lastError = lastWarning = 0;
    }
};

}  // namespace rso
