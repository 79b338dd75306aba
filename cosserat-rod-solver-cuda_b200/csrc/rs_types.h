// rs_types.h -- plain-old-data shared by the host driver and the sm_100a kernels.
//
// Device layout ("packed order"): ropes are packed whole into bins; one bin is one CTA of
// BLOCK threads, one thread per vertex, and a rope never straddles two bins. Device vertex
// arrays are in bin order; `uidx` maps every device vertex back to the caller's flat order
// (rope-major, as in the reference's RopeBatch: rope e owns [start_e, start_e + V_e)).
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define RS_HD __host__ __device__
#else
#define RS_HD
#endif

namespace rs {

// Vertex flags. Bits 0-3 keep the meaning of YarnBall's VertexFlags (YarnBall.h:52-58);
// bit 5 marks a rope's first vertex (the driven root).
enum : uint32_t {
    F_PREV = 1u,         // has a previous vertex on the same rope
    F_NEXT = 2u,         // has a next vertex (owns segment i -> i+1)
    F_NEXT_ORIENT = 4u,  // segment i has a next segment (bending with i+1)
    F_FIX_ORIENT = 8u,   // frame of segment i is held (clamped root, rope end)
    F_ROOT = 32u,        // first vertex of its rope
};

constexpr int kMaxSdf = 64;      // meshes per solver (YarnBall.h:153)
constexpr int kMaxCand = 8;      // broad-phase list length before "visit every mesh"
constexpr int kMaxPlanes = 8;
constexpr int kMaxCols = 128;    // rope-rope candidates per segment (YarnBall.h:38)

// Solver status words (YarnBall.h:204-208).
enum : int { ERR_NONE = 0, ERR_MAX_COLLISIONS = 1, WARN_INTERPENETRATION = 2 };

// Checked builds (-DROPESIM_CHECKED): the frame and adjoint kernels test every index that the
// topology or the data could push out of range and record the first failing check's code in the
// fourth status word (the access is then skipped or redirected in range; nothing traps). The
// regular build compiles the checks away.
#ifdef ROPESIM_CHECKED
constexpr bool kChecked = true;
#else
constexpr bool kChecked = false;
#endif
enum : int {
    CHK_NONE = 0,
    CHK_BIN = 1,         // a bin's vertex range outside [0, n) or larger than the CTA
    CHK_NEXT = 2,        // a next-vertex / next-segment flag on the bin's last vertex (reads t + 1)
    CHK_PREV = 3,        // a previous-vertex read (t - 1) at the bin's first vertex
    CHK_CALLER = 4,      // a caller-order index or rope (env) index out of range
    CHK_GROUP = 5,       // a rope-rope contact group or rope range outside the bin
    CHK_CANDIDATE = 6,   // a rope-rope candidate segment outside the bin
    CHK_POSE = 7,        // a pose-cache slot outside the cache, or a mesh bit beyond num_sdf
    CHK_LATTICE = 8,     // a lattice node outside its grid
    CHK_BLOCK = 9,       // a lattice block-bound index outside its table
};

// One bin = one CTA: a contiguous range of device vertices and of device ropes.
struct Bin {
    int vstart, vcount;   // device vertices [vstart, vstart + vcount)
    int rstart, rcount;   // device ropes [rstart, rstart + rcount)
};

// One rope in device order.
struct Rope {
    int dstart, count;    // device vertices
    int ustart;           // first vertex in the caller's flat order
    int user;             // caller's rope index (= env of its meshes, row of its root program)
};

// A signed-distance lattice: values[nx, ny, nz] (C order) at origin + ijk * h, object frame.
// bmin[bx, by, bz]: the smallest node value of each block of kSdfBlock^3 cells (nodes of the
// block's faces included), a lower bound of the trilinear field inside the block.
constexpr int kSdfBlock = 8;
struct GridDesc {
    const float* v;
    const float* bmin;
    int nx, ny, nz;
    float ox, oy, oz;
    float h, invH;
    float muS, muK;
    int by, bz;
    int bcount, boff;  // blocks of this lattice, and its offset in the CTA-staged bound tables
    // object-frame box of the blocks where contact at the current radius is possible (their
    // bound <= radius + 1e-5), padded by 1e-4; never = 1 when no block qualifies
    float tlo[3], thi[3];
    int never;
    int* status;   // the batch's status words (checked builds record lattice index failures there)
    // 1 / L, rounded down, with L = |(Dx, Dy, Dz)| and D the largest node difference along an axis
    // divided by the spacing: the trilinear field is Lipschitz with constant L, so a probe moved by
    // |d| changes phi by at most L |d| (the persistent kernel's per-substep contact slack)
    float lip_inv;
};

// Kinematic pose of (env, mesh) at the end of a substep: position, rotor (x, y, z, w),
// velocity of the origin, angular velocity (world), world AABB of the lattice.
struct Pose {
    float px, py, pz, vx;
    float qx, qy, qz, qw;
    float vy, vz, wx, wy;
    float wz, lox, loy, loz;
    float hix, hiy, hiz, pad_;
};

// One frame of motion of (env, mesh): start pose, translation, world rotation vector.
struct Motion {
    float p0x, p0y, p0z, dpx;
    float qx, qy, qz, qw;
    float dpy, dpz, rx, ry;
    float rz, pad0, pad1, pad2;
};

// Host staging of a caller-side pose target: position + rotor.
struct Pose7 {
    float px, py, pz, qx, qy, qz, qw, pad_;
};

// Root driving of one frame.
enum : int { ROOT_NONE = 0, ROOT_PROGRAM = 1, ROOT_SET = 2 };

// Everything one persistent frame launch needs, passed by value.
struct FrameArgs {
    // topology (device order)
    const Bin* bins;
    int num_bins;
    // the work queue (rs_frame.cu, frame_kernel): with `queue` set, resident CTAs take bins from
    // *queue (zeroed before the launch) in the order `order` gives; `bin_cost` receives each bin's
    // time in SM cycles (both may be null)
    int* queue;
    const int* order;
    float* bin_cost;
    const Rope* ropes;
    const int4* topo;        // (flags, local rope within the bin, uidx, env)
    // state (device order), updated in place
    float4* pos;             // (x, y, z, invMass)
    float4* vel;             // (vx, vy, vz, lRest)
    float4* lvel;            // (last substep's start velocity xyz, kStretch)
    float4* q;               // segment frame rotor
    const float4* qrest;     // rest rotation (scaled by the bending stiffness)
    // caller-order outputs (the zero-copy views)
    float* out_pos;          // [n, 3]
    float* out_vel;          // [n, 3]
    float* out_q;            // [n, 4]
    float* out_force;        // [n, 3] contact force readout (forces on)
    float* wrench;           // [envs, 64, 6] mesh wrench readout (forces on)
    int* status;             // [2] error, warning
    // root program rows [R, 17] = (p0, v0, p1, q0, q1), caller rope order
    const float* prog;
    int root_mode, has_q0, has_q1;
    // step
    float h, last_h, dt;
    int substeps, iters;
    // physics
    float gx, gy, gz;
    float damping, drag, drag_quad, drag_quad_t, accel;
    // surface contact
    int num_planes;
    float4 planes[kMaxPlanes];
    float c_radius, c_kappa, c_mu_s, c_mu_k, c_vslip;
    int num_sdf, sdf_moving, forces_on;
    int pose_cache;          // pose cache entries per buffer (= max ropes per bin * num_sdf)
    const Pose* poses;       // [envs * 64] committed static poses
    const Motion* motion;    // [envs * 64] this frame's motion (sdf_moving)
    // rope-rope contact (YarnBall.h:175-192; batch.cu:19-49, 367-385)
    int rope_contact;        // 0 = off
    int n;                   // vertices (stride of the candidate lists)
    int num_ropes;           // ropes (rows of the root program, envs of the mesh poses)
    float rc_radius, rc_barrier, rc_kcol, rc_mu, rc_kfric;
    float det_radius, sdet_radius;  // radius + barrier/2, and that times the detection scaler
    const int4* grp;         // per device vertex: (group start, group end, rope start, rope end)
    int* cols;               // [kMaxCols * n] candidate lists, cols[c * n + i] (scratch)
    int* ncols;              // [n] candidate counts (plain engine)
    float* maxstep;          // [n] step limits (plain engine)
    float* pad;              // [n] detection paddings (plain engine)
    GridDesc grids[kMaxSdf];
    int sdf_skip;            // 1: a lattice block whose lower bound clears the radius skips the sample
    int surf_cull;           // 1: the persistent kernel skips surface terms below the substep's slack (exact)
    int sdf_btab;            // floats of block bounds staged per CTA in shared memory (0 = read from L2)
    // differentiable frames: when set, the state after each substep's root program is written to
    // tape[(s * 4 + f) * n + u] for f = x, v, lv (previous substep's start velocity), q and the
    // caller-order index u
    float4* tape;
    // and, when set (no rope-rope contact), every iterate of frame step k = 0 .. I-1: d^{k+1} at
    // itape[(s * 3I + k) * n + u] (.w: the step's two sign tests, frame_signs_encode), q^{k+1} at
    // itape[(s * 3I + I + k) * n + u] and the step's blend rotor b at itape[(s * 3I + 2I + k) * n + u]
    float4* itape;
};

// One frame's backward (rs_adjoint.cu). Arrays are caller order; null outputs are skipped and
// null upstream adjoints read as zero.
struct AdjArgs {
    const float4* tape;                          // [S][4][n] caller order, written by a frame launch
    const float4* itape;                         // [S][3I][n] caller order iterates, or null (recompute)
    const float *g_pos, *g_vel, *g_lvel, *g_q;   // adjoints of the frame-end state [n,3] x3, [n,4]
    float *o_pos, *o_vel, *o_lvel, *o_q;         // adjoints of the frame-start state
    float *o_ea, *o_ei, *o_mass;                 // [n] adjoints of EA, EI (segment i -> i+1), mass
    float *o_p0, *o_v0, *o_p1;                   // [R,3] adjoints of the root program rows
};

// HBM arrays of the per-launch adjoint (contact groups larger than one CTA, or the plain engine),
// one float4 (or word) per device vertex unless noted.
struct PlainAdjBufs {
    float4* ld;           // [(iters + 1) n] displacement iterates d^k (.w: the step limit's scale)
    float4* lq;           // [(iters + 1) n] frame iterates q^k
    float4* x;            // substep-start positions (+ invMass)
    float4* y;            // inertial targets
    uint64_t* cand;       // broad-phase mesh mask of the substep (from the tape)
    float4 *gx, *gv, *gl, *gq;  // (x̄, k̄s), (v̄, ρ̄), (l̄v, ρ̄ of the previous segment), q̄
    float4 *gp0, *gv0, *gp1;    // program adjoints of driven roots (.w of gv0: w̄, the invMass adjoint)
    float4 *td, *tn, *ty;       // per substep: d̄, v̄ at the substep start, ȳ
    float2* ms;                 // per substep: step-limit adjoints (own segment, previous segment)
    float4 *ea, *eb, *ec;       // frame reverse: shares to the previous / next rotor, segment share
    float4 *ha0, *ha1, *hb0, *hb1;  // collision Hessians at d^k: own share, next vertex's share
    float4 *ef, *ee;            // (F̄, tr H̄) and e = H⁻¹ z̄ of the position reverse
    float4* cd;                 // [2 n] pair shares of d̄ by iteration parity (atomics)
    float4* cx;                 // pair shares of x̄ over the substep (atomics)
    float4* qp;                 // quadratic-drag share on the previous vertex's frame
};

// Uniform-grid broad phase of rope-rope detection for contact groups larger than one CTA:
// segment midpoints hashed into cells of twice the largest reach, counting-sorted by bucket.
struct RopeGrid {
    float4* ms;        // [n] segment midpoint and reach (half length + padded radius); w < 0: no segment
    int* bucket;       // [n] hash bucket of the segment's cell (-1: no segment)
    int* count;        // [T + 1] bucket counts, then fill cursors
    int* start;        // [T + 1] exclusive scan of the counts
    int* sorted;       // [n] segments by bucket
    unsigned* smax;    // the largest reach (float bits)
    void* scan_tmp;    // CUB scan scratch
    size_t scan_bytes;
    int T;             // buckets, a power of two
};

// Global-memory working set of the per-substep-launch (plain) engine.
struct PlainBufs {
    float4* dx;       // displacement iterate
    float4* dxn;      // next iterate (Jacobi output)
    float4* y;        // inertial target
    float4* qprev;    // frame snapshot of the iteration
    float4* lpos;     // positions at the substep start (+ invMass)
    float4* facc;     // contact-force readout accumulated over the frame
    uint64_t* cand;   // broad-phase mesh mask per vertex
    Pose* spose;      // [envs * 64] poses of the current substep (moving meshes)
};

}  // namespace rs
