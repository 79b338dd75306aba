// rs_plain.cu -- the per-substep-launch ("plain") engine: the reference's launch structure
// (batch.cu:352-358 + step.cpp:5-35) over the same per-vertex arithmetic as the persistent
// frame kernel (rs_substep.cuh), used as the in-repo plain path the persistent kernel is
// measured against and as a cross-check of it.
//
// Per substep: root kernel (program roots), pose kernel (moving meshes), init kernel, then one
// CUDA-graph replay of num_itr x (position kernel, frame kernel) + end kernel. State and the
// frame's parameters live in global memory (like YarnBall's MetaData upload), so the captured
// graph stays valid across frames. Position kernel: 128 threads own 127 vertices plus one halo
// vertex that recomputes the previous segment's share (cosserat.cu:16-27, one thread per vertex).
#include <cuda_runtime.h>

#include "rs_kernels.h"
#include "rs_substep.cuh"

namespace rs {

namespace {

constexpr int kPosBlock = 128;
constexpr int kOwned = kPosBlock - 1;
constexpr int kOwnedRope = kPosBlock / 2 - 1;  // rope-rope variant: two threads per vertex

__device__ __forceinline__ const float4* env_poses(const FrameArgs& a, const PlainBufs& b, int env) {
    const Pose* base = (a.sdf_moving ? b.spose : a.poses) + (size_t)env * kMaxSdf;
    return reinterpret_cast<const float4*>(base);
}

// Root program / legacy root of every rope (one thread per device rope), batch.cu:90-159.
__global__ void plain_root_kernel(const FrameArgs* __restrict__ pa, int nropes, int s) {
    const FrameArgs& a = *pa;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nropes) return;
    const Rope rp = a.ropes[r];
    const int d = rp.dstart;
    const float* row = a.prog + (size_t)rp.user * 17;
    float4 P = a.pos[d], Vv = a.vel[d];
    f3 p = xyz(P), v = xyz(Vv);
    float4 q = a.q[d];
    if (a.root_mode == ROOT_PROGRAM) root_program(a, row, s, a.substeps, a.h, p, v, q);
    else if (a.root_mode == ROOT_SET && s == 0) root_set(a, row, p, v, q);
    else return;
    a.pos[d] = f4(p, P.w);
    a.vel[d] = f4(v, Vv.w);
    a.q[d] = q;
}

// Poses of every (env, mesh) at the end of substep s (moving frames), iteration.cu:12-33.
__global__ void plain_pose_kernel(const FrameArgs* __restrict__ pa, PlainBufs b, int envs, int s) {
    const FrameArgs& a = *pa;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= envs * a.num_sdf) return;
    const int en = i / a.num_sdf, m = i % a.num_sdf;
    compute_pose(a, en, m, s, a.substeps, a.h, reinterpret_cast<float4*>(b.spose + (size_t)en * kMaxSdf + m));
}

// Inertial prediction, initial guess, lastPos, iteration.cu:34-68; the first substep of a
// frame resets the broad phase to "every mesh". Differentiable frames tape the substep's start
// state here (after its root program; caller order, broad-phase mask in the .w lanes).
__global__ void plain_init_kernel(const FrameArgs* __restrict__ pa, PlainBufs b, int n, int s) {
    const FrameArgs& a = *pa;
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const int first = s == 0;
    const float4 P = a.pos[d], Vv = a.vel[d], L = a.lvel[d];
    if (first) b.cand[d] = all_meshes(a.num_sdf);
    if (a.tape) {
        const uint64_t cm = b.cand[d];
        float4* tp = a.tape + (size_t)s * 4 * n + a.topo[d].z;
        tp[0] = make_float4(P.x, P.y, P.z, __int_as_float((int)(uint32_t)cm));
        tp[n] = make_float4(Vv.x, Vv.y, Vv.z, __int_as_float((int)(uint32_t)(cm >> 32)));
        tp[2 * (size_t)n] = L;
        tp[3 * (size_t)n] = a.q[d];
    }
    const f3 g = mk3(a.gx, a.gy, a.gz);
    f3 dx, y;
    init_vertex(xyz(Vv), xyz(L), P.w, a.h, a.last_h, g, dot(g, g), dx, y);
    a.lvel[d] = make_float4(Vv.x, Vv.y, Vv.z, L.w);
    b.dx[d] = f4(dx, 0.f);
    b.y[d] = f4(y, 0.f);
    b.lpos[d] = P;
    if (a.rope_contact) a.pad[d] = a.sdet_radius + len(y);
}

// Rope-rope detection of segment d over its contact group (ascending j, cap kMaxCols) and its
// step limit, batch.cu:19-49 and collision.cu:103-136.
__global__ void plain_detect_kernel(const FrameArgs* __restrict__ pa, PlainBufs b, int n) {
    const FrameArgs& a = *pa;
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const uint32_t fl = (uint32_t)a.topo[d].x;
    if (!(fl & F_NEXT)) {
        a.ncols[d] = 0;
        a.maxstep[d] = INFINITY;
        return;
    }
    const int4 gr = a.grp[d];
    float lim;
    const int cnt = detect_group(
        a, d, d, gr.x, gr.y, gr.z, gr.w, xyz(b.lpos[d]), xyz(b.lpos[d + 1]), [&](int j) { return a.pad[j]; },
        [&](int j) { return a.topo[j].x; }, [&](int j) { return xyz(b.lpos[j]); }, lim);
    if (cnt > kMaxCols) atomicMax(a.status, ERR_MAX_COLLISIONS);
    a.ncols[d] = cnt < kMaxCols ? cnt : kMaxCols;
    a.maxstep[d] = lim;
}

// Position step (SNAPSHOT): reads the previous iterate, writes dxNext and the frame snapshot,
// cosserat.cu:23-225.
template <int SURF, bool ROPE>
__global__ void __launch_bounds__(kPosBlock) plain_position_kernel(const FrameArgs* __restrict__ pa, PlainBufs b, int n) {
    const FrameArgs& a = *pa;
    __shared__ float4 sfa[kPosBlock], sfb[kPosBlock];
    __shared__ float sfc[kPosBlock];
    const int lt = threadIdx.x;
    const int d = blockIdx.x * kOwned + lt - 1;
    const bool valid = d >= 0 && d < n;
    uint32_t fl = 0;
    f3 f = zero3(), f2 = zero3(), dx = zero3();
    sym3 H = sym_zero(), H2 = sym_zero();
    float im = 0.f;
    bool touched = false;
    float4 q = make_float4(0.f, 0.f, 0.f, 1.f);
    if (valid) {
        const int4 tp = a.topo[d];
        fl = (uint32_t)tp.x;
        const float4 P = b.lpos[d];
        im = P.w;
        const VConst c = vertex_constants(a, im, a.vel[d].w, a.lvel[d].w);
        const bool hasNext = fl & F_NEXT;
        dx = xyz(b.dx[d]);
        q = a.q[d];
        const f3 p1 = hasNext ? xyz(b.lpos[d + 1]) : zero3();
        const f3 p1dx = hasNext ? xyz(b.dx[d + 1]) : zero3();
        const float4* cache = (SURF == SURF_MESHES) ? env_poses(a, b, tp.w) : nullptr;
        const uint64_t cand = (SURF == SURF_MESHES) ? b.cand[d] : 0ull;
        const float damp = a.damping / a.h;
        touched = position_terms<SURF>(a, cache, cand, c, hasNext, xyz(P), p1, dx, p1dx, xyz(b.y[d]), q, damp, f, H, f2, H2);
        if constexpr (ROPE) {
            const int nc = hasNext ? a.ncols[d] : 0;
            if (nc > 0) {
                f3 fo = zero3(), f2o = zero3();
                sym3 Ho = sym_zero(), H2o = sym_zero();
                for (int cc = 0; cc < nc; cc++) {
                    const int j = a.cols[(size_t)cc * n + d];
                    const f3 b0 = xyz(b.lpos[j]), b1 = xyz(b.lpos[j + 1]), db0 = xyz(b.dx[j]), db1 = xyz(b.dx[j + 1]);
                    if (cc & 1) collision_term(a, damp, xyz(P), p1, dx, p1dx, b0, b1, db0, db1, fo, f2o, Ho, H2o);
                    else collision_term(a, damp, xyz(P), p1, dx, p1dx, b0, b1, db0, db1, f, f2, H, H2);
                }
                if (nc > 1) { f += fo; f2 += f2o; sym_add(H, Ho); sym_add(H2, H2o); }
            }
        }
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
    if constexpr (ROPE) {
        const float lim = (fl & F_PREV) ? fminf(a.maxstep[d], a.maxstep[d - 1]) : a.maxstep[d];
        position_solve_limited(dx, f, H, a.accel, im, lim);
    } else {
        position_solve(dx, f, H, a.accel, im, !touched);
    }
    b.dxn[d] = f4(dx, 0.f);
    b.qprev[d] = q;
}

// Position step with rope-rope terms, two threads per vertex: the reference splits a segment's
// candidates into two sectors (even ones join the own terms, odd ones a partial added after
// them, cosserat.cu:99-182); here each sector runs on its own thread, so the sums are formed in
// the same order with twice the threads (a contact group that exceeds a CTA is too small to fill
// the GPU at one thread per vertex).
template <int SURF>
__global__ void __launch_bounds__(kPosBlock) plain_position_rope_kernel(const FrameArgs* __restrict__ pa, PlainBufs b,
                                                                        int n) {
    const FrameArgs& a = *pa;
    constexpr int V = kPosBlock / 2;
    __shared__ float4 so[V][5];  // sector 1: fo, f2o, Ho, H2o
    __shared__ float4 sfa[V], sfb[V];
    __shared__ float sfc[V];
    const int lt = threadIdx.x, lv = lt >> 1, sec = lt & 1;
    const int d = blockIdx.x * kOwnedRope + lv - 1;
    const bool valid = d >= 0 && d < n;
    uint32_t fl = 0;
    f3 f = zero3(), f2 = zero3(), dx = zero3();
    sym3 H = sym_zero(), H2 = sym_zero();
    float im = 0.f;
    float4 q = make_float4(0.f, 0.f, 0.f, 1.f);
    int nc = 0;
    if (valid) {
        const int4 tp = a.topo[d];
        fl = (uint32_t)tp.x;
        const float4 P = b.lpos[d];
        im = P.w;
        const bool hasNext = fl & F_NEXT;
        dx = xyz(b.dx[d]);
        q = a.q[d];
        const f3 p1 = hasNext ? xyz(b.lpos[d + 1]) : zero3();
        const f3 p1dx = hasNext ? xyz(b.dx[d + 1]) : zero3();
        const float damp = a.damping / a.h;
        nc = hasNext ? a.ncols[d] : 0;
        if (sec == 0) {
            const VConst c = vertex_constants(a, im, a.vel[d].w, a.lvel[d].w);
            const float4* cache = (SURF == SURF_MESHES) ? env_poses(a, b, tp.w) : nullptr;
            const uint64_t cand = (SURF == SURF_MESHES) ? b.cand[d] : 0ull;
            position_terms<SURF>(a, cache, cand, c, hasNext, xyz(P), p1, dx, p1dx, xyz(b.y[d]), q, damp, f, H, f2, H2);
        }
        for (int cc = sec; cc < nc; cc += 2) {
            const int j = a.cols[(size_t)cc * n + d];
            const f3 b0 = xyz(b.lpos[j]), b1 = xyz(b.lpos[j + 1]), db0 = xyz(b.dx[j]), db1 = xyz(b.dx[j + 1]);
            collision_term(a, damp, xyz(P), p1, dx, p1dx, b0, b1, db0, db1, f, f2, H, H2);
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
    position_solve_limited(dx, f, H, a.accel, im, lim);
    b.dxn[d] = f4(dx, 0.f);
    b.qprev[d] = q;
}

// Frame step (SNAPSHOT) and dx <- dxNext, cosserat.cu:227-273.
__global__ void plain_frame_kernel(const FrameArgs* __restrict__ pa, PlainBufs b, int n) {
    const FrameArgs& a = *pa;
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const float4 dxn = b.dxn[d];
    b.dx[d] = dxn;
    const uint32_t fl = (uint32_t)a.topo[d].x;
    if ((fl & F_FIX_ORIENT) || !(fl & F_NEXT)) return;
    const float4 q = b.qprev[d];
    const f3 seg = (xyz(b.lpos[d + 1]) - xyz(b.lpos[d])) + (xyz(b.dxn[d + 1]) - xyz(dxn));
    const bool hp = fl & F_PREV, hn = fl & F_NEXT_ORIENT;
    a.q[d] = frame_update(q, seg, 1.f / a.vel[d].w, a.lvel[d].w, hp, hp ? b.qprev[d - 1] : q, hp ? a.qrest[d - 1] : q, hn,
                          hn ? b.qprev[d + 1] : q, a.qrest[d]);
}

// Velocity, drag, readout, advection and broad phase, iteration.cu:77-129.
template <int SURF>
__global__ void plain_end_kernel(const FrameArgs* __restrict__ pa, PlainBufs b, int n) {
    const FrameArgs& a = *pa;
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const int4 tp = a.topo[d];
    const uint32_t fl = (uint32_t)tp.x;
    float4 P = a.pos[d];
    const f3 dx = xyz(b.dx[d]);
    const float im = P.w;
    const float4* cache = (SURF == SURF_MESHES) ? env_poses(a, b, tp.w) : nullptr;
    const uint64_t cand = (SURF == SURF_MESHES) ? b.cand[d] : 0ull;
    if (im != 0.f) {
        const f3 tg = (a.drag_quad > 0.f) ? ((fl & F_NEXT) ? qtangent(a.q[d]) : qtangent(a.q[d - 1])) : zero3();
        const float4 Vv = a.vel[d];
        a.vel[d] = f4(end_velocity(a, dx, 1.f / a.h, tg), Vv.w);
        if (SURF != SURF_NONE && a.forces_on) {
            const float kap = a.c_kappa / a.h;
            f3 fv = zero3();
            sym3 Hs = sym_zero();
            float* wrow = (SURF == SURF_MESHES && a.num_sdf > 0) ? a.wrench + (size_t)tp.w * kMaxSdf * 6 : nullptr;
            surfaces<SURF>(a, cache, cand, xyz(P), dx, kap * kap / im, a.h, fv, Hs, wrow, &fv);
            b.facc[d] = add4(b.facc[d], f4(fv, 0.f));
        }
    }
    P = f4(xyz(P) + dx, P.w);
    a.pos[d] = P;
    if (SURF == SURF_MESHES && a.num_sdf > 0) b.cand[d] = (im != 0.f) ? build_candidates(a, cache, a.num_sdf, xyz(P), dx) : 0ull;
}

// Frame end: caller-order views, averaged contact forces, non-finite check.
__global__ void plain_finish_kernel(const FrameArgs* __restrict__ pa, PlainBufs b, int n) {
    const FrameArgs& a = *pa;
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const int u = a.topo[d].z;
    const float4 P = a.pos[d], Vv = a.vel[d];
    a.out_pos[3 * (size_t)u] = P.x; a.out_pos[3 * (size_t)u + 1] = P.y; a.out_pos[3 * (size_t)u + 2] = P.z;
    a.out_vel[3 * (size_t)u] = Vv.x; a.out_vel[3 * (size_t)u + 1] = Vv.y; a.out_vel[3 * (size_t)u + 2] = Vv.z;
    reinterpret_cast<float4*>(a.out_q)[u] = a.q[d];
    if (a.forces_on && a.out_force) {
        const float k = 1.f / float(a.substeps);
        const float4 fc = b.facc[d];
        a.out_force[3 * (size_t)u] = fc.x * k; a.out_force[3 * (size_t)u + 1] = fc.y * k; a.out_force[3 * (size_t)u + 2] = fc.z * k;
        b.facc[d] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    if (!(isfinite(P.x) && isfinite(P.y) && isfinite(P.z))) atomicOr(a.status + 2, 1);
}

inline int blocks_of(int n, int t) { return (n + t - 1) / t; }

template <int SURF, bool ROPE>
void capture_inner(const FrameArgs* pa, const PlainBufs& b, int n, int iters, cudaStream_t s) {
    for (int it = 0; it < iters; it++) {
        if constexpr (ROPE) plain_position_rope_kernel<SURF><<<blocks_of(n, kOwnedRope), kPosBlock, 0, s>>>(pa, b, n);
        else plain_position_kernel<SURF, ROPE><<<blocks_of(n, kOwned), kPosBlock, 0, s>>>(pa, b, n);
        plain_frame_kernel<<<blocks_of(n, 128), 128, 0, s>>>(pa, b, n);
    }
    plain_end_kernel<SURF><<<blocks_of(n, 256), 256, 0, s>>>(pa, b, n);
}

}  // namespace

template <bool ROPE>
void record_inner(const FrameArgs* pa, const PlainBufs& b, int n, int iters, int surf, cudaStream_t s) {
    if (surf == SURF_MESHES) capture_inner<SURF_MESHES, ROPE>(pa, b, n, iters, s);
    else if (surf == SURF_PLANES) capture_inner<SURF_PLANES, ROPE>(pa, b, n, iters, s);
    else capture_inner<SURF_NONE, ROPE>(pa, b, n, iters, s);
}

cudaError_t plain_record_inner(const FrameArgs* pa, const PlainBufs& b, int n, int iters, int surf, bool rope,
                               cudaStream_t s) {
    if (rope) record_inner<true>(pa, b, n, iters, surf, s);
    else record_inner<false>(pa, b, n, iters, surf, s);
    return cudaGetLastError();
}

cudaError_t plain_launch_pre(const FrameArgs* pa, const PlainBufs& b, int n, int nropes, int envs, int num_sdf, bool moving,
                             int root_mode, bool rope, int s, const RopeGrid* grid, cudaStream_t st) {
    if (root_mode != ROOT_NONE && (root_mode == ROOT_PROGRAM || s == 0))
        plain_root_kernel<<<blocks_of(nropes, 128), 128, 0, st>>>(pa, nropes, s);
    if (num_sdf > 0 && moving) plain_pose_kernel<<<blocks_of(envs * num_sdf, 128), 128, 0, st>>>(pa, b, envs, s);
    plain_init_kernel<<<blocks_of(n, 256), 256, 0, st>>>(pa, b, n, s);
    if (rope && grid) {
        const cudaError_t e = rope_grid_detect(pa, b.lpos, *grid, n, true, st);
        if (e != cudaSuccess) return e;
    } else if (rope) {
        plain_detect_kernel<<<blocks_of(n, 128), 128, 0, st>>>(pa, b, n);
    }
    return cudaGetLastError();
}

cudaError_t plain_launch_finish(const FrameArgs* pa, const PlainBufs& b, int n, cudaStream_t st) {
    plain_finish_kernel<<<blocks_of(n, 256), 256, 0, st>>>(pa, b, n);
    return cudaGetLastError();
}

}  // namespace rs
