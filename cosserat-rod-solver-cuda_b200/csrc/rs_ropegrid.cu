// rs_ropegrid.cu -- rope-rope detection for contact groups larger than one CTA through a uniform
// grid, with the candidate lists of the brute force (batch.cu:19-49) pair for pair.
//
// The brute force tests every segment pair of a group (O(V²): 10⁹ pairs per substep for a group
// of 32,768 segments). Here each substep: (1) every segment's midpoint m and reach s (half length
// + padded radius) and the largest reach; (2) the midpoint's cell (edge c = 2 s_max + margin)
// hashed into T buckets, counted; (3) an exclusive scan (CUB) and a scatter sort the segments by
// bucket; (4) one thread per (segment, cell) scans the 27 cells around each segment's own and
// appends the accepted candidates; (5) each segment sorts its list. Any pair that passes
// detect_group's early out has midpoints closer than c, so the partner sits in one of those
// cells: the visited set contains every candidate, each visited pair runs detect_group's own pair
// test (pair_accepts), each bucket is scanned once per segment (a hash can alias two neighbour
// cells), and the accepted indices are sorted. That sorted list is the brute force's ascending
// list. A segment with more
// than kMaxCols candidates reruns the brute force, which keeps the first kMaxCols and flags
// MAX_COLLISIONS as the reference does.
#include <cub/cub.cuh>

#include "rs_kernels.h"
#include "rs_substep.cuh"

namespace rs {

namespace {

__device__ __forceinline__ float cell_edge(const RopeGrid& g) {
    return (2.f * __uint_as_float(*g.smax) * 1.0001f + 1e-6f) * 1.001f + 1e-6f;
}
__device__ __forceinline__ int hash_cell(int ix, int iy, int iz, int T) {
    const unsigned h = (unsigned)ix * 73856093u ^ (unsigned)iy * 19349663u ^ (unsigned)iz * 83492791u;
    return (int)(h & (unsigned)(T - 1));
}

__global__ void rg_reach_kernel(const FrameArgs* __restrict__ pa, const float4* __restrict__ pos, RopeGrid g, int n) {
    const FrameArgs& a = *pa;
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    a.ncols[d] = 0;  // the cell pass counts this segment's candidates here
    if (!(a.topo[d].x & F_NEXT)) {
        g.ms[d] = make_float4(0.f, 0.f, 0.f, -1.f);
        return;
    }
    const f3 p = xyz(pos[d]), p1 = xyz(pos[d + 1]);
    const float s = 0.5f * len(p1 - p) + fmaxf(a.pad[d], a.pad[d + 1]);
    const f3 m = (p + p1) * 0.5f;
    if (!(isfinite(s) && isfinite(m.x) && isfinite(m.y) && isfinite(m.z))) {
        // a diverged segment takes no part (the brute force's tests would reject it as well):
        // it must not widen the cells of every other segment
        g.ms[d] = make_float4(0.f, 0.f, 0.f, -1.f);
        return;
    }
    g.ms[d] = f4(m, s);
    atomicMax(g.smax, __float_as_uint(s));  // reaches are positive: their bits order as the floats
}

__global__ void rg_bucket_kernel(RopeGrid g, int n) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const float4 m = g.ms[d];
    if (m.w < 0.f) {
        g.bucket[d] = -1;
        return;
    }
    const float c = cell_edge(g);
    const int b = hash_cell((int)floorf(m.x / c), (int)floorf(m.y / c), (int)floorf(m.z / c), g.T);
    g.bucket[d] = b;
    atomicAdd(g.count + b, 1);
}

__global__ void rg_scatter_kernel(RopeGrid g, int n) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const int b = g.bucket[d];
    if (b < 0) return;
    g.sorted[g.start[b] + atomicAdd(g.count + b, 1)] = d;
}

// Candidates of every segment from the 27 cells around its midpoint, one thread per (segment,
// cell): the thread scans the cell's bucket (skipped when an earlier cell of the same segment
// hashes to the same bucket, so each candidate is found once) and appends the accepted indices,
// unordered, to the segment's column list, counting them in ncols. `pos` are the substep-start
// positions (device order).
__global__ void rg_cells_kernel(const FrameArgs* __restrict__ pa, const float4* __restrict__ pos, RopeGrid g, int n) {
    const FrameArgs& a = *pa;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 27LL * n) return;
    const int d = (int)(t / 27), c = (int)(t - 27LL * d);
    if (!(a.topo[d].x & F_NEXT)) return;
    const float4 md = g.ms[d];
    if (md.w < 0.f) return;  // diverged: no candidates
    const float ce = cell_edge(g);
    const int cx = (int)floorf(md.x / ce), cy = (int)floorf(md.y / ce), cz = (int)floorf(md.z / ce);
    auto bucket_of = [&](int k) { return hash_cell(cx + k % 3 - 1, cy + (k / 3) % 3 - 1, cz + k / 9 - 1, g.T); };
    const int b = bucket_of(c);
    for (int k = 0; k < c; k++)
        if (bucket_of(k) == b) return;
    const int4 gr = a.grp[d];
    const f3 p = xyz(pos[d]), p1 = xyz(pos[d + 1]);
    const f3 a1 = p1 - p;
    const float ri = fmaxf(a.pad[d], a.pad[d + 1]);
    const f3 mt = p + a1 * 0.5f;
    const float ht = 0.5f * len(a1);
    const int e = g.start[b + 1];
    for (int k = g.start[b]; k < e; k++) {
        const int j = g.sorted[k];
        if (j < gr.x || j >= gr.y) continue;
        if (j >= gr.z && j < gr.w && abs(j - d) <= 2) continue;
        // conservative pre-test on the cached midpoints and reaches (one load instead of four): its
        // bound exceeds pair_accepts' own by 1e-4 relative + 1e-6 m, far more than the rounding
        // between the two forms, so it rejects only pairs that pair_accepts rejects as well
        const float4 mj = g.ms[j];
        const f3 dq = xyz(mj) - xyz(md);
        const float rq = (md.w + mj.w) * 1.0002f + 2e-6f;
        if (dot(dq, dq) > rq * rq) continue;
        const f3 pj0 = xyz(pos[j]), pj1 = xyz(pos[j + 1]);
        if (!pair_accepts(p, a1, mt, ht, ri, pj0, pj1, fmaxf(a.pad[j], a.pad[j + 1]))) continue;
        const int q = atomicAdd(a.ncols + d, 1);
        if (q < kMaxCols) a.cols[(size_t)q * n + d] = j;
    }
}

// Per segment: its candidates sorted ascending (the brute force's order) and its step limit; more
// than kMaxCols candidates rerun the brute force, which keeps the first kMaxCols and flags
// MAX_COLLISIONS as the reference does (`flag`).
__global__ void rg_finish_kernel(const FrameArgs* __restrict__ pa, const float4* __restrict__ pos, RopeGrid g, int n,
                                 int flag) {
    const FrameArgs& a = *pa;
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    if (!(a.topo[d].x & F_NEXT) || g.ms[d].w < 0.f) {
        a.ncols[d] = 0;
        a.maxstep[d] = INFINITY;
        return;
    }
    const int4 gr = a.grp[d];
    const f3 p = xyz(pos[d]), p1 = xyz(pos[d + 1]);
    const f3 a1 = p1 - p;
    const int cnt = a.ncols[d];
    float lim;
    if (cnt > kMaxCols) {
        const int total = detect_group(
            a, d, d, gr.x, gr.y, gr.z, gr.w, p, p1, [&](int j) { return a.pad[j]; },
            [&](int j) { return a.topo[j].x; }, [&](int j) { return xyz(pos[j]); }, lim);
        if (flag && total > kMaxCols) atomicMax(a.status, ERR_MAX_COLLISIONS);
        a.ncols[d] = total < kMaxCols ? total : kMaxCols;
    } else {
        int list[kMaxCols];
        for (int q = 0; q < cnt; q++) {  // insertion sort (the lists are short)
            const int j = a.cols[(size_t)q * n + d];
            int at = q;
            while (at > 0 && list[at - 1] > j) {
                list[at] = list[at - 1];
                at--;
            }
            list[at] = j;
        }
        lim = a.pad[d] - a.det_radius;
        for (int q = 0; q < cnt; q++) {
            const int j = list[q];
            a.cols[(size_t)q * n + d] = j;
            lim = fminf(lim, step_limit_of(p, a1, xyz(pos[j]), xyz(pos[j + 1])));
        }
    }
    a.maxstep[d] = lim;
}

inline int blocks_of(int n, int t) { return (n + t - 1) / t; }

}  // namespace

int rope_grid_buckets(int n) {
    int T = 1024;
    while (T < 2 * n) T <<= 1;
    return T;
}

size_t rope_grid_scan_bytes(int T) {
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, (int*)nullptr, (int*)nullptr, T + 1);
    return bytes;
}

cudaError_t rope_grid_detect(const FrameArgs* pa, const float4* pos, const RopeGrid& g, int n, bool flag,
                             cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(g.smax, 0, sizeof(unsigned), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(g.count, 0, sizeof(int) * (size_t)(g.T + 1), st);
    if (e != cudaSuccess) return e;
    rg_reach_kernel<<<blocks_of(n, 256), 256, 0, st>>>(pa, pos, g, n);
    rg_bucket_kernel<<<blocks_of(n, 256), 256, 0, st>>>(g, n);
    size_t bytes = g.scan_bytes;
    e = cub::DeviceScan::ExclusiveSum(g.scan_tmp, bytes, g.count, g.start, g.T + 1, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(g.count, 0, sizeof(int) * (size_t)(g.T + 1), st);
    if (e != cudaSuccess) return e;
    rg_scatter_kernel<<<blocks_of(n, 256), 256, 0, st>>>(g, n);
    rg_cells_kernel<<<(unsigned)((27LL * n + 127) / 128), 128, 0, st>>>(pa, pos, g, n);
    rg_finish_kernel<<<blocks_of(n, 128), 128, 0, st>>>(pa, pos, g, n, flag ? 1 : 0);
    return cudaGetLastError();
}

}  // namespace rs
