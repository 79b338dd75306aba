// rs_sdfbake.cu -- signed-distance lattices of triangle meshes, baked on the GPU.
//
// Replaces the reference's Warp bake (ropesim/sdf.py:96-156, kernel _sdf_kernel at :159-167):
// every lattice node gets the exact distance to the closest point of the mesh, signed by the
// generalized winding number (inside where it exceeds 1/2), then the shell (|phi| - thickness/2)
// and rounding (phi - round) of that function. Node coordinates are the reference's: float32 of
// (float64 origin + float64 spacing * index).
//
// Design (brute force made cheap by exact culling, no BVH):
//  * Triangles are sorted along a Morton curve of their centroids on the host and grouped in
//    tiles of 32 with one AABB per tile.
//  * bake_distance_kernel: one CTA per brick of 4 x 8 x 8 nodes (z fastest, as the lattice's C
//    order), culling per warp (a 1 x 4 x 8 slab): it first evaluates the tile nearest the slab,
//    then visits every tile but skips those whose AABB is farther from the slab than the slab's
//    current largest per-node distance (a warp max): such a tile cannot lower any node's
//    minimum. The test keeps a 1e-4 relative margin for the rounding of the box gap.
//  * bake_sign_rows_kernel: one warp per lattice row along z counts the signed crossings of the
//    row's line with the mesh (one pass over the triangles, tiles skipped by their x-y box); the
//    crossings above a node are its winding number. Crossing predicates are evaluated in double,
//    antisymmetric per shared edge, with a symbolic-perturbation tie-break (a line through an
//    edge or vertex is counted once). A row whose crossings do not cancel (open mesh, or rounding
//    made the predicates inconsistent) falls back to the solid-angle winding number of every
//    node: Van Oosterom and Strackee (IEEE Trans. Biomed. Eng. 30, 1983), tan(W/2) = a.(b x c) /
//    (|a||b||c| + (a.b)|c| + (a.c)|b| + (b.c)|a|), inside where |W| / 4 pi > 1/2.
// The distance kernel is FP32-bound (no contraction; triangle loads are warp broadcasts from L1);
// the row pass is a small fraction of it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#include "rs_device.cuh"
#include "rs_kernels.h"

using namespace rsd;

namespace rs {
namespace {

constexpr int kBX = 4, kBY = 8, kBZ = 8;  // nodes per CTA brick (256 threads)
constexpr int kTile = 32;                 // triangles per culling tile

struct BakeArgs {
    const float4* tri;   // [3 T] vertices a, b, c of each triangle (Morton order)
    const float4* tdist; // [3 T] (a, ab.ab), (ab, ab.ac), (ac, ac.ac) of each triangle, same order
    const float4* tbox;  // [2 tiles] AABB (lo, hi) of each tile of kTile triangles
    int T, tiles;
    double ox, oy, oz, sp;
    int nx, ny, nz;
    float* out;          // [nx, ny, nz]: unsigned distance after the first kernel, phi after the second
    float halft, rnd;    // thickness / 2 (0: signed), round
    unsigned long long* counters;  // NULL or device [3]: point-triangle distances, line-triangle crossing tests, solid angles
};

__device__ __forceinline__ float node_coord(double o, double sp, int i) { return (float)(o + sp * (double)i); }

// Squared distance from p to the triangle a + v ab + w ac (v, w >= 0, v + w <= 1): the closest
// point by the Voronoi region of p (three vertices, three edges, the face), as in Ericson,
// Real-Time Collision Detection (2005), section 5.1.5. The six projections it tests are
// d1 = ab.ap and d2 = ac.ap and their shifts by the triangle's own dot products (ab.ab, ab.ac,
// ac.ac, precomputed per triangle), so one evaluation is two dot products, the region tests and
// the residual ap - v ab - w ac.
__device__ __forceinline__ float tri_dist2(f3 p, float4 r0, float4 r1, float4 r2) {
    const f3 ap = p - xyz(r0), ab = xyz(r1), ac = xyz(r2);
    const float d1 = dot(ab, ap), d2 = dot(ac, ap);
    float v, w;
    if (d1 <= 0.f && d2 <= 0.f) {  // vertex a
        v = 0.f; w = 0.f;
    } else {
        const float d3 = d1 - r0.w, d4 = d2 - r1.w;  // ab.(p - b), ac.(p - b)
        if (d3 >= 0.f && d4 <= d3) {  // vertex b
            v = 1.f; w = 0.f;
        } else {
            const float d5 = d1 - r1.w, d6 = d2 - r2.w;  // ab.(p - c), ac.(p - c)
            const float vc = d1 * d4 - d3 * d2, vb = d5 * d2 - d1 * d6, va = d3 * d6 - d5 * d4;
            if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {  // edge ab
                v = d1 / (d1 - d3); w = 0.f;
            } else if (d6 >= 0.f && d5 <= d6) {  // vertex c
                v = 0.f; w = 1.f;
            } else if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {  // edge ac
                v = 0.f; w = d2 / (d2 - d6);
            } else if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {  // edge bc
                w = (d4 - d3) / ((d4 - d3) + (d5 - d6)); v = 1.f - w;
            } else {  // face
                const float sc = 1.f / (va + vb + vc);
                v = vb * sc; w = vc * sc;
            }
        }
    }
    const f3 d = ap - ab * v - ac * w;
    return dot(d, d);
}

// Solid angle of the triangle (a, b, c) seen from p (positive when p is behind its
// counter-clockwise face).
__device__ __forceinline__ float solid_angle(f3 p, f3 A, f3 B, f3 C) {
    const f3 a = A - p, b = B - p, c = C - p;
    const float la = len(a), lb = len(b), lc = len(c);
    const float num = dot(a, cross(b, c));
    const float den = la * lb * lc + dot(a, b) * lc + dot(a, c) * lb + dot(b, c) * la;
    return 2.f * atan2f(num, den);
}

// Squared gap between two axis-aligned boxes (0 when they overlap).
__device__ __forceinline__ float box_gap2(f3 lo0, f3 hi0, float4 lo1, float4 hi1) {
    const float gx = fmaxf(0.f, fmaxf(lo1.x - hi0.x, lo0.x - hi1.x));
    const float gy = fmaxf(0.f, fmaxf(lo1.y - hi0.y, lo0.y - hi1.y));
    const float gz = fmaxf(0.f, fmaxf(lo1.z - hi0.z, lo0.z - hi1.z));
    return gx * gx + gy * gy + gz * gz;
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// One CTA per brick of 4 x 8 x 8 nodes (z fastest, coalesced stores); each warp culls for its own
// 1 x 4 x 8 slab of the brick: it evaluates the tile nearest its slab first, then skips every
// tile whose AABB is farther from the slab than the slab's largest current minimum (a warp max,
// refreshed after every 4 evaluated tiles), which cannot lower any of its nodes' minima. No CTA
// barriers: warps proceed independently.
__global__ void __launch_bounds__(256) bake_distance_kernel(const BakeArgs A) {
    const int t = threadIdx.x, lane = t & 31;
    const int i0 = blockIdx.x * kBX, j0 = blockIdx.y * kBY, k0 = blockIdx.z * kBZ;
    const int i = i0 + (t >> 6), j = j0 + ((t >> 3) & 7), k = k0 + (t & 7);
    const bool valid = i < A.nx && j < A.ny && k < A.nz;
    if (__ballot_sync(0xffffffffu, valid) == 0u) return;  // a whole warp outside the lattice
    const f3 p = mk3(node_coord(A.ox, A.sp, min(i, A.nx - 1)), node_coord(A.oy, A.sp, min(j, A.ny - 1)),
                     node_coord(A.oz, A.sp, min(k, A.nz - 1)));
    // the warp's slab: node i, rows jw .. jw + 3, columns k0 .. k0 + 7 (clamped to the lattice)
    const int jw = j0 + (((t >> 5) & 1) << 2);
    const f3 blo = mk3(node_coord(A.ox, A.sp, i), node_coord(A.oy, A.sp, jw), node_coord(A.oz, A.sp, k0));
    const f3 bhi = mk3(node_coord(A.ox, A.sp, i), node_coord(A.oy, A.sp, min(jw + 3, A.ny - 1)),
                       node_coord(A.oz, A.sp, min(k0 + kBZ - 1, A.nz - 1)));

    // the tile nearest the slab (smallest box gap, lowest index on ties) seeds the bound
    float lb = INFINITY;
    int tb = 0;
    for (int e = lane; e < A.tiles; e += 32) {
        const float g = box_gap2(blo, bhi, __ldg(A.tbox + 2 * e), __ldg(A.tbox + 2 * e + 1));
        if (g < lb) { lb = g; tb = e; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float g = __shfl_xor_sync(0xffffffffu, lb, o);
        const int e = __shfl_xor_sync(0xffffffffu, tb, o);
        if (g < lb || (g == lb && e < tb)) { lb = g; tb = e; }
    }
    const int seed = tb;

    float best = INFINITY;
    long long evals = 0;
    auto eval_tile = [&](int e) {
        const int q1 = min(A.T, (e + 1) * kTile);
        for (int q = e * kTile; q < q1; q++) {
            const float4* tr = A.tdist + 3 * q;
            best = fminf(best, tri_dist2(p, __ldg(tr), __ldg(tr + 1), __ldg(tr + 2)));
        }
        evals += q1 - e * kTile;
    };
    eval_tile(seed);
    float U2 = warp_max(valid ? best : 0.f);
    int since = 0;
    for (int e = 0; e < A.tiles; e++) {
        if (e == seed) continue;
        const float g = box_gap2(blo, bhi, __ldg(A.tbox + 2 * e), __ldg(A.tbox + 2 * e + 1));
        if (g > U2 * (1.f + 1e-4f)) continue;  // uniform over the warp: same g and U2 in every lane
        eval_tile(e);
        if (++since == 4) {
            since = 0;
            U2 = warp_max(valid ? best : 0.f);
        }
    }
    if (valid) A.out[((size_t)i * A.ny + j) * A.nz + k] = sqrtf(best);
    if (A.counters) {
        const int nvalid = __popc(__ballot_sync(0xffffffffu, valid));
        if (lane == 0) atomicAdd(A.counters, (unsigned long long)(evals * nvalid));
    }
}

// Side of p relative to the directed 2D edge u -> v: +1 left, -1 right, 0 only for a degenerate
// edge. The predicate is evaluated for the edge's lexicographically ordered endpoints and negated
// when the direction is reversed, so two triangles sharing an edge see exactly opposite answers;
// a point exactly on the line is decided by the symbolic perturbation p + (eps, eps^2) (the sign
// of dE/dpx, then of dE/dpy), so that every point belongs to exactly one side.
__device__ __forceinline__ int side2(double ux, double uy, double vx, double vy, double px, double py) {
    const bool sw = (ux > vx) || (ux == vx && uy > vy);
    if (sw) {
        const double tx = ux, ty = uy;
        ux = vx; uy = vy; vx = tx; vy = ty;
    }
    const double e = (vx - ux) * (py - uy) - (vy - uy) * (px - ux);
    int sd;
    if (e > 0.0) sd = 1;
    else if (e < 0.0) sd = -1;
    else if (vy != uy) sd = (vy < uy) ? 1 : -1;  // dE/dpx = -(vy - uy)
    else sd = (vx > ux) ? 1 : ((vx < ux) ? -1 : 0);  // dE/dpy = vx - ux
    return sw ? -sd : sd;
}

// Crossing of the line {x = px, y = py} with triangle (a, b, c): 0 when the line misses it, else
// the orientation of its projection on the x-y plane (+1: counter-clockwise seen from +z, i.e. its
// normal has n.z > 0) with the crossing height in *zc.
__device__ __forceinline__ int z_crossing(double px, double py, float4 a, float4 b, float4 c, double* zc) {
    const int sab = side2(a.x, a.y, b.x, b.y, px, py);
    if (sab == 0) return 0;
    if (side2(b.x, b.y, c.x, c.y, px, py) != sab || side2(c.x, c.y, a.x, a.y, px, py) != sab) return 0;
    const double ax = a.x, ay = a.y, bx = b.x, by = b.y, cx = c.x, cy = c.y;
    const double area2 = (bx - ax) * (cy - ay) - (by - ay) * (cx - ax);
    if (area2 == 0.0) return 0;
    const double la = (bx - px) * (cy - py) - (by - py) * (cx - px);
    const double lb = (cx - px) * (ay - py) - (cy - py) * (ax - px);
    const double lc = (ax - px) * (by - py) - (ay - py) * (bx - px);
    *zc = (la * (double)a.z + lb * (double)b.z + lc * (double)c.z) / area2;
    return sab;
}

// Two-sided shell (thickness > 0): the unsigned distance minus half the thickness, then rounding.
__global__ void bake_shell_kernel(const BakeArgs A, size_t nodes) {
    const size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n < nodes) A.out[n] = (A.out[n] - A.halft) - A.rnd;
}

// Sign (thickness == 0), then rounding, in place over the distances. One warp per lattice row
// (i, j) along z: the signed crossings of the row's line with the mesh, counted above each node,
// are the node's winding number (a closed oriented mesh; overlapping closed parts add up), so one
// pass over the triangles (whole tiles skipped by their x-y box) signs the whole row. A closed
// mesh crosses every line as often upwards as downwards; a row whose crossings do not sum to zero
// (an open mesh, or predicates that rounding made inconsistent) takes the solid-angle winding
// number of every node instead.
constexpr int kRowWarps = 8;
__global__ void __launch_bounds__(32 * kRowWarps) bake_sign_rows_kernel(const BakeArgs A) {
    extern __shared__ int acc_all[];
    const int wp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long r = (long long)blockIdx.x * kRowWarps + wp;
    if (r >= (long long)A.nx * A.ny) return;  // whole warp: this kernel has no block barriers
    int* acc = acc_all + wp * (A.nz + 1);
    const int i = (int)(r / A.ny), j = (int)(r % A.ny);
    const double px = node_coord(A.ox, A.sp, i), py = node_coord(A.oy, A.sp, j);
    for (int k = lane; k <= A.nz; k += 32) acc[k] = 0;
    __syncwarp();
    int total = 0;
    long long tests = 0;
    for (int e = 0; e < A.tiles; e++) {
        const float4 lo = __ldg(A.tbox + 2 * e), hi = __ldg(A.tbox + 2 * e + 1);
        if (px < lo.x || px > hi.x || py < lo.y || py > hi.y) continue;  // uniform over the warp
        tests += min(kTile, A.T - e * kTile);
        const int q = e * kTile + lane;
        if (q >= A.T) continue;
        const float4* tr = A.tri + 3 * q;
        double zc;
        const int sg = z_crossing(px, py, __ldg(tr), __ldg(tr + 1), __ldg(tr + 2), &zc);
        if (sg == 0) continue;
        total += sg;
        // first node at or above the crossing: the nodes below it see the crossing above them
        int kc = (int)fmin(fmax(ceil((zc - A.oz) / A.sp), 0.0), (double)A.nz);
        while (kc > 0 && (double)node_coord(A.oz, A.sp, kc - 1) >= zc) kc--;
        while (kc < A.nz && (double)node_coord(A.oz, A.sp, kc) < zc) kc++;
        atomicAdd(acc + kc, sg);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
    __syncwarp();
    const size_t row = ((size_t)i * A.ny + j) * A.nz;
    long long solid = 0;
    if (total == 0) {
        if (lane == 0) {  // acc[k] <- crossings strictly above node k
            int run = 0;
            for (int k = A.nz; k >= 0; k--) {
                const int t = acc[k];
                acc[k] = run;
                run += t;
            }
        }
        __syncwarp();
        for (int k = lane; k < A.nz; k += 32) {
            const float d = A.out[row + k];
            A.out[row + k] = (acc[k] != 0 ? -d : d) - A.rnd;
        }
    } else {
        for (int k = lane; k < A.nz; k += 32) {
            const f3 p = mk3((float)px, (float)py, node_coord(A.oz, A.sp, k));
            float sa = 0.f;
            for (int q = 0; q < A.T; q++) {
                const float4* tr = A.tri + 3 * q;
                sa += solid_angle(p, xyz(__ldg(tr)), xyz(__ldg(tr + 1)), xyz(__ldg(tr + 2)));
            }
            const float w = sa * (0.25f / 3.14159265358979f);
            const float d = A.out[row + k];
            A.out[row + k] = (fabsf(w) > 0.5f ? -d : d) - A.rnd;
        }
        solid = (long long)A.T * A.nz;
    }
    if (A.counters && lane == 0) {
        atomicAdd(A.counters + 1, (unsigned long long)tests);
        if (solid) atomicAdd(A.counters + 2, (unsigned long long)solid);
    }
}

}  // namespace

// Host side: validation, Morton ordering and tiling of the triangles, launches. Vertices and
// triangles are host arrays; `out` is host (synchronous) or device memory (queued on `s`).
cudaError_t sdf_bake(const float* verts, int nv, const int* tris, int nt, const float* origin, double spacing, int nx, int ny,
                     int nz, float thickness, float round, float* out, bool out_on_device, unsigned long long* counters,
                     cudaStream_t s, std::string* err) {
    auto fail = [&](const std::string& m) { *err = m; return cudaErrorInvalidValue; };
    if (nv < 3 || nt < 1) return fail("bake needs a triangle mesh (>= 3 vertices, >= 1 triangle)");
    if (!(spacing > 0.0) || nx < 2 || ny < 2 || nz < 2) return fail("spacing > 0 and >= 2 nodes per axis required");
    if (!(thickness >= 0.f) || !(round >= 0.f)) return fail("thickness and round must be >= 0");
    if ((double)nx * ny * nz > 2.0e9) return fail("lattice too large (> 2e9 nodes)");
    if (nz > 7000) return fail("lattice too long along z (> 7000 nodes; the sign pass keeps a row in shared memory)");
    for (int q = 0; q < 3 * nt; q++)
        if (tris[q] < 0 || tris[q] >= nv) return fail("triangle indices out of range");
    for (int q = 0; q < 3 * nv; q++)
        if (!std::isfinite(verts[q])) return fail("vertices must be finite");
    // drop zero-area triangles (their points lie on the neighbouring triangles' edges and their
    // solid angle is zero), then order the rest along a Morton curve of the centroids
    std::vector<int> keep;
    keep.reserve(nt);
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int q = 0; q < nt; q++) {
        const float* a = verts + 3 * tris[3 * q];
        const float* b = verts + 3 * tris[3 * q + 1];
        const float* c = verts + 3 * tris[3 * q + 2];
        const double ux = (double)b[0] - a[0], uy = (double)b[1] - a[1], uz = (double)b[2] - a[2];
        const double vx = (double)c[0] - a[0], vy = (double)c[1] - a[1], vz = (double)c[2] - a[2];
        const double cx = uy * vz - uz * vy, cy = uz * vx - ux * vz, cz = ux * vy - uy * vx;
        if (!(cx * cx + cy * cy + cz * cz > 0.0)) continue;
        keep.push_back(q);
        for (const float* v : {a, b, c})
            for (int d = 0; d < 3; d++) { lo[d] = std::min(lo[d], (double)v[d]); hi[d] = std::max(hi[d], (double)v[d]); }
    }
    const int T = (int)keep.size();
    if (T == 0) return fail("every triangle has zero area");
    auto spread = [](uint32_t x) {  // 10 bits -> every third bit
        x &= 0x3ffu;
        x = (x | (x << 16)) & 0x030000ffu;
        x = (x | (x << 8)) & 0x0300f00fu;
        x = (x | (x << 4)) & 0x030c30c3u;
        x = (x | (x << 2)) & 0x09249249u;
        return x;
    };
    std::vector<uint32_t> code(T);
    for (int e = 0; e < T; e++) {
        const int q = keep[e];
        uint32_t m = 0;
        for (int d = 0; d < 3; d++) {
            const double cen = ((double)verts[3 * tris[3 * q] + d] + verts[3 * tris[3 * q + 1] + d] + verts[3 * tris[3 * q + 2] + d]) / 3.0;
            const double ext = hi[d] - lo[d];
            const double u = ext > 0.0 ? (cen - lo[d]) / ext : 0.0;
            m |= spread((uint32_t)std::min(1023.0, std::max(0.0, u * 1023.0))) << d;
        }
        code[e] = m;
    }
    std::vector<int> order(T);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return code[x] < code[y]; });
    const int tiles = (T + kTile - 1) / kTile;
    std::vector<float4> tri((size_t)6 * T), tbox((size_t)2 * tiles);  // vertices, then the distance records
    for (int e = 0; e < T; e++) {
        const int q = keep[order[e]];
        for (int v = 0; v < 3; v++) {
            const float* x = verts + 3 * tris[3 * q + v];
            tri[3 * e + v] = make_float4(x[0], x[1], x[2], 0.f);
        }
        const float4 a = tri[3 * e], b = tri[3 * e + 1], c = tri[3 * e + 2];
        const float abx = b.x - a.x, aby = b.y - a.y, abz = b.z - a.z, acx = c.x - a.x, acy = c.y - a.y, acz = c.z - a.z;
        const double abab = (double)abx * abx + (double)aby * aby + (double)abz * abz;
        const double abac = (double)abx * acx + (double)aby * acy + (double)abz * acz;
        const double acac = (double)acx * acx + (double)acy * acy + (double)acz * acz;
        tri[(size_t)3 * T + 3 * e] = make_float4(a.x, a.y, a.z, (float)abab);
        tri[(size_t)3 * T + 3 * e + 1] = make_float4(abx, aby, abz, (float)abac);
        tri[(size_t)3 * T + 3 * e + 2] = make_float4(acx, acy, acz, (float)acac);
    }
    for (int b = 0; b < tiles; b++) {
        float4 l = make_float4(INFINITY, INFINITY, INFINITY, 0.f), h = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.f);
        for (int e = b * kTile; e < std::min(T, (b + 1) * kTile); e++)
            for (int v = 0; v < 3; v++) {
                const float4 x = tri[3 * e + v];
                l.x = std::min(l.x, x.x); l.y = std::min(l.y, x.y); l.z = std::min(l.z, x.z);
                h.x = std::max(h.x, x.x); h.y = std::max(h.y, x.y); h.z = std::max(h.z, x.z);
            }
        tbox[2 * b] = l;
        tbox[2 * b + 1] = h;
    }

    const size_t nodes = (size_t)nx * ny * nz;
    float4 *dtri = nullptr, *dbox = nullptr;
    float* dout = out_on_device ? out : nullptr;
    unsigned long long* dcnt = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    cudaError_t e = cudaMallocAsync(&dtri, sizeof(float4) * tri.size(), s);
    if (e == cudaSuccess) e = cudaMallocAsync(&dbox, sizeof(float4) * tbox.size(), s);
    if (e == cudaSuccess && !out_on_device) e = cudaMallocAsync(&dout, sizeof(float) * nodes, s);
    if (e == cudaSuccess && counters) e = cudaMallocAsync(&dcnt, 3 * sizeof(unsigned long long), s);
    if (e == cudaSuccess && counters) e = cudaMemsetAsync(dcnt, 0, 3 * sizeof(unsigned long long), s);
    // host-to-device copies from pageable vectors complete before the call returns
    if (e == cudaSuccess) e = cudaMemcpyAsync(dtri, tri.data(), sizeof(float4) * tri.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dbox, tbox.data(), sizeof(float4) * tbox.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        BakeArgs A;
        A.tri = dtri; A.tdist = dtri + (size_t)3 * T; A.tbox = dbox; A.T = T; A.tiles = tiles;
        A.ox = origin[0]; A.oy = origin[1]; A.oz = origin[2]; A.sp = spacing;
        A.nx = nx; A.ny = ny; A.nz = nz;
        A.out = dout;
        A.halft = 0.5f * thickness;
        A.rnd = round;
        A.counters = dcnt;
        const dim3 grid((nx + kBX - 1) / kBX, (ny + kBY - 1) / kBY, (nz + kBZ - 1) / kBZ);
        if (grid.y > 65535 || grid.z > 65535) e = cudaErrorInvalidValue;
        if (e == cudaSuccess && counters) e = cudaEventCreate(&ev[0]);
        if (e == cudaSuccess && counters) e = cudaEventCreate(&ev[1]);
        if (e == cudaSuccess && counters) e = cudaEventRecord(ev[0], s);
        if (e == cudaSuccess) {
            bake_distance_kernel<<<grid, 256, 0, s>>>(A);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess && thickness > 0.f) {
            bake_shell_kernel<<<(unsigned)((nodes + 255) / 256), 256, 0, s>>>(A, nodes);
            e = cudaGetLastError();
        } else if (e == cudaSuccess) {
            const size_t rows = (size_t)nx * ny;
            const size_t smem = sizeof(int) * kRowWarps * ((size_t)nz + 1);
            if (smem > 48 * 1024)
                e = cudaFuncSetAttribute(bake_sign_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e == cudaSuccess) {
                bake_sign_rows_kernel<<<(unsigned)((rows + kRowWarps - 1) / kRowWarps), 32 * kRowWarps, smem, s>>>(A);
                e = cudaGetLastError();
            }
        }
        if (e == cudaSuccess && counters) e = cudaEventRecord(ev[1], s);
    }
    if (e == cudaSuccess && !out_on_device) e = cudaMemcpyAsync(out, dout, sizeof(float) * nodes, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && counters)
        e = cudaMemcpyAsync(counters, dcnt, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
    if (dtri) cudaFreeAsync(dtri, s);
    if (dbox) cudaFreeAsync(dbox, s);
    if (dout && !out_on_device) cudaFreeAsync(dout, s);
    if (dcnt) cudaFreeAsync(dcnt, s);
    if (e == cudaSuccess && (!out_on_device || counters)) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess && counters) {  // device time of the kernels alone (the host preparation excluded)
        float ms = 0.f;
        e = cudaEventElapsedTime(&ms, ev[0], ev[1]);
        counters[3] = (unsigned long long)((double)ms * 1e6);
    }
    for (cudaEvent_t x : ev)
        if (x) cudaEventDestroy(x);
    if (e != cudaSuccess && err->empty()) *err = std::string("sdf bake: ") + cudaGetErrorString(e);
    return e;
}

}  // namespace rs
