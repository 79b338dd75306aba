// rs_sdfbake_oracle.hpp -- TEST INFRASTRUCTURE ONLY: FP64 CPU restatement of the mesh bake
// (ropesim/sdf.py:96-167 of the reference: bake_mesh and its Warp kernel _sdf_kernel).
//
// The reference's kernel asks Warp (warp-lang, not vendored; the reference pins no version)
// for mesh_query_point_sign_winding_number(mesh, p, 1e6, accuracy 2.0, threshold 0.5): the
// exact closest point of the mesh (a BVH search) and the sign from the generalized winding
// number (Jacobson et al. 2013; Warp evaluates it with the fast approximation of Barill et al.
// 2018, which on a closed mesh is 1 inside and 0 outside like the exact sum). This restatement
// evaluates both by brute force over all triangles in double precision:
//  * distance: the plane projection when it falls inside the triangle (barycentric test),
//    otherwise the nearest of the three edge segments -- a different construction from the
//    GPU's Voronoi-region walk, so that the two check each other;
//  * winding number: sum of the triangles' solid angles / 4 pi (Van Oosterom and Strackee);
//    inside where its magnitude exceeds 1/2;
//  * phi = sign * distance, or |distance| - thickness / 2 for thickness > 0, then - round
//    (sdf.py:145-148).
// Node coordinates are float32(origin + spacing * index) as in sdf.py:69-77. Zero-area triangles
// are dropped. Parallel over lattice rows with std::thread.
#pragma once

#include <algorithm>
#include <cmath>
#include <thread>
#include <vector>

namespace rso {

struct BakeOut {
    std::vector<double> phi, dist, wind;
};

namespace bake_detail {
struct D3 {
    double x, y, z;
};
inline D3 sub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline double dotd(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline D3 crossd(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double norm(D3 a) { return std::sqrt(dotd(a, a)); }

inline double seg_dist2(D3 p, D3 a, D3 b) {
    const D3 ab = sub(b, a);
    const double L = dotd(ab, ab);
    double t = L > 0.0 ? dotd(sub(p, a), ab) / L : 0.0;
    t = std::min(1.0, std::max(0.0, t));
    const D3 q = {a.x + t * ab.x, a.y + t * ab.y, a.z + t * ab.z};
    const D3 d = sub(p, q);
    return dotd(d, d);
}

inline double tri_dist2(D3 p, D3 a, D3 b, D3 c) {
    const D3 n = crossd(sub(b, a), sub(c, a));
    const double nn = dotd(n, n);
    // barycentric coordinates of the plane projection
    const double s = dotd(sub(p, a), n) / nn;
    const D3 q = {p.x - s * n.x, p.y - s * n.y, p.z - s * n.z};
    const double wa = dotd(crossd(sub(b, q), sub(c, q)), n), wb = dotd(crossd(sub(c, q), sub(a, q)), n),
                 wc = dotd(crossd(sub(a, q), sub(b, q)), n);
    if (wa >= 0.0 && wb >= 0.0 && wc >= 0.0) return s * s * nn;
    return std::min(seg_dist2(p, a, b), std::min(seg_dist2(p, b, c), seg_dist2(p, c, a)));
}

inline double solid_angle(D3 p, D3 A, D3 B, D3 C) {
    const D3 a = sub(A, p), b = sub(B, p), c = sub(C, p);
    const double la = norm(a), lb = norm(b), lc = norm(c);
    const double num = dotd(a, crossd(b, c));
    const double den = la * lb * lc + dotd(a, b) * lc + dotd(a, c) * lb + dotd(b, c) * la;
    return 2.0 * std::atan2(num, den);
}
}  // namespace bake_detail

inline BakeOut bake_sdf(const float* verts, int nv, const int* tris, int nt, const float* origin, double spacing, int nx,
                        int ny, int nz, double thickness, double round, int threads) {
    using namespace bake_detail;
    (void)nv;
    std::vector<D3> A, B, C;
    for (int q = 0; q < nt; q++) {
        auto v = [&](int k) {
            const float* x = verts + 3 * tris[3 * q + k];
            return D3{(double)x[0], (double)x[1], (double)x[2]};
        };
        const D3 a = v(0), b = v(1), c = v(2);
        const D3 n = crossd(sub(b, a), sub(c, a));
        if (!(dotd(n, n) > 0.0)) continue;
        A.push_back(a);
        B.push_back(b);
        C.push_back(c);
    }
    const size_t nodes = (size_t)nx * ny * nz;
    BakeOut o;
    o.phi.assign(nodes, 0.0);
    o.dist.assign(nodes, 0.0);
    o.wind.assign(nodes, 0.0);
    const int T = (int)A.size();
    auto rows = [&](long long r0, long long r1) {  // rows r = i * ny + j of nz nodes
        for (long long r = r0; r < r1; r++) {
            const int i = (int)(r / ny), j = (int)(r % ny);
            for (int k = 0; k < nz; k++) {
                const D3 p = {(double)(float)((double)origin[0] + spacing * i), (double)(float)((double)origin[1] + spacing * j),
                              (double)(float)((double)origin[2] + spacing * k)};
                double d2 = INFINITY, w = 0.0;
                for (int q = 0; q < T; q++) {
                    d2 = std::min(d2, tri_dist2(p, A[q], B[q], C[q]));
                    w += solid_angle(p, A[q], B[q], C[q]);
                }
                w /= 4.0 * M_PI;
                const double d = std::sqrt(d2);
                const size_t id = ((size_t)i * ny + j) * nz + k;
                o.dist[id] = d;
                o.wind[id] = w;
                const double phi = thickness > 0.0 ? d - 0.5 * thickness : (std::fabs(w) > 0.5 ? -d : d);
                o.phi[id] = phi - round;
            }
        }
    };
    const long long R = (long long)nx * ny;
    threads = (int)std::max(1LL, std::min((long long)threads, R));
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; t++) pool.emplace_back(rows, R * t / threads, R * (t + 1) / threads);
    for (auto& th : pool) th.join();
    return o;
}

}  // namespace rso
